// Diagonal-block kernels: unblocked Cholesky / LU of one nb x nb block held in
// shared memory, and triangular inverses of diagonal blocks (the trsm sweeps
// multiply by these inverses on the tensor cores).
#include "internal.h"

namespace egpu {

constexpr int kDiagThreads = 256;
constexpr int kMaxNB = 128;

// In-place inverse of the uplo triangle of the b x b column-major block S
// (ld b) in shared memory.  unit: the diagonal is taken as 1 and left as 1.
// Row-parallel forward/backward substitution, two barriers per column.  The
// diagonal of a unit triangle is never read, so a unit-lower inverse can share
// S with an upper triangle (the two touch disjoint entries).
__device__ void tri_inverse_smem(double* S, int b, int uplo, int unit) {
  const int i = threadIdx.x;
  if (uplo == EGPU_LOWER) {
    for (int j = b - 1; j >= 0; --j) {
      const double dinv = unit ? 1.0 : 1.0 / S[j + j * b];
      double tmp = 0.0;
      if (i > j && i < b) {
        // X[i, j] = -(sum_{k=j+1..i} X[i,k] L[k,j]) / L[j,j]   (X[i,i] already inverted)
        for (int k = j + 1; k < i; ++k) tmp = fma(S[i + k * b], S[k + j * b], tmp);
        tmp = fma(unit ? 1.0 : S[i + i * b], S[i + j * b], tmp);
      }
      __syncthreads();
      if (i > j && i < b) S[i + j * b] = -tmp * dinv;
      if (i == 0 && !unit) S[j + j * b] = dinv;
      __syncthreads();
    }
  } else {
    for (int j = 0; j < b; ++j) {
      const double dinv = unit ? 1.0 : 1.0 / S[j + j * b];
      double tmp = 0.0;
      if (i < j) {
        // X[i, j] = -(sum_{k=i..j-1} X[i,k] U[k,j]) / U[j,j]
        tmp = (unit ? 1.0 : S[i + i * b]) * S[i + j * b];
        for (int k = i + 1; k < j; ++k) tmp = fma(S[i + k * b], S[k + j * b], tmp);
      }
      __syncthreads();
      if (i < j) S[i + j * b] = -tmp * dinv;
      if (i == 0 && !unit) S[j + j * b] = dinv;
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// Diagonal-block kernels.  The nb x nb block (nb <= 128) lives in shared
// memory with leading dimension kLDS = 129 (odd: row and column sweeps are
// both bank-conflict free), always as a LOWER triangle (an upper triangle is
// handled as the lower triangle of its transpose: UVar3Unb and LVar3Unb
// perform the same operations on A and A^T).
//
// Factorization: 16-column sub-panels.  Inside a sub-panel every column costs
// one barrier: all threads read a_jj, each updates its share of the
// sub-panel columns with  a_ik -= a_ij a_kj / a_jj  (the rank-1 update of
// LVar3Unb, Cholesky/LVar3.hpp:40-46, applied before the column is scaled),
// and the previous column is scaled by 1/sqrt(a_jj) in the same phase (no
// thread reads it any more).  After the sub-panel, the trailing triangle is
// updated by a register-blocked shared-memory mini-GEMM (4x4 per thread).
// The inverse of the factor is built the same way: 16 x 16 diagonal blocks
// inverted in parallel (one per warp), then block columns from the right,
// X21 = -inv(L22) (L21 X11), with 4x4-blocked mini-GEMMs.
// All loops are rolled: straight-line unrolled code run by one warp stalls
// on instruction fetch.
constexpr int kLDS = 129;
constexpr int kSP = 16;  // sub-panel width
constexpr int kDiagSmem = (128 * kLDS + 128) * (int)sizeof(double);

__device__ __forceinline__ double& SE(double* S, int r, int c) { return S[r + c * kLDS]; }

// C[r0.., c0..] (nr x nc, lower part r >= c when tri) -= A[r0.., k0..k0+K) * B[c0.., k0..k0+K)^T
// reading A and B from S; 4x4 register tiles per thread.  sign = +1 or -1 for
// "-=" or "+=" (the inverse uses the opposite sign).
__device__ void smem_syrk_tiles(double* S, int r0, int nr, int c0, int nc, int k0, int K, bool tri) {
  const int tr = (nr + 3) / 4, tc = (nc + 3) / 4;
  for (int t = threadIdx.x; t < tr * tc; t += blockDim.x) {
    const int ti = t % tr, tj = t / tr;
    const int rb = r0 + 4 * ti, cb = c0 + 4 * tj;
    if (tri && rb + 3 < cb) continue;  // tile strictly above the diagonal
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    for (int k = k0; k < k0 + K; ++k) {
      double x[4], y[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        x[a] = (rb + a < r0 + nr) ? SE(S, rb + a, k) : 0.0;
        y[a] = (cb + a < c0 + nc) ? SE(S, cb + a, k) : 0.0;
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(x[a], y[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int r = rb + a, c = cb + b;
        if (r < r0 + nr && c < c0 + nc && (!tri || r >= c)) SE(S, r, c) -= acc[a][b];
      }
  }
}

// Lower Cholesky of the b x b block in S.  Returns 0 or the 1-based column
// of a non-positive pivot ("A was not numerically HPD", LVar3.hpp:37-38); the
// decision is uniform across the block (every thread reads the same a_jj).
__device__ int smem_chol(double* S, int b) {
  __shared__ double s_alpha[128];
  const int tid = threadIdx.x;
  const int row = tid & 127, half = tid >> 7;  // two threads per row
  for (int c0 = 0; c0 < b; c0 += kSP) {
    const int c1 = min(b, c0 + kSP);
    for (int j = c0; j < c1; ++j) {
      const double ajj = SE(S, j, j);
      if (ajj <= 0.0) return j + 1;
      if (tid == 0) s_alpha[j] = sqrt(ajj);
      // column j-1 is read by nobody in this phase: scale it now
      if (j > c0 && half == 1 && row >= j && row < b) SE(S, row, j - 1) /= s_alpha[j - 1];
      if (row > j && row < b) {
        const double lij = SE(S, row, j) / ajj;
        for (int k = j + 1 + half; k < c1 && k <= row; k += 2) SE(S, row, k) -= lij * SE(S, k, j);
      }
      __syncthreads();
    }
    if (half == 0 && row >= c1 && row < b) SE(S, row, c1 - 1) /= s_alpha[c1 - 1];
    if (half == 1 && row >= c0 && row < c1) SE(S, row, row) = s_alpha[row];
    __syncthreads();
    if (c1 < b) {
      smem_syrk_tiles(S, c1, b - c1, c1, b - c1, c0, c1 - c0, true);
      __syncthreads();
    }
  }
  return 0;
}

// In-place inverse of the lower b x b triangle in S (unit: diagonal taken as 1
// and written as 1).  Uses Xs (16 x 16 scratch per warp would not fit; the
// diagonal blocks are inverted in place column by column by their warp).
__device__ void smem_trinv(double* S, int b, int unit) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = (b + kSP - 1) / kSP;
  // 1. 16 x 16 diagonal blocks, one warp each: lane c (< 16) computes column c
  //    of the block inverse by forward substitution, in place is impossible,
  //    so results go to registers first, then back to S.
  for (int blk = warp; blk < nblk; blk += blockDim.x / 32) {
    const int o = blk * kSP, w = min(kSP, b - o);
    double x[kSP];
    const int c = lane;
#pragma unroll
    for (int i = 0; i < kSP; ++i) x[i] = 0.0;
    if (c < w) {
#pragma unroll
      for (int i = 0; i < kSP; ++i) {
        if (i < w && i >= c) {
          double acc = (i == c) ? 1.0 : 0.0;
#pragma unroll
          for (int m = 0; m < kSP; ++m)
            if (m >= c && m < i) acc = fma(-SE(S, o + i, o + m), x[m], acc);
          x[i] = unit ? acc : acc / SE(S, o + i, o + i);
        }
      }
    }
    __syncwarp();
    if (c < w) {
#pragma unroll
      for (int i = 0; i < kSP; ++i)
        if (i < w && i >= c) SE(S, o + i, o + c) = (unit && i == c) ? 1.0 : x[i];
    }
  }
  __syncthreads();
  // 2. block columns from the right: X21 = -inv(L22) * (L21 * X11)
  for (int blk = nblk - 2; blk >= 0; --blk) {
    const int o = blk * kSP, w = min(kSP, b - o), r0 = o + w, R = b - r0;
    // T = L21 * X11 (R x w), computed into registers, written over L21
    {
      const int tr = (R + 3) / 4;
      double acc[4][4];
      const int t = tid;
      const bool act = t < tr * 4;  // tiles: 4 rows x 4 cols, w <= 16 -> 4 col tiles
      const int ti = t % max(tr, 1), tj = t / max(tr, 1);
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[a][q] = 0.0;
      if (act) {
        for (int k = 0; k < w; ++k) {
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const int r = r0 + 4 * ti + a;
            const double l = (r < b) ? SE(S, r, o + k) : 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int cc = 4 * tj + q;
              const double xv = (cc < w && k >= cc) ? SE(S, o + k, o + cc) : 0.0;
              acc[a][q] = fma(l, xv, acc[a][q]);
            }
          }
        }
      }
      __syncthreads();
      if (act)
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = r0 + 4 * ti + a, cc = 4 * tj + q;
            if (r < b && cc < w) SE(S, r, o + cc) = acc[a][q];
          }
      __syncthreads();
      // X21 = -inv(L22) * T : row r of X21 = -sum_{m <= r} X22[r, m] T[m, :]
      if (act) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[a][q] = 0.0;
        const int rmax = min(b - 1, r0 + 4 * ti + 3);
        for (int m = r0; m <= rmax; ++m) {
          double tv[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) tv[q] = (4 * tj + q < w) ? SE(S, m, o + 4 * tj + q) : 0.0;
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const int r = r0 + 4 * ti + a;
            const double xv = (r < b && m <= r) ? (unit && m == r ? 1.0 : SE(S, r, m)) : 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[a][q] = fma(xv, tv[q], acc[a][q]);
          }
        }
      }
      __syncthreads();
      if (act)
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = r0 + 4 * ti + a, cc = 4 * tj + q;
            if (r < b && cc < w) SE(S, r, o + cc) = -acc[a][q];
          }
      __syncthreads();
    }
  }
}

// Cholesky of the b x b diagonal block (cholesky::LVar3Unb,
// lapack-like/Cholesky/LVar3.hpp:19-49, or UVar3Unb, Cholesky/UVar3.hpp:21-50),
// then the inverse of the factor into W (other triangle zeroed).
template <int UPLO>
__global__ void __launch_bounds__(kDiagThreads) potrf_diag_kernel(double* A, long long lda, int b, double* W,
                                                                   int ldw, DevStatus* st, int col_base) {
  extern __shared__ double S[];
  if (st != nullptr && st->code != 0) return;
  const int tid = threadIdx.x;
  for (int c = 0; c < b; ++c)
    for (int r = c + tid; r < b; r += kDiagThreads)
      SE(S, r, c) = (UPLO == EGPU_LOWER) ? A[r + (long long)c * lda] : A[c + (long long)r * lda];
  __syncthreads();
  const int f = smem_chol(S, b);
  if (f) {
    if (tid == 0) set_status(st, kNotHPD, col_base + f);
    return;
  }
  for (int c = 0; c < b; ++c)
    for (int r = c + tid; r < b; r += kDiagThreads) {
      if (UPLO == EGPU_LOWER) A[r + (long long)c * lda] = SE(S, r, c);
      else A[c + (long long)r * lda] = SE(S, r, c);
    }
  __syncthreads();
  smem_trinv(S, b, 0);
  for (int c = 0; c < b; ++c)
    for (int r = tid; r < b; r += kDiagThreads) {
      const double v = (r >= c) ? SE(S, r, c) : 0.0;
      if (UPLO == EGPU_LOWER) W[r + (long long)c * ldw] = v;
      else W[c + (long long)r * ldw] = v;  // inv(U) = inv(L)^T
    }
}

int launch_potrf_diag(cudaStream_t st, int uplo, double* A, long long lda, int b, double* W, int ldw,
                      DevStatus* status, int col_base) {
  if (b <= 0) return EGPU_OK;
  if (b > kMaxNB) return EGPU_ERR_ARG;
  const size_t smem = kDiagSmem;
  TraceMark tm(st, kTraceDiag, (double)b * b * b / 3.0 * 2.0, 16.0 * b * b);
  cudaError_t e;
  if (uplo == EGPU_LOWER) {
    e = cudaFuncSetAttribute(potrf_diag_kernel<EGPU_LOWER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kDiagSmem);
    if (e == cudaSuccess)
      potrf_diag_kernel<EGPU_LOWER><<<1, kDiagThreads, smem, st>>>(A, lda, b, W, ldw, status, col_base);
      count_launch();
  } else {
    e = cudaFuncSetAttribute(potrf_diag_kernel<EGPU_UPPER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kDiagSmem);
    if (e == cudaSuccess)
      potrf_diag_kernel<EGPU_UPPER><<<1, kDiagThreads, smem, st>>>(A, lda, b, W, ldw, status, col_base);
      count_launch();
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "potrf_diag launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

// Inverse of each diagonal block (block i covers rows/cols [i b, min(n, i b + b))),
// lower or upper (as the transpose of a lower), unit or not.
__global__ void __launch_bounds__(kDiagThreads) trtri_blocks_kernel(int uplo, int unit, const double* A,
                                                                     long long lda, int n, int b, double* W,
                                                                     int ldw) {
  extern __shared__ double S[];
  const int blk = blockIdx.x;
  const int off = blk * b;
  const int bb = min(b, n - off);
  const double* Ab = A + off + (long long)off * lda;
  double* Wb = W + (long long)blk * b * ldw;
  const int tid = threadIdx.x;
  for (int c = 0; c < bb; ++c)
    for (int r = c + tid; r < bb; r += kDiagThreads)
      SE(S, r, c) = (uplo == EGPU_LOWER) ? Ab[r + (long long)c * lda] : Ab[c + (long long)r * lda];
  __syncthreads();
  smem_trinv(S, bb, unit);
  for (int c = 0; c < b; ++c)
    for (int r = tid; r < b; r += kDiagThreads) {
      double v = 0.0;
      if (r < bb && c < bb && r >= c) v = SE(S, r, c);
      if (uplo == EGPU_LOWER) Wb[r + (long long)c * ldw] = v;
      else Wb[c + (long long)r * ldw] = v;
    }
}

int launch_trtri_blocks(cudaStream_t st, int uplo, int unit, const double* A, long long lda, int n, int b,
                        double* W, int ldw) {
  if (n <= 0) return EGPU_OK;
  if (b > kMaxNB || b <= 0) return EGPU_ERR_ARG;
  const int count = (n + b - 1) / b;
  TraceMark tm(st, kTraceDiag, (double)count * b * b * b / 3.0, 16.0 * count * b * b);
  cudaError_t e = cudaFuncSetAttribute(trtri_blocks_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kDiagSmem);
  if (e == cudaSuccess) {
    trtri_blocks_kernel<<<count, kDiagThreads, kDiagSmem, st>>>(uplo, unit, A, lda, n, b, W, ldw);
    count_launch();
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_last_error(e, "trtri launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

// Unpivoted LU of the b x b diagonal block (lu::Unb, lapack-like/LU/Local.hpp:61-82);
// W := inv(unit lower L11), W2 := inv(U11).
__global__ void __launch_bounds__(kDiagThreads) getrf_diag_nopiv_kernel(double* A, long long lda, int b, double* W,
                                                                         int ldw, double* W2, DevStatus* st,
                                                                         int col_base) {
  extern __shared__ double S[];
  if (st != nullptr && st->code != 0) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = kDiagThreads / 32;
  for (int idx = tid; idx < b * b; idx += kDiagThreads) S[idx] = A[idx % b + (idx / b) * lda];
  __syncthreads();
  for (int j = 0; j < b; ++j) {
    const double alpha = S[j + j * b];
    if (alpha == 0.0) {
      if (tid == 0) set_status(st, kSingular, col_base + j + 1);
      return;
    }
    const double inv = 1.0 / alpha;
    for (int i = j + 1 + tid; i < b; i += kDiagThreads) S[i + j * b] *= inv;
    __syncthreads();
    for (int c = j + 1 + warp; c < b; c += NW) {
      const double u = S[j + c * b];
      for (int i = j + 1 + lane; i < b; i += 32) S[i + c * b] -= S[i + j * b] * u;
    }
    __syncthreads();
  }
  for (int idx = tid; idx < b * b; idx += kDiagThreads) A[idx % b + (idx / b) * lda] = S[idx];
  __syncthreads();
  // Strict lower (unit L) and upper-with-diagonal (U) are disjoint: invert both in place.
  tri_inverse_smem(S, b, EGPU_LOWER, 1);
  tri_inverse_smem(S, b, EGPU_UPPER, 0);
  for (int idx = tid; idx < b * b; idx += kDiagThreads) {
    const int r = idx % b, c = idx / b;
    W[r + (long long)c * ldw] = r > c ? S[idx] : (r == c ? 1.0 : 0.0);
    W2[r + (long long)c * ldw] = r <= c ? S[idx] : 0.0;
  }
}

int launch_getrf_diag_nopiv(cudaStream_t st, double* A, long long lda, int b, double* W, int ldw, double* W2,
                            DevStatus* status, int col_base) {
  if (b <= 0) return EGPU_OK;
  if (b > kMaxNB) return EGPU_ERR_ARG;
  cudaError_t e = cudaFuncSetAttribute(getrf_diag_nopiv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(sizeof(double) * kMaxNB * kMaxNB));
  if (e == cudaSuccess) {
    getrf_diag_nopiv_kernel<<<1, kDiagThreads, sizeof(double) * b * b, st>>>(A, lda, b, W, ldw, W2, status,
                                                                             col_base);
    count_launch();
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_last_error(e, "getrf_diag launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

__global__ void copy_kernel(int m, int n, const double* src, long long lds, double* dst, long long ldd) {
  const long long total = (long long)m * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(idx % m), c = (int)(idx / m);
    dst[r + c * ldd] = src[r + c * lds];
  }
}

int launch_copy(cudaStream_t st, int m, int n, const double* src, long long lds, double* dst, long long ldd) {
  if (m <= 0 || n <= 0) return EGPU_OK;
  const long long total = (long long)m * n;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 16);
  copy_kernel<<<blocks, 256, 0, st>>>(m, n, src, lds, dst, ldd);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "copy launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

}  // namespace egpu
