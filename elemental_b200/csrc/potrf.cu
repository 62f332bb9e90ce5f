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
// Blocked diagonal-block kernels.  The nb x nb block (nb <= 128) lives in
// shared memory with leading dimension kLDS = 129 (odd, so both row and
// column sweeps are bank-conflict free).  It is processed in 32-column
// sub-blocks: one warp factors / inverts each 32 x 32 diagonal sub-block in
// registers (lane = row, warp shuffles carry the pivots), and all eight warps
// apply the resulting panel solve and trailing update as shared-memory
// mini-GEMMs.  An upper triangle is handled as the lower triangle of its
// transpose (UVar3Unb and LVar3Unb perform the same operations on A and A^T).
constexpr int kLDS = 129;
constexpr int kXLD = 33;
constexpr int kDiagSmem = (128 * kLDS + 4 * 32 * kXLD) * (int)sizeof(double);

// Warp-level Cholesky of the w x w lower sub-block at S[c0.., c0..]
// (cholesky::LVar3Unb arithmetic, Cholesky/LVar3.hpp:19-49) followed by the
// inverse of the factor into X (column-major, ld kXLD).  Returns 0 or the
// 1-based column (within the sub-block) of a non-positive pivot.
__device__ int warp_chol32(double* S, int c0, int w, double* X) {
  const int lane = threadIdx.x & 31;
  double d[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) d[k] = (lane < w && k < w && k <= lane) ? S[c0 + lane + (c0 + k) * kLDS] : 0.0;
  int fail = 0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (j < w && !fail) {
      const double djj = __shfl_sync(0xffffffffu, d[j], j);
      if (djj <= 0.0) {
        fail = j + 1;
      } else {
        const double alpha = sqrt(djj);
        if (lane > j) d[j] /= alpha;
        else if (lane == j) d[j] = alpha;
        const double lj = d[j];
#pragma unroll
        for (int k = j + 1; k < 32; ++k) {
          const double lkj = __shfl_sync(0xffffffffu, lj, k);
          if (lane >= k) d[k] -= lj * lkj;
        }
      }
    }
  }
  if (fail) return fail;
#pragma unroll
  for (int k = 0; k < 32; ++k)
    if (lane < w && k <= lane) S[c0 + lane + (c0 + k) * kLDS] = d[k];
  // inverse: lane c computes column c of X = L^{-1} by forward substitution
  double x[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    double acc = (k == lane) ? 1.0 : 0.0;
#pragma unroll
    for (int m = 0; m < k; ++m) {
      const double lkm = __shfl_sync(0xffffffffu, d[m], k);
      acc = fma(-lkm, x[m], acc);
    }
    const double lkk = __shfl_sync(0xffffffffu, d[k], k);
    x[k] = (k >= lane && k < w) ? acc / lkk : 0.0;
  }
#pragma unroll
  for (int k = 0; k < 32; ++k)
    if (lane < w && k < w) X[k + lane * kXLD] = x[k];
  return 0;
}

// Warp-level inverse of the w x w lower sub-block at S[c0.., c0..] into X
// (unit: the diagonal is taken as 1).
__device__ void warp_trinv32(const double* S, int c0, int w, int unit, double* X) {
  const int lane = threadIdx.x & 31;
  double d[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    double v = (lane < w && k < w && k <= lane) ? S[c0 + lane + (c0 + k) * kLDS] : 0.0;
    if (unit && k == lane) v = 1.0;
    d[k] = v;
  }
  double x[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    double acc = (k == lane) ? 1.0 : 0.0;
#pragma unroll
    for (int m = 0; m < k; ++m) {
      const double lkm = __shfl_sync(0xffffffffu, d[m], k);
      acc = fma(-lkm, x[m], acc);
    }
    const double lkk = __shfl_sync(0xffffffffu, d[k], k);
    x[k] = (k >= lane && k < w) ? (unit ? acc : acc / lkk) : 0.0;
  }
#pragma unroll
  for (int k = 0; k < 32; ++k)
    if (lane < w && k < w) X[k + lane * kXLD] = x[k];
}

// Blocked in-place inverse of the lower b x b triangle in S, given the
// inverses of its 32 x 32 diagonal sub-blocks in Xd (block jb at
// Xd + jb*32*kXLD).  Block columns are processed last to first:
//   X21 = -inv(L22) * (L21 * X11),  inv(L22) already in place.
__device__ void block_trinv_inplace(double* S, int b, const double* Xd) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nsub = (b + 31) / 32;
  for (int jb = nsub - 1; jb >= 0; --jb) {
    const int c0 = 32 * jb, w = min(32, b - c0), r0 = c0 + w, R = b - r0;
    const double* X11 = Xd + jb * 32 * kXLD;
    if (R > 0) {
      double res[12];
#pragma unroll
      for (int i = 0; i < 12; ++i) {  // T = L21 * X11
        const int r = warp + 8 * i;
        double acc = 0.0;
        if (r < R && lane < w)
          for (int k = lane; k < w; ++k) acc = fma(S[r0 + r + (c0 + k) * kLDS], X11[k + lane * kXLD], acc);
        res[i] = acc;
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const int r = warp + 8 * i;
        if (r < R && lane < w) S[r0 + r + (c0 + lane) * kLDS] = res[i];
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < 12; ++i) {  // X21 = -inv(L22) * T
        const int r = warp + 8 * i;
        double acc = 0.0;
        if (r < R && lane < w)
          for (int m = 0; m <= r; ++m) acc = fma(S[r0 + r + (r0 + m) * kLDS], S[r0 + m + (c0 + lane) * kLDS], acc);
        res[i] = -acc;
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const int r = warp + 8 * i;
        if (r < R && lane < w) S[r0 + r + (c0 + lane) * kLDS] = res[i];
      }
    }
    for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
      const int i = idx % w, k = idx / w;
      if (i >= k) S[c0 + i + (c0 + k) * kLDS] = X11[i + k * kXLD];
    }
    __syncthreads();
  }
}

// Cholesky of the b x b diagonal block (cholesky::LVar3Unb,
// lapack-like/Cholesky/LVar3.hpp:19-49, or UVar3Unb, Cholesky/UVar3.hpp:21-50),
// followed by the inverse of the factor into W (other triangle zeroed).
template <int UPLO>
__global__ void __launch_bounds__(kDiagThreads) potrf_diag_kernel(double* A, long long lda, int b, double* W,
                                                                   int ldw, DevStatus* st, int col_base) {
  extern __shared__ double sm[];
  double* S = sm;
  double* Xd = sm + 128 * kLDS;
  __shared__ int s_fail;
  if (st != nullptr && st->code != 0) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int idx = tid; idx < b * b; idx += kDiagThreads) {
    const int r = idx % b, c = idx / b;
    if (r >= c) S[r + c * kLDS] = (UPLO == EGPU_LOWER) ? A[r + (long long)c * lda] : A[c + (long long)r * lda];
  }
  if (tid == 0) s_fail = 0;
  __syncthreads();
  const int nsub = (b + 31) / 32;
  for (int jb = 0; jb < nsub; ++jb) {
    const int c0 = 32 * jb, w = min(32, b - c0), r0 = c0 + w, R = b - r0;
    double* X11 = Xd + jb * 32 * kXLD;
    if (warp == 0) {
      const int f = warp_chol32(S, c0, w, X11);
      if (f && lane == 0) {
        s_fail = 1;
        set_status(st, kNotHPD, col_base + c0 + f);
      }
    }
    __syncthreads();
    if (s_fail) return;  // "A was not numerically HPD" (LVar3.hpp:37-38)
    if (R > 0) {
      // L21 := A21 * inv(L11)^T   (lane = column c: sum_{k<=c} A21[r,k] X11[c,k])
      double res[12];
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const int r = warp + 8 * i;
        double acc = 0.0;
        if (r < R && lane < w)
          for (int k = 0; k <= lane; ++k) acc = fma(S[r0 + r + (c0 + k) * kLDS], X11[lane + k * kXLD], acc);
        res[i] = acc;
      }
      __syncthreads();
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const int r = warp + 8 * i;
        if (r < R && lane < w) S[r0 + r + (c0 + lane) * kLDS] = res[i];
      }
      __syncthreads();
      // A22 -= L21 L21^T (lower)
      for (int c = r0 + warp; c < b; c += 8)
        for (int r = c + lane; r < b; r += 32) {
          double acc = 0.0;
#pragma unroll 8
          for (int k = 0; k < w; ++k) acc = fma(S[r + (c0 + k) * kLDS], S[c + (c0 + k) * kLDS], acc);
          S[r + c * kLDS] -= acc;
        }
      __syncthreads();
    }
  }
  for (int idx = tid; idx < b * b; idx += kDiagThreads) {
    const int r = idx % b, c = idx / b;
    if (r >= c) {
      if (UPLO == EGPU_LOWER) A[r + (long long)c * lda] = S[r + c * kLDS];
      else A[c + (long long)r * lda] = S[r + c * kLDS];
    }
  }
  __syncthreads();
  block_trinv_inplace(S, b, Xd);
  for (int idx = tid; idx < b * b; idx += kDiagThreads) {
    const int r = idx % b, c = idx / b;
    const double v = (r >= c) ? S[r + c * kLDS] : 0.0;
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
// lower or upper (as the transpose of a lower), unit or not.  The 32 x 32
// diagonal sub-blocks are inverted by four warps in parallel, then the
// blocked in-place substitution fills the rest.
__global__ void __launch_bounds__(kDiagThreads) trtri_blocks_kernel(int uplo, int unit, const double* A,
                                                                     long long lda, int n, int b, double* W,
                                                                     int ldw) {
  extern __shared__ double sm[];
  double* S = sm;
  double* Xd = sm + 128 * kLDS;
  const int blk = blockIdx.x;
  const int off = blk * b;
  const int bb = min(b, n - off);
  const double* Ab = A + off + (long long)off * lda;
  double* Wb = W + (long long)blk * b * ldw;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int idx = tid; idx < bb * bb; idx += kDiagThreads) {
    const int r = idx % bb, c = idx / bb;
    if (r >= c) S[r + c * kLDS] = (uplo == EGPU_LOWER) ? Ab[r + (long long)c * lda] : Ab[c + (long long)r * lda];
  }
  __syncthreads();
  const int nsub = (bb + 31) / 32;
  if (warp < nsub) warp_trinv32(S, 32 * warp, min(32, bb - 32 * warp), unit, Xd + warp * 32 * kXLD);
  __syncthreads();
  if (unit)  // the substitution reads unit diagonals from S
    for (int i = tid; i < bb; i += kDiagThreads) S[i + i * kLDS] = 1.0;
  __syncthreads();
  block_trinv_inplace(S, bb, Xd);
  for (int idx = tid; idx < b * b; idx += kDiagThreads) {
    const int r = idx % b, c = idx / b;
    double v = 0.0;
    if (r < bb && c < bb && r >= c) v = S[r + c * kLDS];
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
