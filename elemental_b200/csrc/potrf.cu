// Diagonal-block kernels: unblocked Cholesky / LU of one nb x nb block held in
// shared memory, and triangular inverses of diagonal blocks (the trsm sweeps
// multiply by these inverses on the tensor cores).
#include "diag_common.cuh"
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

// Cholesky of the b x b diagonal block (cholesky::LVar3Unb,
// lapack-like/Cholesky/LVar3.hpp:19-49, or UVar3Unb, Cholesky/UVar3.hpp:21-50),
// then the inverse of the factor into W (other triangle zeroed).
template <int UPLO>
__global__ void __launch_bounds__(kDiagThreads) potrf_diag_kernel(double* A, long long lda, int b, double* W,
                                                                   int ldw, DevStatus* st, int col_base,
                                                                   int store_factor) {
  extern __shared__ double S[];
  if (st != nullptr && st->code != 0) return;
  const int tid = threadIdx.x;
  tri_load_async(S, A, lda, b, UPLO != EGPU_LOWER);
  cp_async_wait_all();
  __syncthreads();
  double* Xl = S + 128 * kLDS + 128;
  double* T = Xl + 8 * 16 * kLeafLD;
  const int bp = pad16_identity(S, b);
  __syncthreads();
  const int f = smem_chol_dmma(S, bp, Xl, T);
  if (f) {
    if (tid == 0) set_status(st, kNotHPD, col_base + f);
    return;
  }
  if (store_factor) tri_store(S, A, lda, b, UPLO != EGPU_LOWER, false);
  __syncthreads();
  smem_trinv_dmma(S, bp, Xl, T);
  tri_store(S, W, ldw, b, UPLO != EGPU_LOWER, true);  // inv(U) = inv(L)^T
  if (b < ldw)  // a short last block: the rest of its ldw x ldw slot is zero (whole-slot readers)
    for (int e = tid; e < ldw * ldw; e += kDiagThreads) {
      const int i = e % ldw, j = e / ldw;
      if (i >= b || j >= b) W[i + (long long)j * ldw] = 0.0;
    }
}

// The mixed path's diagonal block (lower): the FP32 block of the trailing
// matrix, widened on load, factored and inverted in FP64 as above; the
// inverse goes to W (FP64, for the solves) and, split into TF32 hi/lo rows,
// to Wh/Wl (the B operand of the panel's L21 product on the tensor cores).
// Both big transfers go through the TMA engine: the block arrives as one
// 128 x 128 FP32 box (staged in S's first 64 KB, widened in place: every
// thread reads its values before any writes), and W leaves as one 132 x 128
// FP64 box straight from S (pitch 132; the rows past the slot are clipped)
// while the threads write the split.
__global__ void __launch_bounds__(kDiagThreads) potrf_diag_f32_kernel(const __grid_constant__ CUtensorMap mapA,
                                                                       const __grid_constant__ CUtensorMap mapW,
                                                                       int b, float* Wh, float* Wl, long long ldk,
                                                                       DevStatus* st, int col_base) {
  extern __shared__ __align__(128) double S[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_go;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  static_assert(kDiagThreads == 256, "a warp per 16 columns of the 128 x 128 block");
  float* stage = reinterpret_cast<float*>(S);  // the FP32 box, [i + j * 128]
  if (tid == 0) {
    int go = st == nullptr || st->code == 0;
    if (go && smem_u32(S) % 128 != 0) {  // no TMA into a misaligned buffer
      set_status(st, kTimeout, 205);
      go = 0;
    }
    if (go) {
      mbar_init(&bar, 1);
      fence_mbar_init();
      mbar_expect_tx(&bar, 128u * 128u * 4u);
      tma_load_2d(stage, &mapA, &bar, 0, 0);
      if (!mbar_wait_bounded(&bar, 0)) {  // the box never landed: report, do not touch it
        set_status(st, kTimeout, 206);
        go = 0;
      }
    }
    s_go = go;
  }
  __syncthreads();
  if (!s_go) return;
  (void)mbar_wait_bounded(&bar, 0);  // completed: every thread observes the box's arrival
  {  // widen the lower triangle: warp w holds columns w, w + 8, ..
    float v[16][4];
#pragma unroll
    for (int u = 0; u < 16; ++u)
#pragma unroll
      for (int t = 0; t < 4; ++t) v[u][t] = stage[(lane + 32 * t) + (warp + 8 * u) * 128];
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 16; ++u)
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int j = warp + 8 * u, i = lane + 32 * t;
        if (j < b && i >= j && i < b) S[i + j * kLDS] = (double)v[u][t];
      }
  }
  __syncthreads();
  double* Xl = S + 128 * kLDS + 128;
  double* T = Xl + 8 * 16 * kLeafLD;
  const int bp = pad16_identity(S, b);
  __syncthreads();
  const int f = smem_chol_dmma(S, bp, Xl, T);
  if (f) {
    if (tid == 0) set_status(st, kNotHPD, col_base + f);
    return;
  }
  __syncthreads();
  smem_trinv_dmma(S, bp, Xl, T);
  __syncthreads();
  // W's slot: inv(L) below and on the diagonal, zero above it and outside b x b
  for (int j = warp; j < 128; j += kDiagThreads / 32)
    for (int i = lane; i < 128; i += 32)
      if (i < j || i >= b || j >= b) S[i + j * kLDS] = 0.0;
  fence_proxy_async_smem();  // the zeros (and the inverse) are read by the TMA store
  __syncthreads();
  if (tid == 0) {
    tma_store_2d(&mapW, S, 0, 0);
    bulk_commit();
  }
  for (int j = warp; j < 128; j += kDiagThreads / 32) {  // row j of inv(L), a warp per row
    float* wh = Wh + (long long)j * ldk;
    float* wl = Wl + (long long)j * ldk;
    for (int k = lane; k < (int)ldk; k += 32) {
      const double vv = k < 128 ? S[j + k * kLDS] : 0.0;  // zero above the diagonal and outside b x b
      const float hv = tf32_rna((float)vv);
      wh[k] = hv;
      wl[k] = tf32_rna((float)(vv - (double)hv));
    }
  }
  if (tid == 0) bulk_wait_all();  // the store has read S and landed before the block retires
}

int launch_potrf_diag_f32(cudaStream_t st, const float* Af, long long ldf, int b, double* W, int ldw, float* Wh,
                          float* Wl, long long ldk, DevStatus* status, int col_base) {
  if (b <= 0) return EGPU_OK;
  if (b > kMaxNB || ldk < b || ldw > 128 || ldw < b || ldk % 4 != 0 || ldf % 4 != 0 ||
      reinterpret_cast<uintptr_t>(Af) % 16 != 0 || reinterpret_cast<uintptr_t>(W) % 16 != 0)
    return EGPU_ERR_ARG;
  CUtensorMap mapA, mapW;
  if (!make_tma_2d(&mapA, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, Af, b, b, 4ull * ldf, 128, 128, false) ||
      !make_tma_2d(&mapW, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, W, ldw, ldw, 8ull * ldw, kLDS, 128, false))
    return EGPU_ERR_TMA;
  TraceMark tm(st, kTraceDiag, (double)b * b * b / 3.0 * 2.0, 12.0 * b * b);
  cudaError_t e = cudaFuncSetAttribute(potrf_diag_f32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kDiagSmem);
  if (e == cudaSuccess) {
    potrf_diag_f32_kernel<<<1, kDiagThreads, kDiagSmem, st>>>(mapA, mapW, b, Wh, Wl, ldk, status, col_base);
    count_launch();
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_last_error(e, "potrf_diag_f32 launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

int launch_potrf_diag(cudaStream_t st, int uplo, double* A, long long lda, int b, double* W, int ldw,
                      DevStatus* status, int col_base, bool store_factor) {
  if (b <= 0) return EGPU_OK;
  if (b > kMaxNB) return EGPU_ERR_ARG;
  const size_t smem = kDiagSmem;
  TraceMark tm(st, kTraceDiag, (double)b * b * b / 3.0 * 2.0, 16.0 * b * b);
  cudaError_t e;
  if (uplo == EGPU_LOWER) {
    e = cudaFuncSetAttribute(potrf_diag_kernel<EGPU_LOWER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kDiagSmem);
    if (e == cudaSuccess)
      potrf_diag_kernel<EGPU_LOWER><<<1, kDiagThreads, smem, st>>>(A, lda, b, W, ldw, status, col_base,
                                                            store_factor ? 1 : 0);
      count_launch();
  } else {
    e = cudaFuncSetAttribute(potrf_diag_kernel<EGPU_UPPER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kDiagSmem);
    if (e == cudaSuccess)
      potrf_diag_kernel<EGPU_UPPER><<<1, kDiagThreads, smem, st>>>(A, lda, b, W, ldw, status, col_base,
                                                            store_factor ? 1 : 0);
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
  tri_load_async(S, Ab, lda, bb, uplo != EGPU_LOWER);
  cp_async_wait_all();
  __syncthreads();
  double* Xl = S + 128 * kLDS + 128;
  double* T = Xl + 8 * 16 * kLeafLD;
  const int bp = pad16_identity(S, bb);
  __syncthreads();
  const int warp = tid >> 5;
  for (int q = warp; q < bp / 16; q += kDiagThreads / 32)
    warp_trinv16(S, kLDS, 16 * q, unit, Xl + q * 16 * kLeafLD, kLeafLD);
  __syncthreads();
  smem_trinv_dmma(S, bp, Xl, T);
  tri_store(S, Wb, ldw, bb, uplo != EGPU_LOWER, true);
  if (bb < b)  // a short last block: the rest of its b x b slot is zero
    for (int e = tid; e < b * b; e += kDiagThreads) {
      const int i = e % b, j = e / b;
      if (i >= bb || j >= bb) Wb[i + (long long)j * ldw] = 0.0;
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
