// Small kernels behind TriangularInverse / Inverse / HPDInverse, the
// (Safe)Determinant entry points, ReverseCholesky and LDL: an identity fill (the
// right-hand side the inverses are solved against), a triangle copy (the
// inverse written back over the caller's triangle only), a 180-degree
// triangle rotation (the reverse factorization as a forward one), the
// symmetric staging and write-back of LDL's diagonal blocks and one
// deterministic reduction over the diagonal of a factor.
#include "internal.h"

namespace egpu {

namespace {

__global__ void set_identity_kernel(int n, double* X, long long ldx) {
  const long long total = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    X[i + j * ldx] = i == j ? 1.0 : 0.0;
  }
}

// D's uplo triangle (strict: without the diagonal) := S's; the rest of D is
// not touched.
__global__ void copy_triangle_kernel(int uplo, int strict, int n, const double* S, long long lds, double* D,
                                     long long ldd) {
  const long long total = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    const bool in = uplo == EGPU_LOWER ? (strict ? i > j : i >= j) : (strict ? i < j : i <= j);
    if (in) D[i + j * ldd] = S[i + j * lds];
  }
}

// out[0] = sum_i log|a_ii|, out[1] = number of negative a_ii, out[2] = number
// of i with p[i] != i (p may be null).  One block; every thread sums a fixed
// stride, then a fixed-shape tree: the result does not depend on timing.
constexpr int kDiagReduceThreads = 256;
__global__ void __launch_bounds__(kDiagReduceThreads) diag_logsum_kernel(int n, const double* A, long long lda,
                                                                          const int* p, double* out) {
  __shared__ double s_log[kDiagReduceThreads], s_neg[kDiagReduceThreads], s_swp[kDiagReduceThreads];
  const int t = threadIdx.x;
  double lg = 0.0, ng = 0.0, sw = 0.0;
  for (int i = t; i < n; i += kDiagReduceThreads) {
    const double d = A[i + (long long)i * lda];
    lg += log(fabs(d));
    ng += d < 0.0 ? 1.0 : 0.0;
    if (p != nullptr && p[i] != i) sw += 1.0;
  }
  s_log[t] = lg;
  s_neg[t] = ng;
  s_swp[t] = sw;
  __syncthreads();
  for (int w = kDiagReduceThreads / 2; w > 0; w >>= 1) {
    if (t < w) {
      s_log[t] += s_log[t + w];
      s_neg[t] += s_neg[t + w];
      s_swp[t] += s_swp[t + w];
    }
    __syncthreads();
  }
  if (t == 0) {
    out[0] = s_log[0];
    out[1] = s_neg[0];
    out[2] = s_swp[0];
  }
}

// D[n-1-i, n-1-j] := S[i, j] for (i, j) in S's uplo triangle (a 180-degree
// rotation, which maps S's uplo triangle onto D's other triangle).
__global__ void rotate_triangle_kernel(int uplo, int n, const double* S, long long lds, double* D, long long ldd) {
  const long long total = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    if (uplo == EGPU_LOWER ? i >= j : i <= j) D[(n - 1 - i) + (long long)(n - 1 - j) * ldd] = S[i + j * lds];
  }
}

// The b x b symmetric block whose lower triangle is A11's: Blk[i][j] =
// A11[max(i,j)][min(i,j)] (A11's upper triangle is not read).
__global__ void sym_from_lower_kernel(int b, const double* A, long long lda, double* Blk, long long ldb) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < b * b; e += gridDim.x * blockDim.x) {
    const int i = e % b, j = e / b;
    Blk[i + (long long)j * ldb] = i >= j ? A[i + (long long)j * lda] : A[j + (long long)i * lda];
  }
}

// From the unpivoted LU L\U of a symmetric block: A11's strict lower
// triangle := L's, its diagonal (and d, when given) := U's diagonal (D).
__global__ void ldl_block_writeback_kernel(int b, const double* Blk, long long ldb, double* A, long long lda,
                                           double* d) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < b * b; e += gridDim.x * blockDim.x) {
    const int i = e % b, j = e / b;
    if (i < j) continue;
    const double v = Blk[i + (long long)j * ldb];
    A[i + (long long)j * lda] = v;
    if (i == j && d != nullptr) d[i] = v;
  }
}

int grid_for(long long elems) {
  return (int)std::max<long long>(1, std::min<long long>((elems + 255) / 256, 148 * 16));
}

}  // namespace

int launch_set_identity(cudaStream_t st, int n, double* X, long long ldx) {
  if (n <= 0) return EGPU_OK;
  set_identity_kernel<<<grid_for((long long)n * n), 256, 0, st>>>(n, X, ldx);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "set_identity launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

int launch_copy_triangle(cudaStream_t st, int uplo, bool strict, int n, const double* S, long long lds, double* D,
                         long long ldd) {
  if (n <= 0) return EGPU_OK;
  copy_triangle_kernel<<<grid_for((long long)n * n), 256, 0, st>>>(uplo, strict ? 1 : 0, n, S, lds, D, ldd);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "copy_triangle launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

int launch_rotate_triangle(cudaStream_t st, int uplo, int n, const double* S, long long lds, double* D,
                           long long ldd) {
  if (n <= 0) return EGPU_OK;
  rotate_triangle_kernel<<<grid_for((long long)n * n), 256, 0, st>>>(uplo, n, S, lds, D, ldd);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "rotate_triangle launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

int launch_sym_from_lower(cudaStream_t st, int b, const double* A, long long lda, double* Blk, long long ldb) {
  if (b <= 0) return EGPU_OK;
  sym_from_lower_kernel<<<grid_for((long long)b * b), 256, 0, st>>>(b, A, lda, Blk, ldb);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "sym_from_lower launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

int launch_ldl_block_writeback(cudaStream_t st, int b, const double* Blk, long long ldb, double* A, long long lda,
                               double* d) {
  if (b <= 0) return EGPU_OK;
  ldl_block_writeback_kernel<<<grid_for((long long)b * b), 256, 0, st>>>(b, Blk, ldb, A, lda, d);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "ldl_block_writeback launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

int launch_diag_logsum(cudaStream_t st, int n, const double* A, long long lda, const int* p, double* out) {
  diag_logsum_kernel<<<1, kDiagReduceThreads, 0, st>>>(n, A, lda, p, out);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "diag_logsum launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

}  // namespace egpu
