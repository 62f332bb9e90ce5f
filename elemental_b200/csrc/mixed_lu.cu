// Mixed-precision LU solve with partial pivoting: GaussianElimination's x
// (GaussianElimination.hpp:216-232, LU.hpp:144-218 then lu::SolveAfter,
// LU/SolveAfter.hpp:101-146) at FP64-level backward error, the O(n^3) work
// on the tcgen05 tensor cores.
//
// The working matrix is an FP32 copy of A.  Per 128-wide panel k:
//   1. the panel (rows k..n) is widened to FP64 and factored by the FP64
//      pivoting panel kernel (lu::Panel, LU/Panel.hpp:19-89: the first maximal
//      |a| of each column, swaps, scaling, rank-1 updates), which also gives
//      the composed row permutation and W = inv(unit L11);
//   2. the panel goes back into the FP32 matrix and its interchanges are
//      applied to every other column (ApplyRowPivots, ApplyRowPivots.hpp:129-181);
//   3. U12 = W A12 and A22 -= L21 U12 on the tensor cores (TF32 x 3 split
//      products, FP32 accumulation: the Trsm and Gemm of LU.hpp:202-203).
// The factors (FP32-accurate) are widened once, and refinement runs with FP64
// residuals r = b - A x against the untouched A and corrections through the
// factors' one-launch triangular sweeps (pivots, unit-lower L, upper U); when
// plain refinement contracts slowly -- or, with policy 1, when the 1-norm
// condition estimate says so -- GMRES-IR preconditioned by the same factors.
#include <cmath>
#include <vector>

#include "context.h"

// the FP64 LU and its solve (api.cu)
int getrf_core(egpu_context* h, int m, int n, double* A, long long lda, int* dp, double* B, long long ldb, int nrhs,
               bool pivot_left);
int getrs_core(egpu_context* h, int orient, int n, int nrhs, const double* A, long long lda, const int* dp,
               double* B, long long ldb);

namespace egpu {

namespace {

constexpr int kFallbackFp64 = 1000;  // internal: the FP32 factors do not suffice

// D (FP64, ld ldd) = S (FP32, ld lds), m x w
__global__ void widen_kernel(int m, int w, const float* S, long long lds, double* D, long long ldd) {
  for (int c = blockIdx.y; c < w; c += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
      D[i + (long long)c * ldd] = (double)S[i + (long long)c * lds];
}

// D (FP32, ld ldd) = S (FP64, ld lds), m x w
__global__ void narrow_kernel(int m, int w, const double* S, long long lds, float* D, long long ldd) {
  for (int c = blockIdx.y; c < w; c += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
      D[i + (long long)c * ldd] = (float)S[i + (long long)c * lds];
}

// ApplyRowPivots(A, image, preimage) on an FP32 matrix: row i (< b) moves to
// image[i]; row preimage[i] (>= b) moves into row i (the FP64 form is
// apply_composed_kernel, lu_panel.cu).
__global__ void __launch_bounds__(128) apply_composed_f32_kernel(int ncols, float* A, long long lda, int b,
                                                                 const int* image, const int* preimage) {
  const int i = threadIdx.x;
  const int img = (i < b) ? image[i] : 0;
  const int pre = (i < b) ? preimage[i] : 0;
  constexpr int G = 8;
  for (int c0 = blockIdx.x * G; c0 < ncols; c0 += gridDim.x * G) {
    float v1[G], v2[G];
#pragma unroll
    for (int q = 0; q < G; ++q) {
      const int c = c0 + q;
      if (c < ncols && i < b) {
        v1[q] = A[i + (long long)c * lda];
        v2[q] = (pre >= b) ? A[pre + (long long)c * lda] : 0.f;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < G; ++q) {
      const int c = c0 + q;
      if (c < ncols && i < b) {
        A[img + (long long)c * lda] = v1[q];
        if (pre >= b) A[i + (long long)c * lda] = v2[q];
      }
    }
    __syncthreads();
  }
}

// X (k x N block of an FP32 column-major matrix, ld ldx) -> its transpose's
// TF32 split in K-major rows: hi[c * ldk + kk] = X[kk, c] (kk < k; columns k..
// ldk-1 zero), the B operand (N x K) of C = A B^T.
__global__ void split_tf32_t_kernel(int k, int N, const float* X, long long ldx, float* hi, float* lo, long long ldk) {
  const int c = blockIdx.x;
  for (int kk = threadIdx.x; kk < ldk; kk += blockDim.x) {
    const float x = kk < k ? X[kk + (long long)c * ldx] : 0.f;
    const float h = tf32_rna(x);
    hi[(long long)c * ldk + kk] = h;
    lo[(long long)c * ldk + kk] = tf32_rna(x - h);
  }
}

// Row sums (||A||_inf, the backward error's norm) and column sums (||A||_1,
// the condition estimate's) of |A|: rows[i] by one thread per row, cols[j] by
// one warp per column (contiguous loads, fixed summation order)
__global__ void abs_sums_kernel(int n, const double* A, long long lda, double* rows, double* cols) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += fabs(A[t + (long long)j * lda]);
    rows[t] = s;
  }
  const int lane = threadIdx.x & 31, j = t >> 5;
  if (j < n) {
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += fabs(A[i + (long long)j * lda]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) cols[j] = s;
  }
}

// UT := the transpose of Af's upper triangle (32 x 32 tiles through shared
// memory; only tiles on or above Af's diagonal, so UT's lower triangle is U^T)
__global__ void transpose_upper_kernel(int n, const float* Af, long long ldf, float* UT) {
  __shared__ float tile[32][33];
  const int bi = blockIdx.x, bj = blockIdx.y;  // tile row / column of Af
  if (bj < bi) return;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int q = ty; q < 32; q += 8) {
    const int r = bi * 32 + tx, c = bj * 32 + q;
    tile[q][tx] = (r < n && c < n) ? Af[r + (long long)c * ldf] : 0.f;
  }
  __syncthreads();
  for (int q = ty; q < 32; q += 8) {
    const int r = bj * 32 + tx, c = bi * 32 + q;  // UT(r, c) = Af(c, r)
    if (r < n && c < n) UT[r + (long long)c * ldf] = tile[tx][q];
  }
}

// The 128 x 128 diagonal blocks of the unit-lower L and of U^T, widened to
// FP64 and packed (block q at q * 128 * 129, ld 128) for the batched inverse.
__global__ void diag_blocks_kernel(int n, const float* Af, long long ldf, double* DL, double* DU) {
  const int q = blockIdx.x, b = min(128, n - q * 128);
  double* dl = DL + (long long)q * 128 * 129;
  double* du = DU + (long long)q * 128 * 129;
  const long long o = (long long)q * 128;
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int i = e % b, j = e / b;
    dl[i + j * 128] = i >= j ? (double)Af[(o + i) + (o + j) * ldf] : 0.0;
    du[i + j * 128] = i >= j ? (double)Af[(o + j) + (o + i) * ldf] : 0.0;
  }
}

}  // namespace

// Workspace of the mixed LU solve.
struct MixedLuLayout {
  size_t as, af, lu, pan, piv, img, pre, w, scr, wh, wl, bh, bl, lh, ll, winvl, winvu, flags, perm, xw, r, norms, gv, gw, gc,
      ut, dl, du, winvut, swl, swu, permi, total;
  long long ldf, lds, ldk;
};

static MixedLuLayout mixed_lu_layout(int n, int nrhs, int nb, int fb, int sm_count, bool copy_a) {
  MixedLuLayout L;
  L.lds = ld_aligned(n);
  L.ldf = L.lds;
  L.ldk = ((long long)fb + 31) / 32 * 32;
  size_t off = 0;
  auto take = [&](size_t bytes) { off = (off + 1023) & ~size_t(1023); size_t o = off; off += bytes; return o; };
  const int r = std::max(nrhs, 1);
  L.as = copy_a ? take(sizeof(double) * L.lds * n) : 0;  // an aligned copy of A for the FP64 products
  L.af = take(sizeof(float) * L.ldf * n);
  L.lu = take(sizeof(double) * L.lds * n);                    // the widened factors (solves)
  L.pan = take(sizeof(double) * L.lds * fb);                   // one FP64 panel
  L.piv = take(sizeof(int) * (size_t)n);
  L.img = take(sizeof(int) * (size_t)fb);
  L.pre = take(sizeof(int) * (size_t)fb);
  L.w = take(sizeof(double) * (size_t)fb * fb);
  L.scr = take(lu_panel_scratch_bytes(n, fb, sm_count));
  L.wh = take(sizeof(float) * (size_t)fb * L.ldk);
  L.wl = take(sizeof(float) * (size_t)fb * L.ldk);
  L.bh = take(sizeof(float) * (size_t)n * L.ldk);
  L.bl = take(sizeof(float) * (size_t)n * L.ldk);
  L.lh = take(sizeof(float) * (size_t)n * L.ldk);
  L.ll = take(sizeof(float) * (size_t)n * L.ldk);
  L.winvl = take(winv_bytes(n, nb));
  L.winvu = take(winv_bytes(n, nb));
  L.flags = take(trsm_skinny_flag_bytes(n, nb));
  if (nrhs <= 32) {  // the FP32 sweeps: U^T, the packed diagonal blocks, two sweep workspaces
    const size_t nblk = (size_t)(n + nb - 1) / nb;
    L.ut = take(sizeof(float) * L.ldf * n);
    L.dl = take(sizeof(double) * nblk * 128 * 129);
    L.du = take(sizeof(double) * nblk * 128 * 129);
    L.winvut = take(winv_bytes(n, nb));
    L.swl = take(sweep32_ws_bytes(n, nrhs));
    L.swu = take(sweep32_ws_bytes(n, nrhs));
  }
  L.perm = take(align_up(sizeof(int) * (size_t)((n + 1) & ~1), 256) + sizeof(double) * (size_t)n * r);
  L.permi = take(sizeof(int) * (size_t)n);  // the inverse row permutation
  L.xw = take(sizeof(double) * L.lds * r);
  L.r = take(sizeof(double) * L.lds * r);
  L.norms = take(sizeof(double) * (2 * (size_t)n + 4 * (size_t)r));
  L.gv = take(sizeof(double) * L.lds * r * (kGmresRestart + 1));
  L.gw = take(sizeof(double) * L.lds * r);
  L.gc = take(sizeof(double) * (size_t)r * (kGmresRestart + 2) * 2);
  L.total = (off + 4095) & ~size_t(4095);
  return L;
}

// An FP64 LU solve refined the same way, for the matrices whose low-precision
// factors do not precondition well enough (the condition estimate asks for it,
// or GMRES-IR stagnates): GaussianElimination's plain path on a copy of A.
// getrf_core and getrs_core carve their scratch from the start of the
// workspace; the copy, pivots and refinement vectors sit past a bound on it.

static int dgesv_fp64_refined(egpu_context* h, int n, int nrhs, const double* A, long long lda, const double* B,
                              long long ldb, double* X, long long ldx, int max_iter, double tol, int* iters,
                              double* berr) {
  const int nb = h->nb;
  const long long lds = ld_aligned(n);
  const size_t core = align_up(4 * winv_bytes(n, nb) + trsm_skinny_flag_bytes(n, nb) + sizeof(int) * (size_t)n +
                                   sizeof(double) * (size_t)n * nrhs + lu_panel_scratch_bytes(n, nb, h->sm_count) +
                                   2 * (sizeof(double) * (size_t)nb * nb + 2 * sizeof(int) * nb + 512) + (64 << 10),
                               1 << 20);
  size_t off = core;
  auto take = [&](size_t bytes) { off = align_up(off, 1024); const size_t o = off; off += bytes; return o; };
  const size_t o_lu = take(sizeof(double) * lds * n), o_piv = take(sizeof(int) * (size_t)n),
               o_xw = take(sizeof(double) * lds * nrhs), o_r = take(sizeof(double) * lds * nrhs),
               o_nrm = take(sizeof(double) * (2 * (size_t)n + 4 * (size_t)nrhs));
  TRY(ensure_ws(h, off + 4096));
  unsigned char* ws = static_cast<unsigned char*>(h->ws);
  double* LU = reinterpret_cast<double*>(ws + o_lu);
  int* piv = reinterpret_cast<int*>(ws + o_piv);
  double* Xw = reinterpret_cast<double*>(ws + o_xw);
  double* R = reinterpret_cast<double*>(ws + o_r);
  double* norms = reinterpret_cast<double*>(ws + o_nrm);
  cudaStream_t st = h->stream;
  TRY(launch_copy_cols(st, n, n, A, lda, LU, lds, 0));
  TRY(::getrf_core(h, n, n, LU, lds, piv, nullptr, 0, 0, true));
  TRY(read_status_now(h, nullptr));
  TRY(launch_copy_cols(st, n, nrhs, B, ldb, Xw, lds, 0));
  TRY(::getrs_core(h, EGPU_NORMAL, n, nrhs, LU, lds, piv, Xw, lds));
  abs_sums_kernel<<<(32 * n + 255) / 256, 256, 0, st>>>(n, A, lda, norms, norms + n);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  std::vector<double> rs(n);
  EGPU_CUDA_TRY(cudaMemcpyAsync(rs.data(), norms, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  EGPU_CUDA_TRY(cudaStreamSynchronize(st));
  double anorm = 0.0;
  for (double v : rs) anorm = std::max(anorm, v);
  int it = iters ? *iters : 0;
  double e = INFINITY;
  for (;;) {
    TRY(launch_copy_cols(st, n, nrhs, B, ldb, R, lds, 0));
    int rg = launch_dgemm_skinny(st, n, nrhs, n, -1.0, A, lda, Xw, lds, R, lds, h->sm_count, h->dstatus);
    if (rg == EGPU_ERR_UNSUPPORTED)
      rg = launch_dgemm(st, false, true, n, nrhs, n, -1.0, A, lda, Xw, lds, 1.0, R, lds, 0, false, h->dstatus);
    TRY(rg);
    const double e_prev = e;
    TRY(mixed_berr(h, n, nrhs, R, Xw, B, ldb, lds, anorm, norms + 2 * n, &e));
    if (e <= tol || it >= max_iter || !std::isfinite(e) || e > 0.5 * e_prev) break;
    TRY(::getrs_core(h, EGPU_NORMAL, n, nrhs, LU, lds, piv, R, lds));
    TRY(launch_copy_cols(st, n, nrhs, R, lds, Xw, lds, 1));
    ++it;
  }
  TRY(launch_copy_cols(st, n, nrhs, Xw, lds, X, ldx, 0));
  if (iters) *iters = it;
  if (berr) *berr = e;
  TRY(read_status_now(h, nullptr));
  return e <= tol ? EGPU_OK : EGPU_NO_CONVERGENCE;
}

int dgesv_mixed_core(egpu_context* h, int n, int nrhs, const double* A, long long lda, const double* B, long long ldb,
                     double* X, long long ldx, int max_iter, double tol, int* iters, double* berr) {
  const int nb = 128;  // the solves' diagonal blocks
  // the factorization's panel width: the handle's block size (a multiple of
  // 32 up to 128)
  const int fb = std::max(32, std::min(128, h->nb / 32 * 32));
  cudaStream_t st = h->stream;
  const bool copy_a = !tma_compatible(A, lda);
  const MixedLuLayout L = mixed_lu_layout(n, nrhs, nb, fb, h->sm_count, copy_a);
  TRY(ensure_ws(h, L.total + 4096));
  unsigned char* ws = static_cast<unsigned char*>(h->ws);
  if (copy_a) {  // the residual products read A through 16-byte loads
    double* As = reinterpret_cast<double*>(ws + L.as);
    TRY(launch_copy_cols(st, n, n, A, lda, As, L.lds, 0));
    A = As;
    lda = L.lds;
  }
  float* Af = reinterpret_cast<float*>(ws + L.af);
  double* LU = reinterpret_cast<double*>(ws + L.lu);
  double* P = reinterpret_cast<double*>(ws + L.pan);
  int* piv = reinterpret_cast<int*>(ws + L.piv);
  int* image = reinterpret_cast<int*>(ws + L.img);
  int* preimage = reinterpret_cast<int*>(ws + L.pre);
  double* W = reinterpret_cast<double*>(ws + L.w);
  float *Wh = reinterpret_cast<float*>(ws + L.wh), *Wl = reinterpret_cast<float*>(ws + L.wl);
  float *Bh = reinterpret_cast<float*>(ws + L.bh), *Bl = reinterpret_cast<float*>(ws + L.bl);
  float *Lh = reinterpret_cast<float*>(ws + L.lh), *Ll = reinterpret_cast<float*>(ws + L.ll);
  double* WinvL = reinterpret_cast<double*>(ws + L.winvl);
  double* WinvU = reinterpret_cast<double*>(ws + L.winvu);
  int* flags = reinterpret_cast<int*>(ws + L.flags);
  int* perm = reinterpret_cast<int*>(ws + L.perm);
  double* Xw = reinterpret_cast<double*>(ws + L.xw);
  double* R = reinterpret_cast<double*>(ws + L.r);
  double* norms = reinterpret_cast<double*>(ws + L.norms);
  const long long ldf = L.ldf, lds = L.lds, ldk = L.ldk;
  EGPU_CUDA_TRY(cudaMemsetAsync(h->dstatus, 0, sizeof(DevStatus), st));
  // ---- the FP32 working matrix
  {
    dim3 grid((n + 255) / 256, std::min(n, 65535));
    // narrow A column by column (FP64 -> FP32)
    narrow_kernel<<<grid, 256, 0, st>>>(n, n, A, lda, Af, ldf);
    count_launch();
    EGPU_CUDA_TRY(cudaGetLastError());
  }
  // ---- factorization
  for (int k = 0; k < n; k += fb) {
    const int b = std::min(fb, n - k), m = n - k, n2 = n - k - b;
    float* Ak = Af + k + (long long)k * ldf;
    {
      TraceMark tm(st, kTraceOther, 0.0, 12.0 * m * b);
      widen_kernel<<<dim3((m + 255) / 256, b), 256, 0, st>>>(m, b, Ak, ldf, P, lds);
      count_launch();
      EGPU_CUDA_TRY(cudaGetLastError());
    }
    TRY(launch_lu_panel(st, m, b, P, lds, piv + k, k, image, preimage, W, fb, ws + L.scr, h->dstatus, h->sm_count));
    {
      TraceMark tm(st, kTraceOther, 0.0, 12.0 * m * b);
      narrow_kernel<<<dim3((m + 255) / 256, b), 256, 0, st>>>(m, b, P, lds, Ak, ldf);
      count_launch();
      EGPU_CUDA_TRY(cudaGetLastError());
    }
    // interchanges on the columns left and right of the panel (rows k..n)
    {
      TraceMark tm(st, kTraceSwap, 0.0, 16.0 * b * (n - b));
      if (k > 0) {
        apply_composed_f32_kernel<<<std::min((k + 7) / 8, 148 * 8), 128, 0, st>>>(k, Af + k, ldf, b, image,
                                                                                   preimage);
        count_launch();
      }
      if (n2 > 0) {
        apply_composed_f32_kernel<<<std::min((n2 + 7) / 8, 148 * 8), 128, 0, st>>>(
            n2, Af + k + (long long)(k + b) * ldf, ldf, b, image, preimage);
        count_launch();
      }
      EGPU_CUDA_TRY(cudaGetLastError());
    }
    if (n2 == 0) continue;
    float* A12 = Af + k + (long long)(k + b) * ldf;
    float* A22 = Af + (k + b) + (long long)(k + b) * ldf;
    // U12 = W A12: A = W (b x b, K-major rows), B = A12^T (n2 x b)
    TRY(launch_split_tf32(st, b, b, W, fb, Wh, Wl, ldk));
    {
      TraceMark tm(st, kTraceOther, 0.0, 12.0 * b * n2);
      split_tf32_t_kernel<<<n2, 128, 0, st>>>(b, n2, A12, ldf, Bh, Bl, ldk);
      count_launch();
      EGPU_CUDA_TRY(cudaGetLastError());
    }
    TRY(launch_tc_gemm(st, b, n2, b, 1.0f, Wh, Wl, Bh, Bl, ldk, 0.0f, A12, ldf, 0, 3, h->dstatus));
    // A22 -= L21 U12: A = L21 (n2 x b, from the FP64 panel), B = U12^T (n2 x b)
    TRY(launch_split_tf32(st, n2, b, P + b, lds, Lh, Ll, ldk));
    {
      TraceMark tm(st, kTraceOther, 0.0, 12.0 * b * n2);
      split_tf32_t_kernel<<<n2, 128, 0, st>>>(b, n2, A12, ldf, Bh, Bl, ldk);
      count_launch();
      EGPU_CUDA_TRY(cudaGetLastError());
    }
    TRY(launch_tc_gemm(st, n2, n2, b, -1.0f, Lh, Ll, Bh, Bl, ldk, 1.0f, A22, ldf, 0, 3, h->dstatus));
  }
  TRY(read_status_now(h, nullptr));  // an exact zero pivot: SingularMatrixException
  // ---- the solves.  With nrhs <= 32 the refinement's corrections and the
  // condition estimate sweep the FP32 factors directly (L from Af, U through
  // its transpose UT; one-launch dataflow sweeps over explicit super-block
  // inverses); GMRES-IR, which needs its preconditioner applied in FP64,
  // sweeps an FP64 copy of the factors made when it is first needed.
  const bool use32 = nrhs <= 32;
  const int nblk = (n + nb - 1) / nb;
  float* UT = use32 ? reinterpret_cast<float*>(ws + L.ut) : nullptr;
  void* swl = use32 ? static_cast<void*>(ws + L.swl) : nullptr;
  void* swu = use32 ? static_cast<void*>(ws + L.swu) : nullptr;
  if (use32) {
    double* DL = reinterpret_cast<double*>(ws + L.dl);
    double* DU = reinterpret_cast<double*>(ws + L.du);
    double* WinvUT = reinterpret_cast<double*>(ws + L.winvut);
    const int nt = (n + 31) / 32;
    transpose_upper_kernel<<<dim3(nt, nt), dim3(32, 8), 0, st>>>(n, Af, ldf, UT);
    count_launch();
    diag_blocks_kernel<<<nblk, 256, 0, st>>>(n, Af, ldf, DL, DU);
    count_launch();
    EGPU_CUDA_TRY(cudaGetLastError());
    TRY(launch_trtri_blocks(st, EGPU_LOWER, 1, DL, 128, n, nb, WinvL, nb));
    TRY(launch_trtri_blocks(st, EGPU_LOWER, 0, DU, 128, n, nb, WinvUT, nb));
    TRY(sweep32_prepare(st, n, Af, ldf, WinvL, swl));
    TRY(sweep32_prepare(st, n, UT, ldf, WinvUT, swu));
  }
  // V := A^-1 V (trans 0) or A^-T V (trans 1) through the factors
  // (lu::SolveAfter, LU/SolveAfter.hpp:101-146): pivots, then the unit-lower
  // and upper sweeps (or their transposes in the opposite order)
  // the row permutation of the pivots and its inverse, composed once
  int* permF = perm;
  int* permI = reinterpret_cast<int*>(ws + L.permi);
  double* ptmp = reinterpret_cast<double*>(perm + ((n + 1) & ~1));
  TRY(launch_compose_perm(st, 0, n, piv, n, permF));
  TRY(launch_compose_perm(st, 1, n, piv, n, permI));
  bool have64 = false;
  int epoch = 0;
  auto materialize64 = [&]() -> int {  // FP64 factors and their block inverses
    if (have64) return EGPU_OK;
    widen_kernel<<<dim3((n + 255) / 256, std::min(n, 65535)), 256, 0, st>>>(n, n, Af, ldf, LU, lds);
    count_launch();
    EGPU_CUDA_TRY(cudaGetLastError());
    if (!use32) TRY(launch_trtri_blocks(st, EGPU_LOWER, 1, LU, lds, n, nb, WinvL, nb));
    TRY(launch_trtri_blocks(st, EGPU_UPPER, 0, LU, lds, n, nb, WinvU, nb));
    EGPU_CUDA_TRY(cudaMemsetAsync(flags, 0, trsm_skinny_flag_bytes(n, nb), st));
    have64 = true;
    return EGPU_OK;
  };
  auto lu_solve64 = [&](double* V, int ncols, int trans) -> int {
    TRY(materialize64());
    if (!trans) {
      TRY(launch_permute_rows(st, n, ncols, permF, V, lds, ptmp));
      TRY(launch_trsm_skinny(st, 0, 0, n, ncols, LU, lds, WinvL, nb, V, lds, flags, ++epoch, h->sm_count,
                             h->dstatus));
      return launch_trsm_skinny(st, 1, 0, n, ncols, LU, lds, WinvU, nb, V, lds, flags, ++epoch, h->sm_count,
                                h->dstatus);
    }
    TRY(launch_trsm_skinny(st, 0, 1, n, ncols, LU, lds, WinvU, nb, V, lds, flags, ++epoch, h->sm_count,
                           h->dstatus));
    TRY(launch_trsm_skinny(st, 1, 1, n, ncols, LU, lds, WinvL, nb, V, lds, flags, ++epoch, h->sm_count,
                           h->dstatus));
    return launch_permute_rows(st, n, ncols, permI, V, lds, ptmp);
  };
  auto lu_solve = [&](double* V, int ncols, int trans) -> int {
    if (!use32) return lu_solve64(V, ncols, trans);
    if (!trans) {  // P^T L U x = v: x = U^-1 L^-1 P v; U x = y is (U^T)^T x = y
      TRY(launch_permute_rows(st, n, ncols, permF, V, lds, ptmp));
      TRY(sweep32_solve(st, 0, n, ncols, Af, ldf, V, lds, swl, h->sm_count, h->dstatus));
      return sweep32_solve(st, 1, n, ncols, UT, ldf, V, lds, swu, h->sm_count, h->dstatus);
    }
    TRY(sweep32_solve(st, 0, n, ncols, UT, ldf, V, lds, swu, h->sm_count, h->dstatus));
    TRY(sweep32_solve(st, 1, n, ncols, Af, ldf, V, lds, swl, h->sm_count, h->dstatus));
    return launch_permute_rows(st, n, ncols, permI, V, lds, ptmp);
  };
  auto residual = [&]() -> int {  // R = B - A Xw
    TRY(launch_copy_cols(st, n, nrhs, B, ldb, R, lds, 0));
    int rg = launch_dgemm_skinny(st, n, nrhs, n, -1.0, A, lda, Xw, lds, R, lds, h->sm_count, h->dstatus);
    if (rg == EGPU_ERR_UNSUPPORTED)
      rg = launch_dgemm(st, false, true, n, nrhs, n, -1.0, A, lda, Xw, lds, 1.0, R, lds, 0, false, h->dstatus);
    return rg;
  };
  // ||A||_inf and ||A||_1
  abs_sums_kernel<<<(32 * n + 255) / 256, 256, 0, st>>>(n, A, lda, norms, norms + n);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  std::vector<double> rs(2 * (size_t)n);
  EGPU_CUDA_TRY(cudaMemcpyAsync(rs.data(), norms, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, st));
  EGPU_CUDA_TRY(cudaStreamSynchronize(st));
  double anorm = 0.0, anorm1 = 0.0;
  for (int i = 0; i < n; ++i) {
    anorm = std::max(anorm, rs[i]);
    anorm1 = std::max(anorm1, rs[n + i]);
  }
  // ---- refinement
  TRY(launch_copy_cols(st, n, nrhs, B, ldb, Xw, lds, 0));
  TRY(lu_solve(Xw, nrhs, 0));
  int it = 0;
  double e = INFINITY, e_prev = INFINITY;
  h->gmres_inner = 0;
  h->mixed_kappa = -1.0;
  bool to_gmres = false, to_fp64 = false;
  h->mixed_mode = 0;
  double* V = reinterpret_cast<double*>(ws + L.gv);
  auto estimate = [&]() -> int {
    const std::function<int(double*, int)> solve = [&](double* v, int trans) -> int { return lu_solve(v, 1, trans); };
    TRY(cond1_estimate(h, n, solve, anorm1, V, &h->mixed_kappa));
    to_gmres = h->mixed_kappa * 5.9604644775390625e-08 > 50.0;
    to_fp64 = h->mixed_kappa * 5.9604644775390625e-08 > 1e3;
    return EGPU_OK;
  };
  if (h->mixed_policy == 1) TRY(estimate());
  for (;;) {
    TRY(residual());
    TRY(mixed_berr(h, n, nrhs, R, Xw, B, ldb, lds, anorm, norms + 2 * n, &e));
    if (e <= tol || it >= max_iter || !std::isfinite(e)) break;
    if (h->mixed_policy == 0 && it == 1 && e > 0.2 * e_prev && h->mixed_kappa < 0) TRY(estimate());
    if (to_gmres) break;
    if (it >= 2 && e > 0.25 * e_prev) break;
    e_prev = e;
    TRY(lu_solve(R, nrhs, 0));
    TRY(launch_copy_cols(st, n, nrhs, R, lds, Xw, lds, 1));
    ++it;
  }
  if (to_fp64) {
    if (iters) *iters = it;
    h->mixed_mode = 2;
    return kFallbackFp64;
  }
  if (e > tol && std::isfinite(e) && it < max_iter) {
    h->mixed_mode = 1;
    GmresWork gw{reinterpret_cast<double*>(ws + L.gv), reinterpret_cast<double*>(ws + L.gw),
                 reinterpret_cast<double*>(ws + L.gc), reinterpret_cast<double*>(ws + L.gc) + nrhs};
    const BlockOp apply_a = [&](const double* Vi, double* Wo) -> int {
      EGPU_CUDA_TRY(cudaMemsetAsync(Wo, 0, sizeof(double) * lds * nrhs, st));
      int rg = launch_dgemm_skinny(st, n, nrhs, n, 1.0, A, lda, Vi, lds, Wo, lds, h->sm_count, h->dstatus);
      if (rg == EGPU_ERR_UNSUPPORTED)
        rg = launch_dgemm(st, false, true, n, nrhs, n, 1.0, A, lda, Vi, lds, 0.0, Wo, lds, 0, false, h->dstatus);
      return rg;
    };
    const BlockSolve precond = [&](double* Wo) -> int { return lu_solve64(Wo, nrhs, 0); };
    int inner = 0;
    double e_best = e;
    while (it < max_iter) {
      TRY(gmres_correction(h, n, nrhs, lds, apply_a, precond, R, R, gw, 1e-10, &inner));
      TRY(launch_copy_cols(st, n, nrhs, R, lds, Xw, lds, 1));
      ++it;
      TRY(residual());
      TRY(mixed_berr(h, n, nrhs, R, Xw, B, ldb, lds, anorm, norms + 2 * n, &e));
      if (e <= tol || !std::isfinite(e) || e > 0.9 * e_best) break;
      e_best = e;
    }
    h->gmres_inner = inner;
    if (e > tol && std::isfinite(e)) {  // GMRES-IR stagnated
      if (iters) *iters = it;
      h->mixed_mode = 2;
      return kFallbackFp64;
    }
  }
  TRY(launch_copy_cols(st, n, nrhs, Xw, lds, X, ldx, 0));
  if (iters) *iters = it;
  if (berr) *berr = e;
  TRY(read_status_now(h, nullptr));
  return e <= tol ? EGPU_OK : EGPU_NO_CONVERGENCE;
}

}  // namespace egpu

using namespace egpu;

extern "C" int egpu_dgesv_mixed(egpu_handle h, int n, int nrhs, const double* dA, int lda, const double* dB, int ldb,
                                double* dX, int ldx, int max_iter, double tol, int* iters, double* berr) {
  if (iters) *iters = 0;
  if (berr) *berr = 0.0;
  if (!h) return EGPU_ERR_ARG;
  if (n < 0 || nrhs < 0 || nrhs > 64 || lda < std::max(1, n) || ldb < std::max(1, n) || ldx < std::max(1, n) ||
      max_iter < 0)
    return EGPU_ERR_ARG;
  if (n == 0 || nrhs == 0) return EGPU_OK;
  Enter en(h);
  const int rc = dgesv_mixed_core(h, n, nrhs, dA, lda, dB, ldb, dX, ldx, max_iter, tol, iters, berr);
  if (rc != kFallbackFp64) return rc;
  return dgesv_fp64_refined(h, n, nrhs, dA, lda, dB, ldb, dX, ldx, max_iter, tol, iters, berr);
}
