// Mixed-precision HPD solve: Cholesky with the trailing updates on the
// tcgen05 tensor cores (TF32 x 3 split products, FP32 accumulation, FP32
// trailing matrix), the diagonal blocks and panel solves in FP64, and
// iterative refinement with FP64 residuals to an FP64-level backward error.
//
// Per block column k (nb = the handle's block size):
//   1. the panel columns [k, k+b) of the FP32 working matrix are widened into
//      the FP64 factor buffer Lf;
//   2. potrf of the b x b diagonal block and its inverse (FP64, the same
//      kernel as the plain path: cholesky::LVar3Unb, Cholesky/LVar3.hpp:19-49);
//   3. L21 := A21 inv(L11)^T (FP64 DMMA GEMM);
//   4. L21 is split into TF32 hi/lo parts in K-major layout;
//   5. A22 -= L21 L21^T on the lower triangle of the FP32 matrix with
//      tcgen05.mma kind::tf32 (hi*hi + hi*lo + lo*hi).
// The factor Lf (FP64 storage, FP32-level accuracy) then drives the
// refinement: x = Lf^-T Lf^-1 b, and while the normwise backward error
//   max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf)
// is above the tolerance: r = b - A x (FP64 GEMM on a full symmetric copy of
// A), d = Lf^-T Lf^-1 r, x += d.
#include <cmath>
#include <functional>
#include <vector>

#include "context.h"

namespace egpu {

namespace {

// A (uplo triangle valid) -> As (full symmetric FP64, ld lds) and Af (lower FP32, ld ldf)
__global__ void mixed_prepare_kernel(int uplo, int n, const double* A, long long lda, double* As, long long lds,
                                     float* Af, long long ldf) {
  __shared__ double tile[32][33];
  const int bi = blockIdx.x * 32, bj = blockIdx.y * 32;  // tile rows bi.., cols bj..
  if (bi < bj) return;                                  // lower tiles (and their mirrors) only
  const int tx = threadIdx.x, ty = threadIdx.y;         // 32 x 8
  for (int q = ty; q < 32; q += 8) {
    const int r = bi + tx, c = bj + q;
    double v = 0.0;
    if (r < n && c < n && r >= c) v = (uplo == EGPU_LOWER) ? A[r + (long long)c * lda] : A[c + (long long)r * lda];
    tile[tx][q] = v;
    if (r < n && c < n && r >= c) {
      As[r + (long long)c * lds] = v;
      Af[r + (long long)c * ldf] = (float)v;
    }
  }
  __syncthreads();
  for (int q = ty; q < 32; q += 8) {  // mirror: As[c, r] = A(r, c) for r > c
    const int c = bj + tx, r = bi + q;
    if (r < n && c < n && r > c) As[c + (long long)r * lds] = tile[q][tx];
  }
}

// Lf[i, c] = Af[i, c] for the whole m x b block (a panel's L21)
__global__ void widen_panel_kernel(int m, int b, const float* Af, long long ldf, double* Lf, long long ldl) {
  const int c = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    Lf[i + (long long)c * ldl] = (double)Af[i + (long long)c * ldf];
}


// X (rows x cols, column-major FP64 or FP32) -> hi/lo TF32 in K-major rows:
// hi[r*ldk + c] for c < width (zero for c >= cols)
template <typename T>
__global__ void split_tf32_kernel(int rows, int cols, const T* X, long long ldx, float* hi, float* lo,
                                  long long ldk, int width) {
  __shared__ double tile[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int q = ty; q < 32; q += 8) {
    const int r = r0 + tx, c = c0 + q;
    tile[q][tx] = (r < rows && c < cols) ? (double)X[r + (long long)c * ldx] : 0.0;
  }
  __syncthreads();
  for (int q = ty; q < 32; q += 8) {
    const int r = r0 + q, c = c0 + tx;
    if (r < rows && c < width) {
      const double x = (c < cols) ? tile[tx][q] : 0.0;
      const float h = tf32_rna((float)x);
      hi[(long long)r * ldk + c] = h;
      lo[(long long)r * ldk + c] = tf32_rna((float)(x - (double)h));
    }
  }
}

// per-column max |X[:, j]| into out[j] (one block per column)
__global__ void colmax_kernel(int n, int ncols, const double* X, long long ldx, double* out) {
  const int j = blockIdx.x;
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(X[i + (long long)j * ldx]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) out[j] = m;
  }
}

// ||As||_inf = max_i sum_j |As[i, j]| : per-row sums, one thread per row
// rows[j] = sum_i |As[i, j]|: the row sums of the symmetric As, as column
// sums (a warp per column, contiguous loads, fixed summation order)
__global__ void rowsum_abs_kernel(int n, const double* As, long long lds, double* rows) {
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (j >= n) return;
  const double* col = As + (long long)j * lds;
  double s = 0.0;
  for (int i = lane; i < n; i += 32) s += fabs(col[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) rows[j] = s;
}

// Y = X (n x ncols) ; Y += X
__global__ void copy_cols_kernel(int n, int ncols, const double* X, long long ldx, double* Y, long long ldy,
                                 int add) {
  for (int j = blockIdx.y; j < ncols; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      const double x = X[i + (long long)j * ldx];
      double* y = &Y[i + (long long)j * ldy];
      *y = add ? *y + x : x;
    }
}

// out[j * nrhs + c] = sum_i V_j[i, c] W[i, c] for j < nv (V_j = V + j * vstride); one block per (j, c)
__global__ void block_dots_kernel(int n, const double* V, long long ldv, long long vstride, const double* W,
                                  long long ldw, double* out, int nrhs) {
  const int j = blockIdx.x, c = blockIdx.y;
  const double* v = V + j * vstride + (long long)c * ldv;
  const double* w = W + (long long)c * ldw;
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s = fma(v[i], w[i], s);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[j * nrhs + c] = s;
  }
}

// W[:, c] -= sum_{j < nv} coef[j * nrhs + c] V_j[:, c]
__global__ void block_axpy_kernel(int n, int nv, const double* V, long long ldv, long long vstride,
                                  const double* coef, double* W, long long ldw, int nrhs) {
  const int c = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int j = 0; j < nv; ++j) acc = fma(coef[j * nrhs + c], V[j * vstride + (long long)c * ldv + i], acc);
    W[(long long)c * ldw + i] -= acc;
  }
}

// Y[:, c] = s[c] X[:, c]
__global__ void col_scale_kernel(int n, const double* X, long long ldx, const double* s, double* Y, long long ldy) {
  const int c = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    Y[(long long)c * ldy + i] = s[c] * X[(long long)c * ldx + i];
}

}  // namespace

int launch_copy_cols(cudaStream_t st, int n, int ncols, const double* X, long long ldx, double* Y, long long ldy,
                     int add) {
  if (n <= 0 || ncols <= 0) return EGPU_OK;
  copy_cols_kernel<<<dim3((n + 255) / 256, std::min(ncols, 65535)), 256, 0, st>>>(n, ncols, X, ldx, Y, ldy, add);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  return EGPU_OK;
}

int launch_split_tf32(cudaStream_t st, int rows, int cols, const double* X, long long ldx, float* hi, float* lo,
                      long long ldk, int width) {
  if (rows <= 0 || cols <= 0) return EGPU_OK;
  if (width < 0) width = (int)ldk;
  TraceMark tm(st, kTraceOther, 0.0, (double)rows * (8.0 * cols + 8.0 * width));
  dim3 grid((rows + 31) / 32, (width + 31) / 32), block(32, 8);
  split_tf32_kernel<double><<<grid, block, 0, st>>>(rows, cols, X, ldx, hi, lo, ldk, width);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  return EGPU_OK;
}

int launch_split_tf32_f32(cudaStream_t st, int rows, int cols, const float* X, long long ldx, float* hi, float* lo,
                          long long ldk) {
  if (rows <= 0 || cols <= 0) return EGPU_OK;
  TraceMark tm(st, kTraceOther, 0.0, (double)rows * (4.0 * cols + 8.0 * ldk));
  dim3 grid((rows + 31) / 32, (int)((ldk + 31) / 32)), block(32, 8);
  split_tf32_kernel<float><<<grid, block, 0, st>>>(rows, cols, X, ldx, hi, lo, ldk, (int)ldk);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  return EGPU_OK;
}


// Workspace layout of the mixed solve.
struct MixedLayout {
  size_t as, af, lf, pkh, pkl, wsh, wsl, xw, r, yt, winv, norms, flags, gv, gw, gc, sw, total;
  long long lds, ldf, ldk;
};

static MixedLayout mixed_layout(int n, int nrhs, int nb) {
  MixedLayout L;
  L.lds = std::max<long long>(32, ((long long)n + 31) / 32 * 32);
  L.ldf = L.lds;
  L.ldk = ((long long)nb + 31) / 32 * 32;
  size_t off = 0;
  auto take = [&](size_t bytes) { off = (off + 1023) & ~size_t(1023); size_t o = off; off += bytes; return o; };
  L.as = take(sizeof(double) * L.lds * n);
  L.af = take(sizeof(float) * L.ldf * n);
  L.lf = take(sizeof(double) * L.lds * n);
  L.pkh = take(2 * sizeof(float) * (size_t)n * L.ldk);  // two buffers (look-ahead)
  L.pkl = take(2 * sizeof(float) * (size_t)n * L.ldk);
  L.wsh = take(sizeof(float) * 128 * (size_t)L.ldk);  // TF32 split of the current diagonal inverse
  L.wsl = take(sizeof(float) * 128 * (size_t)L.ldk);
  L.xw = take(sizeof(double) * L.lds * std::max(nrhs, 1));
  L.r = take(sizeof(double) * L.lds * std::max(nrhs, 1));
  L.yt = take(sizeof(double) * L.lds * std::max(nrhs, 1));
  L.winv = take(winv_bytes(n, nb));
  L.norms = take(sizeof(double) * ((size_t)n + 4 * (size_t)std::max(nrhs, 1)));
  L.flags = take(trsm_skinny_flag_bytes(n, nb));
  L.gv = take(sizeof(double) * L.lds * std::max(nrhs, 1) * (kGmresRestart + 1));  // GMRES basis
  L.gw = take(sizeof(double) * L.lds * std::max(nrhs, 1));                        // GMRES work vector
  L.gc = take(sizeof(double) * (size_t)std::max(nrhs, 1) * (kGmresRestart + 2));  // coefficients
  L.sw = take(sweep32_ws_bytes(n, nrhs));  // FP32 sweeps: super-block inverses, work vectors
  L.total = (off + 4095) & ~size_t(4095);
  return L;
}

// X := Lf^-T Lf^-1 X.  Prescaled (nrhs <= 64): the off-diagonal blocks of Lf
// hold M2 = L D^-1 (D the diagonal blocks, W their inverses), and the two
// cooperative sweeps are the column-prescaled forward sweep over M2 (z in X,
// Y := W z) and the row-prescaled backward sweep over M2^T (Y in, X out).
// Otherwise Lf holds L and the blocked multiply-by-inverse form runs.
struct SweepFlags {
  int* flags;
  int epoch;
  bool prescaled;
  double* Y;
  const float* Lf32;  // non-null: the FP32 super-block sweeps over this factor
  long long ldf;
  void* sw;           // their workspace (super-block inverses prepared)
};
static int mixed_solve(egpu_context* h, int n, int nrhs, const double* Lf, long long lds, const double* Winv,
                       double* X, SweepFlags& fl) {
  if (fl.Lf32) return sweep32_solve(h->stream, 2, n, nrhs, fl.Lf32, fl.ldf, X, lds, fl.sw, h->sm_count, h->dstatus);
  if (fl.prescaled) {
    TRY(launch_trsm_skinny(h->stream, 0, 0, n, nrhs, Lf, lds, Winv, h->nb, X, lds, fl.flags, ++fl.epoch,
                           h->sm_count, h->dstatus, fl.Y));
    return launch_trsm_skinny(h->stream, 1, 1, n, nrhs, Lf, lds, Winv, h->nb, X, lds, fl.flags, ++fl.epoch,
                              h->sm_count, h->dstatus, fl.Y, true);
  }
  TRY(trsm_blocked(h->stream, EGPU_LEFT, EGPU_LOWER, 0, n, nrhs, Lf, lds, Winv, h->nb, X, lds, h->dstatus));
  return trsm_blocked(h->stream, EGPU_LEFT, EGPU_LOWER, 1, n, nrhs, Lf, lds, Winv, h->nb, X, lds, h->dstatus);
}

// M2 for block column j0 in place: Lf(r, j) := L(r, j) W_j below the
// diagonal block (the 128-wide tile keeps each row panel in one CTA).  The
// panel's TF32 split was taken from L before this runs.
static int mixed_prescale_step(egpu_context* h, cudaStream_t st, int n, int j0, double* Lf, long long lds,
                               const double* Winv) {
  const int nb = h->nb;
  const int bj = std::min(nb, n - j0);
  const double* Wj = Winv + (size_t)(j0 / nb) * nb * nb;
  const int below = n - j0 - bj;
  if (below > 0) {
    double* P = Lf + (j0 + bj) + (long long)j0 * lds;
    TRY(launch_dgemm(st, false, true, below, bj, bj, 1.0, P, lds, Wj, nb, 0.0, P, lds, 0, true, h->dstatus));
  }
  return EGPU_OK;
}

// Backward error of the current iterate: max_j ||r_j|| / (||A|| ||x_j|| + ||b_j||), inf-norms.
int mixed_berr(egpu_context* h, int n, int nrhs, const double* R, const double* Xw, const double* B,
                      long long ldb, long long lds, double anorm, double* norms, double* berr) {
  cudaStream_t st = h->stream;
  colmax_kernel<<<nrhs, 256, 0, st>>>(n, nrhs, R, lds, norms);
  colmax_kernel<<<nrhs, 256, 0, st>>>(n, nrhs, Xw, lds, norms + nrhs);
  colmax_kernel<<<nrhs, 256, 0, st>>>(n, nrhs, B, ldb, norms + 2 * nrhs);
  count_launch(3);
  EGPU_CUDA_TRY(cudaGetLastError());
  std::vector<double> hn(3 * (size_t)nrhs);
  EGPU_CUDA_TRY(cudaMemcpyAsync(hn.data(), norms, sizeof(double) * 3 * nrhs, cudaMemcpyDeviceToHost, st));
  EGPU_CUDA_TRY(cudaStreamSynchronize(st));
  double e = 0.0;
  for (int j = 0; j < nrhs; ++j) {
    const double den = anorm * hn[nrhs + j] + hn[2 * nrhs + j];
    e = std::max(e, den > 0.0 ? hn[j] / den : (hn[j] > 0.0 ? INFINITY : 0.0));
  }
  *berr = e;
  return EGPU_OK;
}

// GMRES-IR correction: solve A d = r with GMRES left-preconditioned by the
// low-precision factor (M = Lf Lf^T applied by mixed_solve), FP64 everywhere
// else, one Krylov basis per right-hand side advanced in lockstep; classical
// Gram-Schmidt applied twice, Givens rotations on the host.  Stops when every
// column's preconditioned residual fell below inner_tol times its start, or
// after kGmresRestart vectors.  R is consumed; D receives the correction.
int gmres_correction(egpu_context* h, int n, int nrhs, long long lds, const BlockOp& apply_a,
                     const BlockSolve& precond, double* R, double* D, GmresWork& gw, double inner_tol,
                     int* inner_iters) {
  cudaStream_t st = h->stream;
  const long long vs = lds * nrhs;  // stride between basis blocks
  const int m = kGmresRestart;
  dim3 vgrid((n + 255) / 256, nrhs);
  auto dots = [&](int nv, const double* W, std::vector<double>& out) -> int {  // out[j*nrhs+c] = <V_j, W>
    block_dots_kernel<<<dim3(nv, nrhs), 256, 0, st>>>(n, gw.V, lds, vs, W, lds, gw.dots, nrhs);
    count_launch();
    EGPU_CUDA_TRY(cudaGetLastError());
    out.resize((size_t)nv * nrhs);
    EGPU_CUDA_TRY(cudaMemcpyAsync(out.data(), gw.dots, sizeof(double) * nv * nrhs, cudaMemcpyDeviceToHost, st));
    EGPU_CUDA_TRY(cudaStreamSynchronize(st));
    return EGPU_OK;
  };
  auto self_norms = [&](const double* W, std::vector<double>& out) -> int {  // ||W[:, c]||
    block_dots_kernel<<<dim3(1, nrhs), 256, 0, st>>>(n, W, lds, 0, W, lds, gw.dots, nrhs);
    count_launch();
    EGPU_CUDA_TRY(cudaGetLastError());
    out.resize(nrhs);
    EGPU_CUDA_TRY(cudaMemcpyAsync(out.data(), gw.dots, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st));
    EGPU_CUDA_TRY(cudaStreamSynchronize(st));
    for (double& v : out) v = std::sqrt(std::max(v, 0.0));
    return EGPU_OK;
  };
  auto scale_into = [&](const double* X, const std::vector<double>& s, double* Y) -> int {
    EGPU_CUDA_TRY(cudaMemcpyAsync(gw.coef, s.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, st));
    col_scale_kernel<<<vgrid, 256, 0, st>>>(n, X, lds, gw.coef, Y, lds);
    count_launch();
    EGPU_CUDA_TRY(cudaGetLastError());
    return EGPU_OK;
  };
  auto axpy = [&](int nv, const std::vector<double>& c, double* W) -> int {  // W -= sum_j c_j V_j
    EGPU_CUDA_TRY(cudaMemcpyAsync(gw.coef, c.data(), sizeof(double) * nv * nrhs, cudaMemcpyHostToDevice, st));
    block_axpy_kernel<<<vgrid, 256, 0, st>>>(n, nv, gw.V, lds, vs, gw.coef, W, lds, nrhs);
    count_launch();
    EGPU_CUDA_TRY(cudaGetLastError());
    return EGPU_OK;
  };
  // z = M^-1 r, beta = ||z||, V_0 = z / beta
  TRY(precond(R));
  std::vector<double> beta, inv(nrhs), hv, nrm;
  TRY(self_norms(R, beta));
  for (int c = 0; c < nrhs; ++c) inv[c] = beta[c] > 0.0 ? 1.0 / beta[c] : 0.0;
  TRY(scale_into(R, inv, gw.V));
  // per column: Hessenberg (column-major (m+1) x m), rotations, rhs g
  std::vector<double> H((size_t)nrhs * (m + 1) * m, 0.0), cs((size_t)nrhs * m), sn((size_t)nrhs * m),
      g((size_t)nrhs * (m + 1), 0.0);
  auto Hc = [&](int c, int i, int j) -> double& { return H[((size_t)c * m + j) * (m + 1) + i]; };
  for (int c = 0; c < nrhs; ++c) g[(size_t)c * (m + 1)] = beta[c];
  int k = 0;
  for (int i = 0; i < m; ++i) {
    double* Vi = gw.V + i * vs;
    // W = M^-1 A V_i
    TRY(apply_a(Vi, gw.W));
    TRY(precond(gw.W));
    for (int pass = 0; pass < 2; ++pass) {  // classical Gram-Schmidt, twice
      TRY(dots(i + 1, gw.W, hv));
      TRY(axpy(i + 1, hv, gw.W));
      for (int c = 0; c < nrhs; ++c)
        for (int j = 0; j <= i; ++j) Hc(c, j, i) += hv[(size_t)j * nrhs + c];
    }
    TRY(self_norms(gw.W, nrm));
    for (int c = 0; c < nrhs; ++c) {
      Hc(c, i + 1, i) = nrm[c];
      inv[c] = nrm[c] > 0.0 ? 1.0 / nrm[c] : 0.0;
    }
    TRY(scale_into(gw.W, inv, gw.V + (i + 1) * vs));
    bool done = true;
    for (int c = 0; c < nrhs; ++c) {
      double* cc = &cs[(size_t)c * m];
      double* ss = &sn[(size_t)c * m];
      double* gg = &g[(size_t)c * (m + 1)];
      for (int j = 0; j < i; ++j) {  // earlier rotations on the new column
        const double a = Hc(c, j, i), b = Hc(c, j + 1, i);
        Hc(c, j, i) = cc[j] * a + ss[j] * b;
        Hc(c, j + 1, i) = -ss[j] * a + cc[j] * b;
      }
      const double a = Hc(c, i, i), b = Hc(c, i + 1, i);
      const double rr = std::hypot(a, b);
      cc[i] = rr > 0.0 ? a / rr : 1.0;
      ss[i] = rr > 0.0 ? b / rr : 0.0;
      Hc(c, i, i) = rr;
      Hc(c, i + 1, i) = 0.0;
      gg[i + 1] = -ss[i] * gg[i];
      gg[i] = cc[i] * gg[i];
      if (beta[c] > 0.0 && std::fabs(gg[i + 1]) > inner_tol * beta[c]) done = false;
    }
    k = i + 1;
    if (done) break;
  }
  // y = H(0:k, 0:k)^-1 g(0:k) per column; D = sum_j y_j V_j
  std::vector<double> y((size_t)k * nrhs, 0.0);
  for (int c = 0; c < nrhs; ++c) {
    const double* gg = &g[(size_t)c * (m + 1)];
    for (int j = k - 1; j >= 0; --j) {
      double s = gg[j];
      for (int l = j + 1; l < k; ++l) s -= Hc(c, j, l) * y[(size_t)l * nrhs + c];
      const double d = Hc(c, j, j);
      y[(size_t)j * nrhs + c] = d != 0.0 ? s / d : 0.0;
    }
  }
  for (double& v : y) v = -v;  // axpy subtracts
  EGPU_CUDA_TRY(cudaMemsetAsync(D, 0, sizeof(double) * vs, st));
  TRY(axpy(k, y, D));
  if (inner_iters) *inner_iters += k;
  return EGPU_OK;
}

// 1-norm condition estimate of A from its low-precision factor: kappa_1 =
// ||A||_1 ||A^-1||_1 with ||A^-1||_1 estimated by Hager's method (W. W.
// Hager, "Condition estimates", SIAM J. Sci. Stat. Comput. 5, 1984, as
// refined by N. J. Higham, ACM TOMS 14, 1988: the algorithm of LAPACK's
// dlacon), with A^-1 and A^-T applied as the factor's solves.  At most 5 iterations of two solves each, plus the closing test with
// the alternating vector; the small vector logic runs on the host.  V: two
// work columns of ld lds on the device.
// solve(V, trans): V := A^-1 V (trans 0) or A^-T V (trans 1), one column.
int cond1_estimate(egpu_context* h, int n, const std::function<int(double*, int)>& solve, double anorm, double* V,
                   double* kappa) {
  cudaStream_t st = h->stream;
  std::vector<double> x(n), y(n), z(n), xi(n), xi_old(n, 0.0);
  auto apply = [&](std::vector<double>& v, int trans) -> int {
    EGPU_CUDA_TRY(cudaMemcpyAsync(V, v.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
    TRY(solve(V, trans));
    EGPU_CUDA_TRY(cudaMemcpyAsync(v.data(), V, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    EGPU_CUDA_TRY(cudaStreamSynchronize(st));
    return EGPU_OK;
  };
  auto norm1 = [&](const std::vector<double>& v) {
    double t = 0.0;
    for (double a : v) t += std::fabs(a);
    return t;
  };
  for (int i = 0; i < n; ++i) x[i] = 1.0 / n;
  double est = 0.0;
  for (int k = 1; k <= 5; ++k) {
    y = x;
    TRY(apply(y, 0));
    const double ny = norm1(y);
    if (k > 1 && ny <= est) break;  // no increase
    est = ny;
    bool same = k > 1;
    for (int i = 0; i < n; ++i) {
      xi[i] = y[i] >= 0.0 ? 1.0 : -1.0;
      same = same && xi[i] == xi_old[i];
    }
    if (same) break;  // the sign pattern repeats: converged
    z = xi;
    TRY(apply(z, 1));
    int j = 0;
    double zx = 0.0;
    for (int i = 0; i < n; ++i) {
      if (std::fabs(z[i]) > std::fabs(z[j])) j = i;
      zx += z[i] * x[i];
    }
    if (k > 1 && std::fabs(z[j]) <= zx) break;  // no better column
    std::fill(x.begin(), x.end(), 0.0);
    x[j] = 1.0;
    xi_old = xi;
  }
  // the alternating test vector guards against the method's known failures
  for (int i = 0; i < n; ++i) x[i] = (i % 2 ? -1.0 : 1.0) * (1.0 + (n > 1 ? (double)i / (n - 1) : 0.0));
  TRY(apply(x, 0));
  est = std::max(est, 2.0 * norm1(x) / (3.0 * n));
  *kappa = anorm * est;
  return EGPU_OK;
}

// Refinement mode from a 1-norm condition estimate and the low-precision
// factor's unit roundoff u (2^-24 for the FP32-accurate factor): plain
// refinement contracts while kappa_1 u stays below kGmresAbove (kappa_1
// overestimates the 2-norm condition that governs the contraction, by up to
// ~sqrt(n) on the matrices measured), GMRES-IR preconditioned by the same
// factor beyond that.
constexpr double kFactorU = 5.9604644775390625e-08;
constexpr double kGmresAbove = 50.0;

int dposv_mixed_core_impl(egpu_context* h, int uplo, int n, int nrhs, const double* A, long long lda, const double* B,
                     long long ldb, double* X, long long ldx, int max_iter, double tol, int* iters, double* berr) {
  const int nb = h->nb;
  cudaStream_t st = h->stream;
  const MixedLayout L = mixed_layout(n, nrhs, nb);
  h->gmres_inner = 0;
  h->mixed_mode = 0;
  TRY(ensure_ws(h, L.total + 4096));
  unsigned char* ws = static_cast<unsigned char*>(h->ws);
  double* As = reinterpret_cast<double*>(ws + L.as);
  float* Af = reinterpret_cast<float*>(ws + L.af);
  double* Lf = reinterpret_cast<double*>(ws + L.lf);
  float* PKh = reinterpret_cast<float*>(ws + L.pkh);
  float* PKl = reinterpret_cast<float*>(ws + L.pkl);
  float* Wsh = reinterpret_cast<float*>(ws + L.wsh);
  float* Wsl = reinterpret_cast<float*>(ws + L.wsl);
  double* Xw = reinterpret_cast<double*>(ws + L.xw);
  double* R = reinterpret_cast<double*>(ws + L.r);
  double* Winv = reinterpret_cast<double*>(ws + L.winv);
  double* norms = reinterpret_cast<double*>(ws + L.norms);
  // prescaled sweeps where the one-launch sweep kernel takes the shape
  const bool prescale = nrhs <= 64 && nb >= 8 && nb <= 128 && nb % 2 == 0;
  SweepFlags fl{reinterpret_cast<int*>(ws + L.flags), 0, prescale, reinterpret_cast<double*>(ws + L.yt), nullptr,
                0, ws + L.sw};
  // the FP32 super-block sweeps take the corrections when the panels are 128
  // wide and the FP32 factor is TMA-addressable; the FP64 copy of L (and its
  // prescaled M2 form) is then only built if GMRES-IR needs it
  const bool use32 = nb == 128 && nrhs <= 32 && L.ldf % 4 == 0;
  bool have_lf = false;  // Lf holds the FP64 copy (prescaled when `prescale`)
  EGPU_CUDA_TRY(cudaMemsetAsync(fl.flags, 0, trsm_skinny_flag_bytes(n, nb), st));
  const long long lds = L.lds, ldf = L.ldf;
  // The factorization: the fast form computes every panel's L21 on the
  // tensor cores (TF32 x 3); `accurate` keeps L21 in FP64 (DMMA), a second
  // attempt for matrices whose fast factorization meets a non-positive pivot.
  auto factor = [&](bool accurate) -> int {
    EGPU_CUDA_TRY(cudaMemsetAsync(h->dstatus, 0, sizeof(DevStatus), st));
    {
      dim3 grid((n + 31) / 32, (n + 31) / 32), block(32, 8);
      mixed_prepare_kernel<<<grid, block, 0, st>>>(uplo, n, A, lda, As, lds, Af, ldf);
      count_launch();
      EGPU_CUDA_TRY(cudaGetLastError());
    }
    // ---- factorization, look-ahead depth 1: the panel chain of step k+1
    // (diagonal block, L21, split) runs on the high-priority side stream
    // as soon as the main stream has updated block column k+1; the rest of
    // step k's trailing update follows on the main stream.  The split panel is
    // double-buffered (step parity).
    float* PKh2[2] = {PKh, PKh + (size_t)n * L.ldk};
    float* PKl2[2] = {PKl, PKl + (size_t)n * L.ldk};
    cudaStream_t sd = h->side;
    // The panel chain, all on the TF32 x 3 tensor-core path except the
    // diagonal block: the FP32 diagonal block is factored and inverted in FP64
    // (inverse kept for the solves, its TF32 split for the next product), then
    // L21 = A21 inv(L11)^T on the tensor cores, in place in the FP32 panel, and
    // its TF32 split for the trailing updates.
    auto panel_chain = [&](int k, cudaStream_t s) -> int {
      const int b = std::min(nb, n - k);
      const int m2 = n - k - b;
      const int par = (k / nb) & 1;
      double* Wk = Winv + (size_t)(k / nb) * nb * nb;
      TRY(launch_potrf_diag_f32(s, Af + k + (long long)k * ldf, ldf, b, Wk, nb, Wsh, Wsl, L.ldk, h->dstatus, k));
      if (m2 == 0) return EGPU_OK;
      float* A21 = Af + (k + b) + (long long)k * ldf;
      if (accurate) {  // L21 = A21 inv(L11)^T in FP64 (DMMA) from the widened panel
        double* L21 = Lf + (k + b) + (long long)k * lds;
        dim3 grid((m2 + 255) / 256, b);
        widen_panel_kernel<<<grid, 256, 0, s>>>(m2, b, A21, ldf, L21, lds);
        count_launch();
        EGPU_CUDA_TRY(cudaGetLastError());
        TRY(launch_dgemm(s, false, false, m2, b, b, 1.0, L21, lds, Wk, nb, 0.0, L21, lds, 0, true, h->dstatus));
        TRY(launch_split_tf32(s, m2, b, L21, lds, PKh2[par], PKl2[par], L.ldk));
      } else {
        // A21's split: from the previous step's block-column update (its
        // epilogue), or here for the first panel; L21's split is written by the
        // product's epilogue over it (a tile's output rows are the rows it read)
        if (k == 0) TRY(launch_split_tf32_f32(s, m2, b, A21, ldf, PKh2[par], PKl2[par], L.ldk));
        else EGPU_CUDA_TRY(cudaStreamWaitEvent(s, h->ev_a21[par], 0));
        TRY(launch_tc_gemm(s, m2, b, b, 1.0f, PKh2[par], PKl2[par], Wsh, Wsl, L.ldk, 0.0f, A21, ldf, 0, 3,
                           h->dstatus, PKh2[par], PKl2[par], L.ldk, 0, (int)L.ldk));
      }
      EGPU_CUDA_TRY(cudaEventRecord(h->ev_split[par], s));  // L21 final: its FP64 copy may start
      return EGPU_OK;
    };
    // Off the chain, on the lowest-priority stream: the FP64 copy of panel k's
    // L21 for the solves, and M2 in place over it when prescaled
    auto l21_copy = [&](int k, int par) -> int {
      const int b = std::min(nb, n - k), m2 = n - k - b;
      if (m2 <= 0) return EGPU_OK;
      EGPU_CUDA_TRY(cudaStreamWaitEvent(h->aux, h->ev_split[par], 0));
      if (!accurate) {  // the FP32 panel holds L21
        TraceMark tm(h->aux, kTraceOther, 0.0, 12.0 * m2 * b);
        dim3 grid((m2 + 255) / 256, b);
        widen_panel_kernel<<<grid, 256, 0, h->aux>>>(m2, b, Af + (k + b) + (long long)k * ldf, ldf,
                                                     Lf + (k + b) + (long long)k * lds, lds);
        count_launch();
        EGPU_CUDA_TRY(cudaGetLastError());
      }
      if (prescale) TRY(mixed_prescale_step(h, h->aux, n, k, Lf, lds, Winv));
      return EGPU_OK;
    };
    EGPU_CUDA_TRY(cudaEventRecord(h->ev_fork, st));
    EGPU_CUDA_TRY(cudaStreamWaitEvent(sd, h->ev_fork, 0));
    TRY(panel_chain(0, sd));
    for (int k = 0; k < n; k += nb) {
      const int b = std::min(nb, n - k);
      const int m2 = n - k - b;
      const int par = (k / nb) & 1;
      EGPU_CUDA_TRY(cudaEventRecord(h->ev_panel[par], sd));
      if (m2 == 0) break;
      EGPU_CUDA_TRY(cudaStreamWaitEvent(st, h->ev_panel[par], 0));
      const int b2 = std::min(nb, m2);
      float* A22 = Af + (k + b) + (long long)(k + b) * ldf;
      // (a) block column k+1: its diagonal block first (releases the next
      // diagonal factorization), then the rows below it, which are the next
      // panel's A21 (split into the other buffer; its L21 product waits for it)
      TRY(launch_tc_gemm(st, b2, b2, b, -1.0f, PKh2[par], PKl2[par], PKh2[par], PKl2[par], L.ldk, 1.0f, A22, ldf, 1,
                         3, h->dstatus));
      EGPU_CUDA_TRY(cudaEventRecord(h->ev_rest[par], st));
      EGPU_CUDA_TRY(cudaStreamWaitEvent(sd, h->ev_rest[par], 0));
      if (m2 > b2) {
        TRY(launch_tc_gemm(st, m2 - b2, b2, b, -1.0f, PKh2[par] + (size_t)b2 * L.ldk, PKl2[par] + (size_t)b2 * L.ldk,
                           PKh2[par], PKl2[par], L.ldk, 1.0f, A22 + b2, ldf, 0, 3, h->dstatus, PKh2[par ^ 1],
                           PKl2[par ^ 1], L.ldk, 0, (int)L.ldk));
        EGPU_CUDA_TRY(cudaEventRecord(h->ev_a21[par ^ 1], st));
      }
      TRY(panel_chain(k + b, sd));
      // (b) the rest of the trailing lower triangle
      const int m3 = m2 - b2;
      if (m3 > 0)
        TRY(launch_tc_gemm(st, m3, m3, b, -1.0f, PKh2[par] + (size_t)b2 * L.ldk, PKl2[par] + (size_t)b2 * L.ldk,
                           PKh2[par] + (size_t)b2 * L.ldk, PKl2[par] + (size_t)b2 * L.ldk, L.ldk, 1.0f,
                           A22 + b2 + (long long)b2 * ldf, ldf, 1, 3, h->dstatus));
      if (accurate || !use32) TRY(l21_copy(k, par));
    }
    EGPU_CUDA_TRY(cudaEventRecord(h->ev_join, sd));
    EGPU_CUDA_TRY(cudaStreamWaitEvent(st, h->ev_join, 0));
    EGPU_CUDA_TRY(cudaEventRecord(h->ev_aux, h->aux));
    EGPU_CUDA_TRY(cudaStreamWaitEvent(st, h->ev_aux, 0));

    return read_status_now(h, nullptr);
  };
  bool accurate = false;
  int frc = factor(false);
  if (frc == EGPU_NOT_HPD) {
    accurate = true;
    frc = factor(true);
  }
  TRY(frc);  // the status word (pivot column) stays readable by the caller
  if (use32 && !accurate) {  // L in the FP32 working matrix: super-block inverses
    TRY(sweep32_prepare(st, n, Af, ldf, Winv, fl.sw));
    fl.Lf32 = Af;
    fl.ldf = ldf;
  } else {
    have_lf = true;
  }
  // The FP64 copy of L (M2 when prescaled) on demand, for GMRES-IR: widen the
  // FP32 factor's panels and prescale them (the same work the factorization
  // does on its auxiliary stream when the FP32 sweeps are not used).
  auto materialize_lf = [&]() -> int {
    if (have_lf) return EGPU_OK;
    for (int k = 0; k + nb < n; k += nb) {
      const int b = std::min(nb, n - k), m2 = n - k - b;
      TraceMark tm(st, kTraceOther, 0.0, 12.0 * m2 * b);
      dim3 grid((m2 + 255) / 256, b);
      widen_panel_kernel<<<grid, 256, 0, st>>>(m2, b, Af + (k + b) + (long long)k * ldf, ldf,
                                               Lf + (k + b) + (long long)k * lds, lds);
      count_launch();
      EGPU_CUDA_TRY(cudaGetLastError());
      if (prescale) TRY(mixed_prescale_step(h, st, n, k, Lf, lds, Winv));
    }
    have_lf = true;
    fl.Lf32 = nullptr;
    return EGPU_OK;
  };
  // ---- refinement
  {
    rowsum_abs_kernel<<<(n + 7) / 8, 256, 0, st>>>(n, As, lds, norms);
    count_launch();
    EGPU_CUDA_TRY(cudaGetLastError());
  }
  std::vector<double> rs(n);
  EGPU_CUDA_TRY(cudaMemcpyAsync(rs.data(), norms, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  EGPU_CUDA_TRY(cudaStreamSynchronize(st));
  double anorm = 0.0;
  for (double v : rs) anorm = std::max(anorm, v);
  dim3 cgrid((n + 255) / 256, nrhs);
  copy_cols_kernel<<<cgrid, 256, 0, st>>>(n, nrhs, B, ldb, Xw, lds, 0);
  count_launch();
  TRY(mixed_solve(h, n, nrhs, Lf, lds, Winv, Xw, fl));
  int it = 0;
  double e = INFINITY, e_prev = INFINITY;
  h->gmres_inner = 0;
  h->mixed_mode = 0;
  h->mixed_kappa = -1.0;
  bool to_gmres = false;
  double* V = reinterpret_cast<double*>(ws + L.gv);  // the GMRES basis is free until GMRES-IR runs
  auto estimate = [&]() -> int {
    // A symmetric: A^-T = A^-1
    const std::function<int(double*, int)> solve = [&](double* v, int) -> int {
      return mixed_solve(h, n, 1, Lf, lds, Winv, v, fl);
    };
    TRY(cond1_estimate(h, n, solve, anorm, V, &h->mixed_kappa));
    to_gmres = h->mixed_kappa * kFactorU > kGmresAbove;
    return EGPU_OK;
  };
  if (h->mixed_policy == 1) TRY(estimate());
  for (;;) {
    copy_cols_kernel<<<cgrid, 256, 0, st>>>(n, nrhs, B, ldb, R, lds, 0);
    count_launch();
    int rg = launch_dgemm_skinny(st, n, nrhs, n, -1.0, As, lds, Xw, lds, R, lds, h->sm_count, h->dstatus);
    if (rg == EGPU_ERR_UNSUPPORTED)
      rg = launch_dgemm(st, false, true, n, nrhs, n, -1.0, As, lds, Xw, lds, 1.0, R, lds, 0, false, h->dstatus);
    TRY(rg);
    TRY(mixed_berr(h, n, nrhs, R, Xw, B, ldb, lds, anorm, norms + n, &e));
    if (e <= tol || it >= max_iter || !std::isfinite(e)) break;
    // the condition estimate sends ill-conditioned systems to GMRES-IR: at
    // once (policy 1), or when the first correction contracted slowly
    if (h->mixed_policy == 0 && it == 1 && e > 0.2 * e_prev && h->mixed_kappa < 0) TRY(estimate());
    if (to_gmres) break;
    // a safety net for estimates that were too low: slow contraction later on
    if (it >= 2 && e > 0.25 * e_prev) break;
    e_prev = e;
    TRY(mixed_solve(h, n, nrhs, Lf, lds, Winv, R, fl));
    copy_cols_kernel<<<cgrid, 256, 0, st>>>(n, nrhs, R, lds, Xw, lds, 1);
    count_launch();
    ++it;
  }
  // GMRES-IR when plain refinement contracts slowly (the factor is good enough
  // to precondition but too far from A to contract): R holds the residual of Xw
  if (e > tol && std::isfinite(e) && it < max_iter) {
    TRY(materialize_lf());
    GmresWork gw{reinterpret_cast<double*>(ws + L.gv), reinterpret_cast<double*>(ws + L.gw),
                 reinterpret_cast<double*>(ws + L.gc), reinterpret_cast<double*>(ws + L.gc) + nrhs};
    int inner = 0;
    double e_best = e;
    while (it < max_iter) {
      const BlockOp apply_a = [&](const double* Vi, double* Wo) -> int {
        EGPU_CUDA_TRY(cudaMemsetAsync(Wo, 0, sizeof(double) * lds * nrhs, st));
        int rg = launch_dgemm_skinny(st, n, nrhs, n, 1.0, As, lds, Vi, lds, Wo, lds, h->sm_count, h->dstatus);
        if (rg == EGPU_ERR_UNSUPPORTED)
          rg = launch_dgemm(st, false, true, n, nrhs, n, 1.0, As, lds, Vi, lds, 0.0, Wo, lds, 0, false, h->dstatus);
        return rg;
      };
      const BlockSolve precond = [&](double* Wo) -> int { return mixed_solve(h, n, nrhs, Lf, lds, Winv, Wo, fl); };
      TRY(gmres_correction(h, n, nrhs, lds, apply_a, precond, R, R, gw, 1e-10, &inner));
      copy_cols_kernel<<<cgrid, 256, 0, st>>>(n, nrhs, R, lds, Xw, lds, 1);
      count_launch();
      ++it;
      copy_cols_kernel<<<cgrid, 256, 0, st>>>(n, nrhs, B, ldb, R, lds, 0);
      count_launch();
      int rg = launch_dgemm_skinny(st, n, nrhs, n, -1.0, As, lds, Xw, lds, R, lds, h->sm_count, h->dstatus);
      if (rg == EGPU_ERR_UNSUPPORTED)
        rg = launch_dgemm(st, false, true, n, nrhs, n, -1.0, As, lds, Xw, lds, 1.0, R, lds, 0, false, h->dstatus);
      TRY(rg);
      TRY(mixed_berr(h, n, nrhs, R, Xw, B, ldb, lds, anorm, norms + n, &e));
      if (e <= tol || !std::isfinite(e) || e > 0.9 * e_best) break;
      e_best = e;
    }
    h->gmres_inner = inner;
    h->mixed_mode = 1;
  }
  copy_cols_kernel<<<cgrid, 256, 0, st>>>(n, nrhs, Xw, lds, X, ldx, 0);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  if (iters) *iters = it;
  if (berr) *berr = e;
  TRY(read_status_now(h, nullptr));
  return e <= tol ? EGPU_OK : EGPU_NO_CONVERGENCE;
}

}  // namespace egpu

extern "C" int egpu_dposv_mixed(egpu_handle h, int uplo, int n, int nrhs, const double* dA, int lda,
                                const double* dB, int ldb, double* dX, int ldx, int max_iter, double tol,
                                int* iters, double* berr) {
  if (iters) *iters = 0;
  if (berr) *berr = 0.0;
  if (!h) return EGPU_ERR_ARG;
  if (n < 0 || nrhs < 0 || lda < std::max(1, n) || ldb < std::max(1, n) || ldx < std::max(1, n) ||
      (uplo != EGPU_LOWER && uplo != EGPU_UPPER) || max_iter < 0)
    return EGPU_ERR_ARG;
  if (n == 0 || nrhs == 0) return EGPU_OK;
  Enter en(h);
  return egpu::dposv_mixed_core_impl(h, uplo, n, nrhs, dA, lda, dB, ldb, dX, ldx, max_iter, tol, iters, berr);
}

extern "C" int egpu_mixed_gmres_iterations(egpu_handle h) { return h ? h->gmres_inner : -1; }

extern "C" int egpu_set_mixed_policy(egpu_handle h, int policy) {
  if (!h || policy < 0 || policy > 1) return EGPU_ERR_ARG;
  h->mixed_policy = policy;
  return EGPU_OK;
}

extern "C" int egpu_mixed_mode(egpu_handle h) { return h ? h->mixed_mode : -1; }

extern "C" int egpu_mixed_condition_estimate(egpu_handle h, double* kappa1) {
  if (!h || !kappa1) return EGPU_ERR_ARG;
  *kappa1 = h->mixed_kappa;
  return EGPU_OK;
}

// Testing entry for the tcgen05 engine: C (FP32) = alpha A B^T + beta C with
// A (M x K) and B (N x K) given column-major in FP64 and split into TF32 parts.
extern "C" int egpu_tc_gemm_split(egpu_handle h, int M, int N, int K, double alpha, const double* dA, int lda,
                                  const double* dB, int ldb, double beta, float* dC, int ldc, int lower, int terms) {
  if (!h) return EGPU_ERR_ARG;
  if (M < 0 || N < 0 || K < 1 || lda < std::max(1, M) || ldb < std::max(1, N) || ldc < std::max(1, M))
    return EGPU_ERR_ARG;
  if (M == 0 || N == 0) return EGPU_OK;
  Enter en(h);
  const long long ldk = ((long long)K + 31) / 32 * 32;
  const size_t ab = sizeof(float) * (size_t)M * ldk, bb = sizeof(float) * (size_t)N * ldk;
  auto up = [](size_t x) { return (x + 1023) & ~size_t(1023); };
  TRY(ensure_ws(h, 2 * up(ab) + 2 * up(bb) + 4096));
  unsigned char* ws = static_cast<unsigned char*>(h->ws);
  float* Ah = reinterpret_cast<float*>(ws);
  float* Al = reinterpret_cast<float*>(ws + up(ab));
  float* Bh = reinterpret_cast<float*>(ws + 2 * up(ab));
  float* Bl = reinterpret_cast<float*>(ws + 2 * up(ab) + up(bb));
  cudaStream_t st = h->stream;
  EGPU_CUDA_TRY(cudaMemsetAsync(h->dstatus, 0, sizeof(DevStatus), st));
  TRY(launch_split_tf32(st, M, K, dA, lda, Ah, Al, ldk));
  TRY(launch_split_tf32(st, N, K, dB, ldb, Bh, Bl, ldk));
  TRY(launch_tc_gemm(st, M, N, K, (float)alpha, Ah, Al, Bh, Bl, ldk, (float)beta, dC, ldc, lower ? 1 : 0, terms,
                     h->dstatus));
  return read_status_now(h, nullptr);
}

int dposv_mixed_core(egpu_context* h, int uplo, int n, int nrhs, const double* A, long long lda, const double* B,
                     long long ldb, double* X, long long ldx, int max_iter, double tol, int* iters, double* berr) {
  return egpu::dposv_mixed_core_impl(h, uplo, n, nrhs, A, lda, B, ldb, X, ldx, max_iter, tol, iters, berr);
}
