// LU panel factorization with partial pivoting and the row-interchange
// kernels.
//
// lu::Panel (lapack-like/LU/Panel.hpp:19-89) is inherently column-sequential:
// each column's pivot is the first entry of maximal |a| after all previous
// columns' updates.  On the GPU the m x b panel is split row-wise over P
// co-resident CTAs, each holding its rows in shared memory for the whole
// panel.  Per column: every CTA finds its local argmax (warp shuffles + one
// block reduction) and publishes the candidate together with the candidate's
// full row; one bounded grid barrier; then every CTA picks the global winner
// (largest |a|, ties -> lowest row, i.e. the reference's strict '>' scan),
// the two owners swap rows through the published copies, and every CTA scales
// and rank-1 updates its own rows.  One grid barrier per column.
#include "diag_common.cuh"
#include "internal.h"

namespace egpu {

constexpr int kPanelThreads = 256;
constexpr int kPanelMaxRowsPerCta = 192;

struct PanelCand {
  double absv;
  double val;
  int row;
  int pad;
};

struct PanelScratchLayout {
  size_t counter, cand, rowbuf, jrow, total;
};

static PanelScratchLayout panel_layout(int P, int b) {
  PanelScratchLayout L;
  size_t off = 0;
  L.counter = off; off += 256;
  L.cand = off; off += sizeof(PanelCand) * 2 * (size_t)P; off = (off + 255) & ~size_t(255);
  L.rowbuf = off; off += sizeof(double) * 2 * (size_t)P * b; off = (off + 255) & ~size_t(255);
  L.jrow = off; off += sizeof(double) * 2 * (size_t)b; off = (off + 255) & ~size_t(255);
  L.total = off;
  return L;
}

static int panel_rows_per_cta(int m, int sm_count) {
  int R = 128;
  while ((m + R - 1) / R > sm_count && R < kPanelMaxRowsPerCta) R += 32;
  return R;
}

size_t lu_panel_scratch_bytes(int m, int b, int sm_count) {
  const int R = panel_rows_per_cta(m, sm_count);
  const int P = (m + R - 1) / R;
  return panel_layout(P, b).total;
}

__device__ __forceinline__ bool cand_better(double a, int ra, double b, int rb) {
  return a > b || (a == b && ra < rb);
}

__global__ void __launch_bounds__(kPanelThreads) lu_panel_kernel(int m, int b, double* A, long long lda, int* p,
                                                                  int offset, int* image, int* preimage,
                                                                  double* W, int ldw, unsigned char* scratch,
                                                                  PanelScratchLayout L, int R, DevStatus* st) {
  extern __shared__ double S[];  // b columns x R rows (ld R), then u[b]
  double* u = S + (size_t)b * R;
  __shared__ double red_abs[kPanelThreads / 32];
  __shared__ int red_row[kPanelThreads / 32];
  __shared__ double red_val[kPanelThreads / 32];
  __shared__ int red_cta[kPanelThreads / 32];
  __shared__ int s_win, s_prow, s_stop;
  __shared__ double s_pval;

  const int P = gridDim.x;
  const int cta = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = cta * R;
  const int rows = min(R, m - r0);
  unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + L.counter);
  PanelCand* cand = reinterpret_cast<PanelCand*>(scratch + L.cand);
  double* rowbuf = reinterpret_cast<double*>(scratch + L.rowbuf);
  double* jrow = reinterpret_cast<double*>(scratch + L.jrow);

  if (st != nullptr && st->code != 0) return;  // uniform across the grid: set before launch

  for (int c = 0; c < b; ++c)
    for (int lr = tid; lr < rows; lr += kPanelThreads) S[c * R + lr] = A[(long long)c * lda + r0 + lr];
  __syncthreads();

  const int ncols = min(b, m);
  for (int j = 0; j < ncols; ++j) {
    const int par = j & 1;
    // 1. local argmax over rows >= j (first maximal |a| wins ties)
    double best = -1.0, bval = 0.0;
    int brow = 0x7fffffff;
    const int lr0 = max(0, j - r0);
    for (int lr = lr0 + tid; lr < rows; lr += kPanelThreads) {
      const double v = S[j * R + lr];
      const double av = fabs(v);
      if (cand_better(av, r0 + lr, best, brow)) { best = av; brow = r0 + lr; bval = v; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_down_sync(0xffffffffu, best, o);
      const int orow = __shfl_down_sync(0xffffffffu, brow, o);
      const double ov = __shfl_down_sync(0xffffffffu, bval, o);
      if (cand_better(ob, orow, best, brow)) { best = ob; brow = orow; bval = ov; }
    }
    if (lane == 0) { red_abs[warp] = best; red_row[warp] = brow; red_val[warp] = bval; }
    __syncthreads();
    if (tid == 0) {
      for (int w = 1; w < kPanelThreads / 32; ++w)
        if (cand_better(red_abs[w], red_row[w], best, brow)) { best = red_abs[w]; brow = red_row[w]; bval = red_val[w]; }
      PanelCand cc;
      cc.absv = best; cc.val = bval; cc.row = brow; cc.pad = 0;
      cand[par * P + cta] = cc;
      red_row[0] = brow;
    }
    __syncthreads();
    {
      const int myrow = red_row[0];
      double* rb = rowbuf + ((size_t)par * P + cta) * b;
      if (myrow != 0x7fffffff)
        for (int c = tid; c < b; c += kPanelThreads) rb[c] = S[c * R + (myrow - r0)];
      if (j >= r0 && j < r0 + rows)
        for (int c = tid; c < b; c += kPanelThreads) jrow[par * b + c] = S[c * R + (j - r0)];
    }
    // 2. one grid-wide barrier per column (its leading __syncthreads orders
    //    this CTA's stores before thread 0's release fence)
    if (!grid_barrier(counter, (unsigned)P * (unsigned)(j + 1))) {
      if (tid == 0) set_status(st, kTimeout, 200 + j);
      return;
    }
    // 3. global winner: largest |a|, ties -> lowest row (the strict '>' scan
    //    of LU/Panel.hpp:52-63).  Thread c reads CTA c's candidate with an
    //    L2-coherent load (.cg), then a block argmax reduction.
    {
      double wb = -1.0, wv = 0.0;
      int wr = 0x7fffffff, wc = 0;
      if (tid < P) {
        const PanelCand* cp = &cand[par * P + tid];
        wb = __ldcg(&cp->absv);
        wr = __ldcg(&cp->row);
        wv = __ldcg(&cp->val);
        wc = tid;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, wb, o);
        const int orow = __shfl_down_sync(0xffffffffu, wr, o);
        const double ov = __shfl_down_sync(0xffffffffu, wv, o);
        const int oc = __shfl_down_sync(0xffffffffu, wc, o);
        if (cand_better(ob, orow, wb, wr)) { wb = ob; wr = orow; wv = ov; wc = oc; }
      }
      if (lane == 0) { red_abs[warp] = wb; red_row[warp] = wr; red_val[warp] = wv; red_cta[warp] = wc; }
      __syncthreads();
      if (tid == 0) {
        for (int w = 1; w < kPanelThreads / 32; ++w)
          if (cand_better(red_abs[w], red_row[w], wb, wr)) { wb = red_abs[w]; wr = red_row[w]; wv = red_val[w]; wc = red_cta[w]; }
        s_win = wc; s_prow = wr; s_pval = wv;
        s_stop = (wv == 0.0);
        if (cta == 0) p[j] = wr + offset;
      }
      __syncthreads();
    }
    const int prow = s_prow;
    const double pval = s_pval;
    const double* wrow = rowbuf + ((size_t)par * P + s_win) * b;
    if (s_stop) {  // exact zero pivot: SingularMatrixException (LU/Panel.hpp:76-77)
      if (cta == 0 && tid == 0) set_status(st, kSingular, offset + j + 1);
      break;
    }
    // swap rows j <-> prow across the whole panel width
    if (prow != j) {
      if (prow >= r0 && prow < r0 + rows)
        for (int c = tid; c < b; c += kPanelThreads) S[c * R + (prow - r0)] = __ldcg(&jrow[par * b + c]);
      if (j >= r0 && j < r0 + rows)
        for (int c = tid; c < b; c += kPanelThreads) S[c * R + (j - r0)] = __ldcg(&wrow[c]);
    }
    for (int c = j + 1 + tid; c < b; c += kPanelThreads) u[c] = __ldcg(&wrow[c]);
    __syncthreads();
    // 4. Scale (multiply by 1/pivot, LU/Panel.hpp:78-79) and Geru (:80) on own rows > j
    const double inv = 1.0 / pval;
    const int lr1 = max(0, j + 1 - r0);
    const int nr = rows - lr1;
    for (int lr = lr1 + tid; lr < rows; lr += kPanelThreads) S[j * R + lr] *= inv;
    __syncthreads();
    if (nr > 0) {
      // threads: (row, column-phase) with consecutive threads on consecutive rows
      const int tpr = (nr >= kPanelThreads) ? 1 : (nr >= kPanelThreads / 2 ? 2 : 4);
      const int ph = tid % tpr;
      for (int lr = lr1 + tid / tpr; lr < rows; lr += kPanelThreads / tpr) {
        const double l = S[j * R + lr];
        for (int c = j + 1 + ph; c < b; c += tpr) S[c * R + lr] -= l * u[c];
      }
    }
    __syncthreads();
  }

  for (int c = 0; c < b; ++c)
    for (int lr = tid; lr < rows; lr += kPanelThreads) A[(long long)c * lda + r0 + lr] = S[c * R + lr];

  if (cta != 0) return;
  __syncthreads();
  if (st != nullptr && ((volatile DevStatus*)st)->code != 0) return;
  // ComposePivots(p, offset, image, preimage), lapack-like/ComposePivots.hpp:81-125
  if (tid < b) {
    const int i = tid;
    int k = p[i] - offset;
    for (int jj = i - 1; jj >= 0; --jj) {
      const int pj = p[jj] - offset;
      if (pj == k) k = jj;
      else if (jj == k) k = pj;
    }
    preimage[i] = k;
    k = i;
    for (int jj = 0; jj < min(k + 1, b); ++jj) {
      const int pj = p[jj] - offset;
      if (pj == k) k = jj;
      else if (jj == k) k = pj;
    }
    image[i] = k;
  }
  // inv(unit lower L11) from the top b x b of the panel (rows owned by CTA 0)
  __syncthreads();
  if (W != nullptr) {
    const int i = tid;
    for (int j = b - 1; j >= 0; --j) {
      double tmp = 0.0;
      if (i > j && i < b) {
        for (int k = j + 1; k < i; ++k) tmp = fma(S[k * R + i], S[j * R + k], tmp);
        tmp += S[j * R + i];
      }
      __syncthreads();
      if (i > j && i < b) S[j * R + i] = -tmp;
      __syncthreads();
    }
    for (int idx = tid; idx < b * b; idx += kPanelThreads) {
      const int r = idx % b, c = idx / b;
      W[r + (long long)c * ldw] = r > c ? S[c * R + r] : (r == c ? 1.0 : 0.0);
    }
  }
}

// Panel dispatch: the register-resident cluster form (lu_panel_rp.cu) takes
// every panel of up to 16 x 1024 rows; taller panels (up to 148 x 192 rows)
// run the cooperative grid form above, one bounded grid barrier per column.
int launch_lu_panel(cudaStream_t st, int m, int b, double* A, long long lda, int* p, int offset, int* image,
                    int* preimage, double* W, int ldw, void* scratch, DevStatus* status, int sm_count) {
  if (m <= 0 || b <= 0) return EGPU_OK;
  if (b > 128) return EGPU_ERR_ARG;
  {
    const int rc = launch_lu_panel_rp(st, m, b, A, lda, p, offset, image, preimage, W, ldw, status, 16);
    if (rc != EGPU_ERR_UNSUPPORTED) return rc;
  }
  const int R = panel_rows_per_cta(m, sm_count);
  const int P = (m + R - 1) / R;
  if (P > sm_count || R < b) return EGPU_ERR_UNSUPPORTED;
  const PanelScratchLayout L = panel_layout(P, b);
  const size_t smem = sizeof(double) * ((size_t)b * R + b);
  TraceMark tm(st, kTracePanel, (double)m * b * b, 16.0 * m * b);
  cudaError_t e = cudaMemsetAsync(static_cast<unsigned char*>(scratch) + L.counter, 0, sizeof(unsigned), st);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(lu_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(double) * (128 * kPanelMaxRowsPerCta + 128)));
  if (e == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P);
    cfg.blockDim = dim3(kPanelThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // all P CTAs co-resident (grid barrier)
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, lu_panel_kernel, m, b, A, lda, p, offset, image, preimage, W, ldw,
                           static_cast<unsigned char*>(scratch), L, R, status);
    count_launch();
  }
  if (e != cudaSuccess) {
    set_last_error(e, "lu_panel launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

// ApplyRowPivots(A, image, preimage), lapack-like/ApplyRowPivots.hpp:129-181:
// row i (< b) moves to image[i]; row preimage[i] (>= b) moves into row i.
// The destination rows are pairwise distinct, so one read phase and one
// write phase per group of columns suffice.
__global__ void __launch_bounds__(128) apply_composed_kernel(int m, int ncols, double* A, long long lda, int b,
                                                            const int* image, const int* preimage,
                                                            const DevStatus* st) {
  if (st != nullptr && st->code != 0) return;
  const int i = threadIdx.x;
  const int img = (i < b) ? image[i] : 0;
  const int pre = (i < b) ? preimage[i] : 0;
  constexpr int G = 8;
  for (int c0 = blockIdx.x * G; c0 < ncols; c0 += gridDim.x * G) {
    double v1[G], v2[G];
#pragma unroll
    for (int q = 0; q < G; ++q) {
      const int c = c0 + q;
      if (c < ncols && i < b) {
        v1[q] = A[i + (long long)c * lda];
        v2[q] = (pre >= b) ? A[pre + (long long)c * lda] : 0.0;
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

int launch_apply_composed(cudaStream_t st, int m, int ncols, double* A, long long lda, int b, const int* image,
                          const int* preimage, const DevStatus* status) {
  if (m <= 0 || ncols <= 0 || b <= 0) return EGPU_OK;
  const int blocks = std::min((ncols + 7) / 8, 148 * 8);
  TraceMark tm(st, kTraceSwap, 0.0, 32.0 * b * ncols);
  apply_composed_kernel<<<blocks, 128, 0, st>>>(m, ncols, A, lda, b, image, preimage, status);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "apply_composed launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

// Compose sequential swaps i <-> p[i] (forward, or reverse for the inverse)
// into perm: after the swaps, row r holds original row perm[r].  The swaps
// are a dependent chain (one thread); with `smem` the permutation and the
// pivots are staged in shared memory first, so each step is a few shared
// accesses instead of dependent global round trips.
__global__ void compose_perm_kernel(int inverse, int m, const int* p, int np, int* perm, int smem) {
  extern __shared__ int sperm[];
  int* q = smem ? sperm : perm;
  int* sp = sperm + m;
  for (int r = threadIdx.x; r < m; r += blockDim.x) q[r] = r;
  if (smem)
    for (int i = threadIdx.x; i < np; i += blockDim.x) sp[i] = p[i];
  __syncthreads();
  const int* pp = smem ? sp : p;
  if (threadIdx.x == 0) {
    // a pivot outside [0, m) (caller data) is skipped, never followed
    if (!inverse) {
      for (int i = 0; i < np; ++i) {
        const int k = pp[i];
        if ((unsigned)k >= (unsigned)m || i >= m) continue;
        const int t = q[i]; q[i] = q[k]; q[k] = t;
      }
    } else {
      for (int i = np - 1; i >= 0; --i) {
        const int k = pp[i];
        if ((unsigned)k >= (unsigned)m || i >= m) continue;
        const int t = q[i]; q[i] = q[k]; q[k] = t;
      }
    }
  }
  __syncthreads();
  if (smem)
    for (int r = threadIdx.x; r < m; r += blockDim.x) perm[r] = q[r];
}

// dst[r, c] = src[perm[r], c]
__global__ void gather_rows_kernel(int m, int n, const int* perm, const double* src, long long lds, double* dst,
                                   long long ldd) {
  const long long total = (long long)m * n;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(idx % m), c = (int)(idx / m);
    dst[r + c * ldd] = src[perm[r] + c * lds];
  }
}

int launch_compose_perm(cudaStream_t st, int inverse, int m, const int* p, int np, int* perm) {
  if (m <= 0) return EGPU_OK;
  const size_t sbytes = sizeof(int) * ((size_t)m + np);
  const bool smem = sbytes <= 200 * 1024;
  static int attr_dev_mask = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (smem && dev < 31 && !(attr_dev_mask & (1 << dev))) {
    EGPU_CUDA_TRY(cudaFuncSetAttribute(compose_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr_dev_mask |= 1 << dev;
  }
  compose_perm_kernel<<<1, 1024, smem ? sbytes : 0, st>>>(inverse, m, p, np, perm, smem ? 1 : 0);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  return EGPU_OK;
}

int launch_permute_rows(cudaStream_t st, int m, int n, const int* perm, double* A, long long lda, double* tmp) {
  if (m <= 0 || n <= 0) return EGPU_OK;
  const long long total = (long long)m * n;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 16);
  gather_rows_kernel<<<blocks, 256, 0, st>>>(m, n, perm, A, lda, tmp, m);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(e, "laswp launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return launch_copy(st, m, n, tmp, m, A, lda);
}

// perm_scratch: int[m] followed by double[m * n] (8-byte aligned after m ints
// rounded up to an even count).
int launch_laswp_seq(cudaStream_t st, int inverse, int m, int n, double* A, long long lda, const int* p, int np,
                     int* perm_scratch) {
  if (m <= 0 || n <= 0 || np <= 0) return EGPU_OK;
  int* perm = perm_scratch;
  double* tmp = reinterpret_cast<double*>(perm_scratch + ((m + 1) & ~1));
  const int rc = launch_compose_perm(st, inverse, m, p, np, perm);
  if (rc != EGPU_OK) return rc;
  return launch_permute_rows(st, m, n, perm, A, lda, tmp);
}

}  // namespace egpu
