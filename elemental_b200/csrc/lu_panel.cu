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

// ---------------------------------------------------------------------------
// Cluster form of the panel for m <= 16 * 192 rows: the P <= 16 CTAs form one
// thread-block cluster.  Candidates are written straight into every CTA's
// shared memory (DSMEM), the per-column barrier is the hardware cluster
// barrier, and the winning row is read from the winner's shared memory.  Each
// CTA keeps private copies of its candidate row and of row j, double-buffered
// by column parity, so one cluster barrier per column suffices: a buffer is
// rewritten two columns later, after every reader has passed the next barrier.
struct ClusterCand {
  double absv, val, row, pad;
};

__global__ void __launch_bounds__(kPanelThreads) lu_panel_cluster_kernel(int m, int b, double* A, long long lda,
                                                                          int* p, int offset, int* image,
                                                                          int* preimage, double* W, int ldw, int R,
                                                                          DevStatus* st) {
  extern __shared__ double S[];  // b x R rows (ld R) | u[b] | crow[2][b] | jbuf[2][b] | cand[2][16]
  double* u = S + (size_t)b * R;
  double* crow = u + b;
  double* jbuf = crow + 2 * b;
  ClusterCand* cand = reinterpret_cast<ClusterCand*>(jbuf + 2 * b);
  __shared__ double red_abs[kPanelThreads / 32];
  __shared__ int red_row[kPanelThreads / 32];
  __shared__ double red_val[kPanelThreads / 32];
  __shared__ int s_win, s_prow, s_stop;
  __shared__ double s_pval;

  const int P = gridDim.x;  // == cluster size
  const unsigned cta = cluster_ctarank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = (int)cta * R;
  const int rows = max(0, min(R, m - r0));
  // An earlier failure (status word) skips the panel.  CTA 0's reading is
  // the cluster's decision, so every CTA leaves at the same point.
  __shared__ int s_skip;
  if (tid == 0) s_skip = (st != nullptr && ((volatile DevStatus*)st)->code != 0);
  for (int c = 0; c < b; ++c)
    for (int lr = tid; lr < rows; lr += kPanelThreads) S[c * R + lr] = A[(long long)c * lda + r0 + lr];
  __syncthreads();
  cluster_arrive_release();  // all CTAs resident and initialised before any DSMEM traffic
  cluster_wait_acquire();
  const int skip = *cluster_map(&s_skip, 0u);
  cluster_arrive_release();  // CTA 0's flag has been read by all before anyone leaves
  cluster_wait_acquire();
  if (skip) return;

  const int ncols = min(b, m);
  for (int j = 0; j < ncols; ++j) {
    const int par = j & 1;
    double best = -1.0, bval = 0.0;
    int brow = 0x7fffffff;
    for (int lr = max(0, j - r0) + tid; lr < rows; lr += kPanelThreads) {
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
    if (warp == 0) {
      best = lane < kPanelThreads / 32 ? red_abs[lane] : -1.0;
      brow = lane < kPanelThreads / 32 ? red_row[lane] : 0x7fffffff;
      bval = lane < kPanelThreads / 32 ? red_val[lane] : 0.0;
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int orow = __shfl_down_sync(0xffffffffu, brow, o);
        const double ov = __shfl_down_sync(0xffffffffu, bval, o);
        if (cand_better(ob, orow, best, brow)) { best = ob; brow = orow; bval = ov; }
      }
      best = __shfl_sync(0xffffffffu, best, 0);
      brow = __shfl_sync(0xffffffffu, brow, 0);
      bval = __shfl_sync(0xffffffffu, bval, 0);
      if (lane < P) {  // candidate into every CTA's slot [par][cta]
        ClusterCand* dst = cluster_map(&cand[par * 16 + cta], (unsigned)lane);
        dst->absv = best; dst->val = bval; dst->row = (double)brow;
      }
      if (lane == 0) red_row[0] = brow;
    }
    __syncthreads();
    {
      const int myrow = red_row[0];
      if (myrow != 0x7fffffff)
        for (int c = tid; c < b; c += kPanelThreads) crow[par * b + c] = S[c * R + (myrow - r0)];
      if (j >= r0 && j < r0 + rows)
        for (int c = tid; c < b; c += kPanelThreads) jbuf[par * b + c] = S[c * R + (j - r0)];
    }
    __syncthreads();
    cluster_arrive_release();
    cluster_wait_acquire();
    if (warp == 0) {
      double wb = -1.0, wv = 0.0;
      int wr = 0x7fffffff, wc = 0;
      if (lane < P) {
        const ClusterCand cc = cand[par * 16 + lane];
        wb = cc.absv; wv = cc.val; wr = (int)cc.row; wc = lane;
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, wb, o);
        const int orow = __shfl_down_sync(0xffffffffu, wr, o);
        const double ov = __shfl_down_sync(0xffffffffu, wv, o);
        const int oc = __shfl_down_sync(0xffffffffu, wc, o);
        if (cand_better(ob, orow, wb, wr)) { wb = ob; wr = orow; wv = ov; wc = oc; }
      }
      if (lane == 0) {
        s_win = wc; s_prow = wr; s_pval = wv;
        s_stop = (wv == 0.0);
        if (cta == 0) p[j] = wr + offset;
      }
    }
    __syncthreads();
    const int prow = s_prow;
    const double pval = s_pval;
    if (s_stop) {  // exact zero pivot: SingularMatrixException (LU/Panel.hpp:76-77)
      if (cta == 0 && tid == 0) set_status(st, kSingular, offset + j + 1);
      break;
    }
    const double* wrow = cluster_map(crow + par * b, (unsigned)s_win);
    if (prow != j) {
      if (prow >= r0 && prow < r0 + rows) {
        const double* jr = cluster_map(jbuf + par * b, (unsigned)(j / R));
        for (int c = tid; c < b; c += kPanelThreads) S[c * R + (prow - r0)] = jr[c];
      }
      if (j >= r0 && j < r0 + rows)
        for (int c = tid; c < b; c += kPanelThreads) S[c * R + (j - r0)] = wrow[c];
    }
    for (int c = j + 1 + tid; c < b; c += kPanelThreads) u[c] = wrow[c];
    const double inv = 1.0 / pval;
    const int lr1 = max(0, j + 1 - r0);
    __syncthreads();
    for (int lr = lr1 + tid; lr < rows; lr += kPanelThreads) S[j * R + lr] *= inv;
    __syncthreads();
    const int nr = rows - lr1;
    if (nr > 0) {
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
  // no CTA may exit while others can still read its shared memory
  __syncthreads();
  cluster_arrive_release();
  cluster_wait_acquire();
  if (cta != 0) return;
  if (st != nullptr && ((volatile DevStatus*)st)->code != 0) return;
  if (tid < b) {  // ComposePivots(p, offset, image, preimage), ComposePivots.hpp:81-125
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
  __syncthreads();
  if (W != nullptr) {  // inv(unit lower L11)
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

// ---------------------------------------------------------------------------
// Sub-panel form of the panel (m <= 16 * kSpMaxR rows): one thread-block
// cluster of P <= 16 CTAs, each owning R consecutive rows.  The panel stays in
// global memory (it is L2-resident); a CTA keeps only the 16 columns of the
// current sub-panel of its rows in shared memory.  Per column: a local argmax,
// one message per CTA written into every CTA's shared memory (candidate |a|,
// value, row, and the sub-panel parts of the candidate row and of row j), one
// hardware cluster barrier, then every warp picks the winner from its local
// copy of the messages, and each CTA swaps / scales / updates the sub-panel
// rows it owns.  After a sub-panel (LU/Panel.hpp:19-89 applied to 16 columns)
// the pivots are applied to the rest of the panel's columns, CTA 0 solves the
// 16 pivot rows of the remaining columns with the unit-lower 16 x 16 factor,
// and every CTA updates its rows of those columns with a 4x4-blocked
// mini-GEMM.  The result equals lu::Panel's (same pivots; the trailing part of
// the panel is updated in 16-column blocks instead of column by column).
constexpr int kSpThreads = 256;
constexpr int kSpW = 16;
constexpr int kSpMsg = 36;  // header 4 + candidate row 16 + row j 16
constexpr int kSpMaxCl = 16;
constexpr int kSpMaxR = 1024;

__host__ __device__ inline size_t sp_panel_doubles(int R) {
  const size_t work = (size_t)kSpW * R + 2 * kSpMaxCl * kSpMsg + kSpW * 128 + 2 * kSpW * 128;
  const size_t inv = 128 * kLDS + 128;
  return work > inv ? work : inv;
}

__global__ void __launch_bounds__(kSpThreads) lu_panel_sp_kernel(int m, int b, double* A, long long lda, int* p,
                                                                  int offset, int* image, int* preimage, double* W,
                                                                  int ldw, int R, DevStatus* st) {
  extern __shared__ double sm[];
  double* SP = sm;                                     // kSpW columns x R rows (ld R)
  double* MSG = SP + (size_t)kSpW * R;                 // [2][kSpMaxCl][kSpMsg]
  double* UB = MSG + 2 * kSpMaxCl * kSpMsg;            // U12 rows: [k][c - c1], ld 128
  double* MV = UB + kSpW * 128;                        // row moves: [2 kSpW][128]
  __shared__ double red_abs[kSpThreads / 32];
  __shared__ int red_row[kSpThreads / 32];
  __shared__ double red_val[kSpThreads / 32];
  __shared__ int s_piv[kSpW], s_img[kSpW], s_pre[kSpW];
  __shared__ int s_skip;

  const int P = gridDim.x;
  const unsigned cta = cluster_ctarank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = (int)cta * R;
  const int rows = max(0, min(R, m - r0));
  if (tid == 0) s_skip = (st != nullptr && ((volatile DevStatus*)st)->code != 0);
  __syncthreads();
  cluster_arrive_release();
  cluster_wait_acquire();
  const int skip = *cluster_map(&s_skip, 0u);
  cluster_arrive_release();
  cluster_wait_acquire();
  if (skip) return;

  const int ncols = min(b, m);
  bool stop = false;
  for (int c0 = 0; c0 < ncols; c0 += kSpW) {
    const int c1 = min(ncols, c0 + kSpW), w = c1 - c0;
    // rows of this CTA may have been rewritten by CTA 0's interchanges: read
    // around L1 (pairs of rows with 16-byte .cg copies; R and r0 are even)
    {
      const int pairs = rows >> 1;
      for (int k = 0; k < w; ++k) {
        const double* src = &A[(long long)(c0 + k) * lda + r0];
        for (int q = tid; q < pairs; q += kSpThreads) cp_async16_cg(&SP[k * R + 2 * q], src + 2 * q);
        if ((rows & 1) && tid == 0) SP[k * R + rows - 1] = __ldcg(src + rows - 1);
      }
      cp_async_wait_all();
      __syncthreads();
    }
    for (int j = c0; j < c1; ++j) {
      const int jj = j - c0, par = j & 1;
      // a. local argmax over own rows >= j (first maximal |a| on ties)
      double best = -1.0, bval = 0.0;
      int brow = 0x7fffffff;
      for (int lr = max(0, j - r0) + tid; lr < rows; lr += kSpThreads) {
        const double v = SP[jj * R + lr];
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
      // b. warp 0: CTA candidate, message into every CTA of the cluster
      if (warp == 0) {
        best = lane < kSpThreads / 32 ? red_abs[lane] : -1.0;
        brow = lane < kSpThreads / 32 ? red_row[lane] : 0x7fffffff;
        bval = lane < kSpThreads / 32 ? red_val[lane] : 0.0;
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
          const double ob = __shfl_down_sync(0xffffffffu, best, o);
          const int orow = __shfl_down_sync(0xffffffffu, brow, o);
          const double ov = __shfl_down_sync(0xffffffffu, bval, o);
          if (cand_better(ob, orow, best, brow)) { best = ob; brow = orow; bval = ov; }
        }
        best = __shfl_sync(0xffffffffu, best, 0);
        brow = __shfl_sync(0xffffffffu, brow, 0);
        bval = __shfl_sync(0xffffffffu, bval, 0);
        const bool has = brow != 0x7fffffff;
        const bool ownj = (j >= r0 && j < r0 + rows);
        const int lb = has ? brow - r0 : 0;
        // stage the message in registers: lane q < 18 holds double2 number q
        // (0: |a|, value; 1: row, owns-j; 2..9: candidate row; 10..17: row j)
        double2 mv = make_double2(0.0, 0.0);
        if (lane == 0) mv = make_double2(best, bval);
        else if (lane == 1) mv = make_double2((double)brow, ownj ? 1.0 : 0.0);
        else if (lane < 10) {
          const int k = 2 * (lane - 2);
          if (has) mv = make_double2(k < w ? SP[k * R + lb] : 0.0, k + 1 < w ? SP[(k + 1) * R + lb] : 0.0);
        } else if (lane < 18) {
          const int k = 2 * (lane - 10);
          if (ownj) mv = make_double2(k < w ? SP[k * R + (j - r0)] : 0.0, k + 1 < w ? SP[(k + 1) * R + (j - r0)] : 0.0);
        }
        const int nq = ownj ? 18 : 10;  // row j travels only from its owner
        double2* slot = reinterpret_cast<double2*>(&MSG[(par * kSpMaxCl + cta) * kSpMsg]);
        if (lane < nq)
          for (int t = 0; t < P; ++t) *cluster_map(slot + lane, (unsigned)t) = mv;
      }
      cluster_arrive_release();
      cluster_wait_acquire();
      // c. winner, computed by every warp from its CTA's copy of the messages
      double wb = -1.0, wv = 0.0;
      int wr = 0x7fffffff, wc = 0;
      if (lane < P) {
        const double* mm = &MSG[(par * kSpMaxCl + lane) * kSpMsg];
        wb = mm[0]; wv = mm[1]; wr = (int)mm[2]; wc = lane;
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, wb, o);
        const int orow = __shfl_down_sync(0xffffffffu, wr, o);
        const double ov = __shfl_down_sync(0xffffffffu, wv, o);
        const int oc = __shfl_down_sync(0xffffffffu, wc, o);
        if (cand_better(ob, orow, wb, wr)) { wb = ob; wr = orow; wv = ov; wc = oc; }
      }
      wr = __shfl_sync(0xffffffffu, wr, 0);
      wv = __shfl_sync(0xffffffffu, wv, 0);
      wc = __shfl_sync(0xffffffffu, wc, 0);
      if (wv == 0.0) {  // exact zero pivot: SingularMatrixException (LU/Panel.hpp:76-77)
        if (cta == 0 && tid == 0) set_status(st, kSingular, offset + j + 1);
        stop = true;
        break;
      }
      if (cta == 0 && tid == 0) p[j] = wr + offset;
      if (tid == 0) s_piv[jj] = wr;
      const double* wmsg = &MSG[(par * kSpMaxCl + wc) * kSpMsg];
      const double* jmsg = &MSG[(par * kSpMaxCl + j / R) * kSpMsg];
      // d. row interchange inside the sub-panel
      if (wr != j) {
        if (j >= r0 && j < r0 + rows && tid < w) SP[tid * R + (j - r0)] = wmsg[4 + tid];
        if (wr >= r0 && wr < r0 + rows && tid < w) SP[tid * R + (wr - r0)] = jmsg[4 + kSpW + tid];
      }
      __syncthreads();
      // e. Scale (x 1/pivot, Panel.hpp:78-79) and rank-1 update (Geru, :80) of own rows > j
      const double inv = 1.0 / wv;
      for (int lr = max(0, j + 1 - r0) + tid; lr < rows; lr += kSpThreads) {
        const double l = SP[jj * R + lr] * inv;
        SP[jj * R + lr] = l;
        for (int k = jj + 1; k < w; ++k) SP[k * R + lr] -= l * wmsg[4 + k];
      }
      __syncthreads();
    }
    if (stop) break;
    // write back the sub-panel
    for (int k = 0; k < w; ++k)
      for (int lr = tid; lr < rows; lr += kSpThreads) A[(long long)(c0 + k) * lda + r0 + lr] = SP[k * R + lr];
    // The sub-panel's interchanges on the panel's other columns ([0, c0) and
    // [c1, b)).  ComposePivots (ComposePivots.hpp:81-125) relative to row c0
    // gives image/preimage; every CTA moves the rows whose destination it owns
    // (all sources are read before any row is written: a source can also be a
    // destination), then CTA 0 solves the pivot rows of the remaining columns.
    if (tid < w) {
      const int i = tid;
      int k = s_piv[i] - c0;
      for (int q = i - 1; q >= 0; --q) {
        const int pq = s_piv[q] - c0;
        if (pq == k) k = q;
        else if (q == k) k = pq;
      }
      s_pre[i] = k;
      k = i;
      for (int q = 0; q < min(k + 1, w); ++q) {
        const int pq = s_piv[q] - c0;
        if (pq == k) k = q;
        else if (q == k) k = pq;
      }
      s_img[i] = k;
    }
    __syncthreads();
    const int nout = b - w;
    // move mv < w: row c0+mv -> row c0+img[mv]; move w+i: row c0+pre[i] -> row c0+i (pre[i] >= w)
    auto move_src = [&](int mv) { return mv < w ? c0 + mv : c0 + s_pre[mv - w]; };
    auto move_dst = [&](int mv) { return mv < w ? c0 + s_img[mv] : c0 + (mv - w); };
    auto move_live = [&](int mv) {
      if (mv >= w && s_pre[mv - w] < w) return false;
      const int d = move_dst(mv);
      return d != move_src(mv) && d >= r0 && d < r0 + rows;
    };
    {
      const int cc = tid & 127;
      for (int mv = tid >> 7; mv < 2 * w; mv += 2)
        if (cc < nout && move_live(mv)) {
          const int col = cc < c0 ? cc : cc + w;
          MV[mv * 128 + cc] = __ldcg(&A[(long long)col * lda + move_src(mv)]);
        }
    }
    cluster_arrive_release();  // every source read before any row is overwritten
    cluster_wait_acquire();
    {
      const int cc = tid & 127;
      for (int mv = tid >> 7; mv < 2 * w; mv += 2)
        if (cc < nout && move_live(mv)) {
          const int col = cc < c0 ? cc : cc + w;
          A[(long long)col * lda + move_dst(mv)] = MV[mv * 128 + cc];
        }
    }
    __syncthreads();
    if (cta == 0) {
      // U12 := inv(unit lower L11_sub) * A12 on rows c0..c1-1, columns [c1, b)
      for (int c = c1 + tid; c < b; c += kSpThreads) {
        double* colp = &A[(long long)c * lda + c0];
        double u[kSpW];
#pragma unroll
        for (int i = 0; i < kSpW; ++i) u[i] = (i < w) ? __ldcg(colp + i) : 0.0;
#pragma unroll
        for (int i = 1; i < kSpW; ++i) {
          double v = u[i];
#pragma unroll
          for (int k = 0; k < kSpW; ++k)
            if (k < i) v = fma(-SP[k * R + c0 + i], u[k], v);
          u[i] = v;
        }
#pragma unroll
        for (int i = 0; i < kSpW; ++i)
          if (i < w) colp[i] = u[i];
      }
    }
    cluster_arrive_release();  // interchanges and U12 visible to the cluster
    cluster_wait_acquire();
    if (c1 < b) {
      // A[r, c1:b) -= L[r, c0:c1) * U12   for own rows r >= c1
      const int nc = b - c1;
      for (int idx = tid; idx < w * nc; idx += kSpThreads) {
        const int k = idx / nc, cc = idx - k * nc;
        UB[k * 128 + cc] = __ldcg(&A[(long long)(c1 + cc) * lda + c0 + k]);
      }
      __syncthreads();
      const int lr0 = max(0, c1 - r0);
      const int nr = rows - lr0;
      if (nr > 0) {
        const int tr = (nr + 3) / 4, tc = (nc + 3) / 4;
        for (int t = tid; t < tr * tc; t += kSpThreads) {
          const int ti = t % tr, tj = t / tr;
          const int lrb = lr0 + 4 * ti, cb = 4 * tj;
          double acc[4][4];
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[a][q] = 0.0;
          for (int k = 0; k < w; ++k) {
            double x[4], y[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) x[a] = (lrb + a < rows) ? SP[k * R + lrb + a] : 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) y[q] = (cb + q < nc) ? UB[k * 128 + cb + q] : 0.0;
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
              for (int q = 0; q < 4; ++q) acc[a][q] = fma(x[a], y[q], acc[a][q]);
          }
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (lrb + a < rows && cb + q < nc) {
                double* ap = &A[(long long)(c1 + cb + q) * lda + r0 + lrb + a];
                *ap = __ldcg(ap) - acc[a][q];
              }
        }
      }
      __syncthreads();
    }
  }
  // every CTA's trailing updates are in global memory before CTA 0 reads L11,
  // and no CTA leaves while others may still address its shared memory
  cluster_arrive_release();
  cluster_wait_acquire();
  if (cta != 0 || stop) return;
  if (tid < b) {  // ComposePivots over the whole panel
    const int i = tid;
    int k = p[i] - offset;
    for (int q = i - 1; q >= 0; --q) {
      const int pq = p[q] - offset;
      if (pq == k) k = q;
      else if (q == k) k = pq;
    }
    preimage[i] = k;
    k = i;
    for (int q = 0; q < min(k + 1, b); ++q) {
      const int pq = p[q] - offset;
      if (pq == k) k = q;
      else if (q == k) k = pq;
    }
    image[i] = k;
  }
  if (W != nullptr) {  // inv(unit lower L11) of the panel's top b x b block
    double* S = sm;
    for (int c = 0; c < b; ++c)
      for (int r = c + tid; r < b; r += kSpThreads) SE(S, r, c) = __ldcg(&A[(long long)c * lda + r]);
    __syncthreads();
    smem_trinv(S, b, 1);
    for (int c = 0; c < b; ++c)
      for (int r = tid; r < b; r += kSpThreads) W[r + (long long)c * ldw] = (r >= c) ? SE(S, r, c) : 0.0;
  }
}

static size_t cluster_panel_smem(int b, int R) {
  return sizeof(double) * ((size_t)b * R + 5 * (size_t)b) + sizeof(ClusterCand) * 32;
}

// Largest usable cluster for the panel (16 needs the non-portable opt-in and
// 16 co-schedulable SMs); 0 when clusters cannot be used.
static int panel_cluster_max() {
  static int cached = -1;
  if (cached >= 0) return cached;
  cached = 0;
  const int R = kPanelMaxRowsPerCta, b = 128;
  const size_t smem = cluster_panel_smem(b, R);
  if (cudaFuncSetAttribute(lu_panel_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return cached;
  }
  cudaFuncSetAttribute(lu_panel_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaGetLastError();
  for (int c : {16, 8}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(kPanelThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, lu_panel_cluster_kernel, &cfg) == cudaSuccess && nclusters > 0) {
      cached = c;
      break;
    }
    cudaGetLastError();
  }
  return cached;
}

int launch_lu_panel(cudaStream_t st, int m, int b, double* A, long long lda, int* p, int offset, int* image,
                    int* preimage, double* W, int ldw, void* scratch, DevStatus* status, int sm_count) {
  if (m <= 0 || b <= 0) return EGPU_OK;
  if (b > 128) return EGPU_ERR_ARG;
  {
    const int rc = launch_lu_panel_rp(st, m, b, A, lda, p, offset, image, preimage, W, ldw, status,
                                      panel_cluster_max());
    if (rc != EGPU_ERR_UNSUPPORTED) return rc;
  }
  // sub-panel cluster form: panel in global memory, 16 columns in shared memory
  {
    static int sp_ok = -1;
    if (sp_ok < 0) {
      sp_ok = 0;
      const size_t smax = sizeof(double) * sp_panel_doubles(kSpMaxR);
      if (cudaFuncSetAttribute(lu_panel_sp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax) ==
              cudaSuccess &&
          cudaFuncSetAttribute(lu_panel_sp_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
              cudaSuccess)
        sp_ok = 1;
      cudaGetLastError();
    }
    const int cmax = panel_cluster_max();
    if (sp_ok && cmax > 0) {
      // R: a multiple of 32 (16-byte cp.async of row pairs needs even R and r0)
      // and >= b (CTA 0 owns the panel's top b rows)
      int R = (std::max(b, 32) + 31) / 32 * 32;
      while ((m + R - 1) / R > cmax) R += 32;
      if (R <= kSpMaxR) {
        const int P = (m + R - 1) / R;
        TraceMark tm(st, kTracePanel, (double)m * b * b, 16.0 * m * b);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(P);
        cfg.blockDim = dim3(kSpThreads);
        cfg.dynamicSmemBytes = sizeof(double) * sp_panel_doubles(R);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = P;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaError_t e = cudaLaunchKernelEx(&cfg, lu_panel_sp_kernel, m, b, A, lda, p, offset, image, preimage,
                                           W, ldw, R, status);
        count_launch();
        if (e != cudaSuccess) {
          set_last_error(e, "lu_panel_sp launch", __FILE__, __LINE__);
          return EGPU_ERR_CUDA;
        }
        return EGPU_OK;
      }
    }
  }
  // cluster form when the panel fits in one cluster's shared memory
  const int cmax = panel_cluster_max();
  if (cmax > 0 && m <= cmax * kPanelMaxRowsPerCta) {
    int R = (std::max(b, 32) + 31) / 32 * 32;
    while ((m + R - 1) / R > cmax) R += 32;
    const int P = (m + R - 1) / R;
    TraceMark tm(st, kTracePanel, (double)m * b * b, 16.0 * m * b);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P);
    cfg.blockDim = dim3(kPanelThreads);
    cfg.dynamicSmemBytes = cluster_panel_smem(b, R);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = P;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, lu_panel_cluster_kernel, m, b, A, lda, p, offset, image, preimage, W,
                                       ldw, R, status);
    count_launch();
    if (e != cudaSuccess) {
      set_last_error(e, "lu_panel_cluster launch", __FILE__, __LINE__);
      return EGPU_ERR_CUDA;
    }
    return EGPU_OK;
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
// into perm: after the swaps, row r holds original row perm[r].
__global__ void compose_perm_kernel(int inverse, int m, const int* p, int np, int* perm) {
  for (int r = threadIdx.x; r < m; r += blockDim.x) perm[r] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    if (!inverse) {
      for (int i = 0; i < np; ++i) {
        const int k = p[i];
        const int t = perm[i]; perm[i] = perm[k]; perm[k] = t;
      }
    } else {
      for (int i = np - 1; i >= 0; --i) {
        const int k = p[i];
        const int t = perm[i]; perm[i] = perm[k]; perm[k] = t;
      }
    }
  }
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

// perm_scratch: int[m] followed by double[m * n] (8-byte aligned after m ints
// rounded up to an even count).
int launch_laswp_seq(cudaStream_t st, int inverse, int m, int n, double* A, long long lda, const int* p, int np,
                     int* perm_scratch) {
  if (m <= 0 || n <= 0 || np <= 0) return EGPU_OK;
  int* perm = perm_scratch;
  double* tmp = reinterpret_cast<double*>(perm_scratch + ((m + 1) & ~1));
  compose_perm_kernel<<<1, 1024, 0, st>>>(inverse, m, p, np, perm);
  count_launch();
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

}  // namespace egpu
