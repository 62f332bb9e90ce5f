// Register-resident LU panel (lu::Panel, lapack-like/LU/Panel.hpp:19-89).
//
// One thread-block cluster of P <= 16 CTAs of 256 threads; CTA c owns rows
// [c R, c R + R), R = RT * 256, and thread t of the CTA owns local rows
// t, t + 256, ... (RT of them).  The panel is processed in 16-column
// sub-panels; a thread keeps the 16 sub-panel entries of each of its rows in
// registers.  Registers cannot be indexed at run time, so the column loop is
// rolled and the register row is rotated by one after each column: the
// current column always sits in position 0, and after 16 rotations the
// original order is back.
//
// Per column (one __syncthreads and one cluster barrier):
//  1. each warp finds its first maximal |a| over rows >= j with three
//     redux.sync reductions (|a| as an order-preserving 64-bit key, then the
//     lowest row among equal keys), and copies the candidate's 16-entry row
//     into shared memory with shuffles;
//  2. every warp picks the CTA's candidate from the 8 warp candidates, and
//     warp w pushes it (plus row j, from the CTA that owns row j) into the
//     shared memory of CTA w and w + 8 of the cluster;
//  3. after the cluster barrier every warp picks the winner from the P
//     messages (first maximal |a|, ties to the lowest row: the reference's
//     strict '>' scan), the owners of row j and of the winner swap their
//     register rows through the messages, and every thread scales and
//     rank-1 updates its rows below j (Panel.hpp:66-80).
// After a sub-panel: the sub-panel is written back, the sub-panel's
// interchanges are applied to the panel's other columns (ComposePivots,
// ComposePivots.hpp:81-125, then row moves by the CTA that owns each
// destination row, all sources read before the cluster barrier), every CTA
// solves the 16 x (b - c1) block U12 = inv(L11) A12 itself (CTA 0 stores it),
// and updates its rows of the remaining panel columns,
// A[r, c1:b) -= L[r, c0:c1) U12.  The result equals lu::Panel's: the same
// pivots, and the panel's trailing columns updated in 16-column blocks.
#include "diag_common.cuh"
#include "internal.h"

namespace egpu {

namespace {

constexpr int kRpThreads = 256;
constexpr int kRpW = 16;         // sub-panel width
constexpr int kRpMsg = 18;       // double2 per message: header, candidate row (8), row j (8)
constexpr int kRpMaxCl = 16;
constexpr int kRpNoRow = 0x7fffffff;

// shared-memory layout (in doubles)
constexpr int kRpOffMsg = 0;                                  // [2][kRpMaxCl][kRpMsg] double2
constexpr int kRpOffCand = kRpOffMsg + 2 * kRpMaxCl * kRpMsg * 2;  // [8 warps][9] double2
constexpr int kRpOffRowJ = kRpOffCand + 8 * 9 * 2;            // [8] double2
constexpr int kRpOffL11 = kRpOffRowJ + 8 * 2;                 // 16 x 16 (ld 17)
constexpr int kRpOffU12 = kRpOffL11 + 16 * 17;                // [16][128]
constexpr int kRpOffMv = kRpOffU12 + 16 * 128;                // [2 * 16][128] row moves
constexpr int kRpWorkDoubles = kRpOffMv + 2 * kRpW * 128;
constexpr int kRpInvDoubles = 128 * kLDS + 128 + kDiagTmpDoubles;  // final inv(L11)
constexpr int kRpSmemDoubles = kRpWorkDoubles > kRpInvDoubles ? kRpWorkDoubles : kRpInvDoubles;

// first maximal key over the warp, ties to the lowest row (all lanes get it)
__device__ __forceinline__ void warp_argmax_key(unsigned long long key, int row, unsigned long long& wkey,
                                                int& wrow) {
  const unsigned hi = __reduce_max_sync(0xffffffffu, (unsigned)(key >> 32));
  const unsigned lo = __reduce_max_sync(0xffffffffu, (unsigned)(key >> 32) == hi ? (unsigned)key : 0u);
  wkey = ((unsigned long long)hi << 32) | lo;
  const unsigned r = __reduce_min_sync(0xffffffffu, key == wkey ? (unsigned)row : (unsigned)kRpNoRow);
  wrow = (int)r;
}

// |a| as a key whose unsigned order is the order of |a| (non-negative doubles)
__device__ __forceinline__ unsigned long long abs_key(double v) {
  return (unsigned long long)__double_as_longlong(fabs(v));
}

template <int RT>
__device__ __forceinline__ void rotate_rows(double (&v)[RT][kRpW]) {
#pragma unroll
  for (int s = 0; s < RT; ++s) {
    const double t0 = v[s][0];
#pragma unroll
    for (int k = 0; k < kRpW - 1; ++k) v[s][k] = v[s][k + 1];
    v[s][kRpW - 1] = t0;
  }
}

}  // namespace

template <int RT>
__global__ void __launch_bounds__(kRpThreads, 1) lu_panel_rp_kernel(int m, int b, double* A, long long lda, int* p,
                                                                     int offset, int* image, int* preimage,
                                                                     double* W, int ldw, DevStatus* st) {
  constexpr int R = RT * kRpThreads;
  extern __shared__ double sm[];
  double2* MSG = reinterpret_cast<double2*>(sm + kRpOffMsg);
  double2* CAND = reinterpret_cast<double2*>(sm + kRpOffCand);
  double2* ROWJ = reinterpret_cast<double2*>(sm + kRpOffRowJ);
  double* L11 = sm + kRpOffL11;
  double* U12 = sm + kRpOffU12;
  double* MV = sm + kRpOffMv;
  __shared__ int s_piv[128], s_img[kRpW], s_pre[kRpW];
  __shared__ int s_skip;

  const int P = gridDim.x;
  const unsigned cta = cluster_ctarank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = (int)cta * R;
  const int rows = max(0, min(R, m - r0));

  // a failed earlier step: every CTA takes CTA 0's reading of the status
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
  double v[RT][kRpW];
  for (int c0 = 0; c0 < ncols && !stop; c0 += kRpW) {
    const int c1 = min(ncols, c0 + kRpW), w = c1 - c0;
    // ---- load the sub-panel rows into registers (own rows; .cg: no stale L1)
#pragma unroll
    for (int s = 0; s < RT; ++s) {
      const int lr = s * kRpThreads + tid;
#pragma unroll
      for (int k = 0; k < kRpW; ++k)
        v[s][k] = (lr < rows && k < w) ? __ldcg(&A[(long long)(c0 + k) * lda + r0 + lr]) : 0.0;
    }
    // ---- column loop
    for (int t = 0; t < w; ++t) {
      const int j = c0 + t, par = j & 1;
      // 1. warp candidate
      unsigned long long key = 0ull;
      int krow = kRpNoRow;
#pragma unroll
      for (int s = 0; s < RT; ++s) {
        const int lr = s * kRpThreads + tid, r = r0 + lr;
        if (lr < rows && r >= j) {
          const unsigned long long kk = abs_key(v[s][0]);
          if (krow == kRpNoRow || kk > key) { key = kk; krow = r; }  // slots ascend in row
        }
      }
      unsigned long long wkey;
      int wrow;
      warp_argmax_key(key, krow, wkey, wrow);
      if (wrow != kRpNoRow) {
        const int wl = (wrow - r0) & 31, ws = (wrow - r0) / kRpThreads;
        double2 pc = make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < kRpW; ++k) {
          double mine = v[0][k];
#pragma unroll
          for (int s = 1; s < RT; ++s)
            if (ws == s) mine = v[s][k];
          const double x = __shfl_sync(0xffffffffu, mine, wl);
          if (lane == (k >> 1)) {
            if (k & 1) pc.y = x;
            else pc.x = x;
          }
        }
        if (lane < 8) CAND[warp * 9 + 1 + lane] = pc;
      }
      if (lane == 8) CAND[warp * 9] = make_double2(__longlong_as_double((long long)wkey), (double)wrow);
      // row j's owner stages it for the message
      if (j >= r0 && j < r0 + rows && ((j - r0) & (kRpThreads - 1)) == tid) {
        const int sj = (j - r0) / kRpThreads;
#pragma unroll
        for (int s = 0; s < RT; ++s)
          if (s == sj)
#pragma unroll
            for (int q = 0; q < 8; ++q) ROWJ[q] = make_double2(v[s][2 * q], v[s][2 * q + 1]);
      }
      __syncthreads();
      // 2. CTA candidate (every warp), pushed by warp w to CTAs w and w + 8
      {
        unsigned long long ck = 0ull;
        int crow = kRpNoRow;
        if (lane < 8) {
          const double2 h = CAND[lane * 9];
          ck = (unsigned long long)__double_as_longlong(h.x);
          crow = (int)h.y;
        }
        unsigned long long bk;
        int brow;
        warp_argmax_key(ck, crow, bk, brow);
        const unsigned cw = __ballot_sync(0xffffffffu, lane < 8 && crow == brow && ck == bk);
        const int wsrc = cw ? __ffs(cw) - 1 : 0;
        const bool ownj = (j >= r0 && j < r0 + rows);
        double2 mv = make_double2(0.0, 0.0);
        if (lane == 0) mv = make_double2(__longlong_as_double((long long)bk), (double)brow);
        else if (lane < 9) mv = CAND[wsrc * 9 + lane];
        else if (lane >= 10 && lane < 18 && ownj) mv = ROWJ[lane - 10];
        const bool send = (lane < 9) || (ownj && lane >= 10 && lane < 18);
        if (send) {
          double2* slot = &MSG[(par * kRpMaxCl + cta) * kRpMsg + lane];
          for (int dst = warp; dst < P; dst += 8) *cluster_map(slot, (unsigned)dst) = mv;
        }
      }
      cluster_arrive_release();
      cluster_wait_acquire();
      // 3. winner over the P messages
      unsigned long long gk = 0ull;
      int grow = kRpNoRow;
      if (lane < P) {
        const double2 h = MSG[(par * kRpMaxCl + lane) * kRpMsg];
        gk = (unsigned long long)__double_as_longlong(h.x);
        grow = (int)h.y;
      }
      unsigned long long wk;
      int wr;
      warp_argmax_key(gk, grow, wk, wr);
      const unsigned cm = __ballot_sync(0xffffffffu, lane < P && grow == wr && gk == wk);
      const int wc = cm ? __ffs(cm) - 1 : 0;
      const double2* wmsg = &MSG[(par * kRpMaxCl + wc) * kRpMsg + 1];          // winner row
      const double2* jmsg = &MSG[(par * kRpMaxCl + j / R) * kRpMsg + 10];      // row j
      const double wv = wmsg[0].x;
      if (wr == kRpNoRow || wv == 0.0) {  // exact zero pivot: SingularMatrixException (Panel.hpp:76-77)
        if (cta == 0 && tid == 0) set_status(st, kSingular, offset + j + 1);
        stop = true;
        break;
      }
      if (tid == 0) s_piv[j] = wr;
      if (cta == 0 && tid == 0) p[j] = wr + offset;
      // row interchange inside the sub-panel (Panel.hpp:66-72)
      if (wr != j) {
#pragma unroll
        for (int s = 0; s < RT; ++s) {
          const int r = r0 + s * kRpThreads + tid;
          if (r == j) {
#pragma unroll
            for (int q = 0; q < 8; ++q) { const double2 x = wmsg[q]; v[s][2 * q] = x.x; v[s][2 * q + 1] = x.y; }
          } else if (r == wr) {
#pragma unroll
            for (int q = 0; q < 8; ++q) { const double2 x = jmsg[q]; v[s][2 * q] = x.x; v[s][2 * q + 1] = x.y; }
          }
        }
      }
      // scale (Panel.hpp:78-79) and rank-1 update (Geru, :80) of own rows > j
      const double inv = 1.0 / wv;
      const int kmax = w - t;  // positions 1 .. kmax-1 are the sub-panel's unprocessed columns
#pragma unroll
      for (int s = 0; s < RT; ++s) {
        const int lr = s * kRpThreads + tid, r = r0 + lr;
        if (lr < rows && r > j) {
          const double l = v[s][0] * inv;
          v[s][0] = l;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const double2 u = wmsg[q];
            if (2 * q > 0 && 2 * q < kmax) v[s][2 * q] = fma(-l, u.x, v[s][2 * q]);
            if (2 * q + 1 < kmax) v[s][2 * q + 1] = fma(-l, u.y, v[s][2 * q + 1]);
          }
        }
      }
      rotate_rows<RT>(v);
    }
    if (stop) break;
    for (int t = w; t < kRpW; ++t) rotate_rows<RT>(v);  // back to column order
    // ---- write the sub-panel back (own rows)
#pragma unroll
    for (int s = 0; s < RT; ++s) {
      const int lr = s * kRpThreads + tid;
      if (lr < rows)
#pragma unroll
        for (int k = 0; k < kRpW; ++k)
          if (k < w) A[(long long)(c0 + k) * lda + r0 + lr] = v[s][k];
    }
    __syncthreads();  // s_piv of the sub-panel's last column
    // ---- ComposePivots (ComposePivots.hpp:81-125) of the sub-panel, relative to row c0
    if (tid < w) {
      const int i = tid;
      int k = s_piv[c0 + i] - c0;
      for (int q = i - 1; q >= 0; --q) {
        const int pq = s_piv[c0 + q] - c0;
        if (pq == k) k = q;
        else if (q == k) k = pq;
      }
      s_pre[i] = k;
      k = i;
      for (int q = 0; q < min(k + 1, w); ++q) {
        const int pq = s_piv[c0 + q] - c0;
        if (pq == k) k = q;
        else if (q == k) k = pq;
      }
      s_img[i] = k;
    }
    __syncthreads();
    // Row moves on the panel's other columns [0, c0) and [c1, b):
    // move mv < w: row c0+mv -> c0+img[mv]; move w+i: row c0+pre[i] -> c0+i (pre[i] >= w).
    // Rows c0..c1-1 of columns [c1, b) become U12 and are not moved; U12's
    // input row i is the old row c0+pre[i].
    const int nout = b - w;
    auto move_src = [&](int mv) { return mv < w ? c0 + mv : c0 + s_pre[mv - w]; };
    auto move_dst = [&](int mv) { return mv < w ? c0 + s_img[mv] : c0 + (mv - w); };
    auto move_live = [&](int mv) {
      if (mv >= w && s_pre[mv - w] < w) return false;
      const int d = move_dst(mv);
      return d != move_src(mv) && d >= r0 && d < r0 + rows;
    };
    const int ntr = b - c1;  // trailing panel columns
    {
      // all of a thread's gathers are issued before any is stored, so their
      // L2 latencies overlap
      const int cc = tid & 127;
      double g[kRpW];
#pragma unroll
      for (int q = 0; q < kRpW; ++q) {
        const int mv = 2 * q + (tid >> 7);
        g[q] = 0.0;
        if (mv < 2 * w && cc < nout && move_live(mv)) {
          const int col = cc < c0 ? cc : cc + w;
          const int d = move_dst(mv);
          if (!(col >= c1 && d < c1)) g[q] = __ldcg(&A[(long long)col * lda + move_src(mv)]);
        }
      }
      double gu[kRpW * 128 / kRpThreads];
#pragma unroll
      for (int q = 0; q < kRpW * 128 / kRpThreads; ++q) {
        const int idx = tid + q * kRpThreads, i = idx >> 7, c = idx & 127;
        gu[q] = (i < w && c < ntr) ? __ldcg(&A[(long long)(c1 + c) * lda + c0 + s_pre[i]]) : 0.0;
      }
#pragma unroll
      for (int q = 0; q < kRpW; ++q) {
        const int mv = 2 * q + (tid >> 7);
        if (mv < 2 * w && cc < nout && move_live(mv)) {
          const int col = cc < c0 ? cc : cc + w;
          const int d = move_dst(mv);
          if (!(col >= c1 && d < c1)) MV[mv * 128 + cc] = g[q];
        }
      }
#pragma unroll
      for (int q = 0; q < kRpW * 128 / kRpThreads; ++q) {
        const int idx = tid + q * kRpThreads, i = idx >> 7, c = idx & 127;
        if (i < w && c < ntr) U12[i * 128 + c] = gu[q];
      }
    }
    // every source read (and CTA 0's sub-panel, with L11, written) cluster-wide
    cluster_arrive_release();
    cluster_wait_acquire();
    {
      const int cc = tid & 127;
      for (int mv = tid >> 7; mv < 2 * w; mv += 2)
        if (cc < nout && move_live(mv)) {
          const int col = cc < c0 ? cc : cc + w;
          const int d = move_dst(mv);
          if (!(col >= c1 && d < c1)) A[(long long)col * lda + d] = MV[mv * 128 + cc];
        }
    }
    if (ntr > 0) {
      // L11 of the sub-panel (unit lower, rows/cols c0..c1-1), written by its owner before the barrier
      for (int idx = tid; idx < w * w; idx += kRpThreads) {
        const int i = idx % w, k = idx / w;
        L11[i + k * 17] = __ldcg(&A[(long long)(c0 + k) * lda + c0 + i]);
      }
      __syncthreads();
      // U12 := inv(unit lower L11) A12, one column per thread, in shared memory
      for (int cc = tid; cc < ntr; cc += kRpThreads) {
        double u[kRpW];
#pragma unroll
        for (int i = 0; i < kRpW; ++i) u[i] = (i < w) ? U12[i * 128 + cc] : 0.0;
#pragma unroll
        for (int i = 1; i < kRpW; ++i) {
          double x = u[i];
#pragma unroll
          for (int k = 0; k < kRpW; ++k)
            if (k < i && i < w) x = fma(-L11[i + k * 17], u[k], x);
          u[i] = x;
        }
#pragma unroll
        for (int i = 0; i < kRpW; ++i)
          if (i < w) {
            U12[i * 128 + cc] = u[i];
            if (cta == 0) A[(long long)(c1 + cc) * lda + c0 + i] = u[i];
          }
      }
      __syncthreads();
      // A[r, c1:b) -= L[r, c0:c1) U12 for own rows r >= c1 (L in registers),
      // kB columns at a time: every load of a batch is in flight before the
      // first multiply
      constexpr int kB = RT >= 4 ? 4 : 8;
      for (int cb = 0; cb < ntr; cb += kB) {
        double x[RT][kB];
#pragma unroll
        for (int s = 0; s < RT; ++s) {
          const int lr = s * kRpThreads + tid, r = r0 + lr;
#pragma unroll
          for (int q = 0; q < kB; ++q)
            x[s][q] = (lr < rows && r >= c1 && cb + q < ntr) ? __ldcg(&A[(long long)(c1 + cb + q) * lda + r]) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < kB; ++q) {
          if (cb + q < ntr) {
#pragma unroll
            for (int k = 0; k < kRpW; ++k) {
              const double u = k < w ? U12[k * 128 + cb + q] : 0.0;
#pragma unroll
              for (int s = 0; s < RT; ++s) x[s][q] = fma(-v[s][k], u, x[s][q]);
            }
          }
        }
#pragma unroll
        for (int s = 0; s < RT; ++s) {
          const int lr = s * kRpThreads + tid, r = r0 + lr;
#pragma unroll
          for (int q = 0; q < kB; ++q)
            if (lr < rows && r >= c1 && cb + q < ntr) A[(long long)(c1 + cb + q) * lda + r] = x[s][q];
        }
      }
    }
    __syncthreads();
  }
  // all CTAs done with each other's shared memory and with the panel
  cluster_arrive_release();
  cluster_wait_acquire();
  if (cta != 0 || stop) return;
  if (tid < ncols) {  // ComposePivots over the whole panel
    const int i = tid;
    int k = s_piv[i];
    for (int q = i - 1; q >= 0; --q) {
      const int pq = s_piv[q];
      if (pq == k) k = q;
      else if (q == k) k = pq;
    }
    preimage[i] = k;
    k = i;
    for (int q = 0; q < min(k + 1, ncols); ++q) {
      const int pq = s_piv[q];
      if (pq == k) k = q;
      else if (q == k) k = pq;
    }
    image[i] = k;
  }
  if (W != nullptr) {  // inv(unit lower L11) of the panel's top b x b block
    const int bb = ncols;
    double* S = sm;
    for (int e = tid; e < bb * bb; e += kRpThreads) {  // .cg: rows written by this CTA's other threads
      const int r = e % bb, c = e / bb;
      if (r >= c) SE(S, r, c) = __ldcg(&A[(long long)c * lda + r]);
    }
    __syncthreads();
    double* Xl = S + 128 * kLDS + 128;
    double* T = Xl + 8 * 16 * kLeafLD;
    const int bp = pad16_identity(S, bb);
    __syncthreads();
    for (int q = warp; q < bp / 16; q += kRpThreads / 32) warp_trinv16(S, kLDS, 16 * q, 1, Xl + q * 16 * kLeafLD, kLeafLD);
    __syncthreads();
    smem_trinv_dmma(S, bp, Xl, T);
    for (int e = tid; e < bb * bb; e += kRpThreads) {
      const int r = e % bb, c = e / bb;
      W[r + (long long)c * ldw] = (r > c) ? SE(S, r, c) : (r == c ? 1.0 : 0.0);
    }
  }
}

// Launch the register-resident panel when m fits one cluster (m <= 16 * 1024
// rows with a 16-CTA cluster) and b <= 128.  Returns EGPU_ERR_UNSUPPORTED when it does not apply.
int launch_lu_panel_rp(cudaStream_t st, int m, int b, double* A, long long lda, int* p, int offset, int* image,
                       int* preimage, double* W, int ldw, DevStatus* status, int cluster_max) {
  if (b > 128 || b < 1 || cluster_max < 1) return EGPU_ERR_UNSUPPORTED;
  const size_t smem = sizeof(double) * kRpSmemDoubles;
  static int cl_max[3] = {-1, -1, -1};  // per RT: largest cluster the kernel can be scheduled with
  auto kern_of = [](int rt) {
    return rt == 1 ? lu_panel_rp_kernel<1> : (rt == 2 ? lu_panel_rp_kernel<2> : lu_panel_rp_kernel<4>);
  };
  int RT = 0, P = 0;
  for (int ai = 0; ai < 3 && RT == 0; ++ai) {  // fewest rows per thread that fit one cluster
    const int rt = 1 << ai;
    if (cl_max[ai] < 0) {
      cl_max[ai] = 0;
      auto kern = kern_of(rt);
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
          cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
        for (int c : {16, 8}) {
          cudaLaunchConfig_t cfg = {};
          cfg.gridDim = dim3(c);
          cfg.blockDim = dim3(kRpThreads);
          cfg.dynamicSmemBytes = smem;
          cudaLaunchAttribute attr[1];
          attr[0].id = cudaLaunchAttributeClusterDimension;
          attr[0].val.clusterDim.x = c;
          attr[0].val.clusterDim.y = 1;
          attr[0].val.clusterDim.z = 1;
          cfg.attrs = attr;
          cfg.numAttrs = 1;
          int ncl = 0;
          if (cudaOccupancyMaxActiveClusters(&ncl, kern, &cfg) == cudaSuccess && ncl > 0) {
            cl_max[ai] = c;
            break;
          }
        }
      }
      cudaGetLastError();
    }
    const int cmax = std::min(cl_max[ai], cluster_max > 0 ? kRpMaxCl : 0);
    const int pp = (m + rt * kRpThreads - 1) / (rt * kRpThreads);
    if (cmax > 0 && pp <= cmax) { RT = rt; P = pp; }
  }
  if (RT == 0) return EGPU_ERR_UNSUPPORTED;
  auto kern = kern_of(RT);
  TraceMark tm(st, kTracePanel, (double)m * b * b, 16.0 * m * b);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P);
  cfg.blockDim = dim3(kRpThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = P;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, kern, m, b, A, lda, p, offset, image, preimage, W, ldw, status);
  count_launch();
  if (e != cudaSuccess) {
    set_last_error(e, "lu_panel_rp launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

}  // namespace egpu
