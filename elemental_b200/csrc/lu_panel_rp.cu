// Register-resident LU panel (lu::Panel, lapack-like/LU/Panel.hpp:19-89).
//
// One thread-block cluster of P <= 16 CTAs of 256 threads; CTA c owns rows
// [c R, c R + R), R = RT * 256, and thread t of the CTA owns local rows
// t, t + 256, ... (RT of them).  The panel is processed in 16-column
// sub-panels; a thread keeps the 16 sub-panel entries of each of its rows in
// registers.  Registers cannot be indexed at run time, so the 16-column loop
// is unrolled: column t of the sub-panel is register t, and the rank-1 update
// of column t touches registers t + 1 .. 15 only.
//
// Per column (one __syncthreads and one local mbarrier wait):
//  1. each warp finds its first maximal |a| over rows >= j with three
//     redux.sync reductions (|a| as an order-preserving 64-bit key, then the
//     lowest row among equal keys); the lane that owns the candidate stages
//     its 16-entry row and the reciprocal of its pivot in shared memory;
//  2. warps 0 and 1 pick the CTA's candidate from the 8 warp candidates and
//     store the message (candidate, its row, its reciprocal, and row j from
//     the CTA that owns row j) into every CTA's shared memory with
//     asynchronous stores (st.async), four lanes per destination, counted in
//     bytes on the destination's mbarrier for this column (each CTA arms its
//     own mbarrier with the column's byte count);
//  3. every thread waits (bounded) on its own CTA's mbarrier, picks the winner
//     from the P messages (first maximal |a|, ties to the lowest row: the
//     reference's strict '>' scan), the owners of row j and of the winner swap
//     their register rows through the messages, and every thread scales
//     (by the sender's 1/pivot, Panel.hpp:78-79) and rank-1 updates its rows
//     below j (Panel.hpp:80).
// The message buffers alternate between two slots by column parity: a CTA
// writes slot s for column j + 2 only after it has received every CTA's
// column j + 1 message, which each CTA sends after all its threads are done
// with column j's slot, and a CTA re-arms slot s for column j + 2 before it
// sends column j + 1.  Stopping (an exact zero pivot, seen by every CTA in
// the same column, or a wait that ran out, which is broadcast to every CTA)
// is made CTA-uniform at the next __syncthreads_or, and every CTA executes
// the same number of cluster barriers (one per sub-panel, one at the end)
// whatever happens, so a stop cannot strand a CTA at a barrier.
// After a sub-panel: the sub-panel is written back, the sub-panel's
// interchanges are applied to the panel's other columns (ComposePivots,
// ComposePivots.hpp:81-125, then row moves by the CTA that owns each
// destination row, all sources read before the cluster barrier), every CTA
// solves the 16 x (b - c1) block U12 = inv(L11) A12 itself (CTA 0 stores it;
// L11 is captured from the pivot rows as they arrive), and updates its rows of
// the remaining panel columns, A[r, c1:b) -= L[r, c0:c1) U12.  The result
// equals lu::Panel's: the same pivots, and the panel's trailing columns
// updated in 16-column blocks.  Last, CTA 0 forms inv(unit lower L11) of the
// panel's top block (16 x 16 diagonal-block inverses, then DMMA doubling).
#include "diag_common.cuh"
#include "internal.h"

namespace egpu {

namespace {

constexpr int kRpThreads = 256;
constexpr int kRpW = 16;         // sub-panel width
constexpr int kRpCandU = 10;     // double2 per candidate: header, 1/pivot, candidate row (8)
constexpr int kRpMsg = 18;       // double2 per message: a candidate, then row j (8)
constexpr int kRpMaxCl = 16;
constexpr int kRpNoRow = 0x7fffffff;

// shared-memory layout (in doubles)
constexpr int kRpOffMsg = 0;                                        // [2][kRpMaxCl][kRpMsg] double2
constexpr int kRpOffCand = kRpOffMsg + 2 * kRpMaxCl * kRpMsg * 2;   // [2][8 warps][kRpCandU] double2 (staging)
constexpr int kRpOffRowJ = kRpOffCand + 2 * 8 * kRpCandU * 2;       // [2][8] double2 (staging)
constexpr int kRpOffL11 = kRpOffRowJ + 2 * 8 * 2;                   // 16 x 16 (ld 17)
constexpr int kRpOffU12 = kRpOffL11 + 16 * 17;                      // [16][128]
constexpr int kRpOffMv = kRpOffU12 + 16 * 128;                      // [2 * 16][128] row moves
constexpr int kRpWorkDoubles = kRpOffMv + 2 * kRpW * 128;
constexpr int kRpInvDoubles = 128 * kLDS + 128 + kDiagTmpDoubles;  // the final inv(L11)
constexpr int kRpSmemDoubles = kRpWorkDoubles > kRpInvDoubles ? kRpWorkDoubles : kRpInvDoubles;
constexpr uint32_t kRpColBytes(int P) { return (uint32_t)(P * kRpCandU * 16 + 8 * 16); }

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

// 32-bit shared::cluster address of the same object in CTA `rank`
__device__ __forceinline__ uint32_t map_rank(const void* p, unsigned rank) {
  uint32_t out;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(smem_u32(p)), "r"(rank));
  return out;
}
__device__ __forceinline__ void st_cluster(uint32_t addr, int v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
// asynchronous 16-byte store into another CTA of the cluster, counted (bytes)
// on the mbarrier `bar` of that CTA
__device__ __forceinline__ void st_async(uint32_t addr, double2 v, uint32_t bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(addr),
               "d"(v.x), "d"(v.y), "r"(bar)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

}  // namespace

template <int RT>
__global__ void __launch_bounds__(kRpThreads, 1) lu_panel_rp_kernel(int m, int b, double* A, long long lda, int* p,
                                                                     int offset, int* image, int* preimage,
                                                                     double* W, int ldw, DevStatus* st) {
  constexpr int R = RT * kRpThreads;
  extern __shared__ double sm[];
  double2* MSG = reinterpret_cast<double2*>(sm + kRpOffMsg);
  double2* CANDB = reinterpret_cast<double2*>(sm + kRpOffCand);
  double2* ROWJB = reinterpret_cast<double2*>(sm + kRpOffRowJ);
  double* L11 = sm + kRpOffL11;
  double* U12 = sm + kRpOffU12;
  double* MV = sm + kRpOffMv;
  __shared__ int s_piv[128], s_pre[kRpW];
  __shared__ int s_msrc[2 * kRpW], s_mdst[2 * kRpW];  // the sub-panel's row moves (dst -1: none here)
  __shared__ int s_skip, s_abort;
  __shared__ __align__(8) uint64_t s_bar[2];

  const int P = gridDim.x;
  const unsigned cta = cluster_ctarank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = (int)cta * R;
  const int rows = max(0, min(R, m - r0));

  // a failed earlier step: every CTA takes CTA 0's reading of the status
  if (tid == 0) {
    s_skip = (st != nullptr && ((volatile DevStatus*)st)->code != 0);
    s_abort = 0;
    // one phase per column: this CTA's arrival with the byte count of every
    // CTA's candidate, plus row j
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
    mbar_expect_tx(&s_bar[0], kRpColBytes(P));
    mbar_expect_tx(&s_bar[1], kRpColBytes(P));
  }
  __syncthreads();
  cluster_arrive_release();
  cluster_wait_acquire();
  const int skip = *cluster_map(&s_skip, 0u);
  cluster_arrive_release();
  cluster_wait_acquire();
  if (skip) return;

  const int ncols = min(b, m);
  bool stop = false;  // CTA-uniform
  int lstop = 0;      // this thread saw a zero pivot or a wait that ran out
  bool abort_sent = false;
  double v[RT][kRpW];
  for (int c0 = 0; c0 < ncols; c0 += kRpW) {
    const int c1 = min(ncols, c0 + kRpW), w = c1 - c0;
    if (!stop) {
      // ---- load the sub-panel rows into registers (own rows; .cg: no stale L1)
#pragma unroll
      for (int s = 0; s < RT; ++s) {
        const int lr = s * kRpThreads + tid;
#pragma unroll
        for (int k = 0; k < kRpW; ++k)
          v[s][k] = (lr < rows && k < w) ? __ldcg(&A[(long long)(c0 + k) * lda + r0 + lr]) : 0.0;
      }
      // ---- column loop (unrolled: column t of the sub-panel is register t)
#pragma unroll
      for (int t = 0; t < kRpW; ++t) {
        if (t >= w) break;
        const int j = c0 + t, par = j & 1;
        const uint32_t phase = (uint32_t)(j >> 1) & 1u;
        double2* CAND = CANDB + par * 8 * kRpCandU;
        double2* ROWJ = ROWJB + par * 8;
        // 1. warp candidate; its owner stages the row and 1/pivot
        unsigned long long key = 0ull;
        int krow = kRpNoRow;
#pragma unroll
        for (int s = 0; s < RT; ++s) {
          const int lr = s * kRpThreads + tid, r = r0 + lr;
          if (lr < rows && r >= j) {
            const unsigned long long kk = abs_key(v[s][t]);
            if (krow == kRpNoRow || kk > key) { key = kk; krow = r; }  // slots ascend in row
          }
        }
        unsigned long long wkey;
        int wrow;
        warp_argmax_key(key, krow, wkey, wrow);
        double2* cw = &CAND[warp * kRpCandU];
        if (wrow == kRpNoRow) {
          if (lane == 0) cw[0] = make_double2(0.0, (double)kRpNoRow);
        } else {
#pragma unroll
          for (int s = 0; s < RT; ++s)
            if (r0 + s * kRpThreads + tid == wrow) {
              cw[0] = make_double2(__longlong_as_double((long long)wkey), (double)wrow);
              cw[1] = make_double2(__drcp_rn(v[s][t]), 0.0);  // the correctly rounded 1 / pivot
#pragma unroll
              for (int q = 0; q < 8; ++q) cw[2 + q] = make_double2(v[s][2 * q], v[s][2 * q + 1]);
            }
        }
        // row j's owner stages it for the message
        const bool ownj = j >= r0 && j < r0 + rows;
        if (ownj && ((j - r0) & (kRpThreads - 1)) == tid) {
          const int sj = (j - r0) / kRpThreads;
#pragma unroll
          for (int s = 0; s < RT; ++s)
            if (s == sj)
#pragma unroll
              for (int q = 0; q < 8; ++q) ROWJ[q] = make_double2(v[s][2 * q], v[s][2 * q + 1]);
        }
        if (__syncthreads_or(lstop)) {
          stop = true;
          break;
        }
        // 2. CTA candidate; lane L of warps 0-1 stores units L%4, L%4 + 4, ...
        //    of the message into CTA L/4 (asynchronous stores counted on that
        //    CTA's mbarrier for this column)
        if (warp < 2) {
          unsigned long long ck = 0ull;
          int crow = kRpNoRow;
          if (lane < 8) {
            const double2 h = CAND[lane * kRpCandU];
            ck = (unsigned long long)__double_as_longlong(h.x);
            crow = (int)h.y;
          }
          unsigned long long bk;
          int brow;
          warp_argmax_key(ck, crow, bk, brow);
          const unsigned cwm = __ballot_sync(0xffffffffu, lane < 8 && crow == brow && ck == bk);
          const int wsrc = cwm ? __ffs(cwm) - 1 : 0;
          const int nunits = ownj ? kRpMsg : kRpCandU;
          const int L = warp * 32 + lane, d = L >> 2;
          if (d < P) {
            const uint32_t dst = map_rank(&MSG[(par * kRpMaxCl + (int)cta) * kRpMsg], (unsigned)d);
            const uint32_t bar = map_rank(&s_bar[par], (unsigned)d);
            for (int u = L & 3; u < nunits; u += 4)
              st_async(dst + 16u * (uint32_t)u, u < kRpCandU ? CAND[wsrc * kRpCandU + u] : ROWJ[u - kRpCandU], bar);
          }
        }
        // 3. every CTA's message (bounded wait; a wait that runs out stops the cluster)
        {
          bool got = false;
          for (long long it = 0; it < kSpinLimit; ++it) {
            if (mbar_try_wait_cluster(&s_bar[par], phase)) {
              got = true;
              break;
            }
            if (*(volatile int*)&s_abort) break;
            if (it > 64) __nanosleep(64);
          }
          // re-arm this slot for column j + 2: no CTA can send that column
          // before every CTA has sent column j + 1, which this CTA does after this
          if (got && tid == 0) mbar_expect_tx(&s_bar[par], kRpColBytes(P));
          if (!got) {
            lstop = 1;
            if (!abort_sent) {
              abort_sent = true;
              set_status(st, kTimeout, 41);
              for (int d = 0; d < P; ++d) st_cluster(map_rank(&s_abort, (unsigned)d), 1);
            }
          }
        }
        if (!lstop) {
          // winner over the P messages (first maximal |a|, lowest row on ties)
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
          const double2* wm = &MSG[(par * kRpMaxCl + wc) * kRpMsg];
          const double2* wmsg = wm + 2;                                               // winner row
          const double2* jmsg = &MSG[(par * kRpMaxCl + j / R) * kRpMsg + kRpCandU];   // row j
          const double2 pv = wmsg[t / 2];
          const double wv = (t & 1) ? pv.y : pv.x;  // the pivot
          if (wr == kRpNoRow || wv == 0.0) {  // exact zero pivot: SingularMatrixException (Panel.hpp:76-77)
            if (cta == 0 && tid == 0) set_status(st, kSingular, offset + j + 1);
            lstop = 1;
          } else {
            if (tid == 0) s_piv[j] = wr;
            if (cta == 0 && tid == 0) p[j] = wr + offset;
            // the pivot row is final: its entries left of t are row t of L11
            if (tid == 32) {
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                const double2 x = wmsg[q];
                if (2 * q < t) L11[t + (2 * q) * 17] = x.x;
                if (2 * q + 1 < t) L11[t + (2 * q + 1) * 17] = x.y;
              }
            }
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
            double u[kRpW];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              const double2 x = wmsg[q];
              u[2 * q] = x.x;
              u[2 * q + 1] = x.y;
            }
            // scale (Panel.hpp:78-79) and rank-1 update (Geru, :80) of own rows > j
            const double inv = wm[1].x;
#pragma unroll
            for (int s = 0; s < RT; ++s) {
              const int lr = s * kRpThreads + tid, r = r0 + lr;
              if (lr < rows && r > j) {
                const double l = v[s][t] * inv;
                v[s][t] = l;
#pragma unroll
                for (int k = t + 1; k < kRpW; ++k) v[s][k] = fma(-l, u[k], v[s][k]);
              }
            }
          }
        }
      }
    }
    stop = __syncthreads_or(stop || lstop);
    if (!stop) {
      // ---- write the sub-panel back (own rows)
#pragma unroll
      for (int s = 0; s < RT; ++s) {
        const int lr = s * kRpThreads + tid;
        if (lr < rows)
#pragma unroll
          for (int k = 0; k < kRpW; ++k)
            if (k < w) A[(long long)(c0 + k) * lda + r0 + lr] = v[s][k];
      }
    }
    // ---- ComposePivots (ComposePivots.hpp:81-125) of the sub-panel, relative
    // to row c0, and the row moves it implies: move i takes row c0+i to
    // c0+img[i]; move w+i takes row c0+pre[i] to c0+i when pre[i] >= w (a row
    // from below the sub-panel).  A move is kept when this CTA owns its
    // destination.
    if (!stop && tid < w) {
      const int i = tid;
      int k = s_piv[c0 + i] - c0;
      for (int q = i - 1; q >= 0; --q) {
        const int pq = s_piv[c0 + q] - c0;
        if (pq == k) k = q;
        else if (q == k) k = pq;
      }
      const int pre = k;
      k = i;
      for (int q = 0; q < min(k + 1, w); ++q) {
        const int pq = s_piv[c0 + q] - c0;
        if (pq == k) k = q;
        else if (q == k) k = pq;
      }
      const int img = k;
      s_pre[i] = pre;
      int src = c0 + i, d = c0 + img;
      s_msrc[i] = src;
      s_mdst[i] = (d != src && d >= r0 && d < r0 + rows) ? d : -1;
      src = c0 + pre;
      d = c0 + i;
      s_msrc[w + i] = src;
      s_mdst[w + i] = (pre >= w && d != src && d >= r0 && d < r0 + rows) ? d : -1;
    }
    __syncthreads();
    // The moves apply to the panel's other columns [0, c0) and [c1, b); rows
    // c0..c1-1 of columns [c1, b) become U12 and are not moved; U12's input
    // row i is the old row c0+pre[i].
    const int nout = b - w;
    const int ntr = b - c1;  // trailing panel columns
    if (!stop) {
      // all of a thread's gathers are issued before any is stored, so their
      // L2 latencies overlap
      const int cc = tid & 127;
      double g[kRpW];
#pragma unroll
      for (int q = 0; q < kRpW; ++q) {
        const int mv = 2 * q + (tid >> 7);
        const int d = mv < 2 * w ? s_mdst[mv] : -1;
        g[q] = 0.0;
        if (d >= 0 && cc < nout) {
          const int col = cc < c0 ? cc : cc + w;
          if (!(col >= c1 && d < c1)) g[q] = __ldcg(&A[(long long)col * lda + s_msrc[mv]]);
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
        const int d = mv < 2 * w ? s_mdst[mv] : -1;
        if (d >= 0 && cc < nout) {
          const int col = cc < c0 ? cc : cc + w;
          if (!(col >= c1 && d < c1)) MV[mv * 128 + cc] = g[q];
        }
      }
#pragma unroll
      for (int q = 0; q < kRpW * 128 / kRpThreads; ++q) {
        const int idx = tid + q * kRpThreads, i = idx >> 7, c = idx & 127;
        if (i < w && c < ntr) U12[i * 128 + c] = gu[q];
      }
    }
    // every source read (and CTA 0's sub-panel written) cluster-wide
    cluster_arrive_release();
    cluster_wait_acquire();
    if (!stop) {
      const int cc = tid & 127;
      for (int mv = tid >> 7; mv < 2 * w; mv += 2) {
        const int d = s_mdst[mv];
        if (d >= 0 && cc < nout) {
          const int col = cc < c0 ? cc : cc + w;
          if (!(col >= c1 && d < c1)) A[(long long)col * lda + d] = MV[mv * 128 + cc];
        }
      }
    }
    __syncthreads();
    if (!stop && ntr > 0) {
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
    }
    __syncthreads();
    if (!stop && ntr > 0) {
      // A[r, c1:b) -= L[r, c0:c1) U12 for own rows r >= c1 (L in registers),
      // kB columns at a time, the next batch's loads in flight while the
      // current one is updated
      constexpr int kB = RT >= 4 ? 4 : 8;
      double xa[RT][kB], xb[RT][kB];
      auto load = [&](double (&x)[RT][kB], int cb) {
#pragma unroll
        for (int s = 0; s < RT; ++s) {
          const int lr = s * kRpThreads + tid, r = r0 + lr;
#pragma unroll
          for (int q = 0; q < kB; ++q)
            x[s][q] = (lr < rows && r >= c1 && cb + q < ntr) ? __ldcg(&A[(long long)(c1 + cb + q) * lda + r]) : 0.0;
        }
      };
      auto update = [&](double (&x)[RT][kB], int cb) {
        // U12 pairs as 16-byte shared loads (cb is even): one load feeds 2 RT FMAs
#pragma unroll
        for (int k = 0; k < kRpW; ++k) {
          if (k < w) {
            double2 uu[kB / 2];
#pragma unroll
            for (int h = 0; h < kB / 2; ++h) uu[h] = *reinterpret_cast<const double2*>(&U12[k * 128 + cb + 2 * h]);
#pragma unroll
            for (int q = 0; q < kB; ++q) {
              const double u = (q & 1) ? uu[q / 2].y : uu[q / 2].x;
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
      };
      load(xa, 0);
      for (int cb = 0; cb < ntr; cb += 2 * kB) {
        if (cb + kB < ntr) load(xb, cb + kB);
        update(xa, cb);
        if (cb + kB < ntr) {
          if (cb + 2 * kB < ntr) load(xa, cb + 2 * kB);
          update(xb, cb + kB);
        }
      }
    }
    __syncthreads();
  }
  // all CTAs done with each other's shared memory and with the panel
  cluster_arrive_release();
  cluster_wait_acquire();
  if (stop) return;
  if (cta == 0 && tid < ncols) {  // ComposePivots over the whole panel
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
  if (W == nullptr) return;
  // inv(unit lower L11) of the panel's top bb x bb block, by CTA 0: 16 x 16
  // diagonal-block inverses by warps, then the DMMA doubling steps
  if (cta != 0) return;
  const int bb = ncols;
  double* S = sm;
  for (int e0 = tid; e0 < bb * bb; e0 += 8 * kRpThreads) {  // .cg: rows written by other CTAs
    double x[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = e0 + q * kRpThreads, r = e % bb, c = e / bb;
      x[q] = (e < bb * bb && r >= c) ? __ldcg(&A[(long long)c * lda + r]) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = e0 + q * kRpThreads, r = e % bb, c = e / bb;
      if (e < bb * bb && r >= c) SE(S, r, c) = x[q];
    }
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
