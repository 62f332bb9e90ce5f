// Triangular solve X := inv(T) X with few right-hand sides (nrhs <= 64), the
// Trsm(LEFT, ...) calls of cholesky::SolveAfter (Cholesky/SolveAfter.hpp:
// 20-75) and lu::SolveAfter (LU/SolveAfter.hpp:101-146), in one cooperative
// launch.  The triangle T is described by the stored matrix A and two flags:
//   amode 0: T's block (r, j) is A's block (r, j)        (T = A)
//   amode 1: T's block (r, j) is A's block (j, r)^T      (T = A^T)
//   bwd    : T is upper triangular (solve from the last block up)
// so lower L x = b is (fwd, 0), L^T x = b is (bwd, 1), U^T x = b is (fwd, 1)
// and U x = b is (bwd, 0).  Winv holds inv(A_rr) of every diagonal block
// (transposed on use when amode is 1).
//
// Block rows of X (nb rows each) are owned round-robin by the CTAs; a CTA
// processes its block rows in solve order, left-looking: acc = B_r -
// sum_j T(r, j) X_j over the blocks j already solved, then X_r = inv(T_rr)
// acc with the pre-inverted diagonal block, and publishes X_r with a release
// flag.  Each off-diagonal block is read once, so the sweep streams the
// triangle from HBM once while the dependency chain only waits on flags
// (bounded spins), not on kernel boundaries.  The first chunk of each
// off-diagonal block is requested before the wait for the X block it
// multiplies.
//
// Column-prescaled form (mode 1): A holds the off-diagonal blocks already
// multiplied by the inverse of the diagonal block of the column they act on,
// M(r, j) = T(r, j) inv(T_jj).  Then z_r = b_r - sum_j M(r, j) z_j needs no
// inverse on the dependency chain: a CTA publishes z_r (in X) as soon as the
// sum is done and forms Y_r = inv(T_rr) z_r afterwards.
//
// Row-prescaled form (mode 2): the blocks are M(r, j) = inv(T_rr) T(r, j), so
// x_r = inv(T_rr) b_r - sum_j M(r, j) x_j: every task forms inv(T_rr) b_r
// (b read from Y) before its first wait, and publishes x_r (in X) with no
// inverse after the sum.  With M2 = L D^-1 stored, L y = b is the
// column-prescaled sweep over M2 and L^T x = y the row-prescaled sweep over
// M2^T (amode 1): inv(L_rr^T) L_jr^T = (L_jr inv(L_rr))^T = M2(j, r)^T.
//
// Products are 16 x 8 x 8 DMMA fragments from shared memory: the whole
// off-diagonal block (ld 132, or its transpose with ld 132: conflict-free
// fragment loads) and the matching X block, 16-byte cp.async copies in four
// 32-deep groups that all are in flight at once.  Requires nrhs <= 64, nb <= 128 even, lda and ldx even,
// A, Winv, X (and Y) 16-byte aligned.
#include "internal.h"

namespace egpu {

namespace {

constexpr int kTsThreads = 256;  // 8 warps: warp w owns rows 16w .. 16w+15 of the block
constexpr int kTsKC = 32;        // k chunk (one cp.async group each)
constexpr int kTsLD = 132;       // leading dimension of the staged blocks (conflict-free fragment loads)
constexpr int kTsMaxRhs = 64;
constexpr int kTsA = 128 * kTsLD;          // doubles: a whole off-diagonal block, [a + k*132] or [k + a*132]
constexpr int kTsX = kTsMaxRhs * kTsLD;    // doubles: the matching X block, [k + c*132]
// The off-diagonal products of a block row run through a ring of kTsStages
// k chunks: stage = A chunk (amode 0: [a + k*132], amode 1: [k + a*36]) and
// X chunk ([k + c*36]); ld 132 and 36 are both 4 mod 16 (conflict-free
// 8-byte fragment loads).
constexpr int kTsStages = 4;
constexpr int kTsCT = 36;                        // ld of the chunk-transposed layouts
constexpr int kTsRA = 128 * kTsCT;               // doubles: A chunk (the larger of 32*132 and 128*36)
constexpr int kTsRX = kTsMaxRhs * kTsCT;         // doubles: X chunk
constexpr int kTsRStage = kTsRA + kTsRX;
constexpr int kTsSmemDoubles = (kTsA + kTsX) > kTsStages * kTsRStage ? (kTsA + kTsX) : kTsStages * kTsRStage;
static_assert(32 * kTsLD <= kTsRA, "A chunk fits its stage");

struct TsParams {
  const double* L;
  long long lda;
  const double* Winv;  // block i at Winv + i*nb*nb, ld nb
  double* X;
  long long ldx;
  double* Y;  // mode 1: Y_r = inv(T_rr) z_r (z published in X); mode 2: the right-hand side (X receives x)
  int n, nrhs, nb, nblk, bwd, amode;
  int mode;        // 0 plain, 1 column-prescaled, 2 row-prescaled
  int strips, hs;  // tasks per block row and their height (prescaled form: 2)
  int* flags;
  int epoch;
  DevStatus* status;
};

// block row of solve step s
__device__ __forceinline__ int ts_block(const TsParams& p, int s) { return p.bwd ? p.nblk - 1 - s : s; }

// Stage the k chunk [k0, k0+32) of an m x K operand A (m <= 128 rows) into
// the whole-block buffer with 16-byte .cg copies.  amode 0: A(a, k) =
// G[a + k lda] (column-major block), kept as sA[a + k * 132]; amode 1:
// A(a, k) = G[k + a lda] (the transpose of a column-major block), kept as
// sA[k + a * 132].  Out-of-range entries are zero.  lda even, G 16-byte
// aligned, k0 even.
__device__ __forceinline__ void ts_stage_a(double* sA, const double* G, long long lda, int amode, int m, int K,
                                           int k0) {
  const int tid = threadIdx.x;
  if (amode == 0) {
    for (int e = tid; e < 64 * kTsKC; e += kTsThreads) {  // row pairs
      const int a = 2 * (e & 63), k = k0 + (e >> 6);
      double* d = &sA[a + k * kTsLD];
      const double* src = &G[a + (long long)k * lda];
      if (k < K && a + 1 < m) cp_async16_cg(d, src);
      else {
        d[0] = (k < K && a < m) ? src[0] : 0.0;
        d[1] = 0.0;
      }
    }
  } else {
    for (int e = tid; e < 128 * (kTsKC / 2); e += kTsThreads) {  // k pairs
      const int k = k0 + 2 * (e & 15), a = e >> 4;
      double* d = &sA[k + a * kTsLD];
      const double* src = &G[k + (long long)a * lda];
      if (a < m && k + 1 < K) cp_async16_cg(d, src);
      else {
        d[0] = (a < m && k < K) ? src[0] : 0.0;
        d[1] = 0.0;
      }
    }
  }
}

// The matching rows [k0, k0+32) of X (K x nrhs) into sX[k + c * 132]:
// 16-byte .cg copies (L2, never a stale L1 line of a block another CTA has
// just published); ldx even and X 16-byte aligned.
__device__ __forceinline__ void ts_stage_x(double* sX, int K, int k0, const double* Xg, long long ldx, int nrhs) {
  for (int e = threadIdx.x; e < (kTsKC / 2) * nrhs; e += kTsThreads) {
    const int k = k0 + 2 * (e & 15), c = e >> 4;
    double* d = &sX[k + c * kTsLD];
    const double* src = &Xg[k + (long long)c * ldx];
    if (k + 1 < K) {
      cp_async16_cg(d, src);
    } else {
      d[0] = (k < K) ? __ldcg(src) : 0.0;
      d[1] = 0.0;
    }
  }
}

__device__ __forceinline__ void ts_wait_groups(int pending) {
  switch (pending) {  // cp.async.wait_group takes an immediate
    case 0: asm volatile("cp.async.wait_group 0;" ::: "memory"); break;
    case 1: asm volatile("cp.async.wait_group 1;" ::: "memory"); break;
    case 2: asm volatile("cp.async.wait_group 2;" ::: "memory"); break;
    default: asm volatile("cp.async.wait_group 3;" ::: "memory"); break;
  }
}

// Bounded wait (thread 0) for the arrival counter *flag to reach `epoch`
// (strips x sweep number), then a CTA barrier.  Returns
// false (all threads) when the wait ran out.
__device__ __forceinline__ bool ts_wait_flag(const int* flag, int epoch, DevStatus* status) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    int ok = 1;
    long long it = 0;
    while (true) {
      int v;
      asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
      if (v >= epoch) break;
      if (++it > kSpinLimit) { ok = 0; set_status(status, kTimeout, 201); break; }
      if (it > 4096) __nanosleep(64);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Chunk [k0, k0+32) of the strip's A operand into a ring stage: one TMA box
// issued by thread 0, completing on `bar`.  amode 0: the box is rows r0 ..
// r0+hs+3 x columns j0+k0 .. +31 of the stored matrix, landing as
// sA[a + kl*(hs+4)]; amode 1: rows j0+k0 .. +35 x columns r0 .. r0+hs-1,
// landing as sA[kl + a*36].  Both pitches are 4 mod 16 (conflict-free
// fragment loads); the extra rows are read and ignored, and the parts of the
// box past the matrix (a short last block) arrive as zeros.
__device__ __forceinline__ void ts_tma_a(double* sA, const CUtensorMap* map, const TsParams& p, int r0, int j0,
                                         int k0, uint64_t* bar) {
  if (threadIdx.x != 0) return;
  const uint32_t bytes = p.amode == 0 ? (uint32_t)((p.hs + 4) * kTsKC * 8) : (uint32_t)(kTsCT * p.hs * 8);
  mbar_expect_tx(bar, bytes);
  if (p.amode == 0) tma_load_2d(sA, map, bar, r0, j0 + k0);
  else tma_load_2d(sA, map, bar, j0 + k0, r0);
}

// Rows [k0, k0+32) of X (K x nrhs) into a ring stage, sX[kl + c*36]: 16-byte
// .cg copies by every thread (X was published by other CTAs and acquired
// through a flag: read through L2 in the generic proxy), each thread's copies
// arriving on `bar` (initial count: the block size).  Rows past K are zero.
__device__ __forceinline__ void ts_async_x(double* sX, int K, int k0, const double* Xg, long long ldx, int nrhs,
                                           uint64_t* bar) {
  for (int e = threadIdx.x; e < (kTsKC / 2) * nrhs; e += kTsThreads) {
    const int kl = 2 * (e & 15), c = e >> 4, k = k0 + kl;
    double* dd = &sX[kl + c * kTsCT];
    const double* src = &Xg[k + (long long)c * ldx];
    if (k + 1 < K) {
      cp_async16_cg(dd, src);
    } else {
      dd[0] = (k < K) ? __ldcg(src) : 0.0;
      dd[1] = 0.0;
    }
  }
  cp_async_arrive_noinc(bar);
}

// Error exit: wait (bounded) for the copies of every piece already issued,
// chunks [from, a_end) of A and [from, x_end) of X, so no copy still targets
// this CTA's shared memory when it returns.
__device__ __forceinline__ void ts_ring_drain(uint64_t* barA, uint64_t* barX, int gq, int from, int a_end, int x_end) {
  for (int q = from; q < a_end; ++q)
    (void)mbar_wait_bounded(&barA[(gq + q) % kTsStages], (uint32_t)((gq + q) / kTsStages) & 1u);
  for (int q = from; q < x_end; ++q)
    (void)mbar_wait_bounded(&barX[(gq + q) % kTsStages], (uint32_t)((gq + q) / kTsStages) & 1u);
}

// Both pieces of ring chunk `gq` (this CTA's running chunk count) landed:
// every thread waits on the stage's two mbarrier phases (bounded).
__device__ __forceinline__ bool ts_ring_wait(uint64_t* barA, uint64_t* barX, int gq, DevStatus* status) {
  const int slot = gq % kTsStages;
  const uint32_t par = (uint32_t)(gq / kTsStages) & 1u;
  if (mbar_wait_bounded(&barA[slot], par) && mbar_wait_bounded(&barX[slot], par)) return true;
  set_status(status, kTimeout, 202);
  return false;
}

// acc -= sum over solve steps sj < s of T(strip, j) X_j (j = the block row of
// step sj): every product's k chunks stream through the kTsStages-deep ring
// as one sequence, so the loads of the next chunks (and of the next product)
// overlap the DMMAs of the current one.  A pieces are single TMA boxes
// (thread 0) issued up to kTsStages chunks ahead with no flag; X pieces are
// small copies by every thread once X_j is published:
// a poll that runs behind the DMMAs while loaded chunks remain, a bounded
// wait when nothing else is left.  gq: the CTA's running chunk count (the
// stage mbarriers' phases).  Returns false when a wait ran out.
template <int NT>
__device__ bool ts_ring_products(double (&acc)[8][4], double* sm, uint64_t* barA, uint64_t* barX, int& gq,
                                 const CUtensorMap* mapA, const TsParams& p, int s, int r0, int mr, int target) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int cpp = (p.nb + kTsKC - 1) / kTsKC;  // chunks per product
  const int Q = s * cpp;
  int a_issued = 0, x_issued = 0, ready = 0;
  int pv_prev = 0, pidx_prev = -1;  // the previous chunk's poll (thread 0)
  if (threadIdx.x == 0) fence_proxy_async_smem();  // the stages were last written in the generic proxy
  const int ldA = p.amode == 0 ? p.hs + 4 : kTsCT;  // A stage pitch
  for (int qc = 0; qc < Q; ++qc) {
    // X pieces first (they gate the next chunks)
    for (; x_issued < Q && x_issued < qc + kTsStages; ++x_issued) {
      const int sj = x_issued / cpp, c = x_issued - sj * cpp;
      const int j = ts_block(p, sj), j0 = j * p.nb, mj = min(p.nb, p.n - j0);
      if (sj >= ready) {
        if (x_issued > qc) break;  // loaded chunks remain: the poll below runs behind them
        if (!ts_wait_flag(&p.flags[j], target, p.status)) {
          ts_ring_drain(barA, barX, gq, qc, a_issued, x_issued);
          return false;
        }
        ready = sj + 1;
      }
      const int sl = (gq + x_issued) % kTsStages;
      ts_async_x(sm + sl * kTsRStage + kTsRA, mj, c * kTsKC, p.X + j0, p.ldx, p.nrhs, &barX[sl]);
    }
    // A pieces (no flag) up to kTsStages chunks ahead
    for (; a_issued < Q && a_issued < qc + kTsStages; ++a_issued) {
      const int sj = a_issued / cpp, c = a_issued - sj * cpp;
      const int sl = (gq + a_issued) % kTsStages;
      ts_tma_a(sm + sl * kTsRStage, mapA, p, r0, ts_block(p, sj) * p.nb, c * kTsKC, &barA[sl]);
    }
    // poll for the first product not yet known published: a relaxed load
    // issued now and read at the next chunk's closing barrier, so its round
    // trip hides behind the DMMAs
    int pv = 0;
    const int pidx = ready < s ? ready : -1;
    if (pidx >= 0 && threadIdx.x == 0)
      asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(pv) : "l"(&p.flags[ts_block(p, pidx)]) : "memory");
    const int slot = (gq + qc) % kTsStages;
    if (!ts_ring_wait(barA, barX, gq + qc, p.status)) {
      ts_ring_drain(barA, barX, gq, qc + 1, a_issued, x_issued);
      return false;
    }
    __syncthreads();  // the X pieces' ordinary-store parts (zero rows) are visible
    const int sj = qc / cpp, c = qc - sj * cpp;
    const int mj = min(p.nb, p.n - ts_block(p, sj) * p.nb);
    if (c * kTsKC < mj && 16 * warp < mr) {
      const double* sA = sm + slot * kTsRStage;
      const double* sX = sA + kTsRA;
      const int ra = 16 * warp + g;
#pragma unroll
      for (int kk = 0; kk < kTsKC; kk += 8) {
        double a[4];
        if (p.amode == 0) {
          a[0] = -sA[ra + (kk + t) * ldA];
          a[1] = -sA[ra + 8 + (kk + t) * ldA];
          a[2] = -sA[ra + (kk + t + 4) * ldA];
          a[3] = -sA[ra + 8 + (kk + t + 4) * ldA];
        } else {
          a[0] = -sA[(kk + t) + ra * kTsCT];
          a[1] = -sA[(kk + t) + (ra + 8) * kTsCT];
          a[2] = -sA[(kk + t + 4) + ra * kTsCT];
          a[3] = -sA[(kk + t + 4) + (ra + 8) * kTsCT];
        }
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          double bf[2];
          bf[0] = sX[(kk + t) + (8 * nt + g) * kTsCT];
          bf[1] = sX[(kk + t + 4) + (8 * nt + g) * kTsCT];
          dmma_16x8x8(acc[nt], a, bf);
        }
      }
    }
    // the stage is free for chunk qc + kTsStages; the previous chunk's poll
    // answer, made an acquire by thread 0's fence before the barrier that
    // publishes it
    int seen = 0;
    if (threadIdx.x == 0 && pidx_prev >= 0 && pidx_prev == ready && pv_prev >= target) {
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
      seen = 1;
    }
    if (__syncthreads_or(seen)) ready = ready + 1;
    pv_prev = pv;
    pidx_prev = pidx;
  }
  gq += Q;
  return true;
}

// acc[nt] (16 x 8 fragments, rows 16 warp.., columns 8 nt..) += sign * A(m x K) * X(K x nrhs), K <= 128.
// Every chunk of A is requested at once (one cp.async group each) before the
// wait for X to be published (`flag`), then every chunk of X, so one product
// costs one memory round trip plus its DMMAs.  x_in_smem: X already sits in
// the X buffer (the staged accumulator).
template <int NT>
__device__ bool ts_product(double (&acc)[8][4], double sign, double* sm, const double* G, long long lda, int amode,
                           int m, int K, const double* Xg, long long ldx, int nrhs, bool x_in_smem,
                           const int* flag = nullptr, int epoch = 0, DevStatus* status = nullptr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int nch = (K + kTsKC - 1) / kTsKC;
  double* sA = sm;
  double* sX = sm + kTsA;
  for (int c = 0; c < nch; ++c) {
    ts_stage_a(sA, G, lda, amode, m, K, c * kTsKC);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  if (flag != nullptr && !ts_wait_flag(flag, epoch, status)) {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    return false;
  }
  if (!x_in_smem)
    for (int c = 0; c < nch; ++c) {
      ts_stage_x(sX, K, c * kTsKC, Xg, ldx, nrhs);
      asm volatile("cp.async.commit_group;" ::: "memory");
    }
  for (int c = 0; c < nch; ++c) {
    ts_wait_groups(nch - 1 - c);  // A chunk c (and X chunk c) landed for this thread
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTsKC; kk += 8) {
      const int k = c * kTsKC + kk;
      double a[4];
      const int ra = 16 * warp + g;
      if (amode == 0) {
        a[0] = sA[ra + (k + t) * kTsLD];
        a[1] = sA[ra + 8 + (k + t) * kTsLD];
        a[2] = sA[ra + (k + t + 4) * kTsLD];
        a[3] = sA[ra + 8 + (k + t + 4) * kTsLD];
      } else {
        a[0] = sA[(k + t) + ra * kTsLD];
        a[1] = sA[(k + t) + (ra + 8) * kTsLD];
        a[2] = sA[(k + t + 4) + ra * kTsLD];
        a[3] = sA[(k + t + 4) + (ra + 8) * kTsLD];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) a[q] *= sign;
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        double bf[2];
        bf[0] = sX[(k + t) + (8 * nt + g) * kTsLD];
        bf[1] = sX[(k + t + 4) + (8 * nt + g) * kTsLD];
        dmma_16x8x8(acc[nt], a, bf);
      }
    }
  }
  __syncthreads();  // the buffers are free for the next product
  return true;
}

}  // namespace

// NT: 8-column tiles of the right-hand side (a compile-time count: a DMMA
// skipped under a run-time predicate still costs its issue slots).
template <int NT>
__global__ void __launch_bounds__(kTsThreads, 1) trsm_skinny_kernel(const __grid_constant__ CUtensorMap mapA,
                                                                    TsParams p) {
  // TMA boxes land at stage starts: the dynamic region must be 128-byte
  // aligned (it follows the static barriers)
  extern __shared__ __align__(128) double sm[];
  double* accS = sm + kTsA;  // the X buffer: the accumulator is the next product's right operand
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  __shared__ __align__(8) uint64_t barA[kTsStages], barX[kTsStages];
  if (tid == 0) {
    for (int i = 0; i < kTsStages; ++i) {
      mbar_init(&barA[i], 1);
      mbar_init(&barX[i], kTsThreads);
    }
    fence_mbar_init();
  }
  __syncthreads();
  int gq = 0;  // ring chunks issued by this CTA so far
  const int mode = p.mode;
  const int S = p.strips, hs = p.hs, target = p.strips * p.epoch;
  if (p.status != nullptr && ((volatile DevStatus*)p.status)->code != 0) return;
  if (smem_u32(sm) % 128 != 0) {  // no TMA into a misaligned stage: report and stop
    if (tid == 0) set_status(p.status, kTimeout, 203);
    return;
  }
  for (int task = blockIdx.x; task < p.nblk * S; task += gridDim.x) {
    const int s = task / S, q = task - s * S;
    const int r = ts_block(p, s);
    const int rb0 = r * p.nb, mb = min(p.nb, p.n - rb0);  // the block row
    const int r0 = rb0 + q * hs, mr = min(hs, mb - q * hs);  // this task's strip of it (may be empty)
    double acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[nt][e] = 0.0;
    if (mr > 0) {
      if (mode == 2) {
        // acc = inv(T_rr)(strip rows, :) b_r, before the first wait
        const double* Wr = p.Winv + (long long)r * p.nb * p.nb;
        const double* G = p.amode == 0 ? Wr + q * hs : Wr + (long long)q * hs * p.nb;
        ts_product<NT>(acc, 1.0, sm, G, p.nb, p.amode, mr, mb, p.Y + rb0, p.ldx, p.nrhs, false);
      } else {
        // acc = B(strip)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int row = 16 * warp + g + ((e >= 2) ? 8 : 0), col = 8 * nt + 2 * t + (e & 1);
            if (nt < NT && row < mr && col < p.nrhs) acc[nt][e] = __ldcg(&p.X[(r0 + row) + (long long)col * p.ldx]);
          }
      }
      // acc -= T(strip, j) X_j for the blocks j solved before r
      if (!ts_ring_products<NT>(acc, sm, barA, barX, gq, &mapA, p, s, r0, mr, target)) return;
    }
    if (mode == 1) {
      // column-prescaled form: publish the strip of z_r = acc first (the others need only z) ...
      if (mr > 0)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int row = 16 * warp + g + ((e >= 2) ? 8 : 0), col = 8 * nt + 2 * t + (e & 1);
            if (nt < NT && row < mr && col < p.nrhs) p.X[(r0 + row) + (long long)col * p.ldx] = acc[nt][e];
          }
      __syncthreads();  // the block's stores happen before thread 0's release (barrier + cumulative release)
      if (tid == 0) asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(&p.flags[r]) : "memory");
      if (mr <= 0) continue;
      // ... then Y(strip) = inv(T_rr)(strip rows, :) z_r once every strip of z_r is out
#pragma unroll
      for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[nt][e] = 0.0;
      const double* Wr = p.Winv + (long long)r * p.nb * p.nb;
      const double* G = p.amode == 0 ? Wr + q * hs : Wr + (long long)q * hs * p.nb;
      if (!ts_product<NT>(acc, 1.0, sm, G, p.nb, p.amode, mr, mb, p.X + rb0, p.ldx, p.nrhs, false, &p.flags[r], target,
                      p.status))
        return;
    } else if (mode == 0) {
      // X_r = inv(T_rr) acc (one strip per block: the whole accumulator is in this CTA)
#pragma unroll
      for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int row = 16 * warp + g + ((e >= 2) ? 8 : 0), col = 8 * nt + 2 * t + (e & 1);
          // rows past the strip hold products of stale stage rows: they are the
          // product's zero K tail here
          if (nt < NT) accS[row + col * kTsLD] = row < mr ? acc[nt][e] : 0.0;
          acc[nt][e] = 0.0;
        }
      __syncthreads();
      const double* Wr = p.Winv + (long long)r * p.nb * p.nb;
      ts_product<NT>(acc, 1.0, sm, Wr, p.nb, p.amode, mr, mr, accS, kTsLD, p.nrhs, true);
    }
    double* out = mode == 1 ? p.Y : p.X;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int row = 16 * warp + g + ((e >= 2) ? 8 : 0), col = 8 * nt + 2 * t + (e & 1);
        if (nt < NT && row < mr && col < p.nrhs) out[(r0 + row) + (long long)col * p.ldx] = acc[nt][e];
      }
    if (mode != 1) {
      __syncthreads();  // the block's stores happen before thread 0's release (barrier + cumulative release)
      if (tid == 0) asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(&p.flags[r]) : "memory");
    }
  }
}

size_t trsm_skinny_flag_bytes(int n, int nb) { return sizeof(int) * (size_t)((n + nb - 1) / nb) + 256; }

// flags: device array of ceil(n/nb) arrival counters, zero before the first
// sweep of a sequence; sweep number `epoch` (1, 2, ...) of the sequence
// waits for counters to reach strips x epoch.
int launch_trsm_skinny(cudaStream_t st, int bwd, int amode, int n, int nrhs, const double* L, long long lda,
                       const double* Winv, int nb, double* X, long long ldx, int* flags, int epoch, int sm_count,
                       DevStatus* status, double* Y, bool row_prescaled) {
  if (n <= 0 || nrhs <= 0) return EGPU_OK;
  if (nrhs > kTsMaxRhs || nb > 128 || nb < 8 || nb % 2 != 0 || ldx % 2 != 0 || lda % 2 != 0 ||
      reinterpret_cast<uintptr_t>(X) % 16 != 0 || reinterpret_cast<uintptr_t>(L) % 16 != 0 ||
      reinterpret_cast<uintptr_t>(Winv) % 16 != 0 || reinterpret_cast<uintptr_t>(Y) % 16 != 0)
    return EGPU_ERR_UNSUPPORTED;
  TsParams p;
  p.L = L; p.lda = lda; p.Winv = Winv; p.X = X; p.ldx = ldx; p.Y = Y;
  p.n = n; p.nrhs = nrhs; p.nb = nb; p.nblk = (n + nb - 1) / nb; p.bwd = bwd; p.amode = amode;
  p.mode = Y == nullptr ? 0 : row_prescaled ? 2 : 1;
  // prescaled form: two strips per block row, so the dependency chain's product is half a block,
  // while a CTA holds at most two tasks (its second task starts after the first and still has to
  // catch up with all the products of its block row)
  p.strips = (p.mode != 0 && nb >= 32 && (n + nb - 1) / nb <= sm_count) ? 2 : 1;
  p.hs = p.strips == 1 ? nb : ((nb + 1) / 2 + 15) / 16 * 16;
  p.flags = flags; p.epoch = epoch; p.status = status;
  // A's ring pieces: TMA boxes over the stored n x n matrix (see ts_tma_a)
  CUtensorMap mapA;
  const bool mok = amode == 0 ? make_tma_2d(&mapA, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, L, n, n, 8ull * lda,
                                            (uint32_t)(p.hs + 4), kTsKC, false)
                              : make_tma_2d(&mapA, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, L, n, n, 8ull * lda, kTsCT,
                                            (uint32_t)p.hs, false);
  if (!mok) return EGPU_ERR_UNSUPPORTED;
  const size_t smem = sizeof(double) * kTsSmemDoubles;
  const int nt = nrhs <= 8 ? 1 : nrhs <= 16 ? 2 : nrhs <= 32 ? 4 : 8;
  void (*kern)(const CUtensorMap, TsParams) = nt == 1 ? trsm_skinny_kernel<1>
                           : nt == 2 ? trsm_skinny_kernel<2>
                           : nt == 4 ? trsm_skinny_kernel<4> : trsm_skinny_kernel<8>;
  static bool attr[4] = {false, false, false, false};
  const int ai = nt == 1 ? 0 : nt == 2 ? 1 : nt == 4 ? 2 : 3;
  if (!attr[ai]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      cudaGetLastError();
      return EGPU_ERR_UNSUPPORTED;
    }
    attr[ai] = true;
  }
  const int grid = std::min(p.nblk * p.strips, sm_count);
  TraceMark tm(st, kTraceSolve, (double)n * n * nrhs, 4.0 * (double)n * n + 16.0 * n * nrhs);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kTsThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr1[1];
  attr1[0].id = cudaLaunchAttributeCooperative;  // every CTA resident: the flag waits always end
  attr1[0].val.cooperative = 1;
  cfg.attrs = attr1;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, kern, mapA, p);
  count_launch();
  if (e != cudaSuccess) {
    set_last_error(e, "trsm_skinny launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

}  // namespace egpu
