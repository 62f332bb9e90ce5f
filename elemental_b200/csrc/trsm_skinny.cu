// Triangular solve X := inv(T) X with few right-hand sides (nrhs <= 64), the
// Trsm(LEFT, ...) calls of cholesky::SolveAfter (Cholesky/SolveAfter.hpp:
// 20-75) and lu::SolveAfter (LU/SolveAfter.hpp:101-146), in one cooperative
// launch.  The triangle T is described by the stored matrix A and two flags:
//   amode 0: T's block (r, j) is A's block (r, j)        (T = A)
//   amode 1: T's block (r, j) is A's block (j, r)^T      (T = A^T)
//   bwd    : T is upper triangular (solve from the last block up)
// so lower L x = b is (fwd, 0), L^T x = b is (bwd, 1), U^T x = b is (fwd, 1)
// and U x = b is (bwd, 0).  Winv holds inv(A_rr) of every diagonal block
// (transposed on use when amode is 1), each in a zero-padded nb x nb slot.
//
// Block rows of X (nb rows each, optionally split into two strips) are owned
// by the CTAs in solve order, left-looking: acc = B_r - sum_j T(r, j) X_j
// over the blocks j already solved, then X_r = inv(T_rr) acc, published with
// a release counter.  Each off-diagonal block is read once, so the sweep
// streams the triangle from HBM once while the dependency chain only waits
// on counters (bounded spins), not on kernel boundaries.
//
// Column-prescaled form (mode 1): A holds the off-diagonal blocks already
// multiplied by the inverse of the diagonal block of the column they act on,
// M(r, j) = T(r, j) inv(T_jj).  Then z_r = b_r - sum_j M(r, j) z_j needs no
// inverse on the dependency chain: a CTA publishes z_r (in X) as soon as the
// sum is done and forms Y_r = inv(T_rr) z_r afterwards.
//
// Row-prescaled form (mode 2): the blocks are M(r, j) = inv(T_rr) T(r, j), so
// x_r = inv(T_rr) b_r - sum_j M(r, j) x_j: every task forms inv(T_rr) b_r
// (b read from Y) first, with no counter to wait for, and publishes x_r (in
// X) with no inverse after the sum.  With M2 = L D^-1 stored, L y = b is the
// column-prescaled sweep over M2 and L^T x = y the row-prescaled sweep over
// M2^T (amode 1): inv(L_rr^T) L_jr^T = (L_jr inv(L_rr))^T = M2(j, r)^T.
//
// Warp-specialized: every product (an off-diagonal block times X_j, or the
// diagonal inverse times a block of X) streams through a ring of kTsStages
// k chunks of 32.  A producer warp issues each chunk's A piece as one TMA box
// (up to kTsStages chunks ahead) and its X piece as 16-byte copies once X_j
// is published (it alone spins on the counters), both completing on the
// stage's full barriers; eight consumer warps only wait, multiply (16 x 8 x 8
// DMMA fragments from shared memory) and release the stage.  Requires
// nrhs <= 64, nb <= 128 even, lda and ldx even, A, Winv, X (and Y) 16-byte
// aligned.
#include "internal.h"

namespace egpu {

namespace {

constexpr int kTsConsumers = 256;              // 8 warps: warp w owns rows 16w .. 16w+15 of the strip
constexpr int kTsThreads = kTsConsumers + 32;  // + the producer warp
constexpr int kTsKC = 32;                      // k chunk
constexpr int kTsMaxRhs = 64;
// A ring stage holds an A chunk (amode 0: [a + kl*(hs+4)], amode 1:
// [kl + a*36]) and an X chunk ([kl + c*36]); both pitches are 4 mod 16
// (conflict-free 8-byte fragment loads) and every stage starts on a
// 128-byte boundary (TMA destination).
constexpr int kTsStages = 4;
constexpr int kTsCT = 36;                 // pitch of the k-contiguous layouts
constexpr int kTsRA = 128 * kTsCT;        // doubles: A chunk (>= 32 * 132 and 36 * 128)
constexpr int kTsRX = kTsMaxRhs * kTsCT;  // doubles: X chunk
constexpr int kTsRStage = kTsRA + kTsRX;
constexpr int kTsSmemDoubles = kTsStages * kTsRStage;
static_assert(32 * 132 <= kTsRA, "A chunk fits its stage");
static_assert((kTsRStage * 8) % 128 == 0 && (kTsRA * 8) % 128 == 0, "stage starts are 128-byte aligned");

struct TsParams {
  const double* L;
  long long lda;
  const double* Winv;  // block i at Winv + i*nb*nb, ld nb
  double* X;
  long long ldx;
  double* Y;  // mode 1: Y_r = inv(T_rr) z_r (z published in X); mode 2: the right-hand side (X receives x)
  int n, nrhs, nb, nblk, bwd, amode;
  int mode;        // 0 plain, 1 column-prescaled, 2 row-prescaled
  int strips, hs;  // tasks per block row and their height
  int* flags;
  int epoch;
  DevStatus* status;
};

// block row of solve step s
__device__ __forceinline__ int ts_block(const TsParams& p, int s) { return p.bwd ? p.nblk - 1 - s : s; }

// One task: strip q of the block row r solved at step s.
struct TsTask {
  int s, q, r, rb0, mb, r0, mr;
};
__device__ __forceinline__ TsTask ts_task(const TsParams& p, int task) {
  TsTask t;
  t.s = task / p.strips;
  t.q = task - t.s * p.strips;
  t.r = ts_block(p, t.s);
  t.rb0 = t.r * p.nb;
  t.mb = min(p.nb, p.n - t.rb0);
  t.r0 = t.rb0 + t.q * p.hs;
  t.mr = min(p.hs, t.mb - t.q * p.hs);  // may be empty
  return t;
}

// Product pi of a task: the s off-diagonal products (solve steps, sign -1)
// and one diagonal product inv(T_rr)(strip rows, :) times a block of X (sign
// +1): last in modes 0 and 1, first in mode 2.  Its X: block j of X
// (counter j), the staged accumulator (mode 0), z_r (mode 1: counter r, all
// strips) or b_r from Y (mode 2, no counter).
struct TsProd {
  int step;            // off-diagonal solve step, or -1 for the diagonal product
  int j0, K;           // first row of the X block, its height
  const double* xsrc;  // X block (global), or null: staged by the consumers
  const int* flag;     // counter to wait for, or null
};
__device__ __forceinline__ TsProd ts_prod(const TsParams& p, const TsTask& t, int pi) {
  TsProd d;
  const bool diag = p.mode == 2 ? pi == 0 : pi == t.s;
  d.step = diag ? -1 : (p.mode == 2 ? pi - 1 : pi);
  if (!diag) {
    const int j = ts_block(p, d.step);
    d.j0 = j * p.nb;
    d.K = min(p.nb, p.n - d.j0);
    d.xsrc = p.X + d.j0;
    d.flag = &p.flags[j];
  } else {
    d.j0 = t.rb0;
    d.K = t.mb;
    d.xsrc = p.mode == 0 ? nullptr : (p.mode == 1 ? p.X : p.Y) + t.rb0;
    d.flag = p.mode == 1 ? &p.flags[t.r] : nullptr;
  }
  return d;
}

// Bounded wait on an mbarrier phase for the chunk pipeline: spins (the
// try_wait itself suspends briefly) before it starts to sleep.
__device__ __forceinline__ bool ts_mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long long it = 0; it < kSpinLimit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it > 4096) __nanosleep(64);
  }
  return false;
}

// Consumers only (warps 0..7): named barrier 1.
__device__ __forceinline__ void ts_consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kTsConsumers) : "memory"); }

}  // namespace

// Barrier counts: fullA completes on thread 0's expect_tx arrival plus the
// TMA bytes; fullX on two arrivals per producer lane (its copies' completion,
// and an ordinary release arrival covering its zero stores); empty on one
// arrival per consumer warp.
constexpr uint32_t kTsFullXCount = 64;
constexpr uint32_t kTsEmptyCount = kTsConsumers / 32;

// The producer warp: every chunk of every product of this CTA's tasks, A
// pieces up to kTsStages chunks ahead of the X pieces (a stage is reused
// once its consumers released it), X pieces once their block is published.
// Nothing here blocks: the loop polls stage releases and counters and idles
// (bounded) only when neither moves.
__device__ void ts_producer(const CUtensorMap* mapL, const CUtensorMap* mapW, const TsParams& p, double* sm,
                            uint64_t* fullA, uint64_t* fullX, uint64_t* empty) {
  const int lane = threadIdx.x & 31;
  const int cpp = (p.nb + kTsKC - 1) / kTsKC;  // chunks per product
  const int target = p.strips * p.epoch;
  const uint32_t a_bytes = p.amode == 0 ? (uint32_t)((p.hs + 4) * kTsKC * 8) : (uint32_t)(kTsCT * p.hs * 8);
  if (lane == 0) {
    tma_prefetch_desc(mapL);
    tma_prefetch_desc(mapW);
  }
  int gq = 0;  // chunks of this CTA so far
  for (int task = blockIdx.x; task < p.nblk * p.strips; task += gridDim.x) {
    const TsTask t = ts_task(p, task);
    if (t.mr <= 0) continue;
    const int Q = (t.s + 1) * cpp;
    int a_next = 0, x_next = 0, known = -1;
    long long idle = 0;
    // one polling loop: A pieces whose stage is free (tested, never waited
    // for), and the next X piece as soon as its stage is ours and its block
    // is published, so no X piece queues behind a stage release
    while (x_next < Q) {
      bool progress = false;
      while (a_next < Q && a_next < x_next + kTsStages) {
        const int g = gq + a_next, slot = g % kTsStages;
        if (g >= kTsStages) {  // lane 0's test decides for the warp
          const int freed = mbar_test(&empty[slot], ((uint32_t)(g / kTsStages) & 1u) ^ 1u);
          if (!__shfl_sync(0xffffffffu, freed, 0)) break;
        }
        if (lane == 0) {
          const int pi = a_next / cpp, k0 = (a_next - pi * cpp) * kTsKC;
          const TsProd d = ts_prod(p, t, pi);
          double* sA = sm + slot * kTsRStage;
          mbar_expect_tx(&fullA[slot], a_bytes);
          if (d.step >= 0) {  // rows of the strip x columns of block j of the stored matrix (or its transpose)
            if (p.amode == 0) tma_load_2d(sA, mapL, &fullA[slot], t.r0, d.j0 + k0);
            else tma_load_2d(sA, mapL, &fullA[slot], d.j0 + k0, t.r0);
          } else {  // the strip's rows of inv(T_rr): slot r of the Winv tensor (columns r*nb ..)
            const int wc = t.r * p.nb;
            if (p.amode == 0) tma_load_2d(sA, mapW, &fullA[slot], t.q * p.hs, wc + k0);
            else tma_load_2d(sA, mapW, &fullA[slot], k0, wc + t.q * p.hs);
          }
        }
        ++a_next;
        progress = true;
      }
      while (x_next < a_next) {  // X pieces whose stage holds their A piece
        const int pi = x_next / cpp, c = x_next - pi * cpp;
        const TsProd d = ts_prod(p, t, pi);
        if (d.xsrc != nullptr && d.flag != nullptr && known != pi) {
          int v = 0;
          if (lane == 0) asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(d.flag) : "memory");
          v = __shfl_sync(0xffffffffu, v, 0);  // lane 0's acquire, then every lane's copies
          if (v < target) break;
          known = pi;
        }
        const int slot = (gq + x_next) % kTsStages;
        if (d.xsrc != nullptr) {
          double* sX = sm + slot * kTsRStage + kTsRA;
          const int k0 = c * kTsKC;
          for (int e = lane; e < (kTsKC / 2) * p.nrhs; e += 32) {
            const int kl = 2 * (e & 15), col = e >> 4, k = k0 + kl;
            double* dd = &sX[kl + col * kTsCT];
            const double* src = &d.xsrc[k + (long long)col * p.ldx];
            if (k + 1 < d.K) {
              cp_async16_cg(dd, src);
            } else {
              dd[0] = (k < d.K) ? __ldcg(src) : 0.0;
              dd[1] = 0.0;
            }
          }
        }
        // staged pieces (written by the consumers) still complete the phase
        cp_async_arrive_noinc(&fullX[slot]);
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&fullX[slot])) : "memory");
        ++x_next;
        progress = true;
      }
      if (progress) {
        idle = 0;
      } else if (++idle > kSpinLimit) {
        if (lane == 0) set_status(p.status, kTimeout, 212);
        return;
      } else if (idle > 4096) {
        __nanosleep(64);
      }
    }
    gq += Q;
  }
}

// The consumer warps: acc for the task's strip through all its products,
// then the store and the release of the block's counter.
template <int NT>
__device__ void ts_consumers(const TsParams& p, double* sm, uint64_t* fullA, uint64_t* fullX, uint64_t* empty) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g8 = lane >> 2, t4 = lane & 3;
  const int cpp = (p.nb + kTsKC - 1) / kTsKC;
  const int ldA = p.amode == 0 ? p.hs + 4 : kTsCT;  // A stage pitch
  int gq = 0;
  for (int task = blockIdx.x; task < p.nblk * p.strips; task += gridDim.x) {
    const TsTask t = ts_task(p, task);
    double acc[NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[nt][e] = 0.0;
    if (t.mr > 0) {
      if (p.mode != 2) {  // acc = B(strip)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int row = 16 * warp + g8 + ((e >= 2) ? 8 : 0), col = 8 * nt + 2 * t4 + (e & 1);
            if (row < t.mr && col < p.nrhs) acc[nt][e] = __ldcg(&p.X[(t.r0 + row) + (long long)col * p.ldx]);
          }
      }
      const int P = t.s + 1;
      for (int pi = 0; pi < P; ++pi) {
        const TsProd d = ts_prod(p, t, pi);
        if (d.step < 0 && p.mode == 1) {
          // column-prescaled form: publish the strip of z_r = acc (the other
          // tasks need only z), then Y(strip) = inv(T_rr)(strip, :) z_r
#pragma unroll
          for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int row = 16 * warp + g8 + ((e >= 2) ? 8 : 0), col = 8 * nt + 2 * t4 + (e & 1);
              if (row < t.mr && col < p.nrhs) p.X[(t.r0 + row) + (long long)col * p.ldx] = acc[nt][e];
              acc[nt][e] = 0.0;
            }
          ts_consumer_sync();  // the consumers' stores happen before thread 0's (cumulative) release
          if (tid == 0) asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(&p.flags[t.r]) : "memory");
        }
        if (d.xsrc == nullptr) {
          // plain form: X_r = inv(T_rr) acc; the accumulator is the product's
          // X, staged in the X slots of its chunks (row k in the slot of
          // chunk k / 32; rows past the strip are the zero K tail) once every
          // consumer is done with the earlier chunks
          ts_consumer_sync();
          const int gd = gq + pi * cpp;
#pragma unroll
          for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int row = 16 * warp + g8 + ((e >= 2) ? 8 : 0), col = 8 * nt + 2 * t4 + (e & 1);
              double* sXr = sm + ((gd + row / kTsKC) % kTsStages) * kTsRStage + kTsRA;
              sXr[(row % kTsKC) + col * kTsCT] = row < t.mr ? acc[nt][e] : 0.0;
              acc[nt][e] = 0.0;
            }
          ts_consumer_sync();
        }
        const double sgn = d.step >= 0 ? -1.0 : 1.0;
        for (int c = 0; c < cpp; ++c) {
          const int g = gq + pi * cpp + c, slot = g % kTsStages;
          const uint32_t par = (uint32_t)(g / kTsStages) & 1u;
          if (!ts_mbar_wait(&fullA[slot], par) || !ts_mbar_wait(&fullX[slot], par)) {
            if (lane == 0) set_status(p.status, kTimeout, 213);
            return;
          }
          if (c * kTsKC < d.K && 16 * warp < t.mr) {
            const double* sA = sm + slot * kTsRStage;
            const double* sX = sA + kTsRA;
            const int ra = 16 * warp + g8;
#pragma unroll
            for (int kk = 0; kk < kTsKC; kk += 8) {
              double a[4];
              if (p.amode == 0) {
                a[0] = sgn * sA[ra + (kk + t4) * ldA];
                a[1] = sgn * sA[ra + 8 + (kk + t4) * ldA];
                a[2] = sgn * sA[ra + (kk + t4 + 4) * ldA];
                a[3] = sgn * sA[ra + 8 + (kk + t4 + 4) * ldA];
              } else {
                a[0] = sgn * sA[(kk + t4) + ra * kTsCT];
                a[1] = sgn * sA[(kk + t4) + (ra + 8) * kTsCT];
                a[2] = sgn * sA[(kk + t4 + 4) + ra * kTsCT];
                a[3] = sgn * sA[(kk + t4 + 4) + (ra + 8) * kTsCT];
              }
#pragma unroll
              for (int nt = 0; nt < NT; ++nt) {
                double bf[2];
                bf[0] = sX[(kk + t4) + (8 * nt + g8) * kTsCT];
                bf[1] = sX[(kk + t4 + 4) + (8 * nt + g8) * kTsCT];
                dmma_16x8x8(acc[nt], a, bf);
              }
            }
          }
          __syncwarp();
          // the slot's refill is a TMA write: order this warp's reads of it first
          if (lane == 0) {
            fence_proxy_async_smem();
            mbar_arrive(&empty[slot]);
          }
        }
      }
      gq += P * cpp;
      double* out = p.mode == 1 ? p.Y : p.X;
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int row = 16 * warp + g8 + ((e >= 2) ? 8 : 0), col = 8 * nt + 2 * t4 + (e & 1);
          if (row < t.mr && col < p.nrhs) out[(t.r0 + row) + (long long)col * p.ldx] = acc[nt][e];
        }
    }
    if (p.mode != 1 || t.mr <= 0) {  // publish x_r (every strip releases once, an empty one too)
      ts_consumer_sync();
      if (tid == 0) asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(&p.flags[t.r]) : "memory");
    }
  }
}

// NT: 8-column tiles of the right-hand side (a compile-time count: a DMMA
// skipped under a run-time predicate still costs its issue slots).
template <int NT>
__global__ void __launch_bounds__(kTsThreads, 1) trsm_skinny_kernel(const __grid_constant__ CUtensorMap mapL,
                                                                    const __grid_constant__ CUtensorMap mapW,
                                                                    TsParams p) {
  // TMA boxes land at stage starts: the dynamic region must be 128-byte
  // aligned (it follows the static barriers)
  extern __shared__ __align__(128) double sm[];
  __shared__ __align__(8) uint64_t fullA[kTsStages], fullX[kTsStages], empty[kTsStages];
  __shared__ int s_go;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int i = 0; i < kTsStages; ++i) {
      mbar_init(&fullA[i], 1);
      mbar_init(&fullX[i], kTsFullXCount);
      mbar_init(&empty[i], kTsEmptyCount);
    }
    fence_mbar_init();
    int go = p.status == nullptr || ((volatile DevStatus*)p.status)->code == 0;
    if (go && smem_u32(sm) % 128 != 0) {  // no TMA into a misaligned stage: report and stop
      set_status(p.status, kTimeout, 203);
      go = 0;
    }
    s_go = go;
  }
  __syncthreads();
  if (!s_go) return;
  if (tid >= kTsConsumers) ts_producer(&mapL, &mapW, p, sm, fullA, fullX, empty);
  else ts_consumers<NT>(p, sm, fullA, fullX, empty);
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
  // prescaled forms: two strips per block row, so the dependency chain's product is half a block,
  // while a CTA holds at most two tasks (its second task starts after the first and still has to
  // catch up with all the products of its block row)
  p.strips = (p.mode != 0 && nb >= 32 && p.nblk <= sm_count) ? 2 : 1;
  p.hs = p.strips == 1 ? nb : ((nb + 1) / 2 + 15) / 16 * 16;
  p.flags = flags; p.epoch = epoch; p.status = status;
  // the A pieces: TMA boxes over the stored n x n matrix and over the Winv
  // slots (nb rows x nblk*nb columns), the same box for both
  const uint32_t bi = amode == 0 ? (uint32_t)(p.hs + 4) : (uint32_t)kTsCT;
  const uint32_t bo = amode == 0 ? (uint32_t)kTsKC : (uint32_t)p.hs;
  CUtensorMap mapL, mapW;
  if (!make_tma_2d(&mapL, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, L, n, n, 8ull * lda, bi, bo, false) ||
      !make_tma_2d(&mapW, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, Winv, nb, (uint64_t)p.nblk * nb, 8ull * nb, bi, bo,
                   false))
    return EGPU_ERR_UNSUPPORTED;
  const size_t smem = sizeof(double) * kTsSmemDoubles;
  const int nt = nrhs <= 8 ? 1 : nrhs <= 16 ? 2 : nrhs <= 32 ? 4 : 8;
  void (*kern)(const CUtensorMap, const CUtensorMap, TsParams) = nt == 1   ? trsm_skinny_kernel<1>
                                                                 : nt == 2 ? trsm_skinny_kernel<2>
                                                                 : nt == 4 ? trsm_skinny_kernel<4>
                                                                           : trsm_skinny_kernel<8>;
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
  attr1[0].id = cudaLaunchAttributeCooperative;  // every CTA resident: the counter waits always end
  attr1[0].val.cooperative = 1;
  cfg.attrs = attr1;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, kern, mapL, mapW, p);
  count_launch();
  if (e != cudaSuccess) {
    set_last_error(e, "trsm_skinny launch", __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  }
  return EGPU_OK;
}

}  // namespace egpu
