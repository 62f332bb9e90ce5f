// FP32 triangular sweeps for the correction solves of the mixed-precision
// refinement: X := L^-1 X (forward), L^-T X (backward) or L^-T L^-1 X with L
// the low-precision Cholesky factor (FP32, lower triangle of the working
// matrix).
//
// The refinement's residual is FP64 and its corrections only need the
// accuracy of the factor itself (FP32), so the sweeps read L in FP32 and
// compute in FP32 (half the bytes of an FP64 copy, twice the SIMT rate).  The
// dependency chain of a triangular solve is cut to n / S steps by explicit
// inverses of the S x S diagonal super-blocks (S = 4 panels = 512):
//   forward, super-block R:  y_R = W_R (z0_R + dz_R)          (phase A)
//                            dz_Q -= L_QR y_R, Q > R + 1      (phase B)
//                            dz_R+1 -= M_R (z0_R + dz_R)      (kind 2)
//   backward, R downwards:   x_R = W_R^T (v_R + dv_R)          (phase A)
//                            dv_Q -= L_RQ^T x_R, Q < R - 1    (phase B)
//                            dv_R-1 -= P_R^T (v_R + dv_R)     (kind 2)
// with M_R = L_{R+1,R} W_R and P_R = W_R L_{R,R-1} formed once per factor:
// the next super-block's deltas then need the same input as phase A of R, so
// one step of the chain is one round of tile products instead of two.
// Every piece of work is a tile item -- out(128 x 32) += T(128 x k) v(k x 32)
// with T a 128-row tile of W_R, M_R, P_R or L read through TMA -- and one
// cooperative launch works through a queue of items in an order that
// respects their dependencies (R's kind-2 items and phase A of R, then the
// bulk phase-B items of the previous super-block, then R + 1's, ...).
// CTAs take items from an atomic counter, start the item's TMA tile loads at
// once, then wait (bounded) only for the counters of the items it depends on:
// phase A and the kind-2 items of Q wait for all delta items that target Q,
// phase B of R for the phase-A items of R.  Every item's dependencies lie
// earlier in the queue, so the co-resident CTAs always make progress; no grid
// barrier separates the steps, and the bulk of phase B overlaps the chain.
// All results are accumulated with FP32 vector reductions into arrays zeroed
// at the start.
//
// The super-block inverses are built once per factorization from the 128 x
// 128 diagonal-block inverses W_k (FP64, from the diagonal kernels) and the
// off-diagonal blocks of L: X_kk = W_k, X_ij = -W_i sum_{k=j}^{i-1} L_ik X_kj
// (block rows i = 1..3 of each super-block, one launch per i, all
// super-blocks at once), then M_R and P_R (one launch).
#include <vector>

#include "context.h"

namespace egpu {

namespace {

constexpr int kS = 512;          // super-block order
constexpr int kPB = 128;         // panel (block) order inside a super-block
constexpr int kTM = 128;         // tile: rows (M-contiguous) or columns (K-contiguous) of T
constexpr int kTK = 32;          // k per TMA stage
constexpr int kStages = 4;
constexpr int kThreads = 256;
constexpr int kRhs = 32;         // right-hand sides (nrhs <= 32 per launch)
// Granularity of the items on the sweep's chain: the k split of the next
// super-block's delta items and the k width of phase-A tiles (smaller: more,
// shorter items per chain step)
#ifndef EGPU_SWEEP_CRIT_SPLIT
#define EGPU_SWEEP_CRIT_SPLIT 4
#endif
#ifndef EGPU_SWEEP_A_K
#define EGPU_SWEEP_A_K 128
#endif
constexpr int kCritSplit = EGPU_SWEEP_CRIT_SPLIT;
constexpr int kAK = EGPU_SWEEP_A_K;
static_assert(kS % (kCritSplit * kTK) == 0 && kTM % kAK == 0 && kAK % kTK == 0, "chain item granularity");

// shared-memory carve (floats), 1024-byte aligned pieces
constexpr int kStageFloats = kTM * kTK;                     // 4096 floats = 16 KB
constexpr int kOffStages = 0;
constexpr int kOffV = kOffStages + kStages * kStageFloats;  // kS x kRhs floats = 64 KB
constexpr int kSmemFloats = kOffV + kS * kRhs;
constexpr int kSmemBytes = kSmemFloats * 4 + 1024 + 128;  // + alignment slack + mbarriers / scalars

// An item: out[out_row .. +128) (+/-)= T[tile] * v[v_row + kbeg .. v_row + kend)
struct Item {
  short map;      // 0 L (rows contiguous), 1 L (columns), 2 W (rows contiguous), 3 W (columns),
                  // 4 M (rows contiguous), 5 P (columns)
  short dir;      // 0 forward arrays, 1 backward arrays
  short kind;     // 0 phase A (out: y/x of super-block, +), 1 phase B (out: deltas, -),
                  // 2 the next super-block's deltas from phase A's input (M / P tile, -)
  short nk;       // TMA stages
  int tm;         // tile coordinate along M (row of T, or column of T for maps 1/3)
  int tk;         // coordinate of k = kbeg along K in the tensor
  int vrow;       // first row of v for k = kbeg
  int orow;       // first output row
  int orows;      // output rows valid (from orow)
  int dep0, need0;  // counter index and the count it must reach
  int dep1, need1;  // second dependency (or -1)
  int done;       // counter incremented on completion
};

struct SweepDF {
  int n, nrhs, items;
  const Item* table;
  float* Z0;   // n x 32: the right-hand side (X converted)
  float* Df;   // forward deltas
  float* Yf;   // forward results y
  float* Db;   // backward deltas
  float* Yb;   // backward results x
  double* X;   // in / out, FP64 column-major
  long long ldx;
  int out_backward;  // X := Yb (else Yf)
  int* counters;     // [0] queue, [1] abort, [2...] item counters; zeroed before launch
  unsigned* bar;     // grid barrier counter, zeroed before launch
  DevStatus* status;
};

__device__ __forceinline__ float* align1024(float* p) {
  return reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

// Bounded wait until *c >= need (thread 0).  false: timed out or aborted.
__device__ bool wait_counter(const int* c, int need, const int* abort) {
  for (long long it = 0; it < kSpinLimit; ++it) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(c) : "memory");
    if (v >= need) return true;
    int a;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(a) : "l"(abort) : "memory");
    if (a) return false;
    if (it > 16) __nanosleep(32);
  }
  return false;
}

__device__ __forceinline__ void issue(const CUtensorMap* map, bool mcontig, float* stages, uint64_t* full, int s,
                                      int tm, int kc) {
  mbar_expect_tx(&full[s], kStageFloats * 4);
  if (mcontig) {  // M-contiguous: 4 boxes of {32 rows, 32 k}
    for (int b = 0; b < kTM / 32; ++b)
      tma_load_2d(stages + s * kStageFloats + b * 32 * kTK, map, &full[s], tm + 32 * b, kc);
  } else {  // K-contiguous: one box {32 k, 128 columns}, 128-byte swizzle
    tma_load_2d(stages + s * kStageFloats, map, &full[s], kc, tm);
  }
}

__global__ void __launch_bounds__(kThreads, 1) sweep32_kernel(const __grid_constant__ CUtensorMap mL0,
                                                              const __grid_constant__ CUtensorMap mL1,
                                                              const __grid_constant__ CUtensorMap mW0,
                                                              const __grid_constant__ CUtensorMap mW1,
                                                              const __grid_constant__ CUtensorMap mM0,
                                                              const __grid_constant__ CUtensorMap mP1,
                                                              SweepDF p) {
  extern __shared__ float smem_raw[];
  float* sm = align1024(smem_raw);
  float* stages = sm + kOffStages;
  float* vs = sm + kOffV;
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + kSmemFloats);
  int* s_item = reinterpret_cast<int*>(full + kStages);
  int* s_ok = s_item + 1;
  const int tid = threadIdx.x;
  const int G = gridDim.x;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t phase_bits = 0;
  int* abort = p.counters + 1;

  // X (FP64, column-major) -> Z0; deltas and results zero
  const long long nz = (long long)p.n * kRhs;
  for (long long e = blockIdx.x * (long long)kThreads + tid; e < nz; e += (long long)G * kThreads) {
    const int r = (int)(e / kRhs), c = (int)(e % kRhs);
    p.Z0[e] = c < p.nrhs ? (float)p.X[r + (long long)c * p.ldx] : 0.f;
    p.Df[e] = 0.f; p.Yf[e] = 0.f; p.Db[e] = 0.f; p.Yb[e] = 0.f;
  }
  unsigned target = G;
  bool ok = grid_barrier(p.bar, target);

  const int rg = ((tid >> 5) & 3) * 8 + (tid & 7);   // 4-row (or 4-column) group 0..31
  const int cg = (tid >> 7) * 4 + ((tid >> 3) & 3);  // 4-rhs group 0..7
  while (ok) {
    if (tid == 0) *s_item = atomicAdd(p.counters, 1);
    __syncthreads();
    const int idx = *s_item;
    __syncthreads();
    if (idx >= p.items) break;
    const Item it = p.table[idx];
    const bool mcontig = it.map == 0 || it.map == 2 || it.map == 4;
    const CUtensorMap* mp = it.map == 0   ? &mL0
                            : it.map == 1 ? &mL1
                            : it.map == 2 ? &mW0
                            : it.map == 3 ? &mW1
                            : it.map == 4 ? &mM0
                                          : &mP1;
    // the tile does not depend on anything: start its loads now
    if (tid == 0) {
      for (int s = 0; s < min(kStages, (int)it.nk); ++s) issue(mp, mcontig, stages, full, s, it.tm, it.tk + s * kTK);
      bool w = wait_counter(p.counters + it.dep0, it.need0, abort);
      if (w && it.dep1 >= 0) w = wait_counter(p.counters + it.dep1, it.need1, abort);
      if (!w) {
        set_status(p.status, kTimeout, 9002);
        atomicExch(abort, 1);
      }
      *s_ok = w;
    }
    __syncthreads();
    ok = *s_ok != 0;
    // v rows [vrow, vrow + 32 nk) -> smem.  Phase A (and kind 2): forward
    // z0 + dz; backward (y, or z0 when only the backward sweep runs) + dv.
    // Phase B: the super-block's results y / x.  Four rows' loads are in
    // flight before any is stored.
    {
      const float* s0;
      const float* s1 = nullptr;
      if (it.kind != 1) {
        s0 = it.dir == 0 ? p.Z0 : (p.out_backward == 2 ? p.Yf : p.Z0);
        s1 = it.dir == 0 ? p.Df : p.Db;
      } else {
        s0 = it.dir == 0 ? p.Yf : p.Yb;
      }
      const int total = it.nk * kTK * (kRhs / 4);
      for (int e0 = tid; e0 < total; e0 += 4 * kThreads) {
        float4 v[4], d[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int e = e0 + u * kThreads;
          const int gr = it.vrow + e / (kRhs / 4), q = e % (kRhs / 4);
          v[u] = make_float4(0.f, 0.f, 0.f, 0.f);
          d[u] = v[u];
          if (e < total && gr < p.n) {
            v[u] = __ldcg(reinterpret_cast<const float4*>(s0 + (size_t)gr * kRhs) + q);
            if (s1 != nullptr) d[u] = __ldcg(reinterpret_cast<const float4*>(s1 + (size_t)gr * kRhs) + q);
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int e = e0 + u * kThreads;
          if (e < total) {
            const float4 w4 = make_float4(v[u].x + d[u].x, v[u].y + d[u].y, v[u].z + d[u].z, v[u].w + d[u].w);
            reinterpret_cast<float4*>(vs + (e / (kRhs / 4)) * kRhs)[e % (kRhs / 4)] = w4;
          }
        }
      }
    }
    __syncthreads();
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
    for (int ks = 0; ks < it.nk; ++ks) {
      const int s = ks % kStages;
      if (!mbar_wait_bounded(&full[s], (phase_bits >> s) & 1)) {
        if (tid == 0) {
          set_status(p.status, kTimeout, 9001);
          atomicExch(abort, 1);
        }
        ok = false;
      }
      phase_bits ^= 1u << s;
      const float* st = stages + s * kStageFloats;
      const float* vk = vs + ks * kTK * kRhs;
      if (mcontig) {
        // stage = 4 boxes of [32 k][32 rows]: row m = 32 b + q at [b][k][q]
        const int b = rg >> 3, q = (rg & 7) * 4;
#pragma unroll 8
        for (int k = 0; k < kTK; ++k) {
          const float4 lv = *reinterpret_cast<const float4*>(st + b * 32 * kTK + k * 32 + q);
          const float4 yv = *reinterpret_cast<const float4*>(vk + k * kRhs + cg * 4);
          const float l4[4] = {lv.x, lv.y, lv.z, lv.w}, y4[4] = {yv.x, yv.y, yv.z, yv.w};
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int bb = 0; bb < 4; ++bb) acc[a][bb] = fmaf(l4[a], y4[bb], acc[a][bb]);
        }
      } else {
        // stage = [128 columns j][32 k] with the 128-byte swizzle: 16-byte
        // chunk c of row j at chunk c ^ (j & 7); columns rg + 32 a
#pragma unroll 2
        for (int kc = 0; kc < kTK / 4; ++kc) {
          float l4[4][4];
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const int j = rg + 32 * a;
            const float4 v = *reinterpret_cast<const float4*>(st + j * kTK + ((kc ^ (j & 7)) << 2));
            l4[a][0] = v.x; l4[a][1] = v.y; l4[a][2] = v.z; l4[a][3] = v.w;
          }
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const float4 yv = *reinterpret_cast<const float4*>(vk + (kc * 4 + kk) * kRhs + cg * 4);
            const float y4[4] = {yv.x, yv.y, yv.z, yv.w};
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
              for (int bb = 0; bb < 4; ++bb) acc[a][bb] = fmaf(l4[a][kk], y4[bb], acc[a][bb]);
          }
        }
      }
      if (ks + kStages < it.nk) {  // stage s is refilled (item-uniform): every thread done with it first
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) issue(mp, mcontig, stages, full, s, it.tm, it.tk + (ks + kStages) * kTK);
      }
    }
    // out rows: phase A adds into the results, phase B and kind 2 subtract
    // into the deltas
    {
      float* out = it.kind == 0 ? (it.dir == 0 ? p.Yf : p.Yb) : (it.dir == 0 ? p.Df : p.Db);
      const float sg = it.kind == 0 ? 1.f : -1.f;
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const int m = mcontig ? rg * 4 + a : rg + 32 * a;
        if (m < it.orows) {
          float* z = out + (size_t)(it.orow + m) * kRhs + cg * 4;
          asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(z), "f"(sg * acc[a][0]),
                       "f"(sg * acc[a][1]), "f"(sg * acc[a][2]), "f"(sg * acc[a][3])
                       : "memory");
        }
      }
    }
    __threadfence();
    fence_proxy_async_smem();  // this item's stage reads before the next item's TMA writes
    __syncthreads();
    if (tid == 0) atomicAdd(p.counters + it.done, 1);
  }
  // the results to X once every item is done
  target += G;
  ok = grid_barrier(p.bar, target) && ok;
  const float* res = p.out_backward ? p.Yb : p.Yf;
  for (long long e = blockIdx.x * (long long)kThreads + tid; e < nz; e += (long long)G * kThreads) {
    const int r = (int)(e / kRhs), c = (int)(e % kRhs);
    if (c < p.nrhs) p.X[r + (long long)c * p.ldx] = (double)__ldcg(res + e);
  }
  if (!ok && tid == 0) set_status(p.status, kTimeout, 9000);
}

// ---- super-block inverses ----------------------------------------------

// C (128 x 128, FP32, column-major ldc) = sum over `terms` of A_t (128 x 128)
// B_t (128 x 128), A_t / B_t FP32 column-major; the result is scaled by
// `alpha` and stored.  256 threads, an 8 x 8 register tile each, k chunks of
// 32 through shared memory.
struct Prod {
  const float* A;
  long long lda;
  const float* B;
  long long ldb;
};

constexpr int kBsLd = 129;  // padded: consecutive k of one column land in distinct banks

// A rows from a_rows on, and rows k0 + k >= k_rows[t] of every B_t, read as
// zero (they may lie past the matrix); the output's rows [0, out_rows) x
// columns [0, out_cols) are stored.
__device__ void tile128_products(const Prod* prods, int terms, float alpha, float* C, long long ldc,
                                 float* As, float* Bs, int a_rows, int out_rows, int out_cols,
                                 const int* k_rows = nullptr) {
  const int tid = threadIdx.x;
  const int tr = (tid & 15) * 8, tc = (tid >> 4) * 8;
  float acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = 0.f;
  for (int t = 0; t < terms; ++t) {
    for (int k0 = 0; k0 < kPB; k0 += 32) {
      // As[k][128 rows] = A(:, k0 + k); Bs[k][128 cols] = B(k0 + k, :)
      for (int e = tid; e < 32 * 128; e += kThreads) {
        const int k = e >> 7, r = e & 127;
        As[k * 128 + r] = r < a_rows ? prods[t].A[r + (long long)(k0 + k) * prods[t].lda] : 0.f;
      }
      const int kr = k_rows ? k_rows[t] : kPB;
      for (int e = tid; e < 32 * 128; e += kThreads) {  // consecutive threads: consecutive k
        const int k = e & 31, c = e >> 5;
        Bs[k * kBsLd + c] = (k0 + k) < kr ? prods[t].B[(k0 + k) + (long long)c * prods[t].ldb] : 0.f;
      }
      __syncthreads();
#pragma unroll 4
      for (int k = 0; k < 32; ++k) {
        float a8[8], b8[8];
#pragma unroll
        for (int a = 0; a < 8; ++a) a8[a] = As[k * 128 + tr + a];
#pragma unroll
        for (int b = 0; b < 8; ++b) b8[b] = Bs[k * kBsLd + tc + b];
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
          for (int b = 0; b < 8; ++b) acc[a][b] = fmaf(a8[a], b8[b], acc[a][b]);
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int b = 0; b < 8; ++b)
#pragma unroll
    for (int a = 0; a < 8; ++a)
      if (tr + a < out_rows && tc + b < out_cols) C[(tr + a) + (long long)(tc + b) * ldc] = alpha * acc[a][b];
}

// W (FP64 nb x nb blocks, ld nb) -> the diagonal blocks of every super-block
// in Wc (FP32); the rest of Wc zero.
__global__ void superinv_init_kernel(int n, int nsuper, const double* Winv, float* Wc) {
  const long long total = (long long)nsuper * kS * kS;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int R = (int)(e / ((long long)kS * kS));
    const int rem = (int)(e % ((long long)kS * kS));
    const int i = rem % kS, j = rem / kS;  // column-major in the super-block
    const int bi = i / kPB, bj = j / kPB;
    float v = 0.f;
    const int gi = R * kS + i, gj = R * kS + j;
    if (bi == bj && gi < n && gj < n) {
      const int k = R * (kS / kPB) + bi;  // global panel index
      v = (float)Winv[(size_t)k * kPB * kPB + (i % kPB) + (size_t)(j % kPB) * kPB];
    }
    Wc[e] = v;
  }
}

// Block row `bi` (1..3) of every super-block: for j < bi,
//   T = sum_{k=j}^{bi-1} L(bi, k) X(k, j),  X(bi, j) = -W_bi T
// one CTA per (super-block, j); T in the output slot first, then W_bi T into
// the temporary and copied back.
__global__ void __launch_bounds__(kThreads) superinv_row_kernel(int n, int nsuper, int bi, const float* L,
                                                                long long ldl, float* Wc, float* tmp) {
  extern __shared__ float sh[];
  float* As = sh;
  float* Bs = sh + 32 * 128;  // 32 x kBsLd
  const int R = blockIdx.y, j = blockIdx.x;
  if (j >= bi) return;
  const int r0 = R * kS;
  if (r0 + bi * kPB >= n) return;  // block row past the matrix
  float* X = Wc + (size_t)R * kS * kS;
  Prod prods[3];
  int terms = 0;
  for (int k = j; k < bi; ++k) {
    prods[terms].A = L + (r0 + bi * kPB) + (long long)(r0 + k * kPB) * ldl;  // L(bi, k)
    prods[terms].lda = ldl;
    prods[terms].B = X + k * kPB + (size_t)(j * kPB) * kS;  // X(k, j)
    prods[terms].ldb = kS;
    ++terms;
  }
  const int rows_valid = min(kPB, n - (r0 + bi * kPB));
  float* T = tmp + ((size_t)R * 4 + j) * kPB * kPB;  // 128 x 128, ld 128
  // T is written whole (rows past the matrix are zero): the next product
  // reads all of it, and stale workspace contents times W's zero columns
  // would otherwise give 0 * NaN
  tile128_products(prods, terms, 1.f, T, kPB, As, Bs, rows_valid, kPB, kPB);
  __syncthreads();
  __threadfence_block();
  Prod w;
  w.A = X + bi * kPB + (size_t)(bi * kPB) * kS;  // X(bi, bi) = W_bi
  w.lda = kS;
  w.B = T;
  w.ldb = kPB;
  tile128_products(&w, 1, -1.f, X + bi * kPB + (size_t)(j * kPB) * kS, kS, As, Bs, kPB, rows_valid, kPB);
}

// The products that put one super-block step of each sweep on one phase:
//   forward  (z = 0):  M_R = L_{R+1,R} W_R   for R = 0 .. nsuper - 2, in Mc
//   backward (z = 1):  P_R = W_R L_{R,R-1}   for R = 1 .. nsuper - 1, in Pc
// (Mc / Pc: kS rows, block R at columns R kS .. R kS + kS - 1, ld kS, as Wc.)
// One CTA per 128 x 128 output tile (blockIdx.x = 4 mt + nt); W_R is lower
// triangular, so only the k blocks where it is nonzero are multiplied.  Rows
// and k indices past the matrix read as zero and every tile is written whole.
__global__ void __launch_bounds__(kThreads) superprod_kernel(int n, int nsuper, const float* L, long long ldl,
                                                             const float* Wc, float* Mc, float* Pc) {
  extern __shared__ float sh[];
  float* As = sh;
  float* Bs = sh + 32 * 128;
  const int mt = blockIdx.x >> 2, nt = blockIdx.x & 3;
  const int z = blockIdx.z;
  const int R = z == 0 ? (int)blockIdx.y : (int)blockIdx.y + 1;
  const float* W = Wc + (size_t)R * kS * kS;
  Prod prods[4];
  int kr[4];
  int terms = 0, a_rows = kPB;
  if (z == 0) {  // M_R(mt, nt) = sum_t L_{R+1,R}(mt, t) W_R(t, nt), t >= nt
    const long long r0 = (long long)(R + 1) * kS + mt * kPB;
    a_rows = (int)max(0LL, min((long long)kPB, (long long)n - r0));
    for (int t = nt; t < 4; ++t) {
      prods[terms].A = L + r0 + (long long)(R * kS + t * kPB) * ldl;
      prods[terms].lda = ldl;
      prods[terms].B = W + t * kPB + (size_t)(nt * kPB) * kS;
      prods[terms].ldb = kS;
      kr[terms] = kPB;
      ++terms;
    }
    if (a_rows == 0) terms = 0;  // the tile lies past the matrix: zeros
  } else {  // P_R(mt, nt) = sum_t W_R(mt, t) L_{R,R-1}(t, nt), t <= mt, rows of R inside the matrix
    for (int t = 0; t <= mt; ++t) {
      const long long k0 = (long long)R * kS + t * kPB;
      if (k0 >= n) break;
      prods[terms].A = W + mt * kPB + (size_t)(t * kPB) * kS;
      prods[terms].lda = kS;
      prods[terms].B = L + k0 + (long long)((R - 1) * kS + nt * kPB) * ldl;
      prods[terms].ldb = ldl;
      kr[terms] = (int)min((long long)kPB, (long long)n - k0);
      ++terms;
    }
  }
  float* out = (z == 0 ? Mc : Pc) + (size_t)R * kS * kS + mt * kPB + (size_t)(nt * kPB) * kS;
  tile128_products(prods, terms, 1.f, out, kS, As, Bs, a_rows, kPB, kPB, kr);
}

}  // namespace

// ---- host: the item queue --------------------------------------------

// Counter layout: [0] queue, [1] abort, then per direction d and super-block R:
// cY(d, R) (phase-A items of R done), cD(d, R) (phase-B items targeting R done).
struct CounterIx {
  int nsuper;
  int cy(int d, int R) const { return 2 + (d * nsuper + R) * 2; }
  int cd(int d, int R) const { return 3 + (d * nsuper + R) * 2; }
  int count() const { return 2 + 4 * nsuper; }
};

// Items of one sweep direction in dependency order.  G: grid size (decides
// how finely the bulk phase-B tiles are split along k).
static void build_items(int n, int G, int dir, bool after_forward, std::vector<Item>& out, const CounterIx& cx) {
  const int nsuper = (n + kS - 1) / kS;
  auto sb_of = [&](int R) { return std::min(kS, n - R * kS); };
  std::vector<int> cd_need(nsuper, 0);  // delta items (kinds 1 and 2) that will target each super-block
  // Delta items of super-block R: critical -- the next super-block of the
  // sweep, from the M_R / P_R products and phase A's input (kind 2, k split
  // kCritSplit ways), so they run beside phase A of R -- or bulk (phase B,
  // the others)
  auto b_items = [&](int R, bool critical, std::vector<Item>& v) {
    const int r0 = R * kS, sb = sb_of(R);
    // targets: forward rows of later super-blocks; backward columns of earlier ones
    std::vector<int> targets;
    if (dir == 0)
      for (int Q = R + 1; Q < nsuper; ++Q) targets.push_back(Q);
    else
      for (int Q = R - 1; Q >= 0; --Q) targets.push_back(Q);
    int bulk_tiles = 0;
    for (size_t t = 1; t < targets.size(); ++t) bulk_tiles += (sb_of(targets[t]) + kTM - 1) / kTM;
    int ksplit_bulk = 1;
    while (ksplit_bulk < 4 && bulk_tiles * ksplit_bulk * 2 <= G) ksplit_bulk *= 2;
    for (size_t t = critical ? 0 : 1; t < (critical ? std::min<size_t>(1, targets.size()) : targets.size()); ++t) {
      const int Q = targets[t], q0 = Q * kS, sq = sb_of(Q);
      const int ksplit = t == 0 ? kCritSplit : ksplit_bulk;  // the next super-block's items are on the chain
      const int kch = kS / ksplit;
      for (int m = 0; m < sq; m += kTM)
        for (int kp = 0; kp < ksplit; ++kp) {
          const int kb = kp * kch, ke = std::min(sb, kb + kch);
          if (ke <= kb) continue;
          Item it{};
          it.dir = dir;
          it.nk = (ke - kb + kTK - 1) / kTK;
          it.vrow = r0 + kb;
          it.orow = q0 + m;
          it.orows = std::min(kTM, sq - m);
          it.need0 = 0;  // filled below
          it.dep1 = -1;
          if (critical) {
            // forward: rows m of M_R (block R at Mc columns R kS ..); backward:
            // columns R kS + m of Pc, k along P_R's rows
            it.map = dir == 0 ? 4 : 5;
            it.kind = 2;
            it.tm = dir == 0 ? m : R * kS + m;
            it.tk = dir == 0 ? R * kS + kb : kb;
            it.dep0 = cx.cd(dir, R);
            if (dir == 1 && after_forward) {  // its input y_R: the forward phase A of R
              it.dep1 = cx.cy(0, R);
              it.need1 = 0;  // filled by the caller
            }
          } else {
            it.map = dir == 0 ? 0 : 1;
            it.kind = 1;
            it.tm = q0 + m;      // forward: rows of L; backward: columns of L
            it.tk = r0 + kb;     // forward: columns of L; backward: rows of L
            it.dep0 = cx.cy(dir, R);
          }
          it.done = cx.cd(dir, Q);
          ++cd_need[Q];
          v.push_back(it);
        }
    }
  };
  auto a_items = [&](int R, std::vector<Item>& v) {
    const int r0 = R * kS, sb = sb_of(R);
    for (int mt = 0; mt < sb; mt += kTM)
      for (int kt = 0; kt < sb; kt += kAK) {
        // W_R lower: the forward tile (rows mt.., k kt..) is nonzero when
        // kt < mt + kTM; W_R^T upper: when kt + kAK > mt
        if (dir == 0 ? kt >= mt + kTM : kt + kAK <= mt) continue;
        Item it{};
        it.map = dir == 0 ? 2 : 3;
        it.dir = dir;
        it.kind = 0;
        it.nk = (std::min(kAK, sb - kt) + kTK - 1) / kTK;
        // W_R block in the (kS x kS nsuper) tensor: rows i, columns R kS + j
        it.tm = dir == 0 ? mt : R * kS + mt;
        it.tk = dir == 0 ? R * kS + kt : kt;
        it.vrow = r0 + kt;
        it.orow = r0 + mt;
        it.orows = std::min(kTM, sb - mt);
        it.dep0 = cx.cd(dir, R);
        it.need0 = 0;  // filled below
        it.dep1 = -1;
        if (dir == 1 && after_forward) {  // x_R needs y_R: all forward phase-A items of R
          it.dep1 = cx.cy(0, R);
          it.need1 = 0;  // filled by the caller
        }
        it.done = cx.cy(dir, R);
        v.push_back(it);
      }
  };
  const size_t first = out.size();
  // dependency order with the chain first: R's items for the next
  // super-block and phase A of R (both wait for the deltas of R only), then
  // the bulk of the previous super-block's phase B (phase A of R + 1 needs
  // those and R's critical items, all queued before it)
  for (int s = 0; s <= nsuper; ++s) {
    const int R = dir == 0 ? s : nsuper - 1 - s;
    const int Rp = dir == 0 ? s - 1 : nsuper - s;  // the previous super-block of the sweep
    if (s < nsuper) b_items(R, true, out);
    if (s < nsuper) a_items(R, out);
    if (s >= 1) b_items(Rp, false, out);
  }
  // needs: phase A of R and R's critical items wait for every delta item
  // targeting R; phase B of R for all phase-A items of R
  std::vector<int> a_count(nsuper, 0);
  for (size_t i = first; i < out.size(); ++i)
    if (out[i].kind == 0) ++a_count[(out[i].orow) / kS];
  for (size_t i = first; i < out.size(); ++i) {
    Item& it = out[i];
    if (it.kind == 0) it.need0 = cd_need[it.orow / kS];
    else if (it.kind == 2) it.need0 = cd_need[it.vrow / kS];
    else it.need0 = a_count[it.vrow / kS];
  }
}

// The whole queue of one launch: forward (trans 0), backward (1) or both
// (2), the backward phase A and kind-2 items of R then also waiting for the
// forward phase A of R (whose y they read).
static void build_queue(int n, int trans, int sm_count, std::vector<Item>& items) {
  const int nsuper = (n + kS - 1) / kS;
  const CounterIx cx{nsuper};
  if (trans == 0 || trans == 2) build_items(n, sm_count, 0, false, items, cx);
  if (trans == 1 || trans == 2) {
    const size_t b0 = items.size();
    build_items(n, sm_count, 1, trans == 2, items, cx);
    if (trans == 2) {
      std::vector<int> ay(nsuper, 0);
      for (size_t i = 0; i < b0; ++i)
        if (items[i].kind == 0) ++ay[items[i].orow / kS];
      for (size_t i = b0; i < items.size(); ++i)  // the super-block whose y the item reads
        if (items[i].dep1 >= 0) items[i].need1 = ay[(items[i].kind == 2 ? items[i].vrow : items[i].orow) / kS];
    }
  }
}

size_t sweep32_ws_bytes(int n, int nrhs) {
  (void)nrhs;
  const int nsuper = (n + kS - 1) / kS;
  size_t b = 0;
  b += (size_t)nsuper * kS * kS * sizeof(float) + 1024;      // Wc
  b += 2 * ((size_t)nsuper * kS * kS * sizeof(float) + 1024);  // Mc, Pc
  b += (size_t)nsuper * 4 * kPB * kPB * sizeof(float);       // temporaries of the inverse
  b += 5 * ((size_t)n * kRhs * sizeof(float) + 1024);        // Z0, Df, Yf, Db, Yb
  b += (size_t)(2 + 4 * nsuper) * sizeof(int) + 1024;        // counters
  b += 1024;                                                  // barrier
  b += (size_t)2 * (nsuper * (4 * (kS / kAK) + 4 * kCritSplit) + nsuper * nsuper * 16 + 64) * sizeof(Item) +
       1024;  // item table (bound)
  return b + 16 * 1024;  // every piece is 1024-aligned
}

namespace {
struct SweepWs {
  float *Wc, *Mc, *Pc, *tmp, *Z0, *Df, *Yf, *Db, *Yb;
  int* counters;
  unsigned* bar;
  Item* table;
};
SweepWs carve(void* ws, int n) {
  const int nsuper = (n + kS - 1) / kS;
  SweepWs w;
  uintptr_t b = reinterpret_cast<uintptr_t>(ws);
  auto take = [&](size_t bytes) { b = align_up(b, 1024); uintptr_t o = b; b += bytes; return o; };
  w.Wc = reinterpret_cast<float*>(take((size_t)nsuper * kS * kS * sizeof(float)));
  w.Mc = reinterpret_cast<float*>(take((size_t)nsuper * kS * kS * sizeof(float)));
  w.Pc = reinterpret_cast<float*>(take((size_t)nsuper * kS * kS * sizeof(float)));
  w.tmp = reinterpret_cast<float*>(take((size_t)nsuper * 4 * kPB * kPB * sizeof(float)));
  w.Z0 = reinterpret_cast<float*>(take((size_t)n * kRhs * sizeof(float)));
  w.Df = reinterpret_cast<float*>(take((size_t)n * kRhs * sizeof(float)));
  w.Yf = reinterpret_cast<float*>(take((size_t)n * kRhs * sizeof(float)));
  w.Db = reinterpret_cast<float*>(take((size_t)n * kRhs * sizeof(float)));
  w.Yb = reinterpret_cast<float*>(take((size_t)n * kRhs * sizeof(float)));
  w.counters = reinterpret_cast<int*>(take((size_t)(2 + 4 * nsuper) * sizeof(int)));
  w.bar = reinterpret_cast<unsigned*>(take(256));
  w.table = reinterpret_cast<Item*>(take(0));
  return w;
}
}  // namespace

// Build the super-block inverses from L (FP32, ld ldl) and the FP64 panel
// inverses Winv (nb = 128, one nb x nb block per panel).  ws: sweep32_ws_bytes.
int sweep32_prepare(cudaStream_t st, int n, const float* L, long long ldl, const double* Winv, void* ws) {
  const int nsuper = (n + kS - 1) / kS;
  const SweepWs w = carve(ws, n);
  TraceMark tm(st, kTraceOther, (double)nsuper * 4.0 * kS * kS * kS / 3.0, 12.0 * nsuper * kS * kS);
  superinv_init_kernel<<<std::min<long long>(((long long)nsuper * kS * kS + 255) / 256, 148 * 16), 256, 0, st>>>(
      n, nsuper, Winv, w.Wc);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  static bool attr = false;
  const int shb = (32 * 128 + 32 * kBsLd) * (int)sizeof(float);
  if (!attr) {
    EGPU_CUDA_TRY(cudaFuncSetAttribute(superinv_row_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, shb));
    attr = true;
  }
  for (int bi = 1; bi < kS / kPB; ++bi) {
    superinv_row_kernel<<<dim3(bi, nsuper), kThreads, shb, st>>>(n, nsuper, bi, L, ldl, w.Wc, w.tmp);
    count_launch();
    EGPU_CUDA_TRY(cudaGetLastError());
  }
  if (nsuper > 1) {  // the one-phase chain products M_R and P_R (shb < 48 KB: no attribute needed)
    TraceMark tp(st, kTraceOther, 2.0 * (nsuper - 1) * 2.0 * kS * kS * kS * 0.625, 24.0 * (nsuper - 1) * kS * kS);
    superprod_kernel<<<dim3(16, nsuper - 1, 2), kThreads, shb, st>>>(n, nsuper, L, ldl, w.Wc, w.Mc, w.Pc);
    count_launch();
    EGPU_CUDA_TRY(cudaGetLastError());
  }
  return EGPU_OK;
}

// X := L^-1 X (trans 0), L^-T X (trans 1) or L^-T L^-1 X (trans 2); X FP64 n
// x nrhs (nrhs <= 32, ld ldx), L FP32 (ld ldl, 16-byte aligned base and ld a
// multiple of 4), ws prepared by sweep32_prepare for this L.
int sweep32_solve(cudaStream_t st, int trans, int n, int nrhs, const float* L, long long ldl, double* X,
                  long long ldx, void* ws, int sm_count, DevStatus* status) {
  if (n <= 0 || nrhs <= 0) return EGPU_OK;
  if (nrhs > kRhs || trans < 0 || trans > 2) return EGPU_ERR_UNSUPPORTED;
  if (reinterpret_cast<uintptr_t>(L) % 16 != 0 || ldl % 4 != 0) return EGPU_ERR_ALIGN;
  const int nsuper = (n + kS - 1) / kS;
  const SweepWs w = carve(ws, n);
  const CounterIx cx{nsuper};
  std::vector<Item> items;
  build_queue(n, trans, sm_count, items);
  CUtensorMap m[6];
  // L: {n rows, n columns}; W: {kS rows, kS * nsuper columns}
  if (!make_tma_2d(&m[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, L, n, n, ldl * 4, 32, kTK, false) ||
      !make_tma_2d(&m[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, L, n, n, ldl * 4, kTK, kTM, true) ||
      !make_tma_2d(&m[2], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, w.Wc, kS, (uint64_t)kS * nsuper, kS * 4, 32, kTK, false) ||
      !make_tma_2d(&m[3], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, w.Wc, kS, (uint64_t)kS * nsuper, kS * 4, kTK, kTM, true) ||
      !make_tma_2d(&m[4], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, w.Mc, kS, (uint64_t)kS * nsuper, kS * 4, 32, kTK, false) ||
      !make_tma_2d(&m[5], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, w.Pc, kS, (uint64_t)kS * nsuper, kS * 4, kTK, kTM, true))
    return EGPU_ERR_TMA;
  static int attr_dev_mask = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 31 && !(attr_dev_mask & (1 << dev))) {
    EGPU_CUDA_TRY(cudaFuncSetAttribute(sweep32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
    attr_dev_mask |= 1 << dev;
  }
  EGPU_CUDA_TRY(cudaMemcpyAsync(w.table, items.data(), sizeof(Item) * items.size(), cudaMemcpyHostToDevice, st));
  EGPU_CUDA_TRY(cudaMemsetAsync(w.counters, 0, sizeof(int) * cx.count(), st));
  EGPU_CUDA_TRY(cudaMemsetAsync(w.bar, 0, sizeof(unsigned), st));
  SweepDF p;
  p.n = n; p.nrhs = nrhs; p.items = (int)items.size(); p.table = w.table;
  p.Z0 = w.Z0; p.Df = w.Df; p.Yf = w.Yf; p.Db = w.Db; p.Yb = w.Yb;
  p.X = X; p.ldx = ldx;
  p.out_backward = trans == 0 ? 0 : (trans == 2 ? 2 : 1);
  p.counters = w.counters; p.bar = w.bar; p.status = status;
  TraceMark tm(st, kTraceSolve, (trans == 2 ? 2.0 : 1.0) * n * n * nrhs,
               (trans == 2 ? 2.0 : 1.0) * (2.0 * n * n + 16.0 * n * nrhs));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(sm_count);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kSmemBytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  EGPU_CUDA_TRY(cudaLaunchKernelEx(&cfg, sweep32_kernel, m[0], m[1], m[2], m[3], m[4], m[5], p));
  count_launch();
  // (a copy from pageable host memory returns once the data is staged, so the
  // table's host vector may go)
  return EGPU_OK;
}

// ---- test / profiling entry --------------------------------------------

namespace {
// D (FP64, ld ldd) = the lower b x b diagonal blocks of L (FP32): block q of
// size min(128, n - 128 q) at D + 128 q (1 + ldd)
__global__ void widen_diag_blocks_kernel(int n, const float* L, long long ldl, double* D, long long ldd) {
  const int q = blockIdx.x, b = min(kPB, n - q * kPB);
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int i = e % b, j = e / b;
    const long long r = (long long)q * kPB + i, c = (long long)q * kPB + j;
    D[r + c * ldd] = i >= j ? (double)L[r + c * ldl] : 0.0;
  }
}
}  // namespace

}  // namespace egpu

using namespace egpu;

// Host-only view of the queue (no device work): 14 ints per item.
extern "C" int egpu_sweep32_queue(int n, int trans, int sm_count, int* out, int max_items) {
  if (n < 1 || trans < 0 || trans > 2 || sm_count < 1 || max_items < 0) return EGPU_ERR_ARG;
  std::vector<Item> items;
  build_queue(n, trans, sm_count, items);
  const int cnt = (int)items.size();
  if (out != nullptr) {
    for (int i = 0; i < std::min(cnt, max_items); ++i) {
      const Item& it = items[i];
      const int v[14] = {it.map, it.dir, it.kind, it.nk, it.tm, it.tk, it.vrow, it.orow, it.orows,
                         it.dep0, it.need0, it.dep1, it.need1, it.done};
      for (int k = 0; k < 14; ++k) out[(size_t)i * 14 + k] = v[k];
    }
  }
  return cnt;
}

extern "C" int egpu_sweep32_solve(egpu_handle h, int trans, int n, int nrhs, const float* dL, int ldl, double* dX,
                                  int ldx) {
  if (!h) return EGPU_ERR_ARG;
  if (n < 0 || nrhs < 0 || nrhs > 32 || ldl < std::max(1, n) || ldx < std::max(1, n) || trans < 0 || trans > 2)
    return EGPU_ERR_ARG;
  if (n == 0 || nrhs == 0) return EGPU_OK;
  Enter en(h);
  const long long ldd = ld_aligned(n);
  const size_t dbytes = align_up(sizeof(double) * (size_t)ldd * n, 1024);
  const size_t wbytes = align_up(winv_bytes(n, kPB), 1024);
  TRY(ensure_ws(h, dbytes + wbytes + sweep32_ws_bytes(n, nrhs) + 4096));
  unsigned char* ws = static_cast<unsigned char*>(h->ws);
  double* D = reinterpret_cast<double*>(ws);
  double* Winv = reinterpret_cast<double*>(ws + dbytes);
  void* sw = ws + dbytes + wbytes;
  cudaStream_t st = h->stream;
  EGPU_CUDA_TRY(cudaMemsetAsync(h->dstatus, 0, sizeof(DevStatus), st));
  widen_diag_blocks_kernel<<<(n + kPB - 1) / kPB, 256, 0, st>>>(n, dL, ldl, D, ldd);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  TRY(launch_trtri_blocks(st, EGPU_LOWER, 0, D, ldd, n, kPB, Winv, kPB));
  TRY(sweep32_prepare(st, n, dL, ldl, Winv, sw));
  TRY(sweep32_solve(st, trans, n, nrhs, dL, ldl, dX, ldx, sw, h->sm_count, h->dstatus));
  return read_status_now(h, nullptr);
}
