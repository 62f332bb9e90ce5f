// FP32 triangular sweeps for the correction solves of the mixed-precision
// refinement: X := L^-1 X (forward) or X := L^-T X (backward) with L the
// low-precision Cholesky factor (FP32, lower triangle of the working matrix).
//
// The refinement's residual is FP64 and its corrections only need the
// accuracy of the factor itself (FP32), so the sweeps read L in FP32 and
// compute in FP32 (half the bytes of an FP64 copy, twice the SIMT rate).  The
// dependency chain of a triangular solve is cut to n / S steps by explicit
// inverses of the S x S diagonal super-blocks (S = 4 panels = 512):
//   forward, super-block R:  y_R = W_R z_R              (phase A)
//                            z_i -= L_iR y_R, i > R      (phase B)
//   backward, R downwards:   x_R = W_R^T v_R            (phase A)
//                            v_j -= L_Rj^T x_R, j < R    (phase B)
// One cooperative launch runs all super-steps with two bounded grid
// barriers each.  Phase A spreads the rows of W_R over the grid (a warp per
// row, W_R's rows read contiguously from the copy laid out for the
// direction); phase B deals 128-row (forward) or 128-column (backward) tiles
// of L out to the CTAs, each streaming its 128 x 512 block of L through a
// TMA ring (32 columns or rows per stage) against y_R / x_R held in shared
// memory, 4 x 4 register tiles per thread.
//
// The super-block inverses are built once per factorization from the 128 x
// 128 diagonal-block inverses W_k (FP64, from the diagonal kernels) and the
// off-diagonal blocks of L: X_kk = W_k, X_ij = -W_i sum_{k=j}^{i-1} L_ik X_kj
// (block rows i = 1..3 of each super-block, one launch per i, all
// super-blocks at once).
#include "context.h"

namespace egpu {

namespace {

constexpr int kS = 512;          // super-block order
constexpr int kPB = 128;         // panel (block) order inside a super-block
constexpr int kTM = 128;         // phase-B tile: rows (forward) / columns (backward)
constexpr int kTK = 32;          // k per TMA stage
constexpr int kStages = 4;
constexpr int kThreads = 256;
constexpr int kRhs = 32;         // right-hand sides per pass

// shared-memory carve (floats), 1024-byte aligned pieces
constexpr int kStageFloats = kTM * kTK;                 // 4096 floats = 16 KB
constexpr int kOffStages = 0;
constexpr int kOffY = kOffStages + kStages * kStageFloats;  // kS x kRhs floats = 64 KB
constexpr int kSmemFloats = kOffY + kS * kRhs;
constexpr int kSmemBytes = kSmemFloats * 4 + 1024 + 64;  // + alignment slack + mbarriers

struct Sweep32Params {
  int n, nrhs, trans, nsuper;
  const float* Wc;   // W_R column-major (S x S per super-block, stride S*S)
  const float* Wr;   // W_R row-major
  float* Z;          // n x ldz row-major work (right-hand sides contiguous)
  int ldz;
  float* Yb;         // S x ldz row-major: y_R / x_R of the current super-block
  double* X;         // in: right-hand side, out: solution (FP64, column-major)
  long long ldx;
  unsigned* counter; // grid barrier counter, zero at launch
  DevStatus* status;
};

__device__ __forceinline__ float* align1024(float* p) {
  return reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

// Phase A: rows of the current super-block, a warp per row.  out = Wrow * zs
// over k in [klo, khi); zs = the super-block's right-hand sides (sb x 32).
// The row's W values are loaded first (up to 16 per lane, all in flight at
// once), then broadcast with shuffles.  Results go to Yb (and to X when
// write_x).
__device__ void phase_a(const Sweep32Params& p, const float* Wrow_base, bool lower_rows, int r0, int sb, int pass,
                        const float* zs, bool write_x) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gw = blockIdx.x * (kThreads / 32) + warp, nw = gridDim.x * (kThreads / 32);
  const int c = pass * kRhs + lane;
  for (int i = gw; i < sb; i += nw) {
    // forward: W_R row i, k = 0..i (W_R lower); backward: W_R^T row i = W_R
    // column i, k = i..sb-1
    const int klo = lower_rows ? 0 : i, khi = lower_rows ? i + 1 : sb;
    const float* w = Wrow_base + (size_t)i * kS;
    float wl[kS / 32];
#pragma unroll
    for (int q = 0; q < kS / 32; ++q) {
      const int k = q * 32 + lane;
      wl[q] = (k >= klo && k < khi) ? w[k] : 0.f;
    }
    float acc = 0.f, acc2 = 0.f;  // two chains: even and odd k
#pragma unroll
    for (int q = 0; q < kS / 32; ++q) {
      if (q * 32 >= khi || q * 32 + 32 <= klo) continue;
#pragma unroll
      for (int t = 0; t < 32; t += 2) {
        acc = fmaf(__shfl_sync(0xffffffffu, wl[q], t), zs[(q * 32 + t) * kRhs + lane], acc);
        acc2 = fmaf(__shfl_sync(0xffffffffu, wl[q], t + 1), zs[(q * 32 + t + 1) * kRhs + lane], acc2);
      }
    }
    acc += acc2;
    p.Yb[(size_t)i * p.ldz + c] = acc;
    if (write_x && c < p.nrhs) p.X[(r0 + i) + (long long)c * p.ldx] = (double)acc;
  }
}

// Stage rows [0, rows) x 32 columns (pass) of a row-major array into smem
// (rows beyond `rows` up to kS are zero).
__device__ void stage_rows(float* dst, const float* src, int ldz, int rows, int pass) {
  for (int e = threadIdx.x; e < kS * (kRhs / 4); e += kThreads) {
    const int r = e / (kRhs / 4), q = e % (kRhs / 4);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (r < rows) v = __ldcg(reinterpret_cast<const float4*>(src + (size_t)r * ldz + pass * kRhs) + q);
    reinterpret_cast<float4*>(dst + r * kRhs)[q] = v;
  }
}

// The phase-B work items of one super-step: tiles of 128 rows (forward) or
// columns (backward) of the trailing part, each tile's k range split into
// `ksplit` parts when there are few tiles.
struct BItems {
  int lo, hi, ntiles, ksplit, kchunk, items;
};
__device__ __forceinline__ BItems b_items(int fwd, int n, int r0, int r1, int G) {
  BItems b;
  b.lo = fwd ? r1 : 0;
  b.hi = fwd ? n : r0;
  b.ntiles = b.hi > b.lo ? (b.hi - b.lo + kTM - 1) / kTM : 0;
  b.ksplit = 1;
  while (b.ksplit < 4 && b.ntiles * b.ksplit * 2 <= G) b.ksplit *= 2;
  b.kchunk = kS / b.ksplit;
  b.items = b.ntiles * b.ksplit;
  return b;
}

// Issue the TMA loads of k-stage `kn` of an item into ring slot `s`.
__device__ __forceinline__ void issue_stage(const CUtensorMap* mapF, const CUtensorMap* mapB, int fwd, float* stages,
                                            uint64_t* full, int s, int m0, int kglob) {
  mbar_expect_tx(&full[s], kStageFloats * 4);
  if (fwd) {
    for (int b = 0; b < kTM / 32; ++b)
      tma_load_2d(stages + s * kStageFloats + b * 32 * kTK, mapF, &full[s], m0 + 32 * b, kglob);
  } else {
    tma_load_2d(stages + s * kStageFloats, mapB, &full[s], kglob, m0);
  }
}

// mode 0: X := L^-1 X; 1: X := L^-T X; 2: both (forward then backward in the
// same launch, y kept in Z between them).
__global__ void __launch_bounds__(kThreads, 1) sweep32_kernel(const __grid_constant__ CUtensorMap mapF,
                                                              const __grid_constant__ CUtensorMap mapB,
                                                              Sweep32Params p) {
  extern __shared__ float smem_raw[];
  float* sm = align1024(smem_raw);
  float* stages = sm + kOffStages;
  float* ys = sm + kOffY;
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + kSmemFloats);
  const int tid = threadIdx.x;
  const int G = gridDim.x;
  unsigned target = 0;
  bool ok = true;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t phase_bits = 0;  // parity of each stage's mbarrier

  // X (FP64, column-major) -> Z (FP32, row-major; padding columns zero)
  for (long long e = blockIdx.x * (long long)kThreads + tid; e < (long long)p.n * p.ldz;
       e += (long long)G * kThreads) {
    const int r = (int)(e / p.ldz), c = (int)(e % p.ldz);
    p.Z[(size_t)r * p.ldz + c] = c < p.nrhs ? (float)p.X[r + (long long)c * p.ldx] : 0.f;
  }
  target += G;
  ok = grid_barrier(p.counter, target);

  const int passes = (p.nrhs + kRhs - 1) / kRhs;
  const int rg = ((tid >> 5) & 3) * 8 + (tid & 7);   // 4-row (or 4-column) group 0..31
  const int cg = (tid >> 7) * 4 + ((tid >> 3) & 3);  // 4-rhs group 0..7
  const int nsteps = p.trans == 2 ? 2 * p.nsuper : p.nsuper;
  for (int step = 0; step < nsteps && ok; ++step) {
    const int fwd = p.trans == 0 || (p.trans == 2 && step < p.nsuper);
    const int lstep = step < p.nsuper ? step : step - p.nsuper;
    const int R = fwd ? lstep : p.nsuper - 1 - lstep;
    const int r0 = R * kS, sb = min(kS, p.n - r0), r1 = r0 + sb;
    const float* WR = (fwd ? p.Wr : p.Wc) + (size_t)R * kS * kS;
    const bool write_x = !(p.trans == 2 && fwd);
    const BItems bi = b_items(fwd, p.n, r0, r1, G);
    const bool has_a = blockIdx.x * (kThreads / 32) < sb;
    // The first phase-B item's L stages do not depend on y_R: start them now
    bool prefetched = false;
    if (tid == 0 && passes == 1 && (int)blockIdx.x < bi.items) {
      const int t = blockIdx.x / bi.ksplit, kpart = blockIdx.x % bi.ksplit;
      const int kbeg = kpart * bi.kchunk, kend = min(sb, kbeg + bi.kchunk);
      const int nk = kend > kbeg ? (kend - kbeg + kTK - 1) / kTK : 0;
      for (int s = 0; s < min(kStages, nk); ++s)
        issue_stage(&mapF, &mapB, fwd, stages, full, s, bi.lo + t * kTM, r0 + kbeg + s * kTK);
    }
    prefetched = passes == 1 && (int)blockIdx.x < bi.items;
    // ---- phase A
    if (has_a) {
      for (int pass = 0; pass < passes; ++pass) {
        stage_rows(ys, p.Z + (size_t)r0 * p.ldz, p.ldz, sb, pass);
        __syncthreads();
        phase_a(p, WR, fwd, r0, sb, pass, ys, write_x);
        __syncthreads();
      }
    }
    target += G;
    if (!(ok = grid_barrier(p.counter, target))) break;
    // ---- phase B.  When there are fewer tiles than CTAs, each tile's k
    // range is split into 2 or 4 parts (work items) whose results are added
    // to Z with FP32 reductions, so that the late super-steps keep the grid
    // busy.  Forward steps of mode 2 also move y_R into Z's rows of R (no
    // phase B writes them) for the backward steps.
    if (p.trans == 2 && fwd) {
      for (int e = blockIdx.x * kThreads + tid; e < sb * p.ldz; e += G * kThreads)
        p.Z[(size_t)r0 * p.ldz + e] = __ldcg(p.Yb + e);
    }
    for (int pass = 0; pass < passes; ++pass) {
      if ((int)blockIdx.x >= bi.items) break;
      stage_rows(ys, p.Yb, p.ldz, sb, pass);
      __syncthreads();
      for (int it = blockIdx.x; it < bi.items; it += G) {
        const int t = it / bi.ksplit, kpart = it % bi.ksplit;
        const int m0 = bi.lo + t * kTM;
        const int kbeg = kpart * bi.kchunk, kend = min(sb, kbeg + bi.kchunk);
        const int nk = kend > kbeg ? (kend - kbeg + kTK - 1) / kTK : 0;
        if (nk == 0) continue;
        if (tid == 0 && !(prefetched && it == (int)blockIdx.x && pass == 0))
          for (int s = 0; s < min(kStages, nk); ++s)
            issue_stage(&mapF, &mapB, fwd, stages, full, s, m0, r0 + kbeg + s * kTK);
        float acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
        for (int ks = 0; ks < nk; ++ks) {
          const int s = ks % kStages;
          if (!mbar_wait_bounded(&full[s], (phase_bits >> s) & 1)) {
            set_status(p.status, kTimeout, 9001);
            ok = false;
          }
          phase_bits ^= 1u << s;
          const float* st = stages + s * kStageFloats;
          const float* yk = ys + (kbeg + ks * kTK) * kRhs;
          if (fwd) {
            // stage = 4 boxes of [32 k][32 rows]: row m = 32 b + q at [b][k][q]
            const int b = rg >> 3, q = (rg & 7) * 4;
#pragma unroll 8
            for (int k = 0; k < kTK; ++k) {
              const float4 lv = *reinterpret_cast<const float4*>(st + b * 32 * kTK + k * 32 + q);
              const float4 yv = *reinterpret_cast<const float4*>(yk + k * kRhs + cg * 4);
              const float l4[4] = {lv.x, lv.y, lv.z, lv.w}, y4[4] = {yv.x, yv.y, yv.z, yv.w};
#pragma unroll
              for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) acc[a][bb] = fmaf(l4[a], y4[bb], acc[a][bb]);
            }
          } else {
            // stage = [128 columns j][32 k] with the 128-byte swizzle: 16-byte
            // chunk c of row j at chunk c ^ (j & 7)
#pragma unroll 2
            for (int kc = 0; kc < kTK / 4; ++kc) {
              float l4[4][4];
#pragma unroll
              for (int a = 0; a < 4; ++a) {
                const int j = rg + 32 * a;  // 8 lanes read 8 consecutive columns: distinct chunks
                const float4 v = *reinterpret_cast<const float4*>(st + j * kTK + ((kc ^ (j & 7)) << 2));
                l4[a][0] = v.x; l4[a][1] = v.y; l4[a][2] = v.z; l4[a][3] = v.w;
              }
#pragma unroll
              for (int kk = 0; kk < 4; ++kk) {
                const float4 yv = *reinterpret_cast<const float4*>(yk + (kc * 4 + kk) * kRhs + cg * 4);
                const float y4[4] = {yv.x, yv.y, yv.z, yv.w};
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                  for (int bb = 0; bb < 4; ++bb) acc[a][bb] = fmaf(l4[a][kk], y4[bb], acc[a][bb]);
              }
            }
          }
          fence_proxy_async_smem();
          __syncthreads();  // every thread is done with stage s
          if (tid == 0 && ks + kStages < nk)
            issue_stage(&mapF, &mapB, fwd, stages, full, s, m0, r0 + kbeg + (ks + kStages) * kTK);
        }
        // Z[m, c] -= acc for the tile's rows (forward: 4 consecutive rows per
        // thread) / columns (backward: columns rg + 32 a); L1 is bypassed since
        // other CTAs wrote these rows in earlier super-steps
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          const int m = m0 + (fwd ? rg * 4 + a : rg + 32 * a);
          if (m < bi.hi) {
            float* z = p.Z + (size_t)m * p.ldz + pass * kRhs + cg * 4;
            if (bi.ksplit == 1) {
              float4 v = __ldcg(reinterpret_cast<const float4*>(z));
              v.x -= acc[a][0]; v.y -= acc[a][1]; v.z -= acc[a][2]; v.w -= acc[a][3];
              *reinterpret_cast<float4*>(z) = v;
            } else {
              asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(z), "f"(-acc[a][0]),
                           "f"(-acc[a][1]), "f"(-acc[a][2]), "f"(-acc[a][3])
                           : "memory");
            }
          }
        }
      }
      __syncthreads();
    }
    target += G;
    if (!(ok = grid_barrier(p.counter, target))) break;
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

// A rows from a_rows on read as zero (they may lie past the matrix); the
// output's rows [0, out_rows) x columns [0, out_cols) are stored.
__device__ void tile128_products(const Prod* prods, int terms, float alpha, float* C, long long ldc,
                                 float* As, float* Bs, int a_rows, int out_rows, int out_cols) {
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
      for (int e = tid; e < 32 * 128; e += kThreads) {  // consecutive threads: consecutive k
        const int k = e & 31, c = e >> 5;
        Bs[k * kBsLd + c] = prods[t].B[(k0 + k) + (long long)c * prods[t].ldb];
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

// Wr = Wc^T per super-block (row-major copy for the forward sweep)
__global__ void transpose_blocks_kernel(int nsuper, const float* Wc, float* Wr) {
  __shared__ float t[32][33];
  const int R = blockIdx.z;
  const float* src = Wc + (size_t)R * kS * kS;
  float* dst = Wr + (size_t)R * kS * kS;
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int q = threadIdx.y; q < 32; q += 8) t[q][threadIdx.x] = src[(bx + threadIdx.x) + (size_t)(by + q) * kS];
  __syncthreads();
  for (int q = threadIdx.y; q < 32; q += 8) dst[(by + threadIdx.x) + (size_t)(bx + q) * kS] = t[threadIdx.x][q];
}

}  // namespace

size_t sweep32_ws_bytes(int n, int nrhs) {
  const int nsuper = (n + kS - 1) / kS;
  const int ldz = ((std::max(nrhs, 1) + kRhs - 1) / kRhs) * kRhs;
  size_t b = 0;
  b += 2 * (size_t)nsuper * kS * kS * sizeof(float);        // Wc, Wr
  b += (size_t)nsuper * 4 * kPB * kPB * sizeof(float);       // temporaries of the inverse
  b += (size_t)n * ldz * sizeof(float) + 1024;                // Z
  b += (size_t)kS * ldz * sizeof(float) + 1024;               // Yb
  b += 4096;                                                  // counter
  return b + 8 * 1024;
}

// Build the super-block inverses from L (FP32, ld ldl) and the FP64 panel
// inverses Winv (nb = 128, one nb x nb block per panel).  ws: sweep32_ws_bytes.
int sweep32_prepare(cudaStream_t st, int n, const float* L, long long ldl, const double* Winv, void* ws) {
  const int nsuper = (n + kS - 1) / kS;
  unsigned char* b = static_cast<unsigned char*>(ws);
  float* Wc = reinterpret_cast<float*>(b);
  float* Wr = Wc + (size_t)nsuper * kS * kS;
  float* tmp = Wr + (size_t)nsuper * kS * kS;
  TraceMark tm(st, kTraceOther, (double)nsuper * 4.0 * kS * kS * kS / 3.0, 12.0 * nsuper * kS * kS);
  superinv_init_kernel<<<std::min<long long>(((long long)nsuper * kS * kS + 255) / 256, 148 * 16), 256, 0, st>>>(
      n, nsuper, Winv, Wc);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  static bool attr = false;
  const int shb = (32 * 128 + 32 * kBsLd) * (int)sizeof(float);
  if (!attr) {
    EGPU_CUDA_TRY(cudaFuncSetAttribute(superinv_row_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, shb));
    attr = true;
  }
  for (int bi = 1; bi < kS / kPB; ++bi) {
    superinv_row_kernel<<<dim3(bi, nsuper), kThreads, shb, st>>>(n, nsuper, bi, L, ldl, Wc, tmp);
    count_launch();
    EGPU_CUDA_TRY(cudaGetLastError());
  }
  transpose_blocks_kernel<<<dim3(kS / 32, kS / 32, nsuper), dim3(32, 8), 0, st>>>(nsuper, Wc, Wr);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  return EGPU_OK;
}

// X := L^-1 X (trans 0) or L^-T X (trans 1); X FP64 n x nrhs (ld ldx), L FP32
// (ld ldl, 16-byte aligned base and ld a multiple of 4), ws prepared by
// sweep32_prepare for this L.
int sweep32_solve(cudaStream_t st, int trans, int n, int nrhs, const float* L, long long ldl, double* X,
                  long long ldx, void* ws, int sm_count, DevStatus* status) {
  if (n <= 0 || nrhs <= 0) return EGPU_OK;
  if (reinterpret_cast<uintptr_t>(L) % 16 != 0 || ldl % 4 != 0) return EGPU_ERR_ALIGN;
  const int nsuper = (n + kS - 1) / kS;
  const int ldz = ((nrhs + kRhs - 1) / kRhs) * kRhs;
  unsigned char* b = static_cast<unsigned char*>(ws);
  float* Wc = reinterpret_cast<float*>(b);
  float* Wr = Wc + (size_t)nsuper * kS * kS;
  float* tmp = Wr + (size_t)nsuper * kS * kS;
  unsigned char* after = reinterpret_cast<unsigned char*>(tmp + (size_t)nsuper * 4 * kPB * kPB);
  float* Z = reinterpret_cast<float*>(align_up(reinterpret_cast<uintptr_t>(after), 1024));
  float* Yb = reinterpret_cast<float*>(align_up(reinterpret_cast<uintptr_t>(Z + (size_t)n * ldz), 1024));
  unsigned* counter = reinterpret_cast<unsigned*>(align_up(reinterpret_cast<uintptr_t>(Yb + (size_t)kS * ldz), 256));
  CUtensorMap mapF, mapB;
  // forward: boxes of 32 rows (inner) x 32 columns; backward: 32 rows (inner)
  // x 128 columns, 128-byte swizzle
  if (!make_tma_2d(&mapF, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, L, n, n, ldl * 4, 32, kTK, false) ||
      !make_tma_2d(&mapB, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, L, n, n, ldl * 4, kTK, kTM, true))
    return EGPU_ERR_TMA;
  static int attr_dev_mask = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 31 && !(attr_dev_mask & (1 << dev))) {
    EGPU_CUDA_TRY(cudaFuncSetAttribute(sweep32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes));
    attr_dev_mask |= 1 << dev;
  }
  EGPU_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned), st));
  Sweep32Params p;
  p.n = n; p.nrhs = nrhs; p.trans = trans; p.nsuper = nsuper;  // trans 2: forward + backward
  p.Wc = Wc; p.Wr = Wr; p.Z = Z; p.ldz = ldz; p.Yb = Yb; p.X = X; p.ldx = ldx; p.counter = counter;
  p.status = status;
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
  EGPU_CUDA_TRY(cudaLaunchKernelEx(&cfg, sweep32_kernel, mapF, mapB, p));
  count_launch();
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

extern "C" int egpu_sweep32_solve(egpu_handle h, int trans, int n, int nrhs, const float* dL, int ldl, double* dX,
                                  int ldx) {
  if (!h) return EGPU_ERR_ARG;
  if (n < 0 || nrhs < 0 || nrhs > 64 || ldl < std::max(1, n) || ldx < std::max(1, n) || trans < 0 || trans > 2)
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
