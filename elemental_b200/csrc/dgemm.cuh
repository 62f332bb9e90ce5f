// FP64 tensor-core GEMM / SYRK engine for sm_100a.
//
// C[MxN] = alpha * op(A)[MxK] * op(B)[KxN] + beta * C, optionally restricted
// to the lower (tri=1) or upper (tri=2) triangle of C.  This single engine
// carries every level-3 call of the factor-and-solve path:
//   * Herk/Syrk trailing update of Cholesky  (Cholesky/LVar3.hpp:114,
//     UVar3.hpp:113; dsyrk_ at src/core/imports/blas.cpp:1043)
//   * Gemm trailing update of LU             (LU.hpp:203; dgemm_ at blas.cpp:930)
//   * Trsm panel / row-panel solves, run as a multiply by the explicitly
//     inverted diagonal block                 (LVar3.hpp:113, LU.hpp:202)
//
// Operands are staged global->shared by TMA (cp.async.bulk.tensor, one
// elected thread, mbarrier completion), 4-stage ring, BK = 16.  The math is
// FP64 DMMA (mma.sync m16n8k8 f64): Blackwell's tcgen05 has no f64 kind, and
// DMMA reaches the FP64 peak (37.2 TFLOP/s measured, DFMA 34.1).
//
// Shared-memory layouts (no bank conflicts on any fragment load):
//   MN-major operand (m or n contiguous in global): BM/16 boxes of 16 m x
//     16 k, each [16 k][16 m] (128 B per k row) with the 128B swizzle (16-byte
//     chunk c of row k at chunk c ^ (k & 7)); one 16-byte load gives two
//     adjacent rows -> feeds two m16 tiles (row-interleaved tile pairs).  The
//     four lanes of a quad read k rows 2t (+1) of the same chunk, which the
//     swizzle spreads over distinct banks (plain [16 k][BM] rows, 8 BM bytes
//     apart, would put all four in the same banks).
//   K-major operand (k contiguous in global): smem [BM][16 k], 128B swizzle;
//     one 16-byte load gives the k pair (2t, 2t+1) of one row.
// The k index inside each k8 step is permuted (logical t <-> physical 2t,
// t+4 <-> 2t+1) identically for A and B, which leaves the product unchanged.
#pragma once
#include "common.cuh"

namespace egpu {

struct GemmParams {
  double* C;
  long long ldc;
  int M, N, K;
  double alpha, beta;
  int tri;  // 0 full, 1 lower (row >= col), 2 upper (row <= col)
  int tiles_m, tiles_n;
  int cvec;  // C base 16-byte aligned and ldc even: paired 16-byte epilogue
  DevStatus* status;
};

constexpr int kBK = 16;
constexpr int kStages = 4;

template <int WARPS_M, int WARPS_N>
struct GemmShape {
  static constexpr int BM = 64 * WARPS_M;
  static constexpr int BN = 32 * WARPS_N;
  static constexpr int kThreads = 32 * WARPS_M * WARPS_N;
  static constexpr int kStageBytes = (BM + BN) * kBK * 8;
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024 /*align*/ + 16 * kStages /*barriers*/;
};

// Map a linear CTA index onto (tile_m, tile_n) for the triangular modes with
// BM = 2*BN (tile-row i covers rows [BM i, BM i + BM), tile-col j covers
// [BN j, BN j + BN)).  Lower: column j needs rows i >= j/2 (count
// max(0, MT - j/2)); upper: rows i <= j/2 (count min(j/2 + 1, MT)).
// cum(j) = number of tiles in columns < j.
__device__ __forceinline__ long long tri_S(long long j) {  // sum_{j'<j} floor(j'/2)
  const long long a = j / 2;
  return (j & 1) ? a * a : a * (a - 1);
}
__device__ __forceinline__ long long tri_cum_lower(int j, int MT) {
  const long long jj = min((long long)j, 2ll * MT);
  return jj * MT - tri_S(jj);
}
__device__ __forceinline__ long long tri_cum_upper(int j, int MT) {
  const long long J0 = 2ll * MT;
  if (j <= J0) return tri_S(j) + j;
  return tri_S(J0) + J0 + (j - J0) * MT;
}

__device__ __forceinline__ bool map_tile(const GemmParams& p, int& ti, int& tj) {
  const long long L = blockIdx.x;
  if (p.tri == 0) {
    ti = (int)(L % p.tiles_m);
    tj = (int)(L / p.tiles_m);
    return tj < p.tiles_n;
  }
  int lo = 0, hi = p.tiles_n;  // find largest j with cum(j) <= L
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    long long c = p.tri == 1 ? tri_cum_lower(mid, p.tiles_m) : tri_cum_upper(mid, p.tiles_m);
    if (c <= L) lo = mid; else hi = mid;
  }
  tj = lo;
  if (p.tri == 1) {
    ti = tj / 2 + (int)(L - tri_cum_lower(tj, p.tiles_m));
  } else {
    ti = (int)(L - tri_cum_upper(tj, p.tiles_m));
  }
  return ti < p.tiles_m && tj < p.tiles_n;
}

template <bool AK, bool BK, int WARPS_M, int WARPS_N>
__global__ void __launch_bounds__(32 * WARPS_M * WARPS_N, (WARPS_M * WARPS_N <= 4) ? 2 : 1)
    dgemm_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const GemmParams p) {
  using S = GemmShape<WARPS_M, WARPS_N>;
  constexpr int BM = S::BM, BN = S::BN;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * S::kStageBytes);
  uint64_t* empty = full + kStages;  // one arrival per warp when it is done with a stage

  int ti, tj;
  if (!map_tile(p, ti, tj)) return;
  if (p.status != nullptr && p.status->code != 0) return;  // an earlier step failed
  const int row0 = ti * BM, col0 = tj * BN;
  const int KT = (p.K + kBK - 1) / kBK;

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp % WARPS_M, wn = warp / WARPS_M;

  if (tid == 0) {
    tma_prefetch_desc(&tmA);
    tma_prefetch_desc(&tmB);
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], S::kThreads / 32);
    }
    fence_mbar_init();
  }
  __syncthreads();

  auto issue = [&](int kt) {
    const int s = kt % kStages;
    double* sA = reinterpret_cast<double*>(smem + s * S::kStageBytes);
    double* sB = sA + BM * kBK;
    mbar_expect_tx(&full[s], S::kStageBytes);
    if (AK) {
      tma_load_2d(sA, &tmA, &full[s], kt * kBK, row0);
    } else {
#pragma unroll
      for (int b = 0; b < BM / 16; ++b) tma_load_2d(sA + b * 256, &tmA, &full[s], row0 + 16 * b, kt * kBK);
    }
    if (BK) {
      tma_load_2d(sB, &tmB, &full[s], kt * kBK, col0);
    } else {
#pragma unroll
      for (int b = 0; b < BN / 16; ++b) tma_load_2d(sB + b * 256, &tmB, &full[s], col0 + 16 * b, kt * kBK);
    }
  };

  int issued = 0;  // k-tiles whose loads thread 0 has issued
  if (tid == 0) {
    for (int kt = 0; kt < kStages && kt < KT; ++kt) issue(kt);
    issued = min(kStages, KT);
  }
  // Pull this tile of C into L2 while the main loop runs, so the epilogue's
  // read-modify-write does not wait on HBM (one bulk prefetch per column).
  if (p.beta != 0.0 && p.cvec) {
    const int nrow = min(BM, p.M - row0);
    const int ncol = min(BN, p.N - col0);
    const unsigned bytes = (unsigned)((nrow * 8) & ~15);  // never past the column's end
    for (int c = tid; c < ncol && bytes > 0; c += S::kThreads) {
      const double* src = p.C + (long long)(col0 + c) * p.ldc + row0;
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
    }
  }

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

  bool ok = true;
  for (int kt = 0; kt < KT; ++kt) {
    const int s = kt % kStages;
    const uint32_t parity = (kt / kStages) & 1;
    // warp-uniform outcome: the DMMAs below need the whole warp converged
    ok = __all_sync(0xffffffffu, ok && mbar_wait_bounded(&full[s], parity));
    const double* sA = reinterpret_cast<const double*>(smem + s * S::kStageBytes);
    const double* sB = sA + BM * kBK;
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      double af[4][4], bf[4][2];
      const int ke = ks * 8 + 2 * t;  // physical k pair (ke, ke+1)
      if (AK) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r0 = wm * 64 + i * 16 + g;
          const int r1 = r0 + 8;
          const int ch = ks * 4 + t;
          const double2 v0 = *reinterpret_cast<const double2*>(sA + r0 * 16 + ((ch ^ (r0 & 7)) << 1));
          const double2 v1 = *reinterpret_cast<const double2*>(sA + r1 * 16 + ((ch ^ (r1 & 7)) << 1));
          af[i][0] = v0.x; af[i][2] = v0.y; af[i][1] = v1.x; af[i][3] = v1.y;
        }
      } else {
        // box (wm * 64 + pr * 32) / 16 (+1 for rows +16), chunk g of rows ke, ke + 1
        const int c0 = (g ^ (ke & 7)) << 1, c1 = (g ^ ((ke + 1) & 7)) << 1;
#pragma unroll
        for (int pr = 0; pr < 2; ++pr) {
          const double* bx = sA + (wm * 4 + pr * 2) * 256;
          const double2 v00 = *reinterpret_cast<const double2*>(bx + ke * 16 + c0);
          const double2 v01 = *reinterpret_cast<const double2*>(bx + (ke + 1) * 16 + c1);
          const double2 v10 = *reinterpret_cast<const double2*>(bx + 256 + ke * 16 + c0);
          const double2 v11 = *reinterpret_cast<const double2*>(bx + 256 + (ke + 1) * 16 + c1);
          af[2 * pr][0] = v00.x; af[2 * pr][1] = v10.x; af[2 * pr][2] = v01.x; af[2 * pr][3] = v11.x;
          af[2 * pr + 1][0] = v00.y; af[2 * pr + 1][1] = v10.y; af[2 * pr + 1][2] = v01.y; af[2 * pr + 1][3] = v11.y;
        }
      }
      if (BK) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int n = wn * 32 + j * 8 + g;
          const int ch = ks * 4 + t;
          const double2 v = *reinterpret_cast<const double2*>(sB + n * 16 + ((ch ^ (n & 7)) << 1));
          bf[j][0] = v.x; bf[j][1] = v.y;
        }
      } else {
        const int c0 = (g ^ (ke & 7)) << 1, c1 = (g ^ ((ke + 1) & 7)) << 1;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const double* bx = sB + (wn * 2 + q) * 256;  // box of n rows wn * 32 + q * 16 ..
          const double2 v0 = *reinterpret_cast<const double2*>(bx + ke * 16 + c0);
          const double2 v1 = *reinterpret_cast<const double2*>(bx + (ke + 1) * 16 + c1);
          bf[2 * q][0] = v0.x; bf[2 * q][1] = v1.x;
          bf[2 * q + 1][0] = v0.y; bf[2 * q + 1][1] = v1.y;
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_16x8x8(acc[i][j], af[i], bf[j]);
    }
    // This warp is done with stage s.  The refill is a TMA write into the
    // same bytes, and an mbarrier release alone does not order this warp's
    // generic-proxy reads before an async-proxy write: lane 0 fences (after
    // the warp has converged) and arrives.  Warp 0 refills the stage for
    // k-tile kt + kStages once every warp has arrived (the whole warp waits,
    // lane 0 issues, so warp 0 stays converged); the other warps run ahead
    // into the stages already loaded instead of meeting at a CTA barrier.
    __syncwarp();
    if (lane == 0) {
      fence_proxy_async_smem();
      mbar_arrive(&empty[s]);
    }
    if (warp == 0 && kt + kStages < KT) {
      ok = __all_sync(0xffffffffu, ok && mbar_wait_bounded(&empty[s], parity));
      if (ok && lane == 0) issue(kt + kStages);
      if (ok) issued = kt + kStages + 1;
      __syncwarp();
    }
    if (!ok) break;
  }

  // a warp that gave up (bounded wait) leaves early; all meet here
  if (!__syncthreads_and(ok)) {
    if (tid == 0) {
      set_status(p.status, kTimeout, 100);
      // Drain copies still in flight before the CTA's shared memory goes away.
      for (int r = max(0, issued - kStages); r < issued; ++r)
        (void)mbar_wait_bounded(&full[r % kStages], (r / kStages) & 1);
    }
    __syncthreads();
    return;
  }

  // Epilogue: C = alpha * acc + beta * C on the valid (and triangle) region.
  // All C loads are issued before any store so their latencies overlap.
  const double alpha = p.alpha, beta = p.beta;
  auto row_of = [&](int i, int r) -> int {
    if (AK) return row0 + wm * 64 + i * 16 + g + ((r >= 2) ? 8 : 0);
    return row0 + wm * 64 + (i >> 1) * 32 + 2 * g + (i & 1) + ((r >= 2) ? 16 : 0);
  };
  auto col_of = [&](int j, int r) -> int {
    const int c = 2 * t + (r & 1);
    if (BK) return col0 + wn * 32 + j * 8 + c;
    return col0 + wn * 32 + (j >> 1) * 16 + 2 * c + (j & 1);
  };
  auto valid = [&](int row, int col) -> bool {
    if (row >= p.M || col >= p.N) return false;
    if (p.tri == 1 && row < col) return false;
    if (p.tri == 2 && row > col) return false;
    return true;
  };
  // MN-major A: tiles 2pr and 2pr+1 hold rows (2g, 2g+1) -> one 16-byte access
  const bool vec = !AK && p.cvec;
  if (vec) {
#pragma unroll
    for (int pr = 0; pr < 2; ++pr)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int row = row_of(2 * pr, r), col = col_of(j, r);
          const bool v0 = valid(row, col), v1 = valid(row + 1, col);
          double* cp = p.C + (long long)col * p.ldc + row;
          double c0 = 0.0, c1 = 0.0;
          if (beta != 0.0) {
            if (v0 && v1) {
              const double2 cc = *reinterpret_cast<const double2*>(cp);
              c0 = cc.x; c1 = cc.y;
            } else {
              if (v0) c0 = cp[0];
              if (v1) c1 = cp[1];
            }
          }
          acc[2 * pr][j][r] = fma(beta, c0, alpha * acc[2 * pr][j][r]);
          acc[2 * pr + 1][j][r] = fma(beta, c1, alpha * acc[2 * pr + 1][j][r]);
        }
#pragma unroll
    for (int pr = 0; pr < 2; ++pr)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int row = row_of(2 * pr, r), col = col_of(j, r);
          const bool v0 = valid(row, col), v1 = valid(row + 1, col);
          double* cp = p.C + (long long)col * p.ldc + row;
          if (v0 && v1) {
            *reinterpret_cast<double2*>(cp) = make_double2(acc[2 * pr][j][r], acc[2 * pr + 1][j][r]);
          } else {
            if (v0) cp[0] = acc[2 * pr][j][r];
            if (v1) cp[1] = acc[2 * pr + 1][j][r];
          }
        }
    return;
  }
  if (beta != 0.0) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int row = row_of(i, r), col = col_of(j, r);
          const double c = valid(row, col) ? p.C[(long long)col * p.ldc + row] : 0.0;
          acc[i][j][r] = fma(beta, c, alpha * acc[i][j][r]);
        }
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[i][j][r] *= alpha;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int row = row_of(i, r), col = col_of(j, r);
        if (valid(row, col)) p.C[(long long)col * p.ldc + row] = acc[i][j][r];
      }
}

}  // namespace egpu
