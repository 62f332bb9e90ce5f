// Shared-memory building blocks for nb x nb diagonal blocks (nb <= 128):
// blocked Cholesky, triangular inverse and register-blocked mini-GEMMs.
#pragma once
#include "internal.h"

namespace egpu {

// ---------------------------------------------------------------------------
// Diagonal-block kernels.  The nb x nb block (nb <= 128) lives in shared
// memory with leading dimension kLDS = 132 (4 mod 16: the 8-byte DMMA
// fragment loads, rows g + 8.. x columns t + 4.., hit 16 distinct bank pairs
// per half warp; even, so every column starts on a 16-byte boundary for
// 16-byte copies), always as a LOWER triangle (an upper triangle is
// handled as the lower triangle of its transpose: UVar3Unb and LVar3Unb
// perform the same operations on A and A^T).
//
// Factorization: 16-column sub-panels.  Inside a sub-panel every column costs
// one barrier: all threads read a_jj, each updates its share of the
// sub-panel columns with  a_ik -= a_ij a_kj / a_jj  (the rank-1 update of
// LVar3Unb, Cholesky/LVar3.hpp:40-46, applied before the column is scaled),
// and the previous column is scaled by 1/sqrt(a_jj) in the same phase (no
// thread reads it any more).  After the sub-panel, the trailing triangle is
// updated by a register-blocked shared-memory mini-GEMM (4x4 per thread).
// The inverse of the factor is built the same way: 16 x 16 diagonal blocks
// inverted in parallel (one per warp), then block columns from the right,
// X21 = -inv(L22) (L21 X11), with 4x4-blocked mini-GEMMs.
// All loops are rolled: straight-line unrolled code run by one warp stalls
// on instruction fetch.
constexpr int kLDS = 132;
constexpr int kSP = 16;  // sub-panel width
constexpr int kDiagSmemBase = (128 * kLDS + 128) * (int)sizeof(double);

template <typename T>
__device__ __forceinline__ T& SE(T* S, int r, int c) { return S[r + c * kLDS]; }

// C[r0.., c0..] (nr x nc, lower part r >= c when tri) -= A[r0.., k0..k0+K) * B[c0.., k0..k0+K)^T
// reading A and B from S; 4x4 register tiles per thread.  sign = +1 or -1 for
// "-=" or "+=" (the inverse uses the opposite sign).
template <typename T>
__device__ inline void smem_syrk_tiles(T* S, int r0, int nr, int c0, int nc, int k0, int K, bool tri) {
  const int tr = (nr + 3) / 4, tc = (nc + 3) / 4;
  for (int t = threadIdx.x; t < tr * tc; t += blockDim.x) {
    const int ti = t % tr, tj = t / tr;
    const int rb = r0 + 4 * ti, cb = c0 + 4 * tj;
    if (tri && rb + 3 < cb) continue;  // tile strictly above the diagonal
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = T(0);
    for (int k = k0; k < k0 + K; ++k) {
      T x[4], y[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        x[a] = (rb + a < r0 + nr) ? SE(S, rb + a, k) : T(0);
        y[a] = (cb + a < c0 + nc) ? SE(S, cb + a, k) : T(0);
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(x[a], y[b], acc[a][b]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int r = rb + a, c = cb + b;
        if (r < r0 + nr && c < c0 + nc && (!tri || r >= c)) SE(S, r, c) -= acc[a][b];
      }
  }
}

// Lower Cholesky of the b x b block in S (T = float or double).  Returns 0 or
// the 1-based column of a non-positive pivot ("A was not numerically HPD",
// LVar3.hpp:37-38); the decision is uniform across the block (every thread
// reads the same a_jj).
template <typename T>
__device__ inline int smem_chol(T* S, int b) {
  __shared__ T s_alpha[128];
  const int tid = threadIdx.x;
  const int row = tid & 127, half = tid >> 7;  // two threads per row
  for (int c0 = 0; c0 < b; c0 += kSP) {
    const int c1 = min(b, c0 + kSP);
    for (int j = c0; j < c1; ++j) {
      const T ajj = SE(S, j, j);
      if (!(ajj > T(0))) return j + 1;  // non-positive or NaN
      if (tid == 0) s_alpha[j] = sqrt(ajj);
      // column j-1 is read by nobody in this phase: scale it now
      if (j > c0 && half == 1 && row >= j && row < b) SE(S, row, j - 1) /= s_alpha[j - 1];
      if (row > j && row < b) {
        const T lij = SE(S, row, j) / ajj;
        for (int k = j + 1 + half; k < c1 && k <= row; k += 2) SE(S, row, k) -= lij * SE(S, k, j);
      }
      __syncthreads();
    }
    if (half == 0 && row >= c1 && row < b) SE(S, row, c1 - 1) /= s_alpha[c1 - 1];
    if (half == 1 && row >= c0 && row < c1) SE(S, row, row) = s_alpha[row];
    __syncthreads();
    if (c1 < b) {
      smem_syrk_tiles(S, c1, b - c1, c1, b - c1, c0, c1 - c0, true);
      __syncthreads();
    }
  }
  return 0;
}

// In-place inverse of the lower b x b triangle in S (unit: diagonal taken as 1
// and written as 1).  Uses Xs (16 x 16 scratch per warp would not fit; the
// diagonal blocks are inverted in place column by column by their warp).
template <typename T>
__device__ inline void smem_trinv(T* S, int b, int unit) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = (b + kSP - 1) / kSP;
  // 1. 16 x 16 diagonal blocks, one warp each: lane c (< 16) computes column c
  //    of the block inverse by forward substitution, in place is impossible,
  //    so results go to registers first, then back to S.
  for (int blk = warp; blk < nblk; blk += blockDim.x / 32) {
    const int o = blk * kSP, w = min(kSP, b - o);
    T x[kSP];
    const int c = lane;
#pragma unroll
    for (int i = 0; i < kSP; ++i) x[i] = T(0);
    if (c < w) {
#pragma unroll
      for (int i = 0; i < kSP; ++i) {
        if (i < w && i >= c) {
          T acc = (i == c) ? T(1) : T(0);
#pragma unroll
          for (int m = 0; m < kSP; ++m)
            if (m >= c && m < i) acc = fma(-SE(S, o + i, o + m), x[m], acc);
          x[i] = unit ? acc : acc / SE(S, o + i, o + i);
        }
      }
    }
    __syncwarp();
    if (c < w) {
#pragma unroll
      for (int i = 0; i < kSP; ++i)
        if (i < w && i >= c) SE(S, o + i, o + c) = (unit && i == c) ? T(1) : x[i];
    }
  }
  __syncthreads();
  // 2. block columns from the right: X21 = -inv(L22) * (L21 * X11)
  for (int blk = nblk - 2; blk >= 0; --blk) {
    const int o = blk * kSP, w = min(kSP, b - o), r0 = o + w, R = b - r0;
    // T = L21 * X11 (R x w), computed into registers, written over L21
    {
      const int tr = (R + 3) / 4;
      T acc[4][4];
      const int t = tid;
      const bool act = t < tr * 4;  // tiles: 4 rows x 4 cols, w <= 16 -> 4 col tiles
      const int ti = t % max(tr, 1), tj = t / max(tr, 1);
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[a][q] = T(0);
      if (act) {
        for (int k = 0; k < w; ++k) {
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const int r = r0 + 4 * ti + a;
            const T l = (r < b) ? SE(S, r, o + k) : T(0);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int cc = 4 * tj + q;
              const T xv = (cc < w && k >= cc) ? SE(S, o + k, o + cc) : T(0);
              acc[a][q] = fma(l, xv, acc[a][q]);
            }
          }
        }
      }
      __syncthreads();
      if (act)
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = r0 + 4 * ti + a, cc = 4 * tj + q;
            if (r < b && cc < w) SE(S, r, o + cc) = acc[a][q];
          }
      __syncthreads();
      // X21 = -inv(L22) * T : row r of X21 = -sum_{m <= r} X22[r, m] T[m, :]
      if (act) {
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[a][q] = T(0);
        const int rmax = min(b - 1, r0 + 4 * ti + 3);
        for (int m = r0; m <= rmax; ++m) {
          T tv[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) tv[q] = (4 * tj + q < w) ? SE(S, m, o + 4 * tj + q) : T(0);
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            const int r = r0 + 4 * ti + a;
            const T xv = (r < b && m <= r) ? (unit && m == r ? T(1) : SE(S, r, m)) : T(0);
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[a][q] = fma(xv, tv[q], acc[a][q]);
          }
        }
      }
      __syncthreads();
      if (act)
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = r0 + 4 * ti + a, cc = 4 * tj + q;
            if (r < b && cc < w) SE(S, r, o + cc) = -acc[a][q];
          }
      __syncthreads();
    }
  }
}


// ---------------------------------------------------------------------------
// DMMA building blocks on shared-memory operands (all column-major).
//
// C = alpha * A * op(B) + beta * C for M % 16 == 0, N % 8 == 0, K % 8 == 0.
// The 16 x 8 output tiles go round-robin to warps w_first .. w_first +
// w_count - 1 (default: all warps); skip_top_left leaves the top-left 16 x 16
// block of C to someone else.
// A_LOWER: A[r][k] = 0 for k > r.  B_TRANS: op(B)[k][c] = B[c][k] (B stored
// N x K).  B_LOWER: op(B)[k][c] = 0 for c > k.  C_LOWER: only r >= c is
// written.  C must not alias A or B.  All warps of the CTA share the 16x8
// output tiles; the caller synchronises afterwards.
template <bool A_LOWER, bool B_TRANS, bool B_LOWER, bool C_LOWER>
__device__ inline void smem_dmma_gemm(const double* A, int lda, const double* B, int ldb, double* C, int ldc,
                                      int M, int N, int K, double alpha, double beta, int w_first = 0,
                                      int w_count = -1, bool skip_top_left = false) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = w_count > 0 ? w_count : (blockDim.x >> 5);
  const int g = lane >> 2, t = lane & 3;
  const int tm = M / 16, tn = N / 8;
  for (int tile = warp - w_first; tile < tm * tn; tile += nw) {
    const int r0 = (tile % tm) * 16, c0 = (tile / tm) * 8;
    if (C_LOWER && r0 + 15 < c0) continue;
    if (skip_top_left && r0 < 16 && c0 < 16) continue;  // another warp owns that block
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const int kend = A_LOWER ? min(K, r0 + 16) : K;  // A is zero right of its diagonal
    const int kbeg = B_LOWER ? (c0 / 8) * 8 : 0;      // op(B) is zero above its diagonal
    for (int k0 = kbeg; k0 < kend; k0 += 8) {
      double a[4], b[2];
      const int ka = k0 + t, kb = k0 + t + 4;
      const int ra = r0 + g, rb = r0 + g + 8;
      a[0] = (!A_LOWER || ka <= ra) ? A[ra + ka * lda] : 0.0;
      a[1] = (!A_LOWER || ka <= rb) ? A[rb + ka * lda] : 0.0;
      a[2] = (!A_LOWER || kb <= ra) ? A[ra + kb * lda] : 0.0;
      a[3] = (!A_LOWER || kb <= rb) ? A[rb + kb * lda] : 0.0;
      const int cc = c0 + g;
      b[0] = (!B_LOWER || cc <= ka) ? (B_TRANS ? B[cc + ka * ldb] : B[ka + cc * ldb]) : 0.0;
      b[1] = (!B_LOWER || cc <= kb) ? (B_TRANS ? B[cc + kb * ldb] : B[kb + cc * ldb]) : 0.0;
      dmma_16x8x8(acc, a, b);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = r0 + g + ((q >= 2) ? 8 : 0), c = c0 + 2 * t + (q & 1);
      if (C_LOWER && r < c) continue;
      double* cp = C + r + c * ldc;
      *cp = (beta == 0.0) ? alpha * acc[q] : fma(alpha, acc[q], beta * *cp);
    }
  }
}

// Columns of X = inv(L) for the 16 x 16 lower block L at S[o.., o..] (read
// with all lanes on the same address: shared-memory broadcasts), given
// rinv = 1 / L[lane][lane] in lane `lane` (< 16).  Lane c < 16 computes column
// c by forward substitution, x[k] = (delta_kc - sum_{m<k} L[k][m] x[m]) rinv_k.
__device__ inline void warp_trinv16_cols(const double* S, int lds, int o, double rinv, double* X, int ldx) {
  const int lane = threadIdx.x & 31;
  double x[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const double rk = __shfl_sync(0xffffffffu, rinv, k);
    double a0 = (k == lane) ? 1.0 : 0.0, a1 = 0.0;
#pragma unroll
    for (int m = 0; m < k; m += 2) {
      a0 = fma(-S[(o + k) + (o + m) * lds], x[m], a0);
      if (m + 1 < k) a1 = fma(-S[(o + k) + (o + m + 1) * lds], x[m + 1], a1);
    }
    x[k] = (k >= lane) ? (a0 + a1) * rk : 0.0;
  }
  if (lane < 16)
#pragma unroll
    for (int k = 0; k < 16; ++k) X[k + lane * ldx] = x[k];
}

// Cholesky of one 16 x 16 lower block at S[o.., o..] by one warp, rows in
// registers (lane i < 16 holds row i), pivots broadcast by shuffles; the
// factor goes back into S and its inverse into X (16 x 16, ld ldx).
// The diagonal uses r = 1/sqrt(a_jj): a_jj r = sqrt(a_jj), a_ij r = l_ij, and
// r is also the reciprocal the inverse needs.
// Returns 0 or the 1-based column of a non-positive pivot (warp-uniform).
__device__ inline int warp_chol16(double* S, int lds, int o, double* X, int ldx) {
  const int lane = threadIdx.x & 31;
  const bool act = lane < 16;
  double d[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) d[k] = (act && k <= lane) ? S[(o + lane) + (o + k) * lds] : 0.0;
  int fail = 0;
  double myr = 1.0;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const double djj = __shfl_sync(0xffffffffu, d[j], j);
    if (!fail) {
      if (djj <= 0.0) {
        fail = j + 1;
      } else {
        const double r = rsqrt(djj);
        if (lane == j) myr = r;
        d[j] *= r;  // lane j: sqrt(a_jj); lanes > j: l_ij
        const double lj = d[j];
#pragma unroll
        for (int k = j + 1; k < 16; ++k) {
          const double lkj = __shfl_sync(0xffffffffu, lj, k);
          if (lane >= k) d[k] = fma(-lj, lkj, d[k]);
        }
      }
    }
  }
  if (fail) return fail;
#pragma unroll
  for (int k = 0; k < 16; ++k)
    if (act && k <= lane) S[(o + lane) + (o + k) * lds] = d[k];
  __syncwarp();
  warp_trinv16_cols(S, lds, o, myr, X, ldx);
  return 0;
}

// Inverse of one 16 x 16 lower block at S[o.., o..] (unit: diagonal taken as
// 1) by one warp, into X (ld ldx).  The 16 reciprocals of the diagonal are
// formed in parallel, one per lane.
__device__ inline void warp_trinv16(const double* S, int lds, int o, int unit, double* X, int ldx) {
  const int lane = threadIdx.x & 31;
  const double rinv = (unit || lane >= 16) ? 1.0 : 1.0 / S[(o + lane) + (o + lane) * lds];
  warp_trinv16_cols(S, lds, o, rinv, X, ldx);
}

// Temporary area of the DMMA diagonal kernels: 16 leaf inverses (ld 17) and
// one 64 x 64 product buffer (ld 68).
constexpr int kLeafLD = 17;
constexpr int kTmpLD = 68;
constexpr int kDiagTmpDoubles = 8 * 16 * kLeafLD + 64 * kTmpLD;
constexpr int kDiagSmem = kDiagSmemBase + kDiagTmpDoubles * (int)sizeof(double);

// Flat (one pass, all copies in flight) transfers of a b x b triangle between
// global memory and S; a column-by-column loop costs one memory round trip
// per column.  `upper`: the global block holds the triangle transposed
// (S(r, c) = G[c + r ld]); consecutive threads always take consecutive
// global addresses.
__device__ inline void tri_load_async(double* S, const double* G, long long ld, int b, bool upper) {
  // a warp per column j, lanes over rows; 16-byte copies when G's columns are
  // 16-byte aligned (the copy may start one row above the diagonal: S's
  // strict upper triangle is never read)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const bool vec = !upper && (ld % 2 == 0) && (reinterpret_cast<uintptr_t>(G) % 16 == 0);
  for (int j = warp; j < b; j += nw) {
    const double* g = G + (long long)j * ld;
    if (vec) {
      for (int i = (j & ~1) + 2 * lane; i < b; i += 64) {
        if (i + 1 < b) cp_async16_cg(&S[i + j * kLDS], &g[i]);
        else cp_async8(&S[i + j * kLDS], &g[i]);
      }
    } else if (!upper) {
      for (int i = j + lane; i < b; i += 32) cp_async8(&S[i + j * kLDS], &g[i]);
    } else {
      for (int i = lane; i <= j; i += 32) cp_async8(&S[j + i * kLDS], &g[i]);  // G(i, j), i <= j
    }
  }
}
// Lower triangle of S (r >= c) into G; the other triangle of the b x b block
// is written as zero when `zero_other`, else left alone.
__device__ inline void tri_store(const double* S, double* G, long long ld, int b, bool upper, bool zero_other) {
  // a warp per column j of G, lanes over rows i; 16-byte stores when aligned
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const bool vec = !upper && (ld % 2 == 0) && (reinterpret_cast<uintptr_t>(G) % 16 == 0);
  for (int j = warp; j < b; j += nw) {
    double* g = G + (long long)j * ld;
    if (vec) {
      const double* s = S + j * kLDS;
      for (int i = (zero_other ? 0 : (j & ~1)) + 2 * lane; i < b; i += 64) {
        const double v0 = i >= j ? s[i] : 0.0;
        if (i + 1 < b && (i >= j || zero_other)) {
          *reinterpret_cast<double2*>(&g[i]) = make_double2(v0, i + 1 >= j ? s[i + 1] : 0.0);
        } else {
          if (i >= j || zero_other) g[i] = v0;
          if (i + 1 < b) g[i + 1] = s[i + 1];  // i + 1 == j: on the diagonal
        }
      }
    } else {
      for (int i = lane; i < b; i += 32) {
        const int r = upper ? j : i, c = upper ? i : j;  // S coordinates
        if (r >= c) g[i] = S[r + c * kLDS];
        else if (zero_other) g[i] = 0.0;
      }
    }
  }
}

// Pad the lower b x b triangle in S to bp = round_up(b, 16) with identity.
__device__ inline int pad16_identity(double* S, int b) {
  const int bp = (b + 15) & ~15;
  for (int e = threadIdx.x; e < (bp - b) * bp; e += blockDim.x) {
    const int r = b + e / bp, c = e % bp;  // rows b..bp-1, all columns
    if (r >= c) S[r + c * kLDS] = (r == c) ? 1.0 : 0.0;
  }
  return bp;
}

// In-place inverse of the lower bp x bp triangle in S (bp a multiple of 16,
// padded with identity), given the inverses of its 16 x 16 diagonal blocks in
// Xl (block q at Xl + q*16*kLeafLD).  Levels of doubling block size:
//   inv([[A, 0], [B, C]]) = [[Ai, 0], [-Ci B Ai, Ci]],  T = B Ai, X21 = -Ci T.
__device__ inline void smem_trinv_dmma(double* S, int bp, const double* Xl, double* T) {
  // leaves into place
  const int nleaf = bp / 16;
  for (int e = threadIdx.x; e < nleaf * 256; e += blockDim.x) {
    const int q = e >> 8, i = (e >> 4) & 15, k = e & 15;
    if (i >= k) S[(16 * q + i) + (16 * q + k) * kLDS] = Xl[q * 16 * kLeafLD + i + k * kLeafLD];
  }
  __syncthreads();
  for (int s = 16; s < bp; s *= 2) {
    for (int o = 0; o + s < bp; o += 2 * s) {
      const int s2 = min(s, bp - o - s);
      // T = B * Ai   (s2 x s), B = S[o+s.., o..], Ai = S[o.., o..] lower
      smem_dmma_gemm<false, false, true, false>(S + (o + s) + o * kLDS, kLDS, S + o + o * kLDS, kLDS, T, kTmpLD,
                                                s2, s, s, 1.0, 0.0);
      __syncthreads();
      // X21 = -Ci * T  (s2 x s), Ci = S[o+s.., o+s..] lower
      smem_dmma_gemm<true, false, false, false>(S + (o + s) + (o + s) * kLDS, kLDS, T, kTmpLD,
                                                S + (o + s) + o * kLDS, kLDS, s2, s, s2, -1.0, 0.0);
      __syncthreads();
    }
  }
}

// L21 := A21 * X11^T in place (A21: m2 x 16 at P, ld kLDS, m2 % 16 == 0;
// X11: 16 x 16, ld kLeafLD): warp w takes 16-row tiles w, w + nw, ...; both
// 8-column halves stay in registers until the whole row tile is read.
__device__ inline void smem_l21_inplace(double* P, int m2, const double* X11) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  for (int rt = warp; rt < m2 / 16; rt += nw) {
    const int r0 = rt * 16;
    double acc0[4] = {0.0, 0.0, 0.0, 0.0}, acc1[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k0 = 0; k0 < 16; k0 += 8) {
      double a[4], b0[2], b1[2];
      a[0] = P[(r0 + g) + (k0 + t) * kLDS];
      a[1] = P[(r0 + g + 8) + (k0 + t) * kLDS];
      a[2] = P[(r0 + g) + (k0 + t + 4) * kLDS];
      a[3] = P[(r0 + g + 8) + (k0 + t + 4) * kLDS];
      b0[0] = X11[g + (k0 + t) * kLeafLD];  // op(B)[k][c] = X11[c][k]
      b0[1] = X11[g + (k0 + t + 4) * kLeafLD];
      b1[0] = X11[(g + 8) + (k0 + t) * kLeafLD];
      b1[1] = X11[(g + 8) + (k0 + t + 4) * kLeafLD];
      dmma_16x8x8(acc0, a, b0);
      dmma_16x8x8(acc1, a, b1);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = r0 + g + ((q >= 2) ? 8 : 0), c = 2 * t + (q & 1);
      P[r + c * kLDS] = acc0[q];
      P[r + (c + 8) * kLDS] = acc1[q];
    }
  }
}

// Lower Cholesky of the bp x bp block in S (bp a multiple of 16; the caller
// pads with identity) in 16-column steps, the diagonal 16 x 16 leaves
// factored and inverted by one warp (X11 into Xl), L21 = A21 X11^T and the
// trailing update A22 -= L21 L21^T on the tensor cores.  Look-ahead: while
// warps 1.. update the rest of A22, warp 0 updates the next diagonal leaf
// first and factors it.  Returns 0 or the 1-based column of a non-positive
// pivot (uniform).
__device__ inline int smem_chol_dmma(double* S, int bp, double* Xl, double* /*T*/) {
  __shared__ int s_fail;
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (warp == 0) {
    const int f = warp_chol16(S, kLDS, 0, Xl, kLeafLD);
    if (threadIdx.x == 0) s_fail = f;
  }
  __syncthreads();
  for (int o = 0; o < bp; o += 16) {
    if (s_fail) return s_fail;
    const int m2 = bp - o - 16;
    if (m2 <= 0) break;
    double* L21 = S + (o + 16) + o * kLDS;
    double* A22 = S + (o + 16) + (o + 16) * kLDS;
    smem_l21_inplace(L21, m2, Xl + (o / 16) * 16 * kLeafLD);
    __syncthreads();
    if (warp == 0) {
      smem_dmma_gemm<false, true, false, true>(L21, kLDS, L21, kLDS, A22, kLDS, 16, 16, 16, -1.0, 1.0, 0, 1);
      __syncwarp();
      const int f = warp_chol16(S, kLDS, o + 16, Xl + ((o + 16) / 16) * 16 * kLeafLD, kLeafLD);
      if (threadIdx.x == 0) s_fail = f ? o + 16 + f : 0;
    } else {
      smem_dmma_gemm<false, true, false, true>(L21, kLDS, L21, kLDS, A22, kLDS, m2, m2, 16, -1.0, 1.0, 1, nw - 1,
                                               true);
    }
    __syncthreads();
  }
  return s_fail;
}

}  // namespace egpu
