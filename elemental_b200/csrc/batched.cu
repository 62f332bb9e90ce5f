// Batched factor-and-solve of many independent systems of uneven sizes in
// persistent launches: HPDSolve (Cholesky + cholesky::SolveAfter) and
// GaussianElimination-style LU + solve, per system, n <= 512.
//
// One CTA owns one system at a time and pulls the next from a size-sorted
// queue (largest first) with an atomic counter, so the uneven sizes balance
// across the SMs.  Per system the CTA runs the blocked right-looking
// algorithm with an NB-wide panel held in shared memory:
//   * Cholesky: the diagonal block is factored by one warp with the block in
//     registers (lane = row, shuffles along the column, no CTA barrier per
//     column); its inverse is formed by the same warp with a short dependent
//     chain (reciprocal diagonal, right-looking column accumulation); the
//     panel solve is a multiply by that inverse; the trailing update runs on
//     the FP64 tensor cores (DMMA m16n8k8, 32x32 warp tiles) over the
//     system's trailing matrix in global memory.
//   * LU: the panel is factored with logical pivoting -- the chosen row is
//     marked done instead of being swapped, every thread tracks the current
//     position of the rows it owns, so a column costs one CTA barrier -- and
//     the panel is then permuted once in shared memory; the interchanges on
//     the columns to its right are gathered by warps (all loads of a column
//     in flight, then all stores).
//   * The solves run on a chunk of <= 8 right-hand sides in shared memory,
//     blocked by NB with the kept diagonal-block inverses.
//
// Storage type T: double for the FP64 plans (the factor overwrites A), float
// for the refined plans: A is converted once into an FP32 working copy, the
// factorization runs on it (arithmetic in FP64 registers, every stored value
// rounded to FP32), and FP64 iterative refinement on A recovers an FP64
// solution (backward error <= 1e-14).  A refined system whose refinement
// stalls is re-solved in FP64 (panel NB / 2, same shared memory).
#include <algorithm>
#include <climits>
#include <new>
#include <vector>

#include "internal.h"

namespace egpu {

#define BTRY(x)                          \
  do {                                   \
    const int rc_ = (x);                 \
    if (rc_ != EGPU_OK) return rc_;      \
  } while (0)

struct BatchItem {
  double* A;  // the system matrix (column-major, lda); FP64 plans factor it in place
  double* B;  // right-hand sides in, solutions out (ldb); null: factor only
  void* F;    // refined plans: the working copy (ldf; room for doubles); FP64 plans: A
  int n, nrhs, lda, ldb, ldf, id;
};

constexpr int kBmaxN = 512;                    // largest order handled by one CTA
constexpr int kBmaxRHS = 16;                   // right-hand sides per system
constexpr int kRC = 8;                         // right-hand sides per shared-memory chunk
constexpr int kPLD = kBmaxN + 32;              // panel leading dimension (rows)
constexpr int kIRMax = 10;                     // refinement corrections before the FP64 fallback
constexpr double kIRTol = 1e-14;               // backward error the refined plans reach
constexpr int kScrDoubles = kBmaxN * 32 + kBmaxN / 2;  // per-CTA scratch: inverses + interchanges

// Shared-memory layout (bytes) for storage type T and panel width NB: the
// panel P, the diagonal-block inverse / solve staging X (NB x (NB + 1)), the
// left-looking dots Y (NB x kRC) and, for refined plans whose panel is
// smaller than two right-hand-side chunks, the solution chunk BS.  The
// solves' chunk R (and the refined plans' solution chunk otherwise) alias
// the panel, which the factorization no longer needs by then.
constexpr size_t kChunkBytes = (size_t)kRC * kBmaxN * 8;
template <typename T, int NB>
struct BL {
  static constexpr int kXLD = NB + 1;
  static constexpr size_t kPBytes = (size_t)NB * kPLD * sizeof(T);
  static constexpr bool kOwnBS = sizeof(T) == 4 && kPBytes < 2 * kChunkBytes;
  static constexpr size_t kOffX = (kPBytes + 15) & ~size_t(15);
  static constexpr size_t kOffY = kOffX + (size_t)NB * kXLD * 8;
  static constexpr size_t kOffB = kOffY + (size_t)NB * kRC * 8;
  static constexpr size_t kBytes = kOffB + (kOwnBS ? kChunkBytes : 0);
  static_assert(kPBytes >= kChunkBytes, "the solves' chunk aliases the panel");
};

struct BatchArgs {
  const BatchItem* items;
  int count;
  int* counter;
  int* info;
  int* iters;
  double* scratch;
};

// ------------------------------------------------------------ element I/O --
template <typename T> struct Pair2;
template <> struct Pair2<double> { using type = double2; };
template <> struct Pair2<float> { using type = float2; };

template <typename T>
__device__ __forceinline__ double ldv(const T* p) { return (double)*p; }
template <typename T>
__device__ __forceinline__ void stv(T* p, double v) { *p = (T)v; }
template <typename T>
__device__ __forceinline__ void ld_pair(const T* p, double& x, double& y) {
  const typename Pair2<T>::type v = *reinterpret_cast<const typename Pair2<T>::type*>(p);
  x = (double)v.x;
  y = (double)v.y;
}
template <typename T>
__device__ __forceinline__ void st_pair(T* p, double x, double y) {
  typename Pair2<T>::type v;
  v.x = (T)x;
  v.y = (T)y;
  *reinterpret_cast<typename Pair2<T>::type*>(p) = v;
}
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_el(T* d, const T* s) {
  if constexpr (sizeof(T) == 8) cp_async8(d, s);
  else cp_async4(d, s);
}

// Max of v over the CTA (every thread gets it).  red: NT/32 doubles.
template <int NT>
__device__ __forceinline__ double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();  // earlier readers of red are done
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double r = red[0];
#pragma unroll
  for (int w = 1; w < NT / 32; ++w) r = fmax(r, red[w]);
  return r;
}

// ------------------------------------------------------- DMMA warp tiles --
// C (32x32 warp tile at (prow, pcol) of the m2 x m2 trailing lower
// triangle, global) -= P[pb + rows] P[pb + cols]^T with P the NB-wide panel
// in shared memory ([k][r], ld kPLD); only r >= c is written.
template <typename T, int NB>
__device__ __forceinline__ void tile_syrk(T* C, long long ldc, bool cvec, const T* P, int prow, int pcol, int m2,
                                          int pb) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  double acc[2][4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int row = prow + 2 * g + ((r >= 2) ? 16 : 0);
      const int col = pcol + (j >> 1) * 16 + 2 * (2 * t + (r & 1)) + (j & 1);
      const bool v0 = row < m2 && col < m2 && row >= col;
      const bool v1 = row + 1 < m2 && col < m2 && row + 1 >= col;
      const T* cp = C + (long long)col * ldc + row;
      double c0 = 0.0, c1 = 0.0;
      if (cvec && v0 && v1) {
        ld_pair(cp, c0, c1);
      } else {
        if (v0) c0 = ldv(cp);
        if (v1) c1 = ldv(cp + 1);
      }
      acc[0][j][r] = -c0;
      acc[1][j][r] = -c1;
    }
#pragma unroll
  for (int ks = 0; ks < NB / 8; ++ks) {
    const int ke = ks * 8 + 2 * t;
    double af[2][4], bf[4][2];
    {
      const int m0 = pb + prow + 2 * g;
      double x00, y00, x01, y01, x10, y10, x11, y11;
      ld_pair(P + ke * kPLD + m0, x00, y00);
      ld_pair(P + (ke + 1) * kPLD + m0, x01, y01);
      ld_pair(P + ke * kPLD + m0 + 16, x10, y10);
      ld_pair(P + (ke + 1) * kPLD + m0 + 16, x11, y11);
      af[0][0] = x00; af[0][1] = x10; af[0][2] = x01; af[0][3] = x11;
      af[1][0] = y00; af[1][1] = y10; af[1][2] = y01; af[1][3] = y11;
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int n0 = pb + pcol + q * 16 + 2 * g;
      double x0, y0, x1, y1;
      ld_pair(P + ke * kPLD + n0, x0, y0);
      ld_pair(P + (ke + 1) * kPLD + n0, x1, y1);
      bf[2 * q][0] = x0; bf[2 * q][1] = x1;
      bf[2 * q + 1][0] = y0; bf[2 * q + 1][1] = y1;
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma_16x8x8(acc[i][j], af[i], bf[j]);
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int row = prow + 2 * g + ((r >= 2) ? 16 : 0);
      const int col = pcol + (j >> 1) * 16 + 2 * (2 * t + (r & 1)) + (j & 1);
      const bool v0 = row < m2 && col < m2 && row >= col;
      const bool v1 = row + 1 < m2 && col < m2 && row + 1 >= col;
      T* cp = C + (long long)col * ldc + row;
      if (cvec && v0 && v1) {
        st_pair(cp, -acc[0][j][r], -acc[1][j][r]);
      } else {
        if (v0) stv(cp, -acc[0][j][r]);
        if (v1) stv(cp + 1, -acc[1][j][r]);
      }
    }
}

// C (32x32 warp tile, global) -= P[pb + rows] * U[:, cols] where P is the
// panel in shared memory and U the NB x ncols row block right of the panel
// in global memory (column-major: the k pairs of one column are adjacent).
template <typename T, int NB>
__device__ __forceinline__ void tile_gemm(T* C, long long ldc, bool cvec, const T* P, const T* U, long long ldu,
                                          int prow, int pcol, int mrows, int ncols, int pb) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  double acc[2][4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int row = prow + 2 * g + ((r >= 2) ? 16 : 0);
      const int col = pcol + 8 * j + 2 * t + (r & 1);
      const bool v0 = row < mrows && col < ncols;
      const bool v1 = row + 1 < mrows && col < ncols;
      const T* cp = C + (long long)col * ldc + row;
      double c0 = 0.0, c1 = 0.0;
      if (cvec && v0 && v1) {
        ld_pair(cp, c0, c1);
      } else {
        if (v0) c0 = ldv(cp);
        if (v1) c1 = ldv(cp + 1);
      }
      acc[0][j][r] = -c0;
      acc[1][j][r] = -c1;
    }
#pragma unroll
  for (int ks = 0; ks < NB / 8; ++ks) {
    const int ke = ks * 8 + 2 * t;
    double af[2][4], bf[4][2];
    {
      const int m0 = pb + prow + 2 * g;
      double x00, y00, x01, y01, x10, y10, x11, y11;
      ld_pair(P + ke * kPLD + m0, x00, y00);
      ld_pair(P + (ke + 1) * kPLD + m0, x01, y01);
      ld_pair(P + ke * kPLD + m0 + 16, x10, y10);
      ld_pair(P + (ke + 1) * kPLD + m0 + 16, x11, y11);
      af[0][0] = x00; af[0][1] = x10; af[0][2] = x01; af[0][3] = x11;
      af[1][0] = y00; af[1][1] = y10; af[1][2] = y01; af[1][3] = y11;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int col = pcol + 8 * j + g;
      bf[j][0] = 0.0;
      bf[j][1] = 0.0;
      if (col < ncols) {
        const T* up = U + (long long)col * ldu + ke;
        if (cvec) {
          ld_pair(up, bf[j][0], bf[j][1]);
        } else {
          bf[j][0] = ldv(up);
          bf[j][1] = ldv(up + 1);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma_16x8x8(acc[i][j], af[i], bf[j]);
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int row = prow + 2 * g + ((r >= 2) ? 16 : 0);
      const int col = pcol + 8 * j + 2 * t + (r & 1);
      const bool v0 = row < mrows && col < ncols;
      const bool v1 = row + 1 < mrows && col < ncols;
      T* cp = C + (long long)col * ldc + row;
      if (cvec && v0 && v1) {
        st_pair(cp, -acc[0][j][r], -acc[1][j][r]);
      } else {
        if (v0) stv(cp, -acc[0][j][r]);
        if (v1) stv(cp + 1, -acc[1][j][r]);
      }
    }
}

// ------------------------------------------------ diagonal-block kernels --
// Lower Cholesky of the b x b top of the panel (b <= NB <= 32) by one warp,
// the LVar3Unb steps (Cholesky/LVar3.hpp:19-49: alpha11 := sqrt(alpha11),
// a21 := a21 / alpha11, A22 -= a21 a21^H) with lane r holding row r in
// registers; the scaling multiplies by the correctly rounded reciprocal.
// Stores L (rounded to T) into P and 1 / L(i,i) of the stored values into
// rd.  Returns 0 or the 1-based column of a non-positive pivot (warp-uniform).
template <typename T, int NB>
__device__ int diag_chol_warp(T* P, int b, double* rd) {
  const int lane = threadIdx.x & 31;
  double a[NB];
#pragma unroll
  for (int k = 0; k < NB; ++k) a[k] = (lane < b && k < b && k <= lane) ? ldv(P + k * kPLD + lane) : 0.0;
  int fail = 0;
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    if (j < b && fail == 0) {
      const double d = __shfl_sync(0xffffffffu, a[j], j);
      if (d <= 0.0) {
        fail = j + 1;
      } else {
        const double s = sqrt(d);
        const double rs = __drcp_rn(s);
        if (lane == j) a[j] = s;
        else if (lane > j) a[j] *= rs;
#pragma unroll
        for (int k = j + 1; k < NB; ++k) {
          const double lkj = __shfl_sync(0xffffffffu, a[j], k);
          if (lane >= k) a[k] = fma(-a[j], lkj, a[k]);
        }
      }
    }
  }
  if (fail) return fail;
#pragma unroll
  for (int k = 0; k < NB; ++k)
    if (lane < b && k < b && k <= lane) stv(P + k * kPLD + lane, a[k]);
  __syncwarp();
  if (lane < b) rd[lane] = __drcp_rn(ldv(P + lane * kPLD + lane));
  __syncwarp();
  return 0;
}

// Column `lane` of the inverse of the b x b triangle in the panel's top
// rows (P[col][row], ld kPLD), by one warp: LOWER (UNIT: unit diagonal) or
// UPPER, rd[m] = 1 / T(m, m).  The inverse's column is formed right-looking
// (x_m = -S_m * rd_m, then S_i += T(i, m) x_m), so the dependent chain per
// step is one multiply and one FMA.  out[m + c * ldo] receives the triangle
// (the unit lower form leaves the diagonal alone).
template <typename T, int NB, bool UPPER, bool UNIT>
__device__ void tri_inv_warp(const T* P, int b, const double* rd, double* out, int ldo) {
  const int c = threadIdx.x & 31;
  double S[NB];
#pragma unroll
  for (int i = 0; i < NB; ++i) S[i] = 0.0;
  if constexpr (!UPPER) {
#pragma unroll
    for (int m = 0; m < NB; ++m) {
      if (m < b) {
        const double r = UNIT ? 1.0 : rd[m];
        double x = (m == c) ? r : -S[m] * r;
        if (m < c) x = 0.0;
        if (c < b && m >= c && !(UNIT && m == c)) out[m + c * ldo] = x;
#pragma unroll
        for (int i = m + 1; i < NB; ++i) S[i] = fma(ldv(P + m * kPLD + i), x, S[i]);
      }
    }
  } else {
#pragma unroll
    for (int m = NB - 1; m >= 0; --m) {
      if (m < b) {
        const double r = rd[m];
        double x = (m == c) ? r : -S[m] * r;
        if (m > c) x = 0.0;
        if (c < b && m <= c) out[m + c * ldo] = x;
#pragma unroll
        for (int i = 0; i < m; ++i) S[i] = fma(ldv(P + m * kPLD + i), x, S[i]);
      }
    }
  }
}

// LU with partial pivoting of the m x b panel in shared memory (lu::Panel,
// LU/Panel.hpp:19-89: the entry of largest magnitude, the first in row
// order on ties; zero pivot -> singular; a21 *= 1/alpha11; A22 -= a21 a12).
// The chosen row is marked done instead of swapped; every thread keeps the
// current position of the rows it owns (rows tid + t * NT), so the sequential
// interchange semantics (position j <-> position p_j) hold and a column
// costs one CTA barrier.  Afterwards the panel rows are permuted into
// position order in place; s_mv receives the (from, to) row moves and
// s_piv[j] the position swapped with j at step j.  Returns 0 or the 1-based
// column of a zero pivot (CTA-uniform).
template <typename T, int NB, int NT>
__device__ int lu_panel_smem(T* P, int m, int b, int* s_piv, int* s_mv, int* s_nmv, double* s_rv, int* s_rp,
                             int* s_rh) {
  constexpr int RPT = kBmaxN / NT;
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int pos[RPT];
  bool done[RPT];
#pragma unroll
  for (int t = 0; t < RPT; ++t) {
    pos[t] = tid + t * NT;
    done[t] = pos[t] >= m;
  }
  for (int j = 0; j < b; ++j) {
    double best = -1.0;
    int bpos = INT_MAX, bphys = -1;
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
      if (!done[t]) {
        const double v = fabs(ldv(P + j * kPLD + tid + t * NT));
        if (v > best || (v == best && pos[t] < bpos)) {
          best = v;
          bpos = pos[t];
          bphys = tid + t * NT;
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int op = __shfl_xor_sync(0xffffffffu, bpos, o);
      const int oh = __shfl_xor_sync(0xffffffffu, bphys, o);
      if (ob > best || (ob == best && op < bpos)) {
        best = ob;
        bpos = op;
        bphys = oh;
      }
    }
    const int par = (j & 1) * NW;
    if (lane == 0) {
      s_rv[par + warp] = best;
      s_rp[par + warp] = bpos;
      s_rh[par + warp] = bphys;
    }
    __syncthreads();
    best = s_rv[par];
    bpos = s_rp[par];
    bphys = s_rh[par];
#pragma unroll
    for (int w = 1; w < NW; ++w) {
      const double ob = s_rv[par + w];
      const int op = s_rp[par + w];
      if (ob > best || (ob == best && op < bpos)) {
        best = ob;
        bpos = op;
        bphys = s_rh[par + w];
      }
    }
    if (bphys < 0) return j + 1;
    const double pv = ldv(P + j * kPLD + bphys);
    if (pv == 0.0) return j + 1;
    if (tid == 0) s_piv[j] = bpos;
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
      if (pos[t] == j) pos[t] = bpos;
      if (tid + t * NT == bphys) {
        done[t] = true;
        pos[t] = j;
      }
    }
    const double rp = __drcp_rn(pv);
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
      if (!done[t]) {
        const int r = tid + t * NT;
        const double l = ldv(P + j * kPLD + r) * rp;
        stv(P + j * kPLD + r, l);
        for (int c = j + 1; c < b; ++c)
          stv(P + c * kPLD + r, fma(-l, ldv(P + c * kPLD + bphys), ldv(P + c * kPLD + r)));
      }
    }
  }
  // the row moves, then the panel rows into position order
  if (tid == 0) *s_nmv = 0;
  __syncthreads();
#pragma unroll
  for (int t = 0; t < RPT; ++t) {
    const int r = tid + t * NT;
    if (r < m && pos[t] != r) {
      const int k = atomicAdd(s_nmv, 1);
      s_mv[2 * k] = r;
      s_mv[2 * k + 1] = pos[t];
    }
  }
  __syncthreads();
  const int nmv = *s_nmv;
  constexpr int kPer = (2 * NB * NB + NT - 1) / NT;
  double v[kPer];
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int e = tid + u * NT;
    if (e < nmv * b) v[u] = ldv(P + (e / nmv) * kPLD + s_mv[2 * (e % nmv)]);
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int e = tid + u * NT;
    if (e < nmv * b) stv(P + (e / nmv) * kPLD + s_mv[2 * (e % nmv) + 1], v[u]);
  }
  __syncthreads();
  return 0;
}

// ------------------------------------------------------------ factorizations --
// Shared-memory work areas of one CTA (pointers into the dynamic block plus
// the static scalars); X is NB x (NB + 1), Y is NB x kBmaxRHS doubles.
struct BWork {
  double* X;
  double* Y;
  double* BS;
  double* rd;
  double* red;
  int* piv;
  int* mv;
  int* nmv;
  int* ri;
  int* rh;
  int* flag;
};

// Lower Cholesky of F (n x n, ldf) in place (LVar3 blocked right-looking,
// Cholesky/LVar3.hpp:83-123), the diagonal-block inverses into Xg (NB x NB
// blocks, ld NB).  Returns 0 or the 1-based column of a non-positive pivot.
template <typename T, int NB, int NT>
__device__ int chol_factor(T* F, long long ldf, int n, T* P, const BWork& w, double* Xg) {
  constexpr int kXLD = NB + 1;
  const int tid = threadIdx.x, warp = tid >> 5;
  const bool cvec = (reinterpret_cast<uintptr_t>(F) % (2 * sizeof(T)) == 0) && (ldf % 2 == 0);
  for (int k0 = 0; k0 < n; k0 += NB) {
    const int b = min(NB, n - k0), m = n - k0;
    for (int c = 0; c < b; ++c)
      for (int r = c + tid; r < m; r += NT) cp_async_el(&P[c * kPLD + r], &F[(long long)(k0 + c) * ldf + k0 + r]);
    cp_async_wait_all();
    __syncthreads();
    if (warp == 0) {
      const int f = diag_chol_warp<T, NB>(P, b, w.rd);
      if (tid == 0) *w.flag = f;
      if (f == 0) tri_inv_warp<T, NB, false, false>(P, b, w.rd, w.X, kXLD);
    }
    __syncthreads();
    if (*w.flag) {
      const int f = k0 + *w.flag;
      __syncthreads();
      return f;
    }
    // keep inv(L11) for the solve; L21 := A21 inv(L11)^T, one row per thread
    double* Xb = Xg + (size_t)(k0 / NB) * NB * NB;
    for (int e = tid; e < NB * NB; e += NT) {
      const int i = e % NB, c = e / NB;
      Xb[e] = (i < b && c < b && i >= c) ? w.X[i + c * kXLD] : 0.0;
    }
    for (int r = b + tid; r < m; r += NT) {
      double a[NB];
#pragma unroll
      for (int k = 0; k < NB; ++k) a[k] = (k < b) ? ldv(P + k * kPLD + r) : 0.0;
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        if (c < b) {
          double s = 0.0;
#pragma unroll
          for (int k = 0; k <= c; ++k) s = fma(a[k], w.X[c + k * kXLD], s);
          stv(P + c * kPLD + r, s);
        }
      }
    }
    __syncthreads();
    for (int c = 0; c < b; ++c)
      for (int r = c + tid; r < m; r += NT) F[(long long)(k0 + c) * ldf + k0 + r] = P[c * kPLD + r];
    const int m2 = m - b;
    if (m2 > 0) {
      const int nt = (m2 + 31) / 32;
      const int ntile = nt * (nt + 1) / 2;
      T* C = F + (long long)(k0 + b) * ldf + (k0 + b);
      for (int tt = warp; tt < ntile; tt += NT / 32) {
        int ti = (int)((sqrt(8.0 * tt + 1.0) - 1.0) * 0.5);  // triangular index -> (ti, tj), ti >= tj
        while ((ti + 1) * (ti + 2) / 2 <= tt) ++ti;
        while (ti * (ti + 1) / 2 > tt) --ti;
        const int tj = tt - ti * (ti + 1) / 2;
        tile_syrk<T, NB>(C, ldf, cvec, P, ti * 32, tj * 32, m2, b);
      }
    }
    __syncthreads();
  }
  return 0;
}

// LU with partial pivoting of F (n x n, ldf) in place (LU.hpp:144-218, the
// RowEchelon form of GaussianElimination.hpp:94-209: a panel's interchanges
// are applied to the panel and the columns right of it).  Xg receives per
// diagonal block inv(unit L11) below the diagonal and inv(U11) on and above
// it; piv[k] the absolute row swapped with row k.  Returns 0 or the 1-based
// column of a zero pivot.
template <typename T, int NB, int NT>
__device__ int lu_factor(T* F, long long ldf, int n, T* P, const BWork& w, double* Xg, int* piv) {
  constexpr int kXLD = NB + 1;
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool cvec = (reinterpret_cast<uintptr_t>(F) % (2 * sizeof(T)) == 0) && (ldf % 2 == 0);
  for (int k0 = 0; k0 < n; k0 += NB) {
    const int b = min(NB, n - k0), m = n - k0;
    for (int c = 0; c < b; ++c)
      for (int r = tid; r < m; r += NT) cp_async_el(&P[c * kPLD + r], &F[(long long)(k0 + c) * ldf + k0 + r]);
    cp_async_wait_all();
    __syncthreads();
    const int f = lu_panel_smem<T, NB, NT>(P, m, b, w.piv, w.mv, w.nmv, w.red, w.ri, w.rh);
    if (f) {
      __syncthreads();
      return k0 + f;
    }
    const int nmv = *w.nmv;
    // panel back in position order; interchanges on the columns to its right
    for (int c = 0; c < b; ++c)
      for (int r = tid; r < m; r += NT) F[(long long)(k0 + c) * ldf + k0 + r] = P[c * kPLD + r];
    if (tid < b) piv[k0 + tid] = k0 + w.piv[tid];
    const int ncr = n - k0 - b;
    for (int c0 = warp; c0 < ncr; c0 += 4 * NW) {
      T v[4][2];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int c = c0 + u * NW;
        if (c < ncr) {
          const T* col = F + (long long)(k0 + b + c) * ldf + k0;
          if (lane < nmv) v[u][0] = col[w.mv[2 * lane]];
          if (lane + 32 < nmv) v[u][1] = col[w.mv[2 * (lane + 32)]];
        }
      }
      __syncwarp();
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int c = c0 + u * NW;
        if (c < ncr) {
          T* col = F + (long long)(k0 + b + c) * ldf + k0;
          if (lane < nmv) col[w.mv[2 * lane + 1]] = v[u][0];
          if (lane + 32 < nmv) col[w.mv[2 * (lane + 32) + 1]] = v[u][1];
        }
      }
    }
    __syncthreads();
    // warps 0 / 1: inv(unit L11) / inv(U11); the others: U12 := inv(unit L11) A12
    if (warp == 1 && lane < b) w.rd[lane] = __drcp_rn(ldv(P + lane * kPLD + lane));
    if (warp == 0) tri_inv_warp<T, NB, false, true>(P, b, w.rd, w.X, kXLD);
    if (warp == 1) {
      __syncwarp();
      tri_inv_warp<T, NB, true, false>(P, b, w.rd, w.X, kXLD);
    }
    for (int c = tid - 64; tid >= 64 && c < ncr; c += NT - 64) {
      T* col = F + (long long)(k0 + b + c) * ldf + k0;
      double u[NB];
#pragma unroll
      for (int i = 0; i < NB; ++i) u[i] = (i < b) ? ldv(col + i) : 0.0;
#pragma unroll
      for (int i = 1; i < NB; ++i) {
        if (i < b) {
          double s = u[i];
#pragma unroll
          for (int q = 0; q < i; ++q) s = fma(-ldv(P + q * kPLD + i), u[q], s);
          u[i] = (double)(T)s;
        }
      }
#pragma unroll
      for (int i = 1; i < NB; ++i)
        if (i < b) stv(col + i, u[i]);
    }
    __syncthreads();
    double* Xb = Xg + (size_t)(k0 / NB) * NB * NB;
    for (int e = tid; e < NB * NB; e += NT) {
      const int i = e % NB, c = e / NB;
      Xb[e] = (i < b && c < b) ? w.X[i + c * kXLD] : 0.0;
    }
    // trailing update A22 -= L21 U12
    const int m2 = m - b;
    if (m2 > 0 && ncr > 0) {
      const int tr = (m2 + 31) / 32, tc = (ncr + 31) / 32;
      T* C = F + (long long)(k0 + b) * ldf + (k0 + b);
      const T* U = F + (long long)(k0 + b) * ldf + k0;
      for (int tt = warp; tt < tr * tc; tt += NW)
        tile_gemm<T, NB>(C, ldf, cvec, P, U, ldf, (tt % tr) * 32, (tt / tr) * 32, m2, ncr, b);
    }
    __syncthreads();
  }
  return 0;
}

// ------------------------------------------------------------------ solves --
// R (shared, R[q * kBmaxN + i], nr <= kRC columns) := op(factor)^-1 R, blocked
// by NB with the diagonal-block inverses in Xg.
//   LU = false: L L^T (cholesky::SolveAfter, Cholesky/SolveAfter.hpp:20-75):
//     forward with L (right-looking), backward with L^T (left-looking dots).
//   LU = true: the panels' interchanges and unit L block by block, then U
//     (the RowEchelon elimination applied to R, then lu::SolveAfter's U step).
template <typename T, int NB, int NT, bool LU>
__device__ void solve_smem(const T* F, long long ldf, int n, int nr, const double* Xg, const int* piv, double* R,
                           const BWork& w) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = NT / 32;
  double* stage = w.X;  // bi x nr
  const int nblk = (n + NB - 1) / NB;
  for (int ib = 0; ib < nblk; ++ib) {
    const int i0 = ib * NB, bi = min(NB, n - i0);
    if (LU) {
      if (tid < nr) {
        double* rq = R + tid * kBmaxN;
        for (int j = 0; j < bi; ++j) {
          const int p = piv[i0 + j];
          if (p != i0 + j) {
            const double t0 = rq[i0 + j];
            rq[i0 + j] = rq[p];
            rq[p] = t0;
          }
        }
      }
      __syncthreads();
    }
    const double* Xi = Xg + (size_t)ib * NB * NB;
    for (int e = tid; e < bi * nr; e += NT) {
      const int i = e % bi, q = e / bi;
      const double* rq = R + q * kBmaxN + i0;
      double s = LU ? rq[i] : 0.0;
      const int kend = LU ? i : i + 1;
      for (int k = 0; k < kend; ++k) s = fma(Xi[i + k * NB], rq[k], s);
      stage[e] = s;
    }
    __syncthreads();
    for (int e = tid; e < bi * nr; e += NT) R[(e / bi) * kBmaxN + i0 + e % bi] = stage[e];
    for (int r = i0 + bi + tid; r < n; r += NT) {
      double acc[kRC];
#pragma unroll
      for (int q = 0; q < kRC; ++q) acc[q] = 0.0;
      for (int k = 0; k < bi; ++k) {
        const double l = ldv(F + (long long)(i0 + k) * ldf + r);
#pragma unroll
        for (int q = 0; q < kRC; ++q)
          if (q < nr) acc[q] = fma(l, stage[k + q * bi], acc[q]);
      }
#pragma unroll
      for (int q = 0; q < kRC; ++q)
        if (q < nr) R[q * kBmaxN + r] -= acc[q];
    }
    __syncthreads();
  }
  for (int ib = nblk - 1; ib >= 0; --ib) {
    const int i0 = ib * NB, bi = min(NB, n - i0);
    const double* Xi = Xg + (size_t)ib * NB * NB;
    if (!LU) {
      // D = L(below, block)^T X(below): one warp per column, lanes over rows
      double* D = w.Y;  // bi x nr
      for (int c = warp; c < bi; c += NW) {
        double acc[kRC];
#pragma unroll
        for (int q = 0; q < kRC; ++q) acc[q] = 0.0;
        const T* lc = F + (long long)(i0 + c) * ldf;
        for (int r = i0 + bi + lane; r < n; r += 32) {
          const double l = ldv(lc + r);
#pragma unroll
          for (int q = 0; q < kRC; ++q)
            if (q < nr) acc[q] = fma(l, R[q * kBmaxN + r], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < kRC; ++q) {
          if (q < nr) {
            double v = acc[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) D[c + q * bi] = v;
          }
        }
      }
      __syncthreads();
      for (int e = tid; e < bi * nr; e += NT) {
        const int i = e % bi, q = e / bi;
        const double* rq = R + q * kBmaxN + i0;
        double s = 0.0;
        for (int k = i; k < bi; ++k) s = fma(Xi[k + i * NB], rq[k] - D[k + q * bi], s);
        stage[e] = s;
      }
      __syncthreads();
      for (int e = tid; e < bi * nr; e += NT) R[(e / bi) * kBmaxN + i0 + e % bi] = stage[e];
      __syncthreads();
    } else {
      for (int e = tid; e < bi * nr; e += NT) {
        const int i = e % bi, q = e / bi;
        const double* rq = R + q * kBmaxN + i0;
        double s = 0.0;
        for (int k = i; k < bi; ++k) s = fma(Xi[i + k * NB], rq[k], s);
        stage[e] = s;
      }
      __syncthreads();
      for (int e = tid; e < bi * nr; e += NT) R[(e / bi) * kBmaxN + i0 + e % bi] = stage[e];
      for (int r = tid; r < i0; r += NT) {
        double acc[kRC];
#pragma unroll
        for (int q = 0; q < kRC; ++q) acc[q] = 0.0;
        for (int k = 0; k < bi; ++k) {
          const double u = ldv(F + (long long)(i0 + k) * ldf + r);
#pragma unroll
          for (int q = 0; q < kRC; ++q)
            if (q < nr) acc[q] = fma(u, stage[k + q * bi], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < kRC; ++q)
          if (q < nr) R[q * kBmaxN + r] -= acc[q];
      }
      __syncthreads();
    }
  }
}

// Chunk [q0, q0 + nr) of B (global) -> R, R -> B.
template <int NT>
__device__ __forceinline__ void load_chunk(double* R, const double* B, long long ldb, int n, int q0, int nr) {
  for (int e = threadIdx.x; e < n * nr; e += NT) R[(e / n) * kBmaxN + e % n] = B[(long long)(q0 + e / n) * ldb + e % n];
}
template <int NT>
__device__ __forceinline__ void store_chunk(const double* R, double* B, long long ldb, int n, int q0, int nr) {
  for (int e = threadIdx.x; e < n * nr; e += NT) B[(long long)(q0 + e / n) * ldb + e % n] = R[(e / n) * kBmaxN + e % n];
}

// ------------------------------------------------------------- refinement --
// F := T(A) (HPD: the lower triangle; GE: all of it), returning ||A||_inf of
// the matrix A stands for (HPD: the symmetric one its lower triangle holds).
template <typename T, bool HPD, int NT>
__device__ double convert_norm(const double* A, long long lda, int n, T* F, long long ldf, double* red) {
  double rmax = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) {
    double rs = 0.0;
    for (int k = 0; k < n; ++k) {
      double a;
      if (HPD) {
        a = (k <= i) ? A[i + (long long)k * lda] : A[k + (long long)i * lda];
        if (k <= i) F[i + (long long)k * ldf] = (T)a;
      } else {
        a = A[i + (long long)k * lda];
        F[i + (long long)k * ldf] = (T)a;
      }
      rs += fabs(a);
    }
    rmax = fmax(rmax, rs);
  }
  return block_max<NT>(rmax, red);
}

// R := B(:, q0 : q0 + nr) - A X (FP64), X = XS (shared); returns the
// backward error max_q ||r_q||_inf / (||A||_inf ||x_q||_inf + ||b_q||_inf).
template <bool HPD, int NT>
__device__ double residual(const double* A, long long lda, int n, const double* B, long long ldb, int q0, int nr,
                           const double* XS, double* R, bool x_zero, double anorm, double* red) {
  double rmax[kRC], xmax[kRC], bmax[kRC];
#pragma unroll
  for (int q = 0; q < kRC; ++q) rmax[q] = xmax[q] = bmax[q] = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) {
    double acc[kRC];
#pragma unroll
    for (int q = 0; q < kRC; ++q) {
      acc[q] = 0.0;
      if (q < nr) {
        acc[q] = B[(long long)(q0 + q) * ldb + i];
        bmax[q] = fmax(bmax[q], fabs(acc[q]));
        xmax[q] = fmax(xmax[q], fabs(XS[q * kBmaxN + i]));
      }
    }
    if (!x_zero) {
#pragma unroll 4
      for (int k = 0; k < n; ++k) {
        const double* ap = HPD ? ((k <= i) ? A + i + (long long)k * lda : A + k + (long long)i * lda)
                               : A + i + (long long)k * lda;
        const double a = *ap;
#pragma unroll
        for (int q = 0; q < kRC; ++q)
          if (q < nr) acc[q] = fma(-a, XS[q * kBmaxN + k], acc[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < kRC; ++q) {
      if (q < nr) {
        R[q * kBmaxN + i] = acc[q];
        rmax[q] = fmax(rmax[q], fabs(acc[q]));
      }
    }
  }
  // one CTA reduction for the 3 x kRC maxima: warps, then across warps
  constexpr int NW = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < kRC; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      rmax[q] = fmax(rmax[q], __shfl_xor_sync(0xffffffffu, rmax[q], o));
      xmax[q] = fmax(xmax[q], __shfl_xor_sync(0xffffffffu, xmax[q], o));
      bmax[q] = fmax(bmax[q], __shfl_xor_sync(0xffffffffu, bmax[q], o));
    }
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < kRC; ++q) {
      red[(3 * q) * NW + warp] = rmax[q];
      red[(3 * q + 1) * NW + warp] = xmax[q];
      red[(3 * q + 2) * NW + warp] = bmax[q];
    }
  __syncthreads();
  if (threadIdx.x < 3 * kRC) {
    double v = red[threadIdx.x * NW];
    for (int k = 1; k < NW; ++k) v = fmax(v, red[threadIdx.x * NW + k]);
    red[3 * kRC * NW + threadIdx.x] = v;
  }
  __syncthreads();
  const double* fin = red + 3 * kRC * NW;
  double berr = 0.0;
  for (int q = 0; q < nr; ++q) {
    const double rr = fin[3 * q], den = anorm * fin[3 * q + 1] + fin[3 * q + 2];
    berr = fmax(berr, den > 0.0 ? rr / den : (rr > 0.0 ? INFINITY : 0.0));
  }
  return berr;
}

// Iterative refinement of chunk [q0, q0 + nr) with the working factor:
// X = 0; repeat r = b - A x (FP64), stop at backward error <= kIRTol,
// d = factor^-1 r, x += d.  X ends in B.  Returns the corrections applied,
// or -1 when the refinement stalls (then B is left unchanged).
template <typename T, int NB, int NT, bool HPD>
__device__ int refine_chunk(const double* A, long long lda, int n, double* B, long long ldb, int q0, int nr,
                            const T* F, long long ldf, const double* Xg, const int* piv, double anorm, double* XS,
                            double* R, const BWork& w) {
  for (int e = threadIdx.x; e < kRC * kBmaxN; e += NT) XS[e] = 0.0;
  __syncthreads();
  double prev = INFINITY;
  for (int it = 0; it <= kIRMax; ++it) {
    const double berr = residual<HPD, NT>(A, lda, n, B, ldb, q0, nr, XS, R, it == 0, anorm, w.red);
    if (berr <= kIRTol) {
      __syncthreads();
      store_chunk<NT>(XS, B, ldb, n, q0, nr);
      __syncthreads();
      return it;
    }
    if (it == kIRMax || !(berr == berr) || (it >= 2 && berr > 0.5 * prev)) {
      __syncthreads();
      return -1;
    }
    prev = berr;
    __syncthreads();
    solve_smem<T, NB, NT, !HPD>(F, ldf, n, nr, Xg, piv, R, w);
    for (int e = threadIdx.x; e < n * nr; e += NT) XS[(e / n) * kBmaxN + e % n] += R[(e / n) * kBmaxN + e % n];
    __syncthreads();
  }
  return -1;
}

// ------------------------------------------------------------------ kernels --
// KIND 0: HPDSolve(LOWER) per system; KIND 1: GaussianElimination per system.
// T double: FP64 plan (A receives the factor, B the solution); T float:
// refined plan (A unchanged, F the FP32 working copy, B the solution).
// info[id] = 0 or the 1-based column where the (FP64) factorization stopped;
// iters[id] = refinement corrections, -1 = solved by the FP64 fallback.
template <typename T, int NB, int NT, int MINB, int KIND>
__global__ void __launch_bounds__(NT, MINB) batched_kernel(BatchArgs args) {
  extern __shared__ __align__(16) unsigned char sm_dyn[];
  using LY = BL<T, NB>;
  constexpr bool kRefined = sizeof(T) == 4;
  constexpr bool kHPD = KIND == 0;
  __shared__ double s_rd[32];
  __shared__ double s_red[3 * kRC * (NT / 32) + 3 * kRC];
  __shared__ int s_piv[32];
  __shared__ int s_mv[2 * 64];
  __shared__ int s_nmv, s_idx, s_flag;
  __shared__ int s_ri[2 * (NT / 32)], s_rh[2 * (NT / 32)];
  T* P = reinterpret_cast<T*>(sm_dyn);
  BWork w;
  w.X = reinterpret_cast<double*>(sm_dyn + LY::kOffX);
  w.Y = reinterpret_cast<double*>(sm_dyn + LY::kOffY);
  w.BS = reinterpret_cast<double*>(sm_dyn + (LY::kOwnBS ? LY::kOffB : kChunkBytes));
  w.rd = s_rd;
  w.red = s_red;
  w.piv = s_piv;
  w.mv = s_mv;
  w.nmv = &s_nmv;
  w.ri = s_ri;
  w.rh = s_rh;
  w.flag = &s_flag;
  const int tid = threadIdx.x;
  double* Xg = args.scratch + (size_t)blockIdx.x * kScrDoubles;
  int* pivg = reinterpret_cast<int*>(Xg + kBmaxN * 32);
  double* R = reinterpret_cast<double*>(sm_dyn);  // the solves' chunk (aliases the panel)
  while (true) {
    if (tid == 0) s_idx = atomicAdd(args.counter, 1);
    __syncthreads();
    const int idx = s_idx;
    __syncthreads();
    if (idx >= args.count) break;
    const BatchItem it = args.items[idx];
    const int n = it.n;
    const int nrhs = it.B ? it.nrhs : 0;
    int fail = 0, iters = 0;
    if constexpr (!kRefined) {
      fail = kHPD ? chol_factor<double, NB, NT>(it.A, it.lda, n, reinterpret_cast<double*>(P), w, Xg)
                  : lu_factor<double, NB, NT>(it.A, it.lda, n, reinterpret_cast<double*>(P), w, Xg, pivg);
      if (!fail) {
        for (int q0 = 0; q0 < nrhs; q0 += kRC) {
          const int nr = min(kRC, nrhs - q0);
          load_chunk<NT>(R, it.B, it.ldb, n, q0, nr);
          __syncthreads();
          solve_smem<double, NB, NT, !kHPD>(it.A, it.lda, n, nr, Xg, pivg, R, w);
          store_chunk<NT>(R, it.B, it.ldb, n, q0, nr);
          __syncthreads();
        }
      }
    } else {
      float* F32 = reinterpret_cast<float*>(it.F);
      const double anorm = convert_norm<float, kHPD, NT>(it.A, it.lda, n, F32, it.ldf, w.red);
      __syncthreads();
      int f32 = kHPD ? chol_factor<float, NB, NT>(F32, it.ldf, n, P, w, Xg)
                     : lu_factor<float, NB, NT>(F32, it.ldf, n, P, w, Xg, pivg);
      int q_fb = f32 ? 0 : -1;  // first chunk left to the FP64 fallback
      for (int q0 = 0; q0 < nrhs && q_fb < 0; q0 += kRC) {
        const int nr = min(kRC, nrhs - q0);
        const int k = refine_chunk<float, NB, NT, kHPD>(it.A, it.lda, n, it.B, it.ldb, q0, nr, F32, it.ldf, Xg,
                                                         pivg, anorm, w.BS, R, w);
        if (k < 0) q_fb = q0;
        else iters = max(iters, k);
      }
      if (q_fb >= 0) {
        // FP64 fallback in the working copy (panel NB / 2: the same bytes)
        constexpr int NB2 = NB / 2;
        double* F64 = reinterpret_cast<double*>(it.F);
        convert_norm<double, kHPD, NT>(it.A, it.lda, n, F64, it.ldf, w.red);
        __syncthreads();
        fail = kHPD ? chol_factor<double, NB2, NT>(F64, it.ldf, n, reinterpret_cast<double*>(P), w, Xg)
                    : lu_factor<double, NB2, NT>(F64, it.ldf, n, reinterpret_cast<double*>(P), w, Xg, pivg);
        if (!fail) {
          for (int q0 = q_fb; q0 < nrhs; q0 += kRC) {
            const int nr = min(kRC, nrhs - q0);
            load_chunk<NT>(R, it.B, it.ldb, n, q0, nr);
            __syncthreads();
            solve_smem<double, NB2, NT, !kHPD>(F64, it.ldf, n, nr, Xg, pivg, R, w);
            store_chunk<NT>(R, it.B, it.ldb, n, q0, nr);
            __syncthreads();
          }
        }
        iters = -1;
      }
    }
    if (tid == 0) {
      args.info[it.id] = fail;
      if (args.iters) args.iters[it.id] = iters;
    }
    __syncthreads();
  }
}

// Copies every system's A (n x n) and B (n x nrhs) to or from a packed
// backup (off[i]: offset of system i's copy), one CTA per system.
__global__ void batch_backup_kernel(const BatchItem* items, int count, double* bk, const long long* off, int dir) {
  for (int s = blockIdx.x; s < count; s += gridDim.x) {
    const BatchItem it = items[s];
    double* base = bk + off[s];
    const long long na = (long long)it.n * it.n, nb = it.B ? (long long)it.n * it.nrhs : 0;
    for (long long e = threadIdx.x; e < na + nb; e += blockDim.x) {
      double* g = e < na ? it.A + (e / it.n) * it.lda + e % it.n
                         : it.B + ((e - na) / it.n) * it.ldb + (e - na) % it.n;
      if (dir == 0) base[e] = *g;
      else *g = base[e];
    }
  }
}

// ------------------------------------------------------------------ variants --
typedef void (*BatchKernel)(BatchArgs);
struct Variant {
  BatchKernel kern[2];
  size_t smem;
  int nb, nt;
};

#define EGPU_BVAR(T, NB, NT, MINB) \
  { {batched_kernel<T, NB, NT, MINB, 0>, batched_kernel<T, NB, NT, MINB, 1>}, BL<T, NB>::kBytes, NB, NT }

// FP64 plans: (panel 32, 256 threads, one CTA per SM), (16, 256, two per SM),
// (16, 128, two per SM).  Refined plans: (32, 256, two per SM), (16, 256, two
// per SM), (32, 128, two per SM).
constexpr int kNumVariants = 3;
static const Variant kVariants[2][kNumVariants] = {
    {EGPU_BVAR(double, 32, 256, 1), EGPU_BVAR(double, 16, 256, 2), EGPU_BVAR(double, 16, 128, 2)},
    {EGPU_BVAR(float, 32, 256, 2), EGPU_BVAR(float, 16, 256, 2), EGPU_BVAR(float, 32, 128, 2)},
};
constexpr int kMaxPerSM = 4;
constexpr int kMaxClass = 3;
static const int kClassMax[kMaxClass] = {512, 256, 128};  // size classes, largest first

// Sets the kernel's shared-memory limit and returns the CTAs per SM it
// reaches (cached per device, so launches inside a stream capture make no
// attribute calls once a shape has run outside one).
static int variant_prepare(const Variant& v, int kind, int* per_sm) {
  constexpr int kMaxDev = 16;
  static int cache[kMaxDev][2][kNumVariants][2];
  int dev = 0;
  EGPU_CUDA_TRY(cudaGetDevice(&dev));
  const int prec = (&v >= &kVariants[1][0]) ? 1 : 0;
  const int vi = static_cast<int>(&v - &kVariants[prec][0]);
  int* slot = (dev < kMaxDev) ? &cache[dev][prec][vi][kind] : nullptr;
  if (slot && *slot > 0) {
    *per_sm = *slot;
    return EGPU_OK;
  }
  EGPU_CUDA_TRY(cudaFuncSetAttribute(v.kern[kind], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem));
  int occ = 0;
  EGPU_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, v.kern[kind], v.nt, v.smem));
  *per_sm = std::max(1, std::min(occ, kMaxPerSM));
  if (slot) *slot = *per_sm;
  return EGPU_OK;
}

static void sort_items(std::vector<BatchItem>& items) {
  std::stable_sort(items.begin(), items.end(), [](const BatchItem& a, const BatchItem& b) { return a.n > b.n; });
}

static bool bad_item(int n, int nrhs, int lda, int ldb, bool hasB) {
  return n < 0 || n > kBmaxN || nrhs < 0 || nrhs > kBmaxRHS || lda < std::max(1, n) ||
         (hasB && nrhs > 0 && ldb < std::max(1, n));
}

// Host side of the one-shot calls (egpu_dposv_batched / egpu_dgesv_batched):
// sort by size, upload the descriptors, launch the default FP64 shape, read
// back the statuses.  Buffers come from the handle workspace.
int egpu_batched_launch(int kind, cudaStream_t st, int sm_count, int count, const int* n, const int* nrhs,
                        double* const* A, const int* lda, double* const* B, const int* ldb, void* ws,
                        size_t ws_bytes, int* info_host) {
  for (int i = 0; i < count; ++i)
    if (bad_item(n[i], nrhs[i], lda[i], B ? ldb[i] : 1, B != nullptr)) return EGPU_ERR_UNSUPPORTED;
  std::vector<BatchItem> items(count);
  for (int i = 0; i < count; ++i) {
    items[i].A = A[i];
    items[i].B = B ? B[i] : nullptr;
    items[i].F = A[i];
    items[i].n = n[i];
    items[i].nrhs = B ? nrhs[i] : 0;
    items[i].lda = lda[i];
    items[i].ldb = B ? ldb[i] : 1;
    items[i].ldf = lda[i];
    items[i].id = i;
  }
  sort_items(items);
  const Variant& v = kVariants[0][0];
  int per_sm = 1;
  BTRY(variant_prepare(v, kind, &per_sm));
  const int grid = std::max(1, std::min(sm_count, count));
  unsigned char* base = static_cast<unsigned char*>(ws);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    off = (off + 255) & ~size_t(255);
    void* p = base + off;
    off += bytes;
    return p;
  };
  BatchItem* d_items = static_cast<BatchItem*>(take(sizeof(BatchItem) * std::max(count, 1)));
  int* d_counter = static_cast<int*>(take(sizeof(int)));
  int* d_info = static_cast<int*>(take(sizeof(int) * std::max(count, 1)));
  double* d_scr = static_cast<double*>(take(sizeof(double) * (size_t)sm_count * kScrDoubles));
  if (off > ws_bytes) return EGPU_ERR_ALLOC;
  if (count == 0) return EGPU_OK;
  EGPU_CUDA_TRY(cudaMemcpyAsync(d_items, items.data(), sizeof(BatchItem) * count, cudaMemcpyHostToDevice, st));
  EGPU_CUDA_TRY(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
  {
    double flops = 0.0;
    for (int i = 0; i < count; ++i) flops += (kind == 0 ? 1.0 / 3.0 : 2.0 / 3.0) * (double)n[i] * n[i] * n[i];
    TraceMark tm(st, kTraceOther, flops, 0.0);
    BatchArgs a{d_items, count, d_counter, d_info, nullptr, d_scr};
    v.kern[kind]<<<grid, v.nt, v.smem, st>>>(a);
    count_launch();
  }
  EGPU_CUDA_TRY(cudaGetLastError());
  EGPU_CUDA_TRY(cudaMemcpyAsync(info_host, d_info, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
  EGPU_CUDA_TRY(cudaStreamSynchronize(st));
  return EGPU_OK;
}

size_t egpu_batched_ws_bytes(int count, int sm_count) {
  return sizeof(BatchItem) * (size_t)std::max(count, 1) + sizeof(int) * (size_t)std::max(count, 1) + 4096 +
         sizeof(double) * (size_t)sm_count * kScrDoubles;
}

// ---------------------------------------------------------------------------
// Batch plans: the size-sorted item list, the queue counters, per-system
// info / refinement counts, the per-CTA scratch and (refined plans) the
// working copies live on the device for the plan's lifetime, so a run is a
// counter reset plus one persistent launch per size class, which a CUDA
// graph can capture and replay.  The launch shape of each size class -- the
// panel width and CTA size (which set how many CTAs share an SM) and the
// persistent grid -- is what egpu_batch_plan_autotune chooses, by timing the
// candidates on the plan's own systems.
struct BatchPlan {
  int kind = 0, precision = 0, count = 0, sm_count = 0, device = 0;
  BatchItem* d_items = nullptr;
  int* d_counter = nullptr;
  int* d_info = nullptr;
  int* d_iters = nullptr;
  double* d_scr = nullptr;
  void* block = nullptr;
  void* farena = nullptr;
  double flops = 0.0;
  std::vector<BatchItem> items;  // sorted, as on the device
  int nclass = 1;
  int cbeg[kMaxClass] = {0, 0, 0}, cend[kMaxClass] = {0, 0, 0};
  int cvar[kMaxClass] = {0, 0, 0}, cgrid[kMaxClass] = {0, 0, 0}, cnmax[kMaxClass] = {kBmaxN, 0, 0};
};

static int plan_default_shape(BatchPlan* p) {
  p->nclass = 1;
  p->cbeg[0] = 0;
  p->cend[0] = p->count;
  p->cvar[0] = 0;
  p->cnmax[0] = kBmaxN;
  int per_sm = 1;
  BTRY(variant_prepare(kVariants[p->precision][0], p->kind, &per_sm));
  p->cgrid[0] = per_sm * p->sm_count;
  return EGPU_OK;
}

int batch_plan_create(int device, int sm_count, int kind, int precision, int count, const int* n, const int* nrhs,
                      double* const* A, const int* lda, double* const* B, const int* ldb, BatchPlan** out) {
  *out = nullptr;
  if (precision != 0 && precision != 1) return EGPU_ERR_ARG;
  for (int i = 0; i < count; ++i)
    if (bad_item(n[i], nrhs[i], lda[i], B ? ldb[i] : 1, B != nullptr)) return EGPU_ERR_UNSUPPORTED;
  BatchPlan* p = new (std::nothrow) BatchPlan;
  if (!p) return EGPU_ERR_ALLOC;
  p->kind = kind; p->precision = precision; p->count = count; p->sm_count = sm_count; p->device = device;
  p->items.resize(count);
  size_t fbytes = 0;
  std::vector<size_t> foff(count);
  for (int i = 0; i < count; ++i) {
    BatchItem& it = p->items[i];
    it.A = A[i];
    it.B = B ? B[i] : nullptr;
    it.n = n[i];
    it.nrhs = B ? nrhs[i] : 0;
    it.lda = lda[i];
    it.ldb = B ? ldb[i] : 1;
    it.id = i;
    it.ldf = precision ? std::max(2, (n[i] + 1) & ~1) : lda[i];
    foff[i] = fbytes;
    fbytes += precision ? (((size_t)it.ldf * std::max(1, n[i]) * sizeof(double)) + 255) & ~size_t(255) : 0;
    p->flops += (kind == 0 ? 1.0 / 3.0 : 2.0 / 3.0) * (double)n[i] * n[i] * n[i];
  }
  const size_t b_items = ((sizeof(BatchItem) * (size_t)std::max(count, 1)) + 255) & ~size_t(255);
  const size_t b_ints = ((sizeof(int) * (size_t)std::max(count, 1)) + 255) & ~size_t(255);
  const size_t b_scr = sizeof(double) * (size_t)kMaxPerSM * sm_count * kScrDoubles;
  cudaError_t e = cudaMalloc(&p->block, b_items + 256 + 2 * b_ints + b_scr);
  if (e == cudaSuccess && fbytes) e = cudaMalloc(&p->farena, fbytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (p->block) cudaFree(p->block);
    delete p;
    return EGPU_ERR_ALLOC;
  }
  unsigned char* base = static_cast<unsigned char*>(p->block);
  p->d_items = reinterpret_cast<BatchItem*>(base);
  p->d_counter = reinterpret_cast<int*>(base + b_items);
  p->d_info = reinterpret_cast<int*>(base + b_items + 256);
  p->d_iters = reinterpret_cast<int*>(base + b_items + 256 + b_ints);
  p->d_scr = reinterpret_cast<double*>(base + b_items + 256 + 2 * b_ints);
  for (int i = 0; i < count; ++i)
    p->items[i].F = precision ? static_cast<void*>(static_cast<unsigned char*>(p->farena) + foff[i])
                              : static_cast<void*>(p->items[i].A);
  sort_items(p->items);
  if (count > 0) e = cudaMemcpy(p->d_items, p->items.data(), sizeof(BatchItem) * count, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(p->d_iters, 0, b_ints);
  int rc = e == cudaSuccess ? plan_default_shape(p) : EGPU_ERR_CUDA;
  if (rc != EGPU_OK) {
    if (e != cudaSuccess) set_last_error(e, "batch plan upload", __FILE__, __LINE__);
    batch_plan_destroy(p);
    return rc;
  }
  *out = p;
  return EGPU_OK;
}

// One persistent launch over systems [beg, end) of the sorted list.
static int plan_launch(BatchPlan* p, cudaStream_t st, int cls, int beg, int end, int var, int grid) {
  if (end <= beg) return EGPU_OK;
  const Variant& v = kVariants[p->precision][var];
  int per_sm = 1;
  BTRY(variant_prepare(v, p->kind, &per_sm));
  grid = std::max(1, std::min(grid, per_sm * p->sm_count));
  double flops = 0.0;
  for (int i = beg; i < end; ++i) {
    const double nn = p->items[i].n;
    flops += (p->kind == 0 ? 1.0 / 3.0 : 2.0 / 3.0) * nn * nn * nn;
  }
  TraceMark tm(st, kTraceOther, flops, 0.0);
  BatchArgs a{p->d_items + beg, end - beg, p->d_counter + cls, p->d_info, p->d_iters, p->d_scr};
  v.kern[p->kind]<<<grid, v.nt, v.smem, st>>>(a);
  count_launch();
  EGPU_CUDA_TRY(cudaGetLastError());
  return EGPU_OK;
}

// Enqueue one run of the plan on `st` (no host synchronisation).
int batch_plan_run(BatchPlan* p, cudaStream_t st) {
  if (p->count == 0) return EGPU_OK;
  EGPU_CUDA_TRY(cudaMemsetAsync(p->d_counter, 0, sizeof(int) * kMaxClass, st));
  for (int c = 0; c < p->nclass; ++c) BTRY(plan_launch(p, st, c, p->cbeg[c], p->cend[c], p->cvar[c], p->cgrid[c]));
  return EGPU_OK;
}

int batch_plan_info(BatchPlan* p, cudaStream_t st, int* info_host) {
  if (p->count == 0) return EGPU_OK;
  EGPU_CUDA_TRY(cudaMemcpyAsync(info_host, p->d_info, sizeof(int) * p->count, cudaMemcpyDeviceToHost, st));
  EGPU_CUDA_TRY(cudaStreamSynchronize(st));
  return EGPU_OK;
}

int batch_plan_iters(BatchPlan* p, cudaStream_t st, int* iters_host) {
  if (p->count == 0) return EGPU_OK;
  EGPU_CUDA_TRY(cudaMemcpyAsync(iters_host, p->d_iters, sizeof(int) * p->count, cudaMemcpyDeviceToHost, st));
  EGPU_CUDA_TRY(cudaStreamSynchronize(st));
  return EGPU_OK;
}

int batch_plan_shape(BatchPlan* p, int* nclass, int* class_nmax, int* panel, int* threads, int* grid) {
  if (nclass) *nclass = p->nclass;
  for (int c = 0; c < p->nclass; ++c) {
    const Variant& v = kVariants[p->precision][p->cvar[c]];
    if (class_nmax) class_nmax[c] = p->cnmax[c];
    if (panel) panel[c] = v.nb;
    if (threads) threads[c] = v.nt;
    if (grid) grid[c] = p->cgrid[c];
  }
  return EGPU_OK;
}

// Autotuning: the candidate shapes of each size class are timed on the
// plan's own systems (inputs restored from a backup before every run, and
// once more at the end), then the per-class choice is compared with the best
// single launch over all systems and the faster kept.
int batch_plan_autotune(BatchPlan* p, cudaStream_t st, int reps, double* best_ms, int* best_grid) {
  if (p->count == 0) {
    if (best_ms) *best_ms = 0.0;
    if (best_grid) *best_grid = p->cgrid[0];
    return EGPU_OK;
  }
  reps = std::max(1, reps);
  std::vector<long long> off(p->count);
  long long tot = 0;
  for (int i = 0; i < p->count; ++i) {
    off[i] = tot;
    tot += (long long)p->items[i].n * p->items[i].n + (long long)p->items[i].n * p->items[i].nrhs;
  }
  double* bk = nullptr;
  long long* d_off = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = EGPU_OK;
  auto fail_cuda = [&](cudaError_t e, const char* what) {
    set_last_error(e, what, __FILE__, __LINE__);
    return EGPU_ERR_CUDA;
  };
  cudaError_t e = cudaMalloc(&bk, sizeof(double) * std::max(1LL, tot));
  if (e == cudaSuccess) e = cudaMalloc(&d_off, sizeof(long long) * p->count);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (bk) cudaFree(bk);
    return EGPU_ERR_ALLOC;
  }
  e = cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * p->count, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const int cgrid_bk = std::min(p->count, 4 * p->sm_count);
  if (e == cudaSuccess) {
    batch_backup_kernel<<<cgrid_bk, 256, 0, st>>>(p->d_items, p->count, bk, d_off, 0);
    count_launch();
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) rc = fail_cuda(e, "batch plan autotune");
  // time one shape on systems [beg, end): restore, launch, reps times
  auto time_shape = [&](int beg, int end, int var, int grid, double* ms_out) -> int {
    double sum = 0.0;
    for (int r = 0; r <= reps; ++r) {
      batch_backup_kernel<<<cgrid_bk, 256, 0, st>>>(p->d_items, p->count, bk, d_off, 1);
      count_launch();
      cudaError_t ee = cudaMemsetAsync(p->d_counter, 0, sizeof(int) * kMaxClass, st);
      if (ee == cudaSuccess) ee = cudaEventRecord(e0, st);
      if (ee != cudaSuccess) return fail_cuda(ee, "batch plan autotune");
      BTRY(plan_launch(p, st, 0, beg, end, var, grid));
      ee = cudaEventRecord(e1, st);
      if (ee == cudaSuccess) ee = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (ee == cudaSuccess) ee = cudaEventElapsedTime(&ms, e0, e1);
      if (ee != cudaSuccess) return fail_cuda(ee, "batch plan autotune");
      if (r > 0) sum += ms;  // the first run is the warm-up
    }
    *ms_out = sum / reps;
    return EGPU_OK;
  };
  int nb[kMaxClass], ne[kMaxClass], nmax[kMaxClass], ncls = 0;
  for (int c = 0; c < kMaxClass && rc == EGPU_OK; ++c) {
    const int hi = kClassMax[c], lo = (c + 1 < kMaxClass) ? kClassMax[c + 1] : 0;
    int b = 0;
    while (b < p->count && p->items[b].n > hi) ++b;
    int en = b;
    while (en < p->count && p->items[en].n > lo) ++en;
    if (en > b) {
      nb[ncls] = b;
      ne[ncls] = en;
      nmax[ncls] = hi;
      ++ncls;
    }
  }
  int bvar[kMaxClass] = {0, 0, 0}, bgrid[kMaxClass] = {0, 0, 0};
  double split_ms = 0.0, single_ms = 1e300;
  int single_var = 0, single_grid = p->sm_count;
  for (int v = 0; v < kNumVariants && rc == EGPU_OK; ++v) {
    int per_sm = 1;
    rc = variant_prepare(kVariants[p->precision][v], p->kind, &per_sm);
    const int full = per_sm * p->sm_count;
    for (int g : {full, full / 2}) {
      if (rc != EGPU_OK || g < 1) continue;
      double ms = 0.0;
      rc = time_shape(0, p->count, v, g, &ms);
      if (rc == EGPU_OK && ms < single_ms) {
        single_ms = ms;
        single_var = v;
        single_grid = g;
      }
    }
  }
  if (ncls > 1) {
    for (int c = 0; c < ncls && rc == EGPU_OK; ++c) {
      double best = 1e300;
      for (int v = 0; v < kNumVariants && rc == EGPU_OK; ++v) {
        int per_sm = 1;
        rc = variant_prepare(kVariants[p->precision][v], p->kind, &per_sm);
        const int full = per_sm * p->sm_count;
        for (int g : {full, full / 2}) {
          if (rc != EGPU_OK || g < 1) continue;
          double ms = 0.0;
          rc = time_shape(nb[c], ne[c], v, g, &ms);
          if (rc == EGPU_OK && ms < best) {
            best = ms;
            bvar[c] = v;
            bgrid[c] = g;
          }
        }
      }
      split_ms += best;
    }
  }
  if (rc == EGPU_OK) {
    if (ncls > 1 && split_ms < single_ms) {
      p->nclass = ncls;
      for (int c = 0; c < ncls; ++c) {
        p->cbeg[c] = nb[c];
        p->cend[c] = ne[c];
        p->cvar[c] = bvar[c];
        p->cgrid[c] = bgrid[c];
        p->cnmax[c] = nmax[c];
      }
    } else {
      p->nclass = 1;
      p->cbeg[0] = 0;
      p->cend[0] = p->count;
      p->cvar[0] = single_var;
      p->cgrid[0] = single_grid;
      p->cnmax[0] = kBmaxN;
    }
    if (best_ms) *best_ms = (ncls > 1 && split_ms < single_ms) ? split_ms : single_ms;
    if (best_grid) *best_grid = p->cgrid[0];
  }
  if (bk) {
    if (rc == EGPU_OK) {
      batch_backup_kernel<<<cgrid_bk, 256, 0, st>>>(p->d_items, p->count, bk, d_off, 1);
      count_launch();
    }
    cudaStreamSynchronize(st);
    cudaFree(bk);
  }
  if (d_off) cudaFree(d_off);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return rc;
}

void batch_plan_set_grid(BatchPlan* p, int grid) {
  for (int c = 0; c < p->nclass; ++c) p->cgrid[c] = std::max(1, std::min(grid, kMaxPerSM * p->sm_count));
}

void batch_plan_destroy(BatchPlan* p) {
  if (!p) return;
  if (p->block) cudaFree(p->block);
  if (p->farena) cudaFree(p->farena);
  delete p;
}

}  // namespace egpu
