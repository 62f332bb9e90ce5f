// Batched factor-and-solve of many independent systems of uneven sizes in one
// persistent launch: HPDSolve (Cholesky + cholesky::SolveAfter) and
// GaussianElimination-style LU + solve, per system, n <= 512.
//
// One CTA owns one system at a time and pulls the next from a size-sorted
// queue (largest first) with an atomic counter, so the uneven sizes balance
// across the SMs.  Per system the CTA runs the blocked right-looking
// algorithm of the single-system path with a 32-wide panel held in shared
// memory: diagonal block factored with one barrier per column, its inverse,
// the panel solve as a multiply by that inverse, and the trailing update on
// the FP64 tensor cores (DMMA m16n8k8, 32x32 warp tiles) reading and
// writing the system's trailing matrix in global memory (L2-resident for the
// systems in flight).  The right-hand sides are solved with the same
// diagonal-block inverses, kept per CTA in a global scratch area.
#include <algorithm>
#include <new>
#include <vector>

#include "internal.h"

namespace egpu {

struct BatchItem {
  double* A;
  double* B;
  int n, nrhs, lda, ldb;
  int id, pad;
};

constexpr int kBT = 256;      // threads per CTA
constexpr int kBnb = 32;      // panel width
constexpr int kBmaxN = 512;   // largest order handled by one CTA
constexpr int kBmaxRHS = 16;  // right-hand sides per system
constexpr int kPLD = kBmaxN + 32;  // panel leading dimension (edge tiles read past row m harmlessly)
constexpr int kXLD = 33;
constexpr int kBSmemDoubles = kBnb * kPLD + kBnb * kXLD + kBmaxN * kBmaxRHS + 64;

// C (32x32 warp tile of the trailing matrix, global) -= P[rows] * P[cols]^T
// with P the 32-wide panel in shared memory ([k][r], ld kPLD).  Rows/cols are
// panel-relative; `tri` keeps only r >= c; `sign` = -1 for Cholesky/LU updates.
__device__ __forceinline__ void warp_tile_update(double* C, long long ldc, bool cvec, const double* P, int prow,
                                                 int pcol, int mrows, int ncols, int pbase_r, int pbase_c,
                                                 bool tri) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  double acc[2][4][4];
  // load C in the accumulator layout (rows 2g + i (+16), cols per n8 pair)
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int row = prow + 2 * g + ((r >= 2) ? 16 : 0);
      const int c = 2 * t + (r & 1);
      const int col = pcol + (j >> 1) * 16 + 2 * c + (j & 1);
      const bool v0 = row < mrows && col < ncols && (!tri || row >= col);
      const bool v1 = row + 1 < mrows && col < ncols && (!tri || row + 1 >= col);
      const double* cp = C + (long long)col * ldc + row;
      if (cvec && v0 && v1) {
        const double2 cc = *reinterpret_cast<const double2*>(cp);
        acc[0][j][r] = cc.x;
        acc[1][j][r] = cc.y;
      } else {
        if (v0) acc[0][j][r] = cp[0];
        if (v1) acc[1][j][r] = cp[1];
      }
    }
  // acc := C - P_rows * P_cols^T : negate, accumulate +, negate back
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = -acc[i][j][r];
#pragma unroll
  for (int ks = 0; ks < kBnb / 8; ++ks) {
    const int ke = ks * 8 + 2 * t;
    double af[2][4], bf[4][2];
    {
      const int m0 = pbase_r + prow + 2 * g;
      const double2 v00 = *reinterpret_cast<const double2*>(P + ke * kPLD + m0);
      const double2 v01 = *reinterpret_cast<const double2*>(P + (ke + 1) * kPLD + m0);
      const double2 v10 = *reinterpret_cast<const double2*>(P + ke * kPLD + m0 + 16);
      const double2 v11 = *reinterpret_cast<const double2*>(P + (ke + 1) * kPLD + m0 + 16);
      af[0][0] = v00.x; af[0][1] = v10.x; af[0][2] = v01.x; af[0][3] = v11.x;
      af[1][0] = v00.y; af[1][1] = v10.y; af[1][2] = v01.y; af[1][3] = v11.y;
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int n0 = pbase_c + pcol + q * 16 + 2 * g;
      const double2 v0 = *reinterpret_cast<const double2*>(P + ke * kPLD + n0);
      const double2 v1 = *reinterpret_cast<const double2*>(P + (ke + 1) * kPLD + n0);
      bf[2 * q][0] = v0.x; bf[2 * q][1] = v1.x;
      bf[2 * q + 1][0] = v0.y; bf[2 * q + 1][1] = v1.y;
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
      const int c = 2 * t + (r & 1);
      const int col = pcol + (j >> 1) * 16 + 2 * c + (j & 1);
      const bool v0 = row < mrows && col < ncols && (!tri || row >= col);
      const bool v1 = row + 1 < mrows && col < ncols && (!tri || row + 1 >= col);
      double* cp = C + (long long)col * ldc + row;
      if (cvec && v0 && v1) {
        *reinterpret_cast<double2*>(cp) = make_double2(-acc[0][j][r], -acc[1][j][r]);
      } else {
        if (v0) cp[0] = -acc[0][j][r];
        if (v1) cp[1] = -acc[1][j][r];
      }
    }
}

// Lower Cholesky of the b x b top of the panel (b <= 32), one barrier per
// column (the LVar3Unb operations, Cholesky/LVar3.hpp:19-49), then the
// inverse of the factor into X (ld kXLD) by warp 0.  Returns 0 or 1-based
// column of a non-positive pivot (uniform over the CTA).
__device__ int batch_diag_chol(double* P, int b, double* X, double* s_alpha) {
  const int tid = threadIdx.x;
  const int row = tid & 31, grp = tid >> 5;  // 8 column groups
  for (int j = 0; j < b; ++j) {
    const double ajj = P[j * kPLD + j];
    if (ajj <= 0.0) return j + 1;
    if (tid == 0) s_alpha[j] = sqrt(ajj);
    if (j > 0 && grp == 0 && row >= j && row < b) P[(j - 1) * kPLD + row] /= s_alpha[j - 1];
    if (row > j && row < b) {
      const double lij = P[j * kPLD + row] / ajj;
      for (int k = j + 1 + grp; k <= row && k < b; k += 8) P[k * kPLD + row] -= lij * P[j * kPLD + k];
    }
    __syncthreads();
  }
  if (grp == 1 && row < b) P[row * kPLD + row] = s_alpha[row];
  __syncthreads();
  // X = inv(L11): lane c of warp 0 computes column c by forward substitution
  if (tid < 32) {
    const int c = tid;
    if (c < b) {
      for (int i = c; i < b; ++i) {
        double acc = (i == c) ? 1.0 : 0.0;
        for (int m = c; m < i; ++m) acc = fma(-P[m * kPLD + i], X[m + c * kXLD], acc);
        X[i + c * kXLD] = acc / P[i * kPLD + i];
      }
    }
  }
  __syncthreads();
  return 0;
}

__global__ void __launch_bounds__(kBT, 1) chol_batched_kernel(const BatchItem* items, int count, int* counter,
                                                               int* info, double* inv_scratch) {
  extern __shared__ double sm[];
  double* P = sm;                      // [kBnb][kPLD]
  double* X = P + kBnb * kPLD;         // [kBnb][kXLD]
  double* BS = X + kBnb * kXLD;        // right-hand sides [rhs][kBmaxN]
  __shared__ double s_alpha[kBnb];
  __shared__ int s_idx;
  const int tid = threadIdx.x, warp = tid >> 5;
  double* Xg = inv_scratch + (size_t)blockIdx.x * (kBmaxN / kBnb) * kBnb * kBnb;  // per-CTA diag inverses
  while (true) {
    if (tid == 0) s_idx = atomicAdd(counter, 1);
    __syncthreads();
    const int idx = s_idx;
    __syncthreads();
    if (idx >= count) break;
    const BatchItem it = items[idx];
    const int n = it.n;
    double* A = it.A;
    const long long lda = it.lda;
    const bool cvec = (reinterpret_cast<uintptr_t>(A) % 16 == 0) && (lda % 2 == 0);
    int fail = 0;
    for (int k0 = 0; k0 < n && !fail; k0 += kBnb) {
      const int b = min(kBnb, n - k0), m = n - k0;
      for (int c = 0; c < b; ++c)
        for (int r = tid; r < m; r += kBT) cp_async8(&P[c * kPLD + r], &A[(long long)(k0 + c) * lda + k0 + r]);
      cp_async_wait_all();
      __syncthreads();
      fail = batch_diag_chol(P, b, X, s_alpha);
      if (fail) {
        fail += k0;
        break;
      }
      // keep inv(L11) for the solve
      for (int e = tid; e < kBnb * kBnb; e += kBT) {
        const int i = e % kBnb, c = e / kBnb;
        Xg[(k0 / kBnb) * kBnb * kBnb + e] = (i < b && c < b && i >= c) ? X[i + c * kXLD] : 0.0;
      }
      // L21 := A21 * inv(L11)^T, one row per thread
      for (int r = b + tid; r < m; r += kBT) {
        double a[kBnb];
#pragma unroll
        for (int k = 0; k < kBnb; ++k) a[k] = (k < b) ? P[k * kPLD + r] : 0.0;
#pragma unroll
        for (int c = 0; c < kBnb; ++c) {
          if (c < b) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k <= c; ++k) s = fma(a[k], X[c + k * kXLD], s);
            P[c * kPLD + r] = s;
          }
        }
      }
      __syncthreads();
      // write the panel back (lower part of the diagonal block + L21)
      for (int c = 0; c < b; ++c)
        for (int r = c + tid; r < m; r += kBT) A[(long long)(k0 + c) * lda + k0 + r] = P[c * kPLD + r];
      // trailing update A22 -= L21 L21^T on the lower triangle, 32x32 DMMA warp tiles
      const int m2 = m - b;
      if (m2 > 0) {
        const int nt = (m2 + 31) / 32;
        const int T = nt * (nt + 1) / 2;
        double* C = A + (long long)(k0 + b) * lda + (k0 + b);
        for (int tt = warp; tt < T; tt += kBT / 32) {
          int ti = 0;  // triangular index -> (ti, tj), ti >= tj
          while ((ti + 1) * (ti + 2) / 2 <= tt) ++ti;
          const int tj = tt - ti * (ti + 1) / 2;
          warp_tile_update(C, lda, cvec, P, ti * 32, tj * 32, m2, m2, b, b, true);
        }
      }
      __syncthreads();
    }
    if (tid == 0) info[it.id] = fail;
    if (fail || it.nrhs <= 0) continue;
    // ---- solve: L L^T X = B (cholesky::SolveAfter, Cholesky/SolveAfter.hpp:20-75)
    const int nrhs = it.nrhs;
    double* Bg = it.B;
    const long long ldb = it.ldb;
    for (int q = 0; q < nrhs; ++q)
      for (int r = tid; r < n; r += kBT) BS[q * kBmaxN + r] = Bg[(long long)q * ldb + r];
    __syncthreads();
    const int nblk = (n + kBnb - 1) / kBnb;
    // forward: Y_i = inv(L_ii) (B_i - sum_{j<i} L_ij Y_j), right-looking
    for (int ib = 0; ib < nblk; ++ib) {
      const int i0 = ib * kBnb, bi = min(kBnb, n - i0);
      const double* Xi = Xg + (size_t)ib * kBnb * kBnb;
      for (int e = tid; e < bi * nrhs; e += kBT) {  // bi * nrhs can exceed the CTA (32 x 16)
        const int i = e % bi, q = e / bi;
        double s = 0.0;
        for (int k = 0; k <= i; ++k) s = fma(Xi[i + k * kBnb], BS[q * kBmaxN + i0 + k], s);
        X[i + q * kXLD] = s;  // staging
      }
      __syncthreads();
      for (int e = tid; e < bi * nrhs; e += kBT) {  // bi * nrhs can exceed the CTA (32 x 16)
        const int i = e % bi, q = e / bi;
        BS[q * kBmaxN + i0 + i] = X[i + q * kXLD];
      }
      __syncthreads();
      for (int r = i0 + bi + tid; r < n; r += kBT) {
        double acc[kBmaxRHS];
#pragma unroll
        for (int q = 0; q < kBmaxRHS; ++q) acc[q] = 0.0;
        for (int k = 0; k < bi; ++k) {
          const double l = A[(long long)(i0 + k) * lda + r];
#pragma unroll
          for (int q = 0; q < kBmaxRHS; ++q)
            if (q < nrhs) acc[q] = fma(l, BS[q * kBmaxN + i0 + k], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < kBmaxRHS; ++q)
          if (q < nrhs) BS[q * kBmaxN + r] -= acc[q];
      }
      __syncthreads();
    }
    // backward: X_i = inv(L_ii)^T (Y_i - sum_{j>i} L_ji^T X_j), right-looking
    for (int ib = nblk - 1; ib >= 0; --ib) {
      const int i0 = ib * kBnb, bi = min(kBnb, n - i0);
      const double* Xi = Xg + (size_t)ib * kBnb * kBnb;
      for (int e = tid; e < bi * nrhs; e += kBT) {  // bi * nrhs can exceed the CTA (32 x 16)
        const int i = e % bi, q = e / bi;
        double s = 0.0;
        for (int k = i; k < bi; ++k) s = fma(Xi[k + i * kBnb], BS[q * kBmaxN + i0 + k], s);
        X[i + q * kXLD] = s;
      }
      __syncthreads();
      for (int e = tid; e < bi * nrhs; e += kBT) {  // bi * nrhs can exceed the CTA (32 x 16)
        const int i = e % bi, q = e / bi;
        BS[q * kBmaxN + i0 + i] = X[i + q * kXLD];
      }
      __syncthreads();
      // rows j < i0: Y_j -= sum_c L[i0 + c][j] X_{i0+c}
      for (int jr = tid; jr < i0; jr += kBT) {
        double acc[kBmaxRHS];
#pragma unroll
        for (int q = 0; q < kBmaxRHS; ++q) acc[q] = 0.0;
        const double* lcol = A + (long long)jr * lda + i0;  // L[i0.., jr], contiguous
        for (int c = 0; c < bi; ++c) {
          const double l = lcol[c];
#pragma unroll
          for (int q = 0; q < kBmaxRHS; ++q)
            if (q < nrhs) acc[q] = fma(l, BS[q * kBmaxN + i0 + c], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < kBmaxRHS; ++q)
          if (q < nrhs) BS[q * kBmaxN + jr] -= acc[q];
      }
      __syncthreads();
    }
    for (int q = 0; q < nrhs; ++q)
      for (int r = tid; r < n; r += kBT) Bg[(long long)q * ldb + r] = BS[q * kBmaxN + r];
    __syncthreads();
  }
}

// C (32x32 warp tile, global) -= P[rows] * U[:, cols] where P is the 32-wide
// panel in shared memory ([k][r]) and U is the 32 x N row block of the
// system in global memory (column-major: k pairs of one column are adjacent,
// loaded straight into the K-major B fragments).
__device__ __forceinline__ void warp_tile_update_gemm(double* C, long long ldc, bool cvec, const double* P,
                                                      const double* U, long long ldu, int prow, int pcol,
                                                      int mrows, int ncols, int pbase_r) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  double acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;
  // K-major B: logical column c of n8 tile j -> pcol + 8 j + c (no interleave)
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int row = prow + 2 * g + ((r >= 2) ? 16 : 0);
      const int col = pcol + 8 * j + 2 * t + (r & 1);
      const bool v0 = row < mrows && col < ncols;
      const bool v1 = row + 1 < mrows && col < ncols;
      const double* cp = C + (long long)col * ldc + row;
      if (cvec && v0 && v1) {
        const double2 cc = *reinterpret_cast<const double2*>(cp);
        acc[0][j][r] = -cc.x;
        acc[1][j][r] = -cc.y;
      } else {
        if (v0) acc[0][j][r] = -cp[0];
        if (v1) acc[1][j][r] = -cp[1];
      }
    }
#pragma unroll
  for (int ks = 0; ks < kBnb / 8; ++ks) {
    const int ke = ks * 8 + 2 * t;
    double af[2][4], bf[4][2];
    {
      const int m0 = pbase_r + prow + 2 * g;
      const double2 v00 = *reinterpret_cast<const double2*>(P + ke * kPLD + m0);
      const double2 v01 = *reinterpret_cast<const double2*>(P + (ke + 1) * kPLD + m0);
      const double2 v10 = *reinterpret_cast<const double2*>(P + ke * kPLD + m0 + 16);
      const double2 v11 = *reinterpret_cast<const double2*>(P + (ke + 1) * kPLD + m0 + 16);
      af[0][0] = v00.x; af[0][1] = v10.x; af[0][2] = v01.x; af[0][3] = v11.x;
      af[1][0] = v00.y; af[1][1] = v10.y; af[1][2] = v01.y; af[1][3] = v11.y;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int col = pcol + 8 * j + g;
      if (col < ncols) {
        const double* up = U + (long long)col * ldu + ke;
        bf[j][0] = up[0];
        bf[j][1] = up[1];
      } else {
        bf[j][0] = 0.0;
        bf[j][1] = 0.0;
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
      double* cp = C + (long long)col * ldc + row;
      if (cvec && v0 && v1) {
        *reinterpret_cast<double2*>(cp) = make_double2(-acc[0][j][r], -acc[1][j][r]);
      } else {
        if (v0) cp[0] = -acc[0][j][r];
        if (v1) cp[1] = -acc[1][j][r];
      }
    }
}

// GaussianElimination(A, B) per system (GaussianElimination.hpp:216-232 with
// the RowEchelon of :94-209): LU with partial pivoting over 32-wide panels,
// the panel's interchanges applied to the columns right of it and to B,
// B eliminated along, then B := inv(U) B.  info[id] = 0 or the 1-based column
// of an exact zero pivot (SingularMatrixException).
__global__ void __launch_bounds__(kBT, 1) lu_batched_kernel(const BatchItem* items, int count, int* counter,
                                                             int* info, double* inv_scratch) {
  extern __shared__ double sm[];
  double* P = sm;               // [kBnb][kPLD]
  double* X = P + kBnb * kPLD;  // [kBnb][kXLD]
  double* BS = X + kBnb * kXLD;
  __shared__ double red_abs[kBT / 32];
  __shared__ int red_row[kBT / 32];
  __shared__ int s_piv[kBnb];
  __shared__ int s_idx, s_fail;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* Xg = inv_scratch + (size_t)blockIdx.x * (kBmaxN / kBnb) * kBnb * kBnb;
  while (true) {
    if (tid == 0) s_idx = atomicAdd(counter, 1);
    __syncthreads();
    const int idx = s_idx;
    __syncthreads();
    if (idx >= count) break;
    const BatchItem it = items[idx];
    const int n = it.n, nrhs = it.nrhs;
    double* A = it.A;
    double* Bg = it.B;
    const long long lda = it.lda, ldb = it.ldb;
    const bool cvec = (reinterpret_cast<uintptr_t>(A) % 16 == 0) && (lda % 2 == 0);
    int fail = 0;
    for (int k0 = 0; k0 < n && !fail; k0 += kBnb) {
      const int b = min(kBnb, n - k0), m = n - k0;
      for (int c = 0; c < b; ++c)
        for (int r = tid; r < m; r += kBT) cp_async8(&P[c * kPLD + r], &A[(long long)(k0 + c) * lda + k0 + r]);
      cp_async_wait_all();
      if (tid == 0) s_fail = 0;
      __syncthreads();
      // ---- panel: lu::Panel (LU/Panel.hpp:19-89) on the m x b panel in shared memory
      for (int j = 0; j < b; ++j) {
        double best = -1.0;
        int brow = 0x7fffffff;
        for (int r = j + tid; r < m; r += kBT) {
          const double av = fabs(P[j * kPLD + r]);
          if (av > best || (av == best && r < brow)) { best = av; brow = r; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double ob = __shfl_down_sync(0xffffffffu, best, o);
          const int orow = __shfl_down_sync(0xffffffffu, brow, o);
          if (ob > best || (ob == best && orow < brow)) { best = ob; brow = orow; }
        }
        if (lane == 0) { red_abs[warp] = best; red_row[warp] = brow; }
        __syncthreads();
        if (tid == 0) {
          for (int w = 1; w < kBT / 32; ++w)
            if (red_abs[w] > best || (red_abs[w] == best && red_row[w] < brow)) { best = red_abs[w]; brow = red_row[w]; }
          s_piv[j] = brow;
          if (P[j * kPLD + brow] == 0.0) s_fail = k0 + j + 1;
        }
        __syncthreads();
        if (s_fail) break;
        const int pr = s_piv[j];
        if (pr != j && tid < b) {  // swap panel rows j and pr
          const double t0 = P[tid * kPLD + j];
          P[tid * kPLD + j] = P[tid * kPLD + pr];
          P[tid * kPLD + pr] = t0;
        }
        __syncthreads();
        const double inv = 1.0 / P[j * kPLD + j];
        for (int r = j + 1 + tid; r < m; r += kBT) {
          const double l = P[j * kPLD + r] * inv;
          P[j * kPLD + r] = l;
          for (int c = j + 1; c < b; ++c) P[c * kPLD + r] -= l * P[c * kPLD + j];
        }
        __syncthreads();
      }
      if (s_fail) {
        fail = s_fail;
        break;
      }
      for (int c = 0; c < b; ++c)
        for (int r = tid; r < m; r += kBT) A[(long long)(k0 + c) * lda + k0 + r] = P[c * kPLD + r];
      // ---- interchanges on the columns right of the panel and on B
      const int ncr = n - k0 - b;
      for (int c = tid; c < ncr + nrhs; c += kBT) {
        double* col = (c < ncr) ? A + (long long)(k0 + b + c) * lda + k0 : Bg + (long long)(c - ncr) * ldb + k0;
        for (int j = 0; j < b; ++j) {
          const int pr = s_piv[j];
          if (pr != j) {
            const double t0 = col[j];
            col[j] = col[pr];
            col[pr] = t0;
          }
        }
      }
      // inv(U11) for the final solve (warp 0, lane c computes column c, backward)
      if (tid < 32) {
        const int c = tid;
        if (c < b) {
          for (int i = c; i >= 0; --i) {
            double acc = (i == c) ? 1.0 : 0.0;
            for (int q = i + 1; q <= c; ++q) acc = fma(-P[q * kPLD + i], X[q + c * kXLD], acc);
            X[i + c * kXLD] = acc / P[i * kPLD + i];
          }
        }
      }
      __syncthreads();
      for (int e = tid; e < kBnb * kBnb; e += kBT) {
        const int i = e % kBnb, c = e / kBnb;
        Xg[(k0 / kBnb) * kBnb * kBnb + e] = (i < b && c < b && i <= c) ? X[i + c * kXLD] : 0.0;
      }
      // ---- U12 := inv(unit L11) A12 and B1 := inv(unit L11) B1 (column by column)
      for (int c = tid; c < ncr + nrhs; c += kBT) {
        double* col = (c < ncr) ? A + (long long)(k0 + b + c) * lda + k0 : Bg + (long long)(c - ncr) * ldb + k0;
        double u[kBnb];
#pragma unroll
        for (int i = 0; i < kBnb; ++i) {
          if (i < b) {
            double v = col[i];
#pragma unroll
            for (int q = 0; q < kBnb; ++q)
              if (q < i) v = fma(-P[q * kPLD + i], u[q], v);
            u[i] = v;
            col[i] = v;
          }
        }
      }
      __syncthreads();
      // ---- trailing update A22 -= L21 U12 and B2 -= L21 B1
      const int m2 = m - b;
      if (m2 > 0) {
        if (ncr > 0) {
          const int tr = (m2 + 31) / 32, tc = (ncr + 31) / 32;
          double* C = A + (long long)(k0 + b) * lda + (k0 + b);
          const double* U = A + (long long)(k0 + b) * lda + k0;
          for (int tt = warp; tt < tr * tc; tt += kBT / 32)
            warp_tile_update_gemm(C, lda, cvec, P, U, lda, (tt % tr) * 32, (tt / tr) * 32, m2, ncr, b);
        }
        for (int r = b + tid; r < m; r += kBT) {
          double acc[kBmaxRHS];
#pragma unroll
          for (int q = 0; q < kBmaxRHS; ++q) acc[q] = 0.0;
          for (int k = 0; k < b; ++k) {
            const double l = P[k * kPLD + r];
#pragma unroll
            for (int q = 0; q < kBmaxRHS; ++q)
              if (q < nrhs) acc[q] = fma(l, Bg[(long long)q * ldb + k0 + k], acc[q]);
          }
#pragma unroll
          for (int q = 0; q < kBmaxRHS; ++q)
            if (q < nrhs) Bg[(long long)q * ldb + k0 + r] -= acc[q];
        }
      }
      __syncthreads();
    }
    if (tid == 0) info[it.id] = fail;
    if (fail || nrhs <= 0) {
      __syncthreads();
      continue;
    }
    // ---- B := inv(U) B, backward over 32-blocks with the kept inv(U_ii)
    for (int q = 0; q < nrhs; ++q)
      for (int r = tid; r < n; r += kBT) BS[q * kBmaxN + r] = Bg[(long long)q * ldb + r];
    __syncthreads();
    const int nblk = (n + kBnb - 1) / kBnb;
    for (int ib = nblk - 1; ib >= 0; --ib) {
      const int i0 = ib * kBnb, bi = min(kBnb, n - i0);
      const double* Xi = Xg + (size_t)ib * kBnb * kBnb;
      for (int e = tid; e < bi * nrhs; e += kBT) {  // bi * nrhs can exceed the CTA (32 x 16)
        const int i = e % bi, q = e / bi;
        double s = 0.0;
        for (int k = i; k < bi; ++k) s = fma(Xi[i + k * kBnb], BS[q * kBmaxN + i0 + k], s);
        X[i + q * kXLD] = s;
      }
      __syncthreads();
      for (int e = tid; e < bi * nrhs; e += kBT) {  // bi * nrhs can exceed the CTA (32 x 16)
        const int i = e % bi, q = e / bi;
        BS[q * kBmaxN + i0 + i] = X[i + q * kXLD];
      }
      __syncthreads();
      for (int r = tid; r < i0; r += kBT) {  // rows above: B_r -= U[r, i0..] X_i
        double acc[kBmaxRHS];
#pragma unroll
        for (int q = 0; q < kBmaxRHS; ++q) acc[q] = 0.0;
        for (int k = 0; k < bi; ++k) {
          const double u = A[(long long)(i0 + k) * lda + r];
#pragma unroll
          for (int q = 0; q < kBmaxRHS; ++q)
            if (q < nrhs) acc[q] = fma(u, BS[q * kBmaxN + i0 + k], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < kBmaxRHS; ++q)
          if (q < nrhs) BS[q * kBmaxN + r] -= acc[q];
      }
      __syncthreads();
    }
    for (int q = 0; q < nrhs; ++q)
      for (int r = tid; r < n; r += kBT) Bg[(long long)q * ldb + r] = BS[q * kBmaxN + r];
    __syncthreads();
  }
}

// Host side: sort by size, upload the descriptors, launch, read back statuses.
// Buffers come from the handle workspace (see egpu_dposv_batched in api.cu).
int egpu_batched_launch(int kind, cudaStream_t st, int sm_count, int count, const int* n, const int* nrhs,
                        double* const* A, const int* lda, double* const* B, const int* ldb, void* ws,
                        size_t ws_bytes, int* info_host) {
  for (int i = 0; i < count; ++i)
    if (n[i] < 0 || n[i] > kBmaxN || nrhs[i] < 0 || nrhs[i] > kBmaxRHS || lda[i] < std::max(1, n[i]) ||
        (nrhs[i] > 0 && ldb[i] < std::max(1, n[i])))
      return EGPU_ERR_UNSUPPORTED;
  std::vector<BatchItem> items(count);
  for (int i = 0; i < count; ++i) {
    items[i].A = A[i];
    items[i].B = B ? B[i] : nullptr;
    items[i].n = n[i];
    items[i].nrhs = B ? nrhs[i] : 0;
    items[i].lda = lda[i];
    items[i].ldb = B ? ldb[i] : 1;
    items[i].id = i;
  }
  std::stable_sort(items.begin(), items.end(), [](const BatchItem& a, const BatchItem& b) { return a.n > b.n; });
  const int grid = sm_count;
  unsigned char* base = static_cast<unsigned char*>(ws);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    off = (off + 255) & ~size_t(255);
    void* p = base + off;
    off += bytes;
    return p;
  };
  BatchItem* d_items = static_cast<BatchItem*>(take(sizeof(BatchItem) * count));
  int* d_counter = static_cast<int*>(take(sizeof(int)));
  int* d_info = static_cast<int*>(take(sizeof(int) * count));
  double* d_inv = static_cast<double*>(take(sizeof(double) * (size_t)grid * kBmaxN * kBnb));
  if (off > ws_bytes) return EGPU_ERR_ALLOC;
  EGPU_CUDA_TRY(cudaMemcpyAsync(d_items, items.data(), sizeof(BatchItem) * count, cudaMemcpyHostToDevice, st));
  EGPU_CUDA_TRY(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
  const size_t smem = sizeof(double) * kBSmemDoubles;
  auto kern = (kind == 0) ? chol_batched_kernel : lu_batched_kernel;
  EGPU_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  {
    double flops = 0.0;
    for (int i = 0; i < count; ++i) flops += (kind == 0 ? 1.0 / 3.0 : 2.0 / 3.0) * (double)n[i] * n[i] * n[i];
    TraceMark tm(st, kTraceOther, flops, 0.0);
    kern<<<grid, kBT, smem, st>>>(d_items, count, d_counter, d_info, d_inv);
    count_launch();
  }
  EGPU_CUDA_TRY(cudaGetLastError());
  EGPU_CUDA_TRY(cudaMemcpyAsync(info_host, d_info, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
  EGPU_CUDA_TRY(cudaStreamSynchronize(st));
  return EGPU_OK;
}

size_t egpu_batched_ws_bytes(int count, int sm_count) {
  return sizeof(BatchItem) * (size_t)count + sizeof(int) * (size_t)count + 4096 +
         sizeof(double) * (size_t)sm_count * kBmaxN * kBnb;
}

// ---------------------------------------------------------------------------
// Batch plans: the size-sorted item list, the queue counter, per-system info
// and the per-CTA inverse scratch live on the device for the plan's lifetime,
// so a run is two stream operations (counter reset + the persistent kernel),
// which a CUDA graph can capture and replay.  The grid (number of persistent
// CTAs) is the tunable launch shape: egpu_batch_plan_autotune times the
// candidates on the plan's own systems and keeps the fastest.
struct BatchPlan {
  int kind = 0, count = 0, grid = 0, sm_count = 0, device = 0;
  BatchItem* d_items = nullptr;
  int* d_counter = nullptr;
  int* d_info = nullptr;
  double* d_inv = nullptr;
  void* block = nullptr;
  double flops = 0.0;
};

int batch_plan_create(int device, int sm_count, int kind, int count, const int* n, const int* nrhs,
                      double* const* A, const int* lda, double* const* B, const int* ldb, BatchPlan** out) {
  *out = nullptr;
  for (int i = 0; i < count; ++i)
    if (n[i] < 0 || n[i] > kBmaxN || nrhs[i] < 0 || nrhs[i] > kBmaxRHS || lda[i] < std::max(1, n[i]) ||
        (B && nrhs[i] > 0 && ldb[i] < std::max(1, n[i])))
      return EGPU_ERR_UNSUPPORTED;
  std::vector<BatchItem> items(count);
  double flops = 0.0;
  for (int i = 0; i < count; ++i) {
    items[i].A = A[i];
    items[i].B = B ? B[i] : nullptr;
    items[i].n = n[i];
    items[i].nrhs = B ? nrhs[i] : 0;
    items[i].lda = lda[i];
    items[i].ldb = B ? ldb[i] : 1;
    items[i].id = i;
    flops += (kind == 0 ? 1.0 / 3.0 : 2.0 / 3.0) * (double)n[i] * n[i] * n[i];
  }
  std::stable_sort(items.begin(), items.end(), [](const BatchItem& a, const BatchItem& b) { return a.n > b.n; });
  BatchPlan* p = new (std::nothrow) BatchPlan;
  if (!p) return EGPU_ERR_ALLOC;
  p->kind = kind; p->count = count; p->grid = sm_count; p->sm_count = sm_count; p->device = device; p->flops = flops;
  const size_t b_items = ((sizeof(BatchItem) * (size_t)std::max(count, 1)) + 255) & ~size_t(255);
  const size_t b_info = ((sizeof(int) * (size_t)std::max(count, 1)) + 255) & ~size_t(255);
  const size_t b_inv = sizeof(double) * (size_t)sm_count * kBmaxN * kBnb;
  cudaError_t e = cudaMalloc(&p->block, b_items + 256 + b_info + b_inv);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete p;
    return EGPU_ERR_ALLOC;
  }
  unsigned char* base = static_cast<unsigned char*>(p->block);
  p->d_items = reinterpret_cast<BatchItem*>(base);
  p->d_counter = reinterpret_cast<int*>(base + b_items);
  p->d_info = reinterpret_cast<int*>(base + b_items + 256);
  p->d_inv = reinterpret_cast<double*>(base + b_items + 256 + b_info);
  if (count > 0) e = cudaMemcpy(p->d_items, items.data(), sizeof(BatchItem) * count, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    set_last_error(e, "batch plan upload", __FILE__, __LINE__);
    cudaFree(p->block);
    delete p;
    return EGPU_ERR_CUDA;
  }
  *out = p;
  return EGPU_OK;
}

// Enqueue one run of the plan on `st` (no host synchronisation).
int batch_plan_run(BatchPlan* p, cudaStream_t st) {
  if (p->count == 0) return EGPU_OK;
  const size_t smem = sizeof(double) * kBSmemDoubles;
  auto kern = (p->kind == 0) ? chol_batched_kernel : lu_batched_kernel;
  static bool attr[2] = {false, false};
  if (!attr[p->kind]) {
    EGPU_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr[p->kind] = true;
  }
  EGPU_CUDA_TRY(cudaMemsetAsync(p->d_counter, 0, sizeof(int), st));
  {
    TraceMark tm(st, kTraceOther, p->flops, 0.0);
    kern<<<std::max(1, std::min(p->grid, p->sm_count)), kBT, smem, st>>>(p->d_items, p->count, p->d_counter,
                                                                        p->d_info, p->d_inv);
    count_launch();
  }
  EGPU_CUDA_TRY(cudaGetLastError());
  return EGPU_OK;
}

int batch_plan_info(BatchPlan* p, cudaStream_t st, int* info_host) {
  if (p->count == 0) return EGPU_OK;
  EGPU_CUDA_TRY(cudaMemcpyAsync(info_host, p->d_info, sizeof(int) * p->count, cudaMemcpyDeviceToHost, st));
  EGPU_CUDA_TRY(cudaStreamSynchronize(st));
  return EGPU_OK;
}

// Time each candidate grid (`reps` runs each, after one untimed run) and keep
// the fastest.  The runs factor the plan's systems in place.
int batch_plan_autotune(BatchPlan* p, cudaStream_t st, int reps, double* best_ms, int* best_grid) {
  const int cands[] = {p->sm_count, (3 * p->sm_count) / 4, p->sm_count / 2, p->sm_count / 4};
  cudaEvent_t e0, e1;
  EGPU_CUDA_TRY(cudaEventCreate(&e0));
  EGPU_CUDA_TRY(cudaEventCreate(&e1));
  double best = 1e300;
  int bg = p->sm_count;
  for (int g : cands) {
    if (g < 1) continue;
    p->grid = g;
    int rc = batch_plan_run(p, st);
    if (rc != EGPU_OK) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
    cudaEventRecord(e0, st);
    for (int r = 0; r < std::max(1, reps); ++r) {
      rc = batch_plan_run(p, st);
      if (rc != EGPU_OK) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
    }
    cudaEventRecord(e1, st);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) {
      set_last_error(e, "batch plan autotune", __FILE__, __LINE__);
      cudaEventDestroy(e0); cudaEventDestroy(e1);
      return EGPU_ERR_CUDA;
    }
    const double per = ms / std::max(1, reps);
    if (per < best) { best = per; bg = g; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  p->grid = bg;
  if (best_ms) *best_ms = best;
  if (best_grid) *best_grid = bg;
  return EGPU_OK;
}

void batch_plan_set_grid(BatchPlan* p, int grid) { p->grid = std::max(1, std::min(grid, p->sm_count)); }

void batch_plan_destroy(BatchPlan* p) {
  if (!p) return;
  if (p->block) cudaFree(p->block);
  delete p;
}

}  // namespace egpu
