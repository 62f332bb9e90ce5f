// C-ABI entry points: handle, workspace, and the blocked right-looking
// drivers that sequence the sm_100a kernels for Cholesky, LU and the solves.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>
#include <new>
#include <string>

#include "context.h"

namespace egpu {

static thread_local std::string t_last_error;
static std::atomic<long long> g_launches{0};

void set_last_error(cudaError_t e, const char* what, const char* file, int line) {
  t_last_error = std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" + std::to_string(line) + ")";
}

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

thread_local Trace* t_trace = nullptr;


TraceMark::TraceMark(cudaStream_t s, int kind, double flops, double bytes) {
  if (t_trace == nullptr || !t_trace->on) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  Trace::Rec r{kind, flops, bytes, t_trace->get(), t_trace->get(), s};
  if (!r.e0 || !r.e1) return;
  t = t_trace;
  st = s;
  idx = (int)t->recs.size();
  cudaEventRecord(r.e0, s);
  t->recs.push_back(r);
}

TraceMark::~TraceMark() {
  if (t) cudaEventRecord(t->recs[idx].e1, st);
}

}  // namespace egpu

using namespace egpu;




// A device matrix argument that may need repacking into an aligned copy for TMA.
struct Operand {
  double* ptr;
  long long ld;
  double* user;
  long long user_ld;
  int rows, cols;
  bool packed = false;
};

// Blocked triangular solve with the diagonal blocks pre-inverted (Winv, one
// nb x nb block per diagonal block, ld nb).  Covers Trsm's eight
// side/uplo/orientation cases (blas-like/level3/Trsm.hpp:49-86); the
// unit/non-unit choice is carried by Winv.  B is m x n; alpha already applied.
int trsm_blocked(cudaStream_t st, int side, int uplo, int trans, int m, int n, const double* A, long long lda,
                 const double* Winv, int nb, double* B, long long ldb, DevStatus* status) {
  const int nt = (side == EGPU_LEFT) ? m : n;  // order of the triangle
  const int nblk = (nt + nb - 1) / nb;
  const bool fwd = (side == EGPU_LEFT) ? ((uplo == EGPU_LOWER) == !trans) : ((uplo == EGPU_UPPER) == !trans);
  for (int s = 0; s < nblk; ++s) {
    const int i = fwd ? s : nblk - 1 - s;
    const int i0 = i * nb;
    const int bi = std::min(nb, nt - i0);
    const double* Wi = Winv + (size_t)i * nb * nb;
    if (side == EGPU_LEFT) {
      double* Bi = B + i0;
      // B_i := op(inv(A_ii)) * B_i   (in place; one CTA holds all bi rows)
      TRY(launch_dgemm(st, trans != 0, true, bi, n, bi, 1.0, Wi, nb, Bi, ldb, 0.0, Bi, ldb, 0, false, status));
      if (fwd) {
        const int r0 = i0 + bi, mr = nt - r0;
        if (mr > 0) {
          // B_below -= op(A)_{below,i} * B_i
          if (!trans)  // A_{below,i} stored rows r0.., cols i0.. : MN-major
            TRY(launch_dgemm(st, false, true, mr, n, bi, -1.0, A + r0 + (size_t)i0 * lda, lda, Bi, ldb, 1.0,
                             B + r0, ldb, 0, false, status));
          else  // (A_{i,below})^T, A_{i,below} = rows i0.., cols r0.. : K-major
            TRY(launch_dgemm(st, true, true, mr, n, bi, -1.0, A + i0 + (size_t)r0 * lda, lda, Bi, ldb, 1.0,
                             B + r0, ldb, 0, false, status));
        }
      } else {
        const int mr = i0;
        if (mr > 0) {
          if (!trans)  // A_{above,i}: rows 0..i0, cols i0.. : MN-major
            TRY(launch_dgemm(st, false, true, mr, n, bi, -1.0, A + (size_t)i0 * lda, lda, Bi, ldb, 1.0, B, ldb, 0,
                             false, status));
          else  // (A_{i,above})^T, A_{i,above}: rows i0.., cols 0..i0 : K-major
            TRY(launch_dgemm(st, true, true, mr, n, bi, -1.0, A + i0, lda, Bi, ldb, 1.0, B, ldb, 0, false,
                             status));
        }
      }
    } else {
      double* Bi = B + (size_t)i0 * ldb;
      // B_i := B_i * op(inv(A_ii))   (in place; one CTA holds all bi columns)
      TRY(launch_dgemm(st, false, trans == 0, m, bi, bi, 1.0, Bi, ldb, Wi, nb, 0.0, Bi, ldb, 0, true, status));
      if (fwd) {
        const int c0 = i0 + bi, nc = nt - c0;
        if (nc > 0) {
          if (!trans)  // op(A) = A_{i,right}: rows i0.., cols c0.. (K x N) : K-major
            TRY(launch_dgemm(st, false, true, m, nc, bi, -1.0, Bi, ldb, A + i0 + (size_t)c0 * lda, lda, 1.0,
                             B + (size_t)c0 * ldb, ldb, 0, false, status));
          else  // op(A) = (A_{right,i})^T: A rows c0.., cols i0.. (N x K) : MN-major
            TRY(launch_dgemm(st, false, false, m, nc, bi, -1.0, Bi, ldb, A + c0 + (size_t)i0 * lda, lda, 1.0,
                             B + (size_t)c0 * ldb, ldb, 0, false, status));
        }
      } else {
        const int nc = i0;
        if (nc > 0) {
          if (!trans)  // A_{i,left}: rows i0.., cols 0.. : K-major
            TRY(launch_dgemm(st, false, true, m, nc, bi, -1.0, Bi, ldb, A + i0, lda, 1.0, B, ldb, 0, false,
                             status));
          else  // (A_{left,i})^T: A rows 0.., cols i0.. : MN-major
            TRY(launch_dgemm(st, false, false, m, nc, bi, -1.0, Bi, ldb, A + (size_t)i0 * lda, lda, 1.0, B, ldb,
                             0, false, status));
        }
      }
    }
  }
  return EGPU_OK;
}

int check_handle(egpu_context* h) { return h ? EGPU_OK : EGPU_ERR_ARG; }

// Workspace carve for diag-block inverses of an order-nt triangle.
size_t winv_bytes(int nt, int nb) { return sizeof(double) * (size_t)((nt + nb - 1) / nb) * nb * nb; }

// ----- core device drivers on TMA-compatible operands -----

// Sequential blocked right-looking Cholesky: per block column, potrf of the
// diagonal block (+ its inverse), the panel Trsm as a multiply by that
// inverse, and the Herk trailing update (LVar3.hpp:83-123 / UVar3.hpp:85-125).
int potrf_seq(egpu_context* h, int uplo, int n, double* A, long long lda, double* W) {
  const int nb = h->nb;
  cudaStream_t st = h->stream;
  for (int k = 0; k < n; k += nb) {
    const int b = std::min(nb, n - k);
    const int m2 = n - k - b;
    double* A11 = A + k + (size_t)k * lda;
    TRY(launch_potrf_diag(st, uplo, A11, lda, b, W, nb, h->dstatus, k));
    if (m2 == 0) continue;
    if (uplo == EGPU_LOWER) {
      double* A21 = A + (k + b) + (size_t)k * lda;
      double* A22 = A + (k + b) + (size_t)(k + b) * lda;
      // Trsm(RIGHT, LOWER, ADJOINT, NON_UNIT, 1, A11, A21): A21 := A21 * inv(L11)^T
      TRY(launch_dgemm(st, false, false, m2, b, b, 1.0, A21, lda, W, nb, 0.0, A21, lda, 0, true, h->dstatus));
      // Herk(LOWER, NORMAL, -1, A21, 1, A22)
      TRY(launch_dgemm(st, false, false, m2, m2, b, -1.0, A21, lda, A21, lda, 1.0, A22, lda, 1, false, h->dstatus));
    } else {
      double* A12 = A + k + (size_t)(k + b) * lda;
      double* A22 = A + (k + b) + (size_t)(k + b) * lda;
      // Trsm(LEFT, UPPER, ADJOINT, NON_UNIT, 1, A11, A12): A12 := inv(U11)^T * A12
      TRY(launch_dgemm(st, true, true, b, m2, b, 1.0, W, nb, A12, lda, 0.0, A12, lda, 0, false, h->dstatus));
      // Herk(UPPER, ADJOINT, -1, A12, 1, A22)
      TRY(launch_dgemm(st, true, true, m2, m2, b, -1.0, A12, lda, A12, lda, 1.0, A22, lda, 2, false, h->dstatus));
    }
  }
  return EGPU_OK;
}

// The Herk update of step k restricted to the trailing block columns
// [c0, c1) (lower) or block rows [c0, c1) (upper).  Rows/cols are global.
int potrf_update_cols(egpu_context* h, cudaStream_t st, int uplo, int n, double* A, long long lda, int k, int b,
                      int c0, int c1) {
  if (c1 <= c0) return EGPU_OK;
  if (uplo == EGPU_LOWER) {
    // A[c0:n, c0:c1] -= A[c0:n, k:k+b] * A[c0:c1, k:k+b]^T   (lower part)
    return launch_dgemm(st, false, false, n - c0, c1 - c0, b, -1.0, A + c0 + (size_t)k * lda, lda,
                        A + c0 + (size_t)k * lda, lda, 1.0, A + c0 + (size_t)c0 * lda, lda, 1, false, h->dstatus);
  }
  // A[c0:c1, c0:n] -= A[k:k+b, c0:c1]^T * A[k:k+b, c0:n]   (upper part)
  return launch_dgemm(st, true, true, c1 - c0, n - c0, b, -1.0, A + k + (size_t)c0 * lda, lda,
                      A + k + (size_t)c0 * lda, lda, 1.0, A + c0 + (size_t)c0 * lda, lda, 2, false, h->dstatus);
}

// The diagonal-block factorization and panel Trsm of step k.
int potrf_panel(egpu_context* h, cudaStream_t st, int uplo, int n, double* A, long long lda, int k, int b,
                double* W) {
  const int nb = h->nb;
  const int m2 = n - k - b;
  TRY(launch_potrf_diag(st, uplo, A + k + (size_t)k * lda, lda, b, W, nb, h->dstatus, k));
  if (m2 == 0) return EGPU_OK;
  if (uplo == EGPU_LOWER) {
    double* A21 = A + (k + b) + (size_t)k * lda;
    return launch_dgemm(st, false, false, m2, b, b, 1.0, A21, lda, W, nb, 0.0, A21, lda, 0, true, h->dstatus);
  }
  double* A12 = A + k + (size_t)(k + b) * lda;
  return launch_dgemm(st, true, true, b, m2, b, 1.0, W, nb, A12, lda, 0.0, A12, lda, 0, false, h->dstatus);
}

// Look-ahead depth 1: the panel of step k+1 (update of block column k+1 by
// step k, diagonal factorization, panel Trsm) runs on a high-priority side
// stream while the rest of step k's trailing update runs on the main stream.
//   side:  [upd(k -> col k+1)] [potrf k+1] [trsm k+1] -> ev_panel
//   main:  wait ev_panel(k) -> [upd(k -> cols >= k+2)] -> ev_rest
// The side stream waits for ev_rest(k-1) before touching column k+1, which
// step k-1's main-stream update also wrote.
int potrf_lookahead(egpu_context* h, int uplo, int n, double* A, long long lda, double* W) {
  const int nb = h->nb;
  const int nblk = (n + nb - 1) / nb;
  cudaStream_t M = h->stream, P = h->side;
  EGPU_CUDA_TRY(cudaEventRecord(h->ev_fork, M));
  EGPU_CUDA_TRY(cudaStreamWaitEvent(P, h->ev_fork, 0));
  TRY(potrf_panel(h, P, uplo, n, A, lda, 0, std::min(nb, n), W));
  EGPU_CUDA_TRY(cudaEventRecord(h->ev_panel[0], P));
  for (int kb = 0; kb < nblk; ++kb) {
    const int k = kb * nb, b = std::min(nb, n - k);
    const int c1 = k + b, c2 = std::min(n, c1 + nb);
    if (kb + 1 < nblk) {
      if (kb >= 1) EGPU_CUDA_TRY(cudaStreamWaitEvent(P, h->ev_rest[(kb - 1) & 1], 0));
      TRY(potrf_update_cols(h, P, uplo, n, A, lda, k, b, c1, c2));
      TRY(potrf_panel(h, P, uplo, n, A, lda, c1, c2 - c1, W));
      EGPU_CUDA_TRY(cudaEventRecord(h->ev_panel[(kb + 1) & 1], P));
    }
    EGPU_CUDA_TRY(cudaStreamWaitEvent(M, h->ev_panel[kb & 1], 0));
    TRY(potrf_update_cols(h, M, uplo, n, A, lda, k, b, c2, n));
    EGPU_CUDA_TRY(cudaEventRecord(h->ev_rest[kb & 1], M));
  }
  EGPU_CUDA_TRY(cudaEventRecord(h->ev_join, P));
  EGPU_CUDA_TRY(cudaStreamWaitEvent(M, h->ev_join, 0));
  return EGPU_OK;
}

// Look-ahead over groups of G panels, so that the trailing update reads and
// writes the matrix once per G panels (K = G nb: the DMMA update's fixed cost
// per pass -- tile fill, C read-modify-write -- amortised over G times the
// flops; FP64 throughout, so the deferral changes only summation order).
//   side:  per panel kb of group g = [g0, g1): update block column kb by the
//          group's earlier panels [g0, kb) (one product, K = (kb - g0) nb),
//          then factor it; after the last panel -> ev_panel(g)
//   main:  wait ev_panel(g); update by the whole group the next group's first
//          block column (-> ev_next), its other block columns (-> ev_rest),
//          then everything beyond it
// Group g+1's first panel waits for ev_next(g), its later panels for
// ev_rest(g); the main stream alone writes columns beyond the group the side
// stream is factoring, so no column is written by both streams at once.
// G <= 0 selects the group size per group from the order of the trailing
// matrix: deep groups while the main-stream update dominates, single panels
// once the side chain (diag + Trsm + column update per panel) is the longer.
// The first groups are kept short (2, then 8 panels): until a group is
// factored the main stream has nothing to update, and the first update (K =
// 2 nb over the whole matrix) is long enough to hide the next group's chain.
static const int kRamp[4] = {2, 8, 16, 16};

static int auto_group(int m_left) {
  return m_left > 12288 ? 16 : m_left > 7168 ? 8 : m_left > 5120 ? 4 : m_left > 3072 ? 2 : 1;
}

int potrf_grouped(egpu_context* h, int uplo, int n, double* A, long long lda, double* W, int G) {
  const int nb = h->nb;
  const int nblk = (n + nb - 1) / nb;
  cudaStream_t M = h->stream, P = h->side;
  EGPU_CUDA_TRY(cudaEventRecord(h->ev_fork, M));
  EGPU_CUDA_TRY(cudaStreamWaitEvent(P, h->ev_fork, 0));
  int Gn = 1;  // the current group's size
  for (int g0 = 0, gi = 0; g0 < nblk; g0 += Gn, ++gi) {
    Gn = G > 0 ? G : std::min(auto_group(n - g0 * nb), kRamp[std::min(gi, 3)]);
    const int g1 = std::min(nblk, g0 + Gn);
    const int kg = g0 * nb, kend = std::min(n, g1 * nb), Kg = kend - kg;  // the group's columns
    for (int kb = g0; kb < g1; ++kb) {
      const int k = kb * nb, b = std::min(nb, n - k);
      if (kb == g0 && gi >= 1) EGPU_CUDA_TRY(cudaStreamWaitEvent(P, h->ev_next[(gi - 1) & 1], 0));
      if (kb == g0 + 1 && gi >= 1) EGPU_CUDA_TRY(cudaStreamWaitEvent(P, h->ev_rest[(gi - 1) & 1], 0));
      if (kb > g0) TRY(potrf_update_cols(h, P, uplo, n, A, lda, kg, k - kg, k, k + b));
      TRY(potrf_panel(h, P, uplo, n, A, lda, k, b, W));
    }
    if (g1 == nblk) break;
    EGPU_CUDA_TRY(cudaEventRecord(h->ev_panel[gi & 1], P));
    EGPU_CUDA_TRY(cudaStreamWaitEvent(M, h->ev_panel[gi & 1], 0));
    // the next group's columns [c1, c3): its size decides which of them the
    // main stream updates before ev_rest
    const int Gnext = G > 0 ? G : std::min(auto_group(n - kend), kRamp[std::min(gi + 1, 3)]);
    const int c1 = kend, c2 = std::min(n, c1 + nb), c3 = std::min(n, c1 + Gnext * nb);
    TRY(potrf_update_cols(h, M, uplo, n, A, lda, kg, Kg, c1, c2));
    EGPU_CUDA_TRY(cudaEventRecord(h->ev_next[gi & 1], M));
    TRY(potrf_update_cols(h, M, uplo, n, A, lda, kg, Kg, c2, c3));
    EGPU_CUDA_TRY(cudaEventRecord(h->ev_rest[gi & 1], M));
    TRY(potrf_update_cols(h, M, uplo, n, A, lda, kg, Kg, c3, n));
  }
  EGPU_CUDA_TRY(cudaEventRecord(h->ev_join, P));
  EGPU_CUDA_TRY(cudaStreamWaitEvent(M, h->ev_join, 0));
  return EGPU_OK;
}

int potrf_core(egpu_context* h, int uplo, int n, double* A, long long lda) {
  const int nb = h->nb;
  TRY(ensure_ws(h, sizeof(double) * (size_t)nb * nb + 4096));
  Carve cv(h->ws);
  double* W = cv.take<double>((size_t)nb * nb);
  if ((h->lookahead < 0 || h->lookahead >= 2) && n > 2 * nb)
    return potrf_grouped(h, uplo, n, A, lda, W, h->lookahead);
  if (h->lookahead && n > nb) return potrf_lookahead(h, uplo, n, A, lda, W);
  return potrf_seq(h, uplo, n, A, lda, W);
}

// Step k of LU after its panel: pivots applied to the block columns [c0, c1)
// (global columns, rows k..m), then the row-panel Trsm (multiply by
// inv(L11)) and the Gemm trailing update of those columns (LU.hpp:198-203).
int getrf_update_cols(egpu_context* h, cudaStream_t st, int m, double* A, long long lda, int k, int b,
                      const double* W, const int* image, const int* preimage, int c0, int c1) {
  if (c1 <= c0) return EGPU_OK;
  const int mr = m - k, nc = c1 - c0;
  TRY(launch_apply_composed(st, mr, nc, A + k + (size_t)c0 * lda, lda, b, image, preimage, h->dstatus));
  double* A12 = A + k + (size_t)c0 * lda;
  TRY(launch_dgemm(st, false, true, b, nc, b, 1.0, W, h->nb, A12, lda, 0.0, A12, lda, 0, false, h->dstatus));
  if (mr - b > 0)
    TRY(launch_dgemm(st, false, true, mr - b, nc, b, -1.0, A + (k + b) + (size_t)k * lda, lda, A12, lda, 1.0,
                     A + (k + b) + (size_t)c0 * lda, lda, 0, false, h->dstatus));
  return EGPU_OK;
}

// Blocked right-looking LU with partial pivoting (LU.hpp:144-218).
// With B != nullptr the n x nrhs block B is carried along as extra trailing
// columns (pivots, row-panel solve and Gemm update applied to it each step),
// which is RowEchelon (GaussianElimination.hpp:94-209); pivot_left = false
// then leaves the already-factored L columns unpermuted, as RowEchelon does.
int getrf_core(egpu_context* h, int m, int n, double* A, long long lda, int* dp, double* B = nullptr,
               long long ldb = 0, int nrhs = 0, bool pivot_left = true) {
  const int nb = h->nb;
  const int mn = std::min(m, n);
  const int nblk = (mn + nb - 1) / nb;
  const size_t panel_bytes = lu_panel_scratch_bytes(m, nb, h->sm_count);
  TRY(ensure_ws(h, 2 * (sizeof(double) * (size_t)nb * nb + 2 * sizeof(int) * nb + 512) + panel_bytes + 4096));
  Carve cv(h->ws);
  double* W[2];
  int *image[2], *preimage[2];
  for (int i = 0; i < 2; ++i) {
    W[i] = cv.take<double>((size_t)nb * nb);
    image[i] = cv.take<int>(nb);
    preimage[i] = cv.take<int>(nb);
  }
  void* pscr = cv.take<unsigned char>(panel_bytes);
  const bool la = h->lookahead && nblk > 1;
  cudaStream_t M = h->stream, P = la ? h->side : h->stream;
  auto rest = [&](cudaStream_t st, int k, int b, int s, int c0) -> int {
    if (pivot_left) TRY(launch_apply_composed(st, m - k, k, A + k, lda, b, image[s], preimage[s], h->dstatus));
    TRY(getrf_update_cols(h, st, m, A, lda, k, b, W[s], image[s], preimage[s], c0, n));
    if (B != nullptr && nrhs > 0) {  // B rides along as columns n .. n + nrhs
      const int mr = m - k;
      double* B1 = B + k;
      TRY(launch_apply_composed(st, mr, nrhs, B1, ldb, b, image[s], preimage[s], h->dstatus));
      TRY(launch_dgemm(st, false, true, b, nrhs, b, 1.0, W[s], nb, B1, ldb, 0.0, B1, ldb, 0, false, h->dstatus));
      if (mr - b > 0)
        TRY(launch_dgemm(st, false, true, mr - b, nrhs, b, -1.0, A + (k + b) + (size_t)k * lda, lda, B1, ldb, 1.0,
                         B + k + b, ldb, 0, false, h->dstatus));
    }
    return EGPU_OK;
  };
  if (la) {
    EGPU_CUDA_TRY(cudaEventRecord(h->ev_fork, M));
    EGPU_CUDA_TRY(cudaStreamWaitEvent(P, h->ev_fork, 0));
  }
  TRY(launch_lu_panel(P, m, std::min(nb, mn), A, lda, dp, 0, image[0], preimage[0], W[0], nb, pscr, h->dstatus,
                      h->sm_count));
  if (la) EGPU_CUDA_TRY(cudaEventRecord(h->ev_panel[0], P));
  for (int kb = 0; kb < nblk; ++kb) {
    const int k = kb * nb, b = std::min(nb, mn - k), s = kb & 1;
    const int c1 = k + b;                 // first column right of the panel
    const int c2 = std::min(n, c1 + nb);  // end of the next block column
    if (!la) {
      TRY(rest(M, k, b, s, c1));
      if (kb + 1 < nblk) {
        const int k1 = c1, b1 = std::min(nb, mn - k1);
        TRY(launch_lu_panel(M, m - k1, b1, A + k1 + (size_t)k1 * lda, lda, dp + k1, k1, image[s ^ 1],
                            preimage[s ^ 1], W[s ^ 1], nb, pscr, h->dstatus, h->sm_count));
      }
      continue;
    }
    if (kb + 1 < nblk) {
      // side stream: bring block column kb+1 up to date, then factor it
      if (kb >= 1) EGPU_CUDA_TRY(cudaStreamWaitEvent(P, h->ev_rest[(kb - 1) & 1], 0));
      TRY(getrf_update_cols(h, P, m, A, lda, k, b, W[s], image[s], preimage[s], c1, c2));
      const int k1 = c1, b1 = std::min(nb, mn - k1);
      TRY(launch_lu_panel(P, m - k1, b1, A + k1 + (size_t)k1 * lda, lda, dp + k1, k1, image[s ^ 1],
                          preimage[s ^ 1], W[s ^ 1], nb, pscr, h->dstatus, h->sm_count));
      EGPU_CUDA_TRY(cudaEventRecord(h->ev_panel[(kb + 1) & 1], P));
    }
    // main stream: pivots on the left columns and the rest of the update
    // (after the last panel nothing ran on the side stream: start at c1)
    EGPU_CUDA_TRY(cudaStreamWaitEvent(M, h->ev_panel[s], 0));
    TRY(rest(M, k, b, s, kb + 1 < nblk ? c2 : c1));
    EGPU_CUDA_TRY(cudaEventRecord(h->ev_rest[s], M));
  }
  if (la) {
    EGPU_CUDA_TRY(cudaEventRecord(h->ev_join, P));
    EGPU_CUDA_TRY(cudaStreamWaitEvent(M, h->ev_join, 0));
  }
  return EGPU_OK;
}

int getrf_nopiv_core(egpu_context* h, int m, int n, double* A, long long lda) {
  const int nb = h->nb;
  const int mn = std::min(m, n);
  cudaStream_t st = h->stream;
  TRY(ensure_ws(h, 2 * sizeof(double) * (size_t)nb * nb + 4096));
  Carve cv(h->ws);
  double* W = cv.take<double>((size_t)nb * nb);
  double* W2 = cv.take<double>((size_t)nb * nb);
  for (int k = 0; k < mn; k += nb) {
    const int b = std::min(nb, mn - k);
    const int m2 = m - k - b, n2 = n - k - b;
    double* A11 = A + k + (size_t)k * lda;
    TRY(launch_getrf_diag_nopiv(st, A11, lda, b, W, nb, W2, h->dstatus, k));
    double* A21 = A + (k + b) + (size_t)k * lda;
    double* A12 = A + k + (size_t)(k + b) * lda;
    double* A22 = A + (k + b) + (size_t)(k + b) * lda;
    // Trsm(RIGHT, UPPER, NORMAL, NON_UNIT, 1, A11, A21): A21 := A21 * inv(U11)
    if (m2 > 0) TRY(launch_dgemm(st, false, true, m2, b, b, 1.0, A21, lda, W2, nb, 0.0, A21, lda, 0, true, h->dstatus));
    // Trsm(LEFT, LOWER, NORMAL, UNIT, 1, A11, A12): A12 := inv(L11) * A12
    if (n2 > 0) TRY(launch_dgemm(st, false, true, b, n2, b, 1.0, W, nb, A12, lda, 0.0, A12, lda, 0, false, h->dstatus));
    // Gemm(NORMAL, NORMAL, -1, A21, A12, 1, A22)
    if (m2 > 0 && n2 > 0)
      TRY(launch_dgemm(st, false, true, m2, n2, b, -1.0, A21, lda, A12, lda, 1.0, A22, lda, 0, false, h->dstatus));
  }
  return EGPU_OK;
}

// Triangular solve of order nt with diag-block inverses computed here.
int trsm_core(egpu_context* h, int side, int uplo, int trans, int unit, int m, int n, double alpha,
              const double* A, long long lda, double* B, long long ldb, size_t ws_offset = 0) {
  const int nb = h->nb;
  const int nt = side == EGPU_LEFT ? m : n;
  if (m == 0 || n == 0) return EGPU_OK;
  cudaStream_t st = h->stream;
  TRY(ensure_ws(h, ws_offset + winv_bytes(nt, nb) + 4096));
  Carve cv(h->ws);
  cv.off = ws_offset;
  double* Winv = cv.take<double>((size_t)((nt + nb - 1) / nb) * nb * nb);
  if (alpha != 1.0) TRY(launch_scale(st, m, n, alpha, B, ldb, 0));
  TRY(launch_trtri_blocks(st, uplo, unit, A, lda, nt, nb, Winv, nb));
  return trsm_blocked(st, side, uplo, trans, m, n, A, lda, Winv, nb, B, ldb, h->dstatus);
}

// Can the one-launch skinny sweep (trsm_skinny.cu) take this right-hand side?
static bool skinny_ok(egpu_context* h, int nrhs, const double* A, long long lda, const double* B, long long ldb) {
  return nrhs >= 1 && nrhs <= 64 && h->nb <= 128 && h->nb % 2 == 0 && ldb % 2 == 0 && lda % 2 == 0 &&
         reinterpret_cast<uintptr_t>(B) % 16 == 0 && reinterpret_cast<uintptr_t>(A) % 16 == 0;
}

// X := inv(T2) inv(T1) X with two skinny sweeps.  Each T is (uplo, unit) for
// the inverted diagonal blocks and (bwd, amode) for the sweep; Winv areas and
// the sweep flags are carved at ws_off.
struct SweepSpec {
  int uplo, unit, bwd, amode;
};
static int skinny_pair(egpu_context* h, int n, int nrhs, const double* A, long long lda, double* B, long long ldb,
                       SweepSpec t1, SweepSpec t2, size_t ws_off) {
  const int nb = h->nb;
  const bool same = t1.uplo == t2.uplo && t1.unit == t2.unit;
  const size_t wb = align_up(winv_bytes(n, nb), 256);
  TRY(ensure_ws(h, ws_off + (same ? 1 : 2) * wb + trsm_skinny_flag_bytes(n, nb) + 4096));
  unsigned char* base = static_cast<unsigned char*>(h->ws) + ws_off;
  double* W1 = reinterpret_cast<double*>(base);
  double* W2 = same ? W1 : reinterpret_cast<double*>(base + wb);
  int* flags = reinterpret_cast<int*>(base + (same ? 1 : 2) * wb);
  cudaStream_t st = h->stream;
  EGPU_CUDA_TRY(cudaMemsetAsync(flags, 0, trsm_skinny_flag_bytes(n, nb), st));
  TRY(launch_trtri_blocks(st, t1.uplo, t1.unit, A, lda, n, nb, W1, nb));
  if (!same) TRY(launch_trtri_blocks(st, t2.uplo, t2.unit, A, lda, n, nb, W2, nb));
  TRY(launch_trsm_skinny(st, t1.bwd, t1.amode, n, nrhs, A, lda, W1, nb, B, ldb, flags, 1, h->sm_count, h->dstatus));
  return launch_trsm_skinny(st, t2.bwd, t2.amode, n, nrhs, A, lda, W2, nb, B, ldb, flags, 2, h->sm_count,
                            h->dstatus);
}

int getrs_core(egpu_context* h, int orient, int n, int nrhs, const double* A, long long lda, const int* dp,
               double* B, long long ldb) {
  // lu::SolveAfter (LU/SolveAfter.hpp:101-146)
  // laswp scratch: perm (n ints) + n*nrhs doubles; placed after the Winv area
  const size_t winv = winv_bytes(n, h->nb);
  const size_t lsw = align_up(sizeof(int) * (size_t)((n + 1) & ~1), 256) + sizeof(double) * (size_t)n * nrhs;
  const size_t skinny_off = align_up(align_up(winv + 4096, 256) + lsw + 4096, 256);
  TRY(ensure_ws(h, align_up(winv + 4096, 256) + lsw + 4096));
  int* perm = reinterpret_cast<int*>(static_cast<unsigned char*>(h->ws) + align_up(winv + 4096, 256));
  const size_t trsm_off = 0;
  const bool sk = skinny_ok(h, nrhs, A, lda, B, ldb);
  if (sk) {  // reserve now: a later growth of the workspace would move perm
    TRY(ensure_ws(h, skinny_off + 2 * align_up(winv_bytes(n, h->nb), 256) + trsm_skinny_flag_bytes(n, h->nb) + 8192));
    perm = reinterpret_cast<int*>(static_cast<unsigned char*>(h->ws) + align_up(winv + 4096, 256));
  }
  if (orient == EGPU_NORMAL) {
    if (dp) TRY(launch_laswp_seq(h->stream, 0, n, nrhs, B, ldb, dp, n, perm));
    if (sk) {
      TRY(skinny_pair(h, n, nrhs, A, lda, B, ldb, {EGPU_LOWER, 1, 0, 0}, {EGPU_UPPER, 0, 1, 0}, skinny_off));
    } else {
      TRY(trsm_core(h, EGPU_LEFT, EGPU_LOWER, 0, 1, n, nrhs, 1.0, A, lda, B, ldb, trsm_off));
      TRY(trsm_core(h, EGPU_LEFT, EGPU_UPPER, 0, 0, n, nrhs, 1.0, A, lda, B, ldb, trsm_off));
    }
  } else {
    if (sk) {
      TRY(skinny_pair(h, n, nrhs, A, lda, B, ldb, {EGPU_UPPER, 0, 0, 1}, {EGPU_LOWER, 1, 1, 1}, skinny_off));
    } else {
      TRY(trsm_core(h, EGPU_LEFT, EGPU_UPPER, 1, 0, n, nrhs, 1.0, A, lda, B, ldb, trsm_off));
      TRY(trsm_core(h, EGPU_LEFT, EGPU_LOWER, 1, 1, n, nrhs, 1.0, A, lda, B, ldb, trsm_off));
    }
    if (dp) TRY(launch_laswp_seq(h->stream, 1, n, nrhs, B, ldb, dp, n, perm));
  }
  return EGPU_OK;
}
int potrs_core(egpu_context* h, int uplo, int n, int nrhs, const double* A, long long lda, double* B,
               long long ldb) {
  // cholesky::SolveAfter (Cholesky/SolveAfter.hpp:20-75); TRANSPOSE only
  // conjugates B, a no-op for real data.
  if (skinny_ok(h, nrhs, A, lda, B, ldb)) {
    if (uplo == EGPU_LOWER) return skinny_pair(h, n, nrhs, A, lda, B, ldb, {EGPU_LOWER, 0, 0, 0}, {EGPU_LOWER, 0, 1, 1}, 0);
    return skinny_pair(h, n, nrhs, A, lda, B, ldb, {EGPU_UPPER, 0, 0, 1}, {EGPU_UPPER, 0, 1, 0}, 0);
  }
  if (uplo == EGPU_LOWER) {
    TRY(trsm_core(h, EGPU_LEFT, EGPU_LOWER, 0, 0, n, nrhs, 1.0, A, lda, B, ldb));
    TRY(trsm_core(h, EGPU_LEFT, EGPU_LOWER, 1, 0, n, nrhs, 1.0, A, lda, B, ldb));
  } else {
    TRY(trsm_core(h, EGPU_LEFT, EGPU_UPPER, 1, 0, n, nrhs, 1.0, A, lda, B, ldb));
    TRY(trsm_core(h, EGPU_LEFT, EGPU_UPPER, 0, 0, n, nrhs, 1.0, A, lda, B, ldb));
  }
  return EGPU_OK;
}

// GaussianElimination (GaussianElimination.hpp:216-232): RowEchelon -- LU
// with partial pivoting with B carried along as trailing columns and the
// L columns left unpermuted (the distributed RowEchelon, :94-209, which a
// 1 x 1 grid runs) -- then B := inv(U) B.
int gesv_core(egpu_context* h, int n, int nrhs, double* A, long long lda, double* B, long long ldb) {
  // pivots of RowEchelon are not returned; keep them in a staging slot
  if (ensure_stage(h, 2, sizeof(int) * (size_t)std::max(n, 1)) != EGPU_OK) return EGPU_ERR_ALLOC;
  int* p = static_cast<int*>(h->stage[2]);
  TRY(getrf_core(h, n, n, A, lda, p, B, ldb, nrhs, false));
  int info = 0;
  int rc = read_status(h, &info);
  if (rc != EGPU_OK) return rc;
  if (nrhs == 0) return EGPU_OK;
  return trsm_core(h, EGPU_LEFT, EGPU_UPPER, 0, 0, n, nrhs, 1.0, A, lda, B, ldb);
}

// TriangularInverse (lapack-like/TriangularInverse.hpp:56-64): the uplo
// triangle of A := its inverse, by the blocked Trsm against the identity in
// staging slot 3; the other triangle (and, for UNIT, the diagonal) is not
// touched.
int trtri_core(egpu_context* h, int uplo, int unit, int n, double* A, long long lda) {
  const long long ldx = ld_aligned(n);
  TRY(ensure_stage(h, 3, sizeof(double) * (size_t)ldx * n));
  double* X = static_cast<double*>(h->stage[3]);
  TRY(launch_set_identity(h->stream, n, X, ldx));
  TRY(trsm_core(h, EGPU_LEFT, uplo, 0, unit, n, n, 1.0, A, lda, X, ldx));
  return launch_copy_triangle(h->stream, uplo, unit != 0, n, X, ldx, A, lda);
}

// Inverse (Inverse.hpp:17-23 -> inverse::LUPartialPiv, Inverse/LUPartialPiv.hpp):
// P A = L U, then A := inv(A) as the solution of A X = I (lu::SolveAfter on
// the identity).  A singular pivot stops with EGPU_SINGULAR (SingularMatrix-
// Exception from lu::Panel), A then holding the partial factorization.
int getri_core(egpu_context* h, int n, double* A, long long lda, int* info) {
  int* dp = static_cast<int*>(h->stage[2]);
  TRY(getrf_core(h, n, n, A, lda, dp));
  TRY(read_status(h, info));
  const long long ldx = ld_aligned(n);
  TRY(ensure_stage(h, 3, sizeof(double) * (size_t)ldx * n));
  double* X = static_cast<double*>(h->stage[3]);
  TRY(launch_set_identity(h->stream, n, X, ldx));
  TRY(getrs_core(h, EGPU_NORMAL, n, n, A, lda, dp, X, ldx));
  return launch_copy(h->stream, n, n, X, ldx, A, lda);
}

// HPDInverse (Inverse.hpp:25-35 -> hpd_inverse::CholeskyLVar2 / UVar2): the
// uplo triangle of A := that of inv(A), from the Cholesky factor and
// cholesky::SolveAfter on the identity; the other triangle is not touched.
// A non-HPD input stops with EGPU_NOT_HPD.
int potri_core(egpu_context* h, int uplo, int n, double* A, long long lda, int* info) {
  TRY(potrf_core(h, uplo, n, A, lda));
  TRY(read_status(h, info));
  const long long ldx = ld_aligned(n);
  TRY(ensure_stage(h, 3, sizeof(double) * (size_t)ldx * n));
  double* X = static_cast<double*>(h->stage[3]);
  TRY(launch_set_identity(h->stream, n, X, ldx));
  TRY(potrs_core(h, uplo, n, n, A, lda, X, ldx));
  return launch_copy_triangle(h->stream, uplo, false, n, X, ldx, A, lda);
}

// ReverseCholesky (lapack-like/Cholesky.hpp:64-76 -> cholesky::ReverseLVar3 /
// ReverseUVar3, Cholesky/LVar3.hpp:125-165): LOWER: A = L^T L, L lower;
// UPPER: A = U U^T, U upper, swept from the bottom-right corner.  With J the
// reversal permutation, the reverse factor of A is J chol(J A J) J with the
// other triangle: the uplo triangle is rotated by 180 degrees into staging
// slot 3 (where it becomes the opposite triangle), factored forward, and the
// factor rotated back.  Only the uplo triangle of A is read or written.
// EGPU_NOT_HPD's info is the 1-based column of A where the reverse sweep
// stopped.
int reverse_potrf_core(egpu_context* h, int uplo, int n, double* A, long long lda, int* info) {
  const long long ldx = ld_aligned(n);
  TRY(ensure_stage(h, 3, sizeof(double) * (size_t)ldx * n));
  double* X = static_cast<double*>(h->stage[3]);
  const int other = uplo == EGPU_LOWER ? EGPU_UPPER : EGPU_LOWER;
  TRY(launch_rotate_triangle(h->stream, uplo, n, A, lda, X, ldx));
  TRY(potrf_core(h, other, n, X, ldx));
  int col = 0;
  const int rc = read_status(h, &col);
  if (rc == EGPU_NOT_HPD && info) *info = n + 1 - col;
  TRY(rc);
  return launch_rotate_triangle(h->stream, other, n, X, ldx, A, lda);
}

// LDLT / LDLH (lapack-like/LDL.hpp -> ldl::Var3, LDL/Var3.hpp): blocked
// LDL^T without pivoting on the lower triangle (the upper one is not read or
// written).  Per block column: the symmetric diagonal block, staged from the
// lower triangle, is factored by the unpivoted LU kernel (a symmetric block
// has U11 = D11 L11^T), L11 and D11 are written back (d receives D when
// given); S21 = A21 inv(L11)^T (= L21 D11) before A21 := L21 = A21 inv(U11)
// (Trsm as a multiply, in place), then A22 -= S21 L21^T on the lower
// triangle.  An exact zero pivot stops with EGPU_SINGULAR
// (SingularMatrixException, LDL/Var3.hpp:44-45).
int ldl_core(egpu_context* h, int n, double* A, long long lda, double* d) {
  const int nb = h->nb;
  cudaStream_t st = h->stream;
  const long long lds = ld_aligned(n);
  TRY(ensure_ws(h, 3 * align_up(sizeof(double) * (size_t)nb * nb, 256) + sizeof(double) * (size_t)lds * nb + 4096));
  Carve cv(h->ws);
  double* W = cv.take<double>((size_t)nb * nb);    // inv(L11), unit lower
  double* W2 = cv.take<double>((size_t)nb * nb);   // inv(U11)
  double* Blk = cv.take<double>((size_t)nb * nb);  // the symmetric diagonal block, ld nb
  double* S21 = cv.take<double>((size_t)lds * nb);
  for (int k = 0; k < n; k += nb) {
    const int b = std::min(nb, n - k), m2 = n - k - b;
    double* A11 = A + k + (size_t)k * lda;
    TRY(launch_sym_from_lower(st, b, A11, lda, Blk, nb));
    TRY(launch_getrf_diag_nopiv(st, Blk, nb, b, W, nb, W2, h->dstatus, k));
    TRY(launch_ldl_block_writeback(st, b, Blk, nb, A11, lda, d ? d + k : nullptr));
    if (m2 == 0) continue;
    double* A21 = A + (k + b) + (size_t)k * lda;
    double* A22 = A + (k + b) + (size_t)(k + b) * lda;
    TRY(launch_dgemm(st, false, false, m2, b, b, 1.0, A21, lda, W, nb, 0.0, S21, lds, 0, false, h->dstatus));
    TRY(launch_dgemm(st, false, true, m2, b, b, 1.0, A21, lda, W2, nb, 0.0, A21, lda, 0, true, h->dstatus));
    TRY(launch_dgemm(st, false, false, m2, m2, b, -1.0, S21, lds, A21, lda, 1.0, A22, lda, 1, false, h->dstatus));
  }
  return EGPU_OK;
}

// SafeDeterminant (Determinant.hpp, determinant::LUPartialPiv,
// Determinant/LUPartialPiv.hpp:17-67) and SafeHPDDeterminant
// (hpd_determinant::Cholesky, Determinant/Cholesky.hpp:17-55) on the work
// matrix W (factored in place): det = rho exp(kappa n).  LU: rho = the signs
// of U's diagonal times (-1)^(pivot parity, PivotParity.hpp:17-33), kappa =
// sum log|u_ii| / n.  Cholesky: rho = 1, kappa = sum log l_ii / (n / 2).  A
// singular (LU) or non-HPD (Cholesky) matrix gives rho = kappa = 0, as the
// reference catches its exception.  Always synchronous: the values return to
// the host.
int safe_det_core(egpu_context* h, int hpd, int uplo, int n, double* W, long long ldw, double* rho,
                  double* kappa) {
  *rho = 1.0;
  *kappa = 0.0;
  if (n == 0) return EGPU_OK;
  const size_t piv_bytes = align_up(sizeof(int) * (size_t)n, 256);
  TRY(ensure_stage(h, 2, piv_bytes + 64));
  int* dp = static_cast<int*>(h->stage[2]);
  double* dout = reinterpret_cast<double*>(static_cast<unsigned char*>(h->stage[2]) + piv_bytes);
  EGPU_CUDA_TRY(cudaMemsetAsync(h->dstatus, 0, sizeof(DevStatus), h->stream));
  if (hpd) TRY(potrf_core(h, uplo, n, W, ldw));
  else TRY(getrf_core(h, n, n, W, ldw, dp));
  int rc = read_status_now(h, nullptr);
  if (rc == (hpd ? EGPU_NOT_HPD : EGPU_SINGULAR)) {
    EGPU_CUDA_TRY(cudaMemsetAsync(h->dstatus, 0, sizeof(DevStatus), h->stream));
    *rho = 0.0;
    return EGPU_OK;
  }
  TRY(rc);
  TRY(launch_diag_logsum(h->stream, n, W, ldw, hpd ? nullptr : dp, dout));
  double out[3];
  EGPU_CUDA_TRY(cudaMemcpyAsync(out, dout, sizeof(out), cudaMemcpyDeviceToHost, h->stream));
  EGPU_CUDA_TRY(cudaStreamSynchronize(h->stream));
  if (hpd) {
    *kappa = out[0] / (0.5 * n);
  } else {
    *kappa = out[0] / n;
    const long long flips = (long long)out[1] + (long long)out[2];
    *rho = (flips & 1) ? -1.0 : 1.0;
  }
  return EGPU_OK;
}

// ----- operand repacking for TMA alignment -----

int pack(egpu_context* h, int slot, Operand& op, bool copy_in) {
  op.packed = false;
  if (tma_compatible(op.ptr, op.ld)) return EGPU_OK;
  const long long ld = ld_aligned(op.rows);
  TRY(ensure_stage(h, slot, sizeof(double) * (size_t)ld * std::max(op.cols, 1)));
  op.user = op.ptr;
  op.user_ld = op.ld;
  op.ptr = static_cast<double*>(h->stage[slot]);
  op.ld = ld;
  op.packed = true;
  if (copy_in) TRY(launch_copy(h->stream, op.rows, op.cols, op.user, op.user_ld, op.ptr, op.ld));
  return EGPU_OK;
}

int unpack(egpu_context* h, const Operand& op) {
  if (!op.packed) return EGPU_OK;
  return launch_copy(h->stream, op.rows, op.cols, op.ptr, op.ld, op.user, op.user_ld);
}

Operand make_op(double* p, long long ld, int rows, int cols) {
  Operand o;
  o.ptr = p; o.ld = ld; o.user = p; o.user_ld = ld; o.rows = rows; o.cols = cols;
  return o;
}

bool bad_ld(long long ld, int rows) { return ld < std::max(1, rows); }


// ======================================================================
extern "C" {

int egpu_create(egpu_handle* out, int device) {
  if (!out) return EGPU_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return EGPU_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return EGPU_ERR_ARG;
  egpu_context* h = new (std::nothrow) egpu_context();
  if (!h) return EGPU_ERR_ALLOC;
  h->device = device;
  DeviceGuard g(device);
  cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&h->dstatus, sizeof(DevStatus)) != cudaSuccess ||
      cudaMallocHost(&h->hstatus, sizeof(DevStatus)) != cudaSuccess) {
    set_last_error(cudaGetLastError(), "egpu_create", __FILE__, __LINE__);
    egpu_destroy(h);
    return EGPU_ERR_CUDA;
  }
  h->stream = h->own_stream;
  {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);  // hi = greatest priority
    bool ok = cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, hi) == cudaSuccess;
    ok = ok && cudaStreamCreateWithPriority(&h->aux, cudaStreamNonBlocking, lo) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&h->ev_aux, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < 2; ++i) {
      ok = ok && cudaEventCreateWithFlags(&h->ev_panel[i], cudaEventDisableTiming) == cudaSuccess;
      ok = ok && cudaEventCreateWithFlags(&h->ev_rest[i], cudaEventDisableTiming) == cudaSuccess;
      ok = ok && cudaEventCreateWithFlags(&h->ev_split[i], cudaEventDisableTiming) == cudaSuccess;
      ok = ok && cudaEventCreateWithFlags(&h->ev_a21[i], cudaEventDisableTiming) == cudaSuccess;
      ok = ok && cudaEventCreateWithFlags(&h->ev_next[i], cudaEventDisableTiming) == cudaSuccess;
    }
    if (!ok) {
      set_last_error(cudaGetLastError(), "egpu_create streams", __FILE__, __LINE__);
      egpu_destroy(h);
      return EGPU_ERR_CUDA;
    }
  }
  cudaMemset(h->dstatus, 0, sizeof(DevStatus));
  *out = h;
  return EGPU_OK;
}

int egpu_destroy(egpu_handle h) {
  if (!h) return EGPU_OK;
  Enter g(h);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->ws) cudaFree(h->ws);
  for (int i = 0; i < egpu_context::kStageSlots; ++i)
    if (h->stage[i]) cudaFree(h->stage[i]);
  if (h->dstatus) cudaFree(h->dstatus);
  if (h->hstatus) cudaFreeHost(h->hstatus);
  if (h->side) cudaStreamSynchronize(h->side);
  if (h->aux) cudaStreamSynchronize(h->aux);
  for (cudaEvent_t e : {h->ev_fork, h->ev_join, h->ev_panel[0], h->ev_panel[1], h->ev_rest[0], h->ev_rest[1],
                        h->ev_split[0], h->ev_split[1], h->ev_aux, h->ev_a21[0], h->ev_a21[1], h->ev_next[0],
                        h->ev_next[1]})
    if (e) cudaEventDestroy(e);
  if (h->side) cudaStreamDestroy(h->side);
  if (h->aux) cudaStreamDestroy(h->aux);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return EGPU_OK;
}

int egpu_set_stream(egpu_handle h, void* s) {
  TRY(check_handle(h));
  h->stream = s ? static_cast<cudaStream_t>(s) : h->own_stream;
  return EGPU_OK;
}

void* egpu_get_stream(egpu_handle h) { return h ? static_cast<void*>(h->stream) : nullptr; }

int egpu_synchronize(egpu_handle h) {
  TRY(check_handle(h));
  Enter g(h);
  EGPU_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return EGPU_OK;
}

int egpu_set_blocksize(egpu_handle h, int nb) {
  TRY(check_handle(h));
  if (nb < 1) return EGPU_ERR_ARG;
  nb = std::min(128, std::max(2, nb));
  h->nb = nb & ~1;
  return EGPU_OK;
}

int egpu_get_blocksize(egpu_handle h) { return h ? h->nb : -1; }

int egpu_set_async(egpu_handle h, int on) {
  TRY(check_handle(h));
  Enter g(h);
  if (h->async && !on) {  // leaving async mode: settle outstanding work
    EGPU_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  h->async = on ? 1 : 0;
  return EGPU_OK;
}

int egpu_get_status(egpu_handle h, int* info) {
  TRY(check_handle(h));
  Enter g(h);
  int rc = read_status_now(h, info);
  EGPU_CUDA_TRY(cudaMemsetAsync(h->dstatus, 0, sizeof(DevStatus), h->stream));
  return rc;
}

int egpu_reserve(egpu_handle h, size_t bytes) {
  TRY(check_handle(h));
  Enter g(h);
  return ensure_ws(h, bytes);
}

int egpu_set_lookahead(egpu_handle h, int depth) {
  TRY(check_handle(h));
  if (depth < -1) return EGPU_ERR_ARG;
  h->lookahead = std::min(depth, 16);
  return EGPU_OK;
}

long long egpu_launch_count(egpu_handle) { return g_launches.load(); }

int egpu_trace_enable(egpu_handle h, int on) {
  TRY(check_handle(h));
  Enter g(h);
  cudaStreamSynchronize(h->stream);
  h->trace.clear();
  h->trace.on = on != 0;
  return EGPU_OK;
}

int egpu_trace_summary(egpu_handle h, int kind, double* total_ms, double* total_flops, double* total_bytes,
                       long long* launches) {
  TRY(check_handle(h));
  Enter g(h);
  double ms = 0, fl = 0, by = 0;
  long long n = 0;
  for (auto& r : h->trace.recs) {
    if (r.kind != kind) continue;
    EGPU_CUDA_TRY(cudaEventSynchronize(r.e1));
    float t = 0;
    EGPU_CUDA_TRY(cudaEventElapsedTime(&t, r.e0, r.e1));
    ms += t; fl += r.flops; by += r.bytes; ++n;
  }
  if (total_ms) *total_ms = ms;
  if (total_flops) *total_flops = fl;
  if (total_bytes) *total_bytes = by;
  if (launches) *launches = n;
  return EGPU_OK;
}

int egpu_trace_busy(egpu_handle h, int kind, double* busy_ms, double* share_ms) {
  TRY(check_handle(h));
  Enter g(h);
  if (kind < -1 || kind >= kTraceKinds) return EGPU_ERR_ARG;
  // every launch as an interval on one time axis (the first launch's start)
  struct Iv { double t0, t1; int kind; };
  std::vector<Iv> iv;
  const int n = (int)h->trace.recs.size();
  if (n > 0) {
    const cudaEvent_t base = h->trace.recs[0].e0;
    iv.reserve(n);
    for (const auto& r : h->trace.recs) {
      EGPU_CUDA_TRY(cudaEventSynchronize(r.e1));
      float a = 0, b = 0;
      EGPU_CUDA_TRY(cudaEventElapsedTime(&a, base, r.e0));
      EGPU_CUDA_TRY(cudaEventElapsedTime(&b, base, r.e1));
      iv.push_back({a, std::max(a, b), r.kind});
    }
  }
  // sweep over the interval end points: a segment counts toward `busy` when a
  // launch of `kind` (any kind for -1) is in flight, and toward `share` by
  // 1 / (number of distinct kinds in flight) when `kind` is one of them
  std::vector<std::pair<double, int>> ev;  // (time, +-(index + 1))
  ev.reserve(2 * iv.size());
  for (int i = 0; i < (int)iv.size(); ++i) {
    ev.push_back({iv[i].t0, i + 1});
    ev.push_back({iv[i].t1, -(i + 1)});
  }
  std::sort(ev.begin(), ev.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
    return a.first < b.first || (a.first == b.first && a.second < b.second);  // ends before starts
  });
  int active[kTraceKinds] = {0};
  double busy = 0, share = 0, prev = ev.empty() ? 0.0 : ev[0].first;
  for (const auto& e : ev) {
    const double dt = e.first - prev;
    if (dt > 0) {
      int kinds = 0, any = 0;
      for (int k = 0; k < kTraceKinds; ++k) kinds += active[k] > 0, any += active[k];
      const bool mine = kind < 0 ? any > 0 : active[kind] > 0;
      if (mine) {
        busy += dt;
        share += kind < 0 ? dt : dt / kinds;
      }
    }
    prev = e.first;
    const Iv& x = iv[std::abs(e.second) - 1];
    active[x.kind] += e.second > 0 ? 1 : -1;
  }
  if (busy_ms) *busy_ms = busy;
  if (share_ms) *share_ms = share;
  return EGPU_OK;
}

int egpu_trace_events(egpu_handle h, int max, int* kind, int* stream_tag, double* start_ms, double* dur_ms) {
  TRY(check_handle(h));
  Enter g(h);
  const int n = (int)h->trace.recs.size();
  if (n == 0) return 0;
  const cudaEvent_t base = h->trace.recs[0].e0;
  for (int i = 0; i < n && i < max; ++i) {
    const auto& r = h->trace.recs[i];
    EGPU_CUDA_TRY(cudaEventSynchronize(r.e1));
    float t0 = 0, t = 0;
    EGPU_CUDA_TRY(cudaEventElapsedTime(&t0, base, r.e0));
    EGPU_CUDA_TRY(cudaEventElapsedTime(&t, r.e0, r.e1));
    if (kind) kind[i] = r.kind;
    if (stream_tag) stream_tag[i] = r.st == h->stream ? 0 : r.st == h->side ? 1 : r.st == h->aux ? 2 : 3;
    if (start_ms) start_ms[i] = t0;
    if (dur_ms) dur_ms[i] = t;
  }
  return n;
}

const char* egpu_error_string(int code) {
  switch (code) {
    case EGPU_OK: return "ok";
    case EGPU_NOT_HPD: return "A was not numerically HPD";
    case EGPU_SINGULAR: return "Matrix was singular";
    case EGPU_TIMEOUT: return "device-side wait timed out";
    case EGPU_ERR_ARG: return "invalid argument";
    case EGPU_ERR_CUDA: return "CUDA error";
    case EGPU_ERR_ALLOC: return "device allocation failed";
    case EGPU_ERR_ALIGN: return "operand not 16-byte aligned";
    case EGPU_ERR_TMA: return "tensor-map encoding failed";
    case EGPU_ERR_UNSUPPORTED: return "unsupported size";
    case EGPU_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown";
  }
}

const char* egpu_last_error_detail(void) { return t_last_error.c_str(); }

// ---------------------------------------------------------- device API --

int egpu_dpotrf(egpu_handle h, int uplo, int n, double* dA, int lda, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || (uplo != EGPU_LOWER && uplo != EGPU_UPPER) || bad_ld(lda, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  Operand A = make_op(dA, lda, n, n);
  TRY(pack(h, 0, A, true));
  TRY(reset_status(h));
  TRY(potrf_core(h, uplo, n, A.ptr, A.ld));
  TRY(unpack(h, A));
  return read_status(h, info);
}

int egpu_dpotrs(egpu_handle h, int uplo, int orient, int n, int nrhs, const double* dA, int lda, double* dB,
                int ldb) {
  TRY(check_handle(h));
  if (n < 0 || nrhs < 0 || bad_ld(lda, n) || bad_ld(ldb, n)) return EGPU_ERR_ARG;
  if (n == 0 || nrhs == 0) return EGPU_OK;
  (void)orient;
  Enter g(h);
  Operand A = make_op(const_cast<double*>(dA), lda, n, n), B = make_op(dB, ldb, n, nrhs);
  TRY(pack(h, 0, A, true));
  TRY(pack(h, 1, B, true));
  TRY(reset_status(h));
  TRY(potrs_core(h, uplo, n, nrhs, A.ptr, A.ld, B.ptr, B.ld));
  TRY(unpack(h, B));
  return read_status(h, nullptr);
}

int egpu_dposv(egpu_handle h, int uplo, int orient, int n, int nrhs, double* dA, int lda, double* dB, int ldb,
               int* info) {
  int rc = egpu_dpotrf(h, uplo, n, dA, lda, info);
  if (rc != EGPU_OK) return rc;
  return egpu_dpotrs(h, uplo, orient, n, nrhs, dA, lda, dB, ldb);
}

int egpu_dgetrf(egpu_handle h, int m, int n, double* dA, int lda, int* dp, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (m < 0 || n < 0 || bad_ld(lda, m) || (!dp && std::min(m, n) > 0)) return EGPU_ERR_ARG;
  if (m == 0 || n == 0) return EGPU_OK;
  Enter g(h);
  Operand A = make_op(dA, lda, m, n);
  TRY(pack(h, 0, A, true));
  TRY(reset_status(h));
  TRY(getrf_core(h, m, n, A.ptr, A.ld, dp));
  TRY(unpack(h, A));
  return read_status(h, info);
}

int egpu_dgetrf_nopiv(egpu_handle h, int m, int n, double* dA, int lda, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (m < 0 || n < 0 || bad_ld(lda, m)) return EGPU_ERR_ARG;
  if (m == 0 || n == 0) return EGPU_OK;
  Enter g(h);
  Operand A = make_op(dA, lda, m, n);
  TRY(pack(h, 0, A, true));
  TRY(reset_status(h));
  TRY(getrf_nopiv_core(h, m, n, A.ptr, A.ld));
  TRY(unpack(h, A));
  return read_status(h, info);
}

int egpu_dgetrs(egpu_handle h, int orient, int n, int nrhs, const double* dA, int lda, const int* dp, double* dB,
                int ldb) {
  TRY(check_handle(h));
  if (n < 0 || nrhs < 0 || bad_ld(lda, n) || bad_ld(ldb, n)) return EGPU_ERR_ARG;
  if (n == 0 || nrhs == 0) return EGPU_OK;
  Enter g(h);
  Operand A = make_op(const_cast<double*>(dA), lda, n, n), B = make_op(dB, ldb, n, nrhs);
  TRY(pack(h, 0, A, true));
  TRY(pack(h, 1, B, true));
  TRY(reset_status(h));
  TRY(getrs_core(h, orient == EGPU_NORMAL ? EGPU_NORMAL : EGPU_TRANSPOSE, n, nrhs, A.ptr, A.ld, dp, B.ptr, B.ld));
  TRY(unpack(h, B));
  return read_status(h, nullptr);
}

int egpu_dgesv(egpu_handle h, int n, int nrhs, double* dA, int lda, double* dB, int ldb, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || nrhs < 0 || bad_ld(lda, n) || bad_ld(ldb, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  Operand A = make_op(dA, lda, n, n), B = make_op(dB, ldb, n, std::max(nrhs, 1));
  B.cols = nrhs;
  TRY(pack(h, 0, A, true));
  if (nrhs > 0) TRY(pack(h, 1, B, true));
  TRY(reset_status(h));
  int rc = gesv_core(h, n, nrhs, A.ptr, A.ld, B.ptr, B.ld);
  if (rc < 0) return rc;
  TRY(unpack(h, A));
  if (nrhs > 0) TRY(unpack(h, B));
  int rc2 = read_status(h, info);
  return rc != EGPU_OK ? rc : rc2;
}

int egpu_dposv_batched(egpu_handle h, int count, const int* n, const int* nrhs, double* const* dA, const int* lda,
                       double* const* dB, const int* ldb, int* info) {
  TRY(check_handle(h));
  if (count < 0 || (count > 0 && (!n || !nrhs || !dA || !lda || !info))) return EGPU_ERR_ARG;
  if (count == 0) return EGPU_OK;
  Enter g(h);
  TRY(ensure_ws(h, egpu_batched_ws_bytes(count, h->sm_count) + 4096));
  return egpu_batched_launch(0, h->stream, h->sm_count, count, n, nrhs, dA, lda, dB, ldb, h->ws, h->ws_bytes,
                             info);
}

// ---- batch plans (device-resident batched solves, capturable runs) ----
struct egpu_batch_plan_s {
  egpu_context* h;
  egpu::BatchPlan* p;
};

int egpu_batch_plan_create_ex(egpu_handle h, int kind, int precision, int count, const int* n, const int* nrhs,
                              double* const* dA, const int* lda, double* const* dB, const int* ldb,
                              egpu_batch_plan* out) {
  TRY(check_handle(h));
  if (!out || (kind != 0 && kind != 1) || (precision != 0 && precision != 1) || count < 0 ||
      (count > 0 && (!n || !nrhs || !dA || !lda)))
    return EGPU_ERR_ARG;
  *out = nullptr;
  Enter g(h);
  egpu::BatchPlan* p = nullptr;
  TRY(egpu::batch_plan_create(h->device, h->sm_count, kind, precision, count, n, nrhs, dA, lda, dB, ldb, &p));
  auto* w = new (std::nothrow) egpu_batch_plan_s{h, p};
  if (!w) {
    egpu::batch_plan_destroy(p);
    return EGPU_ERR_ALLOC;
  }
  *out = w;
  return EGPU_OK;
}

int egpu_batch_plan_create(egpu_handle h, int kind, int count, const int* n, const int* nrhs, double* const* dA,
                           const int* lda, double* const* dB, const int* ldb, egpu_batch_plan* out) {
  return egpu_batch_plan_create_ex(h, kind, 0, count, n, nrhs, dA, lda, dB, ldb, out);
}

int egpu_batch_plan_iters(egpu_batch_plan plan, void* stream, int* iters) {
  if (!plan || !iters) return EGPU_ERR_ARG;
  Enter g(plan->h);
  return egpu::batch_plan_iters(plan->p, stream ? static_cast<cudaStream_t>(stream) : plan->h->stream, iters);
}

int egpu_batch_plan_shape(egpu_batch_plan plan, int* nclass, int* class_nmax, int* panel, int* threads, int* grid) {
  if (!plan) return EGPU_ERR_ARG;
  return egpu::batch_plan_shape(plan->p, nclass, class_nmax, panel, threads, grid);
}

int egpu_batch_plan_run(egpu_batch_plan plan, void* stream) {
  if (!plan) return EGPU_ERR_ARG;
  Enter g(plan->h);
  return egpu::batch_plan_run(plan->p, stream ? static_cast<cudaStream_t>(stream) : plan->h->stream);
}

int egpu_batch_plan_info(egpu_batch_plan plan, void* stream, int* info) {
  if (!plan || !info) return EGPU_ERR_ARG;
  Enter g(plan->h);
  return egpu::batch_plan_info(plan->p, stream ? static_cast<cudaStream_t>(stream) : plan->h->stream, info);
}

int egpu_batch_plan_autotune(egpu_batch_plan plan, void* stream, int reps, double* best_ms, int* best_grid) {
  if (!plan) return EGPU_ERR_ARG;
  Enter g(plan->h);
  return egpu::batch_plan_autotune(plan->p, stream ? static_cast<cudaStream_t>(stream) : plan->h->stream, reps,
                                   best_ms, best_grid);
}

int egpu_batch_plan_set_grid(egpu_batch_plan plan, int grid) {
  if (!plan || grid < 1) return EGPU_ERR_ARG;
  egpu::batch_plan_set_grid(plan->p, grid);
  return EGPU_OK;
}

int egpu_batch_plan_destroy(egpu_batch_plan plan) {
  if (!plan) return EGPU_OK;
  {
    Enter g(plan->h);
    egpu::batch_plan_destroy(plan->p);
  }
  delete plan;
  return EGPU_OK;
}

int egpu_dgesv_batched(egpu_handle h, int count, const int* n, const int* nrhs, double* const* dA, const int* lda,
                       double* const* dB, const int* ldb, int* info) {
  TRY(check_handle(h));
  if (count < 0 || (count > 0 && (!n || !nrhs || !dA || !lda || !info))) return EGPU_ERR_ARG;
  if (count == 0) return EGPU_OK;
  Enter g(h);
  TRY(ensure_ws(h, egpu_batched_ws_bytes(count, h->sm_count) + 4096));
  return egpu_batched_launch(1, h->stream, h->sm_count, count, n, nrhs, dA, lda, dB, ldb, h->ws, h->ws_bytes,
                             info);
}

int egpu_dtrsm(egpu_handle h, int side, int uplo, int orient, int diag, int m, int n, double alpha,
               const double* dA, int lda, double* dB, int ldb) {
  TRY(check_handle(h));
  const int nt = side == EGPU_LEFT ? m : n;
  if (m < 0 || n < 0 || bad_ld(lda, nt) || bad_ld(ldb, m)) return EGPU_ERR_ARG;
  if (m == 0 || n == 0) return EGPU_OK;
  Enter g(h);
  Operand A = make_op(const_cast<double*>(dA), lda, nt, nt), B = make_op(dB, ldb, m, n);
  TRY(pack(h, 0, A, true));
  TRY(pack(h, 1, B, true));
  TRY(reset_status(h));
  TRY(trsm_core(h, side, uplo, orient != EGPU_NORMAL, diag == EGPU_UNIT, m, n, alpha, A.ptr, A.ld, B.ptr, B.ld));
  TRY(unpack(h, B));
  return read_status(h, nullptr);
}

int egpu_dtrsv(egpu_handle h, int uplo, int orient, int diag, int n, const double* dA, int lda, double* dx) {
  return egpu_dtrsm(h, EGPU_LEFT, uplo, orient, diag, n, 1, 1.0, dA, lda, dx, std::max(n, 1));
}

int egpu_dgemm(egpu_handle h, int oA, int oB, int m, int n, int k, double alpha, const double* dA, int lda,
               const double* dB, int ldb, double beta, double* dC, int ldc) {
  TRY(check_handle(h));
  const bool ta = oA != EGPU_NORMAL, tb = oB != EGPU_NORMAL;
  if (m < 0 || n < 0 || k < 0 || bad_ld(lda, ta ? k : m) || bad_ld(ldb, tb ? n : k) || bad_ld(ldc, m))
    return EGPU_ERR_ARG;
  if (m == 0 || n == 0) return EGPU_OK;
  Enter g(h);
  Operand A = make_op(const_cast<double*>(dA), lda, ta ? k : m, ta ? m : k);
  Operand B = make_op(const_cast<double*>(dB), ldb, tb ? n : k, tb ? k : n);
  TRY(pack(h, 0, A, true));
  TRY(pack(h, 1, B, true));
  TRY(reset_status(h));
  TRY(launch_dgemm(h->stream, ta, !tb, m, n, k, alpha, A.ptr, A.ld, B.ptr, B.ld, beta, dC, ldc, 0, false,
                   h->dstatus));
  return read_status(h, nullptr);
}

int egpu_dherk(egpu_handle h, int uplo, int orient, int n, int k, double alpha, const double* dA, int lda,
               double beta, double* dC, int ldc) {
  TRY(check_handle(h));
  const bool tr = orient != EGPU_NORMAL;
  if (n < 0 || k < 0 || bad_ld(lda, tr ? k : n) || bad_ld(ldc, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  Operand A = make_op(const_cast<double*>(dA), lda, tr ? k : n, tr ? n : k);
  TRY(pack(h, 0, A, true));
  TRY(reset_status(h));
  // NORMAL: C = a A A^T  (op(A) = A MN-major, op(B) = A^T MN-major)
  // ADJOINT: C = a A^T A (op(A) = A^T K-major, op(B) = A K-major)
  TRY(launch_dgemm(h->stream, tr, tr, n, n, k, alpha, A.ptr, A.ld, A.ptr, A.ld, beta, dC, ldc,
                   uplo == EGPU_LOWER ? 1 : 2, false, h->dstatus));
  return read_status(h, nullptr);
}

int egpu_dlaswp(egpu_handle h, int inverse, int m, int n, double* dA, int lda, const int* dp, int npiv) {
  TRY(check_handle(h));
  if (m < 0 || n < 0 || npiv < 0 || npiv > m || bad_ld(lda, m)) return EGPU_ERR_ARG;
  if (m == 0 || n == 0 || npiv == 0) return EGPU_OK;
  Enter g(h);
  TRY(ensure_ws(h, align_up(sizeof(int) * (size_t)((m + 1) & ~1), 256) + sizeof(double) * (size_t)m * n + 4096));
  TRY(launch_laswp_seq(h->stream, inverse, m, n, dA, lda, dp, npiv, static_cast<int*>(h->ws)));
  EGPU_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return EGPU_OK;
}

int egpu_dtrtri(egpu_handle h, int uplo, int diag, int n, double* dA, int lda) {
  TRY(check_handle(h));
  if (n < 0 || (uplo != EGPU_LOWER && uplo != EGPU_UPPER) || bad_ld(lda, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  Operand A = make_op(dA, lda, n, n);
  TRY(pack(h, 0, A, true));
  TRY(reset_status(h));
  TRY(trtri_core(h, uplo, diag == EGPU_UNIT, n, A.ptr, A.ld));
  TRY(unpack(h, A));
  return read_status(h, nullptr);
}

int egpu_dgetri(egpu_handle h, int n, double* dA, int lda, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || bad_ld(lda, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  TRY(ensure_stage(h, 2, sizeof(int) * (size_t)n));
  Operand A = make_op(dA, lda, n, n);
  TRY(pack(h, 0, A, true));
  TRY(reset_status(h));
  int rc = getri_core(h, n, A.ptr, A.ld, info);
  TRY(unpack(h, A));
  TRY(rc);
  return read_status(h, info);
}

int egpu_dpotri(egpu_handle h, int uplo, int n, double* dA, int lda, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || (uplo != EGPU_LOWER && uplo != EGPU_UPPER) || bad_ld(lda, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  Operand A = make_op(dA, lda, n, n);
  TRY(pack(h, 0, A, true));
  TRY(reset_status(h));
  int rc = potri_core(h, uplo, n, A.ptr, A.ld, info);
  TRY(unpack(h, A));
  TRY(rc);
  return read_status(h, info);
}

int egpu_dpotrf_reverse(egpu_handle h, int uplo, int n, double* dA, int lda, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || (uplo != EGPU_LOWER && uplo != EGPU_UPPER) || bad_ld(lda, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  TRY(reset_status(h));
  return reverse_potrf_core(h, uplo, n, dA, lda, info);
}

int egpu_dldl(egpu_handle h, int orient, int n, double* dA, int lda, double* dd, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || orient == EGPU_NORMAL || bad_ld(lda, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  Operand A = make_op(dA, lda, n, n);
  TRY(pack(h, 0, A, true));
  TRY(reset_status(h));
  TRY(ldl_core(h, n, A.ptr, A.ld, dd));
  TRY(unpack(h, A));
  return read_status(h, info);
}

// The determinant's work matrix: A itself when overwrite (factored in place),
// else a copy in staging slot 3.
static int safe_det_device(egpu_handle h, int hpd, int uplo, int n, double* dA, int lda, int overwrite, double* rho,
                           double* kappa) {
  TRY(check_handle(h));
  if (!rho || !kappa || n < 0 || bad_ld(lda, n) || (hpd && uplo != EGPU_LOWER && uplo != EGPU_UPPER))
    return EGPU_ERR_ARG;
  Enter g(h);
  if (n == 0) return safe_det_core(h, hpd, uplo, n, dA, lda, rho, kappa);
  if (overwrite) {
    Operand A = make_op(dA, lda, n, n);
    TRY(pack(h, 0, A, true));
    TRY(safe_det_core(h, hpd, uplo, n, A.ptr, A.ld, rho, kappa));
    TRY(unpack(h, A));
    EGPU_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return EGPU_OK;
  }
  const long long ldw = ld_aligned(n);
  TRY(ensure_stage(h, 3, sizeof(double) * (size_t)ldw * n));
  double* W = static_cast<double*>(h->stage[3]);
  TRY(launch_copy(h->stream, n, n, dA, lda, W, ldw));
  return safe_det_core(h, hpd, uplo, n, W, ldw, rho, kappa);
}

int egpu_dsafe_det(egpu_handle h, int n, double* dA, int lda, int overwrite, double* rho, double* kappa) {
  return safe_det_device(h, 0, EGPU_LOWER, n, dA, lda, overwrite, rho, kappa);
}

int egpu_dsafe_hpd_det(egpu_handle h, int uplo, int n, double* dA, int lda, int overwrite, double* rho,
                       double* kappa) {
  return safe_det_device(h, 1, uplo, n, dA, lda, overwrite, rho, kappa);
}

// ------------------------------------------------------------ host API --
// Copy host column-major buffers into handle staging memory (ld multiple of
// 32), run the device path, copy results back.

static int h2d(egpu_context* h, int slot, const double* src, int lda, int rows, int cols, double** dst,
               long long* ldd) {
  *ldd = ld_aligned(rows);
  TRY(ensure_stage(h, slot, sizeof(double) * (size_t)(*ldd) * std::max(cols, 1)));
  *dst = static_cast<double*>(h->stage[slot]);
  if (rows > 0 && cols > 0)
    EGPU_CUDA_TRY(cudaMemcpy2DAsync(*dst, sizeof(double) * (*ldd), src, sizeof(double) * lda,
                                    sizeof(double) * rows, cols, cudaMemcpyHostToDevice, h->stream));
  return EGPU_OK;
}

static int d2h(egpu_context* h, const double* src, long long ldd, double* dst, int lda, int rows, int cols) {
  if (rows > 0 && cols > 0)
    EGPU_CUDA_TRY(cudaMemcpy2DAsync(dst, sizeof(double) * lda, src, sizeof(double) * ldd, sizeof(double) * rows,
                                    cols, cudaMemcpyDeviceToHost, h->stream));
  return EGPU_OK;
}

static int* stage_ints(egpu_context* h, int slot, size_t count) {
  if (ensure_stage(h, slot, sizeof(int) * std::max<size_t>(count, 1)) != EGPU_OK) return nullptr;
  return static_cast<int*>(h->stage[slot]);
}

int egpu_host_dpotrf(egpu_handle h, int uplo, int n, double* A, int lda, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || bad_ld(lda, n) || (uplo != EGPU_LOWER && uplo != EGPU_UPPER)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double* d; long long ld;
  TRY(h2d(h, 0, A, lda, n, n, &d, &ld));
  TRY(reset_status(h));
  int rc = potrf_core(h, uplo, n, d, ld);
  if (rc < 0) return rc;
  TRY(d2h(h, d, ld, A, lda, n, n));
  return read_status(h, info);
}

int egpu_host_dpotrs(egpu_handle h, int uplo, int orient, int n, int nrhs, const double* A, int lda, double* B,
                     int ldb) {
  TRY(check_handle(h));
  (void)orient;
  if (n < 0 || nrhs < 0 || bad_ld(lda, n) || bad_ld(ldb, n)) return EGPU_ERR_ARG;
  if (n == 0 || nrhs == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double *dA, *dB; long long la, lb;
  TRY(h2d(h, 0, A, lda, n, n, &dA, &la));
  TRY(h2d(h, 1, B, ldb, n, nrhs, &dB, &lb));
  TRY(reset_status(h));
  TRY(potrs_core(h, uplo, n, nrhs, dA, la, dB, lb));
  TRY(d2h(h, dB, lb, B, ldb, n, nrhs));
  return read_status(h, nullptr);
}

// Host-memory form of egpu_dposv_mixed: A and B copied in, X copied out.
int egpu_host_dposv_mixed(egpu_handle h, int uplo, int n, int nrhs, const double* A, int lda, const double* B,
                          int ldb, double* X, int ldx, int max_iter, double tol, int* iters, double* berr) {
  TRY(check_handle(h));
  if (iters) *iters = 0;
  if (berr) *berr = 0.0;
  if (n < 0 || nrhs < 0 || bad_ld(lda, n) || bad_ld(ldb, n) || bad_ld(ldx, n) || max_iter < 0) return EGPU_ERR_ARG;
  if (n == 0 || nrhs == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double *dA, *dB, *dX; long long la, lb, lx;
  TRY(h2d(h, 0, A, lda, n, n, &dA, &la));
  TRY(h2d(h, 1, B, ldb, n, nrhs, &dB, &lb));
  TRY(ensure_stage(h, 2, sizeof(double) * (size_t)lb * nrhs));
  dX = static_cast<double*>(h->stage[2]);
  lx = lb;
  int rc = dposv_mixed_core(h, uplo, n, nrhs, dA, la, dB, lb, dX, lx, max_iter, tol, iters, berr);
  if (rc == EGPU_OK || rc == EGPU_NO_CONVERGENCE) {
    TRY(d2h(h, dX, lx, X, ldx, n, nrhs));
    EGPU_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  return rc;
}

int egpu_host_dposv(egpu_handle h, int uplo, int orient, int n, int nrhs, double* A, int lda, double* B, int ldb,
                    int* info) {
  TRY(check_handle(h));
  (void)orient;
  if (info) *info = 0;
  if (n < 0 || nrhs < 0 || bad_ld(lda, n) || bad_ld(ldb, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double *dA, *dB; long long la, lb;
  TRY(h2d(h, 0, A, lda, n, n, &dA, &la));
  TRY(h2d(h, 1, B, ldb, n, nrhs, &dB, &lb));
  TRY(reset_status(h));
  TRY(potrf_core(h, uplo, n, dA, la));
  int rc = read_status(h, info);
  if (rc == EGPU_OK && nrhs > 0) TRY(potrs_core(h, uplo, n, nrhs, dA, la, dB, lb));
  TRY(d2h(h, dA, la, A, lda, n, n));
  if (rc == EGPU_OK && nrhs > 0) TRY(d2h(h, dB, lb, B, ldb, n, nrhs));
  int rc2 = read_status(h, nullptr);
  return rc != EGPU_OK ? rc : rc2;
}

int egpu_host_dgetrf(egpu_handle h, int m, int n, double* A, int lda, int* p, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (m < 0 || n < 0 || bad_ld(lda, m)) return EGPU_ERR_ARG;
  if (m == 0 || n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double* d; long long ld;
  TRY(h2d(h, 0, A, lda, m, n, &d, &ld));
  const int mn = std::min(m, n);
  int* dp = stage_ints(h, 2, mn);
  if (!dp) return EGPU_ERR_ALLOC;
  TRY(reset_status(h));
  int rc = getrf_core(h, m, n, d, ld, dp);
  if (rc < 0) return rc;
  TRY(d2h(h, d, ld, A, lda, m, n));
  EGPU_CUDA_TRY(cudaMemcpyAsync(p, dp, sizeof(int) * mn, cudaMemcpyDeviceToHost, h->stream));
  return read_status(h, info);
}

int egpu_host_dgetrf_nopiv(egpu_handle h, int m, int n, double* A, int lda, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (m < 0 || n < 0 || bad_ld(lda, m)) return EGPU_ERR_ARG;
  if (m == 0 || n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double* d; long long ld;
  TRY(h2d(h, 0, A, lda, m, n, &d, &ld));
  TRY(reset_status(h));
  int rc = getrf_nopiv_core(h, m, n, d, ld);
  if (rc < 0) return rc;
  TRY(d2h(h, d, ld, A, lda, m, n));
  return read_status(h, info);
}

int egpu_host_dgetrs(egpu_handle h, int orient, int n, int nrhs, const double* A, int lda, const int* p,
                     double* B, int ldb) {
  TRY(check_handle(h));
  if (n < 0 || nrhs < 0 || bad_ld(lda, n) || bad_ld(ldb, n)) return EGPU_ERR_ARG;
  if (n == 0 || nrhs == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double *dA, *dB; long long la, lb;
  TRY(h2d(h, 0, A, lda, n, n, &dA, &la));
  TRY(h2d(h, 1, B, ldb, n, nrhs, &dB, &lb));
  int* dp = nullptr;
  if (p) {
    dp = stage_ints(h, 2, n);
    if (!dp) return EGPU_ERR_ALLOC;
    EGPU_CUDA_TRY(cudaMemcpyAsync(dp, p, sizeof(int) * n, cudaMemcpyHostToDevice, h->stream));
  }
  TRY(reset_status(h));
  TRY(getrs_core(h, orient == EGPU_NORMAL ? EGPU_NORMAL : EGPU_TRANSPOSE, n, nrhs, dA, la, dp, dB, lb));
  TRY(d2h(h, dB, lb, B, ldb, n, nrhs));
  return read_status(h, nullptr);
}

int egpu_host_dgesv(egpu_handle h, int n, int nrhs, double* A, int lda, double* B, int ldb, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || nrhs < 0 || bad_ld(lda, n) || bad_ld(ldb, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double *dA, *dB; long long la, lb;
  TRY(h2d(h, 0, A, lda, n, n, &dA, &la));
  TRY(h2d(h, 1, B, ldb, n, std::max(nrhs, 1), &dB, &lb));
  TRY(reset_status(h));
  int rc = gesv_core(h, n, nrhs, dA, la, dB, lb);
  if (rc < 0) return rc;
  TRY(d2h(h, dA, la, A, lda, n, n));
  if (nrhs > 0) TRY(d2h(h, dB, lb, B, ldb, n, nrhs));
  int rc2 = read_status(h, info);
  return rc != EGPU_OK ? rc : rc2;
}

int egpu_host_dtrsm(egpu_handle h, int side, int uplo, int orient, int diag, int m, int n, double alpha,
                    const double* A, int lda, double* B, int ldb) {
  TRY(check_handle(h));
  const int nt = side == EGPU_LEFT ? m : n;
  if (m < 0 || n < 0 || bad_ld(lda, nt) || bad_ld(ldb, m)) return EGPU_ERR_ARG;
  if (m == 0 || n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double *dA, *dB; long long la, lb;
  TRY(h2d(h, 0, A, lda, nt, nt, &dA, &la));
  TRY(h2d(h, 1, B, ldb, m, n, &dB, &lb));
  TRY(reset_status(h));
  TRY(trsm_core(h, side, uplo, orient != EGPU_NORMAL, diag == EGPU_UNIT, m, n, alpha, dA, la, dB, lb));
  TRY(d2h(h, dB, lb, B, ldb, m, n));
  return read_status(h, nullptr);
}

int egpu_host_dgemm(egpu_handle h, int oA, int oB, int m, int n, int k, double alpha, const double* A, int lda,
                    const double* B, int ldb, double beta, double* C, int ldc) {
  TRY(check_handle(h));
  const bool ta = oA != EGPU_NORMAL, tb = oB != EGPU_NORMAL;
  if (m < 0 || n < 0 || k < 0 || bad_ld(lda, ta ? k : m) || bad_ld(ldb, tb ? n : k) || bad_ld(ldc, m))
    return EGPU_ERR_ARG;
  if (m == 0 || n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double *dA, *dB, *dC; long long la, lb, lc;
  TRY(h2d(h, 0, A, lda, ta ? k : m, ta ? m : k, &dA, &la));
  TRY(h2d(h, 1, B, ldb, tb ? n : k, tb ? k : n, &dB, &lb));
  TRY(h2d(h, 2, C, ldc, m, n, &dC, &lc));
  TRY(reset_status(h));
  TRY(launch_dgemm(h->stream, ta, !tb, m, n, k, alpha, dA, la, dB, lb, beta, dC, lc, 0, false, h->dstatus));
  TRY(d2h(h, dC, lc, C, ldc, m, n));
  return read_status(h, nullptr);
}

int egpu_host_dherk(egpu_handle h, int uplo, int orient, int n, int k, double alpha, const double* A, int lda,
                    double beta, double* C, int ldc) {
  TRY(check_handle(h));
  const bool tr = orient != EGPU_NORMAL;
  if (n < 0 || k < 0 || bad_ld(lda, tr ? k : n) || bad_ld(ldc, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double *dA, *dC; long long la, lc;
  TRY(h2d(h, 0, A, lda, tr ? k : n, tr ? n : k, &dA, &la));
  TRY(h2d(h, 2, C, ldc, n, n, &dC, &lc));
  TRY(reset_status(h));
  TRY(launch_dgemm(h->stream, tr, tr, n, n, k, alpha, dA, la, dA, la, beta, dC, lc, uplo == EGPU_LOWER ? 1 : 2,
                   false, h->dstatus));
  TRY(d2h(h, dC, lc, C, ldc, n, n));
  return read_status(h, nullptr);
}

int egpu_host_dlaswp(egpu_handle h, int inverse, int m, int n, double* A, int lda, const int* p, int npiv) {
  TRY(check_handle(h));
  if (m < 0 || n < 0 || npiv < 0 || npiv > m || bad_ld(lda, m)) return EGPU_ERR_ARG;
  if (m == 0 || n == 0 || npiv == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double* dA; long long la;
  TRY(h2d(h, 0, A, lda, m, n, &dA, &la));
  int* dp = stage_ints(h, 2, npiv);
  if (!dp) return EGPU_ERR_ALLOC;
  EGPU_CUDA_TRY(cudaMemcpyAsync(dp, p, sizeof(int) * npiv, cudaMemcpyHostToDevice, h->stream));
  TRY(ensure_ws(h, align_up(sizeof(int) * (size_t)((m + 1) & ~1), 256) + sizeof(double) * (size_t)m * n + 4096));
  TRY(launch_laswp_seq(h->stream, inverse, m, n, dA, la, dp, npiv, static_cast<int*>(h->ws)));
  TRY(d2h(h, dA, la, A, lda, m, n));
  EGPU_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return EGPU_OK;
}

int egpu_host_dtrtri(egpu_handle h, int uplo, int diag, int n, double* A, int lda) {
  TRY(check_handle(h));
  if (n < 0 || (uplo != EGPU_LOWER && uplo != EGPU_UPPER) || bad_ld(lda, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double* d; long long ld;
  TRY(h2d(h, 0, A, lda, n, n, &d, &ld));
  TRY(reset_status(h));
  TRY(trtri_core(h, uplo, diag == EGPU_UNIT, n, d, ld));
  TRY(d2h(h, d, ld, A, lda, n, n));
  return read_status(h, nullptr);
}

int egpu_host_dgetri(egpu_handle h, int n, double* A, int lda, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || bad_ld(lda, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double* d; long long ld;
  TRY(h2d(h, 0, A, lda, n, n, &d, &ld));
  if (!stage_ints(h, 2, n)) return EGPU_ERR_ALLOC;
  TRY(reset_status(h));
  int rc = getri_core(h, n, d, ld, info);
  if (rc < 0) return rc;
  TRY(d2h(h, d, ld, A, lda, n, n));
  TRY(rc);
  return read_status(h, info);
}

int egpu_host_dpotri(egpu_handle h, int uplo, int n, double* A, int lda, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || (uplo != EGPU_LOWER && uplo != EGPU_UPPER) || bad_ld(lda, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double* d; long long ld;
  TRY(h2d(h, 0, A, lda, n, n, &d, &ld));
  TRY(reset_status(h));
  int rc = potri_core(h, uplo, n, d, ld, info);
  if (rc < 0) return rc;
  TRY(d2h(h, d, ld, A, lda, n, n));
  TRY(rc);
  return read_status(h, info);
}

int egpu_host_dldl(egpu_handle h, int orient, int n, double* A, int lda, double* d, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || orient == EGPU_NORMAL || bad_ld(lda, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double* dA; long long ld;
  TRY(h2d(h, 0, A, lda, n, n, &dA, &ld));
  TRY(ensure_stage(h, 2, sizeof(double) * (size_t)n));
  double* dd = static_cast<double*>(h->stage[2]);
  TRY(reset_status(h));
  int rc = ldl_core(h, n, dA, ld, dd);
  if (rc < 0) return rc;
  TRY(d2h(h, dA, ld, A, lda, n, n));
  if (d) EGPU_CUDA_TRY(cudaMemcpyAsync(d, dd, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  return read_status(h, info);
}

int egpu_host_dpotrf_reverse(egpu_handle h, int uplo, int n, double* A, int lda, int* info) {
  TRY(check_handle(h));
  if (info) *info = 0;
  if (n < 0 || (uplo != EGPU_LOWER && uplo != EGPU_UPPER) || bad_ld(lda, n)) return EGPU_ERR_ARG;
  if (n == 0) return EGPU_OK;
  Enter g(h);
  SyncScope ss(h);
  double* d; long long ld;
  TRY(h2d(h, 0, A, lda, n, n, &d, &ld));
  TRY(reset_status(h));
  int rc = reverse_potrf_core(h, uplo, n, d, ld, info);
  if (rc < 0) return rc;
  TRY(d2h(h, d, ld, A, lda, n, n));
  EGPU_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return rc;
}

static int safe_det_host(egpu_handle h, int hpd, int uplo, int n, double* A, int lda, int overwrite, double* rho,
                         double* kappa) {
  TRY(check_handle(h));
  if (!rho || !kappa || n < 0 || bad_ld(lda, n) || (hpd && uplo != EGPU_LOWER && uplo != EGPU_UPPER))
    return EGPU_ERR_ARG;
  Enter g(h);
  SyncScope ss(h);
  double* d = nullptr; long long ld = 1;
  if (n > 0) TRY(h2d(h, 0, A, lda, n, n, &d, &ld));
  TRY(safe_det_core(h, hpd, uplo, n, d, ld, rho, kappa));
  if (overwrite && n > 0) {  // canOverwrite: A receives the factorization
    TRY(d2h(h, d, ld, A, lda, n, n));
    EGPU_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  return EGPU_OK;
}

int egpu_host_dsafe_det(egpu_handle h, int n, double* A, int lda, int overwrite, double* rho, double* kappa) {
  return safe_det_host(h, 0, EGPU_LOWER, n, A, lda, overwrite, rho, kappa);
}

int egpu_host_dsafe_hpd_det(egpu_handle h, int uplo, int n, double* A, int lda, int overwrite, double* rho,
                            double* kappa) {
  return safe_det_host(h, 1, uplo, n, A, lda, overwrite, rho, kappa);
}

}  // extern "C"
