// Internal declarations shared by the .cu translation units.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>

#include "../../include/elemgpu.h"
#include "common.cuh"

namespace egpu {

void set_last_error(cudaError_t e, const char* what, const char* file, int line);

// Process-wide count of kernel launches issued by this library.
void count_launch(int n = 1);

bool tma_compatible(const void* p, long long ld);

// ---- launch tracing (per-kernel-class CUDA-event timing on the launch stream)
enum TraceKind { kTraceUpdate = 0, kTraceTrsm = 1, kTraceDiag = 2, kTracePanel = 3, kTraceSwap = 4,
                 kTraceOther = 5, kTraceTc = 6, kTraceSolve = 7, kTraceKinds = 8 };
struct Trace;
// Records an event pair around one launch when the calling thread has an
// active trace; no-op otherwise.
struct TraceMark {
  Trace* t = nullptr;
  int idx = -1;
  cudaStream_t st = nullptr;
  TraceMark(cudaStream_t s, int kind, double flops, double bytes);
  ~TraceMark();
};

int launch_dgemm(cudaStream_t st, bool a_kmajor, bool b_kmajor, int M, int N, int K, double alpha,
                 const double* A, long long lda, const double* B, long long ldb, double beta, double* C,
                 long long ldc, int tri, bool wide, DevStatus* status);
int launch_scale(cudaStream_t st, int M, int N, double beta, double* C, long long ldc, int tri);

// 2-D TMA tensor map (dtype: a CUtensorMapDataType value) over `outer` rows of
// `inner` contiguous elements, rows ld_bytes apart.
bool make_tma_2d(CUtensorMap* m, int dtype, const void* base, uint64_t inner, uint64_t outer, uint64_t ld_bytes,
                 uint32_t box_inner, uint32_t box_outer, bool swz128);

// tcgen05 TF32 GEMM: C (FP32, col-major) = alpha * sum_t A_t B_t^T + beta * C,
// A_t (M x K) and B_t (N x K) K-major FP32 buffers (row stride ldk elements,
// ldk % 4 == 0, 16-byte aligned) holding TF32 values; terms 1 uses (Ahi, Bhi),
// terms 3 adds (Ahi, Blo) and (Alo, Bhi).  tri 1: only r >= c is written (M >= N).
// Sh/Sl (optional): also the TF32 hi/lo split of the result's rows r >= srow0,
// K-major with row stride sldk (% 32 == 0), columns [0, swidth) (zero past N;
// N <= swidth <= sldk), 16-byte aligned; the A buffers may be the same rows.
int launch_tc_gemm(cudaStream_t st, int M, int N, int K, float alpha, const float* Ahi, const float* Alo,
                   const float* Bhi, const float* Blo, long long ldk, float beta, float* C, long long ldc, int tri,
                   int terms, DevStatus* status, float* Sh = nullptr, float* Sl = nullptr, long long sldk = 0,
                   int srow0 = 0, int swidth = 0);

// X (rows x cols, column-major FP64) -> TF32 hi/lo parts in K-major rows
// (hi[r*ldk + c], row stride ldk), columns cols..width-1 zero (width: ldk
// when negative).
int launch_split_tf32(cudaStream_t st, int rows, int cols, const double* X, long long ldx, float* hi, float* lo,
                      long long ldk, int width = -1);
// The same from a column-major FP32 X (width ldk).
int launch_split_tf32_f32(cudaStream_t st, int rows, int cols, const float* X, long long ldx, float* hi, float* lo,
                          long long ldk);

// X := inv(T) X for nrhs <= 64 in one cooperative launch (trsm_skinny.cu:
// amode/bwd select T from the stored triangle A, Winv the inverted diagonal
// blocks).  flags: ceil(n/nb) ints that hold values other than `epoch`.
// Y != NULL selects a prescaled A: column-prescaled (X: b in, z out; Y :=
// inv(T_rr) z_r) or, with row_prescaled, row-prescaled (Y: b in, X := x).
// Returns EGPU_ERR_UNSUPPORTED when the shape or alignment does not fit.
size_t trsm_skinny_flag_bytes(int n, int nb);
int launch_trsm_skinny(cudaStream_t st, int bwd, int amode, int n, int nrhs, const double* A, long long lda,
                       const double* Winv, int nb, double* X, long long ldx, int* flags, int epoch, int sm_count,
                       DevStatus* status, double* Y = nullptr, bool row_prescaled = false);

// C += alpha A B for N <= 64 (split-K DMMA, FP64 atomics into C); A, B
// 16-byte aligned with even leading dimensions, else EGPU_ERR_UNSUPPORTED.
int launch_dgemm_skinny(cudaStream_t st, int M, int N, int K, double alpha, const double* A, long long lda,
                        const double* B, long long ldb, double* C, long long ldc, int sm_count, DevStatus* status);

// ---- iterative-refinement helpers shared by the mixed solvers (mixed.cu) --
constexpr int kGmresRestart = 20;  // Krylov vectors per GMRES cycle
struct GmresWork {
  double* V;      // kGmresRestart + 1 basis blocks of lds x nrhs
  double* W;      // work block
  double* coef;   // (kGmresRestart + 2) x nrhs device coefficients
  double* dots;   // device scratch for dot products ((kGmresRestart + 1) x nrhs)
};
// apply_a(V, W): W := A V (n x nrhs blocks, ld lds); precond(W): W := M^-1 W.
using BlockOp = std::function<int(const double*, double*)>;
using BlockSolve = std::function<int(double*)>;
// One GMRES-IR correction: GMRES on M^-1 A d = M^-1 r (one basis per
// right-hand side, advanced in lockstep); R is consumed, D receives d.
int gmres_correction(egpu_context* h, int n, int nrhs, long long lds, const BlockOp& apply_a,
                     const BlockSolve& precond, double* R, double* D, GmresWork& gw, double inner_tol,
                     int* inner_iters);
// 1-norm condition estimate (Hager / Higham): solve(V, trans) applies A^-1
// (trans 0) or A^-T (trans 1) to one device column V.
int cond1_estimate(egpu_context* h, int n, const std::function<int(double*, int)>& solve, double anorm, double* V,
                   double* kappa);
// Normwise backward error max_j ||r_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf);
// norms: device scratch of 3 nrhs doubles.  Synchronizes.
int mixed_berr(egpu_context* h, int n, int nrhs, const double* R, const double* Xw, const double* B, long long ldb,
               long long lds, double anorm, double* norms, double* berr);
// Y (n x ncols) := X, or += X when add.
int launch_copy_cols(cudaStream_t st, int n, int ncols, const double* X, long long ldx, double* Y, long long ldy,
                     int add);

// FP32 super-block sweeps (sweep32.cu), the correction solves of the mixed
// refinement: sweep32_prepare builds the inverses of the 512 x 512 diagonal
// super-blocks of the lower factor L (FP32, ld ldl) from the 128 x 128 panel
// inverses Winv (FP64, nb = 128); sweep32_solve then applies X := L^-1 X
// (trans 0), L^-T X (trans 1) or L^-T L^-1 X (trans 2) to X (FP64, n x nrhs)
// in one cooperative launch.  ws: sweep32_ws_bytes(n, nrhs) bytes, 256-byte
// aligned.
size_t sweep32_ws_bytes(int n, int nrhs);
int sweep32_prepare(cudaStream_t st, int n, const float* L, long long ldl, const double* Winv, void* ws);
int sweep32_solve(cudaStream_t st, int trans, int n, int nrhs, const float* L, long long ldl, double* X,
                  long long ldx, void* ws, int sm_count, DevStatus* status);

// Diagonal-block Cholesky (factor in place + triangular inverse into W).
int launch_potrf_diag(cudaStream_t st, int uplo, double* A, long long lda, int b, double* W, int ldw,
                      DevStatus* status, int col_base, bool store_factor = true);
// The mixed path's diagonal block: lower Cholesky of the FP32 b x b block at
// Af (computed in FP64), its inverse into W (FP64, zero-padded ldw x ldw
// slot) and the TF32 hi/lo split of that inverse in row-major 128 x ldk form
// (Wh[j*ldk + k] = inv(L)[j][k], zero outside b x b): the K-major B operand
// of L21 = A21 inv(L)^T on the tensor cores.
int launch_potrf_diag_f32(cudaStream_t st, const float* Af, long long ldf, int b, double* W, int ldw, float* Wh,
                          float* Wl, long long ldk, DevStatus* status, int col_base);

// Batched triangular inverse of `count` diagonal blocks of size b (the last
// one may be smaller: n total), block i at A + i*b*(lda+1), into W + i*b*ldw.
int launch_trtri_blocks(cudaStream_t st, int uplo, int unit, const double* A, long long lda, int n, int b,
                        double* W, int ldw);

// LU panel: factor the m x b panel at A in place with partial pivoting;
// p (device, b entries) receives absolute rows (offset added); image/preimage
// (device, b entries each) receive the composed permutation; W receives
// inv(unit-lower L11).  scratch: see lu_panel_scratch_bytes.
size_t lu_panel_scratch_bytes(int m, int b, int sm_count);
int launch_lu_panel(cudaStream_t st, int m, int b, double* A, long long lda, int* p, int offset, int* image,
                    int* preimage, double* W, int ldw, void* scratch, DevStatus* status, int sm_count);

// Register-resident cluster form of the LU panel (m <= 16384); returns
// EGPU_ERR_UNSUPPORTED when it does not apply.
int launch_lu_panel_rp(cudaStream_t st, int m, int b, double* A, long long lda, int* p, int offset, int* image,
                       int* preimage, double* W, int ldw, DevStatus* status, int cluster_max);

// Apply composed panel pivots (image/preimage of b rows) to columns of the
// m-row block A (ld lda), columns [0, ncols).
int launch_apply_composed(cudaStream_t st, int m, int ncols, double* A, long long lda, int b, const int* image,
                          const int* preimage, const DevStatus* status);

// Apply sequential swaps p[0..np) (absolute rows) to rows of A (m x n).
int launch_laswp_seq(cudaStream_t st, int inverse, int m, int n, double* A, long long lda, const int* p, int np,
                     int* perm_scratch);
// The two halves of it: perm := the sequential swaps composed (row r ends up
// holding original row perm[r]); A := A[perm, :] through tmp (m x n doubles).
int launch_compose_perm(cudaStream_t st, int inverse, int m, const int* p, int np, int* perm);
int launch_permute_rows(cudaStream_t st, int m, int n, const int* perm, double* A, long long lda, double* tmp);

// Unpivoted LU of a b x b diagonal block in place; W receives inv(unit L11),
// W2 receives inv(U11).
int launch_getrf_diag_nopiv(cudaStream_t st, double* A, long long lda, int b, double* W, int ldw, double* W2,
                            DevStatus* status, int col_base);

// Batched (one persistent launch) HPDSolve, lower, n <= 512, nrhs <= 16.
size_t egpu_batched_ws_bytes(int count, int sm_count);
struct BatchPlan;
// precision 0: FP64 (A receives the factor); 1: FP32 working copy + FP64 refinement (A unchanged)
int batch_plan_create(int device, int sm_count, int kind, int precision, int count, const int* n, const int* nrhs,
                      double* const* A, const int* lda, double* const* B, const int* ldb, BatchPlan** out);
int batch_plan_run(BatchPlan* p, cudaStream_t st);
int batch_plan_info(BatchPlan* p, cudaStream_t st, int* info_host);
int batch_plan_iters(BatchPlan* p, cudaStream_t st, int* iters_host);
int batch_plan_shape(BatchPlan* p, int* nclass, int* class_nmax, int* panel, int* threads, int* grid);
int batch_plan_autotune(BatchPlan* p, cudaStream_t st, int reps, double* best_ms, int* best_grid);
void batch_plan_set_grid(BatchPlan* p, int grid);
void batch_plan_destroy(BatchPlan* p);
// kind 0: HPDSolve (lower Cholesky + solve); kind 1: GaussianElimination (LU + solve)
int egpu_batched_launch(int kind, cudaStream_t st, int sm_count, int count, const int* n, const int* nrhs,
                        double* const* A, const int* lda, double* const* B, const int* ldb, void* ws,
                        size_t ws_bytes, int* info_host);

// TriangularInverse / Inverse / Determinant helpers (inverse.cu).
int launch_set_identity(cudaStream_t st, int n, double* X, long long ldx);
// D's uplo triangle (strict: below/above the diagonal only) := S's.
int launch_copy_triangle(cudaStream_t st, int uplo, bool strict, int n, const double* S, long long lds, double* D,
                         long long ldd);
// D[n-1-i, n-1-j] := S[i, j] over S's uplo triangle.
int launch_rotate_triangle(cudaStream_t st, int uplo, int n, const double* S, long long lds, double* D,
                           long long ldd);
// LDL diagonal blocks: the symmetric b x b block from A11's lower triangle;
// and back: A11's strict lower := L, diagonal (and d) := D from an L\U block.
int launch_sym_from_lower(cudaStream_t st, int b, const double* A, long long lda, double* Blk, long long ldb);
int launch_ldl_block_writeback(cudaStream_t st, int b, const double* Blk, long long ldb, double* A, long long lda,
                               double* d);
// out[0..2] = sum log|a_ii|, count of a_ii < 0, count of p[i] != i (p may be
// null); one deterministic block reduction.
int launch_diag_logsum(cudaStream_t st, int n, const double* A, long long lda, const int* p, double* out);

// Copy between strided device matrices.
int launch_copy(cudaStream_t st, int m, int n, const double* src, long long lds, double* dst, long long ldd);

}  // namespace egpu
