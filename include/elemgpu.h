/*
 * elemgpu.h -- C ABI of the B200 (sm_100a) factor-and-solve library.
 *
 * Plain pointers and sizes only.  Matrices are column-major with a leading
 * dimension, indices 0-based, exactly as Elemental's Matrix<F> stores them
 * (core/matrix.hpp:16-183; ldim = max(height,1), src/core/matrix.cpp:76).
 * Pivot vectors follow Elemental's convention: p[i] is the absolute 0-based
 * row swapped with row i at step i (lapack-like/LU/Panel.hpp:64).
 *
 * Two families of entry points:
 *   egpu_d*      operate on DEVICE memory (the matrix stays resident in HBM);
 *                they run on the handle's stream.
 *   egpu_host_d* operate on HOST buffers (the Matrix<F> drop-in path): copy
 *                in, run, copy out, synchronize.
 *
 * Return value: EGPU_OK, a factorization status (EGPU_NOT_HPD,
 * EGPU_SINGULAR, EGPU_TIMEOUT; *info = 1-based global column), or a negative
 * error.  The C++ layer (elemgpu/elemental.hpp) maps the statuses to
 * Elemental's exceptions: std::logic_error("A was not numerically HPD")
 * (Cholesky/LVar3.hpp:37-38) and SingularMatrixException (LU/Panel.hpp:76-77).
 *
 * Enum values equal Elemental's (core/types_decl.hpp:104-155).
 */
#ifndef ELEMGPU_H
#define ELEMGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ---- */
#define EGPU_OK 0
#define EGPU_NOT_HPD 1    /* non-positive pivot in Cholesky */
#define EGPU_SINGULAR 2   /* exact zero pivot in LU */
#define EGPU_TIMEOUT 3    /* a bounded device-side wait ran out */
#define EGPU_NO_CONVERGENCE 4  /* refinement stopped above its tolerance (result still written) */
#define EGPU_ERR_ARG (-1)
#define EGPU_ERR_CUDA (-2)
#define EGPU_ERR_ALLOC (-3)
#define EGPU_ERR_ALIGN (-4)
#define EGPU_ERR_TMA (-5)
#define EGPU_ERR_UNSUPPORTED (-6)
#define EGPU_ERR_NO_DEVICE (-7)

/* ---- enums (Elemental core/types_decl.hpp) ---- */
#define EGPU_LOWER 0       /* UpperOrLower */
#define EGPU_UPPER 1
#define EGPU_NORMAL 0      /* Orientation */
#define EGPU_TRANSPOSE 1
#define EGPU_ADJOINT 2
#define EGPU_LEFT 0        /* LeftOrRight */
#define EGPU_RIGHT 1
#define EGPU_NON_UNIT 0    /* UnitOrNonUnit */
#define EGPU_UNIT 1

#if defined(__GNUC__)
#define EGPU_API __attribute__((visibility("default")))
#else
#define EGPU_API
#endif

typedef struct egpu_context* egpu_handle;

/* ---- handle ---- */
/* One handle per host thread; it owns a stream, side streams for look-ahead
 * and a device workspace.  Replaces the reference's global environment
 * (elem::Initialize, core/environment_decl.hpp:16-38). */
EGPU_API int egpu_create(egpu_handle* h, int device);
EGPU_API int egpu_destroy(egpu_handle h);
/* Use an external cudaStream_t (NULL restores the handle's own stream;
 * cudaStreamLegacy, 0x1, selects the legacy default stream). */
EGPU_API int egpu_set_stream(egpu_handle h, void* cuda_stream);
EGPU_API void* egpu_get_stream(egpu_handle h);
EGPU_API int egpu_synchronize(egpu_handle h);
/* Algorithmic block size, default 128: elem::SetBlocksize / Blocksize
 * (src/core/global.cpp:277-283; default at :194).  The GPU kernels use it as
 * the panel width; values are rounded to an even number in [2, 128]. */
EGPU_API int egpu_set_blocksize(egpu_handle h, int nb);
EGPU_API int egpu_get_blocksize(egpu_handle h);
/* Panel look-ahead (0 = sequential steps on one stream; 1 = the next panel is
 * factored on a high-priority side stream while the current trailing update
 * runs; G >= 2, Cholesky: the trailing update is applied once per group of G
 * panels (a G*nb-deep product) while the side stream factors the next group's
 * panels, each updated just in time; -1 = default: Cholesky picks G per group
 * from the trailing order (16 above 12288, 8 above 7168, 4 above 5120, 2 above
 * 3072, else 1; the first two groups at most 2 and 8 panels).
 * LU treats any nonzero value as 1; values above 16 are clamped.)  Results
 * agree to rounding. */
EGPU_API int egpu_set_lookahead(egpu_handle h, int depth);
/* Asynchronous mode for the device-memory API: calls only enqueue work on the
 * handle's stream and return EGPU_OK; a failure status (not HPD, singular,
 * timeout) is kept on the device, later kernels of the handle skip their work,
 * and egpu_get_status() waits, returns the first failure and clears it.  Needed
 * for CUDA-graph capture of whole factorizations.  Host-memory calls always
 * synchronize. */
EGPU_API int egpu_set_async(egpu_handle h, int on);
EGPU_API int egpu_get_status(egpu_handle h, int* info);
/* Pre-size the device workspace (bytes) so that later calls allocate nothing. */
EGPU_API int egpu_reserve(egpu_handle h, size_t bytes);
EGPU_API const char* egpu_error_string(int code);
/* Text of the last CUDA error seen by this thread (or ""). */
EGPU_API const char* egpu_last_error_detail(void);
/* Number of kernel launches issued by this library so far (process-wide). */
EGPU_API long long egpu_launch_count(egpu_handle h);

/* Launch tracing (the role of the reference's CallStackEntry/Timer,
 * core/environment_decl.hpp:260-272, core/timer_decl.hpp:15-34): when on,
 * every kernel launch issued through this handle is bracketed by CUDA events
 * on its own stream.  Kinds: 0 trailing update (Gemm/Herk), 1 triangular
 * multiply by an inverted diagonal block (Trsm), 2 diagonal-block kernels,
 * 3 LU panel, 4 row interchanges, 5 other (batched kernels, conversions),
 * 6 tcgen05 tensor-core updates, 7 one-launch solve sweeps.  enable() clears the records;
 * summary() waits for the recorded launches and sums their per-launch device
 * times (start-to-end on each launch's own stream), algorithmic flops and
 * algorithmic bytes. */
EGPU_API int egpu_trace_enable(egpu_handle h, int on);
EGPU_API int egpu_trace_summary(egpu_handle h, int kind, double* total_ms, double* total_flops,
                                double* total_bytes, long long* launches);
/* Device time of one launch kind (-1: any kind) on one time axis, the
 * concurrent streams merged: *busy_ms = the time during which at least one
 * traced launch of that kind was in flight (the union of the launches'
 * intervals; with kind -1 the traced region's busy time); *share_ms = that
 * time with every moment split evenly among the kinds in flight, so the
 * shares of all kinds add up to the busy time of kind -1.  Sums of per-launch
 * durations (egpu_trace_summary) count overlapped launches twice. */
EGPU_API int egpu_trace_busy(egpu_handle h, int kind, double* busy_ms, double* share_ms);
/* The traced launches in order: kind (as egpu_trace_summary), stream (0 the
   handle's stream, 1 the look-ahead side stream, 2 the lowest-priority
   auxiliary stream, 3 another), start relative to the first traced launch
   and duration, both in ms.  Fills at most `max` entries; returns the number
   of traced launches (or a negative error code). */
EGPU_API int egpu_trace_events(egpu_handle h, int max, int* kind, int* stream_tag, double* start_ms,
                               double* dur_ms);

/* ---- device-memory API ---- */

/* Cholesky(uplo, Matrix<F>& A), lapack-like/Cholesky.hpp:49-62 (blocked
 * right-looking LVar3 / UVar3, Cholesky/LVar3.hpp:83-123,
 * Cholesky/UVar3.hpp:85-125).  Only the uplo triangle is read and written. */
EGPU_API int egpu_dpotrf(egpu_handle h, int uplo, int n, double* dA, int lda, int* info);

/* cholesky::SolveAfter(uplo, orientation, A, B),
 * lapack-like/Cholesky/SolveAfter.hpp:20-75. */
EGPU_API int egpu_dpotrs(egpu_handle h, int uplo, int orient, int n, int nrhs, const double* dA, int lda, double* dB,
                int ldb);

/* HPDSolve(uplo, orientation, A, B), lapack-like/HPDSolve.hpp:18-28. */
EGPU_API int egpu_dposv(egpu_handle h, int uplo, int orient, int n, int nrhs, double* dA, int lda, double* dB, int ldb,
               int* info);

/* LU(Matrix<F>& A, Matrix<int>& p), lapack-like/LU.hpp:144-218.
 * dp: device int32[min(m,n)]. */
EGPU_API int egpu_dgetrf(egpu_handle h, int m, int n, double* dA, int lda, int* dp, int* info);

/* LU(Matrix<F>& A) without pivoting, lapack-like/LU.hpp:36-74. */
EGPU_API int egpu_dgetrf_nopiv(egpu_handle h, int m, int n, double* dA, int lda, int* info);

/* lu::SolveAfter(orientation, A, p, B), lapack-like/LU/SolveAfter.hpp:101-146;
 * dp == NULL selects the unpivoted overload (:20-57). */
EGPU_API int egpu_dgetrs(egpu_handle h, int orient, int n, int nrhs, const double* dA, int lda, const int* dp,
                double* dB, int ldb);

/* GaussianElimination(A, B), lapack-like/GaussianElimination.hpp:216-232. */
EGPU_API int egpu_dgesv(egpu_handle h, int n, int nrhs, double* dA, int lda, double* dB, int ldb, int* info);

/* Batch plans: a batched HPD solve (kind 0, as egpu_dposv_batched) or
 * GaussianElimination (kind 1, as egpu_dgesv_batched) whose size-sorted
 * system list, queue and scratch stay on the device, so that a run is a
 * counter reset plus one persistent launch per size class, with no host
 * synchronisation (a CUDA graph can capture
 * and replay it; the device pointers are fixed at creation: refill the
 * matrices in place between runs).  egpu_batch_plan_autotune chooses the
 * launch shape: for the whole list and for each size class (n <= 128,
 * <= 256, <= 512) it times the candidate panel widths (16, 32), CTA sizes
 * (128, 256 threads: one or two CTAs per SM) and persistent grids on the
 * plan's own systems -- restoring every input from a backup before each run
 * and once more at the end -- and keeps the faster of the best single launch
 * and the best launch per class (*best_grid: the first class's grid);
 * egpu_batch_plan_info copies the
 * per-system info of the last run to the host and synchronises.  A plan
 * belongs to the handle that made it and must be destroyed before it.
 * No counterpart in the reference (it solves one system per call). */
typedef struct egpu_batch_plan_s* egpu_batch_plan;
EGPU_API int egpu_batch_plan_create(egpu_handle h, int kind, int count, const int* n, const int* nrhs,
                                    double* const* dA, const int* lda, double* const* dB, const int* ldb,
                                    egpu_batch_plan* out);
EGPU_API int egpu_batch_plan_run(egpu_batch_plan plan, void* stream);
EGPU_API int egpu_batch_plan_info(egpu_batch_plan plan, void* stream, int* info);
EGPU_API int egpu_batch_plan_autotune(egpu_batch_plan plan, void* stream, int reps, double* best_ms,
                                      int* best_grid);
EGPU_API int egpu_batch_plan_set_grid(egpu_batch_plan plan, int grid);
/* As egpu_batch_plan_create with a precision: 0 = FP64 (as above); 1 = each
 * system is converted once into an FP32 working copy (plan-owned), factored
 * there (FP64 register arithmetic, values stored in FP32), and its solution
 * refined in FP64 against A until the backward error max_j ||b_j - A x_j||_inf
 * / (||A||_inf ||x_j||_inf + ||b_j||_inf) <= 1e-14; A is left unchanged and B
 * receives X.  A system whose refinement stalls (or whose FP32 factorization
 * breaks down) is re-solved in FP64 within the same launch. */
EGPU_API int egpu_batch_plan_create_ex(egpu_handle h, int kind, int precision, int count, const int* n,
                                       const int* nrhs, double* const* dA, const int* lda, double* const* dB,
                                       const int* ldb, egpu_batch_plan* out);
/* Refinement corrections of each system in the last run (precision 1; -1 =
 * solved by the FP64 fallback; 0 for FP64 plans); synchronises. */
EGPU_API int egpu_batch_plan_iters(egpu_batch_plan plan, void* stream, int* iters);
/* The plan's launch shape: *nclass size classes (largest first), each with
 * its largest order, panel width, CTA size (threads) and persistent grid
 * (arrays of at least 3 entries; any pointer may be NULL). */
EGPU_API int egpu_batch_plan_shape(egpu_batch_plan plan, int* nclass, int* class_nmax, int* panel, int* threads,
                                   int* grid);
EGPU_API int egpu_batch_plan_destroy(egpu_batch_plan plan);

/* Request server (continuous batching on one GPU): no counterpart in the
 * reference.  A dispatcher thread admits queued requests in arrival order
 * against an HBM budget (bytes) and hands them to `slots` worker threads,
 * each with its own handle and stream, so up to `slots` jobs run at once;
 * all queued small requests (n <= 512, nrhs <= 16) of the kind at the head of
 * the queue form one batched job.  mode 0: FP64 solves; mode 1: HPD requests
 * of order >= the mixed threshold take egpu_dposv_mixed (FP64 fallback when
 * it cannot reach the tolerance), the rest stay FP64; a GE request outside
 * the batched jobs whose A is exactly symmetric with a positive diagonal is
 * tried as HPD first
 * (FP64 Cholesky, or the mixed solver from the threshold) and goes to LU only
 * when that factorization fails -- the same x.  kind 0 = HPDSolve(LOWER) (A lower triangle read),
 * kind 1 = GaussianElimination.  A, B, X are host buffers (pinned for
 * speed) that must stay valid until the request completes; A and B are not
 * modified, X receives the solution.  The per-slot handle workspaces are
 * outside the budget's accounting. */
typedef struct egpu_server_s* egpu_server;
EGPU_API int egpu_server_create(int device, size_t hbm_budget_bytes, int slots, int mode, egpu_server* out);
EGPU_API int egpu_server_set_tolerance(egpu_server s, double tol);
/* Mode 1 sends HPD requests of order >= n to the mixed solver (default
 * 6144: below it the FP64 path is faster on B200 for kappa spread
 * log-uniformly up to 1e8, where GMRES-IR makes the mixed solve slower). */
EGPU_API int egpu_server_set_mixed_min_n(egpu_server s, int n);
EGPU_API int egpu_server_submit(egpu_server s, int kind, int n, int nrhs, const double* A, int lda,
                                const double* B, int ldb, double* X, int ldx, unsigned long long* id);
/* Resident matrices (the request loop keeps matrices and factors on the
 * device): egpu_server_register copies A (host, kind 0 HPD / 1 GE) to the
 * device once, charging the budget for A and its factor, and returns *mid.
 * Requests on it (egpu_server_submit_resident) send only B and X: the first
 * one forms the factor (Cholesky; in mode 1 a GE matrix passing the structure
 * test tries Cholesky before LU), later ones reuse it, each an FP64 solve
 * (paths 6 and 7 in egpu_server_query).  egpu_server_unregister waits for the
 * matrix's requests to finish, then frees it. */
EGPU_API int egpu_server_register(egpu_server s, int kind, int n, const double* A, int lda, unsigned long long* mid);
EGPU_API int egpu_server_submit_resident(egpu_server s, unsigned long long mid, int nrhs, const double* B, int ldb,
                                         double* X, int ldx, unsigned long long* id);
EGPU_API int egpu_server_unregister(egpu_server s, unsigned long long mid);
/* *done = 0 while queued or running; once done: *status (EGPU_* code),
 * *latency_ms (completion - submission), *path (0 FP64, 1 mixed, 2 batched,
 * 3 mixed fell back to FP64, 4 GE request solved by the FP64 HPD path, 5 GE
 * request solved by the mixed HPD path, 6 resident matrix factored by this
 * request, 7 resident factor reused), *iters and *berr (mixed path).  wait != 0
 * blocks until the request completes. */
EGPU_API int egpu_server_query(egpu_server s, unsigned long long id, int wait, int* done, int* status,
                               double* latency_ms, int* path, int* iters, double* berr);
EGPU_API int egpu_server_release(egpu_server s, unsigned long long id);
EGPU_API int egpu_server_drain(egpu_server s);
EGPU_API int egpu_server_destroy(egpu_server s);

/* Mixed-precision HPDSolve (HPDSolve.hpp:18-28 computes the same x): no
 * counterpart in the reference, which factors in the working precision only.
 * Cholesky with the trailing updates and the panel solves (L21) on the
 * tcgen05 tensor cores in TF32 x 3 split precision (FP32 accumulation and
 * FP32 trailing matrix) and FP64 diagonal blocks (a factorization that meets
 * a non-positive pivot is redone once with FP64 panel solves before
 * EGPU_NOT_HPD is returned), then iterative refinement with FP64
 * residuals until the normwise backward error
 *   max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf) <= tol
 * or max_iter corrections.  A (uplo triangle read) and B are inputs only;
 * X (n x nrhs) receives the solution.  Returns EGPU_OK, EGPU_NOT_HPD,
 * EGPU_NO_CONVERGENCE (X holds the last iterate) or an error; *iters = the
 * corrections applied, *berr = the final backward error.  Synchronous. */
EGPU_API int egpu_dposv_mixed(egpu_handle h, int uplo, int n, int nrhs, const double* dA, int lda,
                              const double* dB, int ldb, double* dX, int ldx, int max_iter, double tol,
                              int* iters, double* berr);

/* GMRES iterations spent by the handle's last mixed solve: when plain
 * refinement stagnates (the low-precision factor is too far from A to
 * contract, typically kappa >~ 1e7), egpu_dposv_mixed continues with GMRES-IR
 * (GMRES on M^-1 A d = M^-1 r, M the low-precision factor, FP64 residuals and
 * Krylov vectors, 20 vectors per cycle, one cycle per correction); its
 * corrections count in *iters. */
EGPU_API int egpu_mixed_gmres_iterations(egpu_handle h);

/* Mixed-precision GaussianElimination (GaussianElimination.hpp:216-232 and
 * lu::SolveAfter, LU/SolveAfter.hpp:101-146, compute the same x; no
 * counterpart in the reference, which factors in the working precision only):
 * LU with partial pivoting of an FP32 copy of A -- each 128-wide panel
 * factored in FP64 by the pivoting panel kernel (lu::Panel, LU/Panel.hpp:19-89),
 * the row-panel solve and trailing update on the tcgen05 tensor cores in
 * TF32 x 3 split precision -- then iterative refinement with FP64 residuals
 * against A and corrections through the factors (GMRES-IR preconditioned by
 * them when plain refinement contracts slowly, or under policy 1 when the
 * 1-norm condition estimate asks for it; the FP64 LU of a copy of A when the
 * estimate says the FP32 factors cannot precondition, or GMRES-IR stagnates).  A and B are inputs only (an A
 * that is not 16-byte aligned with even lda is copied once); X receives the solution; nrhs <= 64.  Returns EGPU_OK,
 * EGPU_SINGULAR (an exact zero pivot of the low-precision factorization;
 * egpu_get_status gives its column), EGPU_NO_CONVERGENCE or an error.
 * Synchronous. */
EGPU_API int egpu_dgesv_mixed(egpu_handle h, int n, int nrhs, const double* dA, int lda, const double* dB, int ldb,
                              double* dX, int ldx, int max_iter, double tol, int* iters, double* berr);

/* Refinement policy of egpu_dposv_mixed and egpu_dgesv_mixed (no counterpart in the reference):
 * 0 (default) adaptive -- plain iterative refinement, and when the first
 * correction contracts slowly a 1-norm condition estimate of A (Hager's method
 * with A^-1 applied through the low-precision factor) decides between
 * continuing and GMRES-IR; 1 -- the estimate runs after every factorization
 * and an ill-conditioned A goes to GMRES-IR at once.  A matrix the
 * FP32-accurate factorization reports not numerically HPD is refactored with
 * FP64 panel solves (see egpu_dposv_mixed) before any refinement. */
EGPU_API int egpu_set_mixed_policy(egpu_handle h, int policy);
/* The last mixed solve's 1-norm condition estimate kappa_1(A) = ||A||_1
 * ||A^-1||_1 (-1 when that solve did not need one). */
EGPU_API int egpu_mixed_condition_estimate(egpu_handle h, double* kappa1);
/* How the last mixed solve finished: 0 plain refinement, 1 GMRES-IR, 2 the
 * FP64 factorization (egpu_dgesv_mixed only: taken when the condition estimate
 * puts kappa_1 * 2^-24 above 1e3, or when GMRES-IR stagnates); -1 no handle. */
EGPU_API int egpu_mixed_mode(egpu_handle h);

/* Host-memory form of egpu_dposv_mixed (A, B, X in host memory). */
EGPU_API int egpu_host_dposv_mixed(egpu_handle h, int uplo, int n, int nrhs, const double* A, int lda,
                                   const double* B, int ldb, double* X, int ldx, int max_iter, double tol,
                                   int* iters, double* berr);

/* The tcgen05 engine of egpu_dposv_mixed, for tests and benchmarks:
 * C (FP32, M x N, column-major) = alpha A B^T + beta C, with A (M x K) and
 * B (N x K) column-major FP64 split into TF32 hi/lo parts; terms 1 multiplies
 * the hi parts only, terms 3 adds hi*lo + lo*hi.  lower != 0: only the lower
 * triangle of a square C is written.  No counterpart in the reference. */
EGPU_API int egpu_tc_gemm_split(egpu_handle h, int M, int N, int K, double alpha, const double* dA, int lda,
                                const double* dB, int ldb, double beta, float* dC, int ldc, int lower, int terms);

/* The FP32 correction sweep of egpu_dposv_mixed, for tests and profiling (no
 * counterpart in the reference): X := L^-1 X (trans 0), L^-T X (trans 1) or
 * L^-T L^-1 X (trans 2, one launch) with L lower triangular, FP32, column-major (16-byte aligned, ldl a
 * multiple of 4), through 512 x 512 super-block inverses built from L's 128 x
 * 128 diagonal-block inverses; X FP64, nrhs <= 32.  Synchronous. */
EGPU_API int egpu_sweep32_solve(egpu_handle h, int trans, int n, int nrhs, const float* dL, int ldl, double* dX,
                                int ldx);

/* The work queue egpu_sweep32_solve launches for order n (host only, no
 * device needed; for tests and profiling, no counterpart in the reference):
 * returns the number of tile items and, when out != NULL, writes up to
 * max_items of them, 14 ints each in queue order -- tile map (0 L rows, 1 L
 * columns, 2 / 3 super-block inverse rows / columns, 4 L_{R+1,R} W_R rows,
 * 5 W_R L_{R,R-1} columns), direction, kind (0 super-block product, 1 bulk
 * delta, 2 next-block delta from the same input as kind 0), k chunks of 32,
 * tile coordinates (M, K), first input row, first output row, output rows,
 * then the dependency counter / count pairs (second counter -1: none) and the
 * counter the item increments.  Counters: 0 queue, 1 abort, then per
 * direction d and super-block R: 2 + 2 (d nsuper + R) (its kind-0 items
 * done) and 3 + 2 (d nsuper + R) (the delta items targeting R done). */
EGPU_API int egpu_sweep32_queue(int n, int trans, int sm_count, int* out, int max_items);

/* Batched HPDSolve(LOWER, NORMAL, A_i, B_i) (HPDSolve.hpp:18-28) for `count`
 * independent systems of uneven orders n[i] <= 512 with nrhs[i] <= 16, in one
 * persistent launch (one CTA per system at a time, largest first).  n, nrhs,
 * lda, ldb, info: host arrays; dA[i], dB[i]: device pointers (dB may be NULL:
 * factor only).  info[i] = 0, or the 1-based column where A_i stopped being
 * numerically HPD (that system's B_i is left unsolved).  Synchronous. */
EGPU_API int egpu_dposv_batched(egpu_handle h, int count, const int* n, const int* nrhs, double* const* dA,
                                const int* lda, double* const* dB, const int* ldb, int* info);

/* Sharding of independent systems across GPUs (no counterpart in the
 * reference, which distributes one matrix over a process grid instead): owner[i]
 * in [0, parts) for each of `count` systems of order n[i] (kind[i] 0 = HPD
 * solve, cost n^3 / 3; 1 = GaussianElimination, cost 2 n^3 / 3; kind NULL =
 * all HPD), dealt largest first to the least-loaded part.  Deterministic, so
 * every rank computes the same partition; load (optional, `parts` doubles)
 * receives each part's summed cost.  Host-only: no device is touched. */
EGPU_API int egpu_partition_systems(int count, const int* n, const int* kind, int parts, int* owner, double* load);

/* Batched GaussianElimination(A_i, B_i) (GaussianElimination.hpp:216-232) for
 * `count` independent systems, n[i] <= 512, nrhs[i] <= 16, one persistent
 * launch; same argument conventions as egpu_dposv_batched.  info[i] = 0 or the
 * 1-based column of an exact zero pivot (SingularMatrixException). */
EGPU_API int egpu_dgesv_batched(egpu_handle h, int count, const int* n, const int* nrhs, double* const* dA,
                                const int* lda, double* const* dB, const int* ldb, int* info);

/* Trsm(side, uplo, orientation, diag, alpha, A, B),
 * blas-like/level3/Trsm.hpp:49-86 (dtrsm_ at src/core/imports/blas.cpp:1203). */
EGPU_API int egpu_dtrsm(egpu_handle h, int side, int uplo, int orient, int diag, int m, int n, double alpha,
               const double* dA, int lda, double* dB, int ldb);

/* Trsv(uplo, orientation, diag, A, x), blas-like/level2/Trsv.hpp:20-44. */
EGPU_API int egpu_dtrsv(egpu_handle h, int uplo, int orient, int diag, int n, const double* dA, int lda, double* dx);

/* Gemm(orientA, orientB, alpha, A, B, beta, C), blas-like/level3/Gemm.hpp:158-211
 * (dgemm_ at blas.cpp:930-941). */
EGPU_API int egpu_dgemm(egpu_handle h, int orientA, int orientB, int m, int n, int k, double alpha, const double* dA,
               int lda, const double* dB, int ldb, double beta, double* dC, int ldc);

/* Herk(uplo, orientation, alpha, A, beta, C) for real F (= Syrk),
 * blas-like/level3/Herk.hpp:17-27, Syrk.hpp:20-57 (dsyrk_ at blas.cpp:1043).
 * orient NORMAL: C := alpha A A^T + beta C (A n x k); otherwise A^T A. */
EGPU_API int egpu_dherk(egpu_handle h, int uplo, int orient, int n, int k, double alpha, const double* dA, int lda,
               double beta, double* dC, int ldc);

/* ApplyRowPivots(A, p) / ApplyInverseRowPivots(A, p),
 * lapack-like/ApplyRowPivots.hpp:17-79 (sequential swaps i <-> p[i]). */
EGPU_API int egpu_dlaswp(egpu_handle h, int inverse, int m, int n, double* dA, int lda, const int* dp, int npiv);

/* TriangularInverse(uplo, diag, A), lapack-like/TriangularInverse.hpp:56-64
 * (triangular_inverse::LVar3 / UVar3): the uplo triangle of A := its inverse;
 * the other triangle, and for diag = EGPU_UNIT the diagonal, are not
 * touched.  No singularity check (as the reference). */
EGPU_API int egpu_dtrtri(egpu_handle h, int uplo, int diag, int n, double* dA, int lda);

/* Inverse(A), lapack-like/Inverse.hpp:17-23 (inverse::LUPartialPiv,
 * Inverse/LUPartialPiv.hpp): A := inv(A) from P A = L U.  Returns
 * EGPU_SINGULAR (info = the 1-based column of the zero pivot, lu::Panel's
 * SingularMatrixException) with A holding the partial factorization. */
EGPU_API int egpu_dgetri(egpu_handle h, int n, double* dA, int lda, int* info);

/* HPDInverse(uplo, A), lapack-like/Inverse.hpp:25-35 (hpd_inverse::
 * CholeskyLVar2 / CholeskyUVar2): the uplo triangle of A := that of inv(A);
 * the other triangle is not touched.  EGPU_NOT_HPD as egpu_dpotrf. */
EGPU_API int egpu_dpotri(egpu_handle h, int uplo, int n, double* dA, int lda, int* info);

/* LDLT(A[, d]) / LDLH(A[, d]), lapack-like/LDL.hpp (ldl::Var3,
 * LDL/Var3.hpp): A = L D L^T without pivoting, orient EGPU_TRANSPOSE or
 * EGPU_ADJOINT (the same for real F; EGPU_NORMAL is EGPU_ERR_ARG, "Can only
 * perform LDL^T or LDL^H").  Only the lower triangle is read and written:
 * strictly below the diagonal L (unit diagonal implied), on the diagonal D;
 * dd (device, n doubles, or NULL) also receives D.  EGPU_SINGULAR with info =
 * the 1-based column of an exact zero pivot. */
EGPU_API int egpu_dldl(egpu_handle h, int orient, int n, double* dA, int lda, double* dd, int* info);

/* ReverseCholesky(uplo, A), lapack-like/Cholesky.hpp:64-76
 * (cholesky::ReverseLVar3 / ReverseUVar3, Cholesky/LVar3.hpp:125-165): LOWER
 * factors A = L^T L with L lower, UPPER A = U U^T with U upper, in the uplo
 * triangle (the other triangle is not touched).  EGPU_NOT_HPD with info = the
 * 1-based column where the reverse sweep met a non-positive pivot.  dA needs
 * no alignment (the triangle is staged). */
EGPU_API int egpu_dpotrf_reverse(egpu_handle h, int uplo, int n, double* dA, int lda, int* info);

/* SafeDeterminant(A[, canOverwrite]), lapack-like/Determinant.hpp (
 * determinant::LUPartialPiv, Determinant/LUPartialPiv.hpp:17-67 with
 * PivotParity.hpp:17-33): det(A) = rho * exp(kappa * n), rho = +-1, kappa =
 * sum log|u_ii| / n.  A singular matrix gives rho = kappa = 0 and EGPU_OK (the
 * reference catches SingularMatrixException).  overwrite != 0 factors A in
 * place (canOverwrite); otherwise A is copied first and left unchanged.
 * Synchronous in either handle mode (the values return to the host); it
 * clears the handle's device status. */
EGPU_API int egpu_dsafe_det(egpu_handle h, int n, double* dA, int lda, int overwrite, double* rho, double* kappa);

/* SafeHPDDeterminant(uplo, A[, canOverwrite]), Determinant.hpp
 * (hpd_determinant::Cholesky, Determinant/Cholesky.hpp:17-55): rho = 1, kappa
 * = sum log l_ii / (n / 2); a matrix that is not numerically HPD gives rho =
 * kappa = 0 and EGPU_OK.  Otherwise as egpu_dsafe_det. */
EGPU_API int egpu_dsafe_hpd_det(egpu_handle h, int uplo, int n, double* dA, int lda, int overwrite, double* rho,
                                double* kappa);

/* Cholesky factorization that allocates no device memory (no counterpart in
 * the reference).  For callers that cannot let a library allocate: a process
 * that gives all device memory to its own pool at start-up and must not see an
 * allocation fail or synchronise the device mid-run.  Same result as
 * egpu_dpotrf with lookahead 0, on the caller's stream (NULL = the legacy
 * default stream), no handle.  dA must be 16-byte aligned with an even lda
 * (EGPU_ERR_ALIGN otherwise); nb in [2, 128] (EGPU_ERR_UNSUPPORTED otherwise),
 * an odd nb rounded down to the next even value as egpu_set_blocksize does.
 * Scratch: a file-scope 128 KiB + 256 B __device__ array on every GPU that
 * loads the library, held until exit; its device address is looked up on the
 * first call on each device (make that first call before any stream capture).
 * With CUDA's default lazy module loading that first call is also where the
 * driver loads the kernels it launches and places the array, which takes
 * device memory: make one small call at start-up (or set
 * CUDA_MODULE_LOADING=EAGER) so that later calls allocate nothing.  Each call
 * ends by waiting for the caller's stream (the status word is read back).
 * All calls share the array: calls that overlap on the GPU race. */
EGPU_API int egpu_dpotrf_noalloc(void* stream, int uplo, int n, double* dA, int lda, int nb, int* info);

/* ---- host-memory API (Matrix<F> buffers; synchronous) ---- */
EGPU_API int egpu_host_dpotrf(egpu_handle h, int uplo, int n, double* A, int lda, int* info);
EGPU_API int egpu_host_dpotrs(egpu_handle h, int uplo, int orient, int n, int nrhs, const double* A, int lda, double* B,
                     int ldb);
EGPU_API int egpu_host_dposv(egpu_handle h, int uplo, int orient, int n, int nrhs, double* A, int lda, double* B, int ldb,
                    int* info);
EGPU_API int egpu_host_dgetrf(egpu_handle h, int m, int n, double* A, int lda, int* p, int* info);
EGPU_API int egpu_host_dgetrf_nopiv(egpu_handle h, int m, int n, double* A, int lda, int* info);
EGPU_API int egpu_host_dgetrs(egpu_handle h, int orient, int n, int nrhs, const double* A, int lda, const int* p,
                     double* B, int ldb);
EGPU_API int egpu_host_dgesv(egpu_handle h, int n, int nrhs, double* A, int lda, double* B, int ldb, int* info);
EGPU_API int egpu_host_dtrsm(egpu_handle h, int side, int uplo, int orient, int diag, int m, int n, double alpha,
                    const double* A, int lda, double* B, int ldb);
EGPU_API int egpu_host_dgemm(egpu_handle h, int orientA, int orientB, int m, int n, int k, double alpha, const double* A,
                    int lda, const double* B, int ldb, double beta, double* C, int ldc);
EGPU_API int egpu_host_dherk(egpu_handle h, int uplo, int orient, int n, int k, double alpha, const double* A, int lda,
                    double beta, double* C, int ldc);
EGPU_API int egpu_host_dlaswp(egpu_handle h, int inverse, int m, int n, double* A, int lda, const int* p, int npiv);
EGPU_API int egpu_host_dldl(egpu_handle h, int orient, int n, double* A, int lda, double* d, int* info);
EGPU_API int egpu_host_dpotrf_reverse(egpu_handle h, int uplo, int n, double* A, int lda, int* info);
EGPU_API int egpu_host_dtrtri(egpu_handle h, int uplo, int diag, int n, double* A, int lda);
EGPU_API int egpu_host_dgetri(egpu_handle h, int n, double* A, int lda, int* info);
EGPU_API int egpu_host_dpotri(egpu_handle h, int uplo, int n, double* A, int lda, int* info);
/* overwrite != 0 (canOverwrite): A receives the factorization; otherwise A is
 * only read. */
EGPU_API int egpu_host_dsafe_det(egpu_handle h, int n, double* A, int lda, int overwrite, double* rho, double* kappa);
EGPU_API int egpu_host_dsafe_hpd_det(egpu_handle h, int uplo, int n, double* A, int lda, int overwrite, double* rho,
                                     double* kappa);

#ifdef __cplusplus
}
#endif

#endif /* ELEMGPU_H */
