/*
 * Oracle body, included twice by elemref.c (REAL = double / float).
 *
 * TEST INFRASTRUCTURE ONLY.  This is a CPU restatement of Elemental's
 * sequential factor-and-solve path, used by tests/, by smoke() and by
 * bench.py's cpu_baseline / reference arm as the checker.  Nothing in the
 * product (libelemgpu.so, the elem:: headers) links or calls it.
 *
 * Parity status: PINNED to the reference's own code.  The reference ships no
 * golden vectors or known-answer tests for this path (its tests print residual
 * norms from a wall-clock-seeded drand48), so oracle/refbuild/Makefile compiles
 * the reference's sources into oracle/_ref/libelemref.so (a single-process
 * MPI, a hand-written config.h, the scipy wheel's OpenBLAS), and
 * tests/test_oracle_ref.py checks this restatement against it on seeded
 * inputs (pivots index for index, factors and solves to rounding) and against
 * golden vectors it produced (tests/golden/ref_golden.npz).  Two recorded
 * deviations: the reference's sequential RowEchelon crashes (its distributed
 * form, which a 1 x 1 Grid runs, is what GaussianElimination restates), and
 * its blocked ReverseLVar3/UVar3 does not factor A for n > Blocksize() (the
 * restatement follows ReverseLVar3Unb, which it matches exactly for
 * n <= Blocksize()).  tests/test_oracle.py also checks it against LAPACK and
 * exact constructions.
 *
 * The level-3/level-2 arithmetic of the reference lives in whatever external
 * BLAS the build links (Elemental CMakeLists.txt:289-313; call sites
 * src/core/imports/blas.cpp:592 dscal, :690 dger, :901 dtrsv, :930 dgemm,
 * :1043 dsyrk, :1203 dtrsm).  That BLAS is not pinned by the reference; these
 * routines restate the published netlib reference-BLAS loop orders.
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(CAT(oref_, PFX), name)
#define IDX(M, ld, i, j) (M)[(size_t)(i) + (size_t)(j) * (size_t)(ld)]

/* ---------------------------------------------------------------- BLAS-3 */

/* C := alpha*op(A)*op(B) + beta*C  (netlib dgemm loop orders).  Row blocks of
 * C are processed by different threads; each element keeps a fixed summation
 * order, so the result does not depend on the thread count. */
void FN(gemm)(char ta, char tb, int m, int n, int k, REAL alpha,
              const REAL *A, int lda, const REAL *B, int ldb, REAL beta,
              REAL *C, int ldc) {
  const int nota = (ta == 'N' || ta == 'n');
  const int notb = (tb == 'N' || tb == 'n');
  if (m == 0 || n == 0) return;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < n; ++j) {
    if (beta == (REAL)0) {
      for (int i = 0; i < m; ++i) IDX(C, ldc, i, j) = 0;
    } else if (beta != (REAL)1) {
      for (int i = 0; i < m; ++i) IDX(C, ldc, i, j) *= beta;
    }
    if (nota) {
      for (int l = 0; l < k; ++l) {
        REAL t = alpha * (notb ? IDX(B, ldb, l, j) : IDX(B, ldb, j, l));
        if (t == (REAL)0) continue;
        const REAL *a = &IDX(A, lda, 0, l);
        REAL *c = &IDX(C, ldc, 0, j);
        for (int i = 0; i < m; ++i) c[i] += t * a[i];
      }
    } else {
      for (int i = 0; i < m; ++i) {
        REAL s = 0;
        const REAL *a = &IDX(A, lda, 0, i);
        for (int l = 0; l < k; ++l)
          s += a[l] * (notb ? IDX(B, ldb, l, j) : IDX(B, ldb, j, l));
        IDX(C, ldc, i, j) += alpha * s;
      }
    }
  }
}

/* C := alpha*A*A^T + beta*C (trans 'N') or alpha*A^T*A + beta*C ('T'), on the
 * uplo triangle only (netlib dsyrk). */
void FN(syrk)(char uplo, char trans, int n, int k, REAL alpha, const REAL *A,
              int lda, REAL beta, REAL *C, int ldc) {
  const int upper = (uplo == 'U' || uplo == 'u');
  const int notr = (trans == 'N' || trans == 'n');
  if (n == 0) return;
#pragma omp parallel for schedule(dynamic, 8)
  for (int j = 0; j < n; ++j) {
    const int i0 = upper ? 0 : j, i1 = upper ? j + 1 : n;
    if (beta == (REAL)0) {
      for (int i = i0; i < i1; ++i) IDX(C, ldc, i, j) = 0;
    } else if (beta != (REAL)1) {
      for (int i = i0; i < i1; ++i) IDX(C, ldc, i, j) *= beta;
    }
    if (notr) {
      for (int l = 0; l < k; ++l) {
        REAL t = alpha * IDX(A, lda, j, l);
        if (t == (REAL)0) continue;
        for (int i = i0; i < i1; ++i) IDX(C, ldc, i, j) += t * IDX(A, lda, i, l);
      }
    } else {
      for (int i = i0; i < i1; ++i) {
        REAL s = 0;
        for (int l = 0; l < k; ++l) s += IDX(A, lda, l, i) * IDX(A, lda, l, j);
        IDX(C, ldc, i, j) += alpha * s;
      }
    }
  }
}

/* op(A)*X = alpha*B (side 'L') or X*op(A) = alpha*B (side 'R'); B := X.
 * Netlib dtrsm, all eight side/uplo/trans cases. */
void FN(trsm)(char side, char uplo, char transa, char diag, int m, int n,
              REAL alpha, const REAL *A, int lda, REAL *B, int ldb) {
  const int lside = (side == 'L' || side == 'l');
  const int upper = (uplo == 'U' || uplo == 'u');
  const int notr = (transa == 'N' || transa == 'n');
  const int nounit = !(diag == 'U' || diag == 'u');
  if (m == 0 || n == 0) return;
  if (lside) {
    /* columns of B are independent */
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j) {
      REAL *b = &IDX(B, ldb, 0, j);
      if (alpha != (REAL)1)
        for (int i = 0; i < m; ++i) b[i] *= alpha;
      if (notr) {
        if (upper) {
          for (int k = m - 1; k >= 0; --k) {
            if (b[k] == (REAL)0) continue;
            if (nounit) b[k] /= IDX(A, lda, k, k);
            for (int i = 0; i < k; ++i) b[i] -= b[k] * IDX(A, lda, i, k);
          }
        } else {
          for (int k = 0; k < m; ++k) {
            if (b[k] == (REAL)0) continue;
            if (nounit) b[k] /= IDX(A, lda, k, k);
            for (int i = k + 1; i < m; ++i) b[i] -= b[k] * IDX(A, lda, i, k);
          }
        }
      } else {
        if (upper) {
          for (int i = 0; i < m; ++i) {
            REAL t = b[i];
            for (int k = 0; k < i; ++k) t -= IDX(A, lda, k, i) * b[k];
            if (nounit) t /= IDX(A, lda, i, i);
            b[i] = t;
          }
        } else {
          for (int i = m - 1; i >= 0; --i) {
            REAL t = b[i];
            for (int k = i + 1; k < m; ++k) t -= IDX(A, lda, k, i) * b[k];
            if (nounit) t /= IDX(A, lda, i, i);
            b[i] = t;
          }
        }
      }
    }
  } else {
    /* rows of B are independent: split rows over threads */
    const int nth_rows = 64;
    const int nblk = (m + nth_rows - 1) / nth_rows;
#pragma omp parallel for schedule(static)
    for (int rb = 0; rb < nblk; ++rb) {
      const int r0 = rb * nth_rows;
      const int r1 = (r0 + nth_rows < m) ? r0 + nth_rows : m;
      if (notr) {
        if (upper) {
          for (int j = 0; j < n; ++j) {
            if (alpha != (REAL)1)
              for (int i = r0; i < r1; ++i) IDX(B, ldb, i, j) *= alpha;
            for (int k = 0; k < j; ++k) {
              REAL akj = IDX(A, lda, k, j);
              if (akj == (REAL)0) continue;
              for (int i = r0; i < r1; ++i)
                IDX(B, ldb, i, j) -= akj * IDX(B, ldb, i, k);
            }
            if (nounit) {
              REAL t = (REAL)1 / IDX(A, lda, j, j);
              for (int i = r0; i < r1; ++i) IDX(B, ldb, i, j) *= t;
            }
          }
        } else {
          for (int j = n - 1; j >= 0; --j) {
            if (alpha != (REAL)1)
              for (int i = r0; i < r1; ++i) IDX(B, ldb, i, j) *= alpha;
            for (int k = j + 1; k < n; ++k) {
              REAL akj = IDX(A, lda, k, j);
              if (akj == (REAL)0) continue;
              for (int i = r0; i < r1; ++i)
                IDX(B, ldb, i, j) -= akj * IDX(B, ldb, i, k);
            }
            if (nounit) {
              REAL t = (REAL)1 / IDX(A, lda, j, j);
              for (int i = r0; i < r1; ++i) IDX(B, ldb, i, j) *= t;
            }
          }
        }
      } else {
        if (upper) {
          for (int k = n - 1; k >= 0; --k) {
            if (nounit) {
              REAL t = (REAL)1 / IDX(A, lda, k, k);
              for (int i = r0; i < r1; ++i) IDX(B, ldb, i, k) *= t;
            }
            for (int j = 0; j < k; ++j) {
              REAL ajk = IDX(A, lda, j, k);
              if (ajk == (REAL)0) continue;
              for (int i = r0; i < r1; ++i)
                IDX(B, ldb, i, j) -= ajk * IDX(B, ldb, i, k);
            }
            if (alpha != (REAL)1)
              for (int i = r0; i < r1; ++i) IDX(B, ldb, i, k) *= alpha;
          }
        } else {
          for (int k = 0; k < n; ++k) {
            if (nounit) {
              REAL t = (REAL)1 / IDX(A, lda, k, k);
              for (int i = r0; i < r1; ++i) IDX(B, ldb, i, k) *= t;
            }
            for (int j = k + 1; j < n; ++j) {
              REAL ajk = IDX(A, lda, j, k);
              if (ajk == (REAL)0) continue;
              for (int i = r0; i < r1; ++i)
                IDX(B, ldb, i, j) -= ajk * IDX(B, ldb, i, k);
            }
            if (alpha != (REAL)1)
              for (int i = r0; i < r1; ++i) IDX(B, ldb, i, k) *= alpha;
          }
        }
      }
    }
  }
}

/* ---------------------------------------------------------------- BLAS-2 */

/* op(A) x = b, x overwrites b (netlib dtrsv, incx = 1). */
void FN(trsv)(char uplo, char trans, char diag, int n, const REAL *A, int lda,
              REAL *x) {
  FN(trsm)('L', uplo, trans, diag, n, 1, (REAL)1, A, lda, x, n > 0 ? n : 1);
}

/* ---------------------------------------------------- Elemental: Cholesky */

/* cholesky::LVar3Unb, lapack-like/Cholesky/LVar3.hpp:19-49.  Returns 0, or
 * j+1 when the j-th pivot is not positive ("A was not numerically HPD"). */
static int FN(chol_lvar3_unb)(int n, REAL *A, int lda) {
  for (int j = 0; j < n; ++j) {
    REAL alpha = IDX(A, lda, j, j);
    if (alpha <= (REAL)0) return j + 1;
    alpha = (REAL)sqrt((double)alpha);
    IDX(A, lda, j, j) = alpha;
    for (int k = j + 1; k < n; ++k) IDX(A, lda, k, j) /= alpha;
    for (int k = j + 1; k < n; ++k)
      for (int i = k; i < n; ++i)
        IDX(A, lda, i, k) -= IDX(A, lda, i, j) * IDX(A, lda, k, j);
  }
  return 0;
}

/* cholesky::UVar3Unb, lapack-like/Cholesky/UVar3.hpp:21-50. */
static int FN(chol_uvar3_unb)(int n, REAL *A, int lda) {
  for (int j = 0; j < n; ++j) {
    REAL alpha = IDX(A, lda, j, j);
    if (alpha <= (REAL)0) return j + 1;
    alpha = (REAL)sqrt((double)alpha);
    IDX(A, lda, j, j) = alpha;
    for (int k = j + 1; k < n; ++k) IDX(A, lda, j, k) /= alpha;
    for (int k = j + 1; k < n; ++k)
      for (int i = j + 1; i <= k; ++i)
        IDX(A, lda, i, k) -= IDX(A, lda, j, i) * IDX(A, lda, j, k);
  }
  return 0;
}

/* Cholesky(uplo, Matrix&), lapack-like/Cholesky.hpp:49-62, dispatching to the
 * blocked right-looking cholesky::LVar3 (Cholesky/LVar3.hpp:83-123) or UVar3
 * (Cholesky/UVar3.hpp:85-125).  uplo: 0 = LOWER, 1 = UPPER.  Returns 0 or the
 * 1-based global column at which A stopped being numerically HPD. */
int FN(cholesky)(int uplo, int n, REAL *A, int lda, int nb) {
  if (nb < 1) nb = 128;
  for (int k = 0; k < n; k += nb) {
    const int b = (n - k < nb) ? n - k : nb;
    const int m2 = n - k - b;
    REAL *A11 = &IDX(A, lda, k, k);
    int st = uplo == 0 ? FN(chol_lvar3_unb)(b, A11, lda)
                       : FN(chol_uvar3_unb)(b, A11, lda);
    if (st) return k + st;
    if (m2 == 0) continue;
    if (uplo == 0) {
      REAL *A21 = &IDX(A, lda, k + b, k);
      REAL *A22 = &IDX(A, lda, k + b, k + b);
      /* Trsm(RIGHT, LOWER, ADJOINT, NON_UNIT, 1, A11, A21) */
      FN(trsm)('R', 'L', 'T', 'N', m2, b, (REAL)1, A11, lda, A21, lda);
      /* Herk(LOWER, NORMAL, -1, A21, 1, A22) */
      FN(syrk)('L', 'N', m2, b, (REAL)-1, A21, lda, (REAL)1, A22, lda);
    } else {
      REAL *A12 = &IDX(A, lda, k, k + b);
      REAL *A22 = &IDX(A, lda, k + b, k + b);
      /* Trsm(LEFT, UPPER, ADJOINT, NON_UNIT, 1, A11, A12) */
      FN(trsm)('L', 'U', 'T', 'N', b, m2, (REAL)1, A11, lda, A12, lda);
      /* Herk(UPPER, ADJOINT, -1, A12, 1, A22) */
      FN(syrk)('U', 'T', m2, b, (REAL)-1, A12, lda, (REAL)1, A22, lda);
    }
  }
  return 0;
}

/* cholesky::SolveAfter, lapack-like/Cholesky/SolveAfter.hpp:20-75.  For real
 * F the TRANSPOSE conjugations are no-ops, so orientation does not matter. */
void FN(cholesky_solve_after)(int uplo, int orient, int n, int nrhs,
                              const REAL *A, int lda, REAL *B, int ldb) {
  (void)orient;
  if (uplo == 0) {
    FN(trsm)('L', 'L', 'N', 'N', n, nrhs, (REAL)1, A, lda, B, ldb);
    FN(trsm)('L', 'L', 'T', 'N', n, nrhs, (REAL)1, A, lda, B, ldb);
  } else {
    FN(trsm)('L', 'U', 'T', 'N', n, nrhs, (REAL)1, A, lda, B, ldb);
    FN(trsm)('L', 'U', 'N', 'N', n, nrhs, (REAL)1, A, lda, B, ldb);
  }
}

/* HPDSolve, lapack-like/HPDSolve.hpp:18-28. */
int FN(hpd_solve)(int uplo, int orient, int n, int nrhs, REAL *A, int lda,
                  REAL *B, int ldb, int nb) {
  int st = FN(cholesky)(uplo, n, A, lda, nb);
  if (st) return st;
  FN(cholesky_solve_after)(uplo, orient, n, nrhs, A, lda, B, ldb);
  return 0;
}

/* ---------------------------------------------------------- Elemental: LU */

/* ComposePivots(p, pivotOffset, image, preimage),
 * lapack-like/ComposePivots.hpp:81-125: turns b sequential swaps (absolute
 * row indices, offset by pivotOffset) into the image/preimage of rows
 * 0..b-1 of the trailing block. */
void FN(compose_pivots)(const int *p, int b, int offset, int *image,
                        int *preimage) {
  for (int i = 0; i < b; ++i) {
    int k = p[i] - offset;
    for (int j = i - 1; j >= 0; --j) {
      if (p[j] - offset == k)
        k = j;
      else if (j == k)
        k = p[j] - offset;
    }
    preimage[i] = k;
  }
  for (int i = 0; i < b; ++i) {
    int k = i;
    for (int j = 0; j < ((k + 1 < b) ? k + 1 : b); ++j) {
      if (p[j] - offset == k)
        k = j;
      else if (j == k)
        k = p[j] - offset;
    }
    image[i] = k;
  }
}

/* ApplyRowPivots(A, image, preimage), lapack-like/ApplyRowPivots.hpp:129-181:
 * row i of the first b rows moves to row image[i]; row preimage[i] (when it
 * lies below the first b rows) moves into row i. */
void FN(apply_composed_pivots)(int m, int n, REAL *A, int lda, int b,
                               const int *image, const int *preimage) {
  if (m == 0 || n == 0 || b == 0) return;
  REAL *top = (REAL *)malloc(sizeof(REAL) * (size_t)b * (size_t)n);
  REAL *pre = (REAL *)malloc(sizeof(REAL) * (size_t)b * (size_t)n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < b; ++i) top[i + (size_t)j * b] = IDX(A, lda, i, j);
  for (int i = 0; i < b; ++i)
    if (preimage[i] >= b)
      for (int j = 0; j < n; ++j)
        pre[i + (size_t)j * b] = IDX(A, lda, preimage[i], j);
  for (int i = 0; i < b; ++i) {
    for (int j = 0; j < n; ++j) IDX(A, lda, image[i], j) = top[i + (size_t)j * b];
    if (preimage[i] >= b)
      for (int j = 0; j < n; ++j) IDX(A, lda, i, j) = pre[i + (size_t)j * b];
  }
  free(top);
  free(pre);
}

/* ApplyRowPivots(A, p), lapack-like/ApplyRowPivots.hpp:17-47: sequential
 * swaps i <-> p[i], i = 0..np-1. */
void FN(apply_row_pivots)(int m, int n, REAL *A, int lda, const int *p,
                          int np) {
  if (m == 0 || n == 0) return;
  for (int i = 0; i < np; ++i) {
    const int k = p[i];
    if (k == i) continue;
    for (int j = 0; j < n; ++j) {
      REAL t = IDX(A, lda, i, j);
      IDX(A, lda, i, j) = IDX(A, lda, k, j);
      IDX(A, lda, k, j) = t;
    }
  }
}

/* ApplyInverseRowPivots(A, p), ApplyRowPivots.hpp:49-79: the same swaps in
 * reverse order. */
void FN(apply_inverse_row_pivots)(int m, int n, REAL *A, int lda, const int *p,
                                  int np) {
  if (m == 0 || n == 0) return;
  for (int i = np - 1; i >= 0; --i) {
    const int k = p[i];
    if (k == i) continue;
    for (int j = 0; j < n; ++j) {
      REAL t = IDX(A, lda, i, j);
      IDX(A, lda, i, j) = IDX(A, lda, k, j);
      IDX(A, lda, k, j) = t;
    }
  }
}

/* lu::Panel(A, p, pivotOffset), lapack-like/LU/Panel.hpp:19-89.  A is the
 * m x w panel; p[0..w) receives absolute pivot rows (row index + offset).
 * Pivot = first entry of maximal |a| (strict '>' scan).  Returns 0 or the
 * 1-based panel column whose pivot was exactly zero (SingularMatrixException). */
static int FN(lu_panel)(int m, int w, REAL *A, int lda, int *p, int offset) {
  for (int j = 0; j < w && j < m; ++j) {
    REAL pivot = IDX(A, lda, j, j);
    int prow = j;
    for (int i = j + 1; i < m; ++i) {
      REAL v = IDX(A, lda, i, j);
      if (fabs((double)v) > fabs((double)pivot)) {
        pivot = v;
        prow = i;
      }
    }
    p[j] = prow + offset;
    if (prow != j)
      for (int c = 0; c < w; ++c) {
        REAL t = IDX(A, lda, j, c);
        IDX(A, lda, j, c) = IDX(A, lda, prow, c);
        IDX(A, lda, prow, c) = t;
      }
    const REAL alpha = IDX(A, lda, j, j);
    if (alpha == (REAL)0) return j + 1;
    const REAL inv = (REAL)1 / alpha;
    for (int i = j + 1; i < m; ++i) IDX(A, lda, i, j) *= inv; /* Scale */
    for (int c = j + 1; c < w; ++c) {                        /* Geru */
      const REAL u = IDX(A, lda, j, c);
      if (u == (REAL)0) continue;
      for (int i = j + 1; i < m; ++i) IDX(A, lda, i, c) -= IDX(A, lda, i, j) * u;
    }
  }
  return 0;
}

/* LU(A, p), lapack-like/LU.hpp:144-218: blocked right-looking LU with partial
 * pivoting.  p has min(m,n) entries (absolute 0-based rows, sequential-swap
 * semantics).  Returns 0 or the 1-based global column with a zero pivot. */
int FN(lu)(int m, int n, REAL *A, int lda, int *p, int nb) {
  if (nb < 1) nb = 128;
  const int mn = m < n ? m : n;
  int *image = (int *)malloc(sizeof(int) * (size_t)(nb > 0 ? nb : 1));
  int *preimage = (int *)malloc(sizeof(int) * (size_t)(nb > 0 ? nb : 1));
  int status = 0;
  for (int k = 0; k < mn; k += nb) {
    const int b = (mn - k < nb) ? mn - k : nb;
    const int mr = m - k;         /* rows of ABR */
    const int nr = n - k - b;     /* columns right of the panel */
    REAL *ABRL = &IDX(A, lda, k, k);
    int st = FN(lu_panel)(mr, b, ABRL, lda, p + k, k);
    if (st) { status = k + st; break; }
    FN(compose_pivots)(p + k, b, k, image, preimage);
    /* ApplyRowPivots(ABL, ...) and ApplyRowPivots(ABRR, ...) */
    FN(apply_composed_pivots)(mr, k, &IDX(A, lda, k, 0), lda, b, image, preimage);
    FN(apply_composed_pivots)(mr, nr, &IDX(A, lda, k, k + b), lda, b, image, preimage);
    if (nr > 0) {
      REAL *A11 = ABRL, *A12 = &IDX(A, lda, k, k + b);
      REAL *A21 = &IDX(A, lda, k + b, k), *A22 = &IDX(A, lda, k + b, k + b);
      FN(trsm)('L', 'L', 'N', 'U', b, nr, (REAL)1, A11, lda, A12, lda);
      FN(gemm)('N', 'N', mr - b, nr, b, (REAL)-1, A21, lda, A12, lda, (REAL)1, A22, lda);
    }
  }
  free(image);
  free(preimage);
  return status;
}

/* lu::Unb, lapack-like/LU/Local.hpp:61-82 (no pivoting). */
static int FN(lu_unb)(int m, int n, REAL *A, int lda) {
  const int mn = m < n ? m : n;
  for (int j = 0; j < mn; ++j) {
    const REAL alpha = IDX(A, lda, j, j);
    if (alpha == (REAL)0) return j + 1;
    const REAL inv = (REAL)1 / alpha;
    for (int i = j + 1; i < m; ++i) IDX(A, lda, i, j) *= inv;
    for (int c = j + 1; c < n; ++c) {
      const REAL u = IDX(A, lda, j, c);
      if (u == (REAL)0) continue;
      for (int i = j + 1; i < m; ++i) IDX(A, lda, i, c) -= IDX(A, lda, i, j) * u;
    }
  }
  return 0;
}

/* LU(A) without pivoting, lapack-like/LU.hpp:36-74. */
int FN(lu_nopiv)(int m, int n, REAL *A, int lda, int nb) {
  if (nb < 1) nb = 128;
  const int mn = m < n ? m : n;
  for (int k = 0; k < mn; k += nb) {
    const int b = (mn - k < nb) ? mn - k : nb;
    const int m2 = m - k - b, n2 = n - k - b;
    REAL *A11 = &IDX(A, lda, k, k);
    int st = FN(lu_unb)(b, b, A11, lda);
    if (st) return k + st;
    REAL *A21 = &IDX(A, lda, k + b, k), *A12 = &IDX(A, lda, k, k + b);
    REAL *A22 = &IDX(A, lda, k + b, k + b);
    FN(trsm)('R', 'U', 'N', 'N', m2, b, (REAL)1, A11, lda, A21, lda);
    FN(trsm)('L', 'L', 'N', 'U', b, n2, (REAL)1, A11, lda, A12, lda);
    FN(gemm)('N', 'N', m2, n2, b, (REAL)-1, A21, lda, A12, lda, (REAL)1, A22, lda);
  }
  return 0;
}

/* lu::SolveAfter(orientation, A, p, B), lapack-like/LU/SolveAfter.hpp:101-146
 * (p == NULL selects the unpivoted overload, :20-57).  orient: 0 NORMAL,
 * 1 TRANSPOSE, 2 ADJOINT (identical for real F). */
void FN(lu_solve_after)(int orient, int n, int nrhs, const REAL *A, int lda,
                        const int *p, REAL *B, int ldb) {
  if (orient == 0) {
    if (p) FN(apply_row_pivots)(n, nrhs, B, ldb, p, n);
    FN(trsm)('L', 'L', 'N', 'U', n, nrhs, (REAL)1, A, lda, B, ldb);
    FN(trsm)('L', 'U', 'N', 'N', n, nrhs, (REAL)1, A, lda, B, ldb);
  } else {
    FN(trsm)('L', 'U', 'T', 'N', n, nrhs, (REAL)1, A, lda, B, ldb);
    FN(trsm)('L', 'L', 'T', 'U', n, nrhs, (REAL)1, A, lda, B, ldb);
    if (p) FN(apply_inverse_row_pivots)(n, nrhs, B, ldb, p, n);
  }
}

/* GaussianElimination(A, B), lapack-like/GaussianElimination.hpp:216-232,
 * with RowEchelon as the distributed overload states it (:94-209): the panel
 * is [A11; A21]; its pivots are applied to [A12; A22] and to the trailing
 * rows of B, then A12/B1 are solved with unit-lower A11 and A22/B2 updated.
 * (The sequential RowEchelon at :19-92 hands [A12; A22] to lu::Panel, which
 * does not factor the pivot column; the distributed form is the one that
 * computes the documented result, and a 1x1 grid runs it.)  Finally B is
 * solved with the upper triangle of A.  Returns 0 or the 1-based column of a
 * zero pivot. */
int FN(gaussian_elimination)(int n, int nrhs, REAL *A, int lda, REAL *B,
                             int ldb, int nb) {
  if (nb < 1) nb = 128;
  int *p1 = (int *)malloc(sizeof(int) * (size_t)nb);
  int *image = (int *)malloc(sizeof(int) * (size_t)nb);
  int *preimage = (int *)malloc(sizeof(int) * (size_t)nb);
  int status = 0;
  for (int k = 0; k < n; k += nb) {
    const int b = (n - k < nb) ? n - k : nb;
    const int mr = n - k, nr = n - k - b;
    REAL *A11 = &IDX(A, lda, k, k);
    int st = FN(lu_panel)(mr, b, A11, lda, p1, k);
    if (st) { status = k + st; break; }
    FN(compose_pivots)(p1, b, k, image, preimage);
    FN(apply_composed_pivots)(mr, nr, &IDX(A, lda, k, k + b), lda, b, image, preimage);
    FN(apply_composed_pivots)(mr, nrhs, &IDX(B, ldb, k, 0), ldb, b, image, preimage);
    REAL *A12 = &IDX(A, lda, k, k + b), *A21 = &IDX(A, lda, k + b, k);
    REAL *A22 = &IDX(A, lda, k + b, k + b);
    REAL *B1 = &IDX(B, ldb, k, 0), *B2 = &IDX(B, ldb, k + b, 0);
    if (nr > 0) FN(trsm)('L', 'L', 'N', 'U', b, nr, (REAL)1, A11, lda, A12, lda);
    FN(trsm)('L', 'L', 'N', 'U', b, nrhs, (REAL)1, A11, lda, B1, ldb);
    if (nr > 0) {
      FN(gemm)('N', 'N', nr, nr, b, (REAL)-1, A21, lda, A12, lda, (REAL)1, A22, lda);
      FN(gemm)('N', 'N', nr, nrhs, b, (REAL)-1, A21, lda, B1, ldb, (REAL)1, B2, ldb);
    }
  }
  free(p1);
  free(image);
  free(preimage);
  if (status) return status;
  FN(trsm)('L', 'U', 'N', 'N', n, nrhs, (REAL)1, A, lda, B, ldb);
  return 0;
}

#undef FN
#undef IDX
#undef CAT
#undef CAT_
