// C entry points into the reference's own code (TEST INFRASTRUCTURE ONLY).
//
// oracle/refbuild/Makefile compiles the reference's sources where they lie
// (its headers and src/core, src/core/imports, src/core/dist_matrix,
// src/blas-like/Trrk.cpp) together with this file, a single-process MPI
// (mpi.h, mpi_single.cpp), a hand-written config.h and forwarding stubs to the
// OpenBLAS of the scipy wheel, into oracle/_ref/libelemref.so.  Each eref_*
// function wraps column-major caller buffers in elem::Matrix views (no copy;
// Matrix::Attach, core/matrix.hpp:106) and calls the reference's entry point
// unchanged; DistMatrix variants copy into a DistMatrix on a 1 x 1 Grid.
//
// Return codes: 0 ok; 1 the reference threw "A was not numerically HPD"
// (Cholesky/LVar3.hpp:37-38); 2 SingularMatrixException (LU/Panel.hpp:76-77);
// -1 any other exception (eref_last_error() has its message).  Everything but
// the eref_* names has hidden visibility, so the reference's elem:: symbols,
// the MPI names and the BLAS stubs cannot clash with the GPU library or with
// another BLAS in the process.
#include <cstring>
#include <stdexcept>
#include <string>

#include "elemental.hpp"

#define EREF extern "C" __attribute__((visibility("default")))

namespace {

std::string g_err;
bool g_init = false;

void init() {
  if (g_init) return;
  int argc = 1;
  static char name[] = "eref";
  static char* argv0[] = {name, nullptr};
  char** argv = argv0;
  elem::Initialize(argc, argv);
  g_init = true;
}

template <typename Fn>
int guarded(Fn fn) {
  try {
    init();
    fn();
    return 0;
  } catch (elem::SingularMatrixException& e) {
    g_err = e.what();
    return 2;
  } catch (std::logic_error& e) {
    g_err = e.what();
    return g_err == "A was not numerically HPD" ? 1 : -1;
  } catch (std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

elem::UpperOrLower U(int uplo) { return uplo == 0 ? elem::LOWER : elem::UPPER; }
elem::Orientation O(int o) { return o == 0 ? elem::NORMAL : (o == 1 ? elem::TRANSPOSE : elem::ADJOINT); }
elem::LeftOrRight S(int s) { return s == 0 ? elem::LEFT : elem::RIGHT; }
elem::UnitOrNonUnit D(int d) { return d == 0 ? elem::NON_UNIT : elem::UNIT; }

// column-major n x m caller buffer <-> the local matrix of a 1 x 1 DistMatrix
template <typename T, elem::Distribution CD, elem::Distribution RD>
void to_dist(elem::DistMatrix<T, CD, RD>& D, int m, int n, const T* A, int lda) {
  D.ResizeTo(m, n);
  for (int j = 0; j < n; ++j) std::memcpy(D.Matrix().Buffer(0, j), A + (size_t)j * lda, sizeof(T) * m);
}
template <typename T, elem::Distribution CD, elem::Distribution RD>
void from_dist(const elem::DistMatrix<T, CD, RD>& D, T* A, int lda) {
  for (int j = 0; j < D.Width(); ++j)
    std::memcpy(A + (size_t)j * lda, D.LockedMatrix().LockedBuffer(0, j), sizeof(T) * D.Height());
}

}  // namespace

EREF const char* eref_last_error(void) { return g_err.c_str(); }

// elem::SetBlocksize (src/core/global.cpp:277-283); every factorization below
// takes nb and sets it first.
static void set_nb(int nb) {
  if (nb > 0) elem::SetBlocksize(nb);
}

EREF int eref_dcholesky(int uplo, int n, double* A, int lda, int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::Matrix<double> M;
    M.Attach(n, n, A, lda);
    elem::Cholesky(U(uplo), M);  // lapack-like/Cholesky.hpp:49-62
  });
}

EREF int eref_dreverse_cholesky(int uplo, int n, double* A, int lda, int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::Matrix<double> M;
    M.Attach(n, n, A, lda);
    elem::ReverseCholesky(U(uplo), M);  // lapack-like/Cholesky.hpp:64-76
  });
}

EREF int eref_dcholesky_solve_after(int uplo, int orient, int n, int nrhs, const double* A, int lda, double* B,
                                    int ldb) {
  return guarded([&] {
    elem::Matrix<double> M, X;
    M.LockedAttach(n, n, A, lda);
    X.Attach(n, nrhs, B, ldb);
    elem::cholesky::SolveAfter(U(uplo), O(orient), M, X);  // Cholesky/SolveAfter.hpp:20-75
  });
}

EREF int eref_dhpd_solve(int uplo, int orient, int n, int nrhs, double* A, int lda, double* B, int ldb, int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::Matrix<double> M, X;
    M.Attach(n, n, A, lda);
    X.Attach(n, nrhs, B, ldb);
    elem::HPDSolve(U(uplo), O(orient), M, X);  // HPDSolve.hpp:18-28
  });
}

EREF int eref_dlu(int m, int n, double* A, int lda, int* p, int nb) {
  return guarded([&] {
    set_nb(nb);
    const int mn = m < n ? m : n;
    elem::Matrix<double> M;
    elem::Matrix<int> P;
    M.Attach(m, n, A, lda);
    P.Attach(mn, 1, p, mn > 0 ? mn : 1);  // a view: LU does not resize it (LU.hpp:155-156)
    elem::LU(M, P);                       // LU.hpp:144-218
  });
}

EREF int eref_dlu_nopiv(int m, int n, double* A, int lda, int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::Matrix<double> M;
    M.Attach(m, n, A, lda);
    elem::LU(M);  // LU.hpp:36-74
  });
}

EREF int eref_dlu_solve_after(int orient, int n, int nrhs, const double* A, int lda, const int* p, double* B,
                              int ldb) {
  return guarded([&] {
    elem::Matrix<double> M, X;
    elem::Matrix<int> P;
    M.LockedAttach(n, n, A, lda);
    X.Attach(n, nrhs, B, ldb);
    if (p) {
      P.LockedAttach(n, 1, p, n > 0 ? n : 1);
      elem::lu::SolveAfter(O(orient), M, P, X);  // LU/SolveAfter.hpp:101-146
    } else {
      elem::lu::SolveAfter(O(orient), M, X);  // LU/SolveAfter.hpp:20-57
    }
  });
}

// The sequential GaussianElimination (GaussianElimination.hpp:216-232) is not
// wrapped: its RowEchelon (:19-92) hands [A12; A22] -- the columns right of
// the diagonal block -- to lu::Panel and never factors the pivot column, and
// run here it ends in a segmentation fault.  The DistMatrix form
// (eref_dist_dgaussian_elimination: RowEchelon :94-209 on a 1 x 1 Grid) is the
// one the GPU path follows.

EREF int eref_dapply_row_pivots(int inverse, int m, int n, double* B, int ldb, const int* p, int np) {
  return guarded([&] {
    elem::Matrix<double> X;
    elem::Matrix<int> P;
    X.Attach(m, n, B, ldb);
    P.LockedAttach(np, 1, p, np > 0 ? np : 1);
    if (inverse) elem::ApplyInverseRowPivots(X, P);  // ApplyRowPivots.hpp:49-79
    else elem::ApplyRowPivots(X, P);                 // ApplyRowPivots.hpp:17-47
  });
}

EREF int eref_dtrsm(int side, int uplo, int orient, int diag, int m, int n, double alpha, const double* A, int lda,
                    double* B, int ldb) {
  return guarded([&] {
    const int k = side == 0 ? m : n;
    elem::Matrix<double> T, X;
    T.LockedAttach(k, k, A, lda);
    X.Attach(m, n, B, ldb);
    elem::Trsm(S(side), U(uplo), O(orient), D(diag), alpha, T, X);  // blas-like/level3/Trsm.hpp:49-86
  });
}

EREF int eref_dtrsv(int uplo, int orient, int diag, int n, const double* A, int lda, double* x) {
  return guarded([&] {
    elem::Matrix<double> T, X;
    T.LockedAttach(n, n, A, lda);
    X.Attach(n, 1, x, n > 0 ? n : 1);
    elem::Trsv(U(uplo), O(orient), D(diag), T, X);  // blas-like/level2/Trsv.hpp:20-44
  });
}

EREF int eref_dgemm(int oa, int ob, int m, int n, int k, double alpha, const double* A, int lda, const double* B,
                    int ldb, double beta, double* C, int ldc) {
  return guarded([&] {
    elem::Matrix<double> MA, MB, MC;
    MA.LockedAttach(oa == 0 ? m : k, oa == 0 ? k : m, A, lda);
    MB.LockedAttach(ob == 0 ? k : n, ob == 0 ? n : k, B, ldb);
    MC.Attach(m, n, C, ldc);
    elem::Gemm(O(oa), O(ob), alpha, MA, MB, beta, MC);  // blas-like/level3/Gemm.hpp:158-211
  });
}

EREF int eref_dherk(int uplo, int orient, int n, int k, double alpha, const double* A, int lda, double beta,
                    double* C, int ldc) {
  return guarded([&] {
    elem::Matrix<double> MA, MC;
    MA.LockedAttach(orient == 0 ? n : k, orient == 0 ? k : n, A, lda);
    MC.Attach(n, n, C, ldc);
    elem::Herk(U(uplo), O(orient), alpha, MA, beta, MC);  // blas-like/level3/Herk.hpp:17-27
  });
}

EREF int eref_dtriangular_inverse(int uplo, int diag, int n, double* A, int lda, int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::Matrix<double> M;
    M.Attach(n, n, A, lda);
    elem::TriangularInverse(U(uplo), D(diag), M);  // lapack-like/TriangularInverse.hpp:56-64
  });
}

EREF int eref_dinverse(int n, double* A, int lda, int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::Matrix<double> M;
    M.Attach(n, n, A, lda);
    elem::Inverse(M);  // lapack-like/Inverse.hpp:17-23
  });
}

EREF int eref_dhpd_inverse(int uplo, int n, double* A, int lda, int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::Matrix<double> M;
    M.Attach(n, n, A, lda);
    elem::HPDInverse(U(uplo), M);  // lapack-like/Inverse.hpp:25-35
  });
}

EREF int eref_dldl(int orient, int n, double* A, int lda, double* d, int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::Matrix<double> M, dv;
    M.Attach(n, n, A, lda);
    dv.Attach(n, 1, d, n > 0 ? n : 1);
    if (orient == 2) elem::LDLH(M, dv);  // lapack-like/LDL.hpp
    else elem::LDLT(M, dv);
  });
}

EREF int eref_dsafe_determinant(int hpd, int uplo, int n, const double* A, int lda, int nb, double* rho,
                                double* kappa) {
  return guarded([&] {
    set_nb(nb);
    elem::Matrix<double> M;
    M.LockedAttach(n, n, A, lda);
    elem::SafeProduct<double> s = hpd ? elem::SafeHPDDeterminant(U(uplo), M) : elem::SafeDeterminant(M);
    *rho = s.rho;
    *kappa = s.kappa;  // lapack-like/Determinant.hpp
  });
}

// ---- the same entry points on a DistMatrix over a 1 x 1 Grid -----------

EREF int eref_dist_dcholesky(int uplo, int n, double* A, int lda, int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::DistMatrix<double> D(elem::DefaultGrid());
    to_dist(D, n, n, A, lda);
    elem::Cholesky(U(uplo), D);  // Cholesky.hpp:79-101 -> cholesky::LVar3Square
    from_dist(D, A, lda);
  });
}

EREF int eref_dist_dhpd_solve(int uplo, int orient, int n, int nrhs, double* A, int lda, double* B, int ldb,
                              int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::DistMatrix<double> DA(elem::DefaultGrid()), DB(elem::DefaultGrid());
    to_dist(DA, n, n, A, lda);
    to_dist(DB, n, nrhs, B, ldb);
    elem::HPDSolve(U(uplo), O(orient), DA, DB);  // HPDSolve.hpp:30-41
    from_dist(DA, A, lda);
    from_dist(DB, B, ldb);
  });
}

EREF int eref_dist_dlu(int m, int n, double* A, int lda, int* p, int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::DistMatrix<double> DA(elem::DefaultGrid());
    elem::DistMatrix<int, elem::VC, elem::STAR> P(elem::DefaultGrid());
    to_dist(DA, m, n, A, lda);
    elem::LU(DA, P);  // LU.hpp:220-321 (dist lu::Panel with PivotOp, LU/Panel.hpp:91-264)
    from_dist(DA, A, lda);
    from_dist(P, p, P.Height() > 0 ? P.Height() : 1);
  });
}

EREF int eref_dist_dlu_solve_after(int orient, int n, int nrhs, const double* A, int lda, const int* p, double* B,
                                   int ldb) {
  return guarded([&] {
    elem::DistMatrix<double> DA(elem::DefaultGrid()), DB(elem::DefaultGrid());
    elem::DistMatrix<int, elem::VC, elem::STAR> P(elem::DefaultGrid());
    to_dist(DA, n, n, A, lda);
    to_dist(P, n, 1, p, n > 0 ? n : 1);
    to_dist(DB, n, nrhs, B, ldb);
    elem::lu::SolveAfter(O(orient), DA, P, DB);  // LU/SolveAfter.hpp:148-195
    from_dist(DB, B, ldb);
  });
}

EREF int eref_dist_dgaussian_elimination(int n, int nrhs, double* A, int lda, double* B, int ldb, int nb) {
  return guarded([&] {
    set_nb(nb);
    elem::DistMatrix<double> DA(elem::DefaultGrid()), DB(elem::DefaultGrid());
    to_dist(DA, n, n, A, lda);
    to_dist(DB, n, nrhs, B, ldb);
    elem::GaussianElimination(DA, DB);  // GaussianElimination.hpp:234-252 (dist RowEchelon :94-209)
    from_dist(DA, A, lda);
    from_dist(DB, B, ldb);
  });
}

// The BLAS build the reference's level-3 calls land in (OpenBLAS config text).
extern "C" const char* scipy_openblas_get_config(void);
EREF const char* eref_blas_config(void) { return scipy_openblas_get_config(); }
