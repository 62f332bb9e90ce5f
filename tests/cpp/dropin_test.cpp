// Drop-in check written the way the reference's own drivers are
// (tests/lapack-like/Cholesky.cpp, tests/lapack-like/SequentialLU.cpp):
// factor with elem::Cholesky / elem::LU, then apply the factors to a block of
// random vectors and compare against A X.  Exercises Matrix<F> views with
// LDim > Height, the Blocksize stack, DistMatrix on a 1 x 1 Grid, float and
// double, and the exception mapping.  Prints one line per check and exits
// non-zero on the first failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>

#include "elemgpu/elemental.hpp"

using namespace elem;

static std::mt19937_64 gen(12345);

template <typename F>
void Uniform(Matrix<F>& A, int m, int n) {  // U[-1,1], like matrices/Uniform.hpp
  A.ResizeTo(m, n);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) A.Set(i, j, (F)u(gen));
}

template <typename F>
double MaxAbs(const Matrix<F>& A) {
  double r = 0;
  for (int j = 0; j < A.Width(); ++j)
    for (int i = 0; i < A.Height(); ++i) r = std::max(r, std::fabs((double)A.Get(i, j)));
  return r;
}

static int failures = 0;
static void Check(bool ok, const char* what, double value) {
  std::printf("%-48s %s  (%.3e)\n", what, ok ? "ok" : "FAIL", value);
  if (!ok) ++failures;
}

template <typename F>
void TestCholesky(UpperOrLower uplo, int m, double tol) {
  // HPD A = G G^T + m I
  Matrix<F> G, A(m, m), X, Y(m, 100), Z(m, 100);
  Uniform(G, m, m);
  Gemm(NORMAL, TRANSPOSE, F(1), G, G, F(0), A);
  for (int i = 0; i < m; ++i) A.Update(i, i, F(m));
  Uniform(X, m, 100);
  Gemm(NORMAL, NORMAL, F(1), A, X, F(0), Y);  // Y = A X
  Matrix<F> L(A);
  Cholesky(uplo, L);
  // Z = L L^H X (or U^H U X) applied with triangular products built from L
  Matrix<F> T(m, m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) {
      const bool in = uplo == LOWER ? i >= j : i <= j;
      T.Set(i, j, in ? L.Get(i, j) : F(0));
    }
  Matrix<F> W(m, 100);
  if (uplo == LOWER) {
    Gemm(TRANSPOSE, NORMAL, F(1), T, X, F(0), W);
    Gemm(NORMAL, NORMAL, F(1), T, W, F(0), Z);
  } else {
    Gemm(NORMAL, NORMAL, F(1), T, X, F(0), W);
    Gemm(TRANSPOSE, NORMAL, F(1), T, W, F(0), Z);
  }
  double err = 0;
  for (int j = 0; j < 100; ++j)
    for (int i = 0; i < m; ++i) err = std::max(err, std::fabs((double)(Y.Get(i, j) - Z.Get(i, j))));
  Check(err / MaxAbs(Y) < tol, uplo == LOWER ? "Cholesky(LOWER) ||AX - LL^H X|| / ||AX||" : "Cholesky(UPPER)", err / MaxAbs(Y));
  // HPDSolve on the same A recovers X
  Matrix<F> A2(A), B(Y);
  HPDSolve(uplo, NORMAL, A2, B);
  double e2 = 0;
  for (int j = 0; j < 100; ++j)
    for (int i = 0; i < m; ++i) e2 = std::max(e2, std::fabs((double)(B.Get(i, j) - X.Get(i, j))));
  Check(e2 < tol * 10, "HPDSolve recovers X", e2);
}

template <typename F>
void TestLU(int m, double tol) {
  Matrix<F> A, X, Y(m, 100);
  Uniform(A, m, m);
  Uniform(X, m, 100);
  Gemm(NORMAL, NORMAL, F(1), A, X, F(0), Y);
  Matrix<F> LU_(A);
  Matrix<int> p;
  LU(LU_, p);
  Check(p.Height() == m && p.Width() == 1, "LU resizes p to min(m,n) x 1", p.Height());
  Matrix<F> B(Y);
  lu::SolveAfter(NORMAL, LU_, p, B);
  double e = 0;
  for (int j = 0; j < 100; ++j)
    for (int i = 0; i < m; ++i) e = std::max(e, std::fabs((double)(B.Get(i, j) - X.Get(i, j))));
  Check(e < tol * m, "LU + lu::SolveAfter recovers X", e);
  Matrix<F> A3(A), B3(Y);
  GaussianElimination(A3, B3);
  double e3 = 0;
  for (int j = 0; j < 100; ++j)
    for (int i = 0; i < m; ++i) e3 = std::max(e3, std::fabs((double)(B3.Get(i, j) - X.Get(i, j))));
  Check(e3 < tol * m, "GaussianElimination recovers X", e3);
}

// --dist-dump DIR: run the 1 x 1 DistMatrix overloads (and Trsv on a
// Matrix) on the inputs DIR/spd.bin, DIR/ge.bin (n x n) and DIR/rhs.bin
// (n x k), each a header {rows, cols} of int32 followed by the column-major
// doubles, and write every result to DIR/<name>.bin in the same format; the
// Python side compares them with the oracle.
static Matrix<double> ReadBin(const std::string& path) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) { std::printf("cannot open %s\n", path.c_str()); std::exit(2); }
  int hw[2] = {0, 0};
  if (std::fread(hw, sizeof(int), 2, f) != 2) std::exit(2);
  Matrix<double> A(hw[0], hw[1]);
  for (int j = 0; j < hw[1]; ++j)
    if (std::fread(A.Buffer(0, j), sizeof(double), hw[0], f) != (size_t)hw[0]) std::exit(2);
  std::fclose(f);
  return A;
}

template <typename T>
static void WriteBin(const std::string& path, const Matrix<T>& A) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) std::exit(2);
  const int hw[2] = {A.Height(), A.Width()};
  std::fwrite(hw, sizeof(int), 2, f);
  for (int j = 0; j < A.Width(); ++j) std::fwrite(A.LockedBuffer(0, j), sizeof(T), A.Height(), f);
  std::fclose(f);
}

static int DistDump(const std::string& dir) {
  Grid g;
  const Matrix<double> spd = ReadBin(dir + "/spd.bin"), ge = ReadBin(dir + "/ge.bin"), rhs = ReadBin(dir + "/rhs.bin");
  for (UpperOrLower uplo : {LOWER, UPPER}) {
    const char* u = uplo == LOWER ? "L" : "U";
    DistMatrix<double> A(g), B(g), X(g);
    A.Matrix() = spd;
    Cholesky(uplo, A);  // Cholesky.hpp:79-101
    WriteBin(dir + "/chol_" + u + ".bin", A.LockedMatrix());
    X.Matrix() = rhs;
    cholesky::SolveAfter(uplo, NORMAL, A, X);  // Cholesky/SolveAfter.hpp:77-134
    WriteBin(dir + "/solveafter_" + u + ".bin", X.LockedMatrix());
    A.Matrix() = spd;
    B.Matrix() = rhs;
    HPDSolve(uplo, NORMAL, A, B);  // HPDSolve.hpp:30-41
    WriteBin(dir + "/hpdsolve_" + u + ".bin", B.LockedMatrix());
  }
  {
    DistMatrix<double> A(g), B(g);
    DistMatrix<int, VC, STAR> p(g);
    A.Matrix() = ge;
    LU(A, p);  // LU.hpp:220-321
    WriteBin(dir + "/lu.bin", A.LockedMatrix());
    WriteBin(dir + "/lu_p.bin", p.LockedMatrix());
    B.Matrix() = rhs;
    lu::SolveAfter(NORMAL, A, p, B);  // LU/SolveAfter.hpp:148-195
    WriteBin(dir + "/lusolve.bin", B.LockedMatrix());
    A.Matrix() = ge;
    B.Matrix() = rhs;
    GaussianElimination(A, B);  // GaussianElimination.hpp:234-252
    WriteBin(dir + "/gauss.bin", B.LockedMatrix());
  }
  for (UpperOrLower uplo : {LOWER, UPPER})
    for (Orientation o : {NORMAL, TRANSPOSE}) {
      Matrix<double> x(rhs.Height(), 1);
      for (int i = 0; i < rhs.Height(); ++i) x.Set(i, 0, rhs.Get(i, 0));
      Trsv(uplo, o, NON_UNIT, spd, x);  // Trsv.hpp:20-44
      WriteBin(dir + "/trsv_" + (uplo == LOWER ? "L" : "U") + (o == NORMAL ? "N" : "T") + ".bin", x);
    }
  std::printf("DUMPED\n");
  return 0;
}

int main(int argc, char** argv) {
  Initialize(argc, argv);
  if (argc == 3 && std::string(argv[1]) == "--dist-dump") {
    const int rc = DistDump(argv[2]);
    Finalize();
    return rc;
  }
  PushBlocksizeStack(96);
  TestCholesky<double>(LOWER, 500, 1e-12);
  TestCholesky<double>(UPPER, 333, 1e-12);
  PopBlocksizeStack();
  TestCholesky<float>(LOWER, 200, 1e-5);
  TestLU<double>(700, 1e-12);
  TestLU<float>(150, 1e-5);

  // A view with LDim > Height: factor the leading 300 x 300 block in place.
  {
    Matrix<double> big(400, 400);
    Matrix<double> G;
    Uniform(G, 300, 300);
    Matrix<double> view;
    View(view, big, 50, 60, 300, 300);
    Gemm(NORMAL, TRANSPOSE, 1.0, G, G, 0.0, view);
    for (int i = 0; i < 300; ++i) view.Update(i, i, 300.0);
    Matrix<double> copy(view);
    Cholesky(LOWER, view);
    Cholesky(LOWER, copy);
    double d = 0;
    for (int j = 0; j < 300; ++j)
      for (int i = j; i < 300; ++i) d = std::max(d, std::fabs(view.Get(i, j) - copy.Get(i, j)));
    Check(d == 0.0 && big.Get(0, 0) == 0.0 && big.Get(49, 60) == 0.0, "Cholesky on a view (LDim 400)", d);
  }

  // DistMatrix over a 1 x 1 Grid delegates to the sequential path.
  {
    Grid g;
    DistMatrix<double> A(g), B(g);
    Uniform(A.Matrix(), 256, 256);
    for (int i = 0; i < 256; ++i) A.Matrix().Update(i, i, 256.0);
    Uniform(B.Matrix(), 256, 4);
    DistMatrix<double> A0(A), B0(B);
    DistMatrix<int, VC, STAR> p(g);
    LU(A, p);
    lu::SolveAfter(NORMAL, A, p, B);
    Matrix<double> R(256, 4);
    Gemm(NORMAL, NORMAL, 1.0, A0.LockedMatrix(), B.LockedMatrix(), 0.0, R);
    double e = 0;
    for (int j = 0; j < 4; ++j)
      for (int i = 0; i < 256; ++i) e = std::max(e, std::fabs(R.Get(i, j) - B0.Get(i, j)));
    Check(e < 1e-11, "DistMatrix 1x1 LU + SolveAfter", e);
  }

  // Exceptions: non-HPD -> std::logic_error, exact zero pivot -> SingularMatrixException
  {
    Matrix<double> A(50, 50);
    for (int i = 0; i < 50; ++i) A.Set(i, i, i == 30 ? -1.0 : 2.0);
    bool caught = false;
    try { Cholesky(LOWER, A); } catch (std::logic_error& e) { caught = std::string(e.what()) == "A was not numerically HPD"; }
    Check(caught, "Cholesky throws logic_error on non-HPD input", 0);
    Matrix<double> S;
    Uniform(S, 40, 40);
    for (int i = 0; i < 40; ++i) S.Set(i, 7, 0.0);
    Matrix<int> p;
    caught = false;
    try { LU(S, p); } catch (SingularMatrixException&) { caught = true; }
    Check(caught, "LU throws SingularMatrixException", 0);
  }
  // Inverse / HPDInverse / TriangularInverse / (Safe)Determinant, checked by
  // identities: A inv(A) = I, det(A) det(inv(A)) = 1, SafeHPDDeterminant and
  // SafeDeterminant agree on an HPD matrix, a unit triangular inverse keeps
  // the diagonal and the other triangle.
  {
    const int m = 300;
    Matrix<double> A, Ai;
    Uniform(A, m, m);
    for (int i = 0; i < m; ++i) A.Update(i, i, 4.0);
    Ai = A;
    Inverse(Ai);
    Matrix<double> I(m, m);
    Gemm(NORMAL, NORMAL, 1.0, A, Ai, 0.0, I);
    double e = 0;
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) e = std::max(e, std::fabs(I.Get(i, j) - (i == j ? 1.0 : 0.0)));
    Check(e < 1e-12, "Inverse: A inv(A) = I", e);
    SafeProduct<double> d1 = SafeDeterminant(A), d2 = SafeDeterminant(Ai);
    const double s = d1.kappa * d1.n + d2.kappa * d2.n;
    Check(d1.rho * d2.rho == 1.0 && std::fabs(s) < 1e-9, "SafeDeterminant: det(A) det(inv(A)) = 1", s);

    Matrix<double> G, S(m, m), Si;
    Uniform(G, m, m);
    Gemm(NORMAL, TRANSPOSE, 1.0, G, G, 0.0, S);
    for (int i = 0; i < m; ++i) S.Update(i, i, (double)m);
    SafeProduct<double> h = SafeHPDDeterminant(LOWER, S), g = SafeDeterminant(S);
    Check(h.rho == 1.0 && g.rho == 1.0 && std::fabs(h.kappa - g.kappa) < 1e-12 * std::fabs(g.kappa),
          "SafeHPDDeterminant = SafeDeterminant on HPD", std::fabs(h.kappa - g.kappa));
    Si = S;
    HPDInverse(UPPER, Si);
    double eh = 0;  // (S inv(S))_ij from the upper triangle of inv(S) mirrored
    Matrix<double> Sym(m, m);
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) Sym.Set(i, j, i <= j ? Si.Get(i, j) : Si.Get(j, i));
    Gemm(NORMAL, NORMAL, 1.0, S, Sym, 0.0, I);
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) eh = std::max(eh, std::fabs(I.Get(i, j) - (i == j ? 1.0 : 0.0)));
    bool lower_kept = true;
    for (int j = 0; j < m; ++j)
      for (int i = j + 1; i < m; ++i) lower_kept = lower_kept && Si.Get(i, j) == S.Get(i, j);
    Check(eh < 1e-12 && lower_kept, "HPDInverse(UPPER): S inv(S) = I, lower kept", eh);

    Matrix<double> T = A, Ti;  // strictly lower part scaled by 1/m: well conditioned
    for (int j = 0; j < m; ++j)
      for (int i = j + 1; i < m; ++i) T.Set(i, j, A.Get(i, j) / m);
    Ti = T;
    TriangularInverse(LOWER, UNIT, Ti);
    bool kept = true;
    for (int j = 0; j < m; ++j)
      for (int i = 0; i <= j; ++i) kept = kept && Ti.Get(i, j) == T.Get(i, j);
    double et = 0;  // (unit L) inv(unit L) = I
    for (int j = 0; j < m; ++j)
      for (int i = j; i < m; ++i) {
        double acc = 0;
        for (int k = j; k <= i; ++k)
          acc += (k == i ? 1.0 : T.Get(i, k)) * (k == j ? 1.0 : Ti.Get(k, j));
        et = std::max(et, std::fabs(acc - (i == j ? 1.0 : 0.0)));
      }
    Check(kept && et < 1e-10, "TriangularInverse(LOWER, UNIT)", et);

    Matrix<double> R = S;  // ReverseCholesky(LOWER): S = L^T L
    ReverseCholesky(LOWER, R);
    double er = 0;
    for (int j = 0; j < m; ++j)
      for (int i = j; i < m; ++i) {
        double acc = 0;
        for (int k = i; k < m; ++k) acc += R.Get(k, i) * R.Get(k, j);
        er = std::max(er, std::fabs(acc - S.Get(i, j)));
      }
    Check(er < 1e-9 * m, "ReverseCholesky(LOWER): L^T L = S", er);

    Matrix<double> Ld = S, dd;  // LDLT of the HPD S: D > 0 and L D L^T = S
    LDLT(Ld, dd);
    double el = 0;
    bool dpos = dd.Height() == m;
    for (int i = 0; i < m && dpos; ++i) dpos = dd.Get(i, 0) > 0 && dd.Get(i, 0) == Ld.Get(i, i);
    for (int j = 0; j < m; j += 7)
      for (int i = j; i < m; ++i) {
        double acc = 0;
        for (int k = 0; k <= j; ++k) acc += (k == i ? 1.0 : Ld.Get(i, k)) * dd.Get(k, 0) * (k == j ? 1.0 : Ld.Get(j, k));
        el = std::max(el, std::fabs(acc - S.Get(i, j)));
      }
    Check(dpos && el < 1e-9 * m, "LDLT: L D L^T = S, d = diag", el);

    Matrix<double> Z;
    Uniform(Z, 20, 20);
    for (int i = 0; i < 20; ++i) Z.Set(i, 5, 0.0);
    SafeProduct<double> z = SafeDeterminant(Z);
    Check(z.rho == 0.0 && z.kappa == 0.0, "SafeDeterminant of a singular matrix is 0", 0);
  }
  Finalize();
  std::printf("%s\n", failures ? "FAILED" : "PASSED");
  return failures ? 1 : 0;
}
