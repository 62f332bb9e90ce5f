// elemgpu/elemental.hpp -- drop-in C++ front end for Elemental's dense
// factor-and-solve path, backed by the sm_100a kernels through the C ABI in
// elemgpu.h.
//
// It mirrors the names, argument meanings and error behaviour of Elemental's
// own templates so that code written against the reference compiles
// unchanged for this path:
//   Matrix<T>                      core/matrix.hpp:16-183 (column-major, LDim, views)
//   Grid / DistMatrix<T,U,V>       core/grid_decl.hpp:16-103, core/dist_matrix.hpp
//                                  (1 x 1 grid only: every process owns its whole matrix)
//   Blocksize / SetBlocksize / PushBlocksizeStack / PopBlocksizeStack
//                                  src/core/global.cpp:277-287 (default 128, :194)
//   Cholesky, LU, HPDSolve, GaussianElimination, cholesky::SolveAfter,
//   lu::SolveAfter, Trsm, Trsv, Gemm, Herk, Syrk, ApplyRowPivots,
//   ApplyInverseRowPivots          lapack-like/*.hpp, blas-like/level{2,3}/*.hpp
//   SingularMatrixException, NonHPDMatrixException  core/environment_decl.hpp:232-245
//
// F = double runs the FP64 kernels directly.  F = float is promoted to double
// on the host, factored/solved by the FP64 kernels and rounded back (results
// are at least as accurate as a float LAPACK).  Complex F is not provided.
//
// Calls are synchronous, like the reference's.  Each host thread owns one
// egpu handle (created on first use on device 0, or on the device chosen by
// SetDevice before that).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stack>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../elemgpu.h"

namespace elem {

// ----------------------------------------------------------- enums -------
enum UpperOrLower { LOWER, UPPER };
enum Orientation { NORMAL, TRANSPOSE, ADJOINT };
enum LeftOrRight { LEFT, RIGHT };
enum UnitOrNonUnit { NON_UNIT, UNIT };
enum Distribution { MC, MD, MR, VC, VR, STAR, CIRC };

// ------------------------------------------------------- exceptions ------
class SingularMatrixException : public std::runtime_error {
 public:
  SingularMatrixException(const char* msg = "Matrix was singular") : std::runtime_error(msg) {}
};
class NonHPDMatrixException : public std::runtime_error {
 public:
  NonHPDMatrixException(const char* msg = "Matrix was not HPD") : std::runtime_error(msg) {}
};

// ------------------------------------------------------ environment ------
namespace detail {

struct HandleHolder {
  egpu_handle h = nullptr;
  int device = 0;
  ~HandleHolder() {
    if (h) egpu_destroy(h);
  }
};

inline HandleHolder& holder() {
  static thread_local HandleHolder H;
  return H;
}

inline std::stack<int>& blocksize_stack() {
  static thread_local std::stack<int> s;
  if (s.empty()) s.push(128);
  return s;
}

inline egpu_handle handle() {
  HandleHolder& H = holder();
  if (!H.h) {
    int rc = egpu_create(&H.h, H.device);
    if (rc != EGPU_OK) throw std::runtime_error(std::string("elemgpu: ") + egpu_error_string(rc));
  }
  egpu_set_blocksize(H.h, blocksize_stack().top());
  return H.h;
}

// Map a C-ABI return code to the reference's exception types.
inline void check(int rc, int info = 0) {
  switch (rc) {
    case EGPU_OK: return;
    case EGPU_NOT_HPD:  // Cholesky/LVar3.hpp:37-38 throws std::logic_error
      throw std::logic_error("A was not numerically HPD");
    case EGPU_SINGULAR:  // LU/Panel.hpp:76-77
      throw SingularMatrixException();
    default: {
      std::string msg = std::string("elemgpu: ") + egpu_error_string(rc);
      const char* d = egpu_last_error_detail();
      if (d && *d) msg += std::string(" (") + d + ")";
      (void)info;
      throw std::runtime_error(msg);
    }
  }
}

}  // namespace detail

inline void Initialize(int&, char**&) {}
inline void Finalize() {
  detail::HandleHolder& H = detail::holder();
  if (H.h) {
    egpu_destroy(H.h);
    H.h = nullptr;
  }
}
inline bool Initialized() { return true; }
// Choose the CUDA device used by this thread's handle (before the first call).
inline void SetDevice(int device) { detail::holder().device = device; }

inline int Blocksize() { return detail::blocksize_stack().top(); }
inline void SetBlocksize(int blocksize) { detail::blocksize_stack().top() = blocksize; }
inline void PushBlocksizeStack(int blocksize) { detail::blocksize_stack().push(blocksize); }
inline void PopBlocksizeStack() {
  if (detail::blocksize_stack().size() > 1) detail::blocksize_stack().pop();
}

// ------------------------------------------------------------ Matrix -----
template <typename T, typename Int = int>
class Matrix {
 public:
  Matrix(bool fixed = false) : fixed_(fixed) {}
  Matrix(Int height, Int width, bool fixed = false) : fixed_(fixed) { ResizeTo(height, width); }
  Matrix(Int height, Int width, Int ldim, bool fixed = false) : fixed_(fixed) { ResizeTo(height, width, ldim); }
  Matrix(Int height, Int width, const T* buffer, Int ldim, bool fixed = false)
      : height_(height), width_(width), ldim_(ldim), data_(const_cast<T*>(buffer)), viewing_(true), locked_(true),
        fixed_(fixed) {
    CheckDims(height, width, ldim);
  }
  Matrix(Int height, Int width, T* buffer, Int ldim, bool fixed = false)
      : height_(height), width_(width), ldim_(ldim), data_(buffer), viewing_(true), fixed_(fixed) {
    CheckDims(height, width, ldim);
  }
  Matrix(const Matrix& A) { *this = A; }

  Int Height() const { return height_; }
  Int Width() const { return width_; }
  Int LDim() const { return ldim_; }
  Int MemorySize() const { return (Int)memory_.size(); }
  Int DiagonalLength(Int offset = 0) const {
    return offset >= 0 ? std::max<Int>(0, std::min(height_, width_ - offset))
                       : std::max<Int>(0, std::min(height_ + offset, width_));
  }

  T* Buffer() {
    if (locked_) throw std::logic_error("Cannot return non-const buffer of locked Matrix");
    return data_;
  }
  T* Buffer(Int i, Int j) { return Buffer() + i + j * ldim_; }
  const T* LockedBuffer() const { return data_; }
  const T* LockedBuffer(Int i, Int j) const { return data_ + i + j * ldim_; }

  T Get(Int i, Int j) const { return data_[i + j * ldim_]; }
  void Set(Int i, Int j, T alpha) { Buffer()[i + j * ldim_] = alpha; }
  void Update(Int i, Int j, T alpha) { Buffer()[i + j * ldim_] += alpha; }

  bool Owner() const { return !viewing_; }
  bool Viewing() const { return viewing_; }
  bool Locked() const { return locked_; }
  bool FixedSize() const { return fixed_; }

  void Attach(Int height, Int width, T* buffer, Int ldim) {
    CheckDims(height, width, ldim);
    memory_.clear();
    height_ = height; width_ = width; ldim_ = ldim; data_ = buffer; viewing_ = true; locked_ = false;
  }
  void LockedAttach(Int height, Int width, const T* buffer, Int ldim) {
    CheckDims(height, width, ldim);
    memory_.clear();
    height_ = height; width_ = width; ldim_ = ldim; data_ = const_cast<T*>(buffer); viewing_ = true;
    locked_ = true;
  }

  const Matrix& operator=(const Matrix& A) {
    if (this == &A) return *this;
    if (viewing_ && (height_ != A.height_ || width_ != A.width_))
      throw std::logic_error("Cannot assign to a view of different dimensions");
    if (!viewing_) ResizeTo(A.height_, A.width_);
    for (Int j = 0; j < width_; ++j)
      std::memcpy(data_ + j * ldim_, A.data_ + j * A.ldim_, sizeof(T) * height_);
    return *this;
  }

  void Empty() {
    memory_.clear();
    height_ = width_ = 0; ldim_ = 1; data_ = nullptr; viewing_ = locked_ = false;
  }
  void ResizeTo(Int height, Int width) { ResizeTo(height, width, std::max<Int>(height, 1)); }
  void ResizeTo(Int height, Int width, Int ldim) {
    CheckDims(height, width, ldim);
    if (viewing_ && (height > height_ || width > width_ || ldim != ldim_))
      throw std::logic_error("Cannot increase the size of a view");
    height_ = height; width_ = width;
    if (!viewing_) {
      ldim_ = ldim;
      memory_.assign((size_t)ldim * std::max<Int>(width, 1), T(0));
      data_ = memory_.data();
    }
  }

 private:
  static void CheckDims(Int h, Int w, Int ld) {
    if (h < 0 || w < 0) throw std::logic_error("Height and width must be non-negative");
    if (ld < h || ld < 1) throw std::logic_error("Leading dimension must be no less than height and at least 1");
  }
  template <typename U, typename I2> friend void View(Matrix<U, I2>&, Matrix<U, I2>&, I2, I2, I2, I2);
  template <typename U, typename I2> friend void LockedView(Matrix<U, I2>&, const Matrix<U, I2>&, I2, I2, I2, I2);

  Int height_ = 0, width_ = 0, ldim_ = 1;
  T* data_ = nullptr;
  std::vector<T> memory_;
  bool viewing_ = false, locked_ = false, fixed_ = false;
};

// View(A, B, i, j, height, width): A views a block of B (core/view_decl.hpp).
template <typename T, typename Int>
inline void View(Matrix<T, Int>& A, Matrix<T, Int>& B, Int i, Int j, Int height, Int width) {
  if (i < 0 || j < 0 || i + height > B.Height() || j + width > B.Width())
    throw std::logic_error("Trying to view outside of a Matrix");
  A.Attach(height, width, B.Buffer(i, j), B.LDim());
}
template <typename T, typename Int>
inline void LockedView(Matrix<T, Int>& A, const Matrix<T, Int>& B, Int i, Int j, Int height, Int width) {
  if (i < 0 || j < 0 || i + height > B.Height() || j + width > B.Width())
    throw std::logic_error("Trying to view outside of a Matrix");
  A.LockedAttach(height, width, B.LockedBuffer(i, j), B.LDim());
}

// -------------------------------------------------- Grid / DistMatrix ---
// Only the 1 x 1 grid of this path: one process owns every entry, so each
// DistMatrix overload delegates to the sequential routine on A.Matrix(), the
// same local computation the reference performs when p = 1.
class Grid {
 public:
  Grid() = default;
  int Row() const { return 0; }
  int Col() const { return 0; }
  int Rank() const { return 0; }
  int Height() const { return 1; }
  int Width() const { return 1; }
  int Size() const { return 1; }
  bool InGrid() const { return true; }
  bool operator==(const Grid&) const { return true; }
  bool operator!=(const Grid&) const { return false; }
};

inline const Grid& DefaultGrid() {
  static Grid g;
  return g;
}

template <typename T, Distribution U = MC, Distribution V = MR, typename Int = int>
class DistMatrix {
 public:
  explicit DistMatrix(const elem::Grid& g = DefaultGrid()) : grid_(&g) {}
  DistMatrix(Int height, Int width, const elem::Grid& g = DefaultGrid()) : grid_(&g), local_(height, width) {}
  template <Distribution U2, Distribution V2>
  DistMatrix(const DistMatrix<T, U2, V2, Int>& A) : grid_(&A.Grid()), local_(A.LockedMatrix()) {}

  const elem::Grid& Grid() const { return *grid_; }
  Int Height() const { return local_.Height(); }
  Int Width() const { return local_.Width(); }
  Int LocalHeight() const { return local_.Height(); }
  Int LocalWidth() const { return local_.Width(); }
  Int LDim() const { return local_.LDim(); }
  Int ColShift() const { return 0; }
  Int RowShift() const { return 0; }
  bool Viewing() const { return local_.Viewing(); }
  T Get(Int i, Int j) const { return local_.Get(i, j); }
  void Set(Int i, Int j, T a) { local_.Set(i, j, a); }
  void ResizeTo(Int h, Int w) { local_.ResizeTo(h, w); }
  elem::Matrix<T, Int>& Matrix() { return local_; }
  const elem::Matrix<T, Int>& LockedMatrix() const { return local_; }

 private:
  const elem::Grid* grid_;
  elem::Matrix<T, Int> local_;
};

// -------------------------------------------------------- internals -----
namespace detail {

template <typename F>
struct IsSupported : std::integral_constant<bool, std::is_same<F, double>::value || std::is_same<F, float>::value> {};

// Promote a float matrix to a packed double copy; write back on destruction.
template <typename F>
struct AsDouble;

template <>
struct AsDouble<double> {
  double* p;
  int ld;
  AsDouble(const Matrix<double>& A, bool) : p(const_cast<double*>(A.LockedBuffer())), ld(A.LDim()) {}
  void WriteBack(Matrix<double>&) {}
};

template <>
struct AsDouble<float> {
  std::vector<double> buf;
  double* p;
  int ld;
  AsDouble(const Matrix<float>& A, bool) {
    ld = std::max(A.Height(), 1);
    buf.resize((size_t)ld * std::max(A.Width(), 1));
    for (int j = 0; j < A.Width(); ++j)
      for (int i = 0; i < A.Height(); ++i) buf[i + (size_t)j * ld] = A.Get(i, j);
    p = buf.data();
  }
  void WriteBack(Matrix<float>& A) {
    for (int j = 0; j < A.Width(); ++j)
      for (int i = 0; i < A.Height(); ++i) A.Set(i, j, (float)buf[i + (size_t)j * ld]);
  }
};

inline int Ori(Orientation o) { return o == NORMAL ? EGPU_NORMAL : (o == TRANSPOSE ? EGPU_TRANSPOSE : EGPU_ADJOINT); }

}  // namespace detail

// ---------------------------------------------------- BLAS-like (L3) -----

// Gemm(orientA, orientB, alpha, A, B, beta, C), blas-like/level3/Gemm.hpp:158-211.
template <typename T>
inline void Gemm(Orientation oA, Orientation oB, T alpha, const Matrix<T>& A, const Matrix<T>& B, T beta,
                 Matrix<T>& C) {
  static_assert(detail::IsSupported<T>::value, "elemgpu supports float and double");
  const int m = C.Height(), n = C.Width();
  const int k = oA == NORMAL ? A.Width() : A.Height();
  if ((oA == NORMAL ? A.Height() : A.Width()) != m || (oB == NORMAL ? B.Width() : B.Height()) != n ||
      (oB == NORMAL ? B.Height() : B.Width()) != k)
    throw std::logic_error("Nonconformal Gemm");
  detail::AsDouble<T> a(A, false), b(B, false), c(C, true);
  detail::check(egpu_host_dgemm(detail::handle(), detail::Ori(oA), detail::Ori(oB), m, n, k, (double)alpha, a.p,
                                a.ld, b.p, b.ld, (double)beta, c.p, c.ld));
  c.WriteBack(C);
}

// Herk(uplo, orientation, alpha, A, beta, C), blas-like/level3/Herk.hpp:17-27
// (real F: Syrk, Syrk.hpp:20-57).
template <typename T>
inline void Herk(UpperOrLower uplo, Orientation orientation, T alpha, const Matrix<T>& A, T beta, Matrix<T>& C) {
  static_assert(detail::IsSupported<T>::value, "elemgpu supports float and double");
  const int n = C.Height();
  const int k = orientation == NORMAL ? A.Width() : A.Height();
  if (C.Width() != n || (orientation == NORMAL ? A.Height() : A.Width()) != n)
    throw std::logic_error("Nonconformal Herk");
  detail::AsDouble<T> a(A, false), c(C, true);
  detail::check(egpu_host_dherk(detail::handle(), uplo == LOWER ? EGPU_LOWER : EGPU_UPPER, detail::Ori(orientation),
                                n, k, (double)alpha, a.p, a.ld, (double)beta, c.p, c.ld));
  c.WriteBack(C);
}

template <typename T>
inline void Syrk(UpperOrLower uplo, Orientation orientation, T alpha, const Matrix<T>& A, T beta, Matrix<T>& C) {
  Herk(uplo, orientation, alpha, A, beta, C);
}

// Trsm(side, uplo, orientation, diag, alpha, A, B, checkIfSingular),
// blas-like/level3/Trsm.hpp:49-86.
template <typename F>
inline void Trsm(LeftOrRight side, UpperOrLower uplo, Orientation orientation, UnitOrNonUnit diag, F alpha,
                 const Matrix<F>& A, Matrix<F>& B, bool checkIfSingular = false) {
  static_assert(detail::IsSupported<F>::value, "elemgpu supports float and double");
  if (A.Height() != A.Width()) throw std::logic_error("Triangular matrix must be square");
  if ((side == LEFT ? B.Height() : B.Width()) != A.Height()) throw std::logic_error("Nonconformal Trsm");
  if (checkIfSingular && diag != UNIT)
    for (int j = 0; j < A.Height(); ++j)
      if (A.Get(j, j) == F(0)) throw SingularMatrixException();
  detail::AsDouble<F> a(A, false), b(B, true);
  detail::check(egpu_host_dtrsm(detail::handle(), side == LEFT ? EGPU_LEFT : EGPU_RIGHT,
                                uplo == LOWER ? EGPU_LOWER : EGPU_UPPER, detail::Ori(orientation),
                                diag == UNIT ? EGPU_UNIT : EGPU_NON_UNIT, B.Height(), B.Width(), (double)alpha, a.p,
                                a.ld, b.p, b.ld));
  b.WriteBack(B);
}

// Trsv(uplo, orientation, diag, A, x), blas-like/level2/Trsv.hpp:20-44.
template <typename F>
inline void Trsv(UpperOrLower uplo, Orientation orientation, UnitOrNonUnit diag, const Matrix<F>& A, Matrix<F>& x) {
  if (x.Width() != 1 && x.Height() != 1) throw std::logic_error("x must be a vector");
  if (x.Width() == 1) {
    Trsm(LEFT, uplo, orientation, diag, F(1), A, x);
  } else {  // row vector: copy into a column
    Matrix<F> xc(x.Width(), 1);
    for (int i = 0; i < x.Width(); ++i) xc.Set(i, 0, x.Get(0, i));
    Trsm(LEFT, uplo, orientation, diag, F(1), A, xc);
    for (int i = 0; i < x.Width(); ++i) x.Set(0, i, xc.Get(i, 0));
  }
}

// --------------------------------------------------- LAPACK-like ---------

// Cholesky(uplo, A), lapack-like/Cholesky.hpp:49-62.
template <typename F>
inline void Cholesky(UpperOrLower uplo, Matrix<F>& A) {
  static_assert(detail::IsSupported<F>::value, "elemgpu supports float and double");
  if (A.Height() != A.Width()) throw std::logic_error("A must be square");
  detail::AsDouble<F> a(A, true);
  int info = 0;
  int rc = egpu_host_dpotrf(detail::handle(), uplo == LOWER ? EGPU_LOWER : EGPU_UPPER, A.Height(), a.p, a.ld, &info);
  a.WriteBack(A);
  detail::check(rc, info);
}

// LDLT(A[, d]) / LDLH(A[, d]), lapack-like/LDL.hpp (ldl::Var3): A = L D L^T
// without pivoting on the lower triangle; d (resized to n x 1 unless a view)
// receives D.  SingularMatrixException on an exact zero pivot.
namespace detail {
template <typename F>
inline void ldl(Orientation orientation, Matrix<F>& A, Matrix<F>* d) {
  static_assert(IsSupported<F>::value, "elemgpu supports float and double");
  if (A.Height() != A.Width()) throw std::logic_error("A must be square");
  if (orientation == NORMAL) throw std::logic_error("Can only perform LDL^T or LDL^H");
  const int n = A.Height();
  if (d && d->Viewing() && (d->Height() != n || d->Width() != 1))
    throw std::logic_error("d must be a column vector the same height as A");
  if (d && !d->Viewing()) d->ResizeTo(n, 1);
  AsDouble<F> a(A, true);
  std::vector<double> dv(std::max(n, 1));
  int info = 0;
  int rc = egpu_host_dldl(handle(), Ori(orientation), n, a.p, a.ld, dv.data(), &info);
  a.WriteBack(A);
  if (d)
    for (int i = 0; i < n; ++i) d->Set(i, 0, (F)dv[i]);
  check(rc, info);
}
}  // namespace detail
template <typename F>
inline void LDLT(Matrix<F>& A) { detail::ldl(TRANSPOSE, A, (Matrix<F>*)nullptr); }
template <typename F>
inline void LDLT(Matrix<F>& A, Matrix<F>& d) { detail::ldl(TRANSPOSE, A, &d); }
template <typename F>
inline void LDLH(Matrix<F>& A) { detail::ldl(ADJOINT, A, (Matrix<F>*)nullptr); }
template <typename F>
inline void LDLH(Matrix<F>& A, Matrix<F>& d) { detail::ldl(ADJOINT, A, &d); }

// ReverseCholesky(uplo, A), lapack-like/Cholesky.hpp:64-76: A = L^H L (LOWER)
// or U U^H (UPPER), swept from the bottom-right corner.
template <typename F>
inline void ReverseCholesky(UpperOrLower uplo, Matrix<F>& A) {
  static_assert(detail::IsSupported<F>::value, "elemgpu supports float and double");
  if (A.Height() != A.Width()) throw std::logic_error("A must be square");
  detail::AsDouble<F> a(A, true);
  int info = 0;
  int rc = egpu_host_dpotrf_reverse(detail::handle(), uplo == LOWER ? EGPU_LOWER : EGPU_UPPER, A.Height(), a.p, a.ld,
                                    &info);
  a.WriteBack(A);
  detail::check(rc, info);
}

namespace cholesky {
// cholesky::SolveAfter(uplo, orientation, A, B), lapack-like/Cholesky/SolveAfter.hpp:20-75.
template <typename F>
inline void SolveAfter(UpperOrLower uplo, Orientation orientation, const Matrix<F>& A, Matrix<F>& B) {
  if (A.Height() != A.Width()) throw std::logic_error("A must be square");
  if (A.Height() != B.Height()) throw std::logic_error("A and B must be the same height");
  detail::AsDouble<F> a(A, false), b(B, true);
  detail::check(egpu_host_dpotrs(detail::handle(), uplo == LOWER ? EGPU_LOWER : EGPU_UPPER,
                                 detail::Ori(orientation), A.Height(), B.Width(), a.p, a.ld, b.p, b.ld));
  b.WriteBack(B);
}
}  // namespace cholesky

// HPDSolve(uplo, orientation, A, B), lapack-like/HPDSolve.hpp:18-28.
template <typename F>
inline void HPDSolve(UpperOrLower uplo, Orientation orientation, Matrix<F>& A, Matrix<F>& B) {
  Cholesky(uplo, A);
  cholesky::SolveAfter(uplo, orientation, A, B);
}

// LU(A, p), lapack-like/LU.hpp:144-218.  p is resized to min(m,n) x 1 unless
// it is a view (LU.hpp:155-156), in which case it must already conform.
template <typename F>
inline void LU(Matrix<F>& A, Matrix<int>& p) {
  static_assert(detail::IsSupported<F>::value, "elemgpu supports float and double");
  const int mn = std::min(A.Height(), A.Width());
  if (p.Viewing() && (p.Height() != mn || p.Width() != 1))
    throw std::logic_error("p must be a vector of the same height as the min dimension of A");
  if (!p.Viewing()) p.ResizeTo(mn, 1);
  detail::AsDouble<F> a(A, true);
  int info = 0;
  std::vector<int> piv(std::max(mn, 1));
  int rc = egpu_host_dgetrf(detail::handle(), A.Height(), A.Width(), a.p, a.ld, piv.data(), &info);
  a.WriteBack(A);
  for (int i = 0; i < mn; ++i) p.Set(i, 0, piv[i]);
  detail::check(rc, info);
}

// LU(A) without pivoting, lapack-like/LU.hpp:36-74.
template <typename F>
inline void LU(Matrix<F>& A) {
  detail::AsDouble<F> a(A, true);
  int info = 0;
  int rc = egpu_host_dgetrf_nopiv(detail::handle(), A.Height(), A.Width(), a.p, a.ld, &info);
  a.WriteBack(A);
  detail::check(rc, info);
}

namespace lu {
// lu::SolveAfter(orientation, A, B), lapack-like/LU/SolveAfter.hpp:20-57.
template <typename F>
inline void SolveAfter(Orientation orientation, const Matrix<F>& A, Matrix<F>& B) {
  if (A.Height() != A.Width()) throw std::logic_error("A must be square");
  if (A.Height() != B.Height()) throw std::logic_error("A and B must be the same height");
  detail::AsDouble<F> a(A, false), b(B, true);
  detail::check(egpu_host_dgetrs(detail::handle(), detail::Ori(orientation), A.Height(), B.Width(), a.p, a.ld,
                                 nullptr, b.p, b.ld));
  b.WriteBack(B);
}
// lu::SolveAfter(orientation, A, p, B), lapack-like/LU/SolveAfter.hpp:101-146.
template <typename F>
inline void SolveAfter(Orientation orientation, const Matrix<F>& A, const Matrix<int>& p, Matrix<F>& B) {
  if (A.Height() != A.Width()) throw std::logic_error("A must be square");
  if (A.Height() != B.Height()) throw std::logic_error("A and B must be the same height");
  if (p.Height() != A.Height()) throw std::logic_error("A and p must be the same height");
  detail::AsDouble<F> a(A, false), b(B, true);
  std::vector<int> piv(std::max(p.Height(), 1));
  for (int i = 0; i < p.Height(); ++i) piv[i] = p.Get(i, 0);
  detail::check(egpu_host_dgetrs(detail::handle(), detail::Ori(orientation), A.Height(), B.Width(), a.p, a.ld,
                                 piv.data(), b.p, b.ld));
  b.WriteBack(B);
}
}  // namespace lu

// GaussianElimination(A, B), lapack-like/GaussianElimination.hpp:216-232.
template <typename F>
inline void GaussianElimination(Matrix<F>& A, Matrix<F>& B) {
  if (A.Height() != A.Width()) throw std::logic_error("A must be square");
  if (A.Height() != B.Height()) throw std::logic_error("A and B must be the same height");
  detail::AsDouble<F> a(A, true), b(B, true);
  int info = 0;
  int rc = egpu_host_dgesv(detail::handle(), A.Height(), B.Width(), a.p, a.ld, b.p, b.ld, &info);
  a.WriteBack(A);
  b.WriteBack(B);
  detail::check(rc, info);
}

// ApplyRowPivots(A, p) / ApplyInverseRowPivots(A, p), lapack-like/ApplyRowPivots.hpp:17-79.
template <typename F>
inline void ApplyRowPivots(Matrix<F>& A, const Matrix<int>& p) {
  if (p.Width() != 1) throw std::logic_error("p must be a column vector");
  if (p.Height() > A.Height()) throw std::logic_error("p cannot be larger than height of A");
  detail::AsDouble<F> a(A, true);
  std::vector<int> piv(std::max(p.Height(), 1));
  for (int i = 0; i < p.Height(); ++i) piv[i] = p.Get(i, 0);
  detail::check(egpu_host_dlaswp(detail::handle(), 0, A.Height(), A.Width(), a.p, a.ld, piv.data(), p.Height()));
  a.WriteBack(A);
}
template <typename F>
inline void ApplyInverseRowPivots(Matrix<F>& A, const Matrix<int>& p) {
  if (p.Width() != 1) throw std::logic_error("p must be a column vector");
  if (p.Height() > A.Height()) throw std::logic_error("p cannot be larger than height of A");
  detail::AsDouble<F> a(A, true);
  std::vector<int> piv(std::max(p.Height(), 1));
  for (int i = 0; i < p.Height(); ++i) piv[i] = p.Get(i, 0);
  detail::check(egpu_host_dlaswp(detail::handle(), 1, A.Height(), A.Width(), a.p, a.ld, piv.data(), p.Height()));
  a.WriteBack(A);
}

// ------------------------------ inverses and determinants (next rows) -----

// SafeProduct<F> (core/types_decl.hpp:24-31): det = rho * exp(kappa * n).
template <typename F>
struct SafeProduct {
  F rho;
  F kappa;
  int n;
  explicit SafeProduct(int numEntries) : rho(1), kappa(0), n(numEntries) {}
};

// TriangularInverse(uplo, diag, A), lapack-like/TriangularInverse.hpp:56-64.
template <typename F>
inline void TriangularInverse(UpperOrLower uplo, UnitOrNonUnit diag, Matrix<F>& A) {
  static_assert(detail::IsSupported<F>::value, "elemgpu supports float and double");
  if (A.Height() != A.Width()) throw std::logic_error("Nonsquare matrices cannot be triangular");
  detail::AsDouble<F> a(A, true);
  int rc = egpu_host_dtrtri(detail::handle(), uplo == LOWER ? EGPU_LOWER : EGPU_UPPER,
                            diag == UNIT ? EGPU_UNIT : EGPU_NON_UNIT, A.Height(), a.p, a.ld);
  a.WriteBack(A);
  detail::check(rc);
}

// Inverse(A), lapack-like/Inverse.hpp:17-23 (inverse::LUPartialPiv).  Throws
// SingularMatrixException on an exact zero pivot.
template <typename F>
inline void Inverse(Matrix<F>& A) {
  static_assert(detail::IsSupported<F>::value, "elemgpu supports float and double");
  if (A.Height() != A.Width()) throw std::logic_error("Cannot invert non-square matrices");
  detail::AsDouble<F> a(A, true);
  int info = 0;
  int rc = egpu_host_dgetri(detail::handle(), A.Height(), a.p, a.ld, &info);
  a.WriteBack(A);
  detail::check(rc, info);
}

// HPDInverse(uplo, A), lapack-like/Inverse.hpp:25-35 (hpd_inverse::
// CholeskyLVar2 / UVar2): only the uplo triangle of A is written.
template <typename F>
inline void HPDInverse(UpperOrLower uplo, Matrix<F>& A) {
  static_assert(detail::IsSupported<F>::value, "elemgpu supports float and double");
  if (A.Height() != A.Width()) throw std::logic_error("Nonsquare matrices cannot be triangular");
  detail::AsDouble<F> a(A, true);
  int info = 0;
  int rc = egpu_host_dpotri(detail::handle(), uplo == LOWER ? EGPU_LOWER : EGPU_UPPER, A.Height(), a.p, a.ld, &info);
  a.WriteBack(A);
  detail::check(rc, info);
}

namespace detail {
template <typename F>
inline SafeProduct<F> safe_det(int hpd, UpperOrLower uplo, Matrix<F>& A, bool canOverwrite) {
  static_assert(IsSupported<F>::value, "elemgpu supports float and double");
  if (A.Height() != A.Width()) throw std::logic_error("Cannot compute determinant of nonsquare matrix");
  AsDouble<F> a(A, true);
  double rho = 1.0, kappa = 0.0;
  int rc = hpd ? egpu_host_dsafe_hpd_det(handle(), uplo == LOWER ? EGPU_LOWER : EGPU_UPPER, A.Height(), a.p, a.ld,
                                         canOverwrite ? 1 : 0, &rho, &kappa)
               : egpu_host_dsafe_det(handle(), A.Height(), a.p, a.ld, canOverwrite ? 1 : 0, &rho, &kappa);
  if (canOverwrite) a.WriteBack(A);
  check(rc);
  SafeProduct<F> det(A.Height());
  det.rho = F(rho);
  det.kappa = F(kappa);
  return det;
}
}  // namespace detail

// SafeDeterminant(A[, canOverwrite]), lapack-like/Determinant.hpp
// (determinant::LUPartialPiv): rho = kappa = 0 for a singular matrix.
template <typename F>
inline SafeProduct<F> SafeDeterminant(const Matrix<F>& A) {
  Matrix<F> B(A);
  return detail::safe_det(0, LOWER, B, false);
}
template <typename F>
inline SafeProduct<F> SafeDeterminant(Matrix<F>& A, bool canOverwrite = false) {
  return detail::safe_det(0, LOWER, A, canOverwrite);
}

// SafeHPDDeterminant(uplo, A[, canOverwrite]), Determinant.hpp
// (hpd_determinant::Cholesky): rho = kappa = 0 if A is not numerically HPD.
template <typename F>
inline SafeProduct<F> SafeHPDDeterminant(UpperOrLower uplo, const Matrix<F>& A) {
  Matrix<F> B(A);
  return detail::safe_det(1, uplo, B, false);
}
template <typename F>
inline SafeProduct<F> SafeHPDDeterminant(UpperOrLower uplo, Matrix<F>& A, bool canOverwrite = false) {
  return detail::safe_det(1, uplo, A, canOverwrite);
}

// Determinant(A) = rho exp(kappa n); HPDDeterminant(uplo, A) = exp(kappa n)
// (Determinant.hpp).
template <typename F>
inline F Determinant(const Matrix<F>& A) {
  SafeProduct<F> s = SafeDeterminant(A);
  return s.rho * std::exp(s.kappa * s.n);
}
template <typename F>
inline F HPDDeterminant(UpperOrLower uplo, const Matrix<F>& A) {
  SafeProduct<F> s = SafeHPDDeterminant(uplo, A);
  return std::exp(s.kappa * s.n);
}

// ------------------------------------------- 1 x 1 DistMatrix overloads --
// Cholesky.hpp:79-101, LU.hpp:220-321, HPDSolve.hpp:30-41,
// Cholesky/SolveAfter.hpp:77-134, LU/SolveAfter.hpp:148-195,
// GaussianElimination.hpp:234-252.
template <typename F>
inline void Cholesky(UpperOrLower uplo, DistMatrix<F>& A) { Cholesky(uplo, A.Matrix()); }
template <typename F>
inline void LU(DistMatrix<F>& A) { LU(A.Matrix()); }
template <typename F>
inline void LU(DistMatrix<F>& A, DistMatrix<int, VC, STAR>& p) {
  if (!p.Viewing()) p.ResizeTo(std::min(A.Height(), A.Width()), 1);
  LU(A.Matrix(), p.Matrix());
}
template <typename F>
inline void HPDSolve(UpperOrLower uplo, Orientation orientation, DistMatrix<F>& A, DistMatrix<F>& B) {
  HPDSolve(uplo, orientation, A.Matrix(), B.Matrix());
}
template <typename F>
inline void GaussianElimination(DistMatrix<F>& A, DistMatrix<F>& B) { GaussianElimination(A.Matrix(), B.Matrix()); }
namespace cholesky {
template <typename F>
inline void SolveAfter(UpperOrLower uplo, Orientation orientation, const DistMatrix<F>& A, DistMatrix<F>& B) {
  SolveAfter(uplo, orientation, A.LockedMatrix(), B.Matrix());
}
}  // namespace cholesky
namespace lu {
template <typename F>
inline void SolveAfter(Orientation orientation, const DistMatrix<F>& A, DistMatrix<F>& B) {
  SolveAfter(orientation, A.LockedMatrix(), B.Matrix());
}
template <typename F>
inline void SolveAfter(Orientation orientation, const DistMatrix<F>& A, const DistMatrix<int, VC, STAR>& p,
                       DistMatrix<F>& B) {
  SolveAfter(orientation, A.LockedMatrix(), p.LockedMatrix(), B.Matrix());
}
}  // namespace lu
template <typename F>
inline void Trsm(LeftOrRight side, UpperOrLower uplo, Orientation orientation, UnitOrNonUnit diag, F alpha,
                 const DistMatrix<F>& A, DistMatrix<F>& B, bool checkIfSingular = false) {
  Trsm(side, uplo, orientation, diag, alpha, A.LockedMatrix(), B.Matrix(), checkIfSingular);
}
template <typename T>
inline void Gemm(Orientation oA, Orientation oB, T alpha, const DistMatrix<T>& A, const DistMatrix<T>& B, T beta,
                 DistMatrix<T>& C) {
  Gemm(oA, oB, alpha, A.LockedMatrix(), B.LockedMatrix(), beta, C.Matrix());
}
template <typename T>
inline void Herk(UpperOrLower uplo, Orientation orientation, T alpha, const DistMatrix<T>& A, T beta,
                 DistMatrix<T>& C) {
  Herk(uplo, orientation, alpha, A.LockedMatrix(), beta, C.Matrix());
}
template <typename F>
inline void TriangularInverse(UpperOrLower uplo, UnitOrNonUnit diag, DistMatrix<F>& A) {
  TriangularInverse(uplo, diag, A.Matrix());
}
template <typename F>
inline void ReverseCholesky(UpperOrLower uplo, DistMatrix<F>& A) { ReverseCholesky(uplo, A.Matrix()); }
template <typename F>
inline void LDLT(DistMatrix<F>& A) { LDLT(A.Matrix()); }
template <typename F>
inline void LDLH(DistMatrix<F>& A) { LDLH(A.Matrix()); }
template <typename F>
inline void Inverse(DistMatrix<F>& A) { Inverse(A.Matrix()); }
template <typename F>
inline void HPDInverse(UpperOrLower uplo, DistMatrix<F>& A) { HPDInverse(uplo, A.Matrix()); }
template <typename F>
inline SafeProduct<F> SafeDeterminant(const DistMatrix<F>& A) { return SafeDeterminant(A.LockedMatrix()); }
template <typename F>
inline SafeProduct<F> SafeDeterminant(DistMatrix<F>& A, bool canOverwrite = false) {
  return SafeDeterminant(A.Matrix(), canOverwrite);
}
template <typename F>
inline SafeProduct<F> SafeHPDDeterminant(UpperOrLower uplo, const DistMatrix<F>& A) {
  return SafeHPDDeterminant(uplo, A.LockedMatrix());
}
template <typename F>
inline SafeProduct<F> SafeHPDDeterminant(UpperOrLower uplo, DistMatrix<F>& A, bool canOverwrite = false) {
  return SafeHPDDeterminant(uplo, A.Matrix(), canOverwrite);
}
template <typename F>
inline F Determinant(const DistMatrix<F>& A) { return Determinant(A.LockedMatrix()); }
template <typename F>
inline F HPDDeterminant(UpperOrLower uplo, const DistMatrix<F>& A) { return HPDDeterminant(uplo, A.LockedMatrix()); }

}  // namespace elem
