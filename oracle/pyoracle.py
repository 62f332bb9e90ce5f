"""ctypes front end of the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only as the checker.  Every routine mirrors an Elemental
entry point (citations in oracle/oref_impl.h); matrices are numpy arrays in
column-major (Fortran) order, indices are 0-based as in Elemental.

Parity status: pinned -- tests/test_oracle_ref.py checks every routine here
against the reference's own code compiled from its sources (oracle/ref.py,
oracle/_ref) and against the golden vectors it produced (tests/golden/).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

LOWER, UPPER = 0, 1
NORMAL, TRANSPOSE, ADJOINT = 0, 1, 2


def build() -> str:
    """Compile liboracle.so with oracle/Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or (
            os.path.getmtime(_LIB) < os.path.getmtime(os.path.join(_HERE, "oref_impl.h"))
        ):
            build()
        _lib = ctypes.CDLL(_LIB)
        _declare(_lib)
    return _lib


def _declare(L):
    I, D, F, C = ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_char
    P = ctypes.c_void_p
    for pfx, R in (("d", D), ("s", F)):
        g = lambda n: getattr(L, f"oref_{pfx}{n}")  # noqa: E731
        g("gemm").argtypes = [C, C, I, I, I, R, P, I, P, I, R, P, I]
        g("syrk").argtypes = [C, C, I, I, R, P, I, R, P, I]
        g("trsm").argtypes = [C, C, C, C, I, I, R, P, I, P, I]
        g("trsv").argtypes = [C, C, C, I, P, I, P]
        g("cholesky").argtypes = [I, I, P, I, I]
        g("cholesky").restype = I
        g("cholesky_solve_after").argtypes = [I, I, I, I, P, I, P, I]
        g("hpd_solve").argtypes = [I, I, I, I, P, I, P, I, I]
        g("hpd_solve").restype = I
        g("compose_pivots").argtypes = [P, I, I, P, P]
        g("apply_composed_pivots").argtypes = [I, I, P, I, I, P, P]
        g("apply_row_pivots").argtypes = [I, I, P, I, P, I]
        g("apply_inverse_row_pivots").argtypes = [I, I, P, I, P, I]
        g("lu").argtypes = [I, I, P, I, P, I]
        g("lu").restype = I
        g("lu_nopiv").argtypes = [I, I, P, I, I]
        g("lu_nopiv").restype = I
        g("lu_solve_after").argtypes = [I, I, I, P, I, P, P, I]
        g("gaussian_elimination").argtypes = [I, I, P, I, P, I, I]
        g("gaussian_elimination").restype = I
    L.oref_set_threads.argtypes = [I]
    L.oref_get_threads.restype = I


def set_threads(n: int) -> None:
    lib().oref_set_threads(int(n))


def get_threads() -> int:
    return int(lib().oref_get_threads())


def _pfx(a: np.ndarray) -> str:
    if a.dtype == np.float64:
        return "d"
    if a.dtype == np.float32:
        return "s"
    raise TypeError(f"oracle supports float64/float32, got {a.dtype}")


def _f(a, dtype=None):
    a = np.asarray(a, dtype=dtype)
    return np.require(a, requirements=["F", "A", "W"]) if a.ndim == 2 else np.require(a, requirements=["A", "W"])


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _ld(a):
    return max(1, a.shape[0])


def cholesky(A, uplo=LOWER, nb=128):
    """Cholesky(uplo, A): returns (factored copy, status); status = 0 or the
    1-based column where A stopped being numerically HPD."""
    A = _f(A).copy(order="F")
    n = A.shape[0]
    st = getattr(lib(), f"oref_{_pfx(A)}cholesky")(uplo, n, _p(A), _ld(A), nb)
    return A, int(st)


def cholesky_solve_after(A, B, uplo=LOWER, orient=NORMAL):
    B = _f(B).copy(order="F")
    B2 = B.reshape(B.shape[0], -1, order="F")
    getattr(lib(), f"oref_{_pfx(A)}cholesky_solve_after")(
        uplo, orient, A.shape[0], B2.shape[1], _p(_f(A)), _ld(A), _p(B2), _ld(B2))
    return B2.reshape(B.shape, order="F")


def hpd_solve(A, B, uplo=LOWER, orient=NORMAL, nb=128):
    A = _f(A).copy(order="F")
    B = _f(B).copy(order="F")
    B2 = B.reshape(B.shape[0], -1, order="F")
    st = getattr(lib(), f"oref_{_pfx(A)}hpd_solve")(
        uplo, orient, A.shape[0], B2.shape[1], _p(A), _ld(A), _p(B2), _ld(B2), nb)
    return A, B2.reshape(B.shape, order="F"), int(st)


def lu(A, nb=128):
    """LU(A, p): returns (L\\U copy, p int32, status)."""
    A = _f(A).copy(order="F")
    m, n = A.shape
    p = np.zeros(min(m, n), dtype=np.int32)
    st = getattr(lib(), f"oref_{_pfx(A)}lu")(m, n, _p(A), _ld(A), _p(p), nb)
    return A, p, int(st)


def lu_nopiv(A, nb=128):
    A = _f(A).copy(order="F")
    m, n = A.shape
    st = getattr(lib(), f"oref_{_pfx(A)}lu_nopiv")(m, n, _p(A), _ld(A), nb)
    return A, int(st)


def lu_solve_after(A, p, B, orient=NORMAL):
    B = _f(B).copy(order="F")
    B2 = B.reshape(B.shape[0], -1, order="F")
    pp = None if p is None else np.ascontiguousarray(p, dtype=np.int32)
    getattr(lib(), f"oref_{_pfx(A)}lu_solve_after")(
        orient, A.shape[0], B2.shape[1], _p(_f(A)), _ld(A),
        None if pp is None else _p(pp), _p(B2), _ld(B2))
    return B2.reshape(B.shape, order="F")


def gaussian_elimination(A, B, nb=128):
    A = _f(A).copy(order="F")
    B = _f(B).copy(order="F")
    B2 = B.reshape(B.shape[0], -1, order="F")
    st = getattr(lib(), f"oref_{_pfx(A)}gaussian_elimination")(
        A.shape[0], B2.shape[1], _p(A), _ld(A), _p(B2), _ld(B2), nb)
    return A, B2.reshape(B.shape, order="F"), int(st)


def apply_row_pivots(B, p, inverse=False):
    B = _f(B).copy(order="F")
    B2 = B.reshape(B.shape[0], -1, order="F")
    pp = np.ascontiguousarray(p, dtype=np.int32)
    name = "apply_inverse_row_pivots" if inverse else "apply_row_pivots"
    getattr(lib(), f"oref_{_pfx(B)}{name}")(B2.shape[0], B2.shape[1], _p(B2), _ld(B2), _p(pp), len(pp))
    return B2.reshape(B.shape, order="F")


def compose_pivots(p, offset):
    pp = np.ascontiguousarray(p, dtype=np.int32)
    b = len(pp)
    image = np.zeros(b, np.int32)
    pre = np.zeros(b, np.int32)
    lib().oref_dcompose_pivots(_p(pp), b, offset, _p(image), _p(pre))
    return image, pre


def trsm(side, uplo, orient, diag, alpha, A, B):
    """Trsm(side, uplo, orientation, diag, alpha, A, B) with Elemental's
    character mapping (blas-like/level3/Trsm.hpp:49-86)."""
    B = _f(B).copy(order="F")
    m, n = B.shape
    getattr(lib(), f"oref_{_pfx(B)}trsm")(
        side.encode(), uplo.encode(), orient.encode(), diag.encode(), m, n,
        alpha, _p(_f(A)), _ld(A), _p(B), _ld(B))
    return B


def trsv(uplo, orient, diag, A, x):
    """Trsv(uplo, orientation, diag, A, x) (blas-like/level2/Trsv.hpp:20-44,
    dtrsv_ at src/core/imports/blas.cpp:901-904): x := op(A)^-1 x."""
    x = np.array(x, dtype=A.dtype, copy=True).reshape(-1)
    n = x.shape[0]
    getattr(lib(), f"oref_{_pfx(x)}trsv")(uplo.encode(), orient.encode(), diag.encode(), n, _p(_f(A)), _ld(A), _p(x))
    return x


def gemm(ta, tb, alpha, A, B, beta, C):
    C = _f(C).copy(order="F")
    m, n = C.shape
    k = A.shape[1] if ta == "N" else A.shape[0]
    getattr(lib(), f"oref_{_pfx(C)}gemm")(
        ta.encode(), tb.encode(), m, n, k, alpha, _p(_f(A)), _ld(A), _p(_f(B)), _ld(B), beta, _p(C), _ld(C))
    return C


def syrk(uplo, trans, alpha, A, beta, C):
    C = _f(C).copy(order="F")
    n = C.shape[0]
    k = A.shape[1] if trans == "N" else A.shape[0]
    getattr(lib(), f"oref_{_pfx(C)}syrk")(
        uplo.encode(), trans.encode(), n, k, alpha, _p(_f(A)), _ld(A), beta, _p(C), _ld(C))
    return C


# ---- TriangularInverse / Inverse / HPDInverse / (Safe)Determinant ----------
# Compositions of the routines above, in the reference's order of operations.


def triangular_inverse(A, uplo=LOWER, unit=False):
    """TriangularInverse(uplo, diag, A) (lapack-like/TriangularInverse.hpp:56-64):
    the uplo triangle of a copy of A := its inverse (the diagonal too unless
    unit); the other triangle is left as it was.  Computed as Trsm(LEFT, uplo,
    NORMAL, diag, 1, T, I), which is the same inverse as the reference's
    blocked LVar3/UVar3 up to rounding."""
    A = _f(A).copy(order="F")
    n = A.shape[0]
    X = trsm("L", "L" if uplo == LOWER else "U", "N", "U" if unit else "N", 1.0, A, np.eye(n, order="F"))
    tri = np.tril if uplo == LOWER else np.triu
    mask = tri(np.ones((n, n), dtype=bool), -1 if (unit and uplo == LOWER) else (1 if unit else 0))
    A[mask] = X[mask]
    return A


def inverse(A, nb=128):
    """Inverse(A) (Inverse.hpp:17-23) by inverse::LUPartialPiv
    (Inverse/LUPartialPiv.hpp:17-80): P A = L U; TriangularInverse(UPPER,
    NON_UNIT) of U in place; then, over diagonal blocks from the bottom up,
    A1 -= A2 L21 (Gemm) and A1 := A1 inv(L11) (Trsm RIGHT LOWER NORMAL UNIT)
    with L11/L21 copied out and zeroed; finally inv(A) := inv(A) P
    (ApplyInverseColumnPivots).  Returns (inverse, status)."""
    F, p, st = lu(A, nb)
    if st:
        return F, st
    n = F.shape[0]
    F = triangular_inverse(F, UPPER, unit=False)
    ends = list(range(n, 0, -nb))  # blocks aligned to the bottom-right corner
    for e in ends:
        k = max(0, e - nb)
        L11 = F[k:e, k:e].copy(order="F")
        L21 = F[e:, k:e].copy(order="F")
        F[k:e, k:e] = np.triu(F[k:e, k:e])
        F[e:, k:e] = 0.0
        A1 = np.asfortranarray(F[:, k:e])
        if e < n:
            A1 = gemm("N", "N", -1.0, np.asfortranarray(F[:, e:]), L21, 1.0, A1)
        A1 = trsm("R", "L", "N", "U", 1.0, L11, A1)
        F[:, k:e] = A1
    # inv(A) P: the column swaps i <-> p[i] undone in reverse order
    for i in range(n - 1, -1, -1):
        j = int(p[i])
        if j != i:
            F[:, [i, j]] = F[:, [j, i]]
    return F, 0


def hpd_inverse(A, uplo=LOWER, nb=128):
    """HPDInverse(uplo, A) (Inverse.hpp:25-35): the uplo triangle of a copy of
    A := that of inv(A), the other triangle as it was.  Computed from the
    Cholesky factor and cholesky::SolveAfter on the identity (the same inverse
    as hpd_inverse::CholeskyLVar2 / UVar2 up to rounding).  Returns (result,
    status)."""
    F, st = cholesky(A, uplo, nb)
    if st:
        return F, st
    n = F.shape[0]
    X = cholesky_solve_after(F, np.eye(n, order="F"), uplo)
    out = _f(A).copy(order="F")
    tri = np.tril if uplo == LOWER else np.triu
    mask = tri(np.ones((n, n), dtype=bool))
    out[mask] = X[mask]
    return out, 0


def safe_determinant(A, nb=128):
    """SafeDeterminant(A) -> (rho, kappa, n), det = rho exp(kappa n)
    (determinant::LUPartialPiv / AfterLUPartialPiv,
    Determinant/LUPartialPiv.hpp:17-67, PivotParity.hpp:17-33); a singular
    matrix gives rho = kappa = 0."""
    F, p, st = lu(A, nb)
    n = F.shape[0]
    if st:
        return 0.0, 0.0, n
    rho, kappa = 1.0, 0.0
    scale = float(n)
    for i in range(n):
        delta = F[i, i]
        alpha = abs(delta)
        rho *= delta / alpha
        kappa += np.log(alpha) / scale
    odd = sum(1 for i in range(n) if p[i] != i) % 2 == 1
    return (-rho if odd else rho), float(kappa), n


def safe_hpd_determinant(A, uplo=LOWER, nb=128):
    """SafeHPDDeterminant(uplo, A) -> (rho, kappa, n) (hpd_determinant::
    Cholesky / AfterCholesky, Determinant/Cholesky.hpp:17-55): rho = 1, kappa =
    sum log l_ii / (n / 2); a matrix that is not numerically HPD gives rho =
    kappa = 0."""
    F, st = cholesky(A, uplo, nb)
    n = F.shape[0]
    if st:
        return 0.0, 0.0, n
    kappa = 0.0
    scale = n / 2.0
    for i in range(n):
        kappa += np.log(F[i, i]) / scale
    return 1.0, float(kappa), n


def reverse_cholesky(A, uplo=LOWER):
    """ReverseCholesky(uplo, A) (lapack-like/Cholesky.hpp:64-76): LOWER follows
    cholesky::ReverseLVar3Unb (Cholesky/LVar3.hpp:53-81) -- from the last
    column back: alpha = sqrt(a_jj), row j left of the diagonal scaled by
    1/alpha, then A00 -= a10^T a10 on its lower triangle -- giving A = L^T L;
    UPPER is the transpose of the same sweep (A = U U^T).  Unblocked (the
    blocked ReverseLVar3, :125-165, performs the same eliminations).  Returns
    (copy with the factor in the uplo triangle, status): status is the
    1-based column of a non-positive pivot, else 0."""
    A = _f(A).copy(order="F")
    n = A.shape[0]
    W = A if uplo == LOWER else A.T  # the upper case on the transpose: a lower sweep
    for j in range(n - 1, -1, -1):
        alpha = W[j, j]
        if not alpha > 0.0:
            return A, j + 1
        alpha = np.sqrt(alpha)
        W[j, j] = alpha
        W[j, :j] /= alpha
        r = W[j, :j].copy()
        # A00[i, k] -= r[i] r[k] for i >= k (lower triangle of A00)
        W[:j, :j] -= np.tril(np.outer(r, r))
    return A, 0


def ldl(A):
    """LDLT / LDLH(A, d) without pivoting (lapack-like/LDL.hpp), following
    ldl::Var3Unb (LDL/Var3.hpp:19-67) column by column -- d_j = alpha11 (an
    exact zero is SingularMatrixException), A22 -= a21 (a21 / alpha11)^T on its
    lower triangle, a21 /= alpha11 -- which the blocked Var3 reorders only.
    Returns (copy with L strictly below the diagonal and D on it, d, status):
    status is the 1-based column of a zero pivot, else 0.  The upper triangle
    is left as it was."""
    A = _f(A).copy(order="F")
    n = A.shape[0]
    d = np.zeros(n)
    for j in range(n):
        alpha = A[j, j]
        if alpha == 0.0:
            return A, d, j + 1
        d[j] = alpha
        a21 = A[j + 1:, j].copy()
        beta = a21 / alpha
        A[j + 1:, j + 1:] -= np.tril(np.outer(a21, beta))
        A[j + 1:, j] = beta
    return A, d, 0
