"""ctypes front end of oracle/_ref/libelemref.so -- TEST INFRASTRUCTURE ONLY.

libelemref.so is the reference's own code (Elemental's headers and core
sources, compiled unchanged by oracle/refbuild/Makefile against a
single-process MPI and the OpenBLAS of the scipy wheel).  It pins the C
restatement in liboracle.so (tests/test_oracle_ref.py) and, where present,
serves as the CPU baseline.  Only tests/ and bench.py's CPU legs use it, as
the checker; the GPU product never loads it.

Functions mirror oracle/pyoracle.py: numpy column-major arrays in, copies
out; status 0 ok, 1 not HPD, 2 singular (the reference's exceptions)."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libelemref.so")
REF_SRC = "/root/reference"
_lib = None

LOWER, UPPER = 0, 1
NORMAL, TRANSPOSE, ADJOINT = 0, 1, 2


def available() -> bool:
    return os.path.exists(LIB)


def build() -> str | None:
    """Compile libelemref.so from the reference sources (only where they are
    present); returns the library path, or None without the sources."""
    if not os.path.isdir(REF_SRC):
        return LIB if available() else None
    subprocess.run(["make", "-s", "-j", str(os.cpu_count() or 4), "-C", os.path.join(_HERE, "refbuild"),
                    f"REF={REF_SRC}"], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB} is not built (oracle/refbuild/Makefile)")
        L = ctypes.CDLL(LIB)
        I, D, P = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
        sig = {
            "dcholesky": [I, I, P, I, I], "dreverse_cholesky": [I, I, P, I, I],
            "dcholesky_solve_after": [I, I, I, I, P, I, P, I], "dhpd_solve": [I, I, I, I, P, I, P, I, I],
            "dlu": [I, I, P, I, P, I], "dlu_nopiv": [I, I, P, I, I], "dlu_solve_after": [I, I, I, P, I, P, P, I],
            "dapply_row_pivots": [I, I, I, P, I, P, I],
            "dtrsm": [I, I, I, I, I, I, D, P, I, P, I], "dtrsv": [I, I, I, I, P, I, P],
            "dgemm": [I, I, I, I, I, D, P, I, P, I, D, P, I], "dherk": [I, I, I, I, D, P, I, D, P, I],
            "dtriangular_inverse": [I, I, I, P, I, I], "dinverse": [I, P, I, I], "dhpd_inverse": [I, I, P, I, I],
            "dldl": [I, I, P, I, P, I], "dsafe_determinant": [I, I, I, P, I, I, P, P],
            "dist_dcholesky": [I, I, P, I, I], "dist_dhpd_solve": [I, I, I, I, P, I, P, I, I],
            "dist_dlu": [I, I, P, I, P, I], "dist_dlu_solve_after": [I, I, I, P, I, P, P, I],
            "dist_dgaussian_elimination": [I, I, P, I, P, I, I],
        }
        for name, args in sig.items():
            f = getattr(L, "eref_" + name)
            f.argtypes = args
            f.restype = I
        L.eref_last_error.restype = ctypes.c_char_p
        L.eref_blas_config.restype = ctypes.c_char_p
        _lib = L
    return _lib


def blas_config() -> str:
    return lib().eref_blas_config().decode()


def _f(a, dtype=np.float64):
    return np.array(a, dtype=dtype, order="F", copy=True)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _ld(a):
    return max(1, a.shape[0])


def _rc(rc):
    if rc < 0:
        raise RuntimeError("reference raised: " + lib().eref_last_error().decode())
    return int(rc)


def cholesky(A, uplo=LOWER, nb=128, dist=False):
    A = _f(A)
    f = lib().eref_dist_dcholesky if dist else lib().eref_dcholesky
    return A, _rc(f(uplo, A.shape[0], _p(A), _ld(A), nb))


def reverse_cholesky(A, uplo=LOWER, nb=128):
    A = _f(A)
    return A, _rc(lib().eref_dreverse_cholesky(uplo, A.shape[0], _p(A), _ld(A), nb))


def cholesky_solve_after(F, B, uplo=LOWER, orient=NORMAL):
    F, B = _f(F), _f(B).reshape(B.shape[0], -1, order="F")
    _rc(lib().eref_dcholesky_solve_after(uplo, orient, F.shape[0], B.shape[1], _p(F), _ld(F), _p(B), _ld(B)))
    return B


def hpd_solve(A, B, uplo=LOWER, orient=NORMAL, nb=128, dist=False):
    A, B = _f(A), _f(B).reshape(B.shape[0], -1, order="F")
    f = lib().eref_dist_dhpd_solve if dist else lib().eref_dhpd_solve
    st = _rc(f(uplo, orient, A.shape[0], B.shape[1], _p(A), _ld(A), _p(B), _ld(B), nb))
    return A, B, st


def lu(A, nb=128, dist=False):
    A = _f(A)
    m, n = A.shape
    p = np.zeros(max(min(m, n), 1), dtype=np.int32)
    f = lib().eref_dist_dlu if dist else lib().eref_dlu
    st = _rc(f(m, n, _p(A), _ld(A), _p(p), nb))
    return A, p[:min(m, n)], st


def lu_nopiv(A, nb=128):
    A = _f(A)
    return A, _rc(lib().eref_dlu_nopiv(A.shape[0], A.shape[1], _p(A), _ld(A), nb))


def lu_solve_after(F, p, B, orient=NORMAL, dist=False):
    F, B = _f(F), _f(B).reshape(B.shape[0], -1, order="F")
    pp = None if p is None else np.ascontiguousarray(p, dtype=np.int32)
    f = lib().eref_dist_dlu_solve_after if dist else lib().eref_dlu_solve_after
    _rc(f(orient, F.shape[0], B.shape[1], _p(F), _ld(F), None if pp is None else _p(pp), _p(B), _ld(B)))
    return B


def gaussian_elimination(A, B, nb=128):
    """GaussianElimination on a DistMatrix over a 1 x 1 Grid (the distributed
    RowEchelon, GaussianElimination.hpp:94-209, then the upper solve).  The
    sequential form is not offered: the reference's sequential RowEchelon
    (:19-92) crashes when run."""
    A, B = _f(A), _f(B).reshape(B.shape[0], -1, order="F")
    st = _rc(lib().eref_dist_dgaussian_elimination(A.shape[0], B.shape[1], _p(A), _ld(A), _p(B), _ld(B), nb))
    return A, B, st


def apply_row_pivots(B, p, inverse=False):
    B = _f(B).reshape(B.shape[0], -1, order="F")
    pp = np.ascontiguousarray(p, dtype=np.int32)
    _rc(lib().eref_dapply_row_pivots(int(inverse), B.shape[0], B.shape[1], _p(B), _ld(B), _p(pp), pp.shape[0]))
    return B


def trsm(side, uplo, orient, diag, alpha, A, B):
    A, B = _f(A), _f(B)
    _rc(lib().eref_dtrsm(side, uplo, orient, diag, B.shape[0], B.shape[1], float(alpha), _p(A), _ld(A), _p(B),
                         _ld(B)))
    return B


def trsv(uplo, orient, diag, A, x):
    A, x = _f(A), np.array(x, dtype=np.float64, copy=True).reshape(-1)
    _rc(lib().eref_dtrsv(uplo, orient, diag, A.shape[0], _p(A), _ld(A), _p(x)))
    return x


def gemm(oa, ob, alpha, A, B, beta, C):
    A, B, C = _f(A), _f(B), _f(C)
    k = A.shape[1] if oa == NORMAL else A.shape[0]
    _rc(lib().eref_dgemm(oa, ob, C.shape[0], C.shape[1], k, float(alpha), _p(A), _ld(A), _p(B), _ld(B),
                         float(beta), _p(C), _ld(C)))
    return C


def herk(uplo, orient, alpha, A, beta, C):
    A, C = _f(A), _f(C)
    k = A.shape[1] if orient == NORMAL else A.shape[0]
    _rc(lib().eref_dherk(uplo, orient, C.shape[0], k, float(alpha), _p(A), _ld(A), float(beta), _p(C), _ld(C)))
    return C


def triangular_inverse(A, uplo=LOWER, unit=False, nb=128):
    A = _f(A)
    _rc(lib().eref_dtriangular_inverse(uplo, int(unit), A.shape[0], _p(A), _ld(A), nb))
    return A


def inverse(A, nb=128):
    A = _f(A)
    return A, _rc(lib().eref_dinverse(A.shape[0], _p(A), _ld(A), nb))


def hpd_inverse(A, uplo=LOWER, nb=128):
    A = _f(A)
    return A, _rc(lib().eref_dhpd_inverse(uplo, A.shape[0], _p(A), _ld(A), nb))


def ldl(A, orient=TRANSPOSE, nb=128):
    A = _f(A)
    d = np.zeros(max(A.shape[0], 1))
    st = _rc(lib().eref_dldl(orient, A.shape[0], _p(A), _ld(A), _p(d), nb))
    return A, d[:A.shape[0]], st


def safe_determinant(A, hpd=False, uplo=LOWER, nb=128):
    A = _f(A)
    rho, kappa = ctypes.c_double(), ctypes.c_double()
    _rc(lib().eref_dsafe_determinant(int(hpd), uplo, A.shape[0], _p(A), _ld(A), nb, ctypes.byref(rho),
                                     ctypes.byref(kappa)))
    return rho.value, kappa.value
