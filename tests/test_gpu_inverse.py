"""GPU parity of TriangularInverse, Inverse (LU with partial pivoting),
HPDInverse and (Safe)Determinant / (Safe)HPDDeterminant, called through the
C ABI, against the CPU oracle on the same seeded inputs.

Tolerances (FP64, well-conditioned inputs):
  * inverses: entries within 1e-10 * max|oracle inverse| (1e-12 for the
    triangular inverse); the LU inverse also satisfies
    ||A X - I||_1 / (||A||_1 ||X||_1 n eps) <= 4;
  * the triangle an entry point does not own is bit-identical to the input
    (and, for a unit triangular inverse, the diagonal);
  * determinants: rho equal to the oracle's, kappa within 1e-12 * max(1, |kappa|)
    (the GPU sums the logarithms in a different order);
  * a singular / non-HPD matrix: the exception with the oracle's column for
    the inverses, (rho, kappa) = (0, 0) for the safe determinants.
"""
import numpy as np
import pytest

import elemental_b200 as eg
from elemental_b200 import inputs
from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


def cuda(a):
    return eg.colmajor_cuda(a)


def host(t):
    return np.asfortranarray(t.cpu().numpy())


def well_conditioned_triangle(n, seed):
    rs = np.random.default_rng(seed)
    return np.asfortranarray(rs.standard_normal((n, n)) * (0.5 / max(n, 1)) + np.diag(rs.uniform(1.0, 2.0, n)))


def other_triangle(M, uplo):
    return np.triu(M, 1) if uplo == eg.LOWER else np.tril(M, -1)


@pytest.mark.parametrize("n", [1, 7, 128, 129, 300, 1000])
@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
@pytest.mark.parametrize("diag", [eg.NON_UNIT, eg.UNIT])
def test_triangular_inverse(handle, n, uplo, diag):
    T = well_conditioned_triangle(n, 100 + n)
    ref = orc.triangular_inverse(T, uplo, diag == eg.UNIT)
    dT = cuda(T)
    handle.triangular_inverse(dT, uplo, diag)
    X = host(dT)
    tri = np.tril if uplo == eg.LOWER else np.triu
    k = (-1 if uplo == eg.LOWER else 1) if diag == eg.UNIT else 0
    assert np.max(np.abs(tri(X, k) - tri(ref, k))) <= 1e-12 * np.max(np.abs(ref))
    assert np.array_equal(other_triangle(X, uplo), other_triangle(T, uplo))
    if diag == eg.UNIT:
        assert np.array_equal(np.diag(X), np.diag(T))


@pytest.mark.parametrize("n", [1, 2, 7, 130, 257, 700])
def test_inverse_lu(handle, n):
    A = inputs.uniform(n, n, 200 + n)
    ref, st = orc.inverse(A)
    assert st == 0
    dA = cuda(A)
    handle.inverse(dA)
    X = host(dA)
    assert np.max(np.abs(X - ref)) <= 1e-10 * np.max(np.abs(ref))
    res = np.linalg.norm(A @ X - np.eye(n), 1) / (np.linalg.norm(A, 1) * np.linalg.norm(X, 1) * n * EPS)
    assert res <= 4.0


def test_inverse_singular_raises_with_column(handle):
    A = inputs.uniform(40, 40, 7)
    A[:, 17] = 0.0
    _, st = orc.inverse(A)
    with pytest.raises(eg.SingularMatrixError) as e:
        handle.inverse(cuda(A))
    assert e.value.column == st == 18


@pytest.mark.parametrize("n", [1, 100, 300, 1000])
@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
def test_hpd_inverse(handle, n, uplo):
    A = inputs.spd_ggt(n, 300 + n)
    ref, st = orc.hpd_inverse(A, uplo)
    assert st == 0
    dA = cuda(A)
    handle.hpd_inverse(dA, uplo)
    X = host(dA)
    tri = np.tril if uplo == eg.LOWER else np.triu
    assert np.max(np.abs(tri(X) - tri(ref))) <= 1e-10 * np.max(np.abs(ref))
    assert np.array_equal(other_triangle(X, uplo), other_triangle(A, uplo))


def test_hpd_inverse_not_hpd_raises(handle):
    A = inputs.spd_ggt(50, 4)
    A[20, 20] = -1.0
    with pytest.raises(eg.NonHPDError):
        handle.hpd_inverse(cuda(A), eg.LOWER)


@pytest.mark.parametrize("n", [1, 5, 128, 129, 600])
def test_safe_determinant(handle, n):
    A = inputs.uniform(n, n, 400 + n)
    rho_r, kappa_r, _ = orc.safe_determinant(A)
    dA = cuda(A)
    rho, kappa, nn = handle.safe_determinant(dA)
    assert nn == n and rho == rho_r
    assert abs(kappa - kappa_r) <= 1e-12 * max(1.0, abs(kappa_r))
    assert np.array_equal(host(dA), A)  # not overwritten
    # canOverwrite: A holds the LU factors afterwards
    rho2, kappa2, _ = handle.safe_determinant(dA, overwrite=True)
    assert rho2 == rho and abs(kappa2 - kappa) <= 1e-13 * max(1.0, abs(kappa))
    F, _, _ = orc.lu(A)
    assert np.max(np.abs(host(dA) - F)) <= 1e-11 * np.max(np.abs(F))
    if n <= 5:
        assert abs(handle.determinant(cuda(A)) - np.linalg.det(A)) <= 1e-12 * max(1.0, abs(np.linalg.det(A)))


def test_safe_determinant_singular_is_zero(handle):
    A = inputs.uniform(33, 33, 9)
    A[:, 3] = 0.0
    assert handle.safe_determinant(cuda(A)) == (0.0, 0.0, 33)
    # the handle is usable afterwards (the singular status was cleared)
    B = inputs.uniform(33, 33, 10)
    assert handle.safe_determinant(cuda(B))[0] == orc.safe_determinant(B)[0]


@pytest.mark.parametrize("n", [1, 64, 257, 900])
@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
def test_safe_hpd_determinant(handle, n, uplo):
    A = inputs.spd_ggt(n, 500 + n)
    _, kappa_r, _ = orc.safe_hpd_determinant(A, uplo)
    rho, kappa, nn = handle.safe_hpd_determinant(cuda(A), uplo)
    assert nn == n and rho == 1.0
    assert abs(kappa - kappa_r) <= 1e-12 * max(1.0, abs(kappa_r))
    A[n // 2, n // 2] = -1.0
    assert handle.safe_hpd_determinant(cuda(A), uplo) == (0.0, 0.0, n)


def test_inverse_on_view_with_ldim_and_unaligned_pointer(handle):
    import torch
    n, ld = 130, 171
    A = inputs.uniform(n, n, 77)
    ref, _ = orc.inverse(A)
    store = torch.zeros(ld * n + 1, dtype=torch.float64, device="cuda")
    view = torch.as_strided(store, (n, n), (1, ld), storage_offset=1)
    view.copy_(torch.from_numpy(A))
    handle.inverse(view)
    assert np.max(np.abs(np.asfortranarray(view.cpu().numpy()) - ref)) <= 1e-10 * np.max(np.abs(ref))
    assert float(store[0]) == 0.0


def test_host_entry_points(handle):
    n = 150
    A = inputs.uniform(n, n, 61)
    X = A.copy(order="F")
    handle.host_inverse(X)
    ref, _ = orc.inverse(A)
    assert np.max(np.abs(X - ref)) <= 1e-10 * np.max(np.abs(ref))
    S = inputs.spd_ggt(n, 62)
    H = S.copy(order="F")
    handle.host_hpd_inverse(H, eg.UPPER)
    href, _ = orc.hpd_inverse(S, eg.UPPER)
    assert np.max(np.abs(np.triu(H) - np.triu(href))) <= 1e-10 * np.max(np.abs(href))
    T = well_conditioned_triangle(n, 63)
    Ti = T.copy(order="F")
    handle.host_triangular_inverse(Ti, eg.LOWER, eg.NON_UNIT)
    tref = orc.triangular_inverse(T, eg.LOWER, False)
    assert np.max(np.abs(np.tril(Ti) - np.tril(tref))) <= 1e-12 * np.max(np.abs(tref))
    r, k, _ = handle.host_safe_determinant(A)
    rr, kr, _ = orc.safe_determinant(A)
    assert r == rr and abs(k - kr) <= 1e-12 * max(1.0, abs(kr))
    r, k, _ = handle.host_safe_hpd_determinant(S, eg.LOWER)
    assert r == 1.0 and abs(k - orc.safe_hpd_determinant(S)[1]) <= 1e-12 * max(1.0, abs(k))


# ---------------------------------------------------------- ReverseCholesky --

@pytest.mark.parametrize("n", [1, 5, 128, 129, 600])
@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
def test_reverse_cholesky(handle, n, uplo):
    A = inputs.spd_ggt(n, 600 + n)
    ref, st = orc.reverse_cholesky(A, uplo)
    assert st == 0
    dA = cuda(A)
    handle.reverse_cholesky(dA, uplo)
    F = host(dA)
    tri = np.tril if uplo == eg.LOWER else np.triu
    assert np.max(np.abs(tri(F) - tri(ref))) <= 1e-11 * np.max(np.abs(ref))
    assert np.array_equal(other_triangle(F, uplo), other_triangle(A, uplo))
    L = tri(F)
    R = L.T @ L if uplo == eg.LOWER else L @ L.T
    assert np.linalg.norm(A - R, 1) / (n * EPS * np.linalg.norm(A, 1)) <= 4.0


@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
def test_reverse_cholesky_not_hpd_column(handle, uplo):
    A = inputs.spd_ggt(200, 5)
    A[150, 150] = -1.0
    _, st = orc.reverse_cholesky(A, uplo)
    with pytest.raises(eg.NonHPDError) as e:
        handle.reverse_cholesky(cuda(A), uplo)
    assert e.value.column == st


def test_reverse_cholesky_host(handle):
    A = inputs.spd_ggt(300, 6)
    F = A.copy(order="F")
    handle.host_reverse_cholesky(F, eg.LOWER)
    ref, _ = orc.reverse_cholesky(A, eg.LOWER)
    assert np.max(np.abs(np.tril(F) - np.tril(ref))) <= 1e-11 * np.max(np.abs(ref))


# ----------------------------------------------------------------- LDL^T --

def ldl_input(n, seed, garbage_above=True):
    """A = L0 D0 L0^T with L0 unit lower (off-diagonal scaled by 0.5/n) and D0
    of mixed sign (|D0| in [1, 2]): symmetric indefinite with safe unpivoted
    pivots.  The strict upper triangle is overwritten with 7.0, which the
    factorization must neither read nor write."""
    rs = np.random.default_rng(seed)
    L0 = np.tril(rs.standard_normal((n, n)) * (0.5 / max(n, 1)), -1) + np.eye(n)
    D0 = rs.uniform(1.0, 2.0, n) * rs.choice([-1.0, 1.0], n)
    A = np.asfortranarray(L0 @ np.diag(D0) @ L0.T)
    if garbage_above:
        A[np.triu_indices(n, 1)] = 7.0
    return A, L0, D0


@pytest.mark.parametrize("n", [1, 7, 128, 129, 400, 1000])
@pytest.mark.parametrize("orient", [eg.TRANSPOSE, eg.ADJOINT])
def test_ldl(handle, n, orient):
    import torch
    A, L0, D0 = ldl_input(n, 700 + n)
    ref, dref, st = orc.ldl(A)
    assert st == 0
    dA = cuda(A)
    dd = torch.zeros(n, dtype=torch.float64, device="cuda")
    handle.ldl(dA, dd, orient)
    F = host(dA)
    assert np.max(np.abs(np.tril(F) - np.tril(ref))) <= 1e-12 * np.max(np.abs(np.tril(ref)))
    assert np.max(np.abs(dd.cpu().numpy() - dref)) <= 1e-12 * np.max(np.abs(dref))
    assert np.array_equal(np.triu(F, 1), np.triu(A, 1))
    assert np.max(np.abs(np.tril(F, -1) + np.eye(n) - L0)) <= 1e-12


def test_ldl_singular_column_and_normal_rejected(handle):
    A, _, _ = ldl_input(300, 8)
    A[200, :] = 0.0
    A[:, 200] = 0.0
    _, _, st = orc.ldl(A)
    with pytest.raises(eg.SingularMatrixError) as e:
        handle.ldl(cuda(A))
    assert e.value.column == st == 201
    with pytest.raises(eg.ElemGPUError):
        handle.ldl(cuda(A), None, eg.NORMAL)


def test_ldl_host(handle):
    A, _, _ = ldl_input(260, 9)
    F = A.copy(order="F")
    d = handle.host_ldl(F)
    ref, dref, _ = orc.ldl(A)
    assert np.max(np.abs(np.tril(F) - np.tril(ref))) <= 1e-12 * np.max(np.abs(np.tril(ref)))
    assert np.max(np.abs(d - dref)) <= 1e-12 * np.max(np.abs(dref))
