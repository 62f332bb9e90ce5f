"""CPU tests of the oracle (oracle/liboracle.so) -- no GPU needed.

The reference holds no golden vectors for this path, so the oracle is checked
against (a) LAPACK through scipy (dpotrf / dgetrf / dtrtrs), which implement the
same mathematics with the same pivot rule (first maximal |a|), and (b) exact
constructions whose factors are known in advance.
"""
import numpy as np
import pytest
import scipy.linalg as sla

from elemental_b200 import inputs
from oracle import pyoracle as orc

EPS = np.finfo(np.float64).eps
SIZES = [1, 2, 7, 31, 64, 127, 128, 129, 300]


def chol_backward_error(A, F, uplo):
    n = A.shape[0]
    L = np.tril(F) if uplo == orc.LOWER else np.triu(F)
    R = L @ L.T if uplo == orc.LOWER else L.T @ L
    return np.linalg.norm(A - R, 1) / (max(n, 1) * EPS * np.linalg.norm(A, 1))


def lu_backward_error(A, F, p):
    n = A.shape[0]
    L = np.tril(F, -1) + np.eye(n)
    U = np.triu(F)
    PA = orc.apply_row_pivots(A, p)
    return np.linalg.norm(PA - L @ U, 1) / (n * EPS * np.linalg.norm(A, 1))


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("uplo", [orc.LOWER, orc.UPPER])
@pytest.mark.parametrize("nb", [128, 32])
def test_cholesky_vs_lapack(n, uplo, nb):
    A = inputs.spd_ggt(n, seed=n)
    F, st = orc.cholesky(A, uplo, nb)
    assert st == 0
    ref = sla.cholesky(A, lower=(uplo == orc.LOWER))
    tri = np.tril if uplo == orc.LOWER else np.triu
    assert np.max(np.abs(tri(F) - ref)) <= 1e-12 * np.max(np.abs(ref))
    # the other triangle is untouched, bit for bit
    other = np.triu(np.ones((n, n), bool), 1) if uplo == orc.LOWER else np.tril(np.ones((n, n), bool), -1)
    assert np.array_equal(F[other], A[other])
    assert chol_backward_error(A, F, uplo) < 1.0


def test_cholesky_known_factor():
    n = 200
    r = inputs.rng(7)
    # well-conditioned triangle (random unit-scale triangles have exponentially
    # large condition numbers, which no factorization can reproduce exactly)
    L0 = np.tril(r.uniform(-1, 1, (n, n)), -1) / n + np.diag(r.uniform(1, 2, n))
    A = np.asfortranarray(L0 @ L0.T)
    F, st = orc.cholesky(A, orc.LOWER, 64)
    assert st == 0
    assert np.max(np.abs(np.tril(F) - L0)) < 1e-10


def test_cholesky_not_hpd_column():
    n = 150
    A = inputs.spd_ggt(n, 3)
    A[140, 140] = -1.0
    _, st = orc.cholesky(A, orc.LOWER, 128)
    assert st == 141  # 1-based global column


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("nb", [128, 16])
def test_lu_vs_lapack(n, nb):
    A = inputs.uniform(n, n, seed=100 + n)
    F, p, st = orc.lu(A, nb)
    assert st == 0
    lu, piv = sla.lu_factor(A)
    assert np.array_equal(p, piv.astype(np.int32))
    assert np.max(np.abs(F - lu)) <= 1e-11 * max(1.0, np.max(np.abs(lu)))
    assert lu_backward_error(A, F, p) < 2.0


@pytest.mark.parametrize("shape", [(300, 200), (200, 300), (129, 1), (1, 5)])
def test_lu_rectangular(shape):
    m, n = shape
    A = inputs.uniform(m, n, seed=m * 7 + n)
    F, p, st = orc.lu(A, 64)
    lu, piv = sla.lu_factor(A) if m == n else (None, None)
    P, L, U = sla.lu(A)
    assert st == 0
    k = min(m, n)
    Lr = np.tril(F, -1)[:, :k] + np.eye(m, k)
    Ur = np.triu(F)[:k, :]
    PA = orc.apply_row_pivots(A, p)
    assert np.allclose(PA, Lr @ Ur, atol=1e-12 * max(m, n))


def test_lu_known_pivots():
    # Rows arranged so that the pivot of column j sits at row perm[j] by a wide margin.
    n = 96
    r = inputs.rng(11)
    U0 = np.triu(r.uniform(-1, 1, (n, n)), 1) + np.diag(r.uniform(2, 3, n))
    L0 = np.tril(r.uniform(-0.3, 0.3, (n, n)), -1) + np.eye(n)
    A0 = L0 @ U0
    perm = r.permutation(n)
    A = np.asfortranarray(A0[np.argsort(perm)])  # A[perm[i]] = A0[i]
    F, p, st = orc.lu(A, 32)
    assert st == 0
    lu, piv = sla.lu_factor(A)
    assert np.array_equal(p, piv.astype(np.int32))
    assert lu_backward_error(A, F, p) < 2.0


def test_lu_singular_column():
    n = 64
    A = inputs.uniform(n, n, 5)
    A[:, 40] = 0.0
    _, _, st = orc.lu(A, 16)
    assert st == 41


def test_compose_pivots_matches_sequential_swaps():
    r = inputs.rng(1)
    m, b, off = 80, 16, 10
    for trial in range(20):
        p = np.array([off + i + r.integers(0, m - i) for i in range(b)], dtype=np.int32)
        image, pre = orc.compose_pivots(p, off)
        X = inputs.uniform(m, 5, trial)
        seq = X.copy()
        for i in range(b):
            seq[[i, p[i] - off]] = seq[[p[i] - off, i]]
        par = X.copy()
        top = X[:b].copy()
        for i in range(b):
            par[image[i]] = top[i]
            if pre[i] >= b:
                par[i] = X[pre[i]]
        assert np.array_equal(seq, par)


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
def test_trsm_vs_scipy(side, uplo, trans, diag):
    n, k = 70, 9
    r = inputs.rng(3)
    A = np.asfortranarray(r.uniform(-1, 1, (n, n)) + 4 * np.eye(n))
    B = np.asfortranarray(r.standard_normal((n, k) if side == "L" else (k, n)))
    X = orc.trsm(side, uplo, trans, diag, 0.5, A, B)
    Tm = np.tril(A) if uplo == "L" else np.triu(A)
    if diag == "U":
        Tm = Tm - np.diag(np.diag(Tm)) + np.eye(n)
    op = Tm if trans == "N" else Tm.T
    if side == "L":
        assert np.allclose(op @ X, 0.5 * B, atol=1e-12)
    else:
        assert np.allclose(X @ op, 0.5 * B, atol=1e-12)


def test_solves_and_gaussian_elimination():
    n, k = 257, 5
    A = inputs.spd_ggt(n, 4)
    B = inputs.normal(n, k, 5)
    _, X, st = orc.hpd_solve(A, B, orc.LOWER, nb=64)
    assert st == 0
    assert np.allclose(A @ X, B, atol=1e-10)
    _, Xu, st = orc.hpd_solve(A, B, orc.UPPER, nb=64)
    assert np.allclose(Xu, X, atol=1e-12)

    G = inputs.uniform(n, n, 6)
    F, p, st = orc.lu(G, 64)
    Y = orc.lu_solve_after(F, p, B, orc.NORMAL)
    assert np.allclose(G @ Y, B, atol=1e-9)
    Yt = orc.lu_solve_after(F, p, B, orc.TRANSPOSE)
    assert np.allclose(G.T @ Yt, B, atol=1e-9)
    _, Z, st = orc.gaussian_elimination(G, B, 64)
    assert st == 0
    assert np.allclose(Z, Y, atol=1e-9)
    # unpivoted LU on a diagonally dominant matrix
    D = np.asfortranarray(G + n * np.eye(n))
    Fn, st = orc.lu_nopiv(D, 64)
    assert st == 0
    W = orc.lu_solve_after(Fn, None, B, orc.NORMAL)
    assert np.allclose(D @ W, B, atol=1e-10)


def test_gemm_syrk_vs_numpy():
    r = inputs.rng(9)
    A = np.asfortranarray(r.standard_normal((33, 17)))
    B = np.asfortranarray(r.standard_normal((17, 21)))
    C = np.asfortranarray(r.standard_normal((33, 21)))
    out = orc.gemm("N", "N", 2.0, A, B, -1.0, C)
    assert np.allclose(out, 2 * A @ B - C)
    out = orc.gemm("T", "T", 1.0, np.asfortranarray(A.T), np.asfortranarray(B.T), 0.0, C)
    assert np.allclose(out, A @ B)
    S = np.asfortranarray(r.standard_normal((33, 33)))
    outl = orc.syrk("L", "N", -1.0, A, 1.0, S)
    ref = S - A @ A.T
    assert np.allclose(np.tril(outl), np.tril(ref))
    assert np.array_equal(np.triu(outl, 1), np.triu(S, 1))


def test_float_variant():
    A = inputs.spd_ggt(100, 2).astype(np.float32, order="F")
    F, st = orc.cholesky(A, orc.LOWER, 32)
    assert st == 0
    ref = sla.cholesky(A.astype(np.float64), lower=True)
    assert np.max(np.abs(np.tril(F) - ref)) < 1e-4 * np.max(np.abs(ref))


# ---- TriangularInverse / Inverse / HPDInverse / (Safe)Determinant ----------

@pytest.mark.parametrize("n", [1, 7, 130])
def test_inverse_and_determinant_vs_numpy(n):
    rs = np.random.default_rng(40 + n)
    A = np.asfortranarray(rs.uniform(-1, 1, (n, n)))
    X, st = orc.inverse(A, nb=32)
    assert st == 0
    assert np.abs(X @ A - np.eye(n)).max() <= 1e-10
    rho, kappa, nn = orc.safe_determinant(A, nb=32)
    sign, logabs = np.linalg.slogdet(A)
    assert nn == n and rho == sign
    assert abs(kappa * n - logabs) <= 1e-11 * max(1.0, abs(logabs))


def test_inverse_and_determinant_singular():
    A = np.asfortranarray(np.random.default_rng(3).uniform(-1, 1, (9, 9)))
    A[:, 4] = 0.0
    _, st = orc.inverse(A)
    assert st == 5
    assert orc.safe_determinant(A) == (0.0, 0.0, 9)


@pytest.mark.parametrize("uplo", [orc.LOWER, orc.UPPER])
def test_hpd_inverse_and_determinant_vs_numpy(uplo):
    rs = np.random.default_rng(8)
    n = 90
    G = rs.standard_normal((n, n))
    S = np.asfortranarray(G @ G.T + n * np.eye(n))
    H, st = orc.hpd_inverse(S, uplo, nb=32)
    assert st == 0
    tri = np.tril if uplo == orc.LOWER else np.triu
    other = (lambda M: np.triu(M, 1)) if uplo == orc.LOWER else (lambda M: np.tril(M, -1))
    Si = np.linalg.inv(S)
    assert np.abs(tri(H) - tri(Si)).max() <= 1e-12 * np.abs(Si).max()
    assert np.array_equal(other(H), other(S))
    rho, kappa, _ = orc.safe_hpd_determinant(S, uplo, nb=32)
    assert rho == 1.0 and abs(kappa * n - np.linalg.slogdet(S)[1]) <= 1e-11 * n
    S[3, 3] = -1.0
    assert orc.safe_hpd_determinant(S, uplo) == (0.0, 0.0, n)


@pytest.mark.parametrize("uplo", [orc.LOWER, orc.UPPER])
@pytest.mark.parametrize("unit", [False, True])
def test_triangular_inverse_vs_numpy(uplo, unit):
    rs = np.random.default_rng(5)
    n = 60
    T = np.asfortranarray(rs.standard_normal((n, n)) * 0.1 + np.diag(rs.uniform(1, 2, n)))
    X = orc.triangular_inverse(T, uplo, unit)
    tri = np.tril if uplo == orc.LOWER else np.triu
    k = -1 if uplo == orc.LOWER else 1
    Tt = (tri(T, k) + np.eye(n)) if unit else tri(T)
    Xt = (tri(X, k) + np.eye(n)) if unit else tri(X)
    assert np.abs(Xt @ Tt - np.eye(n)).max() <= 1e-13
    other = (lambda M: np.triu(M, 1)) if uplo == orc.LOWER else (lambda M: np.tril(M, -1))
    assert np.array_equal(other(X), other(T))
    if unit:
        assert np.array_equal(np.diag(X), np.diag(T))


def test_ldl_and_reverse_cholesky_oracle():
    rs = np.random.default_rng(12)
    n = 40
    L0 = np.tril(rs.standard_normal((n, n)) * (0.5 / n), -1) + np.eye(n)
    D0 = rs.uniform(1, 2, n) * rs.choice([-1.0, 1.0], n)
    A = np.asfortranarray(L0 @ np.diag(D0) @ L0.T)
    F, d, st = orc.ldl(A)
    assert st == 0 and np.abs(np.tril(F, -1) + np.eye(n) - L0).max() <= 1e-13 and np.abs(d - D0).max() <= 1e-13
    G = rs.standard_normal((n, n))
    S = np.asfortranarray(G @ G.T + n * np.eye(n))
    R, st = orc.reverse_cholesky(S, orc.LOWER)
    L = np.tril(R)
    assert st == 0 and np.abs(L.T @ L - S).max() <= 1e-12 * np.abs(S).max()
