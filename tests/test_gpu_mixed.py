"""Mixed-precision path: the tcgen05 TF32 engine against an FP64 product, and
the mixed HPD solve (TF32 x 3 Cholesky + FP64 iterative refinement) against
the CPU oracle's FP64 solve.

Tolerances: the TF32 x 3 product keeps ~21 bits, so |C - AB^T| is bounded by
about 2^-20 * K * max|A| max|B| (terms 3) and 2^-10 * K * max|A| max|B|
(terms 1, one TF32 product); the refined solve must reach a normwise backward
error <= 1e-14 and agree with the FP64 oracle solution to kappa * 1e-13."""
import numpy as np
import pytest
import torch

import elemental_b200 as eg
from elemental_b200 import inputs
from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu


def _bound(A, B, K, bits):
    return 2.0 ** (-bits) * K * np.abs(A).max() * np.abs(B).max()


@pytest.mark.parametrize("M,N,K", [(128, 128, 32), (300, 250, 200), (1000, 77, 128), (129, 513, 45)])
@pytest.mark.parametrize("terms", [1, 3])
def test_tc_gemm_split_full(handle, M, N, K, terms):
    A = inputs.normal(M, K, 11)
    B = inputs.normal(N, K, 12)
    C0 = inputs.normal(M, N, 13).astype(np.float32)
    dC = eg.colmajor_cuda(C0.astype(np.float64)).float().t().contiguous().t()
    handle.tc_gemm_split(eg.colmajor_cuda(A), eg.colmajor_cuda(B), dC, alpha=-1.0, beta=1.0, terms=terms)
    torch.cuda.synchronize()
    ref = C0.astype(np.float64) - A @ B.T
    err = np.abs(dC.cpu().numpy().astype(np.float64) - ref).max()
    bits = 20 if terms == 3 else 10
    assert err <= _bound(A, B, K, bits) + 2.0 ** -22 * np.abs(ref).max(), err


@pytest.mark.parametrize("n", [384, 1000])
@pytest.mark.parametrize("beta", [0.0, 1.0])
def test_tc_gemm_split_lower_leaves_upper(handle, n, beta):
    # lower-triangle update (the mixed factorization's trailing update); with
    # beta != 0 and ldc a multiple of 4 the C tiles are staged through shared
    # memory by TMA, with a partial last tile row at n = 1000
    K = 128
    A = inputs.normal(n, K, 21)
    C0 = np.full((n, n), 7.0, dtype=np.float32)
    C0[np.tril_indices(n)] = inputs.normal(n, n, 22)[np.tril_indices(n)]
    dC = eg.colmajor_cuda(C0.astype(np.float64)).float().t().contiguous().t()
    dA = eg.colmajor_cuda(A)
    handle.tc_gemm_split(dA, dA, dC, alpha=-1.0, beta=beta, lower=True, terms=3)
    torch.cuda.synchronize()
    out = dC.cpu().numpy().astype(np.float64)
    low = np.tril(np.ones((n, n), bool))
    ref = beta * C0.astype(np.float64) - A @ A.T
    assert np.abs(out[low] - ref[low]).max() <= _bound(A, A, K, 20) + 2.0 ** -22 * np.abs(ref).max()
    assert np.all(out[~low] == 7.0)


def _berr(A, X, B):
    R = B - A @ X
    return np.max(np.abs(R).max(axis=0) / (np.abs(A).sum(axis=1).max() * np.abs(X).max(axis=0) + np.abs(B).max(axis=0)))


@pytest.mark.parametrize("n,nrhs,uplo", [(1000, 4, eg.LOWER), (777, 1, eg.UPPER), (2048, 16, eg.LOWER)])
def test_hpd_solve_mixed_well_conditioned(handle, n, nrhs, uplo):
    A = inputs.spd_ggt(n, 31)
    B = inputs.normal(n, nrhs, 32)
    X, it, be = handle.hpd_solve_mixed(eg.colmajor_cuda(A), eg.colmajor_cuda(B), uplo=uplo)
    Xg = X.cpu().numpy()
    assert be <= 1e-14
    assert _berr(A, Xg, B) <= 1e-14
    _, Xr, st = orc.hpd_solve(A, B, orc.LOWER, nb=128)
    assert st == 0
    assert np.abs(Xg - Xr).max() <= 1e-12 * np.abs(Xr).max()


@pytest.mark.parametrize("kappa", [1e4, 1e6])
def test_hpd_solve_mixed_ill_conditioned(handle, kappa):
    n, nrhs = 1024, 8
    A = inputs.spd_spectrum(n, kappa, 41)
    B = inputs.normal(n, nrhs, 42)
    dA = eg.colmajor_cuda(A)
    X, it, be = handle.hpd_solve_mixed(dA, eg.colmajor_cuda(B))
    assert be <= 1e-14, (it, be)
    assert _berr(A, X.cpu().numpy(), B) <= 1e-14
    _, Xr, st = orc.hpd_solve(A, B, orc.LOWER, nb=128)
    assert np.abs(X.cpu().numpy() - Xr).max() <= kappa * 1e-13 * np.abs(Xr).max()
    # inputs are left unchanged
    assert np.array_equal(dA.cpu().numpy(), A)


def test_hpd_solve_mixed_not_hpd(handle):
    A = inputs.spd_ggt(300, 5)
    A[150, 150] = -1.0
    with pytest.raises(eg.NonHPDError):
        handle.hpd_solve_mixed(eg.colmajor_cuda(A), eg.colmajor_cuda(inputs.normal(300, 2, 6)))


def test_host_hpd_solve_mixed_matches_device():
    """The host-memory entry gives the device entry's solution."""
    h = eg.Handle(0)
    n, k = 700, 5
    A = inputs.spd_spectrum(n, 1e5, 51)
    B = inputs.normal(n, k, 52)
    X = np.zeros((n, k), order="F")
    it, be = h.host_hpd_solve_mixed(A, B, X)
    Xd, it2, be2 = h.hpd_solve_mixed(eg.colmajor_cuda(A), eg.colmajor_cuda(B))
    assert be <= 1e-14 and be2 <= 1e-14
    assert _berr(A, X, B) <= 1e-14
    # both at backward error <= 1e-14: forward errors within kappa * 1e-14 of each other
    assert np.abs(X - Xd.cpu().numpy()).max() <= 1e5 * 1e-14 * np.abs(X).max()
    h.close()


@pytest.mark.parametrize("kappa", [1e8, 1e9])
def test_hpd_solve_mixed_gmres_ir(handle, kappa):
    """Beyond kappa ~ 1e7 the TF32x3 factor no longer contracts plain
    refinement quickly; GMRES-IR preconditioned by it reaches 1e-14."""
    n, nrhs = 1024, 4
    A = inputs.spd_spectrum(n, kappa, 61)
    B = inputs.normal(n, nrhs, 62)
    X, it, be = handle.hpd_solve_mixed(eg.colmajor_cuda(A), eg.colmajor_cuda(B))
    assert be <= 1e-14
    assert _berr(A, X.cpu().numpy(), B) <= 1e-14
    assert handle.mixed_gmres_iterations() > 0


def test_hpd_solve_mixed_config_n16384_kappa1e6(handle):
    # The benchmark configuration: n = 16384, A = Q diag(s) Q^T with s
    # log-spaced over [1, 1e6], 32 right-hand sides ~ N(0,1).  The mixed solve
    # reaches backward error <= 1e-14, and its X agrees with the plain FP64
    # solve (egpu_dposv) on the same A and B to kappa * 1e-13.
    n, k, kappa = 16384, 32, 1e6
    A = inputs.spd_spectrum_torch(n, kappa, 20240, "cuda")
    B = torch.from_numpy(inputs.normal(n, k, 20241)).cuda().t().contiguous().t()
    X, iters, berr = handle.hpd_solve_mixed(A, B, eg.LOWER, 30, 1e-14)
    torch.cuda.synchronize()
    R = B - A @ X
    den = A.abs().sum(1).max() * X.abs().amax(0) + B.abs().amax(0)
    be = float((R.abs().amax(0) / den).max())
    assert be <= 1e-14 and berr <= 1e-14, (be, berr, iters)
    A2, X2 = A.clone(), B.clone()
    handle.hpd_solve(A2, X2, eg.LOWER)
    del A2
    rel = float((X - X2).abs().max() / X2.abs().max())
    assert rel <= kappa * 1e-13, rel


@pytest.mark.parametrize("n", [1, 100, 511, 512, 513, 1000, 2049, 4100])
@pytest.mark.parametrize("nrhs", [1, 7, 32])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_sweep32_solve_matches_fp64_triangular_solve(handle, n, nrhs, trans):
    # the FP32 super-block sweep (egpu_sweep32_solve) against an FP64
    # triangular solve of the same FP32 factor: the Cholesky factor of a
    # well-conditioned HPD matrix, so the FP32 solve is accurate to ~1e-6
    if n > 1000 and nrhs != 32:
        pytest.skip("large orders with the bench's right-hand-side counts only")
    A = torch.from_numpy(inputs.spd_ggt(n, 90 + n)).cuda()
    L = torch.linalg.cholesky(A)
    ld = (n + 31) // 32 * 32
    store = torch.zeros((n, ld), dtype=torch.float32, device="cuda")
    L32 = torch.as_strided(store, (n, n), (1, ld))  # column-major, ld a multiple of 32
    L32.copy_(L.float())
    Bh = inputs.normal(n, nrhs, 91)
    B = torch.from_numpy(Bh).cuda()
    X = eg.colmajor_cuda(Bh)  # column-major FP64
    handle.sweep32_solve(L32, X, trans)
    torch.cuda.synchronize()
    L64 = L32.double().tril()
    if trans == 2:
        ref = torch.linalg.solve_triangular(L64.t(), torch.linalg.solve_triangular(L64, B, upper=False), upper=True)
    else:
        ref = torch.linalg.solve_triangular(L64.t() if trans else L64, B, upper=bool(trans))
    err = float((X - ref).abs().max() / ref.abs().max())
    assert err <= 2e-5, err


@pytest.mark.parametrize("kappa", [1e4, 1e8])
def test_condition_estimate_picks_the_refinement_mode(handle, kappa):
    # policy 1: Hager's 1-norm estimate after the factorization picks plain
    # refinement (kappa 1e4) or GMRES-IR (kappa 1e8); both reach backward
    # error <= 1e-14 and the oracle's FP64 solution to kappa * 1e-13
    n, k = 1024, 4
    A = inputs.spd_spectrum(n, kappa, 33)
    B = inputs.normal(n, k, 34)
    handle.set_mixed_policy(1)
    try:
        X, iters, berr = handle.hpd_solve_mixed(eg.colmajor_cuda(A), eg.colmajor_cuda(B), eg.LOWER, 30, 1e-14)
        est = handle.mixed_condition_estimate()
        gm = handle.mixed_gmres_iterations()
    finally:
        handle.set_mixed_policy(0)
    X = X.cpu().numpy()
    k1 = np.abs(A).sum(0).max() * np.abs(np.linalg.inv(A)).sum(0).max()
    assert k1 / 10 <= est <= k1 * 10, (est, k1)
    assert (gm > 0) == (kappa >= 1e8), (gm, est)
    assert berr <= 1e-14 and _berr(A, X, B) <= 1e-14
    _, Xref, st = orc.hpd_solve(A, B, eg.LOWER, nb=128)
    assert st == 0
    assert np.abs(X - Xref).max() <= kappa * 1e-13 * np.abs(Xref).max()


def test_condition_estimate_skipped_when_refinement_contracts(handle):
    # the default adaptive policy estimates nothing for a well-conditioned A
    n = 800
    A = inputs.spd_spectrum(n, 1e3, 35)
    B = inputs.normal(n, 2, 36)
    X, iters, berr = handle.hpd_solve_mixed(eg.colmajor_cuda(A), eg.colmajor_cuda(B), eg.LOWER, 30, 1e-14)
    assert berr <= 1e-14
    assert handle.mixed_condition_estimate() == -1.0
    assert handle.mixed_gmres_iterations() == 0


def _ge_oracle(A, B):
    _, Xr, st = orc.gaussian_elimination(A, B, 128)
    assert st == 0
    return Xr


@pytest.mark.parametrize("n,nrhs", [(1000, 4), (777, 1), (2048, 16), (129, 3)])
def test_gaussian_elimination_mixed_well_conditioned(handle, n, nrhs):
    A = inputs.uniform(n, n, 71)  # the reference's Uniform test matrix
    B = inputs.normal(n, nrhs, 72)
    dA = eg.colmajor_cuda(A)
    dB = eg.colmajor_cuda(B)
    X, it, be = handle.gaussian_elimination_mixed(dA, dB)
    Xg = X.cpu().numpy()
    assert be <= 1e-14, (it, be)
    assert _berr(A, Xg, B) <= 1e-14
    # A and B are inputs only
    assert np.array_equal(dA.cpu().numpy(), A) and np.array_equal(dB.cpu().numpy(), B)
    Xr = _ge_oracle(A, B)
    kappa = np.linalg.cond(A, 1)
    assert np.abs(Xg - Xr).max() <= kappa * 1e-13 * np.abs(Xr).max()


@pytest.mark.parametrize("kind,kappa,mode", [("general", 1e4, 0), ("general", 3e7, 1), ("general", 1e8, 2),
                                              ("spd", 1e8, 1)])
@pytest.mark.parametrize("policy", [0, 1])
def test_gaussian_elimination_mixed_ill_conditioned(handle, kind, kappa, mode, policy):
    # nonsymmetric U diag(s) V^T and the serving stream's Q diag(s) Q^T: plain
    # refinement, GMRES-IR, or (when the estimate says the FP32 factors cannot
    # precondition) the FP64 factors; every route reaches backward error 1e-14
    n, nrhs = 1024, 8
    A = inputs.general_spectrum(n, kappa, 73) if kind == "general" else inputs.spd_spectrum(n, kappa, 73)
    B = inputs.normal(n, nrhs, 74)
    handle.set_mixed_policy(policy)
    try:
        X, it, be = handle.gaussian_elimination_mixed(eg.colmajor_cuda(A), eg.colmajor_cuda(B))
        est = handle.mixed_condition_estimate()
        got = handle.mixed_mode()
    finally:
        handle.set_mixed_policy(0)
    Xg = X.cpu().numpy()
    assert be <= 1e-14, (it, be, est)
    assert _berr(A, Xg, B) <= 1e-14
    assert got == mode, (got, est)
    Xr = _ge_oracle(A, B)
    assert np.abs(Xg - Xr).max() <= kappa * 1e-13 * np.abs(Xr).max()
    if policy == 1 and mode < 2:
        k1 = np.linalg.cond(A, 1)
        assert k1 / 10 <= est <= k1 * 10, (est, k1)


def test_gaussian_elimination_mixed_singular(handle):
    n = 300
    A = inputs.uniform(n, n, 75)
    A[:, 200] = 0.0
    with pytest.raises(eg.SingularMatrixError):
        handle.gaussian_elimination_mixed(eg.colmajor_cuda(A), eg.colmajor_cuda(inputs.normal(n, 2, 76)))


def test_gaussian_elimination_mixed_n8192(handle):
    # the LU benchmark's size: backward error and the FP64 solve's x
    n, k = 8192, 32
    A = inputs.uniform(n, n, 77)
    B = inputs.normal(n, k, 78)
    dA, dB = eg.colmajor_cuda(A), eg.colmajor_cuda(B)
    X, it, be = handle.gaussian_elimination_mixed(dA, dB)
    assert be <= 1e-14, (it, be)
    A64, X64 = dA.clone(), dB.clone()
    handle.gaussian_elimination(A64, X64)  # FP64 LU: A64 := its factors, X64 := x
    rel = (X - X64).abs().max().item() / X64.abs().max().item()
    assert rel <= 1e-9, rel
