"""GPU parity: the sm_100a kernels, called through the C ABI, against the CPU
oracle on the same seeded inputs.

Tolerances (floating point, FP64):
  * scaled backward error ||A - LL^T||_1 / (n eps ||A||_1) <= 4 (Cholesky) and
    ||PA - LU||_1 / (n eps ||A||_1) <= 4 (LU), for GPU and oracle alike;
  * factor entries within 1e-11 * max|factor| of the oracle's (the inputs are
    well conditioned, so forward differences stay at rounding level);
  * LU pivot vectors identical index for index (inputs without near-ties:
    continuous U[-1,1] entries);
  * the triangle Cholesky does not own is bit-identical to the input;
  * solves: ||A X - B||_1 / (||A||_1 ||X||_1 n eps) <= 4 and X within 1e-9
    relative of the oracle's X.
"""
import os

import numpy as np
import pytest

import elemental_b200 as eg
from elemental_b200 import inputs
from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps
BWD = 4.0


def cuda(a):
    return eg.colmajor_cuda(a)


def host(t):
    return np.asfortranarray(t.cpu().numpy())


def chol_bwd(A, F, uplo):
    n = A.shape[0]
    L = np.tril(F) if uplo == eg.LOWER else np.triu(F)
    R = L @ L.T if uplo == eg.LOWER else L.T @ L
    return np.linalg.norm(A - R, 1) / (n * EPS * np.linalg.norm(A, 1))


def lu_bwd(A, F, p):
    m, n = A.shape
    k = min(m, n)
    L = np.tril(F, -1)[:, :k] + np.eye(m, k)
    U = np.triu(F)[:k, :]
    PA = orc.apply_row_pivots(A, p)
    return np.linalg.norm(PA - L @ U, 1) / (max(m, n) * EPS * np.linalg.norm(A, 1))


def solve_bwd(A, X, B):
    n = A.shape[0]
    return np.linalg.norm(A @ X - B, 1) / (np.linalg.norm(A, 1) * np.linalg.norm(X, 1) * n * EPS)


# ------------------------------------------------------------ level 3 --

@pytest.mark.parametrize("oa", [eg.NORMAL, eg.TRANSPOSE])
@pytest.mark.parametrize("ob", [eg.NORMAL, eg.TRANSPOSE])
@pytest.mark.parametrize("mnk", [(1, 1, 1), (37, 53, 29), (128, 64, 16), (300, 200, 129), (513, 257, 128)])
def test_gemm(handle, oa, ob, mnk):
    m, n, k = mnk
    r = inputs.rng(m + n + k)
    A = np.asfortranarray(r.standard_normal((m, k) if oa == eg.NORMAL else (k, m)))
    B = np.asfortranarray(r.standard_normal((k, n) if ob == eg.NORMAL else (n, k)))
    C = np.asfortranarray(r.standard_normal((m, n)))
    dA, dB, dC = cuda(A), cuda(B), cuda(C)
    handle.gemm(oa, ob, -1.5, dA, dB, 0.5, dC)
    ref = orc.gemm("N" if oa == eg.NORMAL else "T", "N" if ob == eg.NORMAL else "T", -1.5, A, B, 0.5, C)
    assert np.max(np.abs(host(dC) - ref)) <= 1e-13 * k * np.max(np.abs(ref)) + 1e-300


@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
@pytest.mark.parametrize("orient", [eg.NORMAL, eg.TRANSPOSE])
@pytest.mark.parametrize("nk", [(5, 3), (130, 64), (333, 128)])
def test_herk(handle, uplo, orient, nk):
    n, k = nk
    r = inputs.rng(n * k)
    A = np.asfortranarray(r.standard_normal((n, k) if orient == eg.NORMAL else (k, n)))
    C = np.asfortranarray(r.standard_normal((n, n)))
    dA, dC = cuda(A), cuda(C)
    handle.herk(uplo, orient, -1.0, dA, 1.0, dC)
    ref = orc.syrk("L" if uplo == eg.LOWER else "U", "N" if orient == eg.NORMAL else "T", -1.0, A, 1.0, C)
    out = host(dC)
    tri = np.tril if uplo == eg.LOWER else np.triu
    assert np.max(np.abs(tri(out) - tri(ref))) <= 1e-13 * k * np.max(np.abs(ref))
    other = np.triu(np.ones((n, n), bool), 1) if uplo == eg.LOWER else np.tril(np.ones((n, n), bool), -1)
    assert np.array_equal(out[other], C[other])


@pytest.mark.parametrize("side", [eg.LEFT, eg.RIGHT])
@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
@pytest.mark.parametrize("orient", [eg.NORMAL, eg.TRANSPOSE])
@pytest.mark.parametrize("diag", [eg.NON_UNIT, eg.UNIT])
def test_trsm(handle, side, uplo, orient, diag):
    n, k = 301, 17
    r = inputs.rng(side * 8 + uplo * 4 + orient * 2 + diag)
    A = np.asfortranarray(r.uniform(-1, 1, (n, n)) / np.sqrt(n) + 2 * np.eye(n))
    B = np.asfortranarray(r.standard_normal((n, k) if side == eg.LEFT else (k, n)))
    dA, dB = cuda(A), cuda(B)
    handle.trsm(side, uplo, orient, diag, 0.75, dA, dB)
    ref = orc.trsm("L" if side == eg.LEFT else "R", "L" if uplo == eg.LOWER else "U",
                   "N" if orient == eg.NORMAL else "T", "U" if diag == eg.UNIT else "N", 0.75, A, B)
    assert np.max(np.abs(host(dB) - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
@pytest.mark.parametrize("orient", [eg.NORMAL, eg.TRANSPOSE])
@pytest.mark.parametrize("diag", [eg.NON_UNIT, eg.UNIT])
@pytest.mark.parametrize("n", [1, 257, 1030])
def test_trsv(handle, uplo, orient, diag, n):
    # Trsv(uplo, orientation, diag, A, x), blas-like/level2/Trsv.hpp:20-44
    r = inputs.rng(n + 16 * uplo + 4 * orient + diag)
    A = np.asfortranarray(r.uniform(-1, 1, (n, n)) / np.sqrt(n) + 2 * np.eye(n))
    x = r.standard_normal(n)
    dA = cuda(A)
    import torch
    dx = torch.from_numpy(x.copy()).cuda()
    handle.trsv(uplo, orient, diag, dA, dx)
    ref = orc.trsv("L" if uplo == eg.LOWER else "U", "N" if orient == eg.NORMAL else "T",
                   "U" if diag == eg.UNIT else "N", A, x)
    got = dx.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.array_equal(host(dA), A)  # A is read only


# ------------------------------------------------------------- Cholesky --

@pytest.mark.parametrize("n", [1, 2, 7, 127, 128, 129, 300, 1000, 2048])
@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
def test_cholesky(handle, n, uplo):
    A = inputs.spd_ggt(n, seed=n)
    dA = cuda(A)
    handle.cholesky(dA, uplo)
    F = host(dA)
    ref, st = orc.cholesky(A, uplo, 128)
    assert st == 0
    tri = np.tril if uplo == eg.LOWER else np.triu
    assert np.max(np.abs(tri(F) - tri(ref))) <= 1e-11 * np.max(np.abs(tri(ref)))
    other = np.triu(np.ones((n, n), bool), 1) if uplo == eg.LOWER else np.tril(np.ones((n, n), bool), -1)
    assert np.array_equal(F[other], A[other])
    assert chol_bwd(A, F, uplo) <= BWD
    assert chol_bwd(A, ref, uplo) <= BWD


def test_cholesky_not_hpd_raises_with_column(handle):
    n = 300
    A = inputs.spd_ggt(n, 3)
    A[200, 200] = -5.0
    dA = cuda(A)
    with pytest.raises(eg.NonHPDError) as ei:
        handle.cholesky(dA, eg.LOWER)
    _, st = orc.cholesky(A, eg.LOWER, 128)
    assert ei.value.column == st == 201
    # the handle stays usable after a failed factorization
    B = inputs.spd_ggt(64, 4)
    dB = cuda(B)
    handle.cholesky(dB, eg.LOWER)


def test_cholesky_view_with_ldim_and_unaligned_pointer(handle):
    # A view with ldim > height (Matrix<F> views, core/matrix.hpp) and a base
    # pointer that is only 8-byte aligned.
    n, ld = 257, 301
    A = inputs.spd_ggt(n, 9)
    import torch
    store = torch.zeros(ld * n + 1, dtype=torch.float64, device="cuda")
    view = torch.as_strided(store, (n, n), (1, ld), storage_offset=1)
    view.copy_(torch.from_numpy(A))
    handle.cholesky(view, eg.LOWER)
    F = np.asfortranarray(view.cpu().numpy())
    ref, _ = orc.cholesky(A, eg.LOWER, 128)
    assert np.max(np.abs(np.tril(F) - np.tril(ref))) <= 1e-11 * np.max(np.abs(ref))
    assert float(store[0]) == 0.0  # nothing outside the view was written


@pytest.mark.parametrize("nb", [32, 64, 96])
def test_cholesky_blocksize(handle, nb):
    n = 400
    A = inputs.spd_ggt(n, nb)
    handle.set_blocksize(nb)
    try:
        dA = cuda(A)
        handle.cholesky(dA, eg.LOWER)
    finally:
        handle.set_blocksize(128)
    ref, _ = orc.cholesky(A, eg.LOWER, nb)
    assert np.max(np.abs(np.tril(host(dA)) - np.tril(ref))) <= 1e-11 * np.max(np.abs(ref))


# ------------------------------------------------------------------- LU --

@pytest.mark.parametrize("n", [1, 2, 7, 127, 128, 129, 300, 1000, 2048])
def test_lu_pivots_and_factors(handle, n):
    import torch
    A = inputs.uniform(n, n, seed=1000 + n)
    dA = cuda(A)
    dp = torch.zeros(n, dtype=torch.int32, device="cuda")
    handle.lu(dA, dp)
    F, p = host(dA), dp.cpu().numpy()
    ref, pref, st = orc.lu(A, 128)
    assert st == 0
    assert np.array_equal(p, pref), np.nonzero(p != pref)[0][:10]
    assert np.max(np.abs(F - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))
    assert lu_bwd(A, F, p) <= BWD


def test_lu_config_n8192_64rhs(handle):
    # LU with partial pivoting + lu::SolveAfter at the benchmark configuration
    # (n = 8192, nb = 128, A ~ U[-1,1] seeded, 64 right-hand sides ~ N(0,1)):
    # the pivot vector index for index, the factors, the backward error and X
    # against the oracle on the same inputs (LU.hpp:144-218, LU/Panel.hpp:52-64,
    # LU/SolveAfter.hpp:101-146)
    import torch
    n, k = 8192, 64
    A = inputs.uniform(n, n, 20240)
    B = inputs.normal(n, k, 20241)
    dA = cuda(A)
    dp = torch.zeros(n, dtype=torch.int32, device="cuda")
    handle.lu(dA, dp)
    dB = cuda(B)
    handle.lu_solve_after(dA, dp, dB, eg.NORMAL)
    F, p, X = host(dA), dp.cpu().numpy(), host(dB)
    orc.set_threads(os.cpu_count() or 1)
    ref, pref, st = orc.lu(A, 128)
    assert st == 0
    assert np.array_equal(p, pref), np.nonzero(p != pref)[0][:10]
    assert np.max(np.abs(F - ref)) <= 1e-9 * max(1.0, np.max(np.abs(ref)))
    Xref = orc.lu_solve_after(ref, pref, B, orc.NORMAL)
    assert np.max(np.abs(X - Xref)) <= 1e-7 * np.max(np.abs(Xref))
    # backward error through A X - B (the n^3 product of L U is left to the
    # factor comparison above)
    assert solve_bwd(A, X, B) <= BWD * 4


def test_lu_tall_panel_grid_form(handle):
    # m = 20000 rows: taller than one cluster holds (16 x 1024), so the panel
    # runs the cooperative grid form; pivots, factors and solve vs the oracle
    import torch
    m, n = 20000, 320
    A = inputs.uniform(m, n, 4242)
    dA = cuda(A)
    dp = torch.zeros(n, dtype=torch.int32, device="cuda")
    handle.trace_enable(True)
    handle.lu(dA, dp)
    ev = handle.trace_events()
    handle.trace_enable(False)
    assert sum(1 for e in ev if e[0] == "panel") == 3
    ref, pref, st = orc.lu(A, 128)
    assert st == 0
    assert np.array_equal(dp.cpu().numpy(), pref)
    assert np.max(np.abs(host(dA) - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))
    assert lu_bwd(A, host(dA), dp.cpu().numpy()) <= BWD


@pytest.mark.parametrize("shape", [(500, 300), (300, 500), (1000, 129)])
def test_lu_rectangular(handle, shape):
    import torch
    m, n = shape
    A = inputs.uniform(m, n, seed=m + 3 * n)
    dA = cuda(A)
    dp = torch.zeros(min(m, n), dtype=torch.int32, device="cuda")
    handle.lu(dA, dp)
    ref, pref, _ = orc.lu(A, 128)
    assert np.array_equal(dp.cpu().numpy(), pref)
    assert np.max(np.abs(host(dA) - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))


def test_lu_singular_raises_with_column(handle):
    import torch
    n = 300
    A = inputs.uniform(n, n, 77)
    A[:, 150] = 0.0
    dA = cuda(A)
    dp = torch.zeros(n, dtype=torch.int32, device="cuda")
    with pytest.raises(eg.SingularMatrixError) as ei:
        handle.lu(dA, dp)
    _, _, st = orc.lu(A, 128)
    assert ei.value.column == st == 151


def test_lu_nopiv(handle):
    n = 700
    A = np.asfortranarray(inputs.uniform(n, n, 8) + n * np.eye(n))
    dA = cuda(A)
    handle.lu_nopiv(dA)
    ref, st = orc.lu_nopiv(A, 128)
    assert st == 0
    assert np.max(np.abs(host(dA) - ref)) <= 1e-10 * np.max(np.abs(ref))


# --------------------------------------------------------------- solves --

# nrhs <= 64 with an even leading dimension takes the one-launch skinny
# sweep; odd leading dimensions and wider right-hand sides the blocked form
@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
@pytest.mark.parametrize("nrhs", [1, 16, 65])
@pytest.mark.parametrize("n", [1030, 1031])
def test_hpd_solve(handle, uplo, nrhs, n):
    A = inputs.spd_ggt(n, 21)
    B = inputs.normal(n, nrhs, 22)
    dA, dB = cuda(A), cuda(B)
    handle.hpd_solve(dA, dB, uplo)
    X = host(dB)
    _, Xref, st = orc.hpd_solve(A, B, uplo, nb=128)
    assert st == 0
    assert solve_bwd(A, X, B) <= BWD
    assert np.max(np.abs(X - Xref)) <= 1e-9 * np.max(np.abs(Xref))


@pytest.mark.parametrize("orient", [eg.NORMAL, eg.TRANSPOSE])
@pytest.mark.parametrize("nrhs", [1, 64, 65])
@pytest.mark.parametrize("n", [999, 1000])
def test_lu_solve_after(handle, orient, nrhs, n):
    import torch
    A = inputs.uniform(n, n, 31)
    B = inputs.normal(n, nrhs, 32)
    dA = cuda(A)
    dp = torch.zeros(n, dtype=torch.int32, device="cuda")
    handle.lu(dA, dp)
    dB = cuda(B)
    handle.lu_solve_after(dA, dp, dB, orient)
    X = host(dB)
    F, p, _ = orc.lu(A, 128)
    Xref = orc.lu_solve_after(F, p, B, orient)
    Aop = A if orient == eg.NORMAL else A.T
    assert solve_bwd(Aop, X, B) <= BWD * 4
    assert np.max(np.abs(X - Xref)) <= 1e-8 * np.max(np.abs(Xref))


def test_gaussian_elimination(handle):
    n, k = 777, 5
    A = inputs.uniform(n, n, 41)
    B = inputs.normal(n, k, 42)
    dA, dB = cuda(A), cuda(B)
    handle.gaussian_elimination(dA, dB)
    _, Xref, st = orc.gaussian_elimination(A, B, 128)
    assert st == 0
    X = host(dB)
    assert np.max(np.abs(X - Xref)) <= 1e-8 * np.max(np.abs(Xref))
    assert np.allclose(np.triu(host(dA)), np.triu(orc.gaussian_elimination(A, B, 128)[0]), atol=1e-10)


@pytest.mark.parametrize("inverse", [False, True])
def test_apply_row_pivots(handle, inverse):
    import torch
    n, k = 513, 7
    r = inputs.rng(5)
    p = np.array([i + r.integers(0, n - i) for i in range(n)], dtype=np.int32)
    B = inputs.normal(n, k, 6)
    dB = cuda(B)
    handle.apply_row_pivots(dB, torch.from_numpy(p).cuda(), inverse)
    assert np.array_equal(host(dB), orc.apply_row_pivots(B, p, inverse))


# ------------------------------------------------------------- host API --

def test_host_api_matches_device_api(handle):
    n, k = 640, 16
    A = inputs.spd_ggt(n, 51)
    B = inputs.normal(n, k, 52)
    Ah, Bh = A.copy(order="F"), B.copy(order="F")
    handle.host_hpd_solve(Ah, Bh, eg.LOWER)
    dA, dB = cuda(A), cuda(B)
    handle.hpd_solve(dA, dB, eg.LOWER)
    assert np.array_equal(Ah, host(dA))
    assert np.array_equal(Bh, host(dB))
    G = inputs.uniform(n, n, 53)
    Gh = G.copy(order="F")
    p = handle.host_lu(Gh)
    ref, pref, _ = orc.lu(G, 128)
    assert np.array_equal(p, pref)
    assert np.max(np.abs(Gh - ref)) <= 1e-10 * np.max(np.abs(ref))


@pytest.mark.parametrize("uplo", [eg.LOWER, eg.UPPER])
def test_cholesky_lookahead_matches_sequential(handle, uplo):
    n = 1500
    A = inputs.spd_ggt(n, 61)
    out = []
    # 0 sequential, 1 per-panel look-ahead, 2/4 grouped (12 block columns, the
    # last one 92 wide: groups 4+4+4 and 2x6), 5 ragged groups 5+5+2
    for depth in (0, 1, 2, 4, 5, -1):
        handle.set_lookahead(depth)
        dA = cuda(A)
        handle.cholesky(dA, uplo)
        out.append(host(dA))
    handle.set_lookahead(-1)
    tri = np.tril if uplo == eg.LOWER else np.triu
    for o in out[1:]:
        assert np.max(np.abs(tri(out[0]) - tri(o))) <= 1e-13 * np.max(np.abs(out[0]))


def test_lu_lookahead_matches_sequential(handle):
    import torch
    n = 1500
    A = inputs.uniform(n, n, 62)
    res = []
    for depth in (0, 1):
        handle.set_lookahead(depth)
        dA = cuda(A)
        dp = torch.zeros(n, dtype=torch.int32, device="cuda")
        handle.lu(dA, dp)
        res.append((host(dA), dp.cpu().numpy()))
    handle.set_lookahead(-1)
    assert np.array_equal(res[0][1], res[1][1])
    assert np.max(np.abs(res[0][0] - res[1][0])) <= 1e-12 * np.max(np.abs(res[0][0]))


def test_async_mode_keeps_first_failure(handle):
    # async: calls only enqueue; the first failure is reported by get_status
    good = inputs.spd_ggt(300, 71)
    bad = good.copy(order="F")
    bad[100, 100] = -1.0
    handle.set_async(True)
    try:
        d1, d2, d3 = cuda(good), cuda(bad), cuda(good)
        handle.cholesky(d1, eg.LOWER)
        handle.cholesky(d2, eg.LOWER)
        handle.cholesky(d3, eg.LOWER)  # skipped: a failure is pending
        with pytest.raises(eg.NonHPDError) as ei:
            handle.get_status()
        assert ei.value.column == 101
        handle.get_status()  # cleared
    finally:
        handle.set_async(False)
    ref, _ = orc.cholesky(good, eg.LOWER, 128)
    assert np.max(np.abs(np.tril(host(d1)) - np.tril(ref))) <= 1e-11 * np.max(np.abs(ref))
    assert np.array_equal(host(d3), good)  # untouched


def test_trace_records_kernel_classes(handle):
    import torch
    A = inputs.uniform(640, 640, 72)
    dA = cuda(A)
    dp = torch.zeros(640, dtype=torch.int32, device="cuda")
    handle.trace_enable(True)
    handle.lu(dA, dp)
    s = handle.trace_summary()
    handle.trace_enable(False)
    assert s["panel"]["launches"] == 5
    assert s["update"]["launches"] >= 4 and s["update"]["flops"] > 0
    assert all(v["ms"] >= 0 for v in s.values())
