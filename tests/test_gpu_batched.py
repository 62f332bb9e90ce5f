"""Batched uneven factor-and-solve (one persistent launch) against the CPU
oracle, system by system.  Same tolerances as the single-system parity tests:
factors within 1e-11 * max|L| of the oracle's, solutions within 1e-9."""
import numpy as np
import pytest

import elemental_b200 as eg
from elemental_b200 import inputs
from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu


def test_hpd_solve_batched_uneven(handle):
    r = inputs.rng(2024)
    sizes = [1, 2, 31, 32, 33, 64, 127, 128, 129, 300, 511, 512] + list(r.integers(1, 513, 36))
    nrhs = [int(x) for x in r.integers(1, 17, len(sizes))]  # up to the 16-column limit
    As, Bs, dA, dB = [], [], [], []
    for i, (n, k) in enumerate(zip(sizes, nrhs)):
        A = inputs.spd_ggt(int(n), seed=3000 + i)
        B = inputs.normal(int(n), k, seed=4000 + i)
        As.append(A); Bs.append(B)
        dA.append(eg.colmajor_cuda(A)); dB.append(eg.colmajor_cuda(B))
    info = handle.hpd_solve_batched(dA, dB)
    assert info == [0] * len(sizes)
    for i, (A, B) in enumerate(zip(As, Bs)):
        F, X, st = orc.hpd_solve(A, B, orc.LOWER, nb=32)
        assert st == 0
        L = np.tril(dA[i].cpu().numpy())
        assert np.max(np.abs(L - np.tril(F))) <= 1e-11 * np.max(np.abs(F)), i
        Xg = dB[i].cpu().numpy()
        assert np.max(np.abs(Xg - X)) <= 1e-9 * max(1.0, np.max(np.abs(X))), i
        # upper triangle untouched
        n = A.shape[0]
        up = np.triu(np.ones((n, n), bool), 1)
        assert np.array_equal(dA[i].cpu().numpy()[up], A[up])


def test_hpd_batched_reports_failures_per_system(handle):
    good = inputs.spd_ggt(100, 1)
    bad = good.copy(order="F")
    bad[70, 70] = -3.0
    dA = [eg.colmajor_cuda(good), eg.colmajor_cuda(bad), eg.colmajor_cuda(good)]
    dB = [eg.colmajor_cuda(inputs.normal(100, 2, s)) for s in range(3)]
    info = handle.hpd_solve_batched(dA, dB)
    assert info == [0, 71, 0]


def test_gaussian_elimination_batched_uneven(handle):
    r = inputs.rng(77)
    sizes = [1, 2, 31, 32, 33, 64, 100, 255, 256, 257, 511, 512] + list(r.integers(1, 513, 24))
    nrhs = [int(x) for x in r.integers(1, 17, len(sizes))]  # up to the 16-column limit
    As, Bs, dA, dB = [], [], [], []
    for i, (n, k) in enumerate(zip(sizes, nrhs)):
        A = inputs.uniform(int(n), int(n), seed=5000 + i)
        B = inputs.normal(int(n), k, seed=6000 + i)
        As.append(A); Bs.append(B)
        dA.append(eg.colmajor_cuda(A)); dB.append(eg.colmajor_cuda(B))
    info = handle.gaussian_elimination_batched(dA, dB)
    assert info == [0] * len(sizes)
    for i, (A, B) in enumerate(zip(As, Bs)):
        F, X, st = orc.gaussian_elimination(A, B, nb=32)
        assert st == 0
        U = np.triu(dA[i].cpu().numpy())
        assert np.max(np.abs(U - np.triu(F))) <= 1e-10 * max(1.0, np.max(np.abs(F))), i
        Xg = dB[i].cpu().numpy()
        assert np.max(np.abs(Xg - X)) <= 1e-8 * max(1.0, np.max(np.abs(X))), i


def test_gaussian_elimination_batched_singular(handle):
    good = inputs.uniform(80, 80, 1)
    bad = good.copy(order="F")
    bad[:, 45] = 0.0
    dA = [eg.colmajor_cuda(good), eg.colmajor_cuda(bad)]
    dB = [eg.colmajor_cuda(inputs.normal(80, 1, s)) for s in range(2)]
    assert handle.gaussian_elimination_batched(dA, dB) == [0, 46]


@pytest.mark.parametrize("kind", [0, 1])
def test_batch_plan_graph_replay_matches_oracle(handle, kind):
    """A plan run captured in a CUDA graph and replayed on refilled inputs
    gives the oracle's per-system solutions; the autotuner keeps a valid grid."""
    import torch
    r = inputs.rng(77 + kind)
    sizes = [int(x) for x in r.integers(1, 513, 24)] + [512, 1, 33]
    As, Bs, dA, dB = [], [], [], []
    for i, n in enumerate(sizes):
        A = inputs.spd_ggt(n, 500 + i) if kind == 0 else inputs.uniform(n, n, 500 + i)
        B = inputs.normal(n, 1 + i % 16, 600 + i)
        As.append(A); Bs.append(B)
        dA.append(eg.colmajor_cuda(A)); dB.append(eg.colmajor_cuda(B))
    A0 = [a.clone() for a in dA]
    B0 = [b.clone() for b in dB]
    plan = eg.BatchPlan(handle, kind, dA, dB)
    ms, grid = plan.autotune(reps=1)
    assert ms > 0 and 1 <= grid <= torch.cuda.get_device_properties(0).multi_processor_count
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    for a, a0 in zip(dA, A0):
        a.copy_(a0)
    for b, b0 in zip(dB, B0):
        b.copy_(b0)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        plan.run(s)
    torch.cuda.synchronize()
    for rep in range(2):  # refill, replay
        for a, a0 in zip(dA, A0):
            a.copy_(a0)
        for b, b0 in zip(dB, B0):
            b.copy_(b0)
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
    assert plan.info(s) == [0] * len(sizes)
    for i, (A, B) in enumerate(zip(As, Bs)):
        if kind == 0:
            _, X, st = orc.hpd_solve(A, B, orc.LOWER, nb=32)
        else:
            _, X, st = orc.gaussian_elimination(A, B, nb=32)
        assert st == 0
        Xg = dB[i].cpu().numpy()
        assert np.max(np.abs(Xg - X)) <= 1e-8 * max(1.0, np.max(np.abs(X))), i
    plan.close()


def _berr(A, X, B):
    """max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf)."""
    R = B - A @ X
    den = np.abs(A).sum(1).max() * np.abs(X).max(0) + np.abs(B).max(0)
    return float((np.abs(R).max(0) / den).max())


@pytest.mark.parametrize("kind", [0, 1])
def test_refined_plan_uneven(handle, kind):
    """FP32 working copies + FP64 refinement: every system reaches backward
    error <= 1e-14, agrees with the oracle's FP64 solution, and leaves A
    untouched (more than 8 right-hand sides take two chunks)."""
    r = inputs.rng(900 + kind)
    sizes = [1, 2, 31, 32, 33, 64, 127, 128, 129, 255, 256, 257, 300, 511, 512] + \
        [int(x) for x in r.integers(1, 513, 17)]
    As, Bs, dA, dB = [], [], [], []
    for i, n in enumerate(sizes):
        A = inputs.spd_ggt(n, 700 + i) if kind == 0 else inputs.uniform(n, n, 700 + i)
        B = inputs.normal(n, 1 + (i * 5) % 16, 800 + i)
        As.append(A); Bs.append(B)
        dA.append(eg.colmajor_cuda(A)); dB.append(eg.colmajor_cuda(B))
    plan = eg.BatchPlan(handle, kind, dA, dB, precision=1)
    plan.run()
    assert plan.info() == [0] * len(sizes)
    its = plan.iters()
    assert all(0 <= k <= 10 for k in its), its
    for i, (A, B) in enumerate(zip(As, Bs)):
        assert np.array_equal(dA[i].cpu().numpy(), A), i
        Xg = dB[i].cpu().numpy()
        assert _berr(A, Xg, B) <= 1e-14, (i, sizes[i])
        if kind == 0:
            _, X, st = orc.hpd_solve(A, B, orc.LOWER, nb=32)
        else:
            _, X, st = orc.gaussian_elimination(A, B, nb=32)
        assert st == 0
        assert np.max(np.abs(Xg - X)) <= 1e-8 * max(1.0, np.max(np.abs(X))), i
    plan.close()


def test_refined_plan_falls_back_to_fp64(handle):
    """A system too ill-conditioned for the FP32 factor is re-solved in FP64
    (iters -1) to the same backward error; a matrix that is not HPD reports
    its column from the FP64 factorization; the others refine as usual."""
    good = inputs.spd_ggt(200, 1)
    ill = np.asfortranarray(inputs.spd_spectrum(160, 1e12, 2))
    bad = good.copy(order="F")
    bad[70, 70] = -3.0
    mats = [good, ill, bad, inputs.spd_ggt(64, 3)]
    Bs = [inputs.normal(m.shape[0], 3, 10 + i) for i, m in enumerate(mats)]
    dA = [eg.colmajor_cuda(m) for m in mats]
    dB = [eg.colmajor_cuda(b) for b in Bs]
    plan = eg.BatchPlan(handle, 0, dA, dB, precision=1)
    plan.run()
    info, its = plan.info(), plan.iters()
    assert info == [0, 0, 71, 0]
    assert its[1] == -1 and its[2] == -1 and its[0] >= 0 and its[3] >= 0
    for i in (0, 1, 3):
        assert _berr(mats[i], dB[i].cpu().numpy(), Bs[i]) <= 1e-14, i
    plan.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_autotune_restores_inputs_and_reports_shapes(handle, precision):
    """The tile-shape autotuner leaves every input as it found it, reports a
    valid shape per size class, and the tuned plan still solves correctly."""
    import torch
    r = inputs.rng(31 + precision)
    sizes = [int(x) for x in r.integers(32, 513, 40)] + [512, 100, 200]
    As = [inputs.uniform(n, n, 60 + i) for i, n in enumerate(sizes)]
    Bs = [inputs.normal(n, 1 + i % 8, 90 + i) for i, n in enumerate(sizes)]
    dA = [eg.colmajor_cuda(a) for a in As]
    dB = [eg.colmajor_cuda(b) for b in Bs]
    plan = eg.BatchPlan(handle, 1, dA, dB, precision=precision)
    ms, grid = plan.autotune(reps=1)
    torch.cuda.synchronize()
    assert ms > 0 and grid >= 1
    for i in range(len(sizes)):
        assert np.array_equal(dA[i].cpu().numpy(), As[i]), i
        assert np.array_equal(dB[i].cpu().numpy(), Bs[i]), i
    shape = plan.shape()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert 1 <= len(shape) <= 3
    for s in shape:
        assert s["nmax"] in (128, 256, 512) and s["panel"] in (16, 32) and s["threads"] in (128, 256)
        assert 1 <= s["grid"] <= 4 * sms
    plan.run()
    assert plan.info() == [0] * len(sizes)
    for i, (A, B) in enumerate(zip(As, Bs)):
        assert _berr(A, dB[i].cpu().numpy(), B) <= 1e-14, i
    plan.close()
