"""GPU results against the reference itself: the golden vectors that the
reference's own code produced (tests/golden/ref_golden.npz), and, where
oracle/_ref is built, the reference library run on the same seeded inputs at
the benchmark configurations (Cholesky + HPD solve n = 2048 / 16 RHS; LU with
partial pivoting + solve n = 8192 / 64 RHS, pivots index for index).

Tolerances as tests/test_gpu_parity.py: factors 1e-11 (Cholesky) and 1e-10
(LU) of the largest entry, solves 1e-9, pivots identical."""
import os

import numpy as np
import pytest

import elemental_b200 as eg
from elemental_b200 import inputs
from oracle import ref

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "ref_golden.npz")


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b))))


def _host(t):
    return np.asfortranarray(t.cpu().numpy())


def test_gpu_matches_reference_golden_vectors(handle):
    import torch
    g = np.load(GOLDEN)
    for key in [k for k in g.files if k.startswith("chol_in_")]:
        tag = key[len("chol_in_"):]
        n, uplo, nb = (int(x) for x in tag.split("_"))
        handle.set_blocksize(nb)
        try:
            dA = eg.colmajor_cuda(g[key])
            handle.cholesky(dA, uplo)
        finally:
            handle.set_blocksize(128)
        tri = np.tril if uplo == eg.LOWER else np.triu
        assert rel(tri(_host(dA)), tri(g["chol_out_" + tag])) <= 1e-11
    for pre in ("lu", "lurect"):
        for key in [k for k in g.files if k.startswith(pre + "_in_")]:
            tag = key[len(pre + "_in_"):]
            A = g[key]
            dA = eg.colmajor_cuda(A)
            dp = torch.zeros(min(A.shape), dtype=torch.int32, device="cuda")
            handle.lu(dA, dp)
            assert np.array_equal(dp.cpu().numpy(), g[pre + "_piv_" + tag])
            assert rel(_host(dA), g[pre + "_out_" + tag]) <= 1e-10
            if pre == "lu":
                dB = eg.colmajor_cuda(g["lu_rhs_" + tag])
                handle.lu_solve_after(dA, dp, dB, eg.NORMAL)
                assert rel(_host(dB), g["lu_x_" + tag]) <= 1e-9
    dA, dB = eg.colmajor_cuda(g["hpd_A"]), eg.colmajor_cuda(g["hpd_B"])
    handle.hpd_solve(dA, dB, eg.LOWER)
    assert rel(_host(dB), g["hpd_X"]) <= 1e-9
    dA, dB = eg.colmajor_cuda(g["ge_A"]), eg.colmajor_cuda(g["ge_B"])
    handle.gaussian_elimination(dA, dB)
    assert rel(_host(dB), g["ge_X"]) <= 1e-9
    for inv, key in ((False, "swap_out"), (True, "swap_out_inv")):
        dB = eg.colmajor_cuda(g["swap_B"])
        handle.apply_row_pivots(dB, torch.from_numpy(g["swap_p"]).cuda(), inv)
        assert np.array_equal(_host(dB), g[key])


needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


@needs_ref
def test_gpu_matches_reference_cholesky_config_n2048(handle):
    n, k = 2048, 16
    A = inputs.spd_ggt(n, 20240)
    B = inputs.normal(n, k, 20241)
    dA, dB = eg.colmajor_cuda(A), eg.colmajor_cuda(B)
    handle.hpd_solve(dA, dB, eg.LOWER)
    F, X, st = ref.hpd_solve(A, B, ref.LOWER, nb=128)
    assert st == 0
    assert rel(np.tril(_host(dA)), np.tril(F)) <= 1e-11
    assert rel(_host(dB), X) <= 1e-9


@needs_ref
def test_gpu_matches_reference_lu_config_n8192(handle):
    import torch
    n, k = 8192, 64
    A = inputs.uniform(n, n, 20240)
    B = inputs.normal(n, k, 20241)
    dA = eg.colmajor_cuda(A)
    dp = torch.zeros(n, dtype=torch.int32, device="cuda")
    handle.lu(dA, dp)
    dB = eg.colmajor_cuda(B)
    handle.lu_solve_after(dA, dp, dB, eg.NORMAL)
    F, p, st = ref.lu(A, 128)
    assert st == 0
    assert np.array_equal(dp.cpu().numpy(), p), np.nonzero(dp.cpu().numpy() != p)[0][:10]
    assert rel(_host(dA), F) <= 1e-9
    X = ref.lu_solve_after(F, p, B)
    assert rel(_host(dB), X) <= 1e-7
