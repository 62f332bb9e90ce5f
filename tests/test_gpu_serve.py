"""Request server (continuous batching): every result is the same alone and
in the mix (within 1e-10 relative, the difference between the batched
nb = 32 and the single-system nb = 128 blockings), every answer reaches a
normwise backward error <= 1e-14, admission respects the HBM budget, and the
mixed-precision mode falls back to FP64 where refinement cannot converge."""
import numpy as np
import pytest

import elemental_b200 as eg
from elemental_b200 import inputs

pytestmark = pytest.mark.gpu


def _berr(A, X, B):
    R = B - A @ X
    return np.max(np.abs(R).max(axis=0) / (np.abs(A).sum(axis=1).max() * np.abs(X).max(axis=0) + np.abs(B).max(axis=0)))


def _requests(seed, count):
    r = inputs.rng(seed)
    out = []
    for i in range(count):
        kind = int(r.integers(0, 2))
        n = int(np.exp(r.uniform(np.log(16), np.log(1500))))
        k = int(r.integers(1, 20))
        A = inputs.spd_ggt(n, 900 + i) if kind == 0 else inputs.uniform(n, n, 900 + i)
        out.append((kind, A, inputs.normal(n, k, 1900 + i)))
    return out


def _solve_all(srv, reqs):
    Xs, ids = [], []
    for kind, A, B in reqs:
        X = np.zeros(B.shape, order="F")
        ids.append(srv.submit(kind, A, B, X))
        Xs.append(X)
    infos = [srv.query(i, wait=True) for i in ids]
    return Xs, infos


def test_server_mix_equals_alone():
    reqs = _requests(5, 40)
    srv = eg.Server(0, hbm_budget_bytes=8 << 30, slots=4, mode=0)
    Xmix, infos = _solve_all(srv, reqs)
    assert all(f["status"] == 0 for f in infos)
    assert any(f["path"] == 2 for f in infos) and any(f["path"] == 0 for f in infos)
    alone = []
    for kind, A, B in reqs:  # one at a time through the same server
        X = np.zeros(B.shape, order="F")
        rid = srv.submit(kind, A, B, X)
        assert srv.query(rid, wait=True)["status"] == 0
        alone.append(X)
    srv.close()
    for (kind, A, B), Xm, Xa in zip(reqs, Xmix, alone):
        assert _berr(A, Xm, B) <= 1e-14
        assert _berr(A, Xa, B) <= 1e-14
        assert np.max(np.abs(Xm - Xa)) <= 1e-10 * np.max(np.abs(Xa))


def test_server_budget_admission():
    A = inputs.spd_ggt(1200, 3)
    B = inputs.normal(1200, 4, 4)
    per = 8 * (1200 * 1200 + 2 * 1200 * 4) + 8 * 128 * 128 + 8 * 1200 * 4
    srv = eg.Server(0, hbm_budget_bytes=per + 1024, slots=4, mode=0)  # room for one at a time
    Xs, infos = _solve_all(srv, [(0, A, B)] * 6)
    assert all(f["status"] == 0 for f in infos)
    for X in Xs:
        assert _berr(A, X, B) <= 1e-14
    big = inputs.spd_ggt(1600, 5)
    with pytest.raises(eg.ElemGPUError):
        srv.submit(0, big, inputs.normal(1600, 1, 6), np.zeros((1600, 1), order="F"))
    srv.close()


def test_server_mixed_mode_and_fallback():
    srv = eg.Server(0, hbm_budget_bytes=8 << 30, slots=2, mode=1, mixed_min_n=0)
    good = inputs.spd_spectrum(1024, 1e4, 11)
    hard = inputs.spd_spectrum(1024, 1e12, 12)
    B = inputs.normal(1024, 3, 13)
    (Xg, Xh), (fg, fh) = _solve_all(srv, [(0, good, B), (0, hard, B)])
    srv.close()
    assert fg["status"] == 0 and fg["path"] == 1 and fg["berr"] <= 1e-14
    assert _berr(good, Xg, B) <= 1e-14
    assert fh["status"] == 0 and fh["path"] == 3  # TF32x3 factor cannot refine kappa 1e12: FP64 fallback
    assert _berr(hard, Xh, B) <= 1e-14
