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


def test_server_structure_test_routes_symmetric_ge_requests():
    # mode 1: a GE request whose A is exactly symmetric with a positive
    # diagonal is tried as HPD first (path 4: FP64 Cholesky below the mixed
    # threshold, path 5: the mixed solver above it); a symmetric indefinite A
    # fails that factorization and a nonsymmetric A skips it, both ending on
    # the LU path (0).  Every answer is GaussianElimination's x to backward
    # error <= 1e-14.
    n = 700
    spd = inputs.spd_spectrum(n, 1e5, 21)
    indef = np.asfortranarray(spd - 10.0 * np.eye(n))  # eigenvalues from -9: symmetric indefinite
    assert np.all(np.diag(indef) > 0)
    gen = inputs.uniform(n, n, 22)
    B = inputs.normal(n, 3, 23)
    for min_n, spd_path in ((6144, 4), (0, 5)):
        srv = eg.Server(0, hbm_budget_bytes=8 << 30, slots=2, mode=1, mixed_min_n=min_n)
        (Xs, Xi, Xg), (fs, fi, fg) = _solve_all(srv, [(1, spd, B), (1, indef, B), (1, gen, B)])
        srv.close()
        assert fs["status"] == 0 and fs["path"] == spd_path, fs
        assert fi["status"] == 0 and fi["path"] == 0, fi
        assert fg["status"] == 0 and fg["path"] == 0, fg
        for A, X in ((spd, Xs), (indef, Xi), (gen, Xg)):
            assert _berr(A, X, B) <= 1e-14
    # mode 0 never takes the test
    srv = eg.Server(0, hbm_budget_bytes=8 << 30, slots=2, mode=0)
    (X0,), (f0,) = _solve_all(srv, [(1, spd, B)])
    srv.close()
    assert f0["path"] == 0 and _berr(spd, X0, B) <= 1e-14


@pytest.mark.parametrize("mode,n", [(0, 600), (1, 600), (1, 200)])
def test_server_resident_matrices_reuse_their_factor(mode, n):
    # matrices registered once; requests send only B: exactly one request per
    # matrix forms the factor (path 6), the others reuse it (path 7), and
    # every answer equals a one-off request's within 1e-10 and reaches
    # backward error <= 1e-14.  A nonsymmetric GE matrix takes LU, an HPD one
    # Cholesky; a singular matrix fails every request with its status.  Small
    # matrices (n <= 512, which one-off requests would batch) too.
    spd = inputs.spd_spectrum(n, 1e4, 31)
    gen = inputs.uniform(n, n, 32)
    sing = gen.copy(order="F")
    sing[:, 17] = 0.0
    srv = eg.Server(0, hbm_budget_bytes=8 << 30, slots=3, mode=mode)
    mids = [srv.register(0, spd), srv.register(1, gen), srv.register(1, spd), srv.register(1, sing)]
    mats = [spd, gen, spd, sing]
    Bs = [inputs.normal(n, 1 + (i % 5), 40 + i) for i in range(24)]
    ids, Xs = [], []
    for i, B in enumerate(Bs):
        X = np.zeros(B.shape, order="F")
        ids.append(srv.submit_resident(mids[i % 4], B, X))
        Xs.append(X)
    infos = [srv.query(i, wait=True) for i in ids]
    (X1,), (f1,) = _solve_all(srv, [(1, gen, Bs[1])])
    for m in mids:
        srv.unregister(m)
    srv.close()
    for k in range(4):
        paths = [infos[i]["path"] for i in range(k, 24, 4)]
        if k == 3:
            assert all(infos[i]["status"] == eg.SINGULAR for i in range(3, 24, 4))
            continue
        assert sorted(paths) == [6] + [7] * 5, (k, paths)
        for i in range(k, 24, 4):
            assert infos[i]["status"] == 0
            assert _berr(mats[k], Xs[i], Bs[i]) <= 1e-14
    assert f1["status"] == 0 and np.abs(Xs[1] - X1).max() <= 1e-10 * np.abs(X1).max()


def test_server_resident_budget():
    n = 512
    A = inputs.spd_ggt(n, 5)
    per = 2 * 8 * n * n + 4 * n
    srv = eg.Server(0, hbm_budget_bytes=per + 4096, slots=1, mode=0)
    m = srv.register(0, A)
    with pytest.raises(eg.ElemGPUError):
        srv.register(0, A)  # the budget holds one
    srv.unregister(m)
    m = srv.register(0, A)  # room again
    srv.unregister(m)
    srv.close()
