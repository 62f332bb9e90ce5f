"""The FP32 dataflow sweep's work queue, built by the library's own host code
(egpu_sweep32_queue, no device needed), run item by item in queue order on
the CPU: every item must find its dependency counters already reached when
its turn comes (so the co-resident CTAs of the cooperative launch always
make progress), and the items' tile products must add up to the triangular
solves L^-1 X, L^-T X and L^-T L^-1 X.

Item arithmetic, as the kernel does it: out(128 x 32) (+/-)= T(128 x k)
v(k x 32) with T a tile of L, of the 512 x 512 super-block inverses W_R, or
of the chain products M_R = L_{R+1,R} W_R / P_R = W_R L_{R,R-1}, read rows
contiguous (maps 0, 2, 4: T(i, k) = M(tm + i, tk + k)) or as columns (maps
1, 3, 5: T(j, k) = M(tk + k, tm + j))."""
import numpy as np
import pytest

import elemental_b200 as eg

S, TM, TK = 512, 128, 32


def _emulate(n, trans, sm_count, nrhs=3, seed=0):
    r = np.random.default_rng(seed)
    A = r.standard_normal((n, n))
    A = A @ A.T + n * np.eye(n)
    L = np.linalg.cholesky(A)
    ns = (n + S - 1) // S
    P_ = ns * S + S
    Lp = np.zeros((P_, P_))
    Lp[:n, :n] = L
    W = np.zeros((S, S * ns))
    for R in range(ns):
        sb = min(S, n - R * S)
        W[:sb, R * S:R * S + sb] = np.linalg.inv(L[R * S:R * S + sb, R * S:R * S + sb])
    M = np.zeros_like(W)
    Pm = np.zeros_like(W)
    for R in range(ns - 1):
        M[:, R * S:(R + 1) * S] = Lp[(R + 1) * S:(R + 2) * S, R * S:(R + 1) * S] @ W[:, R * S:(R + 1) * S]
    for R in range(1, ns):
        Pm[:, R * S:(R + 1) * S] = W[:, R * S:(R + 1) * S] @ Lp[R * S:(R + 1) * S, (R - 1) * S:R * S]
    mats = {0: Lp[:n, :n], 1: Lp[:n, :n], 2: W, 3: W, 4: M, 5: Pm}

    q = eg.sweep32_queue(n, trans, sm_count)
    X = r.standard_normal((n, nrhs))
    Z0 = np.zeros((P_, nrhs))
    Z0[:n] = X
    Df, Yf, Db, Yb = (np.zeros((P_, nrhs)) for _ in range(4))
    ctr = np.zeros(2 + 4 * ns, dtype=np.int64)
    out_backward = 0 if trans == 0 else (2 if trans == 2 else 1)
    for idx, (mp, d, kind, nk, tm, tk, vrow, orow, orows, dep0, need0, dep1, need1, done) in enumerate(q):
        assert ctr[dep0] >= need0, (idx, dep0, need0, ctr[dep0])
        if dep1 >= 0:
            assert ctr[dep1] >= need1, (idx, dep1, need1, ctr[dep1])
        rows = nk * TK
        if kind != 1:  # phase A and kind 2: forward z0 + dz, backward (y or z0) + dv
            s0 = Z0 if d == 0 else (Yf if out_backward == 2 else Z0)
            s1 = Df if d == 0 else Db
            v = s0[vrow:vrow + rows] + s1[vrow:vrow + rows]
        else:          # phase B: the super-block's results
            v = (Yf if d == 0 else Yb)[vrow:vrow + rows].copy()
        v[np.arange(vrow, vrow + rows) >= n] = 0.0
        Mx = mats[int(mp)]
        T = np.zeros((TM, rows))
        if mp in (0, 2, 4):
            blk = Mx[tm:tm + TM, tk:tk + rows]
        else:
            blk = Mx[tk:tk + rows, tm:tm + TM].T
        T[:blk.shape[0], :blk.shape[1]] = blk
        res = T @ v
        outarr = (Yf if d == 0 else Yb) if kind == 0 else (Df if d == 0 else Db)
        outarr[orow:orow + orows] += (1.0 if kind == 0 else -1.0) * res[:orows]
        ctr[done] += 1
    got = (Yb if out_backward else Yf)[:n]
    if trans == 0:
        ref = np.linalg.solve(L, X)
    elif trans == 1:
        ref = np.linalg.solve(L.T, X)
    else:
        ref = np.linalg.solve(L.T, np.linalg.solve(L, X))
    return float(np.abs(got - ref).max() / np.abs(ref).max()), q


@pytest.mark.parametrize("n", [1, 100, 512, 513, 1000, 2049, 4100])
@pytest.mark.parametrize("trans", [0, 1, 2])
def test_sweep_queue_dependencies_and_result(n, trans):
    err, q = _emulate(n, trans, 148)
    assert err <= 1e-10, err
    kinds = set(int(k) for k in q[:, 2])
    if n > S:  # more than one super-block: the next-block items run beside phase A
        assert 2 in kinds


def test_sweep_queue_with_few_sms():
    # the bulk items' k split depends on the grid: a small grid splits less
    err, q8 = _emulate(2049, 2, 8)
    assert err <= 1e-10
    _, q148 = _emulate(2049, 2, 148)
    assert len(q8) < len(q148)


def test_sweep_queue_rejects_bad_arguments():
    with pytest.raises(eg.ElemGPUError):
        eg.sweep32_queue(0, 0)
    with pytest.raises(eg.ElemGPUError):
        eg.sweep32_queue(100, 3)
