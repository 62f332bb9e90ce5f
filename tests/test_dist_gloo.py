"""The multi-rank plumbing of bench.py (one process per GPU, barrier, max-over-
ranks timing) on two gloo ranks on the CPU: each rank reports its own time
and both end with the slowest; a rank that fails raises in its own process
and the launcher sees a non-zero exit."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out_dir):
    sys.path.insert(0, ROOT)
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(ws),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "EGPU_BENCH_BACKEND": "gloo"})
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (ws, rank, rank)
    bench.barrier(w)
    t = bench.max_over_ranks(w, 10.0 + 5.0 * rank, "cpu")
    bench.barrier(w)
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(repr(t))
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_share_the_max_time(tmp_path):
    ws = 2
    mp.start_processes(_rank_main, args=(ws, _free_port(), str(tmp_path)), nprocs=ws, start_method="spawn",
                       join=True)
    vals = [float(open(tmp_path / f"rank{r}.txt").read()) for r in range(ws)]
    assert vals == [15.0, 15.0]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    saved = {k: os.environ.pop(k, None) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    try:
        assert bench.dist_setup() == (1, 0, 0)
        assert bench.max_over_ranks(1, 3.5, "cpu") == 3.5
        bench.barrier(1)
    finally:
        for k, v in saved.items():
            if v is not None:
                os.environ[k] = v


def _failing_rank_main(rank, ws, port, out_dir):
    _rank_main(rank, ws, port, out_dir)  # all collectives first: nobody waits on the failed rank
    if rank == 1:
        raise RuntimeError("rank 1 failed after its last collective")


@pytest.mark.timeout(180)
def test_failed_rank_is_reported_by_the_launcher(tmp_path):
    with pytest.raises(Exception) as e:
        mp.start_processes(_failing_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2,
                           start_method="spawn", join=True)
    assert "rank 1 failed" in str(e.value)


def _shard_rank_main(rank, ws, port, out_dir):
    # one list of independent systems shared by `ws` ranks: each rank solves
    # the systems the partition gives it (here with the CPU checker, as the
    # host plumbing is what is under test) and the statuses and solutions are
    # gathered on the host
    sys.path.insert(0, ROOT)
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(ws),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "EGPU_BENCH_BACKEND": "gloo"})
    import pickle

    import numpy as np

    import bench
    import torch.distributed as dist
    from elemental_b200 import inputs
    from oracle import pyoracle as orc
    w, r, _ = bench.dist_setup()
    rs = np.random.default_rng(11)
    sizes = [int(x) for x in rs.integers(8, 120, 40)]
    kinds = [int(x) for x in rs.integers(0, 2, 40)]
    mine, load = bench.shard_of(w, r, sizes, kinds)
    res = {}
    for i in mine:
        n = sizes[i]
        A = inputs.spd_ggt(n, 100 + i) if kinds[i] == 0 else inputs.uniform(n, n, 100 + i)
        B = inputs.normal(n, 2, 200 + i)
        _, X, st = orc.hpd_solve(A, B, orc.LOWER, nb=32) if kinds[i] == 0 else orc.gaussian_elimination(A, B, 32)
        res[i] = (st, X)
    parts = bench.gather_to_host(w, (r, mine, res))
    if r == 0:
        with open(os.path.join(out_dir, "gathered.pkl"), "wb") as f:
            pickle.dump({"sizes": sizes, "kinds": kinds, "parts": parts, "load": list(load)}, f)
    bench.barrier(w)
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_shard_one_system_list(tmp_path):
    import pickle

    import numpy as np

    from elemental_b200 import inputs
    from oracle import pyoracle as orc
    ws = 2
    mp.start_processes(_shard_rank_main, args=(ws, _free_port(), str(tmp_path)), nprocs=ws, start_method="spawn",
                       join=True)
    g = pickle.load(open(tmp_path / "gathered.pkl", "rb"))
    sizes, kinds, parts = g["sizes"], g["kinds"], g["parts"]
    owned = sorted(i for _, mine, _ in parts for i in mine)
    assert owned == list(range(len(sizes)))  # every system exactly once
    cost = [(n ** 3) * (2.0 / 3.0 if k else 1.0 / 3.0) for n, k in zip(sizes, kinds)]
    loads = [sum(cost[i] for i in mine) for _, mine, _ in parts]
    assert np.allclose(sorted(loads), sorted(g["load"]))
    assert max(loads) - min(loads) <= max(cost)  # greedy balance bound
    # the gathered statuses and solutions equal a one-rank run of the list
    for _, mine, res in parts:
        for i in mine:
            n = sizes[i]
            A = inputs.spd_ggt(n, 100 + i) if kinds[i] == 0 else inputs.uniform(n, n, 100 + i)
            B = inputs.normal(n, 2, 200 + i)
            _, X, st = orc.hpd_solve(A, B, orc.LOWER, nb=32) if kinds[i] == 0 else orc.gaussian_elimination(A, B, 32)
            assert res[i][0] == st == 0
            assert np.array_equal(res[i][1], X)


def test_partition_is_deterministic_and_balanced():
    sys.path.insert(0, ROOT)
    import numpy as np

    import elemental_b200 as eg
    rs = np.random.default_rng(3)
    n = rs.integers(32, 513, 4096)
    k = rs.integers(0, 2, 4096)
    o1, l1 = eg.partition_systems(n, k, 8)
    o2, l2 = eg.partition_systems(n, k, 8)
    assert np.array_equal(o1, o2) and np.array_equal(l1, l2)
    assert set(np.unique(o1)) == set(range(8))
    cost = n.astype(float) ** 3 * np.where(k == 1, 2 / 3, 1 / 3)
    assert np.allclose([cost[o1 == p].sum() for p in range(8)], l1)
    assert l1.max() - l1.min() <= cost.max()
    o, l = eg.partition_systems(n, None, 1)
    assert np.all(o == 0)
