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
