"""bench.py's multi-GPU logic on CPU: two gloo ranks, replicas only (no data
collective). The job's time is the slowest rank's, and `value` counts every
rank's solve."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, outdir):
    import json
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        local_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        ms = bench.max_over_ranks(local_ms, world, "cpu")
        with open(os.path.join(outdir, f"{rank}.json"), "w") as f:
            json.dump([ms, bench.replica_seconds_per_solve(ms, world)], f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank_and_count_both_solves(tmp_path):
    import json
    world = 2
    port = 29500 + os.getpid() % 1000
    mp.spawn(_rank, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    res = {r: json.load(open(tmp_path / f"{r}.json")) for r in range(world)}
    assert res[0] == res[1]
    ms, value = res[0]
    assert ms == 15.0
    assert value == pytest.approx(15.0 / 1e3 / 2)


def test_one_rank_is_its_own_value():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.replica_seconds_per_solve(20.0, 1) == pytest.approx(0.02)
