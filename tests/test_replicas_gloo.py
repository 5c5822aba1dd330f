"""The N > 1 path of bench.py on CPU: two gloo ranks, each standing in for one
GPU replica with its own device time.  Every rank takes the max over ranks
of each timing (the slowest replica times the job) and rank 0 reports the
whole-job throughput of both replicas."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        step_ms, e2e_ms = 10.0 + 5.0 * rank, 30.0 - 7.0 * rank
        got = bench.reduce_max_over_ranks([step_ms, e2e_ms], world)
        results[rank] = (got, bench.replica_throughput(1000, 20, world, got[0]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_replicas_max_over_ranks_gloo():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        results = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), results), nprocs=world, join=True)
        res = dict(results)
    for rank in range(world):
        (step, e2e), value = res[rank]
        assert step == 15.0 and e2e == 30.0                    # slowest rank's times
        assert value == pytest.approx(world * 1000 * 20 / 15e-3)


def test_single_rank_is_identity():
    import bench
    assert bench.reduce_max_over_ranks([1.5, 2.5], 1) == [1.5, 2.5]
    assert bench.replica_throughput(100, 10, 1, 2.0) == pytest.approx(100 * 10 / 2e-3)
