"""The multi-GPU form is replicas only: every rank runs its own frames and the bench
reduces the ranks' numbers (max of times, sum of particles).  The reduction runs
here as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        vals = [10.0 + rank, 100 * (rank + 1), 1.0 + 2 * rank, 7 * (rank + 1)]
        out[rank] = bench.reduce_replicas(dist, vals, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_reduction_is_max_of_times_and_sum_of_particles():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        ps = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(90)
            assert p.exitcode == 0
        for r in range(2):
            assert out[r] == (11.0, 300.0, 3.0, 21.0)
