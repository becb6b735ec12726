"""bench.py's multi-GPU plumbing, on the host: two replicas over gloo.

The SIMPLE path is not split across GPUs; `bench.py --gpus N` runs N
independent replicas, one per GPU, whose only collectives are barriers and
the max-over-ranks reduction of the timed region.  These tests run that
plumbing as two processes on CPU (gloo), the way torchrun starts the ranks
(RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* in the environment), and check
that every rank sees the slowest rank's time and that the whole-job rate
counts all ranks' units over it.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import bench
    w, r, local, dist = bench.dist_setup(backend="gloo")
    try:
        assert (w, r, local) == (world, rank, rank)
        bench.barrier(dist)
        # rank r "took" 1 + r seconds for its 1000 cells x 10 steps
        t_max = bench.allreduce_max(dist, 1.0 + rank)
        out[rank] = (t_max, bench.job_rate(w, 1000 * 10, t_max))
        bench.barrier(dist)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_replicas_reduce_the_slowest_time(world):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        codes = [p.exitcode for p in procs]
        assert codes == [0] * world, codes
        res = dict(out)
    slowest = float(world)
    for r in range(world):
        t_max, rate = res[r]
        assert t_max == slowest
        assert rate == world * 10000 / slowest


def test_single_process_needs_no_group():
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    world, rank, local, dist = bench.dist_setup()
    assert (world, rank, local, dist) == (1, 0, 0, None)
    assert bench.allreduce_max(None, 2.5) == 2.5
    assert bench.job_rate(1, 100, 2.0) == 50.0
