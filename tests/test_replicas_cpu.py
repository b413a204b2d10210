"""The multi-GPU form is replicas only (the path has no exchange step): each
rank advances its own copy and the job's throughput is set by the slowest
rank.  This checks that aggregation with two gloo ranks on the CPU."""
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [100.0, 250.0][rank]
        e2e_s = [0.5, 0.3][rank]
        value, max_ms, e2e, max_e2e = bench.replica_throughput(ms, e2e_s, 1000, 10, dist, device="cpu")
        out.put((rank, value, max_ms, e2e, max_e2e))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, max_ms, e2e, max_e2e in res:
        assert max_ms == pytest.approx(250.0) and max_e2e == pytest.approx(0.5)
        assert value == pytest.approx(2 * 1000 * 10 / 0.25 / 1e6)  # MLUPS of both replicas over the slow rank
        assert e2e == pytest.approx(2 * 1000 * 10 / 0.5 / 1e6)
