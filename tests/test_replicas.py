"""Multi-rank measurement path of bench.py (replicas, weak scaling) on CPU
with the gloo backend, world size 2: times combine as the max over ranks,
work as the sum."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [300.0, 500.0][rank]
    edges = [1.0e6, 2.0e6][rank]
    v = bench.replica_value(dist, edges, ms, device="cpu")
    m = bench.max_over_ranks(dist, ms, device="cpu")
    s = bench.sum_over_ranks(dist, edges, device="cpu")
    bench.barrier(dist)
    dist.destroy_process_group()
    q.put((rank, v, m, s))


def test_replica_throughput_is_total_work_over_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, v, m, s in out:
        assert m == 500.0
        assert s == 3.0e6
        assert v == pytest.approx(3.0e6 / 0.5)


def test_single_rank_reduces_to_identity():
    import bench
    assert bench.replica_value(None, 10.0, 1000.0) == 10.0
    assert bench.max_over_ranks(None, 7.0) == 7.0
