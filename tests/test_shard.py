"""Sharded construction across ranks (svg_b200/shard.py), world size 2 with
the gloo backend on CPU: each rank builds its contiguous source range - here
with the C restatement of the reference's construction, the CPU stand-in for
the GPU build - and all-gathers its CSR slice; the assembled graph must equal
the single-rank build of every source, bit for bit, on every rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from svg_b200.shard import assemble_csr, shard_ranges, slice_of_csr


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_csr(pos, faces, K, sources):
    from oracle.refbind import CpuOracle
    from tests.helpers import csr_from_padded
    rows = CpuOracle().mesh(pos, faces).build(K, sources, threads=1)
    off, nodes = csr_from_padded(rows.tails, rows.nodes)
    return off, nodes["adj"].copy(), nodes["dist"].copy()


def _mesh():
    from svg_b200 import meshgen
    return meshgen.height_field(18, seed=4)


def _rank(rank, world, port, K, q):
    import torch.distributed as dist
    from svg_b200.shard import gather_csr
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pos, faces = _mesh()
        V = len(pos)
        b, e = shard_ranges(V, world)[rank]
        off, adj, w = _oracle_csr(pos, faces, K, np.arange(b, e, dtype=np.int32))
        degs, adjs, ws = gather_csr(dist, np.diff(off).astype(np.int32), adj, w)
        full = assemble_csr([d.numpy() for d in degs], [a.numpy() for a in adjs], [x.numpy() for x in ws])
        q.put((rank, (b, e), [x.tolist() for x in full]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_sharded_build_gathers_to_the_single_rank_graph(world):
    K = 24
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, K, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pos, faces = _mesh()
    ref = _oracle_csr(pos, faces, K, None)
    ranges = sorted(r for _, r, _ in out)
    assert ranges[0][0] == 0 and ranges[-1][1] == len(pos)
    assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
    for _, _, full in out:
        off, adj, w = (np.asarray(full[0], np.int64), np.asarray(full[1], np.int32), np.asarray(full[2]))
        assert np.array_equal(off, ref[0])
        assert np.array_equal(adj, ref[1])
        assert np.array_equal(w, ref[2])  # float64 lists round-trip exactly


def test_shard_ranges_cover_and_balance():
    assert shard_ranges(10, 3) == [(0, 3), (3, 6), (6, 10)]
    assert shard_ranges(5, 8)[-1] == (4, 5)
    cost = np.r_[np.full(50, 10.0), np.full(50, 1.0)]
    r = shard_ranges(100, 2, cost)
    assert r[0][0] == 0 and r[1][1] == 100 and r[0][1] == r[1][0]
    left = cost[:r[0][1]].sum()
    assert abs(left - cost.sum() / 2) <= 10.0


def test_slice_and_assemble_are_inverse():
    rng = np.random.default_rng(0)
    deg = rng.integers(0, 5, 40).astype(np.int32)
    off = np.r_[0, np.cumsum(deg)].astype(np.int64)
    adj = rng.integers(0, 40, off[-1]).astype(np.int32)
    w = rng.random(off[-1])
    parts = [slice_of_csr(off, adj, w, b, e) for b, e in shard_ranges(40, 3)]
    o2, a2, w2 = assemble_csr(*zip(*parts))
    assert np.array_equal(o2, off) and np.array_equal(a2, adj) and np.array_equal(w2, w)
