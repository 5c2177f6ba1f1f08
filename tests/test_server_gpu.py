"""Serving loop (svg_server_*): requests answered through continuous batching on
several streams give the same results as the synchronous batch calls, alone
and mixed with other requests; builds run through the server, and a budget
too small for every graph evicts and rebuilds them without changing results."""
import numpy as np
import pytest

from oracle.refbind import CpuOracle
from svg_b200 import SVG, Mesh, Server, meshgen
from svg_b200.build_ext import build as build_lib

pytestmark = pytest.mark.gpu
RTOL = 1e-8
MB = 1 << 20


def rel_err(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


@pytest.fixture(scope="module")
def graph():
    build_lib()
    pos, faces = meshgen.torus(1.0, 0.35, 60, 40, 0.02, seed=9)
    m = Mesh.from_arrays(pos, faces)
    s = SVG()
    s.AssignMesh(m)
    s.SetParameters(50)
    s.ConstructSVG()
    return s, m, pos, faces


def _requests(nv, seed, n_sssd, set_sizes):
    rng = np.random.default_rng(seed)
    reqs = [("s", int(a), int(b)) for a, b in rng.integers(0, nv, (n_sssd, 2))]
    for k in set_sizes:
        srcs = rng.choice(nv, k, replace=False).astype(np.int32)
        reqs.append(("m", srcs, rng.uniform(0, 0.2, k)))
    order = rng.permutation(len(reqs))
    return [reqs[i] for i in order]


def _serve(srv, gid, reqs, nv):
    tickets = []
    for r in reqs:
        tickets.append(srv.submit_sssd(gid, r[1], r[2]) if r[0] == "s" else srv.submit_msad(gid, r[1], r[2]))
    out = []
    for r, t in zip(reqs, tickets):
        res = srv.wait(t, 300.0)
        assert res["status"] == 0
        if r[0] == "s":
            srv.take(t)
            out.append(res["dist"])
        else:
            assert res["n"] == nv
            out.append(srv.take(t, nv))
    return out


def _check_against_sync(s, reqs, got):
    for r, g in zip(reqs, got):
        if r[0] == "s":
            assert g == s.sssd_batch(np.array([r[1]], np.int32), np.array([r[2]], np.int32))[0]
        else:
            d, src = s.msad_batch([r[1]], [r[2]])
            assert np.array_equal(g[0], d[0])
            assert (g[1] == src[0]).mean() > 0.999   # equal-distance ties may pick either source


def test_mixed_requests_match_synchronous_calls(graph):
    s, m, pos, faces = graph
    nv = m.vertNum
    reqs = _requests(nv, 3, 400, [1, 2, 7, 30, 200, 1000, 5, 64])
    srv = Server(lanes=3, max_batch=64, slots_per_lane=16, staging_in_bytes=256 << 10,
                 staging_out_bytes=16 * MB, hbm_budget=2048 * MB)
    try:
        gid = srv.add_graph(s)
        got = _serve(srv, gid, reqs, nv)
        st = srv.stats()
        assert st["batched_requests"] == len(reqs)
        assert st["batches"] < len(reqs)          # requests were batched together
    finally:
        srv.close()
    _check_against_sync(s, reqs, got)
    # the same requests alone (one per batch) give the same answers
    srv = Server(lanes=1, max_batch=1, slots_per_lane=4, staging_in_bytes=256 << 10, staging_out_bytes=4 * MB,
                 hbm_budget=2048 * MB)
    try:
        gid = srv.add_graph(s)
        alone = _serve(srv, gid, reqs[:60], nv)
    finally:
        srv.close()
    for r, a, b in zip(reqs[:60], alone, got[:60]):
        if r[0] == "s":
            assert a == b
        else:
            assert np.array_equal(a[0], b[0])


def test_sssd_matches_oracle_astar(graph):
    s, m, pos, faces = graph
    off, adj, dist = s.csr()
    cm = CpuOracle().mesh(pos, faces)
    reqs = _requests(m.vertNum, 5, 200, [])
    srv = Server(lanes=2, max_batch=32, slots_per_lane=8, hbm_budget=2048 * MB,
                 staging_in_bytes=64 << 10, staging_out_bytes=2 * MB)
    try:
        got = np.array(_serve(srv, srv.add_graph(s), reqs, m.vertNum))
    finally:
        srv.close()
    ref, _ = cm.sssd(off, adj, dist, [r[1] for r in reqs], [r[2] for r in reqs])
    assert np.all(rel_err(got, ref) <= RTOL)


def test_bad_requests_fail_alone(graph):
    s, m, pos, faces = graph
    srv = Server(lanes=1, max_batch=8, slots_per_lane=4, hbm_budget=1024 * MB,
                 staging_in_bytes=64 << 10, staging_out_bytes=16 << 10)
    try:
        gid = srv.add_graph(s)
        bad = srv.submit_sssd(gid, 0, m.vertNum)                 # vertex out of range
        big = srv.submit_msad(gid, np.arange(10, dtype=np.int32))  # result larger than staging
        ok = srv.submit_sssd(gid, 0, 17)
        assert srv.wait(bad)["status"] == 1
        assert srv.wait(big)["status"] == 1
        r = srv.wait(ok)
        assert r["status"] == 0
        assert r["dist"] == s.SolveSSSD(0, 17)
        for t in (bad, big, ok):
            srv.take(t)
        with pytest.raises(Exception):
            srv.submit_sssd(gid + 5, 0, 1)                       # unknown graph
    finally:
        srv.close()


def test_builds_evict_and_rebuild_under_budget():
    build_lib()
    meshes, direct = [], []
    for seed in (1, 2, 3):
        pos, faces = meshgen.torus(1.0, 0.35, 125, 80, 0.02, seed=seed)
        m = Mesh.from_arrays(pos, faces)
        g = SVG()
        g.AssignMesh(m)
        g.SetParameters(50)
        g.ConstructSVG()
        meshes.append(m)
        direct.append(g)
    nv = meshes[0].vertNum
    # room for one or two of these graphs beside a build's scratch, never all three
    budget = 160 * MB
    srv = Server(lanes=2, max_batch=64, slots_per_lane=16, hbm_budget=budget,
                 staging_in_bytes=64 << 10, staging_out_bytes=4 * MB)
    try:
        ids, tickets = [], []
        for m in meshes:
            gid, t = srv.submit_build(m, 50)
            ids.append(gid)
            tickets.append(t)
        for t in tickets:
            assert srv.wait(t, 600.0)["status"] == 0
            srv.take(t)
        assert srv.stats()["evictions"] >= 1
        # round-robin over the graphs: evicted ones are rebuilt on demand
        for rnd in range(3):
            for k, gid in enumerate(ids):
                reqs = _requests(nv, 100 * rnd + k, 40, [3, 50])
                got = _serve(srv, gid, reqs, nv)
                _check_against_sync(direct[k], reqs, got)
                assert srv.stats()["resident_bytes"] <= budget
        st = srv.stats()
        assert st["rebuilds"] >= 1
        assert st["resident_graphs"] < 3
    finally:
        srv.close()


def test_msad_results_into_caller_buffers(graph):
    s, m, pos, faces = graph
    nv = m.vertNum
    rng = np.random.default_rng(8)
    sets = [rng.choice(nv, k, replace=False).astype(np.int32) for k in (1, 12, 300)]
    bufs = [(np.zeros(nv), np.zeros(nv, np.int32)) for _ in sets]
    srv = Server(hbm_budget=1024 * MB, staging_in_bytes=64 << 10, staging_out_bytes=4 * MB)
    try:
        gid = srv.add_graph(s)
        tk = [srv.submit_msad(gid, x, out=b) for x, b in zip(sets, bufs)]
        for t in tk:
            r = srv.wait(t, 300.0)
            assert r["status"] == 0 and r["n"] == nv
            srv.take(t)
    finally:
        srv.close()
    d, src = s.msad_batch(sets)
    for q, (bd, bs) in enumerate(bufs):
        assert np.array_equal(bd, d[q])
        assert (bs == src[q]).mean() > 0.999
