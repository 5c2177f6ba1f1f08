"""Parity of the CUDA SVG construction with the reference (GPU).

Bit-exact: neighbour sets, edge lengths and path-end fields of every row
must equal the reference's (golden fixtures) or the oracle's (the C
restatement pinned to the reference) on the same inputs.
"""
import os
import tempfile

import numpy as np
import pytest

from oracle.refbind import CpuOracle
from svg_b200 import MODE_BATCHED, MODE_PLAIN, SVG, Mesh, meshgen
from svg_b200.build_ext import build as build_lib
from tests.helpers import compare_rows, golden_params, load_golden, rows_from_padded, svg_file_bytes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build_lib()


def gpu_build(pos, faces, K, mode=MODE_BATCHED, **kw):
    m = Mesh.from_arrays(pos, faces)
    s = SVG()
    s.AssignMesh(m)
    s.SetParameters(K, kw.pop("split_coef", 10), kw.pop("vert_coef", 2))
    st = s.ConstructSVG(mode=mode, **kw)
    off, nodes = s.CopySVGToHost()
    return off, nodes, st, s, m


@pytest.mark.parametrize("mode", [MODE_BATCHED, MODE_PLAIN])
@pytest.mark.parametrize("name,K", golden_params())
def test_build_matches_reference_golden(name, K, mode):
    """Rows bit-exact against the reference.  Where the reference's fixed
    vertex/split hash tables (K*2, K*10 slots) overflow into their shared sink
    slot, the reference's search is no longer an ICH; such sources must be
    flagged (bit 2) and are excluded, their counters too."""
    g = load_golden(name)
    off, nodes, st, s, _ = gpu_build(g["pos"], g["faces"], K, mode)
    _, _, flags = s.source_stats()
    goff, gnodes = rows_from_padded(g[f"K{K}_tails"], g[f"K{K}_nodes"])
    ok_rows = [r for r in range(len(off) - 1) if not (flags[r] & 2)]
    assert compare_rows(off, nodes, goff, gnodes, rows=ok_rows) == []
    if st["ref_overflow_sources"] == 0:
        assert st["windows_generated"] == int(g[f"K{K}_stats"][:, 0].sum())
    assert st["watchdog_sources"] == 0


def coop_build(pos, faces, K, coop_warps=8, coop_sources=None, **kw):
    """Batched build whose work order comes from a first build's per-source
    costs, with the heaviest `coop_sources` (default: every source) run by
    whole warps (the cooperative form)."""
    m = Mesh.from_arrays(pos, faces)
    s = SVG()
    s.AssignMesh(m)
    s.SetParameters(K, kw.pop("split_coef", 10), kw.pop("vert_coef", 2))
    s.ConstructSVG(heavy_first=0, **kw)   # records the per-source costs on the mesh
    n = len(pos) if coop_sources is None else coop_sources
    st = s.ConstructSVG(heavy_first=1, coop_sources=n, coop_warps=coop_warps, **kw)
    off, nodes = s.CopySVGToHost()
    return off, nodes, st, s, m


@pytest.mark.parametrize("name,K", golden_params())
def test_cooperative_form_matches_reference_golden(name, K):
    """Every source run by a whole warp: the same rows as the reference."""
    g = load_golden(name)
    off, nodes, st, s, _ = coop_build(g["pos"], g["faces"], K)
    assert st["coop_sources"] == len(g["pos"])
    _, _, flags = s.source_stats()
    goff, gnodes = rows_from_padded(g[f"K{K}_tails"], g[f"K{K}_nodes"])
    ok_rows = [r for r in range(len(off) - 1) if not (flags[r] & 2)]
    assert compare_rows(off, nodes, goff, gnodes, rows=ok_rows) == []
    if st["ref_overflow_sources"] == 0:
        assert st["windows_generated"] == int(g[f"K{K}_stats"][:, 0].sum())


@pytest.mark.parametrize("cfg,K,n", [(1, 500, 1200), (0, 100, 1500)])
def test_cooperative_form_matches_oracle_on_benchmark_mesh_samples(cfg, K, n):
    """The heaviest sources of a leading source range run cooperatively (with
    the 1023-entry queue cap binding at K=500), the rest one per lane."""
    pos, faces = meshgen.config_mesh(cfg)
    off, nodes, st, _, _ = coop_build(pos, faces, K, coop_warps=32, coop_sources=n // 3,
                                      source_begin=0, source_end=n)
    assert st["coop_sources"] == n // 3
    (ooff, onodes), rows = _oracle_rows(pos, faces, K, np.arange(0, n, dtype=np.int32))
    assert compare_rows(off[:n + 1], nodes[:off[n]], ooff, onodes) == []
    assert st["windows_generated"] == int(rows.stats[:, 0].sum())


def test_automatic_cooperative_share_keeps_the_graph():
    """The automatic choice (heaviest sources above a lane's average share)
    gives the same CSR as a build with no cooperative warps."""
    pos, faces = meshgen.config_mesh(1, 0.3)
    outs, counts = [], []
    for coop in (0, -1):
        m = Mesh.from_arrays(pos, faces)
        g = SVG()
        g.AssignMesh(m)
        g.SetParameters(300)
        g.ConstructSVG(heavy_first=0)
        st = g.ConstructSVG(heavy_first=1, coop_sources=coop)
        counts.append(st["coop_sources"])
        outs.append(g.csr())
    assert counts[0] == 0
    for x, y in zip(outs[0], outs[1]):
        assert np.array_equal(x, y)


def test_tail_adoption_keeps_the_graph():
    """Warps that adopt their last running lane's source once the queue is
    drained (the default) build the same CSR as warps that do not, and as
    the oracle on a sample of rows."""
    pos, faces = meshgen.config_mesh(1, 0.3)
    outs = []
    for tail in (0, 1):
        m = Mesh.from_arrays(pos, faces)
        g = SVG()
        g.AssignMesh(m)
        g.SetParameters(300)
        g.ConstructSVG(coop_tail=tail, heavy_first=0)
        outs.append(g.CopySVGToHost())
    assert compare_rows(outs[0][0], outs[0][1], outs[1][0], outs[1][1]) == []
    src = np.arange(0, len(pos), 37, dtype=np.int32)
    (ooff, onodes), _ = _oracle_rows(pos, faces, 300, src)
    off, nodes = outs[1]
    got_off = np.concatenate([[0], np.cumsum(np.diff(off)[src])])
    got = np.concatenate([nodes[off[v]:off[v + 1]] for v in src])
    assert compare_rows(got_off, got, ooff, onodes) == []


def test_build_replayed_from_a_captured_cuda_graph_is_identical():
    """opts.graph: the first build captures its device work as a CUDA graph
    kept with the mesh, later builds with the same options replay it; every
    result equals an ordinary build's rows (path ends included), also after
    another mesh's build has re-laid the lane scratch, and an option change
    builds the ordinary way."""
    pos, faces = meshgen.config_mesh(1, 0.3)
    ref_off, ref_nodes, _, _, _ = gpu_build(pos, faces, 200)
    m = Mesh.from_arrays(pos, faces)
    g = SVG()
    g.AssignMesh(m)
    g.SetParameters(200)
    replays = []
    for i in range(3):
        st = g.ConstructSVG(graph=1)
        replays.append(st["graph_replayed"])
        off, nodes = g.CopySVGToHost()
        assert compare_rows(off, nodes, ref_off, ref_nodes) == [], i
        if i == 1:  # another mesh and K re-lay the shared lane scratch
            other = SVG()
            other.AssignMesh(Mesh.from_arrays(*meshgen.torus(1.0, 0.35, 30, 20, 0.02, seed=5)))
            other.SetParameters(40)
            other.ConstructSVG()
    assert replays[0] == 0 and replays[1] == 1
    st = g.ConstructSVG(graph=1, vote_wait=4)  # other options: no replay
    assert st["graph_replayed"] == 0
    off, nodes = g.CopySVGToHost()
    assert compare_rows(off, nodes, ref_off, ref_nodes) == []


def test_autotuned_schedule_keeps_the_graph():
    """The tuner's candidates and its choice change the schedule only: the
    tuned build equals a default build bit for bit (the tuner itself also
    checks every candidate's CSR checksum against the first)."""
    pos, faces = meshgen.config_mesh(1, 0.25)
    m = Mesh.from_arrays(pos, faces)
    g = SVG()
    g.AssignMesh(m)
    g.SetParameters(200)
    g.ConstructSVG(heavy_first=0)
    ref = g.csr()
    best, ms = g.autotune(max_trials=12)
    assert best["autotune"] == 1 and ms > 0
    g.ConstructSVG(autotune=1)
    got = g.csr()
    for x, y in zip(ref, got):
        assert np.array_equal(x, y)


def test_reference_table_overflow_is_flagged():
    """monkey, K=6: the centre reaches 13 vertices, the reference's vertex
    table holds 2K = 12 keys."""
    g = load_golden("monkey")
    _, _, st, s, _ = gpu_build(g["pos"], g["faces"], 6)
    _, _, flags = s.source_stats()
    assert flags[0] & 2
    assert st["ref_overflow_sources"] >= 1


def _oracle_rows(pos, faces, K, src, **kw):
    rows = CpuOracle().mesh(pos, faces).build(K, src, threads=0, **kw)
    return rows_from_padded(rows.tails, rows.nodes), rows


@pytest.mark.parametrize("cfg,K,ranges", [
    (0, 100, [(0, 768), (15000, 15512)]),
    (1, 500, [(0, 300), (36300, 36556)]),
    (1, 100, [(72500, 72900)]),
])
def test_build_matches_oracle_on_benchmark_mesh_samples(cfg, K, ranges):
    pos, faces = meshgen.config_mesh(cfg)
    for a, b in ranges:
        off, nodes, st, _, m = gpu_build(pos, faces, K, source_begin=a, source_end=b)
        src = np.arange(a, b, dtype=np.int32)
        (ooff, onodes), rows = _oracle_rows(pos, faces, K, src)
        sub = off[a:b + 1] - off[a]
        got = nodes[off[a]:off[b]]
        assert compare_rows(sub, got, ooff, onodes) == []
        assert st["windows_generated"] == int(rows.stats[:, 0].sum())
        assert off[b] - off[a] == off[-1]  # rows outside the range are empty


def test_queue_capacity_drops_like_the_reference():
    pos, faces = meshgen.torus(1.0, 0.35, 24, 16, 0.02, seed=3)
    for mode in (MODE_BATCHED, MODE_PLAIN):
        off, nodes, st, _, _ = gpu_build(pos, faces, 30, mode, win_queue_cap=12, pseudo_queue_cap=5)
        (ooff, onodes), rows = _oracle_rows(pos, faces, 30, None, win_cap=12, pseudo_cap=5)
        assert compare_rows(off, nodes, ooff, onodes) == []
        assert st["queue_drop_sources"] > 0


def test_plain_and_batched_builds_are_identical():
    pos, faces = meshgen.height_field(40, seed=7)
    a = gpu_build(pos, faces, 60, MODE_BATCHED)
    b = gpu_build(pos, faces, 60, MODE_PLAIN)
    assert compare_rows(a[0], a[1], b[0], b[1]) == []
    assert a[2]["windows"] == b[2]["windows"]


def test_csr_without_paths_matches():
    pos, faces = meshgen.torus(1.0, 0.35, 30, 20, 0.02, seed=5)
    off, nodes, _, s, _ = gpu_build(pos, faces, 40, with_paths=False)
    coff, adj, dist = s.csr()
    (ooff, onodes), _ = _oracle_rows(pos, faces, 40, None)
    assert np.array_equal(coff, ooff)
    assert np.array_equal(adj, onodes["adj"])
    assert np.array_equal(dist, onodes["dist"])


def test_save_file_is_byte_identical_to_reference_format():
    g = load_golden("monkey")
    K = 20
    _, _, _, s, m = gpu_build(g["pos"], g["faces"], K)
    goff, gnodes = rows_from_padded(g[f"K{K}_tails"], g[f"K{K}_nodes"])
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "m.svg")
        s.SaveSVGToFile(p)
        data = open(p, "rb").read()
        gn = gnodes.copy()
        gn["pad"] = 0
        assert data == svg_file_bytes(goff, gn)
        s2 = SVG()
        s2.AssignMesh(m)
        s2.SetParameters(K)
        s2.LoadSVGFromFile(p)
        off2, n2 = s2.CopySVGToHost()
        assert compare_rows(off2, n2, goff, gnodes) == []


def test_per_source_statistics():
    pos, faces = meshgen.torus(1.0, 0.35, 30, 20, 0.02, seed=5)
    _, _, st, s, _ = gpu_build(pos, faces, 40)
    w, q, f = s.source_stats()
    assert w.sum() == st["windows"]
    assert q.max() == st["max_win_queue"]
    assert (f == 0).all()


def test_bad_arguments_are_reported():
    from svg_b200 import SvgError
    pos, faces = meshgen.torus(1.0, 0.35, 8, 6, 0.02, seed=5)
    with pytest.raises(SvgError):
        gpu_build(pos, faces, 0)
    with pytest.raises(SvgError):
        gpu_build(pos, faces, 10, source_begin=10, source_end=5)


def test_work_order_does_not_change_the_graph():
    """Which lane builds which source, and when, is a scheduling choice: vertex
    order, heaviest-first from the previous build, and the K/10 probe order give
    the same CSR bit for bit."""
    import svg_b200
    from svg_b200 import SVG, Mesh
    pos, faces = meshgen.config_mesh(1, 0.3)
    outs = []
    for hf, warm in ((0, False), (1, True), (2, False)):
        m = Mesh.from_arrays(pos, faces)
        g = SVG()
        g.AssignMesh(m)
        g.SetParameters(200)
        if warm:
            g.ConstructSVG(heavy_first=0)   # leaves per-source costs on the mesh
        g.ConstructSVG(heavy_first=hf)
        outs.append(g.csr())
    for o in outs[1:]:
        for x, y in zip(outs[0], o):
            assert np.array_equal(x, y)
    mem = svg_b200.device_memory()
    assert mem["in_use"] > 0 and mem["peak"] >= mem["in_use"]
