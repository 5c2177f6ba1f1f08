"""Host-side checks that need no GPU: the C-ABI library loads and exports
every declared entry point, and its mesh loader reproduces the reference's
half-edge structure (Mesh::LoadFromFile) exactly."""
import os
import re
import tempfile

import numpy as np
import pytest

import svg_b200
from oracle.refbind import CpuOracle
from svg_b200 import Mesh, SvgError, meshgen
from svg_b200.build_ext import build as build_lib
from tests.helpers import golden_cases, load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _lib_built():
    build_lib()


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "svg_b200.h")).read()
    return sorted(set(re.findall(r"\b(svg_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = svg_b200.lib()
    decl = declared_symbols()
    assert len(decl) >= 20
    missing = [s for s in decl if not hasattr(L, s)]
    assert missing == []
    assert sorted(decl) == sorted(svg_b200.EXPORTS)


def test_version_and_error_string():
    L = svg_b200.lib()
    assert b"sm_100a" in L.svg_version()
    assert L.svg_last_error() is not None


@pytest.mark.parametrize("name", golden_cases())
def test_mesh_loader_matches_reference_on_golden_meshes(name):
    g = load_golden(name)
    m = Mesh.from_arrays(g["pos"], g["faces"])
    ex = m.export()
    assert np.array_equal(ex["he_twin"], g["he_twin"])
    assert np.array_equal(ex["he_len"], g["he_len"])
    assert np.array_equal(ex["angle"], g["angle"])
    assert np.array_equal(ex["first_edge"], g["first_edge"])
    assert np.array_equal(ex["pos"], g["pos"])


@pytest.mark.parametrize("cfg,scale", [(0, 1.0), (1, 1.0), (2, 0.05)])
def test_mesh_loader_matches_oracle_on_benchmark_meshes(cfg, scale):
    pos, faces = meshgen.config_mesh(cfg, scale=scale)
    a = Mesh.from_arrays(pos, faces).export()
    b = CpuOracle().mesh(pos, faces).export()
    for k in ["he_v0", "he_twin", "he_len", "angle", "first_edge"]:
        assert np.array_equal(a[k], b[k]), k


def test_obj_round_trip_is_exact():
    pos, faces = meshgen.height_field(12, seed=4)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "m.obj")
        meshgen.write_obj(p, pos, faces)
        a = Mesh.LoadFromFile(p).export()
    b = Mesh.from_arrays(pos, faces).export()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_obj_accepts_reference_subset_and_slash_indices():
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "m.obj")
        with open(p, "w") as f:
            f.write("# comment\nvn 0 0 1\nvt 0 0\nv 0 0 0\nv\t1 0 0\nv 0 1 0\nv 1 1 0.5\n"
                    "f 1/1/1 2/2/2 3/3/3\nf 2 4 3\n")
        m = Mesh.LoadFromFile(p)
        assert (m.vertNum, m.faceNum) == (4, 2)


def test_obj_errors_are_reported_not_fatal():
    with pytest.raises(SvgError) as e:
        Mesh.LoadFromFile("/nonexistent/mesh.obj")
    assert e.value.code == 2
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "bad.obj")
        with open(p, "w") as f:
            f.write("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n")
        with pytest.raises(SvgError) as e:
            Mesh.LoadFromFile(p)
        assert e.value.code == 5
        p2 = os.path.join(td, "empty.obj")
        open(p2, "w").close()
        with pytest.raises(SvgError) as e:
            Mesh.LoadFromFile(p2)
        assert e.value.code == 5


def test_boundary_half_edges_get_twin_minus_one():
    pos, faces = meshgen.height_field(6, seed=2)
    ex = Mesh.from_arrays(pos, faces).export()
    n = 6
    assert (ex["he_twin"] == -1).sum() == 4 * (n - 1)
    twin = ex["he_twin"]
    inner = twin >= 0
    assert np.all(twin[twin[inner]] == np.nonzero(inner)[0])


def test_isolated_vertex_has_no_first_edge():
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [5, 5, 5]], np.float64)
    faces = np.array([[0, 1, 2]], np.int32)
    ex = Mesh.from_arrays(pos, faces).export()
    assert ex["first_edge"][3] == -1


def test_non_manifold_twins_follow_reference_pairing():
    """Three or more half-edges on one vertex pair (a fin of three triangles, and a
    face repeated with the same orientation): each later half-edge pairs with the
    first of its pair and the first keeps the last, as the reference's map does."""
    from oracle.refbind import RefOracle, ref_available
    if not ref_available():
        pytest.skip("reference oracle not built")
    pos = np.array([[0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, -1, 0], [0.5, 0, 1], [2, 2, 0]], np.float64)
    faces = np.array([[0, 1, 2], [1, 0, 3], [0, 1, 4], [1, 2, 5], [1, 2, 5], [2, 0, 4]], np.int32)
    a = Mesh.from_arrays(pos, faces).export()
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "fin.obj")
        meshgen.write_obj(p, pos, faces)
        b = RefOracle().load(p, fix_boundary=True).export()
    for k in ["he_v0", "he_twin", "he_len", "angle", "first_edge"]:
        assert np.array_equal(a[k], b[k]), k
    assert (a["he_twin"] >= 0).sum() >= 8


@pytest.mark.parametrize("seed", range(12))
def test_random_meshes_match_reference_loader(seed):
    """Random triangles over few vertices (shared, repeated and non-manifold
    edges, both orientations): half-edge twins, lengths, vertex angles and first
    edges equal the reference's loader."""
    from oracle.refbind import RefOracle, ref_available
    if not ref_available():
        pytest.skip("reference oracle not built")
    rng = np.random.default_rng(seed)
    nv = int(rng.integers(5, 25))
    nf = int(rng.integers(4, 60))
    pos = rng.normal(size=(nv, 3))
    faces = np.array([rng.choice(nv, 3, replace=False) for _ in range(nf)], np.int32)
    a = Mesh.from_arrays(pos, faces).export()
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "r.obj")
        meshgen.write_obj(p, pos, faces)
        b = RefOracle().load(p, fix_boundary=True).export()
    for k in ["he_v0", "he_twin", "he_len", "angle", "first_edge"]:
        assert np.array_equal(a[k], b[k]), k
