"""The boundary from compiled callers: include/svg_b200.h from C, and the
header-only C++ wrapper include/svg_b200.hpp (the reference's Mesh / SVG class
and method names, SVG.cuh:52-80, Mesh.cuh:38-39) from a driver written in the
style of the reference's kernel.cu mains (tests/cpp/svg_driver.cpp).

CPU: both compile with warnings as errors and link against the library; the
C program takes the address of every entry point the header declares.
GPU: the driver builds a mesh, saves the .svg file and answers SSSD and MSAD
queries through the wrapper; its file must be byte-identical to the Python
path's, its distances equal to svg_sssd_batch / svg_msad_batch, its paths
and parent pointers valid shortest-path trees of the graph.
"""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import svg_b200
from svg_b200 import SVG, Mesh, meshgen
from svg_b200.build_ext import build as build_lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "svg_b200")
CPP = os.path.join(ROOT, "tests", "cpp")


@pytest.fixture(scope="module", autouse=True)
def _lib_built():
    build_lib()


def _compile(src, out, cxx=True):
    cmd = (["g++", "-std=c++17"] if cxx else ["gcc", "-std=c99"]) + [
        "-O1", "-Wall", "-Wextra", "-Werror", "-I" + INC, src, "-L" + LIBDIR, "-lsvg_b200",
        "-Wl,-rpath," + LIBDIR, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


def test_c_header_compiles_and_every_entry_point_links():
    with tempfile.TemporaryDirectory() as td:
        exe = _compile(os.path.join(CPP, "c_abi_check.c"), os.path.join(td, "c_abi_check"), cxx=False)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    decl = set(re.findall(r"\b(svg_[a-z0-9_]+)\s*\(", open(os.path.join(INC, "svg_b200.h")).read()))
    listed = set(re.findall(r"\(void\*\)(svg_[a-z0-9_]+)", open(os.path.join(CPP, "c_abi_check.c")).read()))
    assert listed == decl
    assert f"{len(decl)} entry points" in out


def test_cpp_wrapper_compiles_with_reference_names():
    with tempfile.TemporaryDirectory() as td:
        _compile(os.path.join(CPP, "svg_driver.cpp"), os.path.join(td, "svg_driver"))


def _parse(out, V):
    sssd, msad = [], []
    lines = out.splitlines()
    i = 0
    while i < len(lines):
        p = lines[i].split()
        if p and p[0] == "sssd":
            s, t, d = int(p[1]), int(p[2]), float(p[3])
            path = [int(x) for x in p[5:]]
            sssd.append((s, t, d, path))
        elif p and p[0] == "msad":
            rows = np.array([[float(x) for x in r.split()] for r in lines[i + 1:i + 1 + V]])
            msad.append((rows[:, 1], rows[:, 2].astype(np.int64), rows[:, 3].astype(np.int64)))
            i += V
        i += 1
    return sssd, msad


@pytest.mark.gpu
def test_cpp_driver_matches_python_path():
    pos, faces = meshgen.torus(1.0, 0.35, 40, 30, 0.02, seed=5)
    V = len(pos)
    K = 60
    rng = np.random.default_rng(9)
    pairs = rng.integers(0, V, (12, 2))
    sets = [rng.choice(V, k, replace=False) for k in (1, 7)]
    wts = [rng.uniform(0, 0.05, len(x)) for x in sets]
    with tempfile.TemporaryDirectory() as td:
        exe = _compile(os.path.join(CPP, "svg_driver.cpp"), os.path.join(td, "svg_driver"))
        obj = os.path.join(td, "torus.obj")
        meshgen.write_obj(obj, pos, faces)
        qf = os.path.join(td, "q.txt")
        with open(qf, "w") as f:
            for s, t in pairs:
                f.write(f"{s} {t}\n")
            f.write(f"{pairs[0][0]} {pairs[0][0]}\n")  # s == t
            for st, w in zip(sets, wts):
                f.write("m %d %s\n" % (len(st), " ".join(f"{int(a)} {float(b)!r}" for a, b in zip(st, w))))
        r = subprocess.run([exe, obj, str(K), qf], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        cpp_file = open(os.path.join(td, "torus.svg"), "rb").read()

        m = Mesh.LoadFromFile(obj)
        g = SVG()
        g.AssignMesh(m)
        g.SetParameters(K, 10, 2)
        g.ConstructSVG()
        py_svg = os.path.join(td, "py.svg")
        g.SaveSVGToFile(py_svg)
        assert cpp_file == open(py_svg, "rb").read()

    off, adj, w = g.csr()
    edge_w = {}
    for u in range(V):
        for e in range(off[u], off[u + 1]):
            edge_w[(u, int(adj[e]))] = float(w[e])
    sssd, msad = _parse(r.stdout, V)
    assert len(sssd) == len(pairs) + 1 and len(msad) == len(sets)
    d_py = g.sssd_batch(pairs[:, 0], pairs[:, 1])
    for (s, t, d, path), dp in zip(sssd, list(d_py) + [0.0]):
        assert d == dp
        assert path[0] == t and path[-1] == s
        # the path runs along graph edges and sums to the distance
        total = 0.0
        for a, b in zip(path[::-1][:-1], path[::-1][1:]):
            total += edge_w[(a, b)]
        assert abs(total - d) <= 1e-12 * max(d, 1e-300)
    dm, sm = g.msad_batch(sets, wts)
    for q, (d, src, par) in enumerate(msad):
        assert np.array_equal(d, dm[q])
        assert np.array_equal(src, sm[q])
        for v in range(V):
            if par[v] >= 0:
                assert d[par[v]] + edge_w[(int(par[v]), v)] == d[v]
            else:
                assert src[v] == v or d[v] == np.finfo(np.float64).max
    # the Python binding of the same entry points agrees
    d2, s2, p2 = g.msad_paths(sets, wts)
    assert np.array_equal(d2, dm) and np.array_equal(p2[1], msad[1][2])
    path, pd, dist = g.sssd_path(int(pairs[0][0]), int(pairs[0][1]))
    assert dist == d_py[0] and path[0] == pairs[0][1] and pd[0] == dist
