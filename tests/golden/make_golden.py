"""Generate the golden fixtures in tests/golden/*.npz from the reference itself.

The reference ships no tests, golden vectors or sample meshes.  Its results
are pinned by running its own ICH (oracle/_ref/libsvgref.so: Mesh.cu,
Geometry.cu, ICHDevice.cu compiled as host C++) on small meshes that reach
the edge cases, and storing the SVG rows it emits:

  tetrahedron   closed, 4 faces: window levels exceed faceNum and are culled
  octahedron    closed, all vertices convex (no pseudo-sources)
  cube          closed, 12 faces, degree-3 and degree-6 vertices
  monkey        open saddle fan (angle sum > 2*pi at the centre) + boundary
  torus_small   closed noisy torus, 16x10 grid (config-0 generator, shrunk)
  hfield_small  open height field, 9x9 grid (config-1 generator, shrunk)
  tiny_grid     open 3x3 grid, K larger than the vertex count

Each file holds the mesh (pos, faces), K, per-source rows in the reference
node layout (tails, nodes) and the reference's ICH counters (stats).

Run:  python tests/golden/make_golden.py     (needs the reference sources)
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.refbind import RefOracle, build_oracles  # noqa: E402
from svg_b200 import meshgen  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def tetrahedron():
    pos = np.array([[0.0, 0.0, 0.0], [1.0, 0.05, 0.0], [0.45, 0.9, 0.02], [0.5, 0.3, 0.85]])
    faces = np.array([[0, 2, 1], [0, 1, 3], [1, 2, 3], [2, 0, 3]], np.int32)
    return pos, faces


def octahedron():
    pos = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float64)
    pos = pos * np.array([1.0, 0.93, 1.07])
    faces = np.array([[0, 2, 4], [2, 1, 4], [1, 3, 4], [3, 0, 4],
                      [2, 0, 5], [1, 2, 5], [3, 1, 5], [0, 3, 5]], np.int32)
    return pos, faces


def cube():
    pos = np.array([[x, y, z] for z in (0.0, 1.0) for y in (0.0, 1.0) for x in (0.0, 1.0)])
    pos += np.random.default_rng(4).uniform(-0.03, 0.03, pos.shape)
    q = [[0, 2, 3, 1], [4, 5, 7, 6], [0, 1, 5, 4], [2, 6, 7, 3], [0, 4, 6, 2], [1, 3, 7, 5]]
    faces = []
    for a, b, c, d in q:
        faces += [[a, b, c], [a, c, d]]
    return pos, np.array(faces, np.int32)


def monkey():
    # centre vertex with a 12-vertex ring whose heights alternate in three
    # lobes (a monkey saddle), then an outer ring: angle sum at the centre > 2*pi
    n = 12
    pos = [[0.0, 0.0, 0.0]]
    for r, amp in ((1.0, 0.55), (2.0, 1.4)):
        for k in range(n):
            a = 2 * np.pi * k / n
            pos.append([r * np.cos(a), r * np.sin(a), amp * np.cos(3 * a)])
    faces = []
    for k in range(n):
        a, b = 1 + k, 1 + (k + 1) % n
        faces.append([0, a, b])
        c, d = 1 + n + k, 1 + n + (k + 1) % n
        faces += [[a, c, d], [a, d, b]]
    return np.array(pos), np.array(faces, np.int32)


def tiny_grid():
    return meshgen.height_field(3, bumps=2, seed=5)


CASES = {
    "tetrahedron": (tetrahedron, [2, 3]),
    "octahedron": (octahedron, [3, 5]),
    "cube": (cube, [4, 7]),
    "monkey": (monkey, [6, 20]),
    "torus_small": (lambda: meshgen.torus(1.0, 0.35, 16, 10, 0.02, seed=0), [8, 30]),
    "hfield_small": (lambda: meshgen.height_field(9, seed=1), [10, 40]),
    "tiny_grid": (tiny_grid, [20]),
}


def main() -> None:
    build_oracles(ref=True)
    ref = RefOracle()
    with tempfile.TemporaryDirectory() as td:
        for name, (fn, Ks) in CASES.items():
            pos, faces = fn()
            obj = os.path.join(td, name + ".obj")
            meshgen.write_obj(obj, pos, faces)
            m = ref.load(obj, fix_boundary=True)
            ex = m.export()
            assert np.array_equal(ex["pos"], pos), name  # %.17g round trip is exact
            data = dict(pos=pos, faces=faces, he_twin=ex["he_twin"], he_len=ex["he_len"], angle=ex["angle"],
                        first_edge=ex["first_edge"])
            for K in Ks:
                rows = m.build(K, threads=1)
                data[f"K{K}_tails"] = rows.tails
                data[f"K{K}_nodes"] = rows.nodes
                data[f"K{K}_stats"] = rows.stats
            data["Ks"] = np.array(Ks, np.int32)
            np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
            print(name, m.nv, m.nf, {K: int(data[f"K{K}_tails"].sum()) for K in Ks})


if __name__ == "__main__":
    main()
