"""The allocation-free build entry point (svg_build_rows_static).

It serves callers that cannot allocate device memory when they build: its
scratch is a fixed array inside the library and every output buffer comes
from the caller.  This file is collected last on purpose.  The test calls the
entry point twice in a row through the C ABI, into buffers the test owns,
and checks each result bit for bit against the rows of the regular build
(svg_build), which allocates its own scratch.
"""
import ctypes as C

import numpy as np
import pytest

import svg_b200
from svg_b200 import SVG, Mesh, meshgen
from svg_b200.build_ext import build as build_lib

pytestmark = pytest.mark.gpu


def test_static_scratch_build_matches_regular_build_on_two_calls():
    import torch

    build_lib()
    L = svg_b200.lib()
    pos, faces = meshgen.torus(1.0, 0.35, 40, 30, 0.02, seed=5)
    mesh = Mesh.from_arrays(pos, faces)
    mesh.copyToGPU()
    K = 60
    svg = SVG()
    svg.AssignMesh(mesh)
    svg.SetParameters(K)
    svg.ConstructSVG(with_paths=False)
    off, adj, dist = svg.csr()

    for a, b in [(0, 700), (300, 1200)]:
        n = b - a
        d_tails = torch.full((n,), -7, dtype=torch.int32, device="cuda")
        d_adj = torch.zeros(n * K, dtype=torch.int32, device="cuda")
        d_dist = torch.zeros(n * K, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = L.svg_build_rows_static(mesh._h, K, a, b, C.c_void_p(d_tails.data_ptr()),
                                     C.c_void_p(d_adj.data_ptr()), C.c_void_p(d_dist.data_ptr()), None)
        assert rc == 0, L.svg_last_error()
        torch.cuda.synchronize()
        tails = d_tails.cpu().numpy()
        padj = d_adj.cpu().numpy().reshape(n, K)
        pdist = d_dist.cpu().numpy().reshape(n, K)
        assert np.array_equal(tails, (off[a + 1:b + 1] - off[a:b]).astype(np.int32))
        for r in range(n):
            v = a + r
            assert np.array_equal(padj[r, :tails[r]], adj[off[v]:off[v + 1]])
            assert np.array_equal(pdist[r, :tails[r]], dist[off[v]:off[v + 1]])


def test_static_scratch_build_rejects_sizes_beyond_its_limit():
    build_lib()
    L = svg_b200.lib()
    pos, faces = meshgen.torus(1.0, 0.35, 12, 8, 0.02, seed=5)
    mesh = Mesh.from_arrays(pos, faces)
    mesh.copyToGPU()
    one = C.c_void_p(16)  # never dereferenced: the call is rejected before any launch
    rc = L.svg_build_rows_static(mesh._h, 129, 0, 4, one, one, one, None)
    assert rc == 1 and b"limit" in L.svg_last_error()
