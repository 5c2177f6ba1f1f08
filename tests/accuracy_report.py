"""SVG approximation error against the exact ICH (full-mesh, FP64, host).

For the 270x270 height field (72,900 vertices, seed 1), 32 seeded random
sources: the exact ICH distances from each source (the reference's ICH with no
K limit, run on the host cores) against the SVG graph distances from the same
source (a one-source MSAD on the GPU SVG built at each K).  Prints one JSON
line with, per K, the relative error (d_svg - d_exact) / d_exact over every
vertex both reach: max, mean, p99, and the fraction above 1e-3.

The exact-ICH oracle is the reference's own ICH run without the K limit, and
it is not exact everywhere: on the 1,900-vertex torus, for example, it reaches
1,889 vertices and the SVG at K = V gives shorter distances than it for about a
quarter of the vertices (by up to 11 %), which a surface path could not do
against true geodesics.  On open meshes it also treats only vertices with angle
>= 2 pi as pseudo-sources, so it misses geodesics that bend around boundary
vertices.  A negative min_rel therefore measures the oracle's shortfall, and
each K also gets the error against the best known distance, the smaller of the
exact ICH and the SVG at the largest K.

Usage (needs a GPU and the oracle built):
    python tests/accuracy_report.py [--K 50,100,200,500] [--sources 32] [--scale 1.0]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle.refbind import CpuOracle, RefOracle, ref_available  # noqa: E402
from svg_b200 import SVG, Mesh, meshgen  # noqa: E402

UNREACHED = 1e300


def exact_ich(pos, faces, sources, threads):
    """Exact ICH distances (K = -1) from each source: the reference's own ICH
    when it is built here, else the C restatement."""
    if ref_available():
        td = tempfile.mkdtemp()
        obj = os.path.join(td, "m.obj")
        meshgen.write_obj(obj, pos, faces)
        mesh = RefOracle().load(obj, fix_boundary=True)
        kind = "reference"
    else:
        mesh = CpuOracle().mesh(pos, faces)
        kind = "port"
    t = time.time()
    d, _, _ = mesh.ich_distances(sources, K=-1, win_cap=1 << 24, pseudo_cap=1 << 22, threads=threads)
    return d, kind, time.time() - t


def svg_distances(svg: SVG, sources):
    d, _ = svg.msad_batch([np.array([s], np.int32) for s in sources], with_src=True)
    return d


def error_stats(d_svg, d_exact):
    both = (d_exact < UNREACHED) & (d_svg < UNREACHED) & (d_exact > 0)
    rel = (d_svg[both] - d_exact[both]) / d_exact[both]
    return {"vertices_compared": int(both.sum()),
            "exact_unreached": int((d_exact >= UNREACHED).sum()),
            "svg_unreached_exact_reached": int(((d_svg >= UNREACHED) & (d_exact < UNREACHED)).sum()),
            "max_rel": float(rel.max()), "mean_rel": float(rel.mean()), "p99_rel": float(np.percentile(rel, 99)),
            "frac_above_1e-3": float((rel > 1e-3).mean()), "min_rel": float(rel.min())}


def run(Ks, n_sources, scale, threads, seed=1, config=1):
    pos, faces = meshgen.config_mesh(config, scale)
    V = len(pos)
    rng = np.random.default_rng(seed)
    sources = rng.choice(V, n_sources, replace=False).astype(np.int32)
    d_exact, kind, secs = exact_ich(pos, faces, sources, threads)
    mesh = Mesh.from_arrays(pos, faces)
    out = {"mesh": {0: "torus", 1: "height_field", 2: "torus_value_noise"}[config], "vertices": V, "sources": sources.tolist(), "oracle": kind,
           "exact_ich_seconds": secs, "threads": threads, "per_K": []}
    d_all = {}
    for K in Ks:
        svg = SVG()
        svg.AssignMesh(mesh)
        svg.SetParameters(K)
        st = svg.ConstructSVG(with_paths=False)
        d_all[K] = svg_distances(svg, sources).reshape(-1)
        row = {"K": K, "edges": st["edges"]}
        row.update(error_stats(d_all[K], d_exact.reshape(-1)))
        out["per_K"].append(row)
        svg.FreeSVGStructure()
    # the exact-ICH oracle itself overestimates some distances (SVG paths at
    # large K come out shorter), so the error is also given against the best
    # known distance: the smaller of the exact ICH and the SVG at the largest K
    best = np.minimum(d_exact.reshape(-1), d_all[max(Ks)])
    for row in out["per_K"]:
        e = error_stats(d_all[row["K"]], best)
        row["vs_best_known"] = {k: e[k] for k in ("max_rel", "mean_rel", "p99_rel", "frac_above_1e-3")}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--K", default="50,100,200,500")
    ap.add_argument("--sources", type=int, default=32)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--config", type=int, default=1, help="0: torus, 1: height field, 2: 750K torus")
    a = ap.parse_args()
    print(json.dumps(run([int(k) for k in a.K.split(",")], a.sources, a.scale, a.threads, config=a.config)),
          flush=True)


if __name__ == "__main__":
    main()
