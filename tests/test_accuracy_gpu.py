"""SVG distances against the reference's ICH run without the K limit, on a
reduced closed torus: the worst overestimate falls as K grows.  (That oracle
itself overestimates some distances, see tests/accuracy_report.py, so a
shorter SVG distance is not asserted against.)"""
import os

import numpy as np
import pytest

from svg_b200.build_ext import build as build_lib
from tests.accuracy_report import run

pytestmark = pytest.mark.gpu


def test_svg_error_against_exact_ich():
    build_lib()
    out = run([20, 80], n_sources=4, scale=0.25, threads=os.cpu_count() or 1, config=0)
    rows = {r["K"]: r for r in out["per_K"]}
    for r in rows.values():
        assert r["vertices_compared"] > 0.99 * out["vertices"] * len(out["sources"]) - r["exact_unreached"]
        # a vertex outside every other vertex's kept K neighbours has no
        # in-edge in the SVG (the reference's graph has the same property)
        assert r["svg_unreached_exact_reached"] < 0.01 * r["vertices_compared"]
    # the worst overestimate against the oracle falls as K grows
    assert rows[80]["max_rel"] < rows[20]["max_rel"]
    assert rows[80]["max_rel"] < 0.05
    assert rows[80]["vs_best_known"]["mean_rel"] < 1e-3
