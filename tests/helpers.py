"""Shared helpers for the parity tests: golden fixtures, row comparison."""
from __future__ import annotations

import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_cases():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def golden_params():
    out = []
    for name in golden_cases():
        g = load_golden(name)
        for K in g["Ks"]:
            out.append((name, int(K)))
    return out


def rows_from_padded(tails: np.ndarray, nodes: np.ndarray):
    """Padded reference rows -> (offsets, packed nodes)."""
    off = np.zeros(len(tails) + 1, np.int64)
    np.cumsum(tails, out=off[1:])
    packed = np.concatenate([nodes[r, : tails[r]] for r in range(len(tails))]) if len(tails) else nodes[:0, 0]
    return off, packed


def compare_rows(off_a, nodes_a, off_b, nodes_b, fields=("adj", "dist", "src_edge", "dst_edge", "src_x", "dst_x"),
                 rows=None):
    """Bit-exact row comparison.  Returns a list of (row, field) mismatches."""
    bad = []
    R = range(len(off_a) - 1) if rows is None else rows
    for r in R:
        a = nodes_a[off_a[r]:off_a[r + 1]]
        b = nodes_b[off_b[r]:off_b[r + 1]]
        if len(a) != len(b):
            bad.append((r, "degree", len(a), len(b)))
            continue
        for f in fields:
            if not np.array_equal(a[f], b[f]):
                bad.append((r, f))
                break
    return bad


def svg_file_bytes(off: np.ndarray, nodes: np.ndarray) -> bytes:
    """The reference's .svg bytes (SVG.cu:208-217): per vertex int32 degree, then nodes."""
    parts = []
    for r in range(len(off) - 1):
        parts.append(np.int32(off[r + 1] - off[r]).tobytes())
        parts.append(nodes[off[r]:off[r + 1]].tobytes())
    return b"".join(parts)


def csr_from_padded(tails: np.ndarray, nodes: np.ndarray):
    """Padded reference rows -> (offsets, packed nodes), vectorised for full meshes."""
    tails = np.asarray(tails)
    off = np.zeros(len(tails) + 1, np.int64)
    np.cumsum(tails, out=off[1:])
    mask = np.arange(nodes.shape[1])[None, :] < tails[:, None]
    return off, nodes[mask]


def first_row_mismatches(off_a, nodes_a, off_b, nodes_b,
                         fields=("adj", "dist", "src_edge", "dst_edge", "src_x", "dst_x"), limit=10):
    """Bit-exact comparison of two CSR row sets over every row at once.
    Returns [] when identical, else up to `limit` (row, reason) entries."""
    if len(off_a) != len(off_b):
        return [(-1, f"row count {len(off_a) - 1} vs {len(off_b) - 1}")]
    deg_a, deg_b = np.diff(off_a), np.diff(off_b)
    bad_deg = np.nonzero(deg_a != deg_b)[0]
    if len(bad_deg):
        return [(int(r), f"degree {deg_a[r]} vs {deg_b[r]}") for r in bad_deg[:limit]]
    out = []
    row_of = np.repeat(np.arange(len(deg_a)), deg_a)
    for f in fields:
        x, y = nodes_a[f], nodes_b[f]
        eq = x == y
        if x.dtype.kind == "f":
            eq |= np.isnan(x) & np.isnan(y)
        diff = np.nonzero(~eq)[0]
        if len(diff):
            rows = np.unique(row_of[diff])[:limit]
            out += [(int(r), f) for r in rows]
    return out[:limit]
