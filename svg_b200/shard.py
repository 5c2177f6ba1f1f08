"""Sharded SVG construction over several ranks (one process per GPU).

Sources are independent (each row of the SVG depends on the mesh and its own
source only; the reference's grid-stride loop over sources, SVG.cu:34, has no
exchange), so a build shards by contiguous source ranges with the mesh
replicated on every rank.  The only collective is one all-gather of the CSR
slices after the build, so that every rank holds the whole graph for queries:
  1. all-gather the slice sizes (row count and edge count per rank);
  2. all-gather the degree, adjacency and length arrays, each padded to the
     largest slice;
  3. concatenate in rank order and rebuild the offsets by a prefix sum of the
     degrees (the rebasing: a slice's local offsets never cross the wire).
With NCCL the tensors are device tensors and the gather runs over NVLink; the
same code runs with gloo on CPU tensors (the multi-rank tests).
"""
from __future__ import annotations

import numpy as np

__all__ = ["shard_ranges", "gather_csr", "assemble_csr", "slice_of_csr"]


def shard_ranges(nv: int, world: int, cost: np.ndarray | None = None) -> list[tuple[int, int]]:
    """Contiguous source ranges, one per rank, covering [0, nv).  With
    per-source costs (e.g. the windows of a previous build), the cut points
    balance the summed cost; otherwise the counts."""
    if world <= 0:
        raise ValueError("world must be positive")
    if cost is None or len(cost) != nv or np.sum(cost) <= 0:
        cuts = [nv * r // world for r in range(world + 1)]
    else:
        c = np.concatenate([[0.0], np.cumsum(np.asarray(cost, np.float64))])
        targets = c[-1] * np.arange(world + 1) / world
        cuts = np.searchsorted(c, targets, side="left").tolist()
        cuts[0], cuts[-1] = 0, nv
        for r in range(1, world + 1):  # monotone, inside [0, nv]
            cuts[r] = int(min(max(cuts[r], cuts[r - 1]), nv))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world)]


def slice_of_csr(off: np.ndarray, adj: np.ndarray, dist: np.ndarray, begin: int, end: int):
    """The rows [begin, end) of a CSR as (degrees, adjacency, lengths)."""
    a, b = int(off[begin]), int(off[end])
    return np.diff(off[begin:end + 1]).astype(np.int32), adj[a:b], dist[a:b]


def assemble_csr(degs: list, adjs: list, dists: list):
    """Slices in rank order -> (offsets int64, adjacency int32, lengths f64)."""
    deg = np.concatenate([np.asarray(d, np.int32) for d in degs]) if degs else np.zeros(0, np.int32)
    off = np.zeros(len(deg) + 1, np.int64)
    np.cumsum(deg, out=off[1:])
    adj = np.concatenate([np.asarray(a, np.int32) for a in adjs]) if adjs else np.zeros(0, np.int32)
    dist = np.concatenate([np.asarray(d, np.float64) for d in dists]) if dists else np.zeros(0)
    return off, adj, dist


def gather_csr(dist_mod, deg, adj, w, device: str = "cpu"):
    """All-gather this rank's CSR slice (torch tensors or numpy arrays:
    int32 degrees of its rows, int32 adjacency, float64 lengths) and return
    every rank's slices as torch tensors on `device`, in rank order:
    (degs, adjs, dists).  Collective: every rank calls it once."""
    import torch

    def t(x, dt):
        if isinstance(x, torch.Tensor):
            return x.to(device=device, dtype=dt).contiguous()
        return torch.as_tensor(np.ascontiguousarray(x), dtype=dt, device=device)

    deg, adj, w = t(deg, torch.int32), t(adj, torch.int32), t(w, torch.float64)
    world = dist_mod.get_world_size()
    sizes = torch.tensor([deg.numel(), adj.numel()], dtype=torch.int64, device=device)
    all_sizes = [torch.zeros_like(sizes) for _ in range(world)]
    dist_mod.all_gather(all_sizes, sizes)
    rows = [int(s[0]) for s in all_sizes]
    edges = [int(s[1]) for s in all_sizes]
    mr, me = max(max(rows), 1), max(max(edges), 1)

    def gather(x, n_max, fill, dt):
        buf = torch.full((n_max,), fill, dtype=dt, device=device)
        buf[:x.numel()] = x
        outs = [torch.empty(n_max, dtype=dt, device=device) for _ in range(world)]
        dist_mod.all_gather(outs, buf)
        return outs

    g_deg = gather(deg, mr, 0, torch.int32)
    g_adj = gather(adj, me, -1, torch.int32)
    g_w = gather(w, me, 0.0, torch.float64)
    return ([g_deg[r][:rows[r]] for r in range(world)], [g_adj[r][:edges[r]] for r in range(world)],
            [g_w[r][:edges[r]] for r in range(world)])
