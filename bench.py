"""Benchmark: SVG construction throughput on one B200 (and N replicas).

Workload (one "step" = one full SVG build): the open height-field mesh, a
270x270 grid (72,900 vertices, 144,722 triangles, 64 seeded Gaussian bumps,
seed 1), K = 500, built by the batched persistent kernel.  Synthetic data of
the benchmark's shape; the reference's Stanford Bunny is not available.

metric  svg_build_edges_per_s: SVG edges emitted per second of build, all ranks.
value   device time of the build (CUDA events on the library stream) with the
        mesh already resident in HBM; a 256 MiB buffer is written between
        steps to flush L2 (126 MB).
e2e     the same metric through the C ABI from host arrays: half-edge mesh
        build, upload of the device mesh from pinned memory, the build, and the
        CSR read back to host memory, every step.
plain   the reference's form (one source per thread, 64x128 grid, full table
        reset per source, O(V) emission scan) on the same GPU, one step.
cpu_baseline / --impl reference
        the reference's own construction (its ICH compiled as host C++,
        oracle/_ref) over a seeded sample of sources on all host cores.

Multi-GPU (--gpus N under torchrun): every rank builds its own replica of the
workload (sources are independent; no data-path collective), scaling "weak";
times are the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(workload="svg_build_height_field_270x270_K500", mesh="height_field", grid=270, vertices=72900,
                K=500, seed=1, mode="batched")
K_BUILD = 500
METRIC = "svg_build_edges_per_s"
UNIT = "edges/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws):
    if ws <= 1:
        return None
    import torch.distributed as dist
    import datetime
    backend = "nccl"
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def _reduce(dist, x: float, op: str, device: str) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(dist, x: float, device: str = "cuda") -> float:
    """Device time of a multi-rank step: the slowest rank's."""
    return _reduce(dist, x, "max", device)


def sum_over_ranks(dist, x: float, device: str = "cuda") -> float:
    """Work of a multi-rank step: every rank's replica counts."""
    return _reduce(dist, x, "sum", device)


def replica_value(dist, edges_this_rank: float, ms_this_rank: float, device: str = "cuda") -> float:
    """Whole-job throughput of N replicas: all ranks' edges over the max time."""
    ms = max_over_ranks(dist, ms_this_rank, device)
    return sum_over_ranks(dist, edges_this_rank, device) / (ms / 1e3)


def barrier(dist):
    if dist is not None:
        dist.barrier()


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        busy = [s for s in sm if s > 0.5 * (max(mx) if mx else 0)] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def workload_mesh():
    from svg_b200 import meshgen
    return meshgen.height_field(WORKLOAD["grid"], seed=WORKLOAD["seed"])


def roofline_figures(st: dict, peaks: dict) -> dict:
    """Roofline of the window-propagation kernel (k_ich_batched).

    Algorithmic bytes per propagated window: 3 half-edge records of the
    unfolded face (3 x 32 B), the apex and two opposite-vertex records
    (3 x 16 B), four vertex-state probes (4 x 32 B), one split-state probe
    (32 B), the window popped (16 B key + 48 B payload) and up to two pushed
    (2 x 64 B): ~450 B; plus 24 B per exported candidate.  HBM-bound by
    construction (no dense contraction); FP64 work ~300 flops per window.
    """
    kernel_s = st["ms_ich"] / 1e3
    bytes_alg = st["windows"] * 450.0 + st["edges"] * 24.0
    achieved = bytes_alg / kernel_s / 1e9 if kernel_s > 0 else 0.0
    peak = peaks.get("hbm_gbs")
    src = "measured"
    if not peak:
        peak, src = 6650.0, "fallback"
    traffic = None
    tp = os.path.join(ROOT, "profiles", "ich_batched_traffic.json")
    if os.path.exists(tp):
        try:
            t = json.load(open(tp))
            # scale the captured per-window traffic to this launch's windows
            traffic = t["dram_bytes_per_window"] * st["windows"]
        except Exception:
            traffic = None
    fp64 = st["windows"] * 300.0 / kernel_s / 1e12 if kernel_s > 0 else 0.0
    return {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 5), "traffic": traffic, "peak_source": src,
            "kernel": "k_ich_batched", "algorithmic_bytes_per_launch": bytes_alg,
            "kernel_ms": st["ms_ich"], "fp64_tflops_est": round(fp64, 4)}


def cpu_reference_run(pos, faces, K, budget_s: float, threads: int, seed: int = 0):
    """The reference's construction (oracle/_ref, else the C restatement) over a
    seeded source sample sized to ~budget_s seconds on `threads` cores."""
    from oracle.refbind import CpuOracle, RefOracle, ref_available
    from svg_b200 import meshgen
    V = len(pos)
    rng = np.random.default_rng(seed)
    if ref_available():
        kind = "reference"
        td = tempfile.mkdtemp()
        obj = os.path.join(td, "m.obj")
        meshgen.write_obj(obj, pos, faces)
        mesh = RefOracle().load(obj, fix_boundary=True)
    else:
        kind = "port"
        mesh = CpuOracle().mesh(pos, faces)
    probe = rng.choice(V, min(V, max(threads * 4, 64)), replace=False).astype(np.int32)
    r = mesh.build(K, probe, threads=threads)
    per_src = max(r.seconds, 1e-6) / len(probe)
    n = int(min(V, max(len(probe), budget_s / per_src)))
    sample = rng.choice(V, n, replace=False).astype(np.int32)
    r = mesh.build(K, sample, threads=threads)
    edges = int(r.tails.sum())
    return {"value": edges / r.seconds, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{n} of {V} sources (seeded), full reference per-source loop incl. O(V) emission",
            "seconds": r.seconds, "edges": edges, "est_full_build_s": r.seconds * V / n}


def run_reference_arm(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    pos, faces = workload_mesh()
    threads = os.cpu_count() or 1
    vals = []
    last = None
    for i in range(args.warmup + args.steps):
        res = cpu_reference_run(pos, faces, K_BUILD, budget_s=args.ref_seconds, threads=threads, seed=i)
        if i >= args.warmup:
            vals.append(res["value"])
            last = res
    v = statistics.mean(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": dict(WORKLOAD, mode="reference_cpu"),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": last["kind"],
                             "sample": last["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "est_full_build_s": last["est_full_build_s"]}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="svg_b200", choices=["svg_b200", "reference"])
    ap.add_argument("--ref-seconds", type=float, default=12.0)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    ws, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    dist = init_dist(ws)
    from svg_b200.build_ext import build as build_lib
    if rank == 0:
        build_lib()
    barrier(dist)
    import svg_b200
    from svg_b200 import SVG, Mesh, MODE_BATCHED, MODE_PLAIN
    L = svg_b200.lib()

    pos, faces = workload_mesh()
    mesh = Mesh.from_arrays(pos, faces)
    mesh.copyToGPU()
    svg = SVG()
    svg.AssignMesh(mesh)
    svg.SetParameters(K_BUILD, 10, 2)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def flush_l2():
        flush.zero_()
        torch.cuda.synchronize()

    def timed_build(mode=MODE_BATCHED):
        flush_l2()
        a = C.c_double()
        L.svg_timer_mark(C.byref(a))
        st = svg.ConstructSVG(mode=mode)
        b = C.c_double()
        L.svg_timer_mark(C.byref(b))
        return b.value, st

    for _ in range(args.warmup):
        timed_build()
    barrier(dist)
    torch.cuda.synchronize()
    clocks = Clocks(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local)
    clocks.start()
    times, kern, edges, launches = [], [], 0, 0
    st = None
    for _ in range(args.steps):
        ms, st = timed_build()
        times.append(ms)
        kern.append(st["ms_total"])
        edges += st["edges"]
        launches += st["launches"]
    torch.cuda.synchronize()
    barrier(dist)
    ck = clocks.stop()
    total_ms = sum(times)
    total_ms_max = max_over_ranks(dist, total_ms)
    value = replica_value(dist, float(edges), total_ms)

    # ---- end to end through the C ABI from host buffers
    posc = np.ascontiguousarray(pos.reshape(-1))
    facc = np.ascontiguousarray(faces.reshape(-1).astype(np.int32))
    e2e_ms, e2e_edges, h2d, d2h = [], 0, 0, 0
    for i in range(args.warmup + args.steps):
        flush_l2()
        a = C.c_double()
        L.svg_timer_mark(C.byref(a))
        t0 = time.perf_counter()
        m2 = Mesh.from_arrays(posc, facc)
        m2.copyToGPU()
        s2 = SVG()
        s2.AssignMesh(m2)
        s2.SetParameters(K_BUILD, 10, 2)
        st2 = s2.ConstructSVG()
        off, adj, dist_h = s2.csr()
        b = C.c_double()
        L.svg_timer_mark(C.byref(b))
        wall = (time.perf_counter() - t0) * 1e3
        if i >= args.warmup:
            e2e_ms.append(max(b.value, wall))
            e2e_edges += st2["edges"]
            h2d = m2.edgeNum * 64 + m2.vertNum * (8 + 24)
            d2h = off.nbytes + adj.nbytes + dist_h.nbytes
        s2.FreeSVGStructure()
        m2.clear()
    e2e_max = max_over_ranks(dist, sum(e2e_ms))
    e2e_val = replica_value(dist, float(e2e_edges), sum(e2e_ms))

    out = None
    if rank == 0:
        peaks = {}
        pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(pp):
            peaks = json.load(open(pp))
        plain = None
        if not args.no_plain:
            ms_p, stp = timed_build(MODE_PLAIN)
            plain = {"build_ms": ms_p, "edges_per_s": stp["edges"] / (ms_p / 1e3),
                     "speedup_batched_vs_plain": (ms_p / (total_ms / args.steps)), "grid": "64x128",
                     "windows": stp["windows"]}
            svg.ConstructSVG(mode=MODE_BATCHED)  # leave the batched graph resident
        cpu = None
        if not args.no_cpu:
            try:
                cpu = cpu_reference_run(pos, faces, K_BUILD, budget_s=args.ref_seconds, threads=os.cpu_count() or 1)
            except Exception as e:  # reported, not fatal
                cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "unavailable",
                       "sample": f"failed: {e}"}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(WORKLOAD, l2="flushed between steps (256 MiB write)", parallelism=f"replicas{ws}",
                           edges_per_build=st["edges"], windows_per_build=st["windows"]),
            "build_s": total_ms_max / args.steps / 1e3,
            "kernel_ms_per_step": statistics.mean(kern),
            "roofline": roofline_figures(st, peaks),
            "cpu_baseline": cpu,
            "plain": plain,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_max / args.steps},
            "gpu_launches": launches,
            "clocks": ck,
            "flags": {k: st[k] for k in ("queue_drop_sources", "ref_overflow_sources", "watchdog_sources",
                                         "undefined_sources", "retried_sources")},
        }
        print(json.dumps(out), flush=True)
    svg.FreeSVGStructure()
    if dist is not None:
        barrier(dist)
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
