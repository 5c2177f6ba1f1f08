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

Multi-GPU (--gpus N under torchrun): the build is sharded - every rank builds
a contiguous range of the sources (sources are independent) and the CSR slices
are all-gathered over NCCL so every rank holds the whole graph; scaling
"strong", a step's time is the max over ranks of build + gather.  --replicas
runs N whole builds instead (scaling "weak", no collective).
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

from svg_b200.shard import gather_csr, shard_ranges  # noqa: E402

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

    def __init__(self, index):
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


def device_view(ptr: int, n: int, typestr: str):
    """A torch tensor over n elements of device memory the library owns (no copy)."""
    import torch

    class _Dev:
        pass

    d = _Dev()
    d.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                  "version": 2, "strides": None}
    return torch.as_tensor(d, device="cuda")


def fma_rate():
    """The GPU's measured FP64 fused-multiply-add rate (svg_device_fp64_rate), or None."""
    try:
        import svg_b200
        x = C.c_double()
        if svg_b200.lib().svg_device_fp64_rate(C.byref(x)) == 0:
            return x.value
    except Exception:
        pass
    return None


def smi_index(local: int) -> str:
    """nvidia-smi's name for this process's GPU: the CUDA_VISIBLE_DEVICES entry
    (an index or a UUID) when that is set, else the local ordinal."""
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if local < len(ids):
            return ids[local]
    return str(local)


def emit(line: dict, args) -> None:
    """Print the JSON line; with --record also write it to that file."""
    text = json.dumps(line)
    print(text, flush=True)
    if getattr(args, "record", None):
        d = os.path.dirname(os.path.abspath(args.record))
        os.makedirs(d, exist_ok=True)
        with open(args.record, "w") as f:
            f.write(text + "\n")


def workload_mesh():
    from svg_b200 import meshgen
    return meshgen.height_field(WORKLOAD["grid"], seed=WORKLOAD["seed"])


def roofline_figures(st: dict, peaks: dict, fma_per_s: float | None = None) -> dict:
    """Roofline of the window-propagation kernel (k_ich_batched).

    HBM form, in the unit of the path's scope table: 250 algorithmic bytes per
    propagated window (3 half-edge records of the unfolded face 60 B, 3
    vertex-state reads 48 B, 1-2 split-state reads ~24 B, one 64 B window
    written and read back 128 B) plus 12 B per output edge (adjacency +
    length).  Beside it, the detailed count of what this kernel's loop reads
    and writes per window: 3 half-edge records (3 x 32 B), the apex and two
    opposite-vertex records (3 x 16 B), four vertex-state probes (4 x 32 B),
    one split-state probe (32 B), the window popped (16 B key + 48 B payload)
    and up to two pushed (2 x 64 B): ~450 B, plus 24 B per exported candidate.
    FP64 form: ~300 FP64 operations per window (adds, multiplies, ~10
    divides, ~12 square roots, no fused multiply-adds) against the measured
    FP64 pipe rate (fused multiply-adds per second: one instruction each).
    Traffic: ncu DRAM bytes per window of a captured launch
    (profiles/ich_batched_traffic.json) x this launch's windows."""
    kernel_s = st["ms_ich"] / 1e3
    peak = peaks.get("hbm_gbs")
    src = "measured"
    if not peak:
        peak, src = 6650.0, "fallback"
    bytes_alg = st["windows"] * 250.0 + st["edges"] * 12.0
    bytes_det = st["windows"] * 450.0 + st["edges"] * 24.0
    achieved = bytes_alg / kernel_s / 1e9 if kernel_s > 0 else 0.0
    ach_det = bytes_det / kernel_s / 1e9 if kernel_s > 0 else 0.0
    traffic = None
    tsrc = None
    tp = os.path.join(ROOT, "profiles", "ich_batched_traffic.json")
    if os.path.exists(tp):
        try:
            t = json.load(open(tp))
            traffic = t["dram_bytes_per_window"] * st["windows"]
            tsrc = t.get("capture")
        except Exception:
            traffic = None
    ops = st["windows"] * 300.0
    fp64 = {"ops_per_window": 300, "achieved_tflops": round(ops / kernel_s / 1e12, 4) if kernel_s > 0 else 0.0}
    if fma_per_s:
        fp64.update({"peak_fma_per_s": fma_per_s, "peak_tflops_fma_as_2": round(2 * fma_per_s / 1e12, 2),
                     "frac_of_pipe": round(ops / kernel_s / fma_per_s, 5) if kernel_s > 0 else 0.0,
                     "peak_source": "measured here (svg_device_fp64_rate: DFMA loop, CUDA events)"})
    return {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 5), "traffic": traffic, "peak_source": src,
            "kernel": "k_ich_batched", "algorithmic_bytes_per_launch": bytes_alg,
            "unit_bytes": "250 B per window + 12 B per edge",
            "detailed": {"bytes_per_launch": bytes_det, "achieved": round(ach_det, 2),
                         "frac": round(ach_det / peak, 5), "unit_bytes": "450 B per window + 24 B per candidate"},
            "traffic_source": tsrc,
            "traffic_per_window": (traffic / st["windows"]) if traffic and st["windows"] else None,
            "kernel_ms": st["ms_ich"], "fp64": fp64}


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


# ---------------------------------------------------------------- other configurations
# `--workload large` (750K-vertex torus builds) and `--workload serve` (serving
# loop on its K=100 graph) print their own JSON line; the default workload is
# the build benchmark above.

LARGE = dict(mesh="torus_value_noise", R=1.0, r=0.4, grid="1000x750", vertices=750000, seed=2)


def _pct(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


def _gpu_setup():
    import torch
    ws, rank, local = dist_env()
    if ws != 1:
        raise SystemExit("this workload runs on one GPU")
    torch.cuda.set_device(local)
    from svg_b200.build_ext import build as build_lib
    build_lib()
    return torch


def work_histogram(windows: np.ndarray) -> dict:
    """Per-source propagated windows: log2 buckets and spread."""
    w = np.asarray(windows, np.int64)
    w = w[w > 0]
    if len(w) == 0:
        return {}
    b = np.floor(np.log2(w)).astype(np.int64)
    cnt = np.bincount(b)
    srt = np.sort(w)[::-1]
    top = max(1, len(w) // 100)
    return {"log2_buckets": {f"[2^{i},2^{i + 1})": int(c) for i, c in enumerate(cnt) if c},
            "min": int(w.min()), "median": float(np.median(w)), "p99": _pct(w, 99), "max": int(w.max()),
            "max_over_median": float(w.max() / np.median(w)),
            "top1pct_share": float(srt[:top].sum() / w.sum())}


def run_large(args):
    """750K-vertex torus (5-octave value noise, seed 2) built at each K with the
    batched kernel under a stated build-scratch budget: time, edges/s, peak
    device memory, per-source work histogram; the plain form on a leading
    slice of sources, extrapolated to the whole mesh (labelled)."""
    torch = _gpu_setup()
    import svg_b200
    from svg_b200 import SVG, Mesh, MODE_PLAIN, meshgen
    L = svg_b200.lib()
    t0 = time.perf_counter()
    pos, faces = meshgen.config_mesh(2, args.scale)
    mesh = Mesh.from_arrays(pos, faces)
    mesh.copyToGPU()
    mesh_s = time.perf_counter() - t0
    V = mesh.vertNum
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    budget = int(args.hbm_budget_gb * (1 << 30))

    def mark():
        x = C.c_double()
        L.svg_timer_mark(C.byref(x))
        return x.value

    out = []
    clocks = Clocks(smi_index(0))
    clocks.start()
    for K in [int(k) for k in args.K.split(",")]:
        svg = SVG()
        svg.AssignMesh(mesh)
        svg.SetParameters(K)
        for _ in range(args.warmup):   # the first build also records per-source costs (heavy-first order)
            svg.ConstructSVG(hbm_budget=budget)
        svg.FreeSVGStructure()
        svg_b200.device_memory(reset_peak=True)
        times, st = [], None
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            mark()
            st = svg.ConstructSVG(hbm_budget=budget)
            times.append(mark())
        mem = svg_b200.device_memory()
        w, q, f = svg.source_stats()
        row = {"K": K, "build_s": statistics.mean(times) / 1e3, "build_s_all": [t / 1e3 for t in times],
               "edges": st["edges"], "edges_per_s": st["edges"] / (statistics.mean(times) / 1e3),
               "windows": st["windows"], "kernel_ms_ich": st["ms_ich"], "kernel_ms_emit": st["ms_emit"],
               "peak_device_bytes": mem["peak"], "scratch_bytes": st["scratch_bytes"],
               "hbm_budget_bytes": budget, "work_histogram": work_histogram(w),
               "flags": {k: st[k] for k in ("queue_drop_sources", "ref_overflow_sources", "watchdog_sources",
                                            "undefined_sources", "retried_sources")}}
        svg.FreeSVGStructure()
        if args.plain_frac > 0:
            n = max(1, int(V * args.plain_frac))
            p = SVG()
            p.AssignMesh(mesh)
            p.SetParameters(K)
            flush.zero_()
            torch.cuda.synchronize()
            mark()
            stp = p.ConstructSVG(mode=MODE_PLAIN, source_begin=0, source_end=n)
            ms = mark()
            p.FreeSVGStructure()
            full = ms / 1e3 * V / n
            row["plain"] = {"sources": n, "build_s": ms / 1e3, "edges": stp["edges"],
                            "est_full_build_s": full, "speedup_batched_vs_plain_est": full / row["build_s"],
                            "note": (f"plain form (64x128 grid, one source per thread), all {V} sources, measured"
                                     if n == V else
                                     f"plain form (64x128 grid, one source per thread) on sources [0,{n}) "
                                     f"of {V}, time scaled by {V}/{n} (extrapolated)")}
        out.append(row)
        log(json.dumps(row))
    line = {"metric": "svg_build_edges_per_s", "value": out[-1]["edges_per_s"], "unit": "edges/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(LARGE, workload=f"svg_build_torus_1000x750_value_noise_K{args.K.replace(',', '_')}",
                           vertices=V, scale=args.scale, l2="flushed between steps (256 MiB write)"),
            "mesh_host_build_and_upload_s": mesh_s, "per_K": out, "clocks": clocks.stop()}
    emit(line, args)
    return 0


def make_stream(V: int, rate: float, duration: float, seed: int = 3):
    """Poisson arrivals at `rate`/s for `duration` s: 70 % SSSD on uniform
    random pairs, 30 % MSAD with log-uniform set sizes in [1, 1000] of uniform
    random vertices (duplicates removed), weights 0."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, int(rate * duration * 1.3) + 64)
    arr = np.cumsum(gaps)
    arr = arr[arr < duration]
    n = len(arr)
    is_sssd = rng.random(n) < 0.7
    reqs = []
    for i in range(n):
        if is_sssd[i]:
            a, b = rng.integers(0, V, 2)
            reqs.append((float(arr[i]), 0, int(a), int(b)))
        else:
            k = int(np.clip(np.rint(np.exp(rng.uniform(0.0, np.log(1000.0)))), 1, 1000))
            reqs.append((float(arr[i]), 1, np.unique(rng.integers(0, V, k)).astype(np.int32), None))
    return reqs


def run_serve(args):
    """Serving on the resident K=100 SVG of the 750K-vertex torus: a Poisson
    stream through the serving loop (continuous batching), then the plain
    form (one query per launch, synchronous) on the stream's first requests."""
    import threading
    torch = _gpu_setup()
    import svg_b200
    from svg_b200 import SVG, Mesh, Server, meshgen
    pos, faces = meshgen.config_mesh(2, args.scale)
    mesh = Mesh.from_arrays(pos, faces)
    mesh.copyToGPU()
    V = mesh.vertNum
    svg = SVG()
    svg.AssignMesh(mesh)
    svg.SetParameters(100)
    bst = svg.ConstructSVG()
    reqs = make_stream(V, args.rate, args.duration)
    n = len(reqs)
    log(f"serve: V={V} edges={bst['edges']} requests={n}")

    srv = Server(lanes=args.lanes, max_batch=args.max_batch, max_batch_msad=args.max_batch_msad,
                 slots_per_lane=args.slots, cluster=args.cluster, hbm_budget=int(args.hbm_budget_gb * (1 << 30)),
                 staging_in_bytes=16 << 20, staging_out_bytes=int(args.staging_out_mb) << 20)
    gid = srv.add_graph(svg)
    # warm-up: a few requests of each kind
    wt = [srv.submit_sssd(gid, i, V - 1 - i) for i in range(64)]
    wt += [srv.submit_msad(gid, np.array([i], np.int32), out=(None, None)) for i in range(8)]
    for t in wt:
        srv.wait(t, 600.0)
        srv.take(t)

    RING = args.ring
    ring_d = [np.zeros(V) for _ in range(RING)]
    ring_s = [np.zeros(V, np.int32) for _ in range(RING)]
    import queue
    ring_free = queue.Queue()
    for i in range(RING):
        ring_free.put(i)
    slot_of = {}
    kind_of = {}
    lat = {0: [], 1: []}
    done_n = [0]
    t_done = [0.0]
    samples = {}
    want = {i for i in range(n) if i < 400}
    ticket_req = {}
    lag = []
    lock = threading.Lock()
    finished = threading.Event()
    stop = threading.Event()
    failed = [0]

    def collector():
        while done_n[0] < n and not stop.is_set():
            res = srv.poll(4096)
            if not res:
                time.sleep(0.0002)
                continue
            for r in res:
                t = r["ticket"]
                with lock:
                    i = ticket_req.get(t)
                if i is None:       # submitted but not yet registered: next poll
                    continue
                k = kind_of[t]
                if r["status"] != 0:
                    failed[0] += 1
                else:
                    lat[k].append(r["latency_ms"])
                if i in want and r["status"] == 0:
                    samples[i] = r["dist"] if k == 0 else ring_d[slot_of[t]].copy()
                srv.take(t)
                if k == 1:
                    ring_free.put(slot_of.pop(t))
                done_n[0] += 1
            t_done[0] = time.perf_counter()
        finished.set()

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    st0 = srv.stats()
    clocks = Clocks(smi_index(0))
    clocks.start()
    t0 = time.perf_counter()
    for i, (ta, kind, a, b) in enumerate(reqs):
        target = t0 + ta
        now = time.perf_counter()
        if now < target:
            time.sleep(max(0.0, target - now - 0.0001))
            while time.perf_counter() < target:
                pass
        lag.append((time.perf_counter() - target) * 1e3)
        if kind == 0:
            t = srv.submit_sssd(gid, a, b)
        else:
            sl = ring_free.get(timeout=args.duration * 2 + 120)   # raises instead of waiting for good
            t = srv.submit_msad(gid, a, out=(ring_d[sl], ring_s[sl]))
            slot_of[t] = sl
        kind_of[t] = kind
        with lock:
            ticket_req[t] = i
    complete = finished.wait(args.duration * 2 + 120)
    wall = (t_done[0] if complete else time.perf_counter()) - t0
    ck = clocks.stop()
    st1 = srv.stats()
    stop.set()
    th.join(5.0)
    srv.close()

    # results equal the synchronous batch calls
    mism = 0
    for i, v in samples.items():
        _, kind, a, b = reqs[i]
        if kind == 0:
            mism += int(v != svg.sssd_batch(np.array([a], np.int32), np.array([b], np.int32))[0])
        else:
            d, _ = svg.msad_batch([a])
            mism += int(not np.array_equal(v, d[0]))

    # one query per launch, synchronous, on the stream's first requests: the
    # plain form (one block per query, the reference's one-search-at-a-time
    # form) and, for the latency floor, the cluster form
    def one_per_launch(form):
        svg.set_query_form(form)
        svg.sssd_batch(np.array([0], np.int32), np.array([1], np.int32))   # query context set-up
        svg.msad_batch([np.array([0], np.int32)])
        tms = {0: [], 1: []}
        tp0 = time.perf_counter()
        for i, (_, kind, a, b) in enumerate(reqs):
            if i >= args.plain_requests or time.perf_counter() - tp0 > args.plain_seconds:
                break
            t1 = time.perf_counter()
            if kind == 0:
                svg.sssd_batch(np.array([a], np.int32), np.array([b], np.int32))
            else:
                svg.msad_batch([a])
            tms[kind].append((time.perf_counter() - t1) * 1e3)
        return tms

    from svg_b200 import QUERY_CLUSTER, QUERY_PLAIN
    plain_t = one_per_launch(QUERY_PLAIN)
    single_t = one_per_launch(QUERY_CLUSTER)
    allp = plain_t[0] + plain_t[1]
    plain_qps = len(allp) / (sum(allp) / 1e3) if allp else None
    alls = single_t[0] + single_t[1]
    alll = lat[0] + lat[1]
    qps = (len(lat[0]) + len(lat[1])) / wall
    line = {"metric": "serve_qps", "value": qps, "unit": "req/s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(LARGE, workload="serve_torus_1000x750_K100_poisson", K=100, vertices=V,
                           rate_per_s=args.rate, duration_s=args.duration, requests=n, sssd_share=0.7,
                           msad_set_size="log-uniform [1,1000]", seed=3, lanes=args.lanes,
                           max_batch=args.max_batch, max_batch_msad=args.max_batch_msad, slots_per_lane=args.slots,
                           cluster=args.cluster, scale=args.scale),
            "offered_per_s": n / args.duration, "wall_s": wall, "complete": bool(complete), "failed": failed[0],
            "latency_ms": {"all": {"p50": _pct(alll, 50), "p99": _pct(alll, 99)},
                           "sssd": {"p50": _pct(lat[0], 50), "p99": _pct(lat[0], 99), "n": len(lat[0])},
                           "msad": {"p50": _pct(lat[1], 50), "p99": _pct(lat[1], 99), "n": len(lat[1])}},
            "submit_lag_ms": {"p50": _pct(lag, 50), "p99": _pct(lag, 99)},
            "batches": st1["batches"] - st0["batches"],
            "mean_batch": (st1["batched_requests"] - st0["batched_requests"]) / max(1, st1["batches"] - st0["batches"]),
            "checked_vs_sync": len(samples), "mismatches_vs_sync": mism,
            "plain": {"requests": len(allp), "qps": plain_qps,
                      "latency_ms": {"all": {"p50": _pct(allp, 50), "p99": _pct(allp, 99)},
                                     "sssd": {"p50": _pct(plain_t[0], 50), "p99": _pct(plain_t[0], 99)},
                                     "msad": {"p50": _pct(plain_t[1], 50), "p99": _pct(plain_t[1], 99)}},
                      "form": "one query per launch, synchronous, inputs from and result to host"},
            "one_per_launch_cluster": {"requests": len(alls), "qps": len(alls) / (sum(alls) / 1e3) if alls else None,
                                       "latency_ms": {"sssd": {"p50": _pct(single_t[0], 50), "p99": _pct(single_t[0], 99)},
                                                      "msad": {"p50": _pct(single_t[1], 50), "p99": _pct(single_t[1], 99)}}},
            "qps_vs_plain": (qps / plain_qps) if plain_qps else None,
            "p99_ms_serving_vs_plain": [_pct(alll, 99), _pct(allp, 99)],
            "build": {"edges": bst["edges"], "ms": bst["ms_total"]},
            "clocks": ck}
    emit(line, args)
    return 0


CONFIG0 = dict(workload="svg_build_torus_200x150_K100_sssd100", mesh="torus", R=1.0, r=0.35, grid="200x150",
               vertices=30000, K=100, seed=0, queries="100 SSSD A*, uniform random pairs (seed 0)")


def run_config0(args):
    """The plain-method configuration: the 30,000-vertex torus (200x150 grid,
    tube radius jittered by 0.02 r N(0,1), seed 0) built at K=100 by the
    batched kernel (timed steps), by the plain form (one source per thread,
    the reference's 64x128 grid and a grid filling every SM) and by the
    reference's own construction on all host cores (every source); then 100
    SSSD A* queries on uniform random vertex pairs: one batch through the C
    ABI (host buffers), one query per launch, and the reference's host A* per
    query on the graph the reference built (SVG.cu:241-251, 369-413)."""
    torch = _gpu_setup()
    import svg_b200
    from svg_b200 import SVG, Mesh, MODE_PLAIN, meshgen
    L = svg_b200.lib()
    K = CONFIG0["K"]
    pos, faces = meshgen.config_mesh(0)
    mesh = Mesh.from_arrays(pos, faces)
    mesh.copyToGPU()
    V = mesh.vertNum
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def mark():
        x = C.c_double()
        L.svg_timer_mark(C.byref(x))
        return x.value

    def fresh():
        flush.zero_()
        torch.cuda.synchronize()
        mark()

    svg = SVG()
    svg.AssignMesh(mesh)
    svg.SetParameters(K)
    for _ in range(args.warmup):
        svg.ConstructSVG()
    clocks = Clocks(smi_index(0))
    clocks.start()
    times, st = [], None
    for _ in range(args.steps):
        fresh()
        st = svg.ConstructSVG()
        times.append(mark())
    build_ms = statistics.mean(times)
    plain = {}
    for name, blocks in (("grid_64x128", 64), ("grid_all_sms", 0)):
        p = SVG()
        p.AssignMesh(mesh)
        p.SetParameters(K)
        if blocks == 0:
            per_sm = torch.cuda.get_device_properties(0).multi_processor_count
            blocks = per_sm * 4
        fresh()
        stp = p.ConstructSVG(mode=MODE_PLAIN, blocks=blocks)
        ms = mark()
        plain[name] = {"blocks": blocks, "threads_per_block": 128, "build_ms": ms,
                       "edges_per_s": stp["edges"] / (ms / 1e3), "speedup_batched_vs_plain": ms / build_ms}
        p.FreeSVGStructure()

    rng = np.random.default_rng(0)
    s = rng.integers(0, V, 100).astype(np.int32)
    t = rng.integers(0, V, 100).astype(np.int32)
    svg.sssd_batch(s[:1], t[:1])   # query context set-up
    fresh()
    w0 = time.perf_counter()
    d_batch = svg.sssd_batch(s, t)
    batch_wall = (time.perf_counter() - w0) * 1e3
    batch_dev = mark()
    per = []
    for i in range(len(s)):
        w0 = time.perf_counter()
        svg.sssd_batch(s[i:i + 1], t[i:i + 1])
        per.append((time.perf_counter() - w0) * 1e3)
    ck = clocks.stop()
    off, nodes = svg.CopySVGToHost()

    cpu = None
    ref_q = None
    if not args.no_cpu:
        # the reference's own construction and A* (test oracle; reported baseline only)
        from oracle.refbind import RefOracle, ref_available
        if ref_available():
            td = tempfile.mkdtemp()
            obj = os.path.join(td, "m.obj")
            meshgen.write_obj(obj, pos, faces)
            rm = RefOracle().load(obj, fix_boundary=True)
            cores = os.cpu_count() or 1
            rows = rm.build(K, None, threads=cores)
            edges = int(rows.tails.sum())
            cpu = {"value": edges / rows.seconds, "unit": UNIT, "cores": cores, "kind": "reference",
                   "sample": f"all {V} sources, the reference's per-source loop incl. its O(V) emission scan",
                   "seconds": rows.seconds, "edges": edges}
            dq, secs = rm.sssd(K, rows.tails, rows.nodes, s, t)
            same_graph = bool(np.array_equal(np.diff(off), rows.tails))
            rel = np.abs(d_batch - dq) / np.maximum(dq, 1e-300)
            ref_q = {"host_ms_per_query": secs * 1e3 / len(s), "host_total_ms": secs * 1e3, "cores": 1,
                     "max_rel_diff_vs_gpu": float(rel.max()), "identical": int((d_batch == dq).sum()),
                     "graph_degrees_identical": same_graph}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "unavailable",
                   "sample": "oracle/_ref not built"}
    line = {"metric": METRIC, "value": st["edges"] / (build_ms / 1e3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": build_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CONFIG0, l2="flushed between steps (256 MiB write)", edges_per_build=st["edges"],
                           windows_per_build=st["windows"]),
            "build_ms_all": times, "plain": plain, "cpu_baseline": cpu,
            "sssd": {"n": len(s), "batch_device_ms": batch_dev, "batch_wall_ms": batch_wall,
                     "one_per_launch_wall_ms": {"mean": statistics.mean(per), "p50": _pct(per, 50),
                                                "p99": _pct(per, 99)},
                     "reference_host": ref_q},
            "clocks": ck,
            "flags": {k: st[k] for k in ("queue_drop_sources", "ref_overflow_sources", "watchdog_sources",
                                         "undefined_sources", "retried_sources")}}
    emit(line, args)
    return 0


def run_case(args):
    """One batched build of the 270x270 height field over sources [0, N) with
    a fixed number of blocks: a small, self-contained launch of the build
    kernel for profilers (N and the block count bound the device memory)."""
    _gpu_setup()
    from svg_b200 import SVG, Mesh, meshgen
    pos, faces = meshgen.config_mesh(1, args.scale)
    mesh = Mesh.from_arrays(pos, faces)
    mesh.copyToGPU()
    svg = SVG()
    svg.AssignMesh(mesh)
    svg.SetParameters(int(args.K.split(",")[0]))
    n = min(args.sources, mesh.vertNum) if args.sources > 0 else mesh.vertNum
    st = svg.ConstructSVG(source_begin=0, source_end=n, blocks=args.blocks, heavy_first=0)
    print(json.dumps({"workload": "case_height_field", "K": svg.K, "sources": n, "blocks": args.blocks,
                      "stats": st}), flush=True)
    return 0


def run_queries(args):
    """Batched query kernels on the resident K=100 SVG of the 750K-vertex
    torus, device buffers only (CUDA events on the library stream): SSSD and
    MSAD batches in the cluster form and the plain form, and one query per
    launch in each.  Roofline of the MSAD kernel: per query every edge is
    relaxed once (4 B adjacency + 8 B length + a 16 B {dist, src} read) and
    every vertex is initialised, read back and written out (16 + 16 + 12 B)."""
    torch = _gpu_setup()
    import svg_b200
    from svg_b200 import SVG, Mesh, QUERY_CLUSTER, QUERY_PLAIN, meshgen
    L = svg_b200.lib()
    P = C.c_void_p
    pos, faces = meshgen.config_mesh(2, args.scale)
    mesh = Mesh.from_arrays(pos, faces)
    mesh.copyToGPU()
    V = mesh.vertNum
    svg = SVG()
    svg.AssignMesh(mesh)
    svg.SetParameters(100)
    svg.ConstructSVG(with_paths=False)
    L.svg_trim_device_cache()
    _, E, _ = svg.counts()
    rng = np.random.default_rng(3)

    def mark():
        x = C.c_double()
        L.svg_timer_mark(C.byref(x))
        return x.value

    NS, NM = args.sssd_batch, args.msad_batch
    S = torch.tensor(rng.integers(0, V, NS), dtype=torch.int32, device="cuda")
    T = torch.tensor(rng.integers(0, V, NS), dtype=torch.int32, device="cuda")
    D = torch.empty(NS, dtype=torch.float64, device="cuda")
    sizes = [int(np.clip(np.rint(np.exp(rng.uniform(0, np.log(1000)))), 1, 1000)) for _ in range(NM)]
    sets = [np.unique(rng.integers(0, V, k)).astype(np.int32) for k in sizes]
    off = np.zeros(NM + 1, np.int64)
    np.cumsum([len(x) for x in sets], out=off[1:])
    d_off = torch.tensor(off, device="cuda")
    d_src = torch.tensor(np.concatenate(sets), device="cuda")
    d_w = torch.zeros(len(d_src), dtype=torch.float64, device="cuda")
    d_dist = torch.empty(NM * V, dtype=torch.float64, device="cuda")
    d_sid = torch.empty(NM * V, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def sssd(n, o=0):
        assert L.svg_sssd_batch_device(svg._g, n, P(S.data_ptr() + 4 * o), P(T.data_ptr() + 4 * o),
                                       P(D.data_ptr())) == 0

    def msad(n, o=0):
        assert L.svg_msad_batch_device(svg._g, n, P(d_off.data_ptr() + 8 * o), P(d_src.data_ptr()),
                                       P(d_w.data_ptr()), P(d_dist.data_ptr()), P(d_sid.data_ptr())) == 0

    def timed(fn, *a):
        flush.zero_()
        torch.cuda.synchronize()
        mark()
        fn(*a)
        return mark()

    out = {}
    clocks = Clocks(smi_index(0))
    clocks.start()
    for name, form in (("cluster", QUERY_CLUSTER), ("plain", QUERY_PLAIN)):
        svg.set_query_form(form)
        sssd(8)
        msad(2)   # context set-up
        mark()
        r = {}
        r["sssd_single_ms_p50"] = float(np.median([timed(sssd, 1, i) for i in range(args.single)]))
        r["msad_single_ms_p50"] = float(np.median([timed(msad, 1, i) for i in range(min(args.single, NM))]))
        ts = [timed(sssd, NS) for _ in range(args.steps)]
        r["sssd_batch_qps"] = NS / (statistics.mean(ts) / 1e3)
        tm = [timed(msad, NM) for _ in range(args.steps)]
        r["msad_batch_ms"] = statistics.mean(tm)
        r["msad_batch_qps"] = NM / (statistics.mean(tm) / 1e3)
        out[name] = r
    svg.set_query_form(QUERY_CLUSTER)
    ck = clocks.stop()
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    peak = peaks.get("hbm_gbs") or 6650.0
    bytes_q = E * 28.0 + V * 44.0
    ach = bytes_q * NM / (out["cluster"]["msad_batch_ms"] / 1e3) / 1e9
    line = {"metric": "msad_batch_qps", "value": out["cluster"]["msad_batch_qps"], "unit": "queries/s", "n_gpus": 1,
            "steps": args.steps, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": dict(LARGE, workload="queries_torus_1000x750_K100", K=100, vertices=V, edges=E,
                           sssd_batch=NS, msad_batch=NM, msad_set_size="log-uniform [1,1000]", seed=3,
                           l2="flushed before every timed call (256 MiB write)", scale=args.scale),
            "forms": out,
            "msad_batch_speedup_cluster_vs_plain": out["cluster"]["msad_batch_qps"] / out["plain"]["msad_batch_qps"],
            "roofline": {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(ach / peak, 4), "traffic": None, "kernel": "k_query_cluster (MSAD)",
                         "algorithmic_bytes_per_query": bytes_q,
                         "peak_source": "measured" if peaks.get("hbm_gbs") else "fallback"},
            "clocks": ck}
    emit(line, args)
    return 0


def run_mixed(args):
    """Mixed build + query serving: the pool of 8 meshes (5K..300K vertices,
    seeds 10-17, tori and height fields), each built once at the start with K
    drawn from {50, 200}, then further builds of random (mesh, K) pairs
    arriving as a Poisson stream, interleaved with a Poisson query stream
    (70 % SSSD, 30 % MSAD with log-uniform set sizes in [1, 1000]) against
    the graphs already built, all under one device-memory budget with
    eviction of least-recently-used graphs and rebuild on demand."""
    import threading
    _gpu_setup()
    from svg_b200 import Mesh, Server, meshgen
    meshes = []
    for pos, faces in meshgen.pool_meshes(args.scale):
        m = Mesh.from_arrays(pos, faces)
        m.copyToGPU()
        meshes.append(m)
    Vs = [m.vertNum for m in meshes]
    rng = np.random.default_rng(4)
    dur = args.duration
    ev = []   # (time, kind, payload): kind 0/1 query, 2 build
    for i in range(len(meshes)):
        ev.append((0.05 * i, 2, (i, int(rng.choice([50, 200])))))
    t = 0.0
    while True:
        t += rng.exponential(1.0 / args.build_rate)
        if t >= dur:
            break
        ev.append((t, 2, (int(rng.integers(0, len(meshes))), int(rng.choice([50, 200])))))
    qa = np.cumsum(rng.exponential(1.0 / args.rate, int(args.rate * dur * 1.3) + 64))
    qa = qa[(qa < dur) & (qa > 0.5)]   # queries start once the first graphs can be resident
    kinds = rng.random(len(qa)) < 0.7
    for ta, k in zip(qa, kinds):
        ev.append((float(ta), 0 if k else 1, None))
    ev.sort(key=lambda e: e[0])
    n_ev = len(ev)

    srv = Server(hbm_budget=int(args.hbm_budget_gb * (1 << 30)), max_batch=args.max_batch,
                 max_batch_msad=args.max_batch_msad, cluster=args.cluster, staging_in_bytes=16 << 20,
                 staging_out_bytes=int(args.staging_out_mb) << 20)
    RING = args.ring
    vmax = max(Vs)
    ring_d = [np.zeros(vmax) for _ in range(RING)]
    ring_s = [np.zeros(vmax, np.int32) for _ in range(RING)]
    import queue
    ring_free = queue.Queue()
    for i in range(RING):
        ring_free.put(i)
    slot_of = {}
    info = {}      # ticket -> (kind, gid)
    lock = threading.Lock()
    lat = {0: [], 1: [], 2: []}
    builds = []
    failed = [0]
    gid_mesh = {}
    done_n = [0]
    t_done = [0.0]
    peak_res = [0]
    finished = threading.Event()

    stop = threading.Event()

    def collector():
        # results drained 256 at a time as a numpy array (no Python object per
        # field), so the thread holds the interpreter lock in short stretches
        # and the submitting loop keeps its schedule
        while done_n[0] < n_ev and not stop.is_set():
            res = srv.poll_array(256)
            if len(res) == 0:
                time.sleep(0.0002)
                continue
            tickets = res["ticket"].tolist()
            status = res["status"].tolist()
            lats = res["latency_ms"].tolist()
            for j, tk in enumerate(tickets):
                with lock:
                    it = info.get(tk)
                if it is None:       # submitted but not yet registered: next poll
                    continue
                kind, gid = it
                if status[j] != 0:
                    failed[0] += 1
                else:
                    lat[kind].append(lats[j])
                    if kind == 2:
                        builds.append((int(res["edges"][j]), float(res["build_ms"][j])))
                srv.take(tk)
                if kind == 1:
                    with lock:
                        sl = slot_of.pop(tk)
                    ring_free.put(sl)
                done_n[0] += 1
            t_done[0] = time.perf_counter()
            time.sleep(0)
        finished.set()

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    clocks = Clocks(smi_index(0))
    clocks.start()
    qrng = np.random.default_rng(5)
    res_ids, res_t = [], [0.0]
    # host time of the submitting loop by call, and how late each submission was
    host_s = {"submit_build": 0.0, "submit_query": 0.0, "resident": 0.0, "msad_slot_wait": 0.0, "stats": 0.0}
    lag = []
    bkw = {} if args.mixed_heavy_first < 0 else {"heavy_first": args.mixed_heavy_first}
    t0 = time.perf_counter()
    last_stats = t0
    for ta, kind, pl in ev:
        target = t0 + ta
        now = time.perf_counter()
        if now < target:
            time.sleep(max(0.0, target - now - 0.0001))
            while time.perf_counter() < target:
                pass
        lag.append((time.perf_counter() - target) * 1e3)
        if kind == 2:
            mi, K = pl
            tc = time.perf_counter()
            gid, tk = srv.submit_build(meshes[mi], K, **bkw)
            host_s["submit_build"] += time.perf_counter() - tc
            gid_mesh[gid] = mi
            with lock:
                info[tk] = (2, gid)
            continue
        # the graphs resident now (refreshed every 20 ms)
        tc = time.perf_counter()
        if time.perf_counter() - res_t[0] > 0.02 or not res_ids:
            res_ids[:] = srv.resident()
            res_t[0] = time.perf_counter()
        while not res_ids:   # nothing built yet: the query waits for the first graph
            time.sleep(0.001)
            res_ids[:] = srv.resident()
        host_s["resident"] += time.perf_counter() - tc
        gids = res_ids
        gid = gids[int(qrng.integers(0, len(gids)))]
        V = Vs[gid_mesh[gid]]
        if kind == 0:
            a, b = qrng.integers(0, V, 2)
            tc = time.perf_counter()
            tk = srv.submit_sssd(gid, int(a), int(b))
            host_s["submit_query"] += time.perf_counter() - tc
        else:
            k = int(np.clip(np.rint(np.exp(qrng.uniform(0.0, np.log(1000.0)))), 1, 1000))
            srcs = np.unique(qrng.integers(0, V, k)).astype(np.int32)
            tc = time.perf_counter()
            sl = ring_free.get(timeout=dur * 2 + 120)   # raises instead of waiting for good
            host_s["msad_slot_wait"] += time.perf_counter() - tc
            tc = time.perf_counter()
            tk = srv.submit_msad(gid, srcs, out=(ring_d[sl][:V], ring_s[sl][:V]))
            host_s["submit_query"] += time.perf_counter() - tc
            with lock:
                slot_of[tk] = sl
        with lock:
            info[tk] = (kind, gid)
        if time.perf_counter() - last_stats > 0.5:
            tc = time.perf_counter()
            peak_res[0] = max(peak_res[0], srv.stats()["resident_bytes"])
            last_stats = time.perf_counter()
            host_s["stats"] += last_stats - tc
    complete = finished.wait(dur * 2 + 120)
    wall = (t_done[0] if complete else time.perf_counter()) - t0
    ck = clocks.stop()
    st = srv.stats()
    stop.set()
    th.join(5.0)
    srv.close()
    nq = len(lat[0]) + len(lat[1])
    be = sum(e for e, _ in builds)
    bms = sum(m for _, m in builds)
    line = {"metric": "mixed_serve_qps", "value": nq / wall, "unit": "req/s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "mixed_build_query_pool8", "meshes": Vs, "K_choices": [50, 200],
                       "hbm_budget_gb": args.hbm_budget_gb, "query_rate_per_s": args.rate,
                       "build_rate_per_s": args.build_rate, "duration_s": dur, "seed": 4, "scale": args.scale},
            "wall_s": wall, "queries": nq, "failed": failed[0], "complete": bool(complete),
            "latency_ms": {"sssd": {"p50": _pct(lat[0], 50), "p99": _pct(lat[0], 99), "n": len(lat[0])},
                           "msad": {"p50": _pct(lat[1], 50), "p99": _pct(lat[1], 99), "n": len(lat[1])},
                           "build": {"p50": _pct(lat[2], 50), "p99": _pct(lat[2], 99), "n": len(lat[2])}},
            "builds": len(builds), "build_edges": be,
            "build_edges_per_s_device": be / (bms / 1e3) if bms > 0 else None,
            "builds_per_s": len(builds) / wall,
            "evictions": st["evictions"], "rebuilds": st["rebuilds"], "resident_graphs_end": st["resident_graphs"],
            "peak_resident_bytes_sampled": peak_res[0],
            "submit_lag_ms": {"p50": _pct(lag, 50), "p99": _pct(lag, 99), "max": max(lag) if lag else None},
            "submit_loop_host_s": {k: round(v, 3) for k, v in host_s.items()},
            "build_heavy_first": "library default" if args.mixed_heavy_first < 0 else args.mixed_heavy_first,
            "clocks": ck}
    emit(line, args)
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
    ap.add_argument("--workload", default="build", choices=["build", "config0", "large", "serve", "mixed", "queries", "case"])
    ap.add_argument("--sources", type=int, default=0, help="case: build sources [0, N)")
    ap.add_argument("--blocks", type=int, default=0, help="case: build kernel blocks (0 = as many as fit)")
    ap.add_argument("--sssd-batch", type=int, default=2048, help="queries: SSSD batch size")
    ap.add_argument("--msad-batch", type=int, default=96, help="queries: MSAD batch size")
    ap.add_argument("--single", type=int, default=8, help="queries: one-query launches timed per kind")
    ap.add_argument("--build-rate", type=float, default=2.0, help="mixed: build requests per s")
    ap.add_argument("--scale", type=float, default=1.0, help="large/serve: grid scale of the 750K torus")
    ap.add_argument("--K", default="100,500", help="large: build K values")
    ap.add_argument("--hbm-budget-gb", type=float, default=40.0)
    ap.add_argument("--plain-frac", type=float, default=0.02, help="large: share of sources built plain")
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--duration", type=float, default=60.0)
    ap.add_argument("--lanes", type=int, default=0, help="serve: 0 = one lane per resident query cluster")
    ap.add_argument("--max-batch", type=int, default=4, help="serve: SSSD requests per batch")
    ap.add_argument("--max-batch-msad", type=int, default=1, help="serve: MSAD requests per batch")
    ap.add_argument("--slots", type=int, default=0, help="serve: queries a lane serves at once (0 = auto)")
    ap.add_argument("--cluster", type=int, default=0, help="serve: blocks per query (0 auto, -1 one block)")
    ap.add_argument("--staging-out-mb", type=int, default=64)
    ap.add_argument("--ring", type=int, default=256)
    ap.add_argument("--plain-requests", type=int, default=400)
    ap.add_argument("--plain-seconds", type=float, default=30.0)
    ap.add_argument("--record", default="", help="also write the JSON line to this file")
    ap.add_argument("--no-autotune", action="store_true", help="time the default schedule, not the tuned one")
    ap.add_argument("--no-graph", action="store_true", help="timed builds without the captured CUDA graph")
    ap.add_argument("--mixed-heavy-first", type=int, default=-1,
                    help="mixed: heavy_first of the served builds (-1 = the library default)")
    ap.add_argument("--e2e-heavy-first", type=int, default=-1,
                    help="e2e: heavy_first of the fresh-mesh build (-1 = the library default)")
    ap.add_argument("--replicas", action="store_true",
                    help="N > 1: N whole builds (weak scaling) instead of one build sharded by source range")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "config0":
        return run_config0(args)
    if args.workload == "large":
        return run_large(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "mixed":
        return run_mixed(args)
    if args.workload == "queries":
        return run_queries(args)
    if args.workload == "case":
        return run_case(args)

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

    # N > 1: every rank builds a contiguous source range and the CSR slices
    # are all-gathered over NCCL (strong scaling); --replicas instead runs N
    # whole builds (weak scaling, no collective)
    shard = ws > 1 and not args.replicas
    V = mesh.vertNum
    sb, se = shard_ranges(V, ws)[rank] if shard else (0, V)

    def gather_slices():
        """Device time (ms) of the all-gather of this rank's CSR slice; every
        rank ends up holding the whole graph."""
        P = C.c_void_p
        o, a, d = P(), P(), P()
        L.svg_graph_device_csr(svg._g, C.byref(o), C.byref(a), C.byref(d))
        nnz = svg.counts()[1]
        off_t = device_view(o.value, V + 1, "<i8")
        deg = (off_t[sb + 1:se + 1] - off_t[sb:se]).to(torch.int32)
        adj_t = device_view(a.value, nnz, "<i4")
        w_t = device_view(d.value, nnz, "<f8")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        gather_csr(dist, deg, adj_t, w_t, device="cuda")
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1)

    def timed_build(mode=MODE_BATCHED, sharded=shard):
        flush_l2()
        a = C.c_double()
        L.svg_timer_mark(C.byref(a))
        # repeated builds of the resident mesh replay the build captured as a
        # CUDA graph by the first (warm-up) build; the plain form is not captured
        gr = int(mode == MODE_BATCHED and not args.no_graph)
        if sharded:
            st = svg.ConstructSVG(mode=mode, source_begin=sb, source_end=se, autotune=int(tune), graph=gr)
        else:
            st = svg.ConstructSVG(mode=mode, autotune=int(tune), graph=gr)
        b = C.c_double()
        L.svg_timer_mark(C.byref(b))
        ms = b.value
        if sharded:
            ms += gather_slices()
        return ms, st

    # untimed: the autotuner times candidate schedules of this build (the
    # graph is the same for all of them) and caches the fastest on the mesh
    tune = not args.no_autotune
    tuned = None
    if tune:
        t0 = time.perf_counter()
        kw = dict(source_begin=sb, source_end=se) if shard else {}
        best, best_ms = svg.autotune(max_trials=16, **kw)
        tuned = {"params": {k: best[k] for k in ("coop_sources", "coop_warps", "blocks", "vote_wait",
                                                 "heavy_waves", "heap_factor", "coop_tail")},
                 "tuned_build_ms": best_ms, "tuning_s": time.perf_counter() - t0}
    for _ in range(args.warmup):
        timed_build()
    barrier(dist)
    torch.cuda.synchronize()
    clocks = Clocks(smi_index(local))
    clocks.start()
    times, kern, edges, launches, replayed = [], [], 0, 0, 0
    st = None
    for _ in range(args.steps):
        ms, st = timed_build()
        times.append(ms)
        kern.append(st["ms_total"])
        edges += st["edges"]
        launches += st["launches"]
        replayed += st["graph_replayed"]
    torch.cuda.synchronize()
    barrier(dist)
    ck = clocks.stop()
    total_ms = sum(times)
    total_ms_max = max_over_ranks(dist, total_ms)
    value = replica_value(dist, float(edges), total_ms)
    edges_per_build = sum_over_ranks(dist, float(st["edges"])) if shard else st["edges"]
    windows_per_build = sum_over_ranks(dist, float(st["windows"])) if shard else st["windows"]

    # ---- end to end through the C ABI from host buffers: the step's inputs in
    # pinned host memory, the CSR read back into pinned host buffers allocated
    # once (as a service reusing its output buffers would)
    def pinned(n, dtype):
        return torch.empty(int(n), dtype=dtype, pin_memory=True).numpy()

    posc = pinned(pos.size, torch.float64)
    posc[:] = pos.reshape(-1)
    facc = pinned(faces.size, torch.int32)
    facc[:] = faces.reshape(-1)
    _, nnz0, _ = svg.counts()
    out_bufs = (pinned(len(pos) + 1, torch.int64), pinned(nnz0 + 1024, torch.int32),
                pinned(nnz0 + 1024, torch.float64))
    e2e_ms, e2e_edges, h2d, d2h = [], 0, 0, 0
    parts = {"mesh_build_upload": [], "build_call": [], "build_device": [], "csr_to_host": []}
    for i in range(args.warmup + args.steps):
        flush_l2()
        a = C.c_double()
        L.svg_timer_mark(C.byref(a))
        t0 = time.perf_counter()
        m2 = Mesh.from_arrays(posc, facc)
        m2.copyToGPU()
        t1 = time.perf_counter()
        s2 = SVG()
        s2.AssignMesh(m2)
        s2.SetParameters(K_BUILD, 10, 2)
        kw = {} if args.e2e_heavy_first < 0 else {"heavy_first": args.e2e_heavy_first}
        st2 = s2.ConstructSVG(source_begin=sb, source_end=se, **kw) if shard else s2.ConstructSVG(**kw)
        t2 = time.perf_counter()
        off, adj, dist_h = s2.csr(out=out_bufs)
        b = C.c_double()
        L.svg_timer_mark(C.byref(b))
        t3 = time.perf_counter()
        wall = (t3 - t0) * 1e3
        if i >= args.warmup:
            parts["mesh_build_upload"].append((t1 - t0) * 1e3)
            parts["build_call"].append((t2 - t1) * 1e3)
            parts["build_device"].append(st2["ms_total"])
            parts["csr_to_host"].append((t3 - t2) * 1e3)
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
            ms_p, stp = timed_build(MODE_PLAIN, sharded=False)
            plain = {"build_ms": ms_p, "edges_per_s": stp["edges"] / (ms_p / 1e3),
                     "speedup_batched_vs_plain": (ms_p / (total_ms_max / args.steps)), "grid": "64x128",
                     "windows": stp["windows"], "gpus": 1}
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
            "scaling": "strong" if shard else "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(WORKLOAD, l2="flushed between steps (256 MiB write)",
                           parallelism=(f"shard{ws}: contiguous source ranges, CSR slices all-gathered over NCCL"
                                        if shard else f"replicas{ws}"),
                           edges_per_build=edges_per_build, windows_per_build=windows_per_build,
                           work_order="timed steps: the autotuned schedule (untimed tuning before the warm-up; "
                                      "heaviest sources first, the heaviest on whole warps, by the per-source "
                                      "costs the earlier builds recorded); e2e: a fresh mesh every step with the "
                                      "default options (no cost record yet: on this mesh, under 4 sources per lane at "
                                      "K >= 160, a K/10 probe build orders the sources; the warps that are "
                                      "left with one running lane adopt it)"),
            "build_s": total_ms_max / args.steps / 1e3,
            "kernel_ms_per_step": statistics.mean(kern),
            "roofline": roofline_figures(st, peaks, fma_rate()),
            "cpu_baseline": cpu,
            "plain": plain,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_max / args.steps,
                    "breakdown_ms_mean": {k: round(statistics.mean(v), 2) for k, v in parts.items() if v},
                    "note": "build_call = the svg_build call's wall time (host set-up, device build, CSR "
                            "allocation); build_device = its CUDA-event time"},
            "gpu_launches": launches,
            "autotune": tuned,
            "graph_replayed_steps": replayed,
            "coop": {"sources": st["coop_sources"], "warps": st["coop_warps"]},
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
