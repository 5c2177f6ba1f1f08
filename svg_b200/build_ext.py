"""Compile the svg_b200 native library in-tree: svg_b200/libsvg_b200.so.

Device code targets sm_100a only and is compiled with --fmad=false: the
geometry must be the plain IEEE sequence of multiplies and adds that decides
the reference's branches, never a fused multiply-add.  Host code uses
-ffp-contract=off for the same reason (mesh precomputation).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsvg_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CU_SOURCES = ["api.cu", "build.cu", "query.cu", "serve.cu"]
CPP_SOURCES = ["mesh.cpp"]
HEADERS = ["svg_internal.h", "engine.h", "ich.cuh"]

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-v",
    "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
]
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra",
             "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "svg_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, log):
    r = subprocess.run(cmd, capture_output=True, text=True)
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"compile failed: {' '.join(cmd[:3])} ... (log {log})")
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False, out_dir: str = OUT_DIR, lib: str = LIB,
          defines: tuple = ()) -> str:
    """Compile (incrementally) into `lib`; `defines` are extra -D flags for the CUDA sources."""
    os.makedirs(out_dir, exist_ok=True)
    jobs = []
    objs = []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(out_dir, s + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append(([NVCC] + NVCC_FLAGS + ["-D" + d for d in defines] + ["-c", src, "-o", obj], obj + ".log"))
    for s in CPP_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(out_dir, s + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append((["g++"] + CXX_FLAGS + ["-c", src, "-o", obj], obj + ".log"))
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            outs = list(ex.map(lambda j: _run(*j), jobs))
        if verbose:
            for o in outs:
                sys.stdout.write(o)
    if jobs or force or not os.path.exists(lib):
        _run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", lib] + objs +
             ["-lcudart_static", "-lrt", "-lpthread", "-ldl"], os.path.join(out_dir, "link.log"))
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
