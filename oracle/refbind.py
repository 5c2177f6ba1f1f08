"""ctypes access to the test oracles.  Test infrastructure only: imported by
tests/, the smoke check and bench.py's CPU-baseline leg, never by the product.

  RefOracle   oracle/_ref/libsvgref.so - the reference's own ICH (Mesh.cu,
              Geometry.cu, ICHDevice.cu compiled as host C++) driven by
              oracle/ref_driver.cpp.
  CpuOracle   oracle/_build/libsvgoracle.so - the plain-C restatement
              (oracle/svg_oracle.c) of the same algorithm.

Both return reference-layout results: per source a row of SVG nodes
(SVG::SVGNode, SVG.cuh:21-27: adj, dist, nextToSrcEdge, nextToDstEdge,
nextToSrcX, nextToDstX) in ascending adjacent-vertex order, at most K.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libsvgref.so")
ORACLE_LIB = os.path.join(HERE, "_build", "libsvgoracle.so")
DBL_MAX = np.finfo(np.float64).max

NODE_DTYPE = np.dtype([
    ("adj", np.int32), ("pad", np.int32), ("dist", np.float64),
    ("src_edge", np.uint32), ("dst_edge", np.uint32),
    ("src_x", np.float64), ("dst_x", np.float64),
])
assert NODE_DTYPE.itemsize == 40

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build_oracles(ref: bool = True) -> None:
    """Compile the C restatement (always) and the reference oracle (when the
    reference sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref:
        # the Makefile's REF names where the reference is checked out;
        # SVG_REFERENCE_DIR overrides it
        src = os.environ.get("SVG_REFERENCE_DIR")
        subprocess.run(["make", "-s", "-C", HERE, "ref"] + (["REF=" + src] if src else []), check=True)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


class SvgRows:
    """Rows of an SVG in reference layout: tails[r] nodes in nodes[r, :tails[r]]."""

    def __init__(self, tails: np.ndarray, nodes: np.ndarray, stats: np.ndarray | None, seconds: float):
        self.tails = tails
        self.nodes = nodes
        self.stats = stats
        self.seconds = seconds

    def row(self, r: int) -> np.ndarray:
        return self.nodes[r, : self.tails[r]]

    def to_csr(self):
        off = np.zeros(len(self.tails) + 1, np.int64)
        np.cumsum(self.tails, out=off[1:])
        flat = np.concatenate([self.row(r) for r in range(len(self.tails))]) if len(self.tails) else \
            np.zeros(0, NODE_DTYPE)
        return off, flat


class RefOracle:
    """The reference's own host-compiled ICH + restated emission loop."""

    def __init__(self, lib_path: str = REF_LIB):
        if not os.path.exists(lib_path):
            raise FileNotFoundError(f"reference oracle not built: {lib_path}")
        L = C.CDLL(lib_path)
        L.ref_mesh_load.restype = C.c_void_p
        L.ref_mesh_load.argtypes = [C.c_char_p, C.c_int]
        L.ref_mesh_free.argtypes = [C.c_void_p]
        L.ref_mesh_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ref_mesh_export.argtypes = [C.c_void_p] + [C.c_void_p] * 11
        L.ref_build.restype = C.c_double
        L.ref_build.argtypes = [C.c_void_p, C.c_int, C.c_uint, C.c_uint, C.c_int, C.c_int,
                                _i32p, C.c_int, C.c_int, _i32p, C.c_void_p, C.c_void_p]
        L.ref_ich_distances.restype = C.c_double
        L.ref_ich_distances.argtypes = [C.c_void_p, C.c_int, C.c_uint, C.c_uint, C.c_int, C.c_int,
                                        _i32p, C.c_int, C.c_int, _f64p, C.c_void_p]
        L.ref_sssd.restype = C.c_double
        L.ref_sssd.argtypes = [C.c_void_p, C.c_int, _i32p, C.c_void_p, C.c_int, _i32p, _i32p, _f64p, C.c_void_p]
        L.ref_msad.restype = C.c_double
        L.ref_msad.argtypes = [C.c_void_p, C.c_int, _i32p, C.c_void_p, C.c_int, _i32p, _f64p, _f64p, C.c_void_p]
        self.L = L

    # ---- mesh ----
    def load(self, obj_path: str, fix_boundary: bool = True) -> "RefMesh":
        h = self.L.ref_mesh_load(obj_path.encode(), int(fix_boundary))
        if not h:
            raise IOError(f"reference loader could not open {obj_path}")
        return RefMesh(self, h)


class RefMesh:
    def __init__(self, oracle: RefOracle, handle):
        self.o = oracle
        self.h = handle
        nv, nf, ne = C.c_int(), C.c_int(), C.c_int()
        oracle.L.ref_mesh_counts(handle, C.byref(nv), C.byref(nf), C.byref(ne))
        self.nv, self.nf, self.ne = nv.value, nf.value, ne.value

    def __del__(self):
        try:
            if self.h:
                self.o.L.ref_mesh_free(self.h)
                self.h = None
        except Exception:
            pass

    def export(self) -> dict:
        V, F, E = self.nv, self.nf, self.ne
        out = dict(pos=np.zeros((V, 3)), faces=np.zeros((F, 3), np.int32),
                   he_v0=np.zeros(E, np.int32), he_v1=np.zeros(E, np.int32),
                   he_twin=np.zeros(E, np.int32), he_next=np.zeros(E, np.int32),
                   he_prev=np.zeros(E, np.int32), he_face=np.zeros(E, np.int32),
                   he_len=np.zeros(E), angle=np.zeros(V), first_edge=np.zeros(V, np.int32))
        keys = ["pos", "faces", "he_v0", "he_v1", "he_twin", "he_next", "he_prev", "he_face",
                "he_len", "angle", "first_edge"]
        self.o.L.ref_mesh_export(self.h, *[out[k].ctypes.data_as(C.c_void_p) for k in keys])
        return out

    def build(self, K: int, sources=None, threads: int = 0, split_coef: int = 10, vert_coef: int = 2,
              win_cap: int = 1023, pseudo_cap: int = 1023, stats: bool = True) -> SvgRows:
        src = np.arange(self.nv, dtype=np.int32) if sources is None else np.ascontiguousarray(sources, np.int32)
        n = len(src)
        tails = np.zeros(n, np.int32)
        nodes = np.zeros((n, K), NODE_DTYPE)
        st = np.zeros((n, 4), np.int32) if stats else None
        secs = self.o.L.ref_build(self.h, K, split_coef, vert_coef, win_cap, pseudo_cap, src, n, threads,
                                  tails, nodes.ctypes.data_as(C.c_void_p),
                                  st.ctypes.data_as(C.c_void_p) if stats else None)
        return SvgRows(tails, nodes, st, secs)

    def ich_distances(self, sources, K: int = -1, split_size: int | None = None, vert_size: int | None = None,
                      win_cap: int = 1 << 22, pseudo_cap: int = 1 << 20, threads: int = 0):
        """Per-vertex ICH distances; K=-1 runs the exhaustive (exact) ICH."""
        src = np.ascontiguousarray(sources, np.int32)
        n = len(src)
        split_size = split_size or 10 * self.nv
        vert_size = vert_size or 2 * self.nv
        d = np.zeros(n * self.nv)
        st = np.zeros((n, 4), np.int32)
        secs = self.o.L.ref_ich_distances(self.h, K, split_size, vert_size, win_cap, pseudo_cap, src, n,
                                          threads, d, st.ctypes.data_as(C.c_void_p))
        return d.reshape(n, self.nv), st, secs

    def sssd(self, K: int, tails: np.ndarray, nodes_padded: np.ndarray, s, t):
        s = np.ascontiguousarray(s, np.int32)
        t = np.ascontiguousarray(t, np.int32)
        d = np.zeros(len(s))
        secs = self.o.L.ref_sssd(self.h, K, np.ascontiguousarray(tails, np.int32),
                                 nodes_padded.ctypes.data_as(C.c_void_p), len(s), s, t, d, None)
        return d, secs

    def msad(self, K: int, tails: np.ndarray, nodes_padded: np.ndarray, srcs, weights):
        srcs = np.ascontiguousarray(srcs, np.int32)
        w = np.ascontiguousarray(weights, np.float64)
        d = np.zeros(self.nv)
        sid = np.zeros(self.nv, np.int32)
        secs = self.o.L.ref_msad(self.h, K, np.ascontiguousarray(tails, np.int32),
                                 nodes_padded.ctypes.data_as(C.c_void_p), len(srcs), srcs, w, d,
                                 sid.ctypes.data_as(C.c_void_p))
        return d, sid, secs


class CpuOracle:
    """The plain-C restatement (oracle/svg_oracle.c)."""

    def __init__(self, lib_path: str = ORACLE_LIB):
        if not os.path.exists(lib_path):
            raise FileNotFoundError(f"C oracle not built: {lib_path}")
        L = C.CDLL(lib_path)
        L.om_mesh_create.restype = C.c_int
        L.om_mesh_create.argtypes = [C.c_int, _f64p, C.c_int, _i32p, C.POINTER(C.c_void_p)]
        L.om_mesh_free.argtypes = [C.c_void_p]
        L.om_mesh_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.om_mesh_export.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        L.om_build.restype = C.c_double
        L.om_build.argtypes = [C.c_void_p, C.c_int, C.c_uint, C.c_uint, C.c_int, C.c_int, _i32p, C.c_int,
                               C.c_int, _i32p, C.c_void_p, C.c_void_p]
        L.om_ich_distances.restype = C.c_double
        L.om_ich_distances.argtypes = [C.c_void_p, C.c_int, C.c_uint, C.c_uint, C.c_int, C.c_int, _i32p,
                                       C.c_int, C.c_int, _f64p, C.c_void_p]
        _i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
        L.om_sssd.restype = C.c_double
        L.om_sssd.argtypes = [C.c_void_p, _i64p, _i32p, _f64p, C.c_int, _i32p, _i32p, _f64p]
        L.om_msad.restype = C.c_double
        L.om_msad.argtypes = [C.c_void_p, _i64p, _i32p, _f64p, C.c_int, _i32p, _f64p, _f64p, C.c_void_p]
        self.L = L

    def mesh(self, pos: np.ndarray, faces: np.ndarray) -> "CpuMesh":
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        faces = np.ascontiguousarray(faces, np.int32).reshape(-1)
        h = C.c_void_p()
        rc = self.L.om_mesh_create(len(pos) // 3, pos, len(faces) // 3, faces, C.byref(h))
        if rc != 0:
            raise RuntimeError("om_mesh_create failed")
        return CpuMesh(self, h.value, pos.reshape(-1, 3))


class CpuMesh:
    def __init__(self, oracle: CpuOracle, handle, pos):
        self.o = oracle
        self.h = handle
        self.pos = pos
        nv, nf, ne = C.c_int(), C.c_int(), C.c_int()
        oracle.L.om_mesh_counts(handle, C.byref(nv), C.byref(nf), C.byref(ne))
        self.nv, self.nf, self.ne = nv.value, nf.value, ne.value

    def __del__(self):
        try:
            if self.h:
                self.o.L.om_mesh_free(self.h)
                self.h = None
        except Exception:
            pass

    def export(self) -> dict:
        out = dict(he_v0=np.zeros(self.ne, np.int32), he_twin=np.zeros(self.ne, np.int32),
                   he_len=np.zeros(self.ne), angle=np.zeros(self.nv), first_edge=np.zeros(self.nv, np.int32))
        self.o.L.om_mesh_export(self.h, *[out[k].ctypes.data_as(C.c_void_p)
                                          for k in ["he_v0", "he_twin", "he_len", "angle", "first_edge"]])
        return out

    def build(self, K: int, sources=None, threads: int = 0, split_coef: int = 10, vert_coef: int = 2,
              win_cap: int = 1023, pseudo_cap: int = 1023) -> SvgRows:
        src = np.arange(self.nv, dtype=np.int32) if sources is None else np.ascontiguousarray(sources, np.int32)
        n = len(src)
        tails = np.zeros(n, np.int32)
        nodes = np.zeros((n, max(K, 1)), NODE_DTYPE)
        st = np.zeros((n, 5), np.int32)
        secs = self.o.L.om_build(self.h, K, split_coef, vert_coef, win_cap, pseudo_cap, src, n, threads, tails,
                                 nodes.ctypes.data_as(C.c_void_p), st.ctypes.data_as(C.c_void_p))
        return SvgRows(tails, nodes, st, secs)

    def ich_distances(self, sources, K: int = -1, split_size: int | None = None, vert_size: int | None = None,
                      win_cap: int = 1 << 22, pseudo_cap: int = 1 << 20, threads: int = 0):
        src = np.ascontiguousarray(sources, np.int32)
        n = len(src)
        d = np.zeros(n * self.nv)
        st = np.zeros((n, 5), np.int32)
        secs = self.o.L.om_ich_distances(self.h, K, split_size or 10 * self.nv, vert_size or 2 * self.nv,
                                         win_cap, pseudo_cap, src, n, threads, d, st.ctypes.data_as(C.c_void_p))
        return d.reshape(n, self.nv), st, secs

    def sssd(self, offsets, adj, w, s, t):
        s = np.ascontiguousarray(s, np.int32)
        d = np.zeros(len(s))
        secs = self.o.L.om_sssd(self.h, np.ascontiguousarray(offsets, np.int64), np.ascontiguousarray(adj, np.int32),
                                np.ascontiguousarray(w, np.float64), len(s), s,
                                np.ascontiguousarray(t, np.int32), d)
        return d, secs

    def msad(self, offsets, adj, w, srcs, weights):
        srcs = np.ascontiguousarray(srcs, np.int32)
        d = np.zeros(self.nv)
        sid = np.zeros(self.nv, np.int32)
        secs = self.o.L.om_msad(self.h, np.ascontiguousarray(offsets, np.int64), np.ascontiguousarray(adj, np.int32),
                                np.ascontiguousarray(w, np.float64), len(srcs), srcs,
                                np.ascontiguousarray(weights, np.float64), d, sid.ctypes.data_as(C.c_void_p))
        return d, sid, secs


def rows_equal(a: SvgRows, b: SvgRows) -> tuple[bool, str]:
    """Bit-exact comparison of two reference-layout SVG row sets."""
    if not np.array_equal(a.tails, b.tails):
        bad = np.nonzero(a.tails != b.tails)[0]
        return False, f"degree differs at rows {bad[:10].tolist()}"
    for r in range(len(a.tails)):
        x, y = a.row(r), b.row(r)
        for f in ("adj", "dist", "src_edge", "dst_edge", "src_x", "dst_x"):
            if not np.array_equal(x[f], y[f]):
                return False, f"row {r} field {f} differs"
    return True, "ok"
