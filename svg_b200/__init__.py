"""svg_b200: B200-native Saddle Vertex Graph geodesics (Python host binding).

A thin ctypes layer over the C ABI of libsvg_b200.so (include/svg_b200.h)
that mirrors the reference's host classes (Mesh.cuh:33-52, SVG.cuh:18-113):

    mesh = Mesh.LoadFromFile("bunny.obj")        # Mesh::LoadFromFile
    svg = SVG(); svg.AssignMesh(mesh)             # SVG::AssignMesh
    svg.SetParameters(100, 10, 2)                 # SVG::SetParameters(K, split, vert)
    svg.ConstructSVG()                            # SVG::ConstructSVG (on the GPU)
    offsets, nodes = svg.CopySVGToHost()          # SVG::CopySVGToHost
    svg.SaveSVGToFile("bunny.svg")                # SVG::SaveSVGToFile (same format)
    d = svg.SolveSSSD(s, t)                       # SVG::SolveSSSD
    dist, src = svg.SolveMSAD(srcs, weights)      # SVG::SolveMSAD

All compute runs on the GPU through the native library; there is no CPU
fallback: if the library cannot be loaded, importing a class that needs it
raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = ["Mesh", "SVG", "BuildOptions", "SvgError", "lib", "NODE_DTYPE", "LIB_PATH",
           "MODE_BATCHED", "MODE_PLAIN", "QUERY_CLUSTER", "QUERY_PLAIN", "Server", "ServerOptions"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SVG_B200_LIB") or os.path.join(HERE, "libsvg_b200.so")
MODE_BATCHED, MODE_PLAIN = 0, 1
QUERY_CLUSTER, QUERY_PLAIN = 0, 1
DBL_MAX = np.finfo(np.float64).max

# svg_node: the reference's SVGNode layout (SVG.cuh:21-27), 40 bytes
NODE_DTYPE = np.dtype([
    ("adj", np.int32), ("pad", np.int32), ("dist", np.float64),
    ("src_edge", np.uint32), ("dst_edge", np.uint32),
    ("src_x", np.float64), ("dst_x", np.float64),
])

STATUS = {0: "ok", 1: "bad argument", 2: "io", 3: "cuda", 4: "out of memory", 5: "mesh", 6: "state"}


class SvgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"svg_b200 error {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


class BuildOptions(C.Structure):
    _fields_ = [
        ("K", C.c_int32), ("split_coef", C.c_uint32), ("vert_coef", C.c_uint32),
        ("win_queue_cap", C.c_int32), ("pseudo_queue_cap", C.c_int32), ("mode", C.c_int32),
        ("threads_per_block", C.c_int32), ("blocks", C.c_int32), ("with_paths", C.c_int32),
        ("heavy_first", C.c_int32), ("hbm_budget", C.c_int64),
        ("source_begin", C.c_int32), ("source_end", C.c_int32),
        ("coop_sources", C.c_int32), ("coop_warps", C.c_int32), ("vote_wait", C.c_int32),
        ("heavy_waves", C.c_int32), ("heap_factor", C.c_int32), ("autotune", C.c_int32),
        ("coop_tail", C.c_int32), ("graph", C.c_int32),
    ]


class BuildStats(C.Structure):
    _fields_ = [
        ("ms_total", C.c_double), ("ms_ich", C.c_double), ("ms_emit", C.c_double),
        ("windows", C.c_int64), ("windows_generated", C.c_int64), ("pseudo_sources", C.c_int64),
        ("edges", C.c_int64), ("sources", C.c_int32), ("max_win_queue", C.c_int32),
        ("max_pseudo_queue", C.c_int32), ("queue_drop_sources", C.c_int32),
        ("ref_overflow_sources", C.c_int32), ("watchdog_sources", C.c_int32),
        ("undefined_sources", C.c_int32), ("retried_sources", C.c_int32), ("launches", C.c_int32),
        ("scratch_bytes", C.c_int64), ("coop_sources", C.c_int32), ("coop_warps", C.c_int32),
        ("graph_replayed", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerOptions(C.Structure):
    _fields_ = [("hbm_budget", C.c_int64), ("lanes", C.c_int32), ("max_batch", C.c_int32),
                ("slots_per_lane", C.c_int32), ("cluster", C.c_int32), ("staging_in_bytes", C.c_int64),
                ("staging_out_bytes", C.c_int64), ("max_batch_msad", C.c_int32), ("build_blocks_per_sm", C.c_int32)]


class ServerResult(C.Structure):
    _fields_ = [("ticket", C.c_int64), ("status", C.c_int32), ("kind", C.c_int32), ("graph_id", C.c_int32),
                ("n", C.c_int32), ("latency_ms", C.c_double), ("dist", C.c_double), ("edges", C.c_int64),
                ("build_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("pending", C.c_int64), ("batches", C.c_int64), ("batched_requests", C.c_int64),
                ("resident_bytes", C.c_int64), ("evictions", C.c_int64), ("rebuilds", C.c_int64),
                ("resident_graphs", C.c_int64)]


_P = C.c_void_p
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

# every symbol include/svg_b200.h declares
EXPORTS = [
    "svg_last_error", "svg_version", "svg_mesh_load_obj", "svg_mesh_from_arrays", "svg_mesh_upload",
    "svg_mesh_free", "svg_mesh_counts", "svg_mesh_export", "svg_build_opts_default", "svg_build",
    "svg_graph_stats", "svg_graph_source_stats", "svg_graph_free", "svg_graph_counts", "svg_graph_copy_csr",
    "svg_graph_copy_nodes", "svg_graph_device_csr", "svg_graph_save", "svg_graph_load", "svg_sssd_batch",
    "svg_msad_batch", "svg_sssd_batch_device", "svg_msad_batch_device", "svg_timer_mark",
    "svg_build_rows_static", "svg_trim_device_cache",
    "svg_server_opts_default", "svg_server_create", "svg_server_free", "svg_server_add_graph",
    "svg_server_submit_build", "svg_server_submit_sssd", "svg_server_submit_msad", "svg_server_wait",
    "svg_server_poll", "svg_server_take", "svg_server_stats", "svg_server_submit_msad_into",
    "svg_device_memory", "svg_graph_set_query_form", "svg_server_resident",
    "svg_msad_batch_paths", "svg_sssd_path", "svg_device_fp64_rate", "svg_build_autotune",
]

_lib = None


def lib() -> C.CDLL:
    """Load libsvg_b200.so (built by svg_b200/build_ext.py).  Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"native library missing: {LIB_PATH} (run python -m svg_b200.build_ext)")
    L = C.CDLL(LIB_PATH)
    L.svg_last_error.restype = C.c_char_p
    L.svg_version.restype = C.c_char_p
    L.svg_mesh_load_obj.argtypes = [C.c_char_p, C.POINTER(_P)]
    L.svg_mesh_from_arrays.argtypes = [C.c_int32, _f64p, C.c_int32, _i32p, C.POINTER(_P)]
    L.svg_mesh_upload.argtypes = [_P]
    L.svg_mesh_free.argtypes = [_P]
    L.svg_mesh_free.restype = None
    L.svg_mesh_counts.argtypes = [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.svg_mesh_export.argtypes = [_P] + [_P] * 6
    L.svg_build_opts_default.argtypes = [C.POINTER(BuildOptions)]
    L.svg_build_opts_default.restype = None
    L.svg_build.argtypes = [_P, C.POINTER(BuildOptions), C.POINTER(_P)]
    L.svg_build_autotune.argtypes = [_P, C.POINTER(BuildOptions), C.c_int32, C.POINTER(BuildOptions),
                                     C.POINTER(C.c_double)]
    L.svg_graph_stats.argtypes = [_P, C.POINTER(BuildStats)]
    L.svg_graph_source_stats.argtypes = [_P, _P, _P, _P]
    L.svg_graph_free.argtypes = [_P]
    L.svg_graph_free.restype = None
    L.svg_graph_counts.argtypes = [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    L.svg_graph_copy_csr.argtypes = [_P, _P, _P, _P]
    L.svg_graph_copy_nodes.argtypes = [_P, _P, _P]
    L.svg_graph_device_csr.argtypes = [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]
    L.svg_graph_save.argtypes = [_P, C.c_char_p]
    L.svg_graph_load.argtypes = [_P, C.c_int32, C.c_char_p, C.POINTER(_P)]
    L.svg_sssd_batch.argtypes = [_P, C.c_int32, _i32p, _i32p, _f64p]
    L.svg_msad_batch.argtypes = [_P, C.c_int32, _i64p, _P, _P, _f64p, _P]
    L.svg_msad_batch_paths.argtypes = [_P, C.c_int32, _i64p, _P, _P, _f64p, _P, _P]
    L.svg_sssd_path.argtypes = [_P, C.c_int32, C.c_int32, C.c_int32, _P, _P, C.POINTER(C.c_int32),
                                C.POINTER(C.c_double)]
    L.svg_sssd_batch_device.argtypes = [_P, C.c_int32, _P, _P, _P]
    L.svg_msad_batch_device.argtypes = [_P, C.c_int32, _P, _P, _P, _P, _P]
    L.svg_timer_mark.argtypes = [C.POINTER(C.c_double)]
    L.svg_device_fp64_rate.argtypes = [C.POINTER(C.c_double)]
    L.svg_build_rows_static.argtypes = [_P, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, _P]
    L.svg_trim_device_cache.restype = C.c_size_t
    L.svg_server_opts_default.argtypes = [C.POINTER(ServerOptions)]
    L.svg_server_opts_default.restype = None
    L.svg_server_create.argtypes = [C.POINTER(ServerOptions), C.POINTER(_P)]
    L.svg_server_free.argtypes = [_P]
    L.svg_server_free.restype = None
    L.svg_server_add_graph.argtypes = [_P, _P, C.POINTER(C.c_int32)]
    L.svg_server_submit_build.argtypes = [_P, _P, C.POINTER(BuildOptions), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    L.svg_server_submit_sssd.argtypes = [_P, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int64)]
    L.svg_server_submit_msad.argtypes = [_P, C.c_int32, C.c_int32, _P, _P, C.POINTER(C.c_int64)]
    L.svg_server_submit_msad_into.argtypes = [_P, C.c_int32, C.c_int32, _P, _P, _P, _P, C.POINTER(C.c_int64)]
    L.svg_device_memory.argtypes = [C.POINTER(C.c_int64)] * 3 + [C.c_int32]
    L.svg_device_memory.restype = None
    L.svg_graph_set_query_form.argtypes = [_P, C.c_int32]
    L.svg_server_resident.argtypes = [_P, C.c_int32, _P, C.POINTER(C.c_int32)]
    L.svg_server_wait.argtypes = [_P, C.c_int64, C.c_double, C.POINTER(ServerResult)]
    L.svg_server_poll.argtypes = [_P, C.c_int32, _P, C.POINTER(C.c_int32)]
    L.svg_server_take.argtypes = [_P, C.c_int64, _P, _P]
    L.svg_server_stats.argtypes = [_P, C.POINTER(ServerStats)]
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != 0:
        raise SvgError(rc, lib().svg_last_error().decode(errors="replace"))


class Mesh:
    """Half-edge triangle mesh (reference Mesh, Mesh.cuh:33-52)."""

    def __init__(self, handle):
        self._h = handle
        nv, nf, ne = C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().svg_mesh_counts(handle, C.byref(nv), C.byref(nf), C.byref(ne)))
        self.vertNum, self.faceNum, self.edgeNum = nv.value, nf.value, ne.value

    @classmethod
    def LoadFromFile(cls, path: str) -> "Mesh":
        h = _P()
        _check(lib().svg_mesh_load_obj(os.fsencode(path), C.byref(h)))
        return cls(h)

    @classmethod
    def from_arrays(cls, pos, faces) -> "Mesh":
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        faces = np.ascontiguousarray(faces, np.int32).reshape(-1)
        h = _P()
        _check(lib().svg_mesh_from_arrays(len(pos) // 3, pos, len(faces) // 3, faces, C.byref(h)))
        return cls(h)

    def copyToGPU(self) -> None:
        _check(lib().svg_mesh_upload(self._h))

    def clear(self) -> None:
        if self._h:
            lib().svg_mesh_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.clear()
        except Exception:
            pass

    def export(self) -> dict:
        V, E = self.vertNum, self.edgeNum
        out = dict(he_v0=np.zeros(E, np.int32), he_twin=np.zeros(E, np.int32), he_len=np.zeros(E),
                   pos=np.zeros((V, 3)), angle=np.zeros(V), first_edge=np.zeros(V, np.int32))
        _check(lib().svg_mesh_export(self._h, *[out[k].ctypes.data_as(_P) for k in
                                                ["he_v0", "he_twin", "he_len", "pos", "angle", "first_edge"]]))
        return out


class SVG:
    """Saddle Vertex Graph on the device (reference SVG, SVG.cuh:18-113)."""

    def __init__(self):
        self.mesh: Mesh | None = None
        self.K = 100
        self.splitInfoCoef = 10
        self.vertInfoCoef = 2
        self._g = None
        self.options = BuildOptions()
        lib().svg_build_opts_default(C.byref(self.options))

    # ---- reference method names
    def AssignMesh(self, mesh: Mesh, d_mesh=None) -> None:
        self.mesh = mesh

    def SetParameters(self, K: int, splitInfoCoef: int = 10, vertInfoCoef: int = 2) -> None:
        self.K, self.splitInfoCoef, self.vertInfoCoef = int(K), int(splitInfoCoef), int(vertInfoCoef)

    def Allocation(self) -> bool:
        """Scratch is allocated inside ConstructSVG; kept for API parity."""
        return True

    def Free(self) -> None:
        """Build scratch is released by the library; kept for API parity."""

    def ConstructSVG(self, mode: int = MODE_BATCHED, with_paths: bool = True, **kw) -> dict:
        if self.mesh is None:
            raise SvgError(6, "AssignMesh first")
        self.FreeSVGStructure()
        o = BuildOptions()
        lib().svg_build_opts_default(C.byref(o))
        o.K, o.split_coef, o.vert_coef = self.K, self.splitInfoCoef, self.vertInfoCoef
        o.mode = mode
        o.with_paths = int(with_paths)
        for k, v in kw.items():
            setattr(o, k, v)
        self.options = o
        h = _P()
        _check(lib().svg_build(self.mesh._h, C.byref(o), C.byref(h)))
        self._g = h
        return self.stats()

    def autotune(self, max_trials: int = 16, **kw) -> tuple:
        """svg_build_autotune: time candidate schedules of the batched build of
        this mesh at K, cache the fastest on the mesh (later ConstructSVG calls
        with autotune=1 use it).  Returns (chosen options as a dict, build ms)."""
        if self.mesh is None:
            raise SvgError(6, "AssignMesh first")
        o = BuildOptions()
        lib().svg_build_opts_default(C.byref(o))
        o.K, o.split_coef, o.vert_coef = self.K, self.splitInfoCoef, self.vertInfoCoef
        for k, v in kw.items():
            setattr(o, k, v)
        best = BuildOptions()
        ms = C.c_double()
        _check(lib().svg_build_autotune(self.mesh._h, C.byref(o), int(max_trials), C.byref(best), C.byref(ms)))
        return {f: getattr(best, f) for f, _ in BuildOptions._fields_}, ms.value

    def FreeSVGStructure(self) -> None:
        if self._g:
            lib().svg_graph_free(self._g)
            self._g = None

    def __del__(self):
        try:
            self.FreeSVGStructure()
        except Exception:
            pass

    def stats(self) -> dict:
        st = BuildStats()
        _check(lib().svg_graph_stats(self._g, C.byref(st)))
        return st.as_dict()

    def source_stats(self):
        V = self.mesh.vertNum
        w, q, f = np.zeros(V, np.int32), np.zeros(V, np.int32), np.zeros(V, np.int32)
        _check(lib().svg_graph_source_stats(self._g, w.ctypes.data_as(_P), q.ctypes.data_as(_P),
                                            f.ctypes.data_as(_P)))
        return w, q, f

    def counts(self):
        nv, nnz, K = C.c_int32(), C.c_int64(), C.c_int32()
        _check(lib().svg_graph_counts(self._g, C.byref(nv), C.byref(nnz), C.byref(K)))
        return nv.value, nnz.value, K.value

    def csr(self, out=None):
        """(offsets[V+1] int64, adj[nnz] int32, dist[nnz] float64) on the host;
        out=(off, adj, dist) reuses caller arrays (e.g. pinned) of at least that size."""
        nv, nnz, _ = self.counts()
        if out is not None:
            off, adj, dist = out
            assert off.dtype == np.int64 and adj.dtype == np.int32 and dist.dtype == np.float64
            assert len(off) >= nv + 1 and len(adj) >= nnz and len(dist) >= nnz
            _check(lib().svg_graph_copy_csr(self._g, off.ctypes.data_as(_P), adj.ctypes.data_as(_P),
                                            dist.ctypes.data_as(_P)))
            return off[:nv + 1], adj[:nnz], dist[:nnz]
        off = np.zeros(nv + 1, np.int64)
        adj = np.zeros(max(nnz, 1), np.int32)
        dist = np.zeros(max(nnz, 1))
        _check(lib().svg_graph_copy_csr(self._g, off.ctypes.data_as(_P), adj.ctypes.data_as(_P),
                                        dist.ctypes.data_as(_P)))
        return off, adj[:nnz], dist[:nnz]

    def CopySVGToHost(self):
        """(offsets, nodes): reference-layout rows packed in CSR order."""
        nv, nnz, _ = self.counts()
        tails = np.zeros(nv, np.int32)
        nodes = np.zeros(max(nnz, 1), NODE_DTYPE)
        _check(lib().svg_graph_copy_nodes(self._g, tails.ctypes.data_as(_P), nodes.ctypes.data_as(_P)))
        off = np.zeros(nv + 1, np.int64)
        np.cumsum(tails, out=off[1:])
        return off, nodes[:nnz]

    def SaveSVGToFile(self, path: str) -> None:
        _check(lib().svg_graph_save(self._g, os.fsencode(path)))

    def LoadSVGFromFile(self, path: str) -> None:
        self.FreeSVGStructure()
        h = _P()
        _check(lib().svg_graph_load(self.mesh._h, self.K, os.fsencode(path), C.byref(h)))
        self._g = h

    # ---- queries
    def set_query_form(self, form: int) -> None:
        """QUERY_CLUSTER (default) or QUERY_PLAIN (one block per query)."""
        _check(lib().svg_graph_set_query_form(self._g, int(form)))

    def sssd_batch(self, s, t) -> np.ndarray:
        s = np.ascontiguousarray(s, np.int32)
        t = np.ascontiguousarray(t, np.int32)
        d = np.zeros(len(s))
        _check(lib().svg_sssd_batch(self._g, len(s), s, t, d))
        return d

    def SolveSSSD(self, s: int, t: int) -> float:
        return float(self.sssd_batch([s], [t])[0])

    def msad_batch(self, sets, weights=None, with_src: bool = True):
        """sets: list of source-id arrays; weights: list of weight arrays (default 0)."""
        V = self.mesh.vertNum
        n = len(sets)
        off = np.zeros(n + 1, np.int64)
        np.cumsum([len(x) for x in sets], out=off[1:])
        srcs = np.ascontiguousarray(np.concatenate(sets) if n else np.zeros(0), np.int32)
        if weights is None:
            w = np.zeros(len(srcs))
        else:
            w = np.ascontiguousarray(np.concatenate(weights) if n else np.zeros(0), np.float64)
        dist = np.zeros(n * V)
        sid = np.zeros(n * V, np.int32) if with_src else None
        _check(lib().svg_msad_batch(self._g, n, off, srcs.ctypes.data_as(_P), w.ctypes.data_as(_P), dist,
                                    sid.ctypes.data_as(_P) if with_src else None))
        dist = dist.reshape(n, V)
        return (dist, sid.reshape(n, V)) if with_src else dist

    def msad_paths(self, sets, weights=None):
        """msad_batch plus parent pointers (pathParentIndex): (dist, src, parent), each (n, V)."""
        V = self.mesh.vertNum
        n = len(sets)
        off = np.zeros(n + 1, np.int64)
        np.cumsum([len(x) for x in sets], out=off[1:])
        srcs = np.ascontiguousarray(np.concatenate(sets) if n else np.zeros(0), np.int32)
        w = np.zeros(len(srcs)) if weights is None else \
            np.ascontiguousarray(np.concatenate(weights) if n else np.zeros(0), np.float64)
        dist = np.zeros(n * V)
        sid = np.zeros(n * V, np.int32)
        par = np.zeros(n * V, np.int32)
        _check(lib().svg_msad_batch_paths(self._g, n, off, srcs.ctypes.data_as(_P), w.ctypes.data_as(_P), dist,
                                          sid.ctypes.data_as(_P), par.ctypes.data_as(_P)))
        return dist.reshape(n, V), sid.reshape(n, V), par.reshape(n, V)

    def sssd_path(self, s: int, t: int, cap: int = 1 << 16):
        """(vertices t ... s along pathParentIndex, their distances from s, the s-t distance)."""
        path = np.zeros(cap, np.int32)
        pd = np.zeros(cap)
        n = C.c_int32()
        d = C.c_double()
        _check(lib().svg_sssd_path(self._g, int(s), int(t), cap, path.ctypes.data_as(_P), pd.ctypes.data_as(_P),
                                   C.byref(n), C.byref(d)))
        return path[:n.value].copy(), pd[:n.value].copy(), d.value

    def SolveMSAD(self, sources, sourceWeights):
        d, s = self.msad_batch([np.asarray(sources)], [np.asarray(sourceWeights, np.float64)])
        return d[0], s[0]


class Server:
    """Serving loop over resident SVGs (svg_server_* in include/svg_b200.h):
    continuous batching of SSSD / MSAD requests on several CUDA streams,
    builds admitted under a device-memory budget with eviction and rebuild."""

    def __init__(self, **opts):
        self.opts = ServerOptions()
        lib().svg_server_opts_default(C.byref(self.opts))
        for k, v in opts.items():
            setattr(self.opts, k, v)
        h = _P()
        _check(lib().svg_server_create(C.byref(self.opts), C.byref(h)))
        self._h = h
        self._keep = []   # meshes/graphs the server refers to stay alive with it

    def close(self):
        if self._h:
            lib().svg_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_graph(self, svg: "SVG") -> int:
        gid = C.c_int32()
        _check(lib().svg_server_add_graph(self._h, svg._g, C.byref(gid)))
        self._keep.append(svg)
        return gid.value

    def submit_build(self, mesh: Mesh, K: int, **kw):
        o = BuildOptions()
        lib().svg_build_opts_default(C.byref(o))
        o.K = K
        for k, v in kw.items():
            setattr(o, k, v)
        gid, t = C.c_int32(), C.c_int64()
        _check(lib().svg_server_submit_build(self._h, mesh._h, C.byref(o), C.byref(gid), C.byref(t)))
        self._keep.append(mesh)
        return gid.value, t.value

    def submit_sssd(self, gid: int, s: int, t: int) -> int:
        tk = C.c_int64()
        _check(lib().svg_server_submit_sssd(self._h, gid, int(s), int(t), C.byref(tk)))
        return tk.value

    def submit_msad(self, gid: int, srcs, weights=None, out=None) -> int:
        """out=(dists, src_ids): float64 / int32 arrays of V entries (either None)
        that receive the result directly; they must outlive the request."""
        srcs = np.ascontiguousarray(srcs, np.int32)
        w = np.zeros(len(srcs)) if weights is None else np.ascontiguousarray(weights, np.float64)
        tk = C.c_int64()
        if out is None:
            _check(lib().svg_server_submit_msad(self._h, gid, len(srcs), srcs.ctypes.data_as(_P),
                                                w.ctypes.data_as(_P), C.byref(tk)))
        else:
            d, sid = out
            assert d is None or (d.dtype == np.float64 and d.flags.c_contiguous)
            assert sid is None or (sid.dtype == np.int32 and sid.flags.c_contiguous)
            _check(lib().svg_server_submit_msad_into(self._h, gid, len(srcs), srcs.ctypes.data_as(_P),
                                                     w.ctypes.data_as(_P),
                                                     None if d is None else d.ctypes.data_as(_P),
                                                     None if sid is None else sid.ctypes.data_as(_P), C.byref(tk)))
        return tk.value

    def wait(self, ticket: int, timeout: float = 600.0) -> dict:
        r = ServerResult()
        _check(lib().svg_server_wait(self._h, ticket, timeout, C.byref(r)))
        return {k: getattr(r, k) for k, _ in r._fields_}

    def take(self, ticket: int, nv: int = 0):
        """Release a finished request; for MSAD return (dists, src_ids) of length nv."""
        d = np.zeros(max(nv, 1))
        s = np.zeros(max(nv, 1), np.int32)
        _check(lib().svg_server_take(self._h, ticket, d.ctypes.data_as(_P) if nv else None,
                                     s.ctypes.data_as(_P) if nv else None))
        return (d[:nv], s[:nv]) if nv else None

    def poll(self, max_n: int = 4096) -> list:
        arr = (ServerResult * max_n)()
        n = C.c_int32()
        _check(lib().svg_server_poll(self._h, max_n, C.cast(arr, _P), C.byref(n)))
        return [{k: getattr(arr[i], k) for k, _ in ServerResult._fields_} for i in range(n.value)]

    _POLL_DT = np.dtype([("ticket", np.int64), ("status", np.int32), ("kind", np.int32), ("graph_id", np.int32),
                         ("n", np.int32), ("latency_ms", np.float64), ("dist", np.float64), ("edges", np.int64),
                         ("build_ms", np.float64)], align=True)

    def poll_array(self, max_n: int = 4096) -> np.ndarray:
        """svg_server_poll into a numpy structured array (the ServerResult
        fields), without a Python object per field: for callers that drain
        thousands of results a second."""
        assert self._POLL_DT.itemsize == C.sizeof(ServerResult)
        out = np.empty(max_n, self._POLL_DT)
        n = C.c_int32()
        _check(lib().svg_server_poll(self._h, max_n, out.ctypes.data_as(_P), C.byref(n)))
        return out[:n.value]

    def resident(self, max_n: int = 4096) -> list:
        """Graph ids resident now, most recently used first."""
        ids = np.zeros(max_n, np.int32)
        n = C.c_int32()
        _check(lib().svg_server_resident(self._h, max_n, ids.ctypes.data_as(_P), C.byref(n)))
        return ids[:n.value].tolist()

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().svg_server_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}


def device_memory(reset_peak: bool = False) -> dict:
    """Device bytes held by the library: in use, high-water mark, cached for reuse."""
    a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
    lib().svg_device_memory(C.byref(a), C.byref(b), C.byref(c), 1 if reset_peak else 0)
    return {"in_use": a.value, "peak": b.value, "cached": c.value}
