"""polymer_b200 -- Python binding of the B200 edgeMap/vertexMap engine.

The engine is libpolymer_b200.so (CUDA kernels for sm_100a behind the C ABI
in include/polymer_b200.h).  This module is a thin ctypes layer over that
ABI, named after the reference applications it replaces:

    g = Graph.from_csr(offsets, edges)            # readGraph (IO-numa.h:745)
    ranks = PageRank(g, maxIter=10)                # numa-PageRank.C:548
    parents, depth = BFS(src, g)                   # numa-BFS.C:476
    labels = Components(g)                         # numa-Components.C:402
    dist = BellmanFord(g, src)                     # numa-BellmanFord.C:400
    y = SPMV(g, x0, maxIter)                       # numa-SPMV.C:335
    logp = BeliefPropagation(g, prior, maxIter)    # numa-BP.C:528

Arrays are numpy (host) or any object exposing a CUDA pointer through
``data_ptr()`` (torch tensors).  There is no CPU fallback: without the
shared library or a GPU every call raises PolymerError.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = [
    "Graph", "PolymerError", "PageRank", "BFS", "BFSAsync", "BFSMulti", "Components", "BellmanFord",
    "BellmanFordMulti", "PageRankDelta", "SPMV",
    "BeliefPropagation", "TraversalStats", "lib", "LIB_PATH", "kernel_launches",
]

# POLYMER_B200_CHECKED=1 loads the checked build (every vertex id the engine
# kernels read is bounds-tested; a bad one fails the call with
# PM_ERR_BAD_GRAPH instead of reading out of bounds).
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                        "libpolymer_b200_check.so" if os.environ.get("POLYMER_B200_CHECKED") == "1"
                        else "libpolymer_b200.so")

PM_MEM_HOST, PM_MEM_DEVICE = 0, 1
PM_GRAPH_SYMMETRIC, PM_GRAPH_SKIP_SELF_LOOPS, PM_LOAD_BINARY, PM_LOAD_DUMP = 2, 4, 16, 32
# Work of one row in the pull's load balance and in the partition cut rule,
# in edges (kRowWork of the kernels).
ROW_WORK = 4
PM_F32, PM_F64, PM_I32 = 0, 1, 2
BF_INF = 1073741823

_STATUS = {
    0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA", 4: "TIMEOUT", 5: "BAD_GRAPH",
    6: "NOT_SUPPORTED", 7: "NO_DEVICE",
}


class PolymerError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__("%s: %s" % (_STATUS.get(status, status), msg))
        self.status = status


class TraversalStats(C.Structure):
    _fields_ = [("rounds", C.c_int32), ("dense_rounds", C.c_int32),
                ("edges_visited", C.c_int64), ("reached", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneReport(C.Structure):
    _fields_ = [("trials", C.c_int64), ("default_ms", C.c_double), ("best_ms", C.c_double)]


# run-time tunables (pm_graph_set_tunable) and applications (pm_tune)
TUNABLES = {"heavy_deg": 0, "cta_expand": 1, "grid_expand": 2, "pull_ctas_per_sm": 3,
            "bfs_div": 4, "cc_div": 5, "bf_div": 6, "cuda_graphs": 7, "heavy_mode": 8,
            "hub_cache": 9, "multi_div": 10, "bf_dense": 11, "cc_mode": 12,
            "bf_delta": 13, "pull_stage": 14, "push_agg": 15}
APPS = {"pagerank": 0, "spmv": 1, "bp": 2, "bfs": 3, "cc": 4, "bellman_ford": 5}

_lib = None


# pm_allgather_fn: (user, buf, elem_bytes, bounds[nranks+1], nranks, stream) -> 0 on success
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64), C.c_int,
                          C.c_void_p)


def lib():
    """Load the engine; raises PolymerError when it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise PolymerError(6, "%s is not built (run polymer_b200/_build.py)" % os.path.basename(LIB_PATH))
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, u32, u64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32, C.c_uint64
    sigs = {
        "pm_graph_create": [vp, vp, i64, i64, u32, u32, C.c_int, C.POINTER(vp)],
        "pm_graph_create_rmat": [C.c_int, C.c_int, u64, u32, C.c_int, C.POINTER(vp)],
        "pm_graph_destroy": [vp],
        "pm_graph_info": [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)],
        "pm_graph_get_csr": [vp, vp, vp, u32],
        "pm_graph_set_weights_i32": [vp, vp, u32],
        "pm_graph_set_weights_f32": [vp, vp, u32],
        "pm_graph_gen_weights_i32": [vp, u64, i32],
        "pm_graph_gen_weights_f32": [vp, u64],
        "pm_graph_get_weights_f32": [vp, vp, u32],
        "pm_graph_get_weights_i32": [vp, vp, u32],
        "pm_fill_uniform_f32": [vp, u64, C.c_int, vp, i64],
        "pm_bfs": [vp, i32, vp, vp, u32, i64, C.POINTER(TraversalStats)],
        "pm_bfs_multi": [vp, vp, C.c_int, vp, u32, i64, C.POINTER(TraversalStats)],
        "pm_bfs_async": [vp, i32, vp, u32, C.POINTER(TraversalStats)],
        "pm_bellman_ford_multi": [vp, vp, C.c_int, vp, u32, i64, C.POINTER(TraversalStats)],
        "pm_ppr": [vp, vp, C.c_int, C.c_int, C.c_double, vp, u32],
        "pm_pagerank_delta": [vp, C.c_int, C.c_double, C.c_double, C.c_int, vp, u32, i64,
                              C.POINTER(TraversalStats)],
        "pm_graph_create_er_batch": [C.c_int, i64, i64, C.c_int, u64, C.c_int, C.POINTER(vp)],
        "pm_graph_set_parts": [vp, vp, C.c_int],
        "pm_graph_get_parts": [vp, vp, C.POINTER(C.c_int)],
        "pm_pagerank_parts": [vp, C.c_int, C.c_double, vp, u32],
        "pm_weighted_pagerank": [vp, C.c_double, C.c_double, C.c_int, vp, u32, C.POINTER(C.c_int),
                                 C.POINTER(C.c_double)],
        "pm_pagerank_adjoint": [vp, C.c_double, C.c_double, C.c_int, vp, vp, vp, vp, u32,
                                C.POINTER(C.c_int), C.POINTER(C.c_double)],
        "pm_spmv_backward": [vp, vp, vp, vp, vp, u32],
        "pm_graph_gen_weights_lognormal": [vp, u64],
        "pm_pagerank_static": [vp, vp, i64, i64, C.c_int, C.c_double, vp, vp],
        "pm_components": [vp, vp, u32, i64, C.POINTER(TraversalStats)],
        "pm_bellman_ford": [vp, i32, vp, u32, i64, C.POINTER(TraversalStats)],
        "pm_pagerank": [vp, C.c_int, C.c_double, C.c_int, vp, u32, vp],
        "pm_spmv": [vp, vp, C.c_int, vp, u32, vp],
        "pm_spmv_f64": [vp, vp, C.c_int, vp, u32, vp],
        "pm_bp": [vp, vp, vp, C.c_int, vp, u32],
        "pm_bp_f64": [vp, vp, vp, C.c_int, vp, u32],
        "pm_timer_begin": [vp],
        "pm_timer_end": [vp, C.POINTER(C.c_float)],
        "pm_profile_enable": [vp, C.c_int],
        "pm_profile_read": [vp, C.c_char_p, C.POINTER(C.c_double), C.POINTER(i64), C.c_int],
        "pm_host_alloc": [u64, C.POINTER(vp)],
        "pm_host_free": [vp],
        "pm_graph_set_tunable": [vp, C.c_int, i64],
        "pm_graph_set_stream": [vp, vp],
        "pm_graph_load_pbbs": [C.c_char_p, u32, C.c_int, C.POINTER(vp)],
        "pm_graph_create_weighted": [vp, vp, vp, C.c_int, i64, i64, u32, u32, C.c_int, C.POINTER(vp)],
        "pm_set_memory_cache": [i64],
        "pm_release_memory_cache": [],
        "pm_memory_cache_info": [C.POINTER(i64)],
        "pm_graph_get_tunable": [vp, C.c_int, C.POINTER(i64)],
        "pm_tune": [vp, C.c_int, C.POINTER(TuneReport)],
        "pm_tune_mix": [vp, vp, C.c_int, C.POINTER(TuneReport)],
        "pm_graph_create_partition": [vp, vp, vp, C.c_int, i64, i64, u32, u32, C.c_int, C.c_int, C.c_int,
                                      C.POINTER(vp)],
        "pm_graph_set_exchange": [vp, EXCHANGE_FN, vp],
        "pm_graph_partition_info": [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), vp],
        "pm_test_fail_alloc_after": [i64],
        "pm_graph_save_dump": [vp, C.c_char_p],
        "pm_test_wait_timeout": [C.c_int, i32],
    }
    for name, args in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.pm_kernel_launches.argtypes = [C.c_int]
    L.pm_kernel_launches.restype = C.c_int64
    L.pm_last_error.restype = C.c_char_p
    L.pm_version.restype = C.c_char_p
    _lib = L
    return L


def _check(status: int) -> None:
    if status != 0:
        raise PolymerError(status, lib().pm_last_error().decode(errors="replace"))


def set_default_tunable(name: str, value: int) -> None:
    """Process-wide value of a tunable for graphs created afterwards."""
    _check(lib().pm_graph_set_tunable(None, TUNABLES[name], int(value)))


def get_default_tunable(name: str) -> int:
    v = C.c_int64()
    _check(lib().pm_graph_get_tunable(None, TUNABLES[name], C.byref(v)))
    return v.value


def save_tuning(path: str, tunables: dict, note: str = "") -> None:
    """Persist a tuning table (e.g. Graph.tune(...)["tunables"] or
    Graph.tunables()) as JSON, with a free-text note (the workload it was
    tuned on)."""
    import json
    bad = sorted(set(tunables) - set(TUNABLES))
    if bad:
        raise PolymerError(1, "unknown tunables %s" % bad)
    with open(path, "w") as f:
        json.dump({"tunables": {k: int(v) for k, v in tunables.items()}, "note": note}, f, indent=1, sort_keys=True)


def load_tuning(path: str, graph: "Graph | None" = None) -> dict:
    """Apply a saved tuning table: to `graph`, or as the process-wide defaults
    of graphs created afterwards (so tables that depend on them are built
    once).  Returns the table."""
    import json
    with open(path) as f:
        table = json.load(f)["tunables"]
    bad = sorted(set(table) - set(TUNABLES))
    if bad:
        raise PolymerError(1, "unknown tunables %s" % bad)
    for k, v in table.items():
        if graph is None:
            set_default_tunable(k, v)
        else:
            graph.set_tunable(k, v)
    return table


def set_memory_cache(max_bytes: int = -1) -> None:
    """Cap of the library's device-memory cache (-1: a quarter of the device, 0: off)."""
    _check(lib().pm_set_memory_cache(int(max_bytes)))


def memory_cached() -> int:
    v = C.c_int64()
    _check(lib().pm_memory_cache_info(C.byref(v)))
    return v.value


def release_memory_cache() -> None:
    _check(lib().pm_release_memory_cache())


def kernel_launches(reset: bool = False) -> int:
    return int(lib().pm_kernel_launches(int(reset)))


def _is_device(a) -> bool:
    return hasattr(a, "data_ptr") and getattr(a, "is_cuda", False)


def _arg(a, dtype):
    """(pointer, mem flag, keep-alive) for a numpy array or CUDA tensor."""
    if a is None:
        return None, PM_MEM_HOST, None
    if _is_device(a):
        return C.c_void_p(a.data_ptr()), PM_MEM_DEVICE, a
    arr = np.ascontiguousarray(a, dtype=dtype)
    return arr.ctypes.data_as(C.c_void_p), PM_MEM_HOST, arr


class Graph:
    """A graph resident on one GPU (CSR + CSC, int32 ids and offsets)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        n, m, md = C.c_int64(), C.c_int64(), C.c_int64()
        _check(lib().pm_graph_info(self._h, C.byref(n), C.byref(m), C.byref(md)))
        self.n, self.m, self.max_out_degree = n.value, m.value, md.value

    @classmethod
    def from_csr(cls, offsets, edges, symmetric: bool = False, skip_self_loops: bool = False,
                 device: int = 0, weights=None) -> "Graph":
        """offsets: n+1 int32 (offsets[n] == m); edges: m int32 destinations;
        weights (optional): m int32 or float32 in CSR order, uploaded while
        the graph is built."""
        n = len(offsets) - 1
        m = len(edges)
        po, mem, ko = _arg(offsets, np.int32)
        pe, mem2, ke = _arg(edges, np.int32)
        if mem != mem2:
            raise PolymerError(1, "offsets and edges must live in the same memory space")
        flags = (PM_GRAPH_SYMMETRIC if symmetric else 0) | (PM_GRAPH_SKIP_SELF_LOOPS if skip_self_loops else 0)
        h = C.c_void_p()
        if weights is None:
            _check(lib().pm_graph_create(po, pe, n, m, flags, mem, device, C.byref(h)))
        else:
            is_float = (np.asarray(weights).dtype.kind == "f") if not _is_device(weights) \
                else weights.is_floating_point()
            pw, mem3, kw = _arg(weights, np.float32 if is_float else np.int32)
            if mem3 != mem:
                raise PolymerError(1, "weights must live with offsets and edges")
            _check(lib().pm_graph_create_weighted(po, pe, pw, PM_F32 if is_float else PM_I32, n, m, flags, mem,
                                                  device, C.byref(h)))
        return cls(h)

    @classmethod
    def partition(cls, offsets, edges, rank: int, nranks: int, exchange, weights=None,
                  skip_self_loops: bool = False, device: int = 0) -> "Graph":
        """This rank's part of one graph spread over nranks processes
        (pm_graph_create_partition): offsets/edges/weights are the WHOLE
        CSR; exchange(buf_ptr, elem_bytes, bounds, stream_ptr) must gather
        every rank's range [bounds[r], bounds[r+1]) of the device array at
        buf_ptr into every rank's copy, in the order of the CUDA stream
        stream_ptr (polymer_b200.distributed.allgather_v builds one over
        torch.distributed)."""
        n = len(offsets) - 1
        m = len(edges)
        po, mem, ko = _arg(offsets, np.int32)
        pe, mem2, ke = _arg(edges, np.int32)
        if mem != mem2:
            raise PolymerError(1, "offsets and edges must live in the same memory space")
        pw, wtype, kw = None, PM_F32, None
        if weights is not None:
            is_float = (np.asarray(weights).dtype.kind == "f") if not _is_device(weights) \
                else weights.is_floating_point()
            pw, mem3, kw = _arg(weights, np.float32 if is_float else np.int32)
            if mem3 != mem:
                raise PolymerError(1, "weights must live with offsets and edges")
            wtype = PM_F32 if is_float else PM_I32
        flags = PM_GRAPH_SKIP_SELF_LOOPS if skip_self_loops else 0
        h = C.c_void_p()
        _check(lib().pm_graph_create_partition(po, pe, pw, wtype, n, m, flags, mem, rank, nranks, device,
                                               C.byref(h)))
        g = cls(h)
        g.set_exchange(exchange)
        return g

    def set_exchange(self, exchange) -> None:
        """Python callable exchange(buf_ptr, elem_bytes, bounds, stream_ptr);
        an exception in it fails the running call (PM_ERR_CUDA)."""
        def cb(user, buf, elem_bytes, bounds, nranks, stream):
            try:
                exchange(buf, int(elem_bytes), [bounds[i] for i in range(nranks + 1)], stream)
                return 0
            except BaseException:  # the library turns nonzero into an error status
                import traceback
                traceback.print_exc()
                return 1
        self._exchange_cb = EXCHANGE_FN(cb)  # kept alive with the handle
        _check(lib().pm_graph_set_exchange(self._h, self._exchange_cb, None))

    def partition_info(self):
        """(rank, nranks, bounds): this handle's rank and every rank's vertex
        range [bounds[r], bounds[r+1])."""
        r, k = C.c_int(), C.c_int()
        _check(lib().pm_graph_partition_info(self._h, C.byref(r), C.byref(k), None))
        b = np.zeros(k.value + 1, np.int64)
        _check(lib().pm_graph_partition_info(self._h, None, None, b.ctypes.data_as(C.c_void_p)))
        return r.value, k.value, b

    @classmethod
    def from_pbbs(cls, offsets_n, edges, **kw) -> "Graph":
        """PBBS AdjacencyGraph arrays: n offsets (no trailing m) and m edges."""
        off = np.append(np.ascontiguousarray(offsets_n, np.int32), np.int32(len(edges)))
        return cls.from_csr(off, np.ascontiguousarray(edges, np.int32), **kw)

    @classmethod
    def load_pbbs(cls, path: str, symmetric: bool = False, skip_self_loops: bool = False,
                  binary: bool = False, device: int = 0) -> "Graph":
        """Read a PBBS file (text, parsed on the GPU; or the binary
        .config/.adj/.idx triple under base name `path`)."""
        h = C.c_void_p()
        flags = (PM_GRAPH_SYMMETRIC if symmetric else 0) | (PM_GRAPH_SKIP_SELF_LOOPS if skip_self_loops else 0) \
            | (PM_LOAD_BINARY if binary else 0)
        _check(lib().pm_graph_load_pbbs(os.fsencode(path), flags, device, C.byref(h)))
        return cls(h)

    @classmethod
    def load_dump(cls, path: str, symmetric: bool = False, skip_self_loops: bool = False,
                  device: int = 0) -> "Graph":
        """Read a graph dump (dumpGraphToBin's layout, parsed on the GPU)."""
        h = C.c_void_p()
        flags = (PM_GRAPH_SYMMETRIC if symmetric else 0) | (PM_GRAPH_SKIP_SELF_LOOPS if skip_self_loops else 0) \
            | PM_LOAD_DUMP
        _check(lib().pm_graph_load_pbbs(os.fsencode(path), flags, device, C.byref(h)))
        return cls(h)

    def save_dump(self, path: str) -> None:
        """Write this graph as a graph dump (both adjacency directions)."""
        _check(lib().pm_graph_save_dump(self._h, os.fsencode(path)))

    @classmethod
    def rmat(cls, scale: int, edge_factor: int = 16, seed: int = 0x5EED0001, symmetric: bool = False,
             device: int = 0) -> "Graph":
        h = C.c_void_p()
        _check(lib().pm_graph_create_rmat(scale, edge_factor, seed,
                                          PM_GRAPH_SYMMETRIC if symmetric else 0, device, C.byref(h)))
        return cls(h)

    @classmethod
    def er_batch(cls, count: int, n_min: int = 1000, n_max: int = 100000, avg_degree: int = 8,
                 seed: int = 0x5EED0006, device: int = 0) -> "Graph":
        """count independent directed Erdos-Renyi graphs as one disjoint union
        (parts(): vertex offsets of the graphs)."""
        h = C.c_void_p()
        _check(lib().pm_graph_create_er_batch(count, n_min, n_max, avg_degree, seed, device,
                                              C.byref(h)))
        return cls(h)

    def set_parts(self, vbase) -> None:
        v = np.ascontiguousarray(vbase, np.int64)
        _check(lib().pm_graph_set_parts(self._h, v.ctypes.data_as(C.c_void_p), len(v) - 1))

    def parts(self) -> np.ndarray:
        c = C.c_int()
        _check(lib().pm_graph_get_parts(self._h, None, C.byref(c)))
        v = np.zeros(c.value + 1, np.int64)
        if c.value:
            _check(lib().pm_graph_get_parts(self._h, v.ctypes.data_as(C.c_void_p), C.byref(c)))
        return v

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pm_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def csr(self):
        off = np.empty(self.n + 1, np.int32)
        idx = np.empty(max(self.m, 1), np.int32)
        _check(lib().pm_graph_get_csr(self._h, off.ctypes.data_as(C.c_void_p),
                                      idx.ctypes.data_as(C.c_void_p), PM_MEM_HOST))
        return off, idx[: self.m]

    def set_weights(self, w) -> None:
        """int32 weights (BellmanFord) or float32 weights (SpMV), CSR order."""
        is_float = (np.asarray(w).dtype.kind == "f") if not _is_device(w) else w.is_floating_point()
        p, mem, keep = _arg(w, np.float32 if is_float else np.int32)
        fn = lib().pm_graph_set_weights_f32 if is_float else lib().pm_graph_set_weights_i32
        _check(fn(self._h, p, mem))

    def gen_weights_int(self, seed: int = 0x5EED0002, wmax: int = 22) -> None:
        _check(lib().pm_graph_gen_weights_i32(self._h, seed, wmax))

    def gen_weights_unit(self, seed: int = 0x5EED0002) -> None:
        _check(lib().pm_graph_gen_weights_f32(self._h, seed))

    def gen_weights_lognormal(self, seed: int = 0x5EED0007) -> None:
        """Lognormal(0,1) float weights normalised per source row."""
        _check(lib().pm_graph_gen_weights_lognormal(self._h, seed))

    def weights_f32(self) -> np.ndarray:
        w = np.empty(max(self.m, 1), np.float32)
        _check(lib().pm_graph_get_weights_f32(self._h, w.ctypes.data_as(C.c_void_p), PM_MEM_HOST))
        return w[: self.m]

    def weights_i32(self) -> np.ndarray:
        w = np.empty(max(self.m, 1), np.int32)
        _check(lib().pm_graph_get_weights_i32(self._h, w.ctypes.data_as(C.c_void_p), PM_MEM_HOST))
        return w[: self.m]

    def timer_begin(self) -> None:
        _check(lib().pm_timer_begin(self._h))

    def timer_end(self) -> float:
        ms = C.c_float()
        _check(lib().pm_timer_end(self._h, C.byref(ms)))
        return ms.value

    def profile(self, enable: bool = True) -> None:
        _check(lib().pm_profile_enable(self._h, int(enable)))

    def profile_read(self, tag: str, reset: bool = False):
        """(total device ms, number of passes) recorded under tag."""
        ms, cnt = C.c_double(), C.c_int64()
        _check(lib().pm_profile_read(self._h, tag.encode(), C.byref(ms), C.byref(cnt), int(reset)))
        return ms.value, cnt.value

    def set_stream(self, stream=None) -> None:
        """Run this graph's work on a torch.cuda.Stream (or a raw cudaStream_t
        handle); None returns to the graph's own stream."""
        h = None if stream is None else getattr(stream, "cuda_stream", stream)
        _check(lib().pm_graph_set_stream(self._h, C.c_void_p(h) if h else None))

    def set_tunable(self, name: str, value: int) -> None:
        _check(lib().pm_graph_set_tunable(self._h, TUNABLES[name], int(value)))

    def get_tunable(self, name: str) -> int:
        v = C.c_int64()
        _check(lib().pm_graph_get_tunable(self._h, TUNABLES[name], C.byref(v)))
        return v.value

    def tunables(self) -> dict:
        return {k: self.get_tunable(k) for k in TUNABLES}

    def tune(self, app) -> dict:
        """Autotune the tunables `app` (a name, or a list of names tuned as
        one mix) uses on this graph; returns the report and the settings kept."""
        r = TuneReport()
        if isinstance(app, str):
            _check(lib().pm_tune(self._h, APPS[app], C.byref(r)))
        else:
            a = np.array([APPS[x] for x in app], np.int32)
            _check(lib().pm_tune_mix(self._h, a.ctypes.data_as(C.c_void_p), len(a), C.byref(r)))
        return {"trials": r.trials, "default_ms": r.default_ms, "best_ms": r.best_ms,
                "tunables": self.tunables()}


def test_fail_alloc_after(k: int) -> None:
    """Failure tests: the k-th device allocation of the library from now on
    fails as an out-of-memory would (k < 1: off)."""
    _check(lib().pm_test_fail_alloc_after(int(k)))


def test_wait_timeout(max_polls: int, device: int = 0) -> None:
    """Failure tests: a bounded device wait on a flag nothing sets; raises
    PolymerError with status 4 (PM_ERR_TIMEOUT)."""
    _check(lib().pm_test_wait_timeout(int(device), int(max_polls)))


class PinnedArray:
    """A numpy view of page-locked host memory from pm_host_alloc."""

    def __init__(self, count: int, dtype):
        self.dtype = np.dtype(dtype)
        self._p = C.c_void_p()
        _check(lib().pm_host_alloc(max(count, 1) * self.dtype.itemsize, C.byref(self._p)))
        buf = (C.c_char * (max(count, 1) * self.dtype.itemsize)).from_address(self._p.value)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=count)

    def free(self) -> None:
        if self._p:
            self.array = None
            lib().pm_host_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _out(like, n, dtype, out=None):
    """Output buffer: `out` if given (numpy array or CUDA tensor of n items),
    else a new one in the memory space of `like` (CUDA tensor) or numpy."""
    if out is not None:
        if _is_device(out):
            if out.numel() != n or out.element_size() != np.dtype(dtype).itemsize:
                raise PolymerError(1, "out must hold %d items of %s" % (n, np.dtype(dtype).name))
            return out, C.c_void_p(out.data_ptr()), PM_MEM_DEVICE
        if out.size != n or out.dtype != np.dtype(dtype) or not out.flags.c_contiguous:
            raise PolymerError(1, "out must be a contiguous %s array of %d items" % (np.dtype(dtype).name, n))
        return out, out.ctypes.data_as(C.c_void_p), PM_MEM_HOST
    if like is not None and _is_device(like):
        import torch
        t = torch.empty(n, dtype={np.int32: torch.int32, np.float32: torch.float32,
                                  np.float64: torch.float64}[dtype], device=like.device)
        return t, C.c_void_p(t.data_ptr()), PM_MEM_DEVICE
    a = np.empty(max(n, 1), dtype)[:n]
    return a, a.ctypes.data_as(C.c_void_p), PM_MEM_HOST


def BFS(start: int, g: Graph, threshold: int = -1, device_out=None, stats: bool = False, out=None):
    """Parents and depths from `start` (numa-BFS.C BFS_F).  threshold < 0:
    direction switch at m/20; 0: dense pull every level as the reference.
    out: optional (parents, depth) buffers to write into."""
    par, pp, mem = _out(device_out, g.n, np.int32, None if out is None else out[0])
    dep, pd, mem2 = _out(device_out, g.n, np.int32, None if out is None else out[1])
    if mem != mem2:
        raise PolymerError(1, "parents and depth must live in the same memory space")
    st = TraversalStats()
    _check(lib().pm_bfs(g.handle, int(start), pp, pd, mem, int(threshold), C.byref(st)))
    return (par, dep, st.as_dict()) if stats else (par, dep)


def BFSAsync(start: int, g: Graph, device_out=None, stats: bool = False, out=None):
    """Reachability with a parent tree from one persistent launch
    (numa-BFS-async-pipe.C): parents over exactly the vertices BFS reaches,
    a valid tree but not a BFS tree."""
    par, pp, mem = _out(device_out, g.n, np.int32, out)
    st = TraversalStats()
    _check(lib().pm_bfs_async(g.handle, int(start), pp, mem, C.byref(st)))
    return (par, st.as_dict()) if stats else par


def _multi_source(fn, sources, g: Graph, threshold, device_out, stats, out):
    src = np.ascontiguousarray(sources, np.int32)
    k = len(src)
    res, pd, mem = _out(device_out, k * g.n, np.int32, None if out is None else out.reshape(-1))
    if mem == PM_MEM_DEVICE:
        import torch
        src_t = torch.from_numpy(src).to(res.device)
        ps = C.c_void_p(src_t.data_ptr())
        torch.cuda.synchronize()
    else:
        ps = src.ctypes.data_as(C.c_void_p)
    st = TraversalStats()
    _check(fn(g.handle, ps, k, pd, mem, int(threshold), C.byref(st)))
    res = res.reshape(k, g.n)
    return (res, st.as_dict()) if stats else res


def BFSMulti(sources, g: Graph, threshold: int = -1, device_out=None, stats: bool = False,
             out=None):
    """Depths from up to 64 sources in one traversal (uint64 source lanes per
    vertex): a (k, n) int32 array, row l = BFS depths from sources[l]."""
    return _multi_source(lib().pm_bfs_multi, sources, g, threshold, device_out, stats, out)


def BellmanFordMulti(sources, g: Graph, threshold: int = -1, device_out=None, stats: bool = False,
                     out=None):
    """Shortest-path distances from up to 64 sources in one traversal (64
    int32 distance lanes per vertex): a (k, n) int32 array, row l = the
    BellmanFord distances from sources[l]."""
    return _multi_source(lib().pm_bellman_ford_multi, sources, g, threshold, device_out, stats, out)


def Components(g: Graph, threshold: int = -1, device_out=None, stats: bool = False, out=None):
    """Min-label connected components (numa-Components.C CC_F)."""
    lab, pl, mem = _out(device_out, g.n, np.int32, out)
    st = TraversalStats()
    _check(lib().pm_components(g.handle, pl, mem, int(threshold), C.byref(st)))
    return (lab, st.as_dict()) if stats else lab


def BellmanFord(g: Graph, start: int, threshold: int = -1, device_out=None, stats: bool = False,
                out=None):
    """Shortest-path distances over the int32 weights (numa-BellmanFord.C BF_F)."""
    dist, pd, mem = _out(device_out, g.n, np.int32, out)
    st = TraversalStats()
    _check(lib().pm_bellman_ford(g.handle, int(start), pd, mem, int(threshold), C.byref(st)))
    return (dist, st.as_dict()) if stats else dist


def PageRank(g: Graph, maxIter: int = 20, damping: float = 0.85, dtype=np.float64,
             device_out=None, resid: bool = False, out=None):
    """Polymer-semantics PageRank (numa-PageRank.C PR_F); dtype float32/float64."""
    dt = np.float64 if np.dtype(dtype) == np.float64 else np.float32
    ranks, pr, mem = _out(device_out, g.n, dt, out)
    res = np.zeros(max(maxIter, 1), np.float64)
    _check(lib().pm_pagerank(g.handle, int(maxIter), float(damping),
                             PM_F64 if dt == np.float64 else PM_F32, pr, mem,
                             res.ctypes.data_as(C.c_void_p) if resid else None))
    return (ranks, res[:maxIter]) if resid else ranks


def PageRankDelta(g: Graph, maxIter: int = 10, damping: float = 0.85, epsilon: float = 0.01,
                  dtype=np.float64, threshold: int = -1, device_out=None, stats: bool = False, out=None):
    """Delta-propagating PageRank (numa-PageRankDelta.C): only vertices whose
    rank moved by more than epsilon of itself push their change."""
    dt = np.float64 if np.dtype(dtype) == np.float64 else np.float32
    ranks, pr, mem = _out(device_out, g.n, dt, out)
    st = TraversalStats()
    _check(lib().pm_pagerank_delta(g.handle, int(maxIter), float(damping), float(epsilon),
                                   PM_F64 if dt == np.float64 else PM_F32, pr, mem, int(threshold),
                                   C.byref(st)))
    return (ranks, st.as_dict()) if stats else ranks


def WeightedPageRank(g: Graph, damping: float = 0.85, tol: float = 1e-6, max_iters: int = 1000,
                     device_out=None, out=None):
    """p = damping * A_W^T p + (1-damping)/n over the float weights, to a
    relative L1 change <= tol: (p, iterations, last relative change)."""
    p, pp, mem = _out(device_out, g.n, np.float32, out)
    it, res = C.c_int(), C.c_double()
    _check(lib().pm_weighted_pagerank(g.handle, float(damping), float(tol), int(max_iters), pp, mem,
                                      C.byref(it), C.byref(res)))
    return p, it.value, res.value


def PageRankAdjoint(g: Graph, p, grad_p, damping: float = 0.85, tol: float = 1e-6,
                    max_iters: int = 1000, with_lambda: bool = False, out=None):
    """dL/dW per CSR edge for the cotangent grad_p at the fixed point p
    (transposed iteration over the CSR): dw (, lambda), iterations."""
    pp, mem, kp = _arg(p, np.float32)
    pg, mem2, kg = _arg(grad_p, np.float32)
    if mem != mem2:
        raise PolymerError(1, "p and grad_p must live in the same memory space")
    like = p if mem == PM_MEM_DEVICE else None
    dw, pdw, _ = _out(like, g.m, np.float32, out)
    lam, pl, _ = _out(like, g.n, np.float32) if with_lambda else (None, None, None)
    it, res = C.c_int(), C.c_double()
    _check(lib().pm_pagerank_adjoint(g.handle, float(damping), float(tol), int(max_iters), pp, pg, pdw,
                                     pl, mem, C.byref(it), C.byref(res)))
    return (dw, lam, it.value) if with_lambda else (dw, it.value)


def SpMVBackward(g: Graph, x, grad_y):
    """Backward of y = A_W^T x: (dx = A_W grad_y, dw[e] = grad_y[v] x[s])."""
    px, mem, kx = _arg(x, np.float32)
    pg, mem2, kg = _arg(grad_y, np.float32)
    if mem != mem2:
        raise PolymerError(1, "x and grad_y must live in the same memory space")
    like = x if mem == PM_MEM_DEVICE else None
    dx, pdx, _ = _out(like, g.n, np.float32)
    dw, pdw, _ = _out(like, g.m, np.float32)
    _check(lib().pm_spmv_backward(g.handle, px, pg, pdx, pdw, mem))
    return dx, dw


def PageRankStatic(offsets, edges, ranks, maxIter: int = 20, damping: float = 0.85, stream=None):
    """PageRank for callers that cannot allocate GPU memory (pm_pagerank_static):
    offsets (n+1 int32), edges (m int32) and ranks (n float32) are contiguous
    CUDA tensors; the working vectors live in a fixed array inside the library
    (n <= 2^20).  Nothing is allocated by this call."""
    import torch
    for t, dt, name in ((offsets, torch.int32, "offsets"), (edges, torch.int32, "edges"),
                        (ranks, torch.float32, "ranks")):
        if not _is_device(t):
            raise PolymerError(1, "PageRankStatic takes CUDA tensors only (%s)" % name)
        if t.dtype != dt or not t.is_contiguous():
            raise PolymerError(1, "%s must be a contiguous %s tensor" % (name, dt))
    n = offsets.numel() - 1
    if ranks.numel() != n:
        raise PolymerError(1, "ranks must hold offsets.numel() - 1 = %d floats" % n)
    _check(lib().pm_pagerank_static(C.c_void_p(offsets.data_ptr()), C.c_void_p(edges.data_ptr()), n,
                                    edges.numel(), int(maxIter), float(damping),
                                    C.c_void_p(ranks.data_ptr()),
                                    None if stream is None else C.c_void_p(stream)))
    return ranks


def PageRankParts(g: Graph, maxIter: int = 20, damping: float = 0.85, device_out=None, out=None):
    """PageRank of every part of a disjoint union (each with its own n), all
    parts in one persistent launch: n float32 in union order."""
    ranks, pr, mem = _out(device_out, g.n, np.float32, out)
    _check(lib().pm_pagerank_parts(g.handle, int(maxIter), float(damping), pr, mem))
    return ranks


def PersonalizedPageRank(g: Graph, seeds, maxIter: int = 20, damping: float = 0.85,
                         device_out=None, out=None):
    """PPR for up to 32 seeds in one SpMM-shaped pass per iteration: (n, k) float32."""
    s = np.ascontiguousarray(seeds, np.int32)
    k = len(s)
    res, po, mem = _out(device_out, g.n * k, np.float32, None if out is None else out.reshape(-1))
    if mem == PM_MEM_DEVICE:
        import torch
        s_t = torch.from_numpy(s).to(res.device)
        torch.cuda.synchronize()
        ps = C.c_void_p(s_t.data_ptr())
    else:
        ps = s.ctypes.data_as(C.c_void_p)
    _check(lib().pm_ppr(g.handle, ps, k, int(maxIter), float(damping), po, mem))
    return res.reshape(g.n, k)


def _arg_typed(a, dtype):
    """_arg with device tensors converted to dtype when they differ."""
    if a is not None and _is_device(a):
        import torch
        want = {np.float32: torch.float32, np.float64: torch.float64}[dtype]
        if a.dtype != want:
            a = a.to(want).contiguous()
    return _arg(a, dtype)


def SPMV(g: Graph, x0, maxIter: int = 10, norms: bool = False, out=None, dtype=np.float32):
    """x <- A_w^T x, maxIter times, over the float weights (numa-SPMV.C SPMV_F);
    dtype float32 (FP32 vectors and sums) or float64 (the FP64 yardstick)."""
    dt = np.float64 if np.dtype(dtype) == np.float64 else np.float32
    px, mem, keep = _arg_typed(x0, dt)
    y, py, mem2 = _out(keep if mem == PM_MEM_DEVICE else None, g.n, dt, out)
    if mem != mem2:
        raise PolymerError(1, "x0 and out must live in the same memory space")
    nrm = np.zeros(max(maxIter, 1), np.float64)
    fn = lib().pm_spmv_f64 if dt == np.float64 else lib().pm_spmv
    _check(fn(g.handle, px, int(maxIter), py, mem, nrm.ctypes.data_as(C.c_void_p) if norms else None))
    return (y, nrm[:maxIter]) if norms else y


def BeliefPropagation(g: Graph, prior, maxIter: int = 10, psi=((0.9, 0.1), (0.1, 0.9)), out=None,
                      dtype=np.float32):
    """2-state BP log-products (n x 2) (numa-BP.C BP_F, normalised messages);
    dtype float32 or float64."""
    dt = np.float64 if np.dtype(dtype) == np.float64 else np.float32
    pp, mem, keep = _arg_typed(prior, dt)
    psi_a = np.ascontiguousarray(psi, dt).reshape(4)
    if mem == PM_MEM_DEVICE:
        import torch
        psi_t = torch.tensor(psi_a, device=keep.device)
        ppsi = C.c_void_p(psi_t.data_ptr())
    else:
        psi_t = psi_a
        ppsi = psi_a.ctypes.data_as(C.c_void_p)
    flat = None if out is None else out.reshape(-1)
    res, po, mem2 = _out(keep if mem == PM_MEM_DEVICE else None, 2 * g.n, dt, flat)
    if mem != mem2:
        raise PolymerError(1, "prior and out must live in the same memory space")
    fn = lib().pm_bp_f64 if dt == np.float64 else lib().pm_bp
    _check(fn(g.handle, pp, ppsi, int(maxIter), po, mem))
    return res.reshape(g.n, 2)


def uniform_f32(g: Graph, count: int, seed: int, open_interval: bool = False):
    """Seeded uniform floats on g's device ([0,1), or (0,1) with open_interval),
    the oracle's pmo_fill_uniform01 / _open rule; returns a torch CUDA tensor."""
    import torch
    x = torch.empty(count, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    _check(lib().pm_fill_uniform_f32(g.handle, seed, int(open_interval), C.c_void_p(x.data_ptr()),
                                     count))
    return x
