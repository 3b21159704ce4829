"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE, not product).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  It loads ``_build/libpm_oracle.so`` (the C
restatement in ``pm_oracle.c``) and drives the reference binaries in ``_ref/``
(compiled from the original Polymer sources by ``oracle/Makefile``).

Graph convention: CSR ``off`` (int32, n+1) and ``idx`` (int32, m), edges
sorted by (source, destination), no self loops, no duplicates.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpm_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

BF_INF = 1073741823  # INT_MAX / 2, numa-BellmanFord.C:283
SEED_GRAPH = 0x5EED0001
SEED_WEIGHT = 0x5EED0002
SEED_X = 0x5EED0003
SEED_PRIOR = 0x5EED0004
SEED_SOURCES = 0x5EED0005

_lib = None

# Where the reference sources lie (read only by the build recipe; the one
# place this path is set).  Absent on machines that only run the prebuilt
# checkers.
REFERENCE_DIR = os.environ.get("POLYMER_REFERENCE", "/root/reference")


def build() -> None:
    """Compile the C restatement (and, when the reference sources are
    present, the reference binaries) with make."""
    targets = ["oracle"]
    if os.path.isdir(REFERENCE_DIR):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, "REF=" + REFERENCE_DIR] + targets, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        i64, u64, i32 = C.c_int64, C.c_uint64, C.c_int32
        sig = {
            "pmo_hash": (u64, [u64, u64]),
            "pmo_rmat_edge": (u64, [C.c_int, u64, u64]),
            "pmo_keys_to_csr": (i64, [u64p, i64, i64, C.c_int, i32p, i32p]),
            "pmo_rmat_graph": (i64, [C.c_int, C.c_int, u64, C.c_int, i32p, i32p]),
            "pmo_fill_weights_int": (None, [i64, i32p, i32p, u64, i32, i32p]),
            "pmo_fill_weights_unit": (None, [i64, i32p, i32p, u64, f32p]),
            "pmo_fill_uniform01": (None, [u64, i64, f32p]),
            "pmo_fill_uniform_open": (None, [u64, i64, f32p]),
            "pmo_pick_sources": (C.c_int, [i64, i32p, u64, C.c_int, i32p]),
            "pmo_transpose": (None, [i64, i32p, i32p, i32p, i32p, C.c_void_p]),
            "pmo_pagerank": (None, [i64, i32p, i32p, C.c_int, C.c_double, f64p, C.c_void_p]),
            "pmo_spmv": (None, [i64, i32p, i32p, f64p, f64p, C.c_int, f64p]),
            "pmo_ppr": (None, [i64, i32p, i32p, i32p, C.c_int, C.c_int, C.c_double, f64p]),
            "pmo_pagerank_delta": (None, [i64, i32p, i32p, C.c_int, C.c_double, C.c_double, f64p,
                                          C.c_void_p]),
            "pmo_weighted_pagerank": (C.c_int, [i64, i32p, i32p, f64p, C.c_double, C.c_double,
                                                C.c_int, f64p]),
            "pmo_pagerank_adjoint": (C.c_int, [i64, i32p, i32p, f64p, C.c_double, C.c_double, C.c_int,
                                               f64p, f64p, f64p, f64p]),
            "pmo_spmv_backward": (None, [i64, i32p, i32p, f64p, f64p, f64p, f64p, f64p]),
            "pmo_lognormal_weights": (None, [i64, i32p, u64, f64p]),
            "pmo_er_part_sizes": (i64, [C.c_int, i64, i64, u64, np.ctypeslib.ndpointer(np.int64)]),
            "pmo_er_batch": (i64, [C.c_int, i64, i64, C.c_int, u64, np.ctypeslib.ndpointer(np.int64),
                                   i32p, i32p]),
            "pmo_bfs": (i64, [i64, i32p, i32p, i32, i32p, C.c_void_p]),
            "pmo_cc": (C.c_int, [i64, i32p, i32p, i32p]),
            "pmo_bellman_ford": (C.c_int, [i64, i32p, i32p, i32p, i32, i32p]),
            "pmo_dijkstra": (None, [i64, i32p, i32p, i32p, i32, i32p]),
            "pmo_bp": (None, [i64, i32p, i32p, f64p, C.c_void_p, f64p, C.c_int, f64p]),
            "pmo_bp_raw": (None, [i64, i32p, i32p, f64p, f64p, C.c_int, C.c_int, f64p]),
            "pmo_write_adj_text": (C.c_int, [C.c_char_p, i64, i32p, i32p, C.c_void_p]),
            "pmo_write_adj_binary": (C.c_int, [C.c_char_p, i64, i32p, i32p]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class Graph:
    n: int
    off: np.ndarray  # int32 [n+1]
    idx: np.ndarray  # int32 [m]

    @property
    def m(self) -> int:
        return int(self.off[-1])

    def transpose(self):
        toff = np.empty(self.n + 1, np.int32)
        tidx = np.empty(max(self.m, 1), np.int32)
        eid = np.empty(max(self.m, 1), np.int32)
        lib().pmo_transpose(self.n, self.off, self.idx, toff, tidx, _ptr(eid))
        return toff, tidx[: self.m], eid[: self.m]

    def out_degree(self) -> np.ndarray:
        return np.diff(self.off).astype(np.int64)


def rmat_graph(scale: int, ef: int, seed: int = SEED_GRAPH, symmetric: bool = False) -> Graph:
    """Seeded R-MAT (a,b,c,d) = (.57,.19,.19,.05), self loops and duplicates
    removed, sorted by source: the synthetic input of every workload."""
    n = 1 << scale
    cap = n * ef * (2 if symmetric else 1)
    off = np.empty(n + 1, np.int32)
    idx = np.empty(max(cap, 1), np.int32)
    m = lib().pmo_rmat_graph(scale, ef, seed, int(symmetric), off, idx)
    return Graph(n, off, idx[:m].copy())


def er_batch(count: int, n_min: int = 1000, n_max: int = 100000, avg_degree: int = 8,
             seed: int = 0x5EED0006):
    """Disjoint union of count seeded directed ER graphs: (Graph, vbase)."""
    vbase = np.zeros(count + 1, np.int64)
    n = lib().pmo_er_part_sizes(count, n_min, n_max, seed, vbase)
    off = np.empty(n + 1, np.int32)
    idx = np.empty(max(n * avg_degree, 1), np.int32)
    m = lib().pmo_er_batch(count, n_min, n_max, avg_degree, seed, vbase, off, idx)
    return Graph(int(n), off, idx[:m].copy()), vbase


def subgraph(g: Graph, v0: int, v1: int) -> Graph:
    """Induced subgraph on the contiguous range [v0, v1) of a graph whose
    edges never leave that range (a part of a disjoint union)."""
    off = (g.off[v0:v1 + 1] - g.off[v0]).astype(np.int32)
    idx = (g.idx[g.off[v0]:g.off[v1]] - v0).astype(np.int32)
    return Graph(v1 - v0, off, idx)


def graph_from_edges(n: int, src, dst, symmetric: bool = False) -> Graph:
    """CSR from an explicit edge list (dedup, self loops dropped)."""
    src = np.asarray(src, np.uint64)
    dst = np.asarray(dst, np.uint64)
    keys = np.empty(max(2 * len(src), 1), np.uint64)
    keys[: len(src)] = (src << np.uint64(32)) | dst
    off = np.empty(n + 1, np.int32)
    idx = np.empty(max(2 * len(src), 1), np.int32)
    m = lib().pmo_keys_to_csr(keys, len(src), n, int(symmetric), off, idx)
    return Graph(n, off, idx[:m].copy())


def weights_int(g: Graph, seed: int = SEED_WEIGHT, wmax: int = 22) -> np.ndarray:
    w = np.empty(max(g.m, 1), np.int32)
    lib().pmo_fill_weights_int(g.n, g.off, g.idx if g.m else np.zeros(1, np.int32), seed, wmax, w)
    return w[: g.m]


def weights_unit(g: Graph, seed: int = SEED_WEIGHT) -> np.ndarray:
    w = np.empty(max(g.m, 1), np.float32)
    lib().pmo_fill_weights_unit(g.n, g.off, g.idx if g.m else np.zeros(1, np.int32), seed, w)
    return w[: g.m]


def uniform01(count: int, seed: int = SEED_X) -> np.ndarray:
    x = np.empty(max(count, 1), np.float32)
    lib().pmo_fill_uniform01(seed, count, x)
    return x[:count]


def uniform_open(count: int, seed: int = SEED_PRIOR) -> np.ndarray:
    x = np.empty(max(count, 1), np.float32)
    lib().pmo_fill_uniform_open(seed, count, x)
    return x[:count]


def pick_sources(g: Graph, k: int, seed: int = SEED_SOURCES) -> np.ndarray:
    out = np.zeros(k, np.int32)
    got = lib().pmo_pick_sources(g.n, g.off, seed, k, out)
    return out[:got]


def _idx(g: Graph):
    return g.idx if g.m else np.zeros(1, np.int32)


def pagerank(g: Graph, iters: int, damping: float = 0.85, with_resid: bool = False):
    out = np.empty(g.n, np.float64)
    resid = np.zeros(max(iters, 1), np.float64)
    lib().pmo_pagerank(g.n, g.off, _idx(g), iters, damping, out, _ptr(resid))
    return (out, resid[:iters]) if with_resid else out


def pagerank_delta(g: Graph, iters: int, damping: float = 0.85, eps2: float = 0.01,
                   with_frontier: bool = False):
    """PageRankDelta restatement (FP64): p after `iters` rounds (and the
    frontier size after each round)."""
    p = np.empty(g.n, np.float64)
    fs = np.zeros(max(iters, 1), np.int64)
    lib().pmo_pagerank_delta(g.n, g.off, _idx(g), iters, damping, eps2, p, fs.ctypes.data_as(C.c_void_p))
    return (p, fs[:iters]) if with_frontier else p


def ppr(g: Graph, seeds, iters: int, damping: float = 0.85) -> np.ndarray:
    """Personalised PageRank of len(seeds) seeds: (n, k) FP64."""
    s = np.ascontiguousarray(seeds, np.int32)
    out = np.empty(g.n * len(s), np.float64)
    lib().pmo_ppr(g.n, g.off, _idx(g), s, len(s), iters, damping, out)
    return out.reshape(g.n, len(s))


def lognormal_weights(g: Graph, seed: int = SEED_WEIGHT) -> np.ndarray:
    """Lognormal(0,1) weights normalised per source row, FP64, CSR order."""
    w = np.empty(max(g.m, 1), np.float64)
    lib().pmo_lognormal_weights(g.n, g.off, seed, w)
    return w[: g.m]


def weighted_pagerank(g: Graph, w, damping: float = 0.85, tol: float = 1e-6, max_iters: int = 1000):
    p = np.empty(g.n, np.float64)
    it = lib().pmo_weighted_pagerank(g.n, g.off, _idx(g), np.ascontiguousarray(w, np.float64),
                                     damping, tol, max_iters, p)
    return p, it


def pagerank_adjoint(g: Graph, w, p, gp, damping: float = 0.85, tol: float = 1e-6,
                     max_iters: int = 1000):
    """(dL/dW per CSR edge, lambda, iterations) for cotangent gp = dL/dp."""
    lam = np.empty(g.n, np.float64)
    dw = np.empty(max(g.m, 1), np.float64)
    it = lib().pmo_pagerank_adjoint(g.n, g.off, _idx(g), np.ascontiguousarray(w, np.float64), damping,
                                    tol, max_iters, np.ascontiguousarray(p, np.float64),
                                    np.ascontiguousarray(gp, np.float64), lam, dw)
    return dw[: g.m], lam, it


def spmv_backward(g: Graph, w, x, gy):
    dx = np.empty(g.n, np.float64)
    dw = np.empty(max(g.m, 1), np.float64)
    lib().pmo_spmv_backward(g.n, g.off, _idx(g), np.ascontiguousarray(w, np.float64),
                            np.ascontiguousarray(x, np.float64), np.ascontiguousarray(gy, np.float64),
                            dx, dw)
    return dx, dw[: g.m]


def induced_subgraph(g: Graph, k: int, w=None):
    """Subgraph on vertices [0, k) keeping the edges between them (and their
    weights when given)."""
    src = np.repeat(np.arange(g.n), np.diff(g.off))
    keep = (src < k) & (g.idx < k)
    s, d = src[keep], g.idx[keep]
    off = np.zeros(k + 1, np.int32)
    np.add.at(off, s + 1, 1)
    off = np.cumsum(off).astype(np.int32)
    sub = Graph(k, off, d.astype(np.int32))
    return (sub, np.asarray(w)[keep]) if w is not None else sub


def spmv(g: Graph, w, x0, iters: int) -> np.ndarray:
    out = np.empty(g.n, np.float64)
    w64 = np.ascontiguousarray(w, np.float64) if g.m else np.zeros(1, np.float64)
    lib().pmo_spmv(g.n, g.off, _idx(g), w64, np.ascontiguousarray(x0, np.float64), iters, out)
    return out


def bfs(g: Graph, src: int):
    depth = np.empty(g.n, np.int32)
    parents = np.empty(g.n, np.int32)
    lib().pmo_bfs(g.n, g.off, _idx(g), src, depth, _ptr(parents))
    return depth, parents


def cc(g: Graph) -> np.ndarray:
    labels = np.empty(g.n, np.int32)
    lib().pmo_cc(g.n, g.off, _idx(g), labels)
    return labels


def bellman_ford(g: Graph, w, src: int) -> np.ndarray:
    dist = np.empty(g.n, np.int32)
    w32 = np.ascontiguousarray(w, np.int32) if g.m else np.zeros(1, np.int32)
    lib().pmo_bellman_ford(g.n, g.off, _idx(g), w32, src, dist)
    return dist


def dijkstra(g: Graph, w, src: int) -> np.ndarray:
    dist = np.empty(g.n, np.int32)
    w32 = np.ascontiguousarray(w, np.int32) if g.m else np.zeros(1, np.int32)
    lib().pmo_dijkstra(g.n, g.off, _idx(g), w32, src, dist)
    return dist


def bp(g: Graph, prior, iters: int, psi_uniform=None, psi_edge=None) -> np.ndarray:
    """Log-products (n x 2) of the 2-state BP restatement."""
    out = np.empty(2 * g.n, np.float64)
    pu = np.ascontiguousarray(
        psi_uniform if psi_uniform is not None else [[0.9, 0.1], [0.1, 0.9]], np.float64
    ).reshape(4)
    pe = None if psi_edge is None else np.ascontiguousarray(psi_edge, np.float64).reshape(-1)
    lib().pmo_bp(g.n, g.off, _idx(g), np.ascontiguousarray(prior, np.float64).reshape(-1),
                 _ptr(pe), pu, iters, out)
    return out.reshape(g.n, 2)


def bp_raw(g: Graph, prior, iters: int, normalize: bool = False, psi=((0.9, 0.1), (0.1, 0.9))) -> np.ndarray:
    """Linear products (n x 2) of BP as the reference writes it (pmo_bp_raw):
    unnormalised beliefs, or with normalize each belief divided by its sum."""
    out = np.empty(2 * g.n, np.float64)
    lib().pmo_bp_raw(g.n, g.off, _idx(g), np.ascontiguousarray(prior, np.float64).reshape(-1),
                     np.ascontiguousarray(psi, np.float64).reshape(4), iters, int(normalize), out)
    return out.reshape(g.n, 2)


def bp_ref_priors(n: int) -> np.ndarray:
    """The priors the patched reference BP sets (ref_patch_bp.py), as float32:
    p0 = (float)(0.2 + 0.6 * ((37 v + 11) mod 101) / 101), p1 = 1 - p0."""
    v = np.arange(n, dtype=np.int64)
    p0 = (0.2 + 0.6 * ((37 * v + 11) % 101).astype(np.float64) / 101.0).astype(np.float32)
    p1 = np.float32(1.0) - p0
    return np.stack([p0, p1], axis=1)


def bfs_depths_from_parents(parents: np.ndarray, src: int) -> np.ndarray:
    """Depth of every vertex by walking the parent array (-1: unreached).
    Raises ValueError on a cycle or a parent chain that misses src."""
    n = len(parents)
    depth = np.full(n, -2, np.int64)
    depth[parents < 0] = -1
    depth[src] = 0
    for v in range(n):
        if depth[v] != -2:
            continue
        chain = []
        u = v
        while depth[u] == -2:
            chain.append(u)
            u = int(parents[u])
            if u < 0 or len(chain) > n:
                raise ValueError("broken parent chain at %d" % v)
        base = depth[u]
        if base < 0:
            raise ValueError("parent chain of %d reaches an unreached vertex" % v)
        for k, x in enumerate(reversed(chain)):
            depth[x] = base + 1 + k
    return depth.astype(np.int32)


# ------------------------------------------------------------------------
# Reference binaries (compiled by oracle/Makefile into _ref/).
# ------------------------------------------------------------------------

def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "numa-PageRank"))


def write_binary(g: Graph, base: str) -> str:
    """Write <base>.config/.adj/.idx and return the base name to pass to the
    reference.  The reference's binary loaders copy "<base>.config" (len+8
    bytes with the NUL) into char[len+7] and "<base>.adj"/".idx" (len+5) into
    char[len+4] stack arrays (IO-numa.h:409-417); the extra byte lands in the
    16-byte alignment padding of those arrays unless len+7 or len+4 is a
    multiple of 16, where the program can abort.  Such lengths get a suffix."""
    while len(base) % 16 in (9, 12):
        base = base + "_"
    if lib().pmo_write_adj_binary(base.encode(), g.n, g.off, _idx(g)) != 0:
        raise OSError("cannot write %s" % base)
    return base


def transpose(g: Graph):
    """In-adjacency of g: CSC offsets and, per destination, its sources in
    ascending order (the order the reference's readGraph gives in-edges,
    IO-numa.h:145-180)."""
    deg = np.diff(g.off).astype(np.int64)
    src = np.repeat(np.arange(g.n, dtype=np.int64), deg)
    order = np.lexsort((src, g.idx.astype(np.int64)))
    in_idx = src[order].astype(np.int32)
    in_off = np.concatenate([[0], np.cumsum(np.bincount(g.idx, minlength=g.n))]).astype(np.int32)
    return in_off, in_idx


def write_dump(g: Graph, path: str) -> None:
    """The graph dump of dumpGraphToBin (IO-numa.h:837-900): int64 total
    bytes, int32 n, int64 m, then per vertex int32 -1, id, out-degree,
    in-degree, out-neighbours, in-neighbours."""
    in_off, in_idx = transpose(g)
    parts = []
    for v in range(g.n):
        o0, o1, i0, i1 = g.off[v], g.off[v + 1], in_off[v], in_off[v + 1]
        parts.append(np.array([-1, v, o1 - o0, i1 - i0], np.int32))
        parts.append(g.idx[o0:o1].astype(np.int32))
        parts.append(in_idx[i0:i1])
    body = np.concatenate(parts).astype(np.int32).tobytes() if parts else b""
    total = 8 + 4 + 8 + len(body)
    with open(path, "wb") as f:
        f.write(np.int64(total).tobytes() + np.int32(g.n).tobytes() + np.int64(len(g.idx)).tobytes() + body)


def read_dump(path: str):
    """The reader of loadGraphFromBin (IO-numa.h:758-830): (n, out_off,
    out_idx, in_off, in_idx); raises ValueError where the reference aborts."""
    raw = open(path, "rb").read()
    total = int(np.frombuffer(raw[:8], np.int64)[0])
    n = int(np.frombuffer(raw[8:12], np.int32)[0])
    m = int(np.frombuffer(raw[12:20], np.int64)[0])
    if total != len(raw):
        raise ValueError("size")
    w = np.frombuffer(raw[20:], np.int32)
    p, out_off, in_off, outs, ins = 0, [0], [0], [], []
    for v in range(n):
        if w[p] != -1 or w[p + 1] != v:
            raise ValueError("record %d" % v)
        od, idg = int(w[p + 2]), int(w[p + 3])
        outs.append(w[p + 4:p + 4 + od])
        ins.append(w[p + 4 + od:p + 4 + od + idg])
        out_off.append(out_off[-1] + od)
        in_off.append(in_off[-1] + idg)
        p += 4 + od + idg
    if p != len(w) or out_off[-1] != m:
        raise ValueError("length")
    cat = lambda xs: np.concatenate(xs).astype(np.int32) if xs else np.zeros(0, np.int32)
    return n, np.array(out_off, np.int32), cat(outs), np.array(in_off, np.int32), cat(ins)


def write_text(g: Graph, path: str, w=None) -> None:
    wp = None if w is None else np.ascontiguousarray(w, np.int32)
    if lib().pmo_write_adj_text(path.encode(), g.n, g.off, _idx(g), _ptr(wp)) != 0:
        raise OSError("cannot write %s" % path)


_TIME_RE = re.compile(r"^(PageRank|BFS|Components|BellmanFord|SPMV|BeliefPropagation)\s*:\s*([0-9.eE+-]+)", re.M)


def _run(args, threads: int | None, timeout: float):
    env = dict(os.environ)
    if threads:
        env["PM_REF_THREADS"] = str(threads)
    p = subprocess.run(args, capture_output=True, text=True, env=env, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError("reference %s failed (%d): %s" % (args[0], p.returncode, p.stderr[-400:]))
    t = _TIME_RE.findall(p.stdout)
    return p.stdout, (float(t[-1][1]) if t else float("nan"))


def ref_pagerank(path: str, iters: int, binary: bool = True, threads=None, result=True, timeout=600, exe=None):
    """numa-PageRank <g> <iters> -1 [-result] [-s] [-b]; returns (ranks|None, seconds).
    exe: another program with the same command line (the application built
    with the B200 binding in place of its PageRank body)."""
    args = [exe or os.path.join(REF_DIR, "numa-PageRank"), path, str(iters), "-1",
            "-result" if result else "-noresult", "-a", "-b" if binary else "-t"]
    out, t = _run(args, threads, timeout)
    if not result:
        return None, t
    vals = re.findall(r"^(\d+)\t([0-9.eE+-]+)$", out, re.M)
    r = np.zeros(len(vals), np.float64)
    for i, v in vals:
        r[int(i)] = float(v)
    return r, t


def ref_bp_result(path: str, iters: int, binary: bool = True, timeout=600):
    """numa-BP-result <g> <iters> -result -a [-b] on one thread (the
    reference multiplies products without atomics); returns (n x 2 products,
    seconds)."""
    args = [os.path.join(REF_DIR, "numa-BP-result"), path, str(iters), "-result", "-a",
            "-b" if binary else "-t"]
    out, t = _run(args, 1, timeout)
    vals = re.findall(r"^prod (\d+) ([0-9.eE+-]+) ([0-9.eE+-]+)$", out, re.M)
    r = np.zeros((len(vals), 2), np.float64)
    for i, a, b in vals:
        r[int(i)] = (float(a), float(b))
    return r, t


def ref_pagerank_delta(path: str, iters: int, binary: bool = True, threads=None, timeout=600):
    """numa-PageRankDelta <g> <iters> -result -a [-b]; returns (p, seconds)."""
    args = [os.path.join(REF_DIR, "numa-PageRankDelta"), path, str(iters), "-result", "-a",
            "-b" if binary else "-t"]
    out, t = _run(args, threads, timeout)
    vals = re.findall(r"^(\d+)\t([0-9.eE+-]+)$", out, re.M)
    r = np.zeros(len(vals), np.float64)
    for i, v in vals:
        r[int(i)] = float(v)
    return r, t


def ref_spmv(path: str, iters: int, threads=None, result=True, timeout=600):
    """numa-SPMV <weighted text> <iters> [-result]; returns (x|None, seconds)."""
    args = [os.path.join(REF_DIR, "numa-SPMV"), path, str(iters), "-result" if result else "-noresult"]
    out, t = _run(args, threads, timeout)
    if not result:
        return None, t
    vals = re.findall(r"^(\d+)\t([0-9.eE+-]+)$", out, re.M)
    r = np.zeros(len(vals), np.float64)
    for i, v in vals:
        r[int(i)] = float(v)
    return r, t


def ref_components(path: str, binary: bool = True, threads=None, result=True, timeout=600):
    """numa-Components <g> -s [-result] [-b]; returns (labels|None, seconds)."""
    args = [os.path.join(REF_DIR, "numa-Components"), path, "-s",
            "-result" if result else "-noresult", "-b" if binary else "-t"]
    out, t = _run(args, threads, timeout)
    if not result:
        return None, t
    vals = re.findall(r"^Result of (\d+) : (-?\d+)$", out, re.M)
    r = np.zeros(len(vals), np.int32)
    for i, v in vals:
        r[int(i)] = int(v)
    return r, t


def ref_bfs(path: str, src: int, binary: bool = True, symmetric: bool = True, threads=None,
            parents=True, timeout=600):
    """numa-BFS (or the parent-printing build) <g> <src> -result [-s] [-b];
    returns (parents|None, visited count, seconds)."""
    exe = "numa-BFS-parents" if parents else "numa-BFS"
    args = [os.path.join(REF_DIR, exe), path, str(src), "-result",
            "-s" if symmetric else "-a", "-b" if binary else "-t"]
    out, t = _run(args, threads, timeout)
    cnt = re.findall(r"^Vert visited: (\d+)", out, re.M)
    par = None
    if parents:
        vals = re.findall(r"^parent (\d+) (-?\d+)$", out, re.M)
        par = np.full(len(vals), -1, np.int32)
        for i, v in vals:
            par[int(i)] = int(v)
    return par, (int(cnt[-1]) if cnt else -1), t


def ref_bellman_ford(path: str, src: int, threads=None, result=False, timeout=600):
    """numa-BellmanFord(-dist) <weighted text> <src> [-result] -s."""
    exe = "numa-BellmanFord-dist" if result else "numa-BellmanFord"
    args = [os.path.join(REF_DIR, exe), path, str(src), "-result" if result else "-noresult", "-s"]
    out, t = _run(args, threads, timeout)
    if not result:
        return None, t
    vals = re.findall(r"^(\d+)\t(-?\d+)$", out, re.M)
    r = np.zeros(len(vals), np.int32)
    for i, v in vals:
        r[int(i)] = int(v)
    return r, t


def ref_bp(path: str, iters: int, binary: bool = True, threads=None, timeout=600):
    """numa-BP <g> <iters> (the reference prints no result); returns seconds."""
    args = [os.path.join(REF_DIR, "numa-BP"), path, str(iters), "-noresult", "-a",
            "-b" if binary else "-t"]
    _, t = _run(args, threads, timeout)
    return t


def tempdir() -> str:
    return tempfile.mkdtemp(prefix="pm_oracle_")
