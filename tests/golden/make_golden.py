"""Generate the golden fixtures of tests/golden/ from the REFERENCE binaries.

Runs the Polymer applications compiled from the original sources
(oracle/_ref, built by `make -C oracle ref`) on small seeded graphs and
stores their outputs, together with the graphs, as .npz files.  The fixtures
pin the CPU oracle (oracle/pm_oracle.c) on machines without the reference
and pin the synthetic-graph generator itself.

    python tests/golden/make_golden.py          # every fixture
    python tests/golden/make_golden.py bp       # the BP fixture only
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import pm_oracle as O  # noqa: E402


def tiny_graph():
    """Hand-built edge cases: a self loop, a 2-cycle, a vertex with no
    in-edges, a sink, two isolated vertices and a second component."""
    edges = [(0, 1), (1, 2), (2, 0), (2, 3), (3, 3), (4, 2), (5, 6), (6, 5), (1, 3), (0, 3)]
    n = 10
    src = [a for a, b in edges]
    dst = [b for a, b in edges]
    # keep the self loop (3,3) in the file: PageRank reads it with SkipRing
    keys = sorted(set(edges))
    off = np.zeros(n + 1, np.int32)
    idx = np.array([b for a, b in keys], np.int32)
    for a, b in keys:
        off[a + 1] += 1
    off = np.cumsum(off).astype(np.int32)
    return n, off, idx, src, dst


def bp_graph():
    """A sparse seeded directed graph (in-degree at most 10), where two rounds
    of the reference's unnormalised FP32 products stay in the normal range."""
    rng = np.random.default_rng(7)
    n, m = 3000, 9000
    return O.graph_from_edges(n, rng.integers(0, n, m), rng.integers(0, n, m))


def bp_fixture(d):
    """numa-BP with its inputs set and its products printed (numa-BP-result,
    oracle/ref_patch_bp.py), one thread, after 1 and 2 rounds."""
    g = bp_graph()
    base = O.write_binary(g, os.path.join(d, "bp"))
    p1, _ = O.ref_bp_result(base, 1)
    p2, _ = O.ref_bp_result(base, 2)
    np.savez_compressed(os.path.join(HERE, "bp_sparse.npz"), off=g.off, idx=g.idx, prod1=p1, prod2=p2)
    return g.n, g.m


def main():
    if not O.ref_available():
        O.build()
    d = O.tempdir()
    out = {}
    if sys.argv[1:] == ["bp"]:
        print("bp_sparse          n=%d m=%d" % bp_fixture(d))
        return
    out["bp_sparse"] = bp_fixture(d)

    # --- directed scale-10 R-MAT: PageRank, SpMV ---------------------------
    g = O.rmat_graph(10, 16)
    base = os.path.join(d, "rmat10")
    base = O.write_binary(g, base)
    pr, _ = O.ref_pagerank(base, 10, threads=4)
    w = O.weights_int(g, wmax=5)
    tpath = os.path.join(d, "rmat10w.txt")
    O.write_text(g, tpath, w)
    sp, _ = O.ref_spmv(tpath, 5, threads=4)
    np.savez_compressed(os.path.join(HERE, "rmat10_directed.npz"), off=g.off, idx=g.idx,
                        pagerank10=pr, spmv_w=w, spmv5=sp)
    out["rmat10_directed"] = (g.n, g.m)

    # --- directed scale-10 R-MAT: PageRankDelta, 3 and 10 rounds ----------
    prd3, _ = O.ref_pagerank_delta(base, 3, threads=4)
    prd10, _ = O.ref_pagerank_delta(base, 10, threads=4)
    np.savez_compressed(os.path.join(HERE, "rmat10_prdelta.npz"), off=g.off, idx=g.idx,
                        prdelta3=prd3, prdelta10=prd10)
    out["rmat10_prdelta"] = (g.n, g.m)

    # --- symmetric scale-10 R-MAT: CC, BFS parents -------------------------
    gs = O.rmat_graph(10, 16, symmetric=True)
    bs = os.path.join(d, "rmat10s")
    bs = O.write_binary(gs, bs)
    cc, _ = O.ref_components(bs, threads=4)
    srcs = O.pick_sources(gs, 3)
    parents, counts = [], []
    for s in srcs:
        par, cnt, _ = O.ref_bfs(bs, int(s), threads=4)
        parents.append(par)
        counts.append(cnt)
    np.savez_compressed(os.path.join(HERE, "rmat10_symmetric.npz"), off=gs.off, idx=gs.idx, cc=cc,
                        bfs_sources=srcs, bfs_parents=np.stack(parents),
                        bfs_counts=np.array(counts, np.int64))
    out["rmat10_symmetric"] = (gs.n, gs.m)

    # --- hand-built edge cases (self loop kept in the file) ----------------
    n, off, idx, _, _ = tiny_graph()
    tg = O.Graph(n, off, idx)
    tb = os.path.join(d, "tiny")
    tb = O.write_binary(tg, tb)
    tpr, _ = O.ref_pagerank(tb, 6, threads=2)
    np.savez_compressed(os.path.join(HERE, "tiny.npz"), off=off, idx=idx, pagerank6=tpr)
    out["tiny"] = (n, len(idx))
    for k, v in out.items():
        print("%-18s n=%d m=%d" % (k, *v))


if __name__ == "__main__":
    main()
