"""The multi-rank partition path on CPU: two `gloo` ranks (world size 2,
127.0.0.1) exchange uneven vertex ranges through
polymer_b200.distributed.allgather_v (an empty range included), and run
PageRank on a 1D partition -- each rank reduces only its own rows with the
reference's frontier semantics (numa-PageRank.C PR_F / PR_Vertex_F /
PR_Vertex_Reset) and the contributions and frontier are gathered after
every pass -- which must equal the oracle's whole-graph PageRank, and
Components by min-label propagation with labels and frontier gathered after
every round -- the oracle's labels, both ranks ending in the same round.  The
ranges come from partition_bounds, the host restatement of the library's
cut rule.  No GPU is used."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _pagerank_partitioned(og, bounds, rank, ex, iters, damping=0.85):
    n = og.n
    deg = np.diff(og.off).astype(np.int64)
    src = np.repeat(np.arange(n), deg)
    lo, hi = int(bounds[rank]), int(bounds[rank + 1])
    own = (og.idx >= lo) & (og.idx < hi)
    s_own, d_own = src[own], og.idx[own].astype(np.int64)
    rows = np.arange(lo, hi)
    pc, pn = np.full(n, 1.0 / n), np.zeros(n)
    c = np.where(deg > 0, pc / np.maximum(deg, 1), 0.0)
    in_f = np.ones(n, np.uint8)  # the frontier: every vertex at the start
    added = (1.0 - damping) / n
    for _ in range(iters):
        act = in_f[s_own] == 1
        acc = np.zeros(n)
        np.add.at(acc, d_own[act], c[s_own[act]])
        hit = np.zeros(n, bool)
        hit[d_own[act]] = True
        nb = pn[rows] + acc[rows]
        f = in_f[rows] == 1
        nb[f] = damping * nb[f] + added  # PR_Vertex_F on frontier vertices
        pc[rows[f]] = 0.0                # PR_Vertex_Reset
        pn[rows] = nb
        c_next, f_next = np.zeros(n), np.zeros(n, np.uint8)
        c_next[rows] = np.where(hit[rows], np.where(deg[rows] > 0, nb / np.maximum(deg[rows], 1), 0.0), 0.0)
        f_next[rows] = hit[rows]
        ex(c_next.ctypes.data, 8, list(bounds), None)
        ex(f_next.ctypes.data, 1, list(bounds), None)
        pc, pn, c, in_f = pn, pc, c_next, f_next
    ex(pc.ctypes.data, 8, list(bounds), None)
    return pc


def _components_partitioned(og, bounds, rank, ex):
    """Min-label propagation (numa-Components.C CC_F) over this rank's rows:
    labels and the frontier are gathered after every round; every rank sees
    the same global frontier, so all stop in the same round."""
    n = og.n
    deg = np.diff(og.off).astype(np.int64)
    src = np.repeat(np.arange(n), deg)
    lo, hi = int(bounds[rank]), int(bounds[rank + 1])
    own = (og.idx >= lo) & (og.idx < hi)
    s_own, d_own = src[own], og.idx[own].astype(np.int64)
    labels = np.arange(n, dtype=np.int32)
    front = np.ones(n, np.uint8)
    rounds = 0
    while front.any():
        act = front[s_own] == 1
        best = labels.copy()
        np.minimum.at(best, d_own[act], labels[s_own[act]])
        nxt = np.zeros(n, np.uint8)
        changed = best[lo:hi] < labels[lo:hi]
        labels[lo:hi] = best[lo:hi]
        nxt[lo:hi] = changed
        ex(labels.ctypes.data, 4, list(bounds), None)
        ex(nxt.ctypes.data, 1, list(bounds), None)
        front = nxt
        rounds += 1
    return labels, rounds


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import pm_oracle
        from polymer_b200 import ROW_WORK
        from polymer_b200.distributed import allgather_v, partition_bounds
        ex = allgather_v(device="cpu")
        # uneven ranges, rank 0's empty
        a = np.full(100, -1, np.int32)
        a[0:100] = np.arange(100) if rank == 1 else -1
        ex(a.ctypes.data, 4, [0, 0, 100], None)
        ok_empty = bool(np.array_equal(a, np.arange(100)))
        b = np.full(70, -1, np.int64)
        b[[slice(0, 64), slice(64, 70)][rank]] = np.arange(70)[[slice(0, 64), slice(64, 70)][rank]] * 3
        ex(b.ctypes.data, 8, [0, 64, 70], None)
        ok_uneven = bool(np.array_equal(b, np.arange(70) * 3))
        og = pm_oracle.rmat_graph(10, 16)
        bounds = partition_bounds(og.off, og.idx, world, row_work=ROW_WORK)
        pr = _pagerank_partitioned(og, bounds, rank, ex, 8)
        want = pm_oracle.pagerank(og, 8)
        sym = pm_oracle.rmat_graph(11, 8, symmetric=True)
        sb = partition_bounds(sym.off, sym.idx, world, row_work=ROW_WORK)
        lab, rounds = _components_partitioned(sym, sb, rank, ex)
        same_cc = bool(np.array_equal(lab, pm_oracle.cc(sym)))
        q.put((rank, ok_empty, ok_uneven, bounds.tolist(), bool(np.allclose(pr, want, rtol=1e-10, atol=0)),
               same_cc, rounds))
    finally:
        dist.destroy_process_group()


def test_partitioned_pagerank_and_components_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=240) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][3] == res[1][3]  # both ranks cut the same ranges
    lo, mid, hi = res[0][3]
    assert lo == 0 and 0 < mid < hi and mid % 32 == 0
    for rank, ok_empty, ok_uneven, _, same, same_cc, rounds in res:
        assert ok_empty and ok_uneven and same and same_cc
    assert res[0][6] == res[1][6] > 1  # both ranks ended in the same round
