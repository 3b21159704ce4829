"""GPU parity: the CUDA engine (through the C ABI) against the CPU oracle on
the same seeded inputs.  Integer results are compared bit-exactly; floating
point within the tolerances stated per test."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

RTOL_F64 = 1e-10     # PageRank FP64 (reference prints %.9e)
RL1_F32 = 1e-5       # relative L1 vs the FP64 oracle for FP32 storage/sums


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def dev_graph(pm, og, symmetric=False, skip=False):
    return pm.Graph.from_csr(og.off, og.idx, symmetric=symmetric, skip_self_loops=skip)


def check_parents(og, src, parents, depth):
    n = og.n
    assert parents[src] == src and depth[src] == 0
    reached = depth >= 0
    assert np.array_equal(reached, parents >= 0)
    v = np.nonzero(reached & (np.arange(n) != src))[0]
    p = parents[v]
    assert np.all(depth[p] == depth[v] - 1), "parent one level up"
    # the edge p -> v exists in the CSR
    for a, b in zip(p[:20000], v[:20000]):
        row = og.idx[og.off[a]:og.off[a + 1]]
        k = np.searchsorted(row, b)
        assert k < len(row) and row[k] == b


# --------------------------------------------------------------------------
def test_rmat_generator_matches_oracle(pm, oracle):
    for scale, ef, sym in ((8, 4, False), (10, 16, True), (14, 16, False), (13, 16, True)):
        og = oracle.rmat_graph(scale, ef, symmetric=sym)
        with pm.Graph.rmat(scale, ef, symmetric=sym) as g:
            off, idx = g.csr()
            assert g.n == og.n and g.m == og.m
            assert np.array_equal(off, og.off) and np.array_equal(idx, og.idx)


def test_graph_create_skip_self_loops(pm, oracle):
    z = load("tiny.npz")
    with pm.Graph.from_csr(z["off"], z["idx"], skip_self_loops=True) as g:
        off, idx = g.csr()
    n = len(z["off"]) - 1
    src = np.repeat(np.arange(n), np.diff(z["off"]))
    keep = src != z["idx"]
    og = oracle.graph_from_edges(n, src[keep], z["idx"][keep])
    assert np.array_equal(off, og.off) and np.array_equal(idx, og.idx)


def test_bad_graph_rejected(pm):
    with pytest.raises(pm.PolymerError) as ei:
        pm.Graph.from_csr(np.array([0, 2, 1], np.int32), np.array([1, 0], np.int32))
    assert ei.value.status == 5
    with pytest.raises(pm.PolymerError):
        pm.Graph.from_csr(np.array([0, 1, 2], np.int32), np.array([1, 7], np.int32))


# --------------------------------------------------------------------------
def test_pagerank_f64_matches_reference_fixture(pm, oracle):
    z = load("rmat10_directed.npz")
    with pm.Graph.from_csr(z["off"], z["idx"]) as g:
        r = pm.PageRank(g, 10, dtype=np.float64)
    assert np.allclose(r, z["pagerank10"], rtol=2e-9, atol=0)


def test_pagerank_tiny_skip_ring_fixture(pm):
    z = load("tiny.npz")
    with pm.Graph.from_csr(z["off"], z["idx"], skip_self_loops=True) as g:
        r = pm.PageRank(g, 6, dtype=np.float64)
    assert np.allclose(r, z["pagerank6"], rtol=2e-9, atol=1e-300)


def test_pagerank_rejects_self_loops(pm):
    z = load("tiny.npz")
    with pm.Graph.from_csr(z["off"], z["idx"]) as g:
        with pytest.raises(pm.PolymerError):
            pm.PageRank(g, 3)


def test_pagerank_config1_f64(pm, oracle):
    """2^16 vertices, edge factor 16, 10 iterations, FP64 (the reference's CPU-sized case)."""
    og = oracle.rmat_graph(16, 16)
    ref, res_ref = oracle.pagerank(og, 10, with_resid=True)
    with pm.Graph.rmat(16, 16) as g:
        r, res = pm.PageRank(g, 10, dtype=np.float64, resid=True)
    assert np.allclose(r, ref, rtol=RTOL_F64, atol=0)
    assert np.allclose(res, res_ref, rtol=1e-9)


def test_pagerank_f32_rel_l1(pm, oracle):
    og = oracle.rmat_graph(18, 16)
    ref = oracle.pagerank(og, 20)
    with pm.Graph.rmat(18, 16) as g:
        r = pm.PageRank(g, 20, dtype=np.float32)
    assert rel_l1(r, ref) < RL1_F32
    assert np.max(np.abs(r - ref) / np.maximum(ref, 1e-30)) < 1e-3


def test_pagerank_deterministic(pm):
    with pm.Graph.rmat(14, 16) as g:
        a = pm.PageRank(g, 7, dtype=np.float32)
        b = pm.PageRank(g, 7, dtype=np.float32)
    assert np.array_equal(a, b)


# --------------------------------------------------------------------------
@pytest.mark.parametrize("threshold", [-1, 0, 1 << 40])
@pytest.mark.parametrize("sym", [True, False])
def test_bfs_depths_exact(pm, oracle, threshold, sym):
    og = oracle.rmat_graph(13, 16, symmetric=sym)
    with dev_graph(pm, og, symmetric=sym) as g:
        for s in oracle.pick_sources(og, 4, seed=0x5EED0005 + sym):
            parents, depth = pm.BFS(int(s), g, threshold=threshold)
            ref, _ = oracle.bfs(og, int(s))
            assert np.array_equal(depth, ref)
            check_parents(og, int(s), parents, depth)


def test_bfs_reference_fixture(pm, oracle):
    z = load("rmat10_symmetric.npz")
    og = oracle.Graph(len(z["off"]) - 1, z["off"], z["idx"])
    with dev_graph(pm, og, symmetric=True) as g:
        for s, par, cnt in zip(z["bfs_sources"], z["bfs_parents"], z["bfs_counts"]):
            _, depth = pm.BFS(int(s), g, threshold=0)   # the reference's always-dense rule
            assert np.array_equal(depth, oracle.bfs_depths_from_parents(par, int(s)))
            assert (depth >= 0).sum() == cnt


def test_bfs_isolated_source_and_heavy_rows(pm, oracle):
    # star: vertex 0 -> 1..5000 (heavy row), 5001 isolated
    n = 5002
    og = oracle.graph_from_edges(n, np.zeros(5000, np.int64), np.arange(1, 5001))
    with dev_graph(pm, og) as g:
        parents, depth, st = pm.BFS(5001, g, stats=True)
        assert depth[5001] == 0 and (depth >= 0).sum() == 1 and st["reached"] == 1
        for thr in (-1, 0, 1 << 40):
            parents, depth = pm.BFS(0, g, threshold=thr)
            assert np.all(depth[1:5001] == 1) and depth[5001] == -1 and np.all(parents[1:5001] == 0)


def test_bfs_sparse_hubs(pm, oracle):
    """Forced sparse rounds on a graph whose hubs exceed the grid-expansion
    degree, and a complete bipartite graph with more hubs than one round can
    hand to the grid kernel (the rest take the CTA path)."""
    og = oracle.rmat_graph(16, 16, symmetric=True)
    assert og.out_degree().max() > 4096
    with dev_graph(pm, og, symmetric=True) as g:
        for s in oracle.pick_sources(og, 3, seed=99):
            parents, depth = pm.BFS(int(s), g, threshold=1 << 40)
            assert np.array_equal(depth, oracle.bfs(og, int(s))[0])
            check_parents(og, int(s), parents, depth)
    a = 4100
    left = np.repeat(np.arange(a), a)
    right = np.tile(np.arange(a, 2 * a), a)
    kb = oracle.graph_from_edges(2 * a, left, right, symmetric=True)
    with dev_graph(pm, kb, symmetric=True) as g:
        for thr in (1 << 40, -1):
            parents, depth, st = pm.BFS(0, g, threshold=thr, stats=True)
            assert np.all(depth[1:a] == 2) and np.all(depth[a:] == 1) and depth[0] == 0
            assert st["reached"] == 2 * a
            assert np.all((parents[1:a] >= a)) and np.all(parents[a:] == 0)


# --------------------------------------------------------------------------
@pytest.mark.parametrize("threshold", [-1, 0, 1 << 40])
@pytest.mark.parametrize("sym,k", [(True, 64), (False, 64), (True, 5)])
def test_bfs_multi_matches_single_source(pm, oracle, threshold, sym, k):
    og = oracle.rmat_graph(13, 16, symmetric=sym)
    srcs = oracle.pick_sources(og, k, seed=0x5EED0015)
    if k == 64:
        srcs[7] = srcs[3]  # a repeated source must give identical rows
    with dev_graph(pm, og, symmetric=sym) as g:
        dep, st = pm.BFSMulti(srcs, g, threshold=threshold, stats=True)
    reached, edges = 0, 0
    deg = og.out_degree()
    for l, s in enumerate(srcs):
        ref, _ = oracle.bfs(og, int(s))
        assert np.array_equal(dep[l], ref), "source %d (lane %d)" % (s, l)
        reached += (ref >= 0).sum()
        edges += deg[ref >= 0].sum()
    assert st["reached"] == reached and st["edges_visited"] == edges


@pytest.mark.parametrize("threshold", [-1, 0])
def test_bfs_multi_long_paths(pm, oracle, threshold):
    """Hundreds of levels (more than the level words kept between depth
    writes): a directed path 0 -> 1 -> ... -> 299 plus a separate 40-vertex
    cycle, sources at both ends, inside, repeated, and on the cycle."""
    n_path, n_cyc = 300, 40
    n = n_path + n_cyc
    src = np.r_[np.arange(n_path - 1), n_path + np.arange(n_cyc)]
    dst = np.r_[np.arange(1, n_path), n_path + (np.arange(n_cyc) + 1) % n_cyc]
    off = np.zeros(n + 1, np.int32)
    np.add.at(off, src + 1, 1)
    off = np.cumsum(off).astype(np.int32)
    idx = dst[np.argsort(src, kind="stable")].astype(np.int32)
    og = oracle.Graph(n, off, idx)
    srcs = [0, 299, 150, 0, n_path + 7, 17, 1]
    with pm.Graph.from_csr(off, idx) as g:
        dep, st = pm.BFSMulti(srcs, g, threshold=threshold, stats=True)
    for l, s in enumerate(srcs):
        assert np.array_equal(dep[l], oracle.bfs(og, s)[0]), "lane %d" % l
    assert st["rounds"] == n_path  # the longest walk (from 0) ends after 299 levels, plus the empty one


def test_bfs_multi_device_out(pm, oracle):
    import torch
    og = oracle.rmat_graph(12, 16, symmetric=True)
    srcs = oracle.pick_sources(og, 64)
    with dev_graph(pm, og, symmetric=True) as g:
        out = torch.empty((64, og.n), dtype=torch.int32, device="cuda")
        dep = pm.BFSMulti(srcs, g, device_out=out, out=out)
        assert dep.is_cuda
        ref = pm.BFSMulti(srcs, g)
    assert np.array_equal(dep.cpu().numpy(), ref)


# --------------------------------------------------------------------------
@pytest.mark.parametrize("cc_mode", [0, 1])
@pytest.mark.parametrize("threshold", [-1, 0, 1 << 40])
def test_components_exact(pm, oracle, threshold, cc_mode):
    """Mode 0: union-find on symmetric graphs; mode 1: the reference's label
    propagation in every direction regime.  Directed graphs always propagate."""
    for sym, scale in ((True, 13), (False, 12)):
        og = oracle.rmat_graph(scale, 8, symmetric=sym)
        with dev_graph(pm, og, symmetric=sym) as g:
            g.set_tunable("cc_mode", cc_mode)
            lab, st = pm.Components(g, threshold=threshold, stats=True)
        assert np.array_equal(lab, oracle.cc(og))
        if sym and cc_mode == 0:
            assert st["dense_rounds"] == 0 and st["edges_visited"] <= og.m


def test_components_union_find_shapes(pm, oracle):
    """Union-find against the oracle on shapes that stress linking: a long
    path under a random vertex order (deep trees before compression), stars
    whose centre has the largest id, many equal components (the sampled
    largest component is one of several), isolated vertices."""
    rng = np.random.default_rng(5)
    n = 40000
    perm = rng.permutation(n)
    src, dst = [], []
    path = perm[:20000]                       # one path over 20000 shuffled ids
    src.append(path[:-1]); dst.append(path[1:])
    for k in range(20):                       # 20 stars of 400 leaves, centre = largest id
        ids = np.sort(perm[20000 + 500 * k: 20000 + 500 * k + 401])
        src.append(np.full(400, ids[-1])); dst.append(ids[:-1])
    for k in range(50):                       # 50 rings of 20 vertices
        ids = perm[30100 + 20 * k: 30100 + 20 * k + 20]
        src.append(ids); dst.append(np.roll(ids, 1))
    og = oracle.graph_from_edges(n, np.concatenate(src), np.concatenate(dst), symmetric=True)
    want = oracle.cc(og)
    with dev_graph(pm, og, symmetric=True) as g:
        for mode in (0, 1):
            g.set_tunable("cc_mode", mode)
            for _ in range(3):
                assert np.array_equal(pm.Components(g), want), mode


def test_components_reference_fixture(pm, oracle):
    z = load("rmat10_symmetric.npz")
    with pm.Graph.from_csr(z["off"], z["idx"], symmetric=True) as g:
        assert np.array_equal(pm.Components(g), z["cc"])


# --------------------------------------------------------------------------
@pytest.mark.parametrize("threshold", [-1, 0, 1 << 40])
def test_bellman_ford_exact(pm, oracle, threshold):
    for sym, scale in ((True, 12), (False, 12)):
        og = oracle.rmat_graph(scale, 16, symmetric=sym)
        w = oracle.weights_int(og)
        with dev_graph(pm, og, symmetric=sym) as g:
            g.set_weights(w)
            for s in oracle.pick_sources(og, 3):
                d = pm.BellmanFord(g, int(s), threshold=threshold)
                assert np.array_equal(d, oracle.dijkstra(og, w, int(s)))


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("threshold", [-1, 0])
def test_bellman_ford_dense_push_exact(pm, oracle, threshold, mode):
    """Dense rounds pushed over the frontier's out-edges: mode 1 through
    edgeMap's DENSE_FORWARD push (k_dense_push, k_heavy_push for rows above
    the heavy cut-off), the option the reference's BellmanFord passes
    (numa-BellmanFord.C:182); mode 2 with atomics whose result is unused and
    the next frontier from the distances that fell (k_bf_push_red,
    k_bf_heavy_red, k_bf_fell).  Distances equal Dijkstra's on R-MAT graphs
    of both kinds, with the heavy cut-off at its default and lowered so that
    the chunk kernels run."""
    for sym, scale in ((True, 13), (False, 13)):
        og = oracle.rmat_graph(scale, 16, symmetric=sym)
        w = oracle.weights_int(og)
        for heavy in (1024, 64):
            with dev_graph(pm, og, symmetric=sym) as g:
                g.set_weights(w)
                g.set_tunable("bf_dense", mode)
                g.set_tunable("heavy_deg", heavy)
                for s in oracle.pick_sources(og, 3):
                    d, st = pm.BellmanFord(g, int(s), threshold=threshold, stats=True)
                    assert np.array_equal(d, oracle.dijkstra(og, w, int(s)))
                    if threshold == 0:
                        assert st["dense_rounds"] == st["rounds"]


@pytest.mark.parametrize("bf_dense", [0, 1, 2])
@pytest.mark.parametrize("delta", [1, 4, 16, 1 << 20])
def test_bellman_ford_delta_stepping_exact(pm, oracle, delta, bf_dense):
    """The delta-stepping schedule (bf_delta): only frontier vertices below a
    moving bound relax each round; distances equal Dijkstra's in every
    direction regime, dense rounds pulled or pushed, on both graph kinds and
    on a hub graph; a huge Delta is the plain schedule."""
    n = 12288
    src = np.concatenate([np.arange(1, n), np.zeros(n - 1, np.int64), np.arange(1, n - 1)])
    dst = np.concatenate([np.zeros(n - 1, np.int64), np.arange(1, n), np.arange(2, n)])
    hub = oracle.graph_from_edges(n, src, dst)
    for og, sym in ((oracle.rmat_graph(13, 16, symmetric=True), True), (oracle.rmat_graph(13, 16), False),
                    (hub, False)):
        w = oracle.weights_int(og)
        with dev_graph(pm, og, symmetric=sym) as g:
            g.set_weights(w)
            g.set_tunable("bf_delta", delta)
            g.set_tunable("bf_dense", bf_dense)
            for s in [int(v) for v in oracle.pick_sources(og, 2)]:
                want = oracle.dijkstra(og, w, s)
                for thr in (-1, 0, 1 << 40):
                    assert np.array_equal(pm.BellmanFord(g, s, threshold=thr), want), (delta, thr, s)


@pytest.mark.parametrize("mode", [1, 2])
def test_bellman_ford_dense_push_hub(pm, oracle, mode):
    """A hub of in- and out-degree 12287 on a ring (three heavy chunks per
    direction, a ragged last chunk): every round dense, pushed."""
    n = 12288
    src = np.concatenate([np.arange(1, n), np.zeros(n - 1, np.int64), np.arange(1, n - 1)])
    dst = np.concatenate([np.zeros(n - 1, np.int64), np.arange(1, n), np.arange(2, n)])
    og = oracle.graph_from_edges(n, src, dst)
    w = oracle.weights_int(og)
    with dev_graph(pm, og) as g:
        g.set_weights(w)
        g.set_tunable("bf_dense", mode)
        for s in (5, 0, 7000, 12287):
            assert np.array_equal(pm.BellmanFord(g, s, threshold=0), oracle.dijkstra(og, w, s))


def _bf_multi_check(pm, oracle, og, sym, srcs, threshold, heavy_deg=None):
    w = oracle.weights_int(og)
    with dev_graph(pm, og, symmetric=sym) as g:
        g.set_weights(w)
        if heavy_deg is not None:
            g.set_tunable("heavy_deg", heavy_deg)
        dist, st = pm.BellmanFordMulti(srcs, g, threshold=threshold, stats=True)
    reached = 0
    for l, s in enumerate(srcs):
        ref = oracle.dijkstra(og, w, int(s))
        assert np.array_equal(dist[l], ref), "source %d (lane %d)" % (s, l)
        reached += (ref < pm.BF_INF).sum()
    assert st["reached"] == reached


@pytest.mark.parametrize("threshold", [-1, 0, 1 << 40])
@pytest.mark.parametrize("sym,k", [(True, 64), (False, 64), (True, 5)])
def test_bellman_ford_multi_matches_dijkstra(pm, oracle, threshold, sym, k):
    # scale 14 has one row above the heavy-row degree in either direction
    og = oracle.rmat_graph(14, 16, symmetric=sym)
    srcs = oracle.pick_sources(og, k, seed=0x5EED0016)
    if k == 64:
        srcs[9] = srcs[2]  # a repeated source must give identical rows
    _bf_multi_check(pm, oracle, og, sym, srcs, threshold)


@pytest.mark.parametrize("threshold", [-1, 0])
def test_bellman_ford_multi_heavy_pieces(pm, oracle, threshold):
    # heavy rows from in-degree 64: most dense-round work goes through the
    # 512-edge pieces and their atomicMin updates
    og = oracle.rmat_graph(14, 16, symmetric=True)
    srcs = oracle.pick_sources(og, 64, seed=0x5EED0017)
    _bf_multi_check(pm, oracle, og, True, srcs, threshold, heavy_deg=64)


@pytest.mark.parametrize("threshold", [-1, 0, 1 << 40])
def test_bellman_ford_multi_hub(pm, oracle, threshold):
    # a hub of in-degree 12287 (three heavy chunks, a ragged last piece) on a
    # ring: lanes fall along the ring and through the hub in the same rounds
    n = 12288
    src = np.concatenate([np.arange(1, n), np.zeros(n - 1, np.int64), np.arange(1, n - 1)])
    dst = np.concatenate([np.zeros(n - 1, np.int64), np.arange(1, n), np.arange(2, n)])
    og = oracle.graph_from_edges(n, src, dst)
    srcs = np.array([5, 0, 7000, 12287, 5, 300, 11111], np.int32)
    _bf_multi_check(pm, oracle, og, False, srcs, threshold)


def test_device_weights_match_oracle(pm, oracle):
    og = oracle.rmat_graph(12, 16, symmetric=True)
    with pm.Graph.rmat(12, 16, symmetric=True) as g:
        g.gen_weights_int()
        assert np.array_equal(g.weights_i32(), oracle.weights_int(og))
        g.gen_weights_unit()
        assert np.array_equal(g.weights_f32(), oracle.weights_unit(og))


# --------------------------------------------------------------------------
def test_spmv_integer_weights_reference_fixture(pm):
    z = load("rmat10_directed.npz")
    n = len(z["off"]) - 1
    with pm.Graph.from_csr(z["off"], z["idx"]) as g:
        g.set_weights(z["spmv_w"].astype(np.float32))
        y = pm.SPMV(g, np.full(n, 1.0 / n, np.float32), 5)
    assert rel_l1(y, z["spmv5"]) < RL1_F32


def test_spmv_f32_rel_l1(pm, oracle):
    og = oracle.rmat_graph(16, 16)
    w = oracle.weights_unit(og)
    x0 = oracle.uniform01(og.n)
    ref = oracle.spmv(og, w.astype(np.float64), x0.astype(np.float64), 10)
    with dev_graph(pm, og) as g:
        g.set_weights(w)
        y, norms = pm.SPMV(g, x0, 10, norms=True)
    assert rel_l1(y, ref) < RL1_F32
    assert abs(norms[-1] / np.abs(ref).sum() - 1) < RL1_F32


def test_spmv_f64_matches_oracle_and_reference(pm, oracle):
    """FP64 vectors and sums: elementwise against the FP64 oracle, and against
    the reference's printed output (%.9e) on its integer-weight fixture."""
    og = oracle.rmat_graph(16, 16)
    w = oracle.weights_unit(og)
    x0 = oracle.uniform01(og.n)
    ref = oracle.spmv(og, w.astype(np.float64), x0.astype(np.float64), 10)
    with dev_graph(pm, og) as g:
        g.set_weights(w)
        y, norms = pm.SPMV(g, x0.astype(np.float64), 10, norms=True, dtype=np.float64)
        y32 = pm.SPMV(g, x0, 10)
    assert y.dtype == np.float64 and np.allclose(y, ref, rtol=RTOL_F64, atol=0)
    assert abs(norms[-1] / np.abs(ref).sum() - 1) < 1e-12
    assert rel_l1(y32, y) < RL1_F32
    z = load("rmat10_directed.npz")
    n = len(z["off"]) - 1
    with pm.Graph.from_csr(z["off"], z["idx"]) as g:
        g.set_weights(z["spmv_w"].astype(np.float32))
        y = pm.SPMV(g, np.full(n, 1.0 / n), 5, dtype=np.float64)
    assert np.allclose(y, z["spmv5"], rtol=2e-9, atol=0)


# --------------------------------------------------------------------------
RL1_PRD_F32 = 1e-5   # FP32 PageRankDelta (measured 1.1e-7 at scale 16; a vertex within FP32
                     # rounding of |Delta| = eps2 * p could take the other side of the test)


@pytest.mark.parametrize("threshold", [0, -1, 1 << 40])
def test_pagerank_delta_f64_matches_oracle(pm, oracle, threshold):
    og = oracle.rmat_graph(14, 16)
    ref, fs = oracle.pagerank_delta(og, 10, with_frontier=True)
    with dev_graph(pm, og) as g:
        p, st = pm.PageRankDelta(g, 10, dtype=np.float64, threshold=threshold, stats=True)
    assert np.allclose(p, ref, rtol=1e-9, atol=1e-15)
    assert st["rounds"] == 10 and st["reached"] == fs[-1]
    if threshold == 0:
        assert st["dense_rounds"] == 10   # the reference's threshold 0: every round pulls
    if threshold == 1 << 40:
        assert st["dense_rounds"] == 1    # only the first round, which commits every vertex


def test_pagerank_delta_reference_fixture(pm):
    z = load("rmat10_prdelta.npz")
    with pm.Graph.from_csr(z["off"], z["idx"]) as g:
        for iters, key in ((3, "prdelta3"), (10, "prdelta10")):
            p = pm.PageRankDelta(g, iters, dtype=np.float64, threshold=0)
            assert np.allclose(p, z[key], rtol=2e-9, atol=0), key


def test_pagerank_delta_f32_rel_l1(pm, oracle):
    og = oracle.rmat_graph(16, 16)
    ref = oracle.pagerank_delta(og, 10)
    with dev_graph(pm, og) as g:
        for thr in (0, -1):
            p = pm.PageRankDelta(g, 10, dtype=np.float32, threshold=thr)
            err = rel_l1(p, ref)
            print("PageRankDelta FP32 threshold %d rel-L1 %.3g" % (thr, err))
            assert err < RL1_PRD_F32, err
        with pytest.raises(pm.PolymerError):
            pm.PageRankDelta(g, 0)


@pytest.mark.parametrize("k", [32, 3])
def test_ppr_matches_oracle(pm, oracle, k):
    og = oracle.rmat_graph(14, 16)
    seeds = oracle.pick_sources(og, k, seed=0x5EED0025)
    ref = oracle.ppr(og, seeds, 20)
    with dev_graph(pm, og) as g:
        out = pm.PersonalizedPageRank(g, seeds, 20)
    assert out.shape == (og.n, k)
    for j in range(k):
        assert rel_l1(out[:, j], ref[:, j]) < RL1_F32, j
    with dev_graph(pm, og) as g:
        assert np.array_equal(pm.PersonalizedPageRank(g, seeds, 0)[seeds, np.arange(k)], np.ones(k))


def test_ppr_heavy_rows(pm, oracle):
    # star into vertex 0 from 5000 sources (a heavy CSC row) plus a chain
    n = 6000
    src = np.concatenate([np.arange(1, 5001), np.arange(5001, 5999)])
    dst = np.concatenate([np.zeros(5000, np.int64), np.arange(5002, 6000)])
    og = oracle.graph_from_edges(n, np.concatenate([src, [0]]), np.concatenate([dst, [5001]]))
    seeds = [1, 2, 5001, 0]
    ref = oracle.ppr(og, seeds, 15)
    with dev_graph(pm, og) as g:
        out = pm.PersonalizedPageRank(g, seeds, 15)
    for j in range(len(seeds)):
        assert rel_l1(out[:, j], ref[:, j]) < RL1_F32


def test_er_batch_generator_and_parts_pagerank(pm, oracle):
    og, vbase = oracle.er_batch(24, 100, 3000, 8, seed=77)
    with pm.Graph.er_batch(24, 100, 3000, 8, seed=77) as g:
        off, idx = g.csr()
        assert np.array_equal(g.parts(), vbase)
        assert np.array_equal(off, og.off) and np.array_equal(idx, og.idx)
        ranks = pm.PageRankParts(g, 20)
    for i in range(24):
        sub = oracle.subgraph(og, int(vbase[i]), int(vbase[i + 1]))
        ref = oracle.pagerank(sub, 20)
        assert rel_l1(ranks[vbase[i]:vbase[i + 1]], ref) < RL1_F32, i


def test_parts_from_user_graph(pm, oracle):
    # two R-MAT graphs side by side as one union, parts declared by the caller
    a = oracle.rmat_graph(10, 8)
    b = oracle.rmat_graph(11, 8, seed=5)
    off = np.concatenate([a.off[:-1], b.off + a.m]).astype(np.int32)
    idx = np.concatenate([a.idx, b.idx + a.n]).astype(np.int32)
    with pm.Graph.from_csr(off, idx) as g:
        g.set_parts([0, a.n, a.n + b.n])
        ranks = pm.PageRankParts(g, 12)
        with pytest.raises(pm.PolymerError):
            g.set_parts([0, 100, a.n + b.n])  # edges cross this split
    assert rel_l1(ranks[:a.n], oracle.pagerank(a, 12)) < RL1_F32
    assert rel_l1(ranks[a.n:], oracle.pagerank(b, 12)) < RL1_F32


# --------------------------------------------------------------------------
def test_bp_matches_oracle(pm, oracle):
    og = oracle.rmat_graph(14, 16)
    prior = oracle.uniform_open(2 * og.n).reshape(og.n, 2)
    ref = oracle.bp(og, prior.astype(np.float64), 10)
    with dev_graph(pm, og) as g:
        out = pm.BeliefPropagation(g, prior, 10)
    err = np.abs(out - ref).sum() / max(np.abs(ref).sum(), 1e-30)
    assert err < RL1_F32, err


def test_bp_f64_matches_oracle(pm, oracle):
    og = oracle.rmat_graph(14, 16)
    prior = oracle.uniform_open(2 * og.n).reshape(og.n, 2).astype(np.float64)
    ref = oracle.bp(og, prior, 10)
    with dev_graph(pm, og) as g:
        out = pm.BeliefPropagation(g, prior, 10, dtype=np.float64)
        out_dev = pm.BeliefPropagation(g, __import__("torch").from_numpy(prior).cuda(), 10,
                                       dtype=np.float64)
    assert out.dtype == np.float64
    assert np.allclose(out, ref, rtol=1e-9, atol=1e-12)
    assert np.array_equal(out_dev.cpu().numpy(), out)


# --------------------------------------------------------------------------
def test_empty_and_single_vertex_graphs(pm, oracle):
    with pm.Graph.from_csr(np.array([0, 0], np.int32), np.zeros(0, np.int32)) as g:
        p, d = pm.BFS(0, g)
        assert d.tolist() == [0] and p.tolist() == [0]
        assert pm.Components(g).tolist() == [0]
        assert np.allclose(pm.PageRank(g, 3), [0.15])
    off = np.zeros(101, np.int32)
    with pm.Graph.from_csr(off, np.zeros(0, np.int32)) as g:
        assert np.array_equal(pm.Components(g), np.arange(100))
        _, d = pm.BFS(7, g)
        assert (d >= 0).sum() == 1


def test_edgeless_graph_all_paths(pm, tmp_path):
    """Every path on 100 vertices and no edges: the batched, asynchronous,
    PageRankDelta, weighted and ingest paths included."""
    n = 100
    off = np.zeros(n + 1, np.int32)
    none = np.zeros(0, np.int32)
    with pm.Graph.from_csr(off, none, weights=none) as g:
        srcs = [3, 50, 99]
        assert np.array_equal(pm.BFSMulti(srcs, g), np.where(np.arange(n)[None, :] == np.array(srcs)[:, None], 0, -1))
        d = pm.BellmanFordMulti(srcs, g)
        assert np.array_equal(d, np.where(np.arange(n)[None, :] == np.array(srcs)[:, None], 0, pm.BF_INF))
        par, st = pm.BFSAsync(7, g, stats=True)
        assert st["reached"] == 1 and (par >= 0).sum() == 1 and par[7] == 7
        p = pm.PageRankDelta(g, 3, dtype=np.float64)
        assert np.allclose(p, 0.15 / n)  # first round: (1-d)/n; later rounds: no in-edges
        x = pm.PersonalizedPageRank(g, [0, 5], 4)
        assert np.allclose(x[0, 0], 0.15) and np.allclose(x[5, 1], 0.15) and x.sum() == pytest.approx(0.3, rel=1e-6)
    path = tmp_path / "none.adj"
    path.write_text("AdjacencyGraph\n%d\n0\n" % n + "0\n" * n)
    with pm.Graph.load_pbbs(str(path)) as g:
        assert g.n == n and g.m == 0


def test_device_pointers_roundtrip(pm, oracle):
    import torch
    og = oracle.rmat_graph(12, 16, symmetric=True)
    off = torch.from_numpy(og.off).cuda()
    idx = torch.from_numpy(og.idx).cuda()
    torch.cuda.synchronize()
    with pm.Graph.from_csr(off, idx, symmetric=True) as g:
        lab = pm.Components(g, device_out=off)
        assert lab.is_cuda and np.array_equal(lab.cpu().numpy(), oracle.cc(og))
        par, dep = pm.BFS(int(oracle.pick_sources(og, 1)[0]), g, device_out=off)
        assert dep.is_cuda


def test_kernel_launch_counter(pm):
    with pm.Graph.rmat(10, 8) as g:
        pm.kernel_launches(reset=True)
        pm.PageRank(g, 5, dtype=np.float32)
        assert pm.kernel_launches() >= 5


def test_bp_on_reference_pinned_inputs(pm, oracle):
    """The graph and priors the patched reference BP was run on
    (tests/golden/bp_sparse.npz): the GPU's FP64 log-products equal the log of
    the reference formula with each message divided by its sum
    (pmo_bp_raw normalize), whose unnormalised form the fixture pins to the
    reference's own output."""
    z = load("bp_sparse.npz")
    og = oracle.Graph(len(z["off"]) - 1, z["off"], z["idx"])
    prior = oracle.bp_ref_priors(og.n)
    with dev_graph(pm, og) as g:
        for it in (1, 2, 4):
            lp = pm.BeliefPropagation(g, prior.astype(np.float64), it, dtype=np.float64)
            want = oracle.bp_raw(og, prior.astype(np.float64), it, normalize=True)
            assert np.allclose(np.exp(lp), want, rtol=1e-9, atol=0), it
            lp32 = pm.BeliefPropagation(g, prior, it)
            assert rel_l1(lp32, np.log(want)) < RL1_F32, it
