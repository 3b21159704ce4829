"""GPU tests of the run-time tunables, the autotuner and the CUDA-graph capture
of the fixed-iteration loops, through the C ABI: results never depend on them
(integer results bit-exact against the oracle; the FP32 pulls reduce in a
fixed order, so PageRank / SpMV / BP / PPR are bit-identical with and without
CUDA graphs)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RL1_F32 = 1e-5


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


def _fp_runs(pm, g, x0, prior):
    return (pm.PageRank(g, 7, dtype=np.float32), pm.PageRank(g, 4, dtype=np.float64),
            pm.SPMV(g, x0, 5), pm.BeliefPropagation(g, prior, 3),
            pm.PersonalizedPageRank(g, [3, 77, 1000], 6))


def test_cuda_graphs_bit_identical(pm):
    with pm.Graph.rmat(15, 16) as g:
        g.gen_weights_unit()
        x0 = pm.uniform_f32(g, g.n, 11).cpu().numpy()
        prior = pm.uniform_f32(g, 2 * g.n, 12, open_interval=True).cpu().numpy()
        assert g.get_tunable("cuda_graphs") == 1
        pm.SPMV(g, x0, 1)  # builds the paired weights once, outside the counts
        pm.kernel_launches(reset=True)
        on = _fp_runs(pm, g, x0, prior)
        on2 = _fp_runs(pm, g, x0, prior)  # replays of the captured loops
        l_on = pm.kernel_launches(reset=True)
        g.set_tunable("cuda_graphs", 0)
        off = _fp_runs(pm, g, x0, prior)
        off2 = _fp_runs(pm, g, x0, prior)
        l_off = pm.kernel_launches(reset=True)
    for a, b, c, d in zip(on, on2, off, off2):
        assert np.array_equal(a, b) and np.array_equal(a, c) and np.array_equal(a, d)
    assert l_on == l_off  # a replayed graph counts the kernels it holds


def test_cuda_graphs_profile_counts_passes(pm):
    with pm.Graph.rmat(14, 16) as g:
        g.profile(True)
        for _ in range(3):
            pm.PageRank(g, 5, dtype=np.float32)
        ms, passes = g.profile_read("pagerank", reset=True)
        assert passes == 15 and ms > 0
        g.set_tunable("cuda_graphs", 0)
        pm.PageRank(g, 5, dtype=np.float32)
        assert g.profile_read("pagerank", reset=True)[1] == 5


@pytest.mark.parametrize("fused", [0, 1, 2])
@pytest.mark.parametrize("heavy", [64, 1024, 4096, 1 << 30])
def test_heavy_degree_results_unchanged(pm, oracle, heavy, fused):
    og = oracle.rmat_graph(14, 16)
    ref = oracle.pagerank(og, 10)
    sym = oracle.rmat_graph(13, 16, symmetric=True)
    w = oracle.weights_int(sym)
    srcs = oracle.pick_sources(sym, 3, seed=0x5EED0021)
    with pm.Graph.from_csr(og.off, og.idx) as g:
        g.set_tunable("heavy_mode", fused)
        g.set_tunable("heavy_deg", heavy)
        assert g.get_tunable("heavy_deg") == heavy
        assert rel_l1(pm.PageRank(g, 10, dtype=np.float32), ref) < RL1_F32
        a = pm.PageRank(g, 10, dtype=np.float64)
        assert np.allclose(a, oracle.pagerank(og, 10), rtol=1e-10, atol=0)
        g.gen_weights_unit()
        x0 = oracle.uniform01(og.n)
        ys = oracle.spmv(og, oracle.weights_unit(og).astype(np.float64), x0.astype(np.float64), 5)
        assert rel_l1(pm.SPMV(g, x0, 5), ys) < RL1_F32
        assert np.array_equal(pm.SPMV(g, x0, 5), pm.SPMV(g, x0, 5))   # fixed reduction order
        g.set_tunable("heavy_deg", 2048)
        assert rel_l1(pm.PageRank(g, 10, dtype=np.float32), ref) < RL1_F32
    with pm.Graph.from_csr(sym.off, sym.idx, symmetric=True) as g:
        g.set_weights(w)
        g.set_tunable("heavy_mode", fused)
        g.set_tunable("heavy_deg", heavy)
        assert np.array_equal(pm.Components(g), oracle.cc(sym))
        for s in srcs:
            _, depth = pm.BFS(int(s), g)
            assert np.array_equal(depth, oracle.bfs(sym, int(s))[0])
            assert np.array_equal(pm.BellmanFord(g, int(s)), oracle.dijkstra(sym, w, int(s)))
        dist = pm.BellmanFordMulti(srcs, g)
        for l, s in enumerate(srcs):
            assert np.array_equal(dist[l], oracle.dijkstra(sym, w, int(s)))


@pytest.mark.parametrize("cta,grid", [(32, 32), (32, 100000), (2048, 2048), (100000, 100000)])
def test_sparse_push_bins_results_unchanged(pm, oracle, cta, grid):
    sym = oracle.rmat_graph(15, 16, symmetric=True)
    srcs = oracle.pick_sources(sym, 3, seed=0x5EED0022)
    with pm.Graph.from_csr(sym.off, sym.idx, symmetric=True) as g:
        g.set_tunable("cta_expand", cta)
        g.set_tunable("grid_expand", grid)
        for s in srcs:
            _, depth = pm.BFS(int(s), g, threshold=1 << 40)   # every round sparse
            assert np.array_equal(depth, oracle.bfs(sym, int(s))[0])
        assert np.array_equal(pm.Components(g, threshold=1 << 40), oracle.cc(sym))


@pytest.mark.parametrize("div", [1, 3, 1 << 20])
def test_direction_divisors(pm, oracle, div):
    sym = oracle.rmat_graph(13, 16, symmetric=True)
    w = oracle.weights_int(sym)
    s = int(oracle.pick_sources(sym, 1, seed=0x5EED0023)[0])
    with pm.Graph.from_csr(sym.off, sym.idx, symmetric=True) as g:
        g.set_weights(w)
        for k in ("bfs_div", "cc_div", "bf_div"):
            g.set_tunable(k, div)
        _, depth, st = pm.BFS(s, g, stats=True)
        assert np.array_equal(depth, oracle.bfs(sym, s)[0])
        if div == 1:
            assert st["dense_rounds"] < st["rounds"]  # m/1: dense only when |F| + outdeg(F) >= m
        assert np.array_equal(pm.Components(g), oracle.cc(sym))
        assert np.array_equal(pm.BellmanFord(g, s), oracle.dijkstra(sym, w, s))


def test_tunable_range_checks(pm):
    with pm.Graph.rmat(10, 8) as g:
        for name, bad in (("heavy_deg", 10), ("cta_expand", 0), ("pull_ctas_per_sm", -1),
                          ("bfs_div", 0), ("cuda_graphs", 2), ("bf_dense", 3),
                          ("cc_mode", -1), ("bf_delta", -1), ("pull_stage", 2), ("push_agg", -1)):
            before = g.get_tunable(name)
            with pytest.raises(pm.PolymerError) as ei:
                g.set_tunable(name, bad)
            assert ei.value.status == 1 and g.get_tunable(name) == before
        with pytest.raises(pm.PolymerError):
            pm._check(pm.lib().pm_graph_set_tunable(g.handle, 99, 1))


@pytest.mark.parametrize("app", ["pagerank", "spmv", "bp", "bfs", "cc", "bellman_ford"])
def test_autotuner_keeps_results(pm, oracle, app):
    sym = app in ("bfs", "cc", "bellman_ford")
    og = oracle.rmat_graph(15, 16, symmetric=sym)
    with pm.Graph.from_csr(og.off, og.idx, symmetric=sym) as g:
        if app == "spmv":
            g.gen_weights_unit()
        if app == "bellman_ford":
            w = oracle.weights_int(og)
            g.set_weights(w)
        rep = g.tune(app)
        assert rep["trials"] >= 3 and 0 < rep["best_ms"] <= rep["default_ms"]
        if app == "pagerank":
            assert rel_l1(pm.PageRank(g, 10, dtype=np.float32), oracle.pagerank(og, 10)) < RL1_F32
        elif app == "bfs":
            s = int(oracle.pick_sources(og, 1)[0])
            assert np.array_equal(pm.BFS(s, g)[1], oracle.bfs(og, s)[0])
        elif app == "cc":
            assert np.array_equal(pm.Components(g), oracle.cc(og))
        elif app == "bellman_ford":
            s = int(oracle.pick_sources(og, 1)[0])
            assert np.array_equal(pm.BellmanFord(g, s), oracle.dijkstra(og, w, s))


def test_defaults_apply_to_new_graphs(pm, oracle):
    og = oracle.rmat_graph(14, 16)
    ref = oracle.pagerank(og, 10)
    try:
        pm.set_default_tunable("heavy_deg", 256)
        pm.set_default_tunable("cuda_graphs", 0)
        with pm.Graph.from_csr(og.off, og.idx) as g:
            assert g.get_tunable("heavy_deg") == 256 and g.get_tunable("cuda_graphs") == 0
            assert rel_l1(pm.PageRank(g, 10, dtype=np.float32), ref) < RL1_F32
    finally:
        pm.set_default_tunable("heavy_deg", 1024)
        pm.set_default_tunable("cuda_graphs", 1)
    with pm.Graph.from_csr(og.off, og.idx) as g:
        assert g.get_tunable("heavy_deg") == 1024


def test_autotuner_mix_keeps_results(pm, oracle):
    sym = oracle.rmat_graph(15, 16, symmetric=True)
    w = oracle.weights_int(sym)
    s = int(oracle.pick_sources(sym, 1, seed=0x5EED0024)[0])
    with pm.Graph.from_csr(sym.off, sym.idx, symmetric=True) as g:
        g.set_weights(w)
        rep = g.tune(["bfs", "cc", "bellman_ford"])
        assert rep["trials"] >= 7 and 0 < rep["best_ms"] <= rep["default_ms"]
        assert np.array_equal(pm.BFS(s, g)[1], oracle.bfs(sym, s)[0])
        assert np.array_equal(pm.Components(g), oracle.cc(sym))
        assert np.array_equal(pm.BellmanFord(g, s), oracle.dijkstra(sym, w, s))
    with pytest.raises(pm.PolymerError):
        with pm.Graph.rmat(10, 8) as g:
            pm._check(pm.lib().pm_tune_mix(g.handle, None, 1, None))


def test_caller_stream(pm, oracle):
    import torch
    og = oracle.rmat_graph(13, 16)
    ref = oracle.pagerank(og, 5)
    s = torch.cuda.Stream()
    with pm.Graph.from_csr(og.off, og.idx) as g:
        g.set_stream(s)
        for _ in range(3):  # runs directly, captures, replays on the caller's stream
            assert np.allclose(pm.PageRank(g, 5), ref, rtol=1e-10, atol=0)
        _, depth = pm.BFS(0, g)
        g.set_stream(None)
        assert np.allclose(pm.PageRank(g, 5), ref, rtol=1e-10, atol=0)
        assert np.array_equal(pm.BFS(0, g)[1], depth)


def test_heavy_mode_overlapped_is_bit_identical(pm):
    """Mode 2 sums the same chunks with the same kernel on a second stream and
    folds them in the same order: results equal mode 0 bit for bit, with and
    without CUDA-graph capture (the fork/join of the two streams is captured)."""
    with pm.Graph.rmat(15, 16) as g:
        g.gen_weights_unit()
        g.set_tunable("heavy_deg", 256)
        x0 = pm.uniform_f32(g, g.n, 21).cpu().numpy()
        prior = pm.uniform_f32(g, 2 * g.n, 22, open_interval=True).cpu().numpy()
        base = _fp_runs(pm, g, x0, prior)
        g.set_tunable("heavy_mode", 2)
        for graphs in (1, 0):
            g.set_tunable("cuda_graphs", graphs)
            for _ in range(3):
                got = _fp_runs(pm, g, x0, prior)
                for a, b in zip(base, got):
                    assert np.array_equal(a, b)


@pytest.mark.parametrize("scale", [10, 15])
def test_pull_stage_bit_identical(pm, oracle, scale):
    """Staged ids (one bulk copy of a batch's CSC ids into shared memory) read
    the same ids in the same order: every pull-reduce result is unchanged bit
    for bit, with batches staged, batches too long to stage and the last ids of
    the array (read from global memory) all on the path."""
    og = oracle.rmat_graph(scale, 16)
    sym = oracle.rmat_graph(scale, 16, symmetric=True)
    w = oracle.weights_int(sym)
    srcs = oracle.pick_sources(sym, 2, seed=0x5EED0025)
    with pm.Graph.from_csr(og.off, og.idx) as g:
        prior = pm.uniform_f32(g, 2 * g.n, 12, open_interval=True).cpu().numpy()
        runs = []
        for st in (0, 1, 0, 1):
            g.set_tunable("pull_stage", st)
            runs.append((pm.PageRank(g, 7, dtype=np.float32), pm.PageRank(g, 4, dtype=np.float64),
                         pm.BeliefPropagation(g, prior, 3)))
        for r in runs[1:]:
            for a, b in zip(runs[0], r):
                assert np.array_equal(a, b)
        assert rel_l1(runs[1][0], oracle.pagerank(og, 7)) < RL1_F32
    with pm.Graph.from_csr(sym.off, sym.idx, symmetric=True) as g:
        g.set_weights(w)
        g.set_tunable("cc_mode", 1)  # label propagation: dense rounds pull-reduce
        g.set_tunable("pull_stage", 1)
        assert np.array_equal(pm.Components(g), oracle.cc(sym))
        for s in srcs:
            assert np.array_equal(pm.BellmanFord(g, int(s)), oracle.dijkstra(sym, w, int(s)))


@pytest.mark.parametrize("scale", [11, 15])
def test_push_agg_results_unchanged(pm, oracle, scale):
    """Warp-aggregated atomicMin pushes (one atomic per target per warp) give
    the labels and distances of one atomic per edge: every round sparse, and
    with the default direction switch."""
    sym = oracle.rmat_graph(scale, 16, symmetric=True)
    w = oracle.weights_int(sym)
    srcs = oracle.pick_sources(sym, 3, seed=0x5EED0026)
    with pm.Graph.from_csr(sym.off, sym.idx, symmetric=True) as g:
        g.set_weights(w)
        g.set_tunable("cc_mode", 1)
        g.set_tunable("push_agg", 1)
        assert g.get_tunable("push_agg") == 1
        for thr in (1 << 40, -1):
            assert np.array_equal(pm.Components(g, threshold=thr), oracle.cc(sym))
            for s in srcs:
                assert np.array_equal(pm.BellmanFord(g, int(s), threshold=thr), oracle.dijkstra(sym, w, int(s)))
