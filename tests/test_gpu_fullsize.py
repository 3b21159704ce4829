"""GPU parity at the benchmark's full sizes: every workload the benchmark
times, on the same seeded inputs, against the CPU oracle (oracle/pm_oracle.c,
FP64 / exact integers).  Slow: the oracle runs its value loops over all host
cores (OpenMP) and the independent oracle computations of a graph run on a
thread pool (its C calls release the GIL) while the GPU computes.

  symmetrised R-MAT scale 22 (graph A): the generator (CSR and int32 weights
    U{1..22}) bit-identical to the oracle's; BFS depths from all 16 seeded
    sources the benchmark uses (pmo_bfs); Components labels (pmo_cc);
    BellmanFord from the first source, dense rounds pulled and pushed
    (pmo_dijkstra: exact shortest paths); 64-source BFS and BellmanFord with
    the benchmark's 64 sources, 8 lanes each against the oracle.
  directed R-MAT scale 24 (graph B): the generator, weights U(0,1] and the
    inputs x0 U[0,1), priors U(0,1) bit-identical to the oracle's; PageRank
    20 iterations FP32 (pmo_pagerank), SpMV 10 iterations (pmo_spmv), BP 10
    iterations (pmo_bp) within relative L1 1e-5 of the FP64 oracle, with the
    max-abs error printed; PPR with the benchmark's 32 seeds, 4 columns
    against pmo_ppr.
  256 Erdos-Renyi graphs, n log-uniform in [1k, 100k], average degree 8: the
    batch generator and PageRank of every part (pmo_pagerank per part)."""
import concurrent.futures as cf

import numpy as np
import pytest

import bench

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

RL1_F32 = 1e-5  # relative L1 of FP32 storage and sums against the FP64 oracle


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


def max_abs(a, b):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max())


@pytest.fixture(scope="module")
def pool():
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        yield ex


@pytest.fixture(scope="module")
def graph_a(pm, oracle):
    """(device graph, oracle graph, weights, the benchmark's 16 sources)."""
    og = oracle.rmat_graph(22, 16, seed=bench.SEED_GRAPH, symmetric=True)
    w = oracle.weights_int(og, seed=bench.SEED_W, wmax=22)
    g = pm.Graph.rmat(22, 16, seed=bench.SEED_GRAPH, symmetric=True)
    g.gen_weights_int(bench.SEED_W, 22)
    yield g, og, w, bench.pick_sources(og.off, 16, bench.SEED_SRC)
    g.close()


@pytest.fixture(scope="module")
def graph_b(pm, oracle):
    og = oracle.rmat_graph(24, 16, seed=bench.SEED_GRAPH)
    g = pm.Graph.rmat(24, 16, seed=bench.SEED_GRAPH)
    g.gen_weights_unit(bench.SEED_W)
    yield g, og
    g.close()


def test_graph_a_generator_and_weights(graph_a):
    g, og, w, _ = graph_a
    off, idx = g.csr()
    assert g.n == 1 << 22 and g.m == og.m
    assert np.array_equal(off, og.off) and np.array_equal(idx, og.idx)
    assert np.array_equal(g.weights_i32(), w)


def test_bfs_all_benchmark_sources_scale22(pm, oracle, graph_a, pool):
    g, og, _, srcs = graph_a
    assert len(srcs) == 16
    refs = [pool.submit(oracle.bfs, og, s) for s in srcs]
    for s, fut in zip(srcs, refs):
        parents, depth = pm.BFS(s, g)
        want = fut.result()[0]
        assert np.array_equal(depth, want), "source %d" % s
        # every parent one level up along an existing edge
        v = np.nonzero((depth > 0))[0]
        assert np.all(depth[parents[v]] == depth[v] - 1)


def test_components_scale22(pm, oracle, graph_a, pool):
    g, og, _, _ = graph_a
    ref = pool.submit(oracle.cc, og)
    assert np.array_equal(pm.Components(g), ref.result())


@pytest.mark.parametrize("bf_dense", [0, 1, 2])
def test_bellman_ford_scale22(pm, oracle, graph_a, pool, bf_dense):
    g, og, w, srcs = graph_a
    ref = pool.submit(oracle.dijkstra, og, w, srcs[0])
    before = g.get_tunable("bf_dense")
    g.set_tunable("bf_dense", bf_dense)
    try:
        d = pm.BellmanFord(g, srcs[0])
    finally:
        g.set_tunable("bf_dense", before)
    assert np.array_equal(d, ref.result())


def test_batched_bfs_and_bellman_ford_scale22(pm, oracle, graph_a, pool):
    g, og, w, _ = graph_a
    src64 = bench.pick_sources(og.off, 64, bench.SEED_SRC + 100)
    lanes = [0, 9, 17, 30, 41, 52, 60, 63]
    ref_bfs = {l: pool.submit(oracle.bfs, og, src64[l]) for l in lanes}
    ref_bf = {l: pool.submit(oracle.dijkstra, og, w, src64[l]) for l in lanes[:4]}
    dep = pm.BFSMulti(src64, g)
    for l in lanes:
        assert np.array_equal(dep[l], ref_bfs[l].result()[0]), "BFS lane %d" % l
    del dep
    dist = pm.BellmanFordMulti(src64, g)
    for l in lanes[:4]:
        assert np.array_equal(dist[l], ref_bf[l].result()), "BellmanFord lane %d" % l


def test_graph_b_generator_and_inputs(pm, oracle, graph_b):
    g, og = graph_b
    off, idx = g.csr()
    assert g.n == 1 << 24 and g.m == og.m
    assert np.array_equal(off, og.off) and np.array_equal(idx, og.idx)
    assert np.array_equal(g.weights_f32(), oracle.weights_unit(og, seed=bench.SEED_W))
    x_dev = pm.uniform_f32(g, g.n, bench.SEED_X).cpu().numpy()
    assert np.array_equal(x_dev, oracle.uniform01(g.n, bench.SEED_X))
    p_dev = pm.uniform_f32(g, 2 * g.n, bench.SEED_PRIOR, open_interval=True).cpu().numpy()
    assert np.array_equal(p_dev, oracle.uniform_open(2 * g.n, bench.SEED_PRIOR))


def test_value_algorithms_scale24(pm, oracle, graph_b, pool):
    """PageRank 20, SpMV 10 and BP 10 iterations in FP32 at scale 24 against
    the FP64 oracle: relative L1 below 1e-5; max-abs printed beside the
    largest magnitude."""
    g, og = graph_b
    n = g.n
    w = oracle.weights_unit(og, seed=bench.SEED_W)
    x0 = oracle.uniform01(n, bench.SEED_X)
    prior = oracle.uniform_open(2 * n, bench.SEED_PRIOR).reshape(n, 2)
    f_pr = pool.submit(oracle.pagerank, og, 20)
    f_spmv = pool.submit(oracle.spmv, og, w.astype(np.float64), x0.astype(np.float64), 10)
    f_bp = pool.submit(oracle.bp, og, prior.astype(np.float64), 10)
    pr = pm.PageRank(g, 20, dtype=np.float32)
    y = pm.SPMV(g, x0, 10)
    lp = pm.BeliefPropagation(g, prior, 10)
    for name, got, fut in (("PageRank", pr, f_pr), ("SpMV", y, f_spmv), ("BP", lp, f_bp)):
        ref = fut.result()
        err = rel_l1(got, ref)
        print("%s scale 24 FP32: rel-L1 %.3g, max-abs %.3g (max |ref| %.3g)" %
              (name, err, max_abs(got, ref), float(np.abs(ref).max())))
        assert err < RL1_F32, (name, err)


def test_ppr_scale24(pm, oracle, graph_b, pool):
    g, og = graph_b
    seeds = bench.pick_sources(og.off, 32, bench.SEED_SRC + 200)
    cols = [0, 11, 22, 31]
    ref = pool.submit(oracle.ppr, og, [seeds[c] for c in cols], 20)
    out = pm.PersonalizedPageRank(g, seeds, 20)
    assert out.shape == (g.n, 32)
    r = ref.result()
    for j, c in enumerate(cols):
        err = rel_l1(out[:, c], r[:, j])
        print("PPR column %d: rel-L1 %.3g" % (c, err))
        assert err < RL1_F32, (c, err)


def test_er_batch_256_parts(pm, oracle, pool):
    og, vbase = oracle.er_batch(256, 1000, 100000, 8)
    assert len(vbase) == 257
    sizes = np.diff(vbase)
    assert sizes.min() >= 1000 and sizes.max() <= 100000
    refs = []
    for i in range(256):
        sub = oracle.subgraph(og, int(vbase[i]), int(vbase[i + 1]))
        refs.append(pool.submit(oracle.pagerank, sub, 20))
    with pm.Graph.er_batch(256, 1000, 100000, 8) as g:
        off, idx = g.csr()
        assert np.array_equal(g.parts(), vbase)
        assert np.array_equal(off, og.off) and np.array_equal(idx, og.idx)
        ranks = pm.PageRankParts(g, 20)
    for i in range(256):
        assert rel_l1(ranks[vbase[i]:vbase[i + 1]], refs[i].result()) < RL1_F32, i
