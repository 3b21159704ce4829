"""GPU tests of the 1D vertex partition (pm_graph_create_partition): one
graph spread over P ranks, each holding the edges whose destination lies in
its vertex range, with the ranges exchanged after every pass.  The P ranks
run as host threads on one GPU (partition_local.LocalGroup); every rank's
result must be the whole graph's result, checked against the oracle:
PageRank and SpMV (FP64) to 1e-10, BFS depths, Components labels and
BellmanFord distances exactly, BP bit for bit against the whole graph."""
import numpy as np
import pytest

from partition_local import LocalGroup
from polymer_b200.distributed import partition_bounds

pytestmark = pytest.mark.gpu


def _part(pm, og, rank, nranks, ex, **kw):
    return pm.Graph.partition(og.off, og.idx, rank, nranks, ex, **kw)


@pytest.mark.parametrize("nranks", [1, 2, 3])
def test_pagerank_spmv_directed(pm, oracle, nranks):
    og = oracle.rmat_graph(13, 16)
    w = oracle.weights_unit(og)
    x0 = oracle.uniform01(og.n)
    want_pr = oracle.pagerank(og, 10)
    want_y = oracle.spmv(og, w, x0, 6)

    def body(rank, ex):
        with _part(pm, og, rank, nranks, ex, weights=w) as g:
            return pm.PageRank(g, 10), pm.SPMV(g, x0, 6, dtype=np.float64), g.partition_info()

    for pr, y, (rank, k, b) in LocalGroup(nranks).run(body):
        assert k == nranks
        assert np.allclose(pr, want_pr, rtol=1e-10, atol=0)
        assert np.allclose(y, want_y, rtol=1e-10, atol=1e-300)


@pytest.mark.parametrize("nranks", [2, 3])
def test_bp_bit_identical(pm, oracle, nranks):
    """BP's pull sums integer counts of frontier in-neighbours, so a partition
    gives the whole graph's log-products bit for bit (FP32 and FP64)."""
    og = oracle.rmat_graph(13, 16)
    prior = oracle.uniform_open(2 * og.n).reshape(-1, 2).astype(np.float32)
    with pm.Graph.from_csr(og.off, og.idx) as g:
        want32 = pm.BeliefPropagation(g, prior, 7)
        want64 = pm.BeliefPropagation(g, prior.astype(np.float64), 7, dtype=np.float64)

    def body(rank, ex):
        with _part(pm, og, rank, nranks, ex) as g:
            return (pm.BeliefPropagation(g, prior, 7),
                    pm.BeliefPropagation(g, prior.astype(np.float64), 7, dtype=np.float64))

    for b32, b64 in LocalGroup(nranks).run(body):
        assert np.array_equal(b32, want32) and np.array_equal(b64, want64)


@pytest.mark.parametrize("nranks", [2, 4])
def test_traversals_symmetric(pm, oracle, nranks):
    og = oracle.rmat_graph(13, 16, symmetric=True)
    w = oracle.weights_int(og)
    srcs = [int(s) for s in oracle.pick_sources(og, 2)]
    want_cc = oracle.cc(og)
    want_d = [oracle.bfs(og, s)[0] for s in srcs]
    want_bf = oracle.dijkstra(og, w, srcs[0])

    def body(rank, ex):
        with _part(pm, og, rank, nranks, ex, weights=w) as g:
            bfs = [pm.BFS(s, g) for s in srcs]
            return bfs, pm.Components(g), pm.BellmanFord(g, srcs[0])

    for bfs, lab, dist in LocalGroup(nranks).run(body):
        assert np.array_equal(lab, want_cc)
        assert np.array_equal(dist, want_bf)
        for s, (par, dep), wd in zip(srcs, bfs, want_d):
            assert np.array_equal(dep, wd)
            v = np.nonzero(dep > 0)[0]  # every parent is an in-neighbour one level up
            assert np.all(dep[par[v]] == dep[v] - 1) and par[s] == s


def test_heavy_rows_and_thresholds(pm, oracle):
    """Rows above the heavy cut-off are chunked inside a rank's range, and
    both traversal directions (threshold 0: dense, huge: sparse) agree."""
    og = oracle.rmat_graph(14, 16, symmetric=True)
    s = int(oracle.pick_sources(og, 1)[0])
    want_cc, want_d = oracle.cc(og), oracle.bfs(og, s)[0]
    want_pr = oracle.pagerank(og, 5)

    def body(rank, ex):
        with _part(pm, og, rank, 3, ex) as g:
            g.set_tunable("heavy_deg", 64)
            out = [pm.PageRank(g, 5)]
            for thr in (0, 1 << 40):
                out.append(pm.Components(g, threshold=thr))
                out.append(pm.BFS(s, g, threshold=thr)[1])
            return out

    for pr, cc0, d0, cc1, d1 in LocalGroup(3).run(body):
        assert np.allclose(pr, want_pr, rtol=1e-10, atol=0)
        assert np.array_equal(cc0, want_cc) and np.array_equal(cc1, want_cc)
        assert np.array_equal(d0, want_d) and np.array_equal(d1, want_d)


def test_bounds_follow_the_cut_rule(pm, oracle):
    og = oracle.rmat_graph(14, 16)
    nranks = 4

    def body(rank, ex):
        with _part(pm, og, rank, nranks, ex) as g:
            r, k, b = g.partition_info()
            off, idx = g.csr()
            return r, b, int(idx.size), bool(np.all((idx >= b[r]) & (idx < b[r + 1])))

    res = LocalGroup(nranks).run(body)
    want = partition_bounds(og.off, og.idx, nranks, row_work=pm.ROW_WORK)
    assert sum(x[2] for x in res) == og.m  # every edge on exactly one rank
    for r, b, m_r, inside in res:
        assert np.array_equal(b, want) and inside
        assert np.all(b[1:-1] % 32 == 0)


def test_whole_graph_calls_refused_and_exchange_errors(pm, oracle):
    og = oracle.rmat_graph(10, 8)

    def body(rank, ex):
        with _part(pm, og, rank, 2, ex) as g:
            with pytest.raises(pm.PolymerError) as ei:
                pm.PersonalizedPageRank(g, [0], 2)
            assert ei.value.status == 6
        return True

    assert all(LocalGroup(2).run(body))

    def failing(buf, elem_bytes, bounds, stream):
        raise RuntimeError("exchange failed on purpose (host side)")

    with pm.Graph.partition(og.off, og.idx, 0, 2, failing) as g:
        with pytest.raises(pm.PolymerError) as ei:
            pm.PageRank(g, 3)
        assert ei.value.status == 3
        # the handle stays usable: a working exchange (rank 1 absent: one rank
        # of a 2-rank group cannot finish) is not needed to query it
        assert g.partition_info()[1] == 2
