"""GPU tests of the asynchronous BFS (pm_bfs_async, numa-BFS-async-pipe.C):
the reached set equals BFS reachability from the oracle, the parents form a
valid tree rooted at the source (every parent edge exists, no cycles), and
the counts match.  Edge cases: an isolated source, a hub split into many
queue chunks, directed and symmetric graphs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def check_tree(oracle, og, src, parents):
    ref, _ = oracle.bfs(og, src)
    reached = ref >= 0
    assert np.array_equal(parents >= 0, reached)
    assert parents[src] == src
    v = np.nonzero(reached & (np.arange(og.n) != src))[0]
    p = parents[v]
    # every parent edge p -> v exists in the CSR (rows are sorted)
    lo = og.off[p]
    hi = og.off[p + 1]
    pos = np.array([np.searchsorted(og.idx[a:b], x) for a, b, x in zip(lo[:50000], hi[:50000], v[:50000])])
    assert np.all(og.idx[lo[:50000] + pos] == v[:50000])
    oracle.bfs_depths_from_parents(parents, src)  # raises on a cycle or a chain that misses src
    return reached


@pytest.mark.parametrize("scale,sym", [(14, False), (15, True), (20, True)])
def test_async_bfs_reaches_what_bfs_reaches(pm, oracle, scale, sym):
    og = oracle.rmat_graph(scale, 16, symmetric=sym)
    deg = og.out_degree()
    with pm.Graph.from_csr(og.off, og.idx, symmetric=sym) as g:
        for s in oracle.pick_sources(og, 3, seed=0x5EED0031):
            par, st = pm.BFSAsync(int(s), g, stats=True)
            reached = check_tree(oracle, og, int(s), par)
            assert st["reached"] == reached.sum()
            assert st["edges_visited"] == deg[reached].sum()


def test_async_bfs_isolated_source_and_hub(pm, oracle):
    # vertex 0 -> 1..10000 (five queue chunks), 1..10000 -> 10001, 10002 isolated
    n = 10003
    src = np.concatenate([np.zeros(10000, np.int64), np.arange(1, 10001)])
    dst = np.concatenate([np.arange(1, 10001), np.full(10000, 10001)])
    og = oracle.graph_from_edges(n, src, dst)
    with pm.Graph.from_csr(og.off, og.idx) as g:
        par, st = pm.BFSAsync(10002, g, stats=True)
        assert st["reached"] == 1 and par[10002] == 10002 and (par >= 0).sum() == 1
        par, st = pm.BFSAsync(0, g, stats=True)
        reached = check_tree(oracle, og, 0, par)
        assert reached.sum() == 10002 and st["reached"] == 10002
        assert np.all(par[1:10001] == 0) and 1 <= par[10001] <= 10000


def test_async_bfs_long_chain(pm, oracle):
    # one item in flight at a time: every warp's batch of slots waits for the chain
    n = 2000
    og = oracle.graph_from_edges(n, np.arange(n - 1), np.arange(1, n))
    with pm.Graph.from_csr(og.off, og.idx) as g:
        par, st = pm.BFSAsync(0, g, stats=True)
        assert st["reached"] == n and par[0] == 0 and np.array_equal(par[1:], np.arange(n - 1))
