"""GPU tests of the hub cache of the FP32 PageRank pull (hub_cache tunable):
the contributions of the highest out-degree sources are read from shared
memory, so every result must be bit-identical to the pull without it -- for
several cache sizes, directed and symmetric graphs, with and without captured
loops, on a partition, and on graphs too small to have hubs."""
import numpy as np
import pytest

from partition_local import LocalGroup

pytestmark = pytest.mark.gpu


def _pr(pm, g, hub, iters=9):
    g.set_tunable("hub_cache", hub)
    return pm.PageRank(g, iters, dtype=np.float32)


@pytest.mark.parametrize("sym", [False, True])
def test_results_bit_identical(pm, oracle, sym):
    og = oracle.rmat_graph(16, 16, symmetric=sym)
    with pm.Graph.from_csr(og.off, og.idx, symmetric=sym) as g:
        assert g.get_tunable("hub_cache") >= 0
        base = _pr(pm, g, 0)
        for hub in (1, 100, 8192, 16384, 0, 16384):
            assert np.array_equal(_pr(pm, g, hub), base), hub
            assert np.array_equal(_pr(pm, g, hub), base), hub  # replay of the captured loop
        g.set_tunable("cuda_graphs", 0)
        assert np.array_equal(_pr(pm, g, 16384), base)
        want = oracle.pagerank(og, 9)
        assert np.sum(np.abs(base - want)) / np.sum(np.abs(want)) < 1e-5


@pytest.mark.parametrize("heavy", [64, 2048])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_with_heavy_rows(pm, oracle, heavy, mode):
    og = oracle.rmat_graph(15, 16)
    with pm.Graph.from_csr(og.off, og.idx) as g:
        g.set_tunable("heavy_deg", heavy)
        g.set_tunable("heavy_mode", mode)
        base = _pr(pm, g, 0, 5)
        assert np.array_equal(_pr(pm, g, 4096, 5), base)


def test_tiny_and_edgeless(pm):
    off = np.array([0, 2, 3, 3], np.int32)
    idx = np.array([1, 2, 0], np.int32)
    with pm.Graph.from_csr(off, idx) as g:
        assert np.array_equal(_pr(pm, g, 16384, 4), _pr(pm, g, 0, 4))
    with pm.Graph.from_csr(np.zeros(9, np.int32), np.zeros(0, np.int32)) as g:
        assert np.array_equal(_pr(pm, g, 16384, 3), _pr(pm, g, 0, 3))


def test_partition_with_hubs(pm, oracle):
    og = oracle.rmat_graph(14, 16)
    with pm.Graph.from_csr(og.off, og.idx) as g:
        g.set_tunable("hub_cache", 0)
        whole = pm.PageRank(g, 6, dtype=np.float32)

    def body(rank, ex):
        with pm.Graph.partition(og.off, og.idx, rank, 2, ex) as g:
            g.set_tunable("hub_cache", 2048)
            return pm.PageRank(g, 6, dtype=np.float32)

    for r in LocalGroup(2).run(body):
        assert np.allclose(r, whole, rtol=1e-6, atol=1e-12)


def test_range_checked(pm):
    with pm.Graph.rmat(8, 4) as g:
        for bad in (-1, 16385):
            with pytest.raises(pm.PolymerError):
                g.set_tunable("hub_cache", bad)
