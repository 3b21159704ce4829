"""GPU test of the library's device-memory cache: buffers of a destroyed
graph are kept and reused by the next graph, results do not change, and
turning the cache off releases it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_cache_reuses_and_releases(pm, oracle):
    og = oracle.rmat_graph(14, 16)
    ref = oracle.pagerank(og, 5)
    pm.set_memory_cache(-1)
    try:
        with pm.Graph.from_csr(og.off, og.idx) as g:
            a = pm.PageRank(g, 5)
        held = pm.memory_cached()
        assert held > 0                       # the destroyed graph's buffers stayed
        with pm.Graph.from_csr(og.off, og.idx) as g:
            assert pm.memory_cached() < held  # ... and the new graph took them
            b = pm.PageRank(g, 5)
        assert np.array_equal(a, b) and np.allclose(a, ref, rtol=1e-10, atol=0)
        pm.set_memory_cache(0)
        assert pm.memory_cached() == 0
        with pm.Graph.from_csr(og.off, og.idx) as g:
            assert np.array_equal(pm.PageRank(g, 5), a)
        assert pm.memory_cached() == 0        # off: freed at once
    finally:
        pm.set_memory_cache(-1)
