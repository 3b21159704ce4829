"""GPU failure tests, made on the host's terms (nothing faults, traps or hangs
the GPU): a bounded device wait that runs out reports PM_ERR_TIMEOUT and
leaves the device usable; an allocation failure injected at any point of a
graph build or of an application call reports PM_ERR_OOM, frees what the
call held, and leaves the library -- and a handle that survived -- usable."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_device_stays_usable(pm, oracle):
    for polls in (1, 20000):
        with pytest.raises(pm.PolymerError) as ei:
            pm.test_wait_timeout(polls)
        assert ei.value.status == 4
    og = oracle.rmat_graph(12, 16, symmetric=True)
    with pm.Graph.from_csr(og.off, og.idx, symmetric=True) as g:
        assert np.array_equal(pm.Components(g), oracle.cc(og))
    with pytest.raises(pm.PolymerError) as ei:
        pm.test_wait_timeout(0)  # out of range: refused before any launch
    assert ei.value.status == 1


@pytest.mark.parametrize("k", [1, 2, 5, 9, 14])
def test_allocation_failure_during_a_build(pm, oracle, k):
    og = oracle.rmat_graph(12, 16)
    w = oracle.weights_unit(og)
    pm.test_fail_alloc_after(k)
    try:
        with pytest.raises(pm.PolymerError) as ei:
            with pm.Graph.from_csr(og.off, og.idx, weights=w) as g:
                pm.PageRank(g, 3)
                pm.SPMV(g, oracle.uniform01(og.n), 2)
        assert ei.value.status == 2 and "injected" in str(ei.value)
    finally:
        pm.test_fail_alloc_after(0)
    with pm.Graph.from_csr(og.off, og.idx, weights=w) as g:  # nothing left broken
        assert np.allclose(pm.PageRank(g, 3), oracle.pagerank(og, 3), rtol=1e-10, atol=0)


def test_allocation_failure_inside_calls_keeps_the_handle(pm, oracle):
    og = oracle.rmat_graph(13, 16, symmetric=True)
    w = oracle.weights_int(og)
    s = int(oracle.pick_sources(og, 1)[0])
    with pm.Graph.from_csr(og.off, og.idx, symmetric=True, weights=w) as g:
        for call in (lambda: pm.BFS(s, g), lambda: pm.Components(g), lambda: pm.BellmanFord(g, s),
                     lambda: pm.BFSMulti([s, 0], g)):
            pm.test_fail_alloc_after(1)  # the call's first new workspace
            try:
                call()  # may find its workspaces already allocated: then nothing fails
            except pm.PolymerError as exc:
                assert exc.status == 2
            finally:
                pm.test_fail_alloc_after(0)
        assert np.array_equal(pm.BFS(s, g)[1], oracle.bfs(og, s)[0])
        assert np.array_equal(pm.Components(g), oracle.cc(og))
        assert np.array_equal(pm.BellmanFord(g, s), oracle.dijkstra(og, w, s))
