"""GPU tests of host threads that drive distinct graph handles at the same
time (the replacement's contract: thread-safe across distinct handles).
Each thread builds, runs and destroys its own graphs in a loop while the
other does the same, so blocks freed by one thread's handles are taken by
the other's through the stream-ordered memory cache; every result must equal
the one computed alone (bit-identical: the kernels reduce in a fixed
order)."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _work_sym(pm, og, w, s):
    with pm.Graph.from_csr(og.off, og.idx, symmetric=True, weights=w) as g:
        return (pm.BFS(s, g)[1], pm.Components(g), pm.BellmanFord(g, s))


def _work_dir(pm, og, x0):
    with pm.Graph.from_csr(og.off, og.idx, weights=np.full(og.m, 0.5, np.float32)) as g:
        return (pm.PageRank(g, 8, dtype=np.float32), pm.SPMV(g, x0, 4, dtype=np.float32))


def _same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("cache", [-1, 0])
def test_two_threads_distinct_handles(pm, oracle, cache):
    sym = oracle.rmat_graph(16, 16, symmetric=True)
    w = oracle.weights_int(sym)
    s = int(oracle.pick_sources(sym, 1)[0])
    dg = oracle.rmat_graph(17, 16)
    x0 = np.random.default_rng(3).random(dg.n).astype(np.float32)
    pm.set_memory_cache(cache)
    try:
        want_sym = _work_sym(pm, sym, w, s)
        want_dir = _work_dir(pm, dg, x0)
        assert np.array_equal(want_sym[1], oracle.cc(sym))
        assert np.array_equal(want_sym[2], oracle.dijkstra(sym, w, s))
        errors, bad = [], []

        def loop(fn, args, want, reps):
            try:
                for _ in range(reps):
                    if not _same(fn(pm, *args), want):
                        bad.append(fn.__name__)
            except Exception as exc:  # reported by the main thread
                errors.append(exc)

        ts = [threading.Thread(target=loop, args=(_work_sym, (sym, w, s), want_sym, 6)),
              threading.Thread(target=loop, args=(_work_dir, (dg, x0), want_dir, 6))]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        assert not errors, errors
        assert not bad, bad
    finally:
        pm.set_memory_cache(-1)


def test_thread_reuses_blocks_freed_by_another(pm, oracle):
    """A graph destroyed in one thread leaves its blocks in the cache; a graph
    built in a second thread takes them and computes the same results."""
    og = oracle.rmat_graph(15, 16)
    ref = oracle.pagerank(og, 5)
    pm.set_memory_cache(-1)
    out = {}

    def run(key):
        with pm.Graph.from_csr(og.off, og.idx) as g:
            out[key] = pm.PageRank(g, 5)

    try:
        for key in ("first", "second"):
            t = threading.Thread(target=run, args=(key,))
            t.start()
            t.join()
            assert pm.memory_cached() > 0
        assert np.array_equal(out["first"], out["second"])
        assert np.allclose(out["second"], ref, rtol=1e-10, atol=0)
    finally:
        pm.set_memory_cache(-1)
