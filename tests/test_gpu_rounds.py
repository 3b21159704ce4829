"""GPU tests of BFS with its rounds driven on the GPU (a CUDA graph whose
WHILE node runs the rounds; on with the cuda_graphs tunable) against the host
loop (cuda_graphs off): the same depths as the oracle, the same round,
direction and edge statistics, for every direction threshold, an isolated
source, a long path (thousands of rounds in one launch) and repeated calls
that replay one captured graph with other sources."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bfs_both(pm, g, s, threshold=-1):
    g.set_tunable("cuda_graphs", 1)
    on = pm.BFS(s, g, threshold=threshold, stats=True)
    g.set_tunable("cuda_graphs", 0)
    off = pm.BFS(s, g, threshold=threshold, stats=True)
    g.set_tunable("cuda_graphs", 1)
    return on, off


@pytest.mark.parametrize("threshold", [-1, 0, 1 << 40])
@pytest.mark.parametrize("sym", [True, False])
def test_device_rounds_match_host_rounds(pm, oracle, threshold, sym):
    og = oracle.rmat_graph(14, 16, symmetric=sym)
    with pm.Graph.from_csr(og.off, og.idx, symmetric=sym) as g:
        for s in oracle.pick_sources(og, 3):
            s = int(s)
            (p1, d1, st1), (p0, d0, st0) = _bfs_both(pm, g, s, threshold)
            want = oracle.bfs(og, s)[0]
            assert np.array_equal(d1, want) and np.array_equal(d0, want)
            for k in ("rounds", "dense_rounds", "reached", "edges_visited"):
                assert st1[k] == st0[k], k
            v = np.nonzero(d1 > 0)[0]
            assert np.all(d1[p1[v]] == d1[v] - 1) and p1[s] == s


def test_isolated_source_and_edgeless(pm):
    off = np.array([0, 2, 2, 3, 3], np.int32)  # 0->1, 0->3, 2->0; vertex 1 and 3 have no out-edges
    idx = np.array([1, 3, 0], np.int32)
    with pm.Graph.from_csr(off, idx) as g:
        (p, d, st), _ = _bfs_both(pm, g, 1)
        assert d.tolist() == [-1, 0, -1, -1] and st["rounds"] == 1 and st["reached"] == 1
        (p, d, st), _ = _bfs_both(pm, g, 2)
        assert d.tolist() == [1, 2, 0, 2]
    with pm.Graph.from_csr(np.zeros(6, np.int32), np.zeros(0, np.int32)) as g:
        (p, d, st), _ = _bfs_both(pm, g, 4)
        assert d.tolist() == [-1, -1, -1, -1, 0]


def test_long_path_in_one_launch(pm):
    n = 3000
    off = np.arange(n + 1, dtype=np.int32)
    off[-1] = n - 1
    idx = np.arange(1, n, dtype=np.int32)  # i -> i+1
    off = np.minimum(off, n - 1).astype(np.int32)
    with pm.Graph.from_csr(off, idx) as g:
        (p, d, st), (_, d0, st0) = _bfs_both(pm, g, 0)
        assert np.array_equal(d, np.arange(n)) and np.array_equal(d0, d)
        assert st["rounds"] == st0["rounds"] == n


def test_replays_with_other_sources(pm, oracle):
    og = oracle.rmat_graph(13, 16, symmetric=True)
    with pm.Graph.from_csr(og.off, og.idx, symmetric=True) as g:
        srcs = [int(s) for s in oracle.pick_sources(og, 6)]
        for s in srcs + srcs[::-1]:
            assert np.array_equal(pm.BFS(s, g)[1], oracle.bfs(og, s)[0])

