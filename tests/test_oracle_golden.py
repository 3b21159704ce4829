"""CPU tests: the oracle restatement against the reference's own outputs.

The fixtures in tests/golden/ were produced by the reference binaries
(oracle/_ref, built from the original Polymer sources) via
tests/golden/make_golden.py.  When oracle/_ref is present the reference is
also run live on fresh graphs.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_generator_reproduces_fixture_graphs(oracle):
    z = load("rmat10_directed.npz")
    g = oracle.rmat_graph(10, 16)
    assert np.array_equal(g.off, z["off"]) and np.array_equal(g.idx, z["idx"])
    z = load("rmat10_symmetric.npz")
    gs = oracle.rmat_graph(10, 16, symmetric=True)
    assert np.array_equal(gs.off, z["off"]) and np.array_equal(gs.idx, z["idx"])


def test_generator_properties(oracle):
    g = oracle.rmat_graph(12, 16)
    src = np.repeat(np.arange(g.n), np.diff(g.off))
    assert np.all(src != g.idx), "self loops must be removed"
    key = src.astype(np.int64) * g.n + g.idx
    assert np.all(np.diff(key) > 0), "edges sorted by (src, dst), no duplicates"
    gs = oracle.rmat_graph(12, 16, symmetric=True)
    s2 = np.repeat(np.arange(gs.n), np.diff(gs.off))
    fwd = set(zip(s2.tolist(), gs.idx.tolist()))
    assert all((b, a) in fwd for a, b in list(fwd)[:5000])


def test_pagerank_matches_reference_fixture(oracle):
    z = load("rmat10_directed.npz")
    g = oracle.Graph(len(z["off"]) - 1, z["off"], z["idx"])
    ours = oracle.pagerank(g, 10)
    ref = z["pagerank10"]
    # the reference prints %.9e
    assert np.allclose(ours, ref, rtol=2e-9, atol=0)


def test_pagerank_frontier_rule_is_not_textbook_pagerank(oracle):
    """The reference's PageRank (numa-PageRank.C:273-335) updates only the
    frontier and takes as the next frontier the targets of the current one,
    so vertices with no in-edges drop out after the first iteration and keep
    what sits in their slots.  A textbook all-vertex iteration (every vertex
    gets 0.15/n + 0.85 * sum each iteration) is measurably different on the
    same graph, while the oracle matches the reference's own output."""
    z = load("rmat10_directed.npz")
    n = len(z["off"]) - 1
    g = oracle.Graph(n, z["off"], z["idx"])
    src = np.repeat(np.arange(n), np.diff(z["off"]))
    deg = np.diff(z["off"]).astype(np.float64)
    p = np.full(n, 1.0 / n)
    for _ in range(10):
        contrib = np.where(deg > 0, p / np.maximum(deg, 1), 0.0)
        q = np.zeros(n)
        np.add.at(q, z["idx"], contrib[src])
        p = 0.15 / n + 0.85 * q
    ours = oracle.pagerank(g, 10)
    assert np.allclose(ours, z["pagerank10"], rtol=2e-9, atol=0)
    indeg = np.bincount(z["idx"], minlength=n)
    assert (indeg == 0).sum() > 0  # the graph has vertices the frontier rule treats differently
    rel = np.abs(p - ours).sum() / np.abs(ours).sum()
    assert rel > 1e-3, rel


def test_pagerank_skip_ring_fixture(oracle):
    z = load("tiny.npz")
    n = len(z["off"]) - 1
    src = np.repeat(np.arange(n), np.diff(z["off"]))
    keep = src != z["idx"]
    g = oracle.graph_from_edges(n, src[keep], z["idx"][keep])
    ours = oracle.pagerank(g, 6)
    assert np.allclose(ours, z["pagerank6"], rtol=2e-9, atol=1e-300)


def test_spmv_matches_reference_fixture(oracle):
    z = load("rmat10_directed.npz")
    g = oracle.Graph(len(z["off"]) - 1, z["off"], z["idx"])
    x0 = np.full(g.n, 1.0 / g.n)
    ours = oracle.spmv(g, z["spmv_w"].astype(np.float64), x0, 5)
    assert np.allclose(ours, z["spmv5"], rtol=2e-9, atol=0)


def test_components_match_reference_fixture(oracle):
    z = load("rmat10_symmetric.npz")
    g = oracle.Graph(len(z["off"]) - 1, z["off"], z["idx"])
    assert np.array_equal(oracle.cc(g), z["cc"])


def test_bfs_depths_match_reference_parents(oracle):
    z = load("rmat10_symmetric.npz")
    g = oracle.Graph(len(z["off"]) - 1, z["off"], z["idx"])
    for s, par, cnt in zip(z["bfs_sources"], z["bfs_parents"], z["bfs_counts"]):
        depth, _ = oracle.bfs(g, int(s))
        assert np.array_equal(oracle.bfs_depths_from_parents(par, int(s)), depth)
        assert (depth >= 0).sum() == cnt


def test_bellman_ford_is_exact(oracle):
    for scale, sym in ((10, True), (11, False)):
        g = oracle.rmat_graph(scale, 8, symmetric=sym)
        w = oracle.weights_int(g)
        for s in oracle.pick_sources(g, 3):
            assert np.array_equal(oracle.bellman_ford(g, w, int(s)), oracle.dijkstra(g, w, int(s)))


def test_weights_rules(oracle):
    g = oracle.rmat_graph(9, 8, symmetric=True)
    w = oracle.weights_int(g)
    assert w.min() >= 1 and w.max() <= 22
    src = np.repeat(np.arange(g.n), np.diff(g.off))
    lookup = dict(zip(zip(src.tolist(), g.idx.tolist()), w.tolist()))
    assert all(lookup[(b, a)] == c for (a, b), c in list(lookup.items())[:3000])
    wu = oracle.weights_unit(g)
    assert wu.min() > 0 and wu.max() <= 1


def test_bp_restatement_small(oracle):
    # two vertices, one edge 0->1: vertex 1 receives one normalised message
    g = oracle.graph_from_edges(2, [0], [1])
    prior = np.array([[0.3, 0.7], [0.6, 0.4]])
    out = oracle.bp(g, prior, 1)
    a0, a1 = 0.6, 0.4
    b0, b1 = 0.9 * a0 + 0.1 * a1, 0.1 * a0 + 0.9 * a1
    assert np.allclose(out[1], [np.log(b0 / (b0 + b1)), np.log(b1 / (b0 + b1))])
    assert np.allclose(out[0], [0, 0])


# The reference's BP prints nothing and leaves its inputs unset; a patched
# copy (oracle/ref_patch_bp.py: seeded priors, products 1, psi
# [[.9,.1],[.1,.9]], products printed) pins the message formula.  Its FP32
# arithmetic against the FP64 restatement: relative 2e-5 over two rounds.
RTOL_BP_FP32 = 2e-5


def test_bp_raw_matches_reference_fixture(oracle):
    z = np.load(os.path.join(GOLDEN, "bp_sparse.npz"))
    g = oracle.Graph(len(z["off"]) - 1, z["off"], z["idx"])
    prior = oracle.bp_ref_priors(g.n).astype(np.float64)
    for it, key in ((1, "prod1"), (2, "prod2")):
        raw = oracle.bp_raw(g, prior, it)
        assert np.allclose(z[key], raw, rtol=RTOL_BP_FP32, atol=0), it


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref",
                                                    "numa-BP-result")), reason="reference binaries not built")
def test_bp_raw_matches_live_reference(oracle, tmp_path):
    rng = np.random.default_rng(11)
    n, m = 2000, 5000
    g = oracle.graph_from_edges(n, rng.integers(0, n, m), rng.integers(0, n, m))
    base = oracle.write_binary(g, str(tmp_path / "bp"))
    prior = oracle.bp_ref_priors(n).astype(np.float64)
    for it in (1, 2):
        ref, _ = oracle.ref_bp_result(base, it)
        assert np.allclose(ref, oracle.bp_raw(g, prior, it), rtol=RTOL_BP_FP32, atol=0), it


def test_bp_log_restatement_is_the_normalised_formula(oracle):
    """pmo_bp (log products of messages divided by their sum) equals the
    reference's formula with each belief divided by its sum, in the linear
    domain: the only change from the reference's messages is that division."""
    rng = np.random.default_rng(3)
    for n, m in ((500, 1500), (4000, 20000)):
        g = oracle.graph_from_edges(n, rng.integers(0, n, m), rng.integers(0, n, m))
        prior = oracle.uniform_open(2 * n, 99).reshape(n, 2).astype(np.float64)
        for it in (1, 2, 4):
            a = np.exp(oracle.bp(g, prior, it))
            b = oracle.bp_raw(g, prior, it, normalize=True)
            assert np.allclose(a, b, rtol=1e-12, atol=0), (n, it)


def test_er_batch_generator(oracle):
    g, vbase = oracle.er_batch(40, 50, 5000, 8, seed=3)
    sizes = np.diff(vbase)
    assert sizes.min() >= 50 and sizes.max() <= 5000 and len(sizes) == 40
    src = np.repeat(np.arange(g.n), np.diff(g.off))
    part = np.searchsorted(vbase, src, side="right") - 1
    assert np.all(g.idx >= vbase[part]) and np.all(g.idx < vbase[part + 1]), "edges stay in their part"
    assert np.all(src != g.idx)
    assert abs(g.m / g.n - 8) < 0.5


def test_ppr_restatement(oracle):
    g = oracle.rmat_graph(9, 8)
    seeds = oracle.pick_sources(g, 4)
    x = oracle.ppr(g, seeds, 30)
    # fixed point check: x = d P^T x + (1-d) e_seed (30 iterations ~ 0.85^30)
    for j, s in enumerate(seeds):
        y = oracle.ppr(g, [s], 31)[:, 0]
        assert np.abs(x[:, j] - y).sum() < 0.05
        assert x[s, j] >= 0.15


def test_pagerank_delta_matches_reference_fixture(oracle):
    z = np.load(os.path.join(GOLDEN, "rmat10_prdelta.npz"))
    g = oracle.Graph(len(z["off"]) - 1, z["off"], z["idx"])
    for iters, key in ((3, "prdelta3"), (10, "prdelta10")):
        p, fs = oracle.pagerank_delta(g, iters, with_frontier=True)
        assert np.allclose(p, z[key], rtol=2e-9, atol=0), key  # the reference prints %.9e
    assert fs[0] > fs[-1] and fs[-1] == 0  # the frontier drains within 10 rounds here


def test_depths_from_parents_rejects_cycles(oracle):
    with pytest.raises(ValueError):
        oracle.bfs_depths_from_parents(np.array([0, 2, 1], np.int32), 0)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref",
                                                    "numa-PageRank")),
                    reason="reference binaries not built here")
def test_live_reference_scale12(oracle, tmp_path):
    g = oracle.rmat_graph(12, 16)
    base = oracle.write_binary(g, str(tmp_path / "g"))
    ref, _ = oracle.ref_pagerank(base, 10, threads=4)
    assert np.allclose(oracle.pagerank(g, 10), ref, rtol=2e-9, atol=0)
    prd, _ = oracle.ref_pagerank_delta(base, 8, threads=4)
    assert np.allclose(oracle.pagerank_delta(g, 8), prd, rtol=2e-9, atol=0)
    gs = oracle.rmat_graph(12, 16, symmetric=True)
    bs = oracle.write_binary(gs, str(tmp_path / "s"))
    lab, _ = oracle.ref_components(bs, threads=4)
    assert np.array_equal(lab, oracle.cc(gs))
    s = int(oracle.pick_sources(gs, 1)[0])
    par, cnt, _ = oracle.ref_bfs(bs, s, threads=4)
    depth, _ = oracle.bfs(gs, s)
    assert np.array_equal(oracle.bfs_depths_from_parents(par, s), depth)


def test_oracle_graph_dump_round_trip(oracle, tmp_path):
    """The oracle's restatement of dumpGraphToBin / loadGraphFromBin reads back
    what it writes (both adjacency directions), on a directed graph."""
    og = oracle.rmat_graph(9, 8)
    path = str(tmp_path / "g.dump")
    oracle.write_dump(og, path)
    n, off, idx, in_off, in_idx = oracle.read_dump(path)
    want_off, want_idx = oracle.transpose(og)
    assert n == og.n and np.array_equal(off, og.off) and np.array_equal(idx, og.idx)
    assert np.array_equal(in_off, want_off) and np.array_equal(in_idx, want_idx)
