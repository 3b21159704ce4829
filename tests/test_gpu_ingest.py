"""GPU tests of pm_graph_load_pbbs: PBBS files written by the oracle's
writers (the format the reference's readers take, IO-numa.h) read back into
device graphs, compared with the oracle's CSR, weights and results; malformed
files end in an error status, never in a graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def same_csr(g, og):
    off, idx = g.csr()
    return g.n == og.n and g.m == og.m and np.array_equal(off, og.off) and np.array_equal(idx, og.idx)


@pytest.mark.parametrize("scale,sym", [(12, False), (13, True), (18, False)])
def test_text_roundtrip(pm, oracle, tmp_path, scale, sym):
    og = oracle.rmat_graph(scale, 16, symmetric=sym)
    path = str(tmp_path / "g.adj")
    oracle.write_text(og, path)
    with pm.Graph.load_pbbs(path, symmetric=sym) as g:
        assert same_csr(g, og)
        if sym:
            assert np.array_equal(pm.Components(g), oracle.cc(og))


def test_weighted_text_sets_weights(pm, oracle, tmp_path):
    og = oracle.rmat_graph(12, 16, symmetric=True)
    w = oracle.weights_int(og)
    path = str(tmp_path / "w.adj")
    oracle.write_text(og, path, w)
    s = int(oracle.pick_sources(og, 1)[0])
    with pm.Graph.load_pbbs(path, symmetric=True) as g:
        assert same_csr(g, og)
        assert np.array_equal(g.weights_i32(), w)
        assert np.array_equal(pm.BellmanFord(g, s), oracle.dijkstra(og, w, s))


def test_binary_roundtrip(pm, oracle, tmp_path):
    og = oracle.rmat_graph(14, 16)
    base = oracle.write_binary(og, str(tmp_path / "b"))
    with pm.Graph.load_pbbs(base, binary=True) as g:
        assert same_csr(g, og)
        assert np.allclose(pm.PageRank(g, 5), oracle.pagerank(og, 5), rtol=1e-10, atol=0)


def test_skip_self_loops_drops_their_weights(pm, oracle, tmp_path):
    # 0->0 (w 7), 0->1 (w 2), 1->1 (w 9), 1->2 (w 3), 2->0 (w 4)
    path = tmp_path / "loops.adj"
    path.write_text("WeightedAdjacencyGraph\n3\n5\n0\n2\n4\n0\n1\n1\n2\n0\n7\n2\n9\n3\n4\n")
    with pm.Graph.load_pbbs(str(path), skip_self_loops=True) as g:
        off, idx = g.csr()
        assert off.tolist() == [0, 1, 2, 3] and idx.tolist() == [1, 2, 0]
        assert g.weights_i32().tolist() == [2, 3, 4]
    with pm.Graph.load_pbbs(str(path)) as g:
        assert g.m == 5 and g.weights_i32().tolist() == [7, 2, 9, 3, 4]
        with pytest.raises(pm.PolymerError):
            pm.PageRank(g, 2)  # self loops kept: PageRank refuses the graph


def test_whitespace_and_signs(pm, tmp_path):
    path = tmp_path / "ws.adj"
    path.write_bytes(b"  AdjacencyGraph\r\n\t4 \r\n5\n+0 2\t3 3\r\n1 2 3  +0\t1\n\n")
    with pm.Graph.load_pbbs(str(path)) as g:
        off, idx = g.csr()
        assert off.tolist() == [0, 2, 3, 3, 5] and idx.tolist() == [1, 2, 3, 0, 1]


@pytest.mark.parametrize("body,what", [
    (b"AdjacencyGraf\n2\n1\n0\n1\n0\n", "header"),
    (b"AdjacencyGraph\n2\n2\n0\n1\n0\n", "count"),
    (b"AdjacencyGraph\n2\n1\n0\n1\n0\n1\n", "count"),
    (b"AdjacencyGraph\n2\n1\n0\n1x\n0\n", "word"),
    (b"AdjacencyGraph\n2\n1\n0\n1\n4294967296\n", "range"),
    (b"AdjacencyGraph\n2\n1\n0\n1\n7\n", "edge id"),
    (b"AdjacencyGraph\n2\n1\n1\n0\n0\n", "offsets"),
    (b"AdjacencyGraph\nx\n1\n0\n1\n0\n", "vertex count"),
])
def test_malformed_files_are_bad_graph(pm, tmp_path, body, what):
    path = tmp_path / "bad.adj"
    path.write_bytes(body)
    with pytest.raises(pm.PolymerError) as ei:
        pm.Graph.load_pbbs(str(path))
    assert ei.value.status == 5, what


def test_missing_files(pm, tmp_path):
    with pytest.raises(pm.PolymerError) as ei:
        pm.Graph.load_pbbs(str(tmp_path / "nothing.adj"))
    assert ei.value.status == 1
    with pytest.raises(pm.PolymerError) as ei:
        pm.Graph.load_pbbs(str(tmp_path / "nothing"), binary=True)
    assert ei.value.status == 1


@pytest.mark.parametrize("device_arrays", [False, True])
def test_create_weighted_equals_create_then_set(pm, oracle, device_arrays):
    import torch
    og = oracle.rmat_graph(13, 16, symmetric=True)
    wi = oracle.weights_int(og)
    wf = oracle.weights_unit(og)
    s = int(oracle.pick_sources(og, 1)[0])
    arr = (lambda a: torch.from_numpy(a).cuda()) if device_arrays else (lambda a: a)
    for w in (wi, wf):
        with pm.Graph.from_csr(arr(og.off), arr(og.idx), symmetric=True, weights=arr(w)) as g:
            assert same_csr(g, og)
            if w.dtype == np.int32:
                assert np.array_equal(g.weights_i32(), w)
                assert np.array_equal(pm.BellmanFord(g, s), oracle.dijkstra(og, w, s))
            else:
                assert np.array_equal(g.weights_f32(), w)


def test_create_weighted_skips_loops_with_their_weights(pm):
    off = np.array([0, 2, 4, 5], np.int32)
    idx = np.array([0, 1, 1, 2, 0], np.int32)
    w = np.array([7, 2, 9, 3, 4], np.int32)
    with pm.Graph.from_csr(off, idx, skip_self_loops=True, weights=w) as g:
        o, i = g.csr()
        assert o.tolist() == [0, 1, 2, 3] and i.tolist() == [1, 2, 0]
        assert g.weights_i32().tolist() == [2, 3, 4]


@pytest.mark.parametrize("sym", [False, True])
def test_graph_dump_load_and_save(pm, oracle, tmp_path, sym):
    """Graph dumps (dumpGraphToBin / loadGraphFromBin layout): the oracle's dump
    loads into the oracle's CSR; the library's dump reads back, in the
    oracle's reader, as the graph's CSR and its transpose."""
    og = oracle.rmat_graph(11, 16, symmetric=sym)
    path = str(tmp_path / "a.dump")
    oracle.write_dump(og, path)
    with pm.Graph.load_dump(path, symmetric=sym) as g:
        assert same_csr(g, og)
        if sym:
            assert np.array_equal(pm.Components(g), oracle.cc(og))
        out = str(tmp_path / "b.dump")
        g.save_dump(out)
    n, off, idx, in_off, in_idx = oracle.read_dump(out)
    want_in_off, want_in_idx = oracle.transpose(og)
    assert n == og.n and np.array_equal(off, og.off) and np.array_equal(idx, og.idx)
    assert np.array_equal(in_off, want_in_off) and np.array_equal(in_idx, want_in_idx)
    assert open(out, "rb").read() == open(path, "rb").read()  # the same bytes as the oracle's writer


def test_graph_dump_malformed(pm, oracle, tmp_path):
    og = oracle.rmat_graph(8, 4)
    good = str(tmp_path / "g.dump")
    oracle.write_dump(og, good)
    raw = bytearray(open(good, "rb").read())

    def bad(mutate, name):
        b = bytearray(raw)
        mutate(b)
        p = str(tmp_path / name)
        open(p, "wb").write(bytes(b))
        with pytest.raises(pm.PolymerError) as ei:
            pm.Graph.load_dump(p)
        assert ei.value.status == 5, name

    bad(lambda b: b.extend(b"\0\0\0\0"), "longer")                    # total size disagrees
    bad(lambda b: b.__setitem__(slice(8, 12), np.int32(og.n + 1).tobytes()), "n")    # record count
    bad(lambda b: b.__setitem__(slice(24, 28), np.int32(5).tobytes()), "id")         # record 0 says 5
    bad(lambda b: b.__setitem__(slice(28, 32), np.int32(-3).tobytes()), "degree")    # negative degree
    bad(lambda b: b.__setitem__(slice(12, 20), np.int64(len(og.idx) + 1).tobytes()), "m")  # m
    with pytest.raises(pm.PolymerError) as ei:
        pm.Graph.load_dump(str(tmp_path / "missing.dump"))
    assert ei.value.status == 1
