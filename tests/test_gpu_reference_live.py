"""GPU results against the reference binaries themselves (oracle/_ref, built
from the unmodified sources and carried with the tree), at the sizes the
benchmark names: PageRank FP64 on the 2^16-vertex directed R-MAT (10
iterations, elementwise to the reference's printed precision), Components
and BFS on the scale-22 symmetrised R-MAT (bit-exact labels; BFS depths
consistent with every parent the reference prints).  The graphs come from
the device generator (bit-identical to the oracle's) and are written in the
reference's binary format.  Skipped where oracle/_ref was not built."""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "numa-PageRank")),
                                 reason="reference binaries not built (make -C oracle ref)")]


def _write(oracle, g, path):
    off, idx = g.csr()
    return oracle.write_binary(oracle.Graph(g.n, off, idx), path)


def test_pagerank_f64_scale16_vs_reference_binary(pm, oracle, tmp_path):
    with pm.Graph.rmat(16, 16) as g:
        r = pm.PageRank(g, 10, dtype=np.float64)
        base = _write(oracle, g, str(tmp_path / "r16"))
    ref, _ = oracle.ref_pagerank(base, 10)
    assert len(ref) == len(r)
    assert np.allclose(r, ref, rtol=2e-9, atol=0)  # the reference prints %.9e


BINDING = os.path.join(ROOT, "tests", "cpp", "_build", "numa-PageRank-b200")


@pytest.mark.skipif(not os.path.exists(BINDING), reason="binding not built (reference sources absent at build time)")
def test_reference_application_with_b200_binding(oracle, tmp_path):
    """The reference's numa-PageRank.C with its PageRank body replaced by the
    B200 binding (tests/cpp/ref_binding/pagerank_b200.inc, the text
    INTEGRATION.md shows), run with the reference's own command line on the
    2^16-vertex R-MAT of the FP64 PageRank workload: its -result output equals
    the unmodified reference program's to the printed precision."""
    og = oracle.rmat_graph(16, 16)
    base = oracle.write_binary(og, str(tmp_path / "b16"))
    got, t_b200 = oracle.ref_pagerank(base, 10, exe=BINDING)
    ref, _ = oracle.ref_pagerank(base, 10)
    assert len(got) == len(ref) == og.n
    assert np.allclose(got, ref, rtol=2e-9, atol=0)
    assert t_b200 == t_b200  # the application's own timer line was printed


def test_components_and_bfs_scale22_vs_reference_binary(pm, oracle, tmp_path):
    with pm.Graph.rmat(22, 16, symmetric=True) as g:
        off, _ = g.csr()
        lab = pm.Components(g)
        nz = np.nonzero(np.diff(off) > 0)[0]
        srcs = [int(nz[17]), int(nz[len(nz) // 2])]
        depths = [pm.BFS(s, g)[1] for s in srcs]
        base = _write(oracle, g, str(tmp_path / "s22"))
    ref_lab, _ = oracle.ref_components(base)
    assert np.array_equal(lab, ref_lab)
    for s, d in zip(srcs, depths):
        par, cnt, _ = oracle.ref_bfs(base, s)
        reached = par >= 0
        assert np.array_equal(reached, d >= 0) and reached.sum() == cnt
        v = np.nonzero(reached)[0]
        v = v[v != s]
        assert d[s] == 0 and np.all(d[v] == d[par[v]] + 1)  # the reference tree's depths


def test_pagerank_delta_and_spmv_scale16_vs_reference_binary(pm, oracle, tmp_path):
    with pm.Graph.rmat(16, 16) as g:
        p = pm.PageRankDelta(g, 10, dtype=np.float64, threshold=0)
        off, idx = g.csr()
        og = oracle.Graph(g.n, off, idx)
        base = oracle.write_binary(og, str(tmp_path / "d16"))
        w = oracle.weights_int(og, wmax=5)  # the reference's SpMV weights are intE
        g.set_weights(w.astype(np.float32))
        y = pm.SPMV(g, np.full(g.n, 1.0 / g.n), 5, dtype=np.float64)
    ref_p, _ = oracle.ref_pagerank_delta(base, 10)
    assert np.allclose(p, ref_p, rtol=2e-9, atol=0)
    text = str(tmp_path / "w16.txt")
    oracle.write_text(og, text, w)
    ref_y, _ = oracle.ref_spmv(text, 5)
    assert np.allclose(y, ref_y, rtol=2e-9, atol=0)
