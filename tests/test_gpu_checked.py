"""GPU tests of the checked build (libpolymer_b200_check.so, loaded with
POLYMER_B200_CHECKED=1): every vertex id the engine kernels read is
bounds-tested, and on valid graphs the checks stay silent -- the applications
give the oracle's results through the same C ABI, in every direction mode
and heavy-row mode.  Run in a child process, since the library is chosen at
import."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_LIB = os.path.join(ROOT, "polymer_b200", "libpolymer_b200_check.so")

SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, ROOT)
sys.path.insert(0, ROOT + "/oracle")
import polymer_b200 as pm
import pm_oracle as oracle
assert pm.LIB_PATH.endswith("libpolymer_b200_check.so"), pm.LIB_PATH
og = oracle.rmat_graph(14, 16, symmetric=True)
w = oracle.weights_int(og)
with pm.Graph.from_csr(og.off, og.idx, symmetric=True, weights=w) as g:
    for mode in (0, 1, 2):
        g.set_tunable("heavy_mode", mode)
        for s in oracle.pick_sources(og, 2):
            s = int(s)
            want = oracle.bfs(og, s)[0]
            for thr in (-1, 0, 1 << 40):
                assert np.array_equal(pm.BFS(s, g, threshold=thr)[1], want), (mode, s, thr)
            assert np.array_equal(pm.BellmanFord(g, s), oracle.dijkstra(og, w, s)), (mode, s)
        for thr in (-1, 0, 1 << 40):
            assert np.array_equal(pm.Components(g, threshold=thr), oracle.cc(og)), (mode, thr)
    srcs = oracle.pick_sources(og, 8)
    dep = pm.BFSMulti(srcs, g)
    for l, s in enumerate(srcs):
        assert np.array_equal(dep[l], oracle.bfs(og, int(s))[0]), l
od = oracle.rmat_graph(14, 16)
wu = oracle.weights_unit(od)
x0 = oracle.uniform01(od.n)
with pm.Graph.from_csr(od.off, od.idx, weights=wu) as g:
    for mode in (0, 1, 2):
        g.set_tunable("heavy_mode", mode)
        pr = pm.PageRank(g, 10)
        assert np.allclose(pr, oracle.pagerank(od, 10), rtol=1e-10, atol=0), mode
        y = pm.SPMV(g, x0.astype(np.float64), 10, dtype=np.float64)
        ref = oracle.spmv(od, wu.astype(np.float64), x0.astype(np.float64), 10)
        assert np.abs(y - ref).sum() / np.abs(ref).sum() < 1e-12, mode
print("checked build ok")
"""


@pytest.mark.skipif(not os.path.exists(CHECK_LIB), reason="checked build not built (__graft_entry__.build())")
def test_checked_build_is_silent_on_valid_graphs(pm):  # pm: skips without a device
    env = dict(os.environ, POLYMER_B200_CHECKED="1")
    p = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + SCRIPT], env=env, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-4000:]
    assert "checked build ok" in p.stdout
