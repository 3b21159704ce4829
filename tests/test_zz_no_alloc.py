"""GPU test of pm_pagerank_static, the entry point for callers that cannot
allocate GPU memory (its working vectors live in a fixed array inside the
library).  Compared, through the C ABI, with pm_pagerank (PM_F32) on the same
graph, on two calls in a row (the second call reuses the array the first one
left behind).  Collected last so that a run stopping at its first failure has
already run every other test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RL1_F32 = 1e-5


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


def test_pagerank_static_matches_pagerank(pm, oracle):
    import torch

    og = oracle.rmat_graph(16, 16)
    with pm.Graph.from_csr(og.off, og.idx) as g:
        ref = pm.PageRank(g, 20, dtype=np.float32)
    off = torch.from_numpy(og.off).cuda()
    idx = torch.from_numpy(og.idx).cuda()
    out1 = torch.empty(og.n, dtype=torch.float32, device="cuda")
    out2 = torch.full((og.n,), -1.0, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    pm.PageRankStatic(off, idx, out1, 20)
    pm.PageRankStatic(off, idx, out2, 20)
    r1, r2 = out1.cpu().numpy(), out2.cpu().numpy()
    assert rel_l1(r1, ref) < RL1_F32
    assert rel_l1(r2, ref) < RL1_F32
    assert rel_l1(r2, r1) < RL1_F32


def test_pagerank_static_rejects_oversize(pm):
    import torch

    n = (1 << 20) + 1
    off = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    idx = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    with pytest.raises(pm.PolymerError) as ei:
        pm.PageRankStatic(off, idx[:0], out, 3)
    assert ei.value.status == 1 and b"1048576" in pm.lib().pm_last_error()
