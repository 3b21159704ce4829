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
    # the second call must not allocate: every library allocation from here
    # on would fail, and the device's free memory must not move
    free_before = torch.cuda.mem_get_info()[0]
    pm.test_fail_alloc_after(1)
    try:
        pm.PageRankStatic(off, idx, out2, 20)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
    finally:
        pm.test_fail_alloc_after(0)
    assert free_after == free_before
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


# Small CSRs the entry point must refuse: (what is wrong, offsets, edges).
BAD_CSRS = [
    ("id out of range", [0, 2, 3, 4], [1, 2, 7, 0]),
    ("negative id", [0, 1, 2, 3], [1, -1, 0]),
    ("self loop", [0, 2, 3, 4], [1, 0, 2, 0]),
    ("offsets[n] != m", [0, 1, 2, 2], [1, 2, 0]),
    ("offsets not monotone", [0, 2, 1, 3], [1, 2, 0]),
    ("offset past m", [0, 1, 5, 3], [1, 2, 0]),
]


def test_pagerank_static_rejects_bad_csr(pm):
    """Each bad CSR is refused with PM_ERR_BAD_GRAPH (the device check reads
    only inside the caller's arrays), and a valid call right after it works
    (the status word is cleared per call)."""
    import torch

    for name, o, e in BAD_CSRS:
        off = torch.tensor(o, dtype=torch.int32, device="cuda")
        idx = torch.tensor(e, dtype=torch.int32, device="cuda")
        out = torch.empty(len(o) - 1, dtype=torch.float32, device="cuda")
        with pytest.raises(pm.PolymerError) as ei:
            pm.PageRankStatic(off, idx, out, 3)
        assert ei.value.status == 5, name  # PM_ERR_BAD_GRAPH
        assert b"invalid CSR" in pm.lib().pm_last_error(), name
    # a 3-cycle: every rank stays 1/3
    off = torch.tensor([0, 1, 2, 3], dtype=torch.int32, device="cuda")
    idx = torch.tensor([1, 2, 0], dtype=torch.int32, device="cuda")
    out = torch.empty(3, dtype=torch.float32, device="cuda")
    pm.PageRankStatic(off, idx, out, 5)
    assert np.allclose(out.cpu().numpy(), 1.0 / 3.0, rtol=1e-6)


def test_pagerank_static_rejects_wrong_tensors(pm):
    import torch

    off = torch.tensor([0, 1, 2, 3], dtype=torch.int32, device="cuda")
    idx = torch.tensor([1, 2, 0], dtype=torch.int32, device="cuda")
    for bad_out in (torch.empty(2, dtype=torch.float32, device="cuda"),
                    torch.empty(3, dtype=torch.float64, device="cuda"),
                    torch.empty(6, dtype=torch.float32, device="cuda")[::2]):
        with pytest.raises(pm.PolymerError):
            pm.PageRankStatic(off, idx, bad_out, 3)
    with pytest.raises(pm.PolymerError):
        pm.PageRankStatic(off.long(), idx, torch.empty(3, dtype=torch.float32, device="cuda"), 3)
