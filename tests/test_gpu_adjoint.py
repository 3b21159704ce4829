"""GPU tests of the differentiation path: weighted PageRank, its adjoint and
the weighted SpMV backward, against the FP64 oracle, FP64 central finite
differences, and through the test-only torch.autograd binding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RL_GRAD = 1e-5   # relative error of gradients vs the FP64 adjoint
TOL = 1e-6       # relative L1 residual of the fixed points


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def weighted_graph(oracle, scale):
    og = oracle.rmat_graph(scale, 16)
    w32 = oracle.lognormal_weights(og).astype(np.float32)
    return og, w32


def targets(oracle, og, k, seed=0x5EED0008, limit=None):
    lim = og.n if limit is None else limit
    t = []
    j = 0
    while len(t) < k:
        v = oracle.lib().pmo_hash(seed, j) % lim
        j += 1
        if v not in t:
            t.append(int(v))
    return np.array(t, np.int64)


def test_weighted_pagerank_matches_oracle(pm, oracle):
    og, w = weighted_graph(oracle, 16)
    ref, it_ref = oracle.weighted_pagerank(og, w.astype(np.float64), tol=TOL)
    with pm.Graph.from_csr(og.off, og.idx) as g:
        g.set_weights(w)
        p, it, res = pm.WeightedPageRank(g, tol=TOL)
    assert res <= TOL and abs(it - it_ref) <= 2
    assert rel(p, ref) < 2e-6


@pytest.mark.parametrize("scale,k", [(14, 64), (20, 1024)])
def test_pagerank_adjoint_vs_fp64_adjoint(pm, oracle, scale, k):
    """Weighted PageRank at scale 20, loss = sum of the ranks of
    1024 seeded targets, gradient for every edge weight."""
    og, w = weighted_graph(oracle, scale)
    w64 = w.astype(np.float64)
    tgt = targets(oracle, og, k)
    gp = np.zeros(og.n)
    gp[tgt] = 1.0
    p_ref, _ = oracle.weighted_pagerank(og, w64, tol=1e-10)
    dw_ref, lam_ref, _ = oracle.pagerank_adjoint(og, w64, p_ref, gp, tol=1e-10)
    with pm.Graph.from_csr(og.off, og.idx) as g:
        g.set_weights(w)
        p, it_f, _ = pm.WeightedPageRank(g, tol=TOL)
        dw, lam, it_a = pm.PageRankAdjoint(g, p, gp.astype(np.float32), tol=TOL, with_lambda=True)
    assert rel(lam, lam_ref) < RL_GRAD
    assert rel(dw, dw_ref) < RL_GRAD
    assert it_a <= 2.5 * it_f


def test_pagerank_gradient_finite_differences(pm, oracle):
    """FP64 central differences, step 1e-6, on 64 random edges of a
    4096-vertex induced subgraph of the scale-20 graph."""
    og, w = weighted_graph(oracle, 20)
    sub, ws = oracle.induced_subgraph(og, 4096, w)
    ws64 = ws.astype(np.float64)
    tgt = targets(oracle, sub, 64, limit=sub.n)
    gp = np.zeros(sub.n)
    gp[tgt] = 1.0
    p, _ = oracle.weighted_pagerank(sub, ws64, tol=1e-14, max_iters=5000)
    dw_ref, _, _ = oracle.pagerank_adjoint(sub, ws64, p, gp, tol=1e-14, max_iters=5000)
    rng = np.random.default_rng(0x5EED)
    edges = rng.choice(sub.m, 64, replace=False)
    h = 1e-6
    fd = np.empty(64)
    for i, e in enumerate(edges):
        wp = ws64.copy()
        wp[e] += h
        wm = ws64.copy()
        wm[e] -= h
        lp = oracle.weighted_pagerank(sub, wp, tol=1e-14, max_iters=5000)[0][tgt].sum()
        lm = oracle.weighted_pagerank(sub, wm, tol=1e-14, max_iters=5000)[0][tgt].sum()
        fd[i] = (lp - lm) / (2 * h)
    # the FP64 adjoint itself; the bound is the FD noise: loss differences of
    # ~1e-14 on a loss of ~1e-2 carry ~1e-6 relative rounding error
    assert rel(dw_ref[edges], fd) < 1e-5
    with pm.Graph.from_csr(sub.off, sub.idx) as g:
        g.set_weights(ws)
        pg, _, _ = pm.WeightedPageRank(g, tol=1e-7)
        dw, _ = pm.PageRankAdjoint(g, pg, gp.astype(np.float32), tol=1e-7)
    assert rel(dw[edges], fd) < 1e-4


def test_spmv_backward_vs_oracle(pm, oracle):
    og, w = weighted_graph(oracle, 20)
    x = oracle.uniform01(og.n, seed=11)
    gy = oracle.uniform01(og.n, seed=12)
    dx_ref, dw_ref = oracle.spmv_backward(og, w.astype(np.float64), x, gy)
    with pm.Graph.from_csr(og.off, og.idx) as g:
        g.set_weights(w)
        dx, dw = pm.SpMVBackward(g, x, gy)
    assert rel(dx, dx_ref) < RL_GRAD
    assert rel(dw, dw_ref) < 1e-7  # a single product per edge


def test_autograd_binding(pm, oracle):
    import torch

    from autograd_binding import WeightedPageRank, WeightedSpMV
    og, w = weighted_graph(oracle, 14)
    tgt = torch.tensor(targets(oracle, og, 32), device="cuda")
    with pm.Graph.from_csr(og.off, og.idx) as g:
        wt = torch.tensor(w, device="cuda", requires_grad=True)
        p = WeightedPageRank.apply(wt, g, 0.85, 1e-7, 1000)
        loss = p[tgt].sum()
        loss.backward()
        gp = np.zeros(og.n)
        gp[tgt.cpu().numpy()] = 1.0
        p_ref, _ = oracle.weighted_pagerank(og, w.astype(np.float64), tol=1e-10)
        dw_ref, _, _ = oracle.pagerank_adjoint(og, w.astype(np.float64), p_ref, gp, tol=1e-10)
        assert rel(wt.grad.cpu().numpy(), dw_ref) < RL_GRAD
        x = torch.tensor(oracle.uniform01(og.n, seed=3), device="cuda", requires_grad=True)
        w2 = torch.tensor(w, device="cuda", requires_grad=True)
        y = WeightedSpMV.apply(x, w2, g)
        (y * y).sum().backward()
        gy = 2 * y.detach().cpu().numpy().astype(np.float64)
        dx_ref, dw2_ref = oracle.spmv_backward(og, w.astype(np.float64), x.detach().cpu().numpy(), gy)
        assert rel(x.grad.cpu().numpy(), dx_ref) < RL_GRAD
        assert rel(w2.grad.cpu().numpy(), dw2_ref) < 1e-6
