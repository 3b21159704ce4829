"""Test-only torch.autograd bindings of the engine's adjoint kernels.

Weighted PageRank p(W) and one weighted SpMV y(x, W) as autograd functions
whose backward passes call pm_pagerank_adjoint / pm_spmv_backward through the
C ABI.  W is a float32 CUDA tensor of per-CSR-edge weights.
"""
import torch

import polymer_b200 as pm


class WeightedPageRank(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w, graph, damping=0.85, tol=1e-6, max_iters=1000):
        graph.set_weights(w.detach().contiguous())
        p = torch.empty(graph.n, dtype=torch.float32, device=w.device)
        torch.cuda.synchronize()
        pm.WeightedPageRank(graph, damping, tol, max_iters, device_out=p, out=p)
        ctx.graph, ctx.damping, ctx.tol, ctx.max_iters = graph, damping, tol, max_iters
        ctx.save_for_backward(w, p)
        return p

    @staticmethod
    def backward(ctx, grad_p):
        w, p = ctx.saved_tensors
        ctx.graph.set_weights(w.detach().contiguous())
        g = grad_p.detach().to(torch.float32).contiguous()
        dw = torch.empty(ctx.graph.m, dtype=torch.float32, device=w.device)
        torch.cuda.synchronize()
        pm.PageRankAdjoint(ctx.graph, p, g, ctx.damping, ctx.tol, ctx.max_iters, out=dw)
        return dw, None, None, None, None


class WeightedSpMV(torch.autograd.Function):
    """y = A_W^T x, i.e. y[v] = sum over edges s->v of W_e x[s]."""

    @staticmethod
    def forward(ctx, x, w, graph):
        graph.set_weights(w.detach().contiguous())
        xs = x.detach().to(torch.float32).contiguous()
        torch.cuda.synchronize()
        y = pm.SPMV(graph, xs, 1)
        ctx.graph = graph
        ctx.save_for_backward(xs, w)
        return y

    @staticmethod
    def backward(ctx, grad_y):
        x, w = ctx.saved_tensors
        ctx.graph.set_weights(w.detach().contiguous())
        torch.cuda.synchronize()
        dx, dw = pm.SpMVBackward(ctx.graph, x, grad_y.detach().to(torch.float32).contiguous())
        return dx, dw, None
