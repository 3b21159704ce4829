"""GPU test of the C++ engine API (include/polymer_b200_engine.cuh): an
application compiled outside the library with its own functors
(tests/cpp/user_max_label.cu: max-label components through edgeMapReduce,
or edgeMap with the DENSE_FORWARD option, vertexMapAll and vertexFilter)
runs on a graph handle of the library and matches the oracle in every
direction regime."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _user_lib(pm):
    sys.path.insert(0, os.path.join(ROOT, "tests", "cpp"))
    import build
    pm.lib()  # the library first: the application links against the same copy
    L = C.CDLL(build.build())
    L.user_max_label.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.user_max_label.restype = C.c_int
    return L


@pytest.mark.parametrize("mode", ["default", "dense", "sparse", "push", "dense_push"])
def test_user_max_label_app(pm, oracle, mode):
    import torch
    L = _user_lib(pm)
    og = oracle.rmat_graph(14, 16, symmetric=True)
    comp = oracle.cc(og)                      # min id of each component
    mx = np.full(og.n, -1, np.int64)
    np.maximum.at(mx, comp, np.arange(og.n))  # max id of each component
    want = mx[comp].astype(np.int32)
    thr = {"default": og.m // 8, "dense": 0, "sparse": 1 << 40, "push": og.m // 8, "dense_push": 0}[mode]
    push = int(mode in ("push", "dense_push"))
    with pm.Graph.from_csr(og.off, og.idx, symmetric=True) as g:
        lab = torch.empty(og.n, dtype=torch.int32, device="cuda")
        roots, rounds, dense = C.c_int64(), C.c_int(), C.c_int()
        torch.cuda.synchronize()
        st = L.user_max_label(g.handle, C.c_void_p(lab.data_ptr()), thr, push, C.byref(roots), C.byref(rounds),
                              C.byref(dense))
        assert st == 0, pm.lib().pm_last_error()
        got = lab.cpu().numpy()
    assert np.array_equal(got, want)
    assert roots.value == len(np.unique(comp))
    if mode in ("dense", "dense_push"):
        assert dense.value == rounds.value
    if mode == "sparse":
        assert dense.value == 0


def _ref_shape_lib(pm):
    sys.path.insert(0, os.path.join(ROOT, "tests", "cpp"))
    import build
    pm.lib()
    L = C.CDLL(build.build("ref_shape_apps"))
    L.ref_components.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int),
                                 C.POINTER(C.c_int)]
    L.ref_components.restype = C.c_int
    L.ref_pagerank.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int64]
    L.ref_pagerank.restype = C.c_int
    return L


@pytest.mark.parametrize("mode", ["default", "dense", "sparse"])
def test_reference_shaped_components(pm, oracle, mode):
    """CC_F / CC_Vertex_F in the reference's shape (numa-Components.C:55-119:
    initFunc / reduceFunc / combineFunc, two-argument updateAtomic, writeMin)
    through pm::edgeMapReduce: min-id labels exactly as the oracle's."""
    import torch
    L = _ref_shape_lib(pm)
    og = oracle.rmat_graph(14, 16, symmetric=True)
    thr = {"default": og.m // 8, "dense": 0, "sparse": 1 << 40}[mode]
    with pm.Graph.from_csr(og.off, og.idx, symmetric=True) as g:
        ids = torch.empty(og.n, dtype=torch.int32, device="cuda")
        prev = torch.empty(og.n, dtype=torch.int32, device="cuda")
        rounds, dense = C.c_int(), C.c_int()
        torch.cuda.synchronize()
        st = L.ref_components(g.handle, C.c_void_p(ids.data_ptr()), C.c_void_p(prev.data_ptr()), thr,
                              C.byref(rounds), C.byref(dense))
        assert st == 0, pm.lib().pm_last_error()
        got = ids.cpu().numpy()
    assert np.array_equal(got, oracle.cc(og))
    if mode == "dense":
        assert dense.value == rounds.value
    if mode == "sparse":
        assert dense.value == 0


@pytest.mark.parametrize("mode", ["dense", "sparse"])
def test_reference_shaped_pagerank(pm, oracle, mode):
    """PR_F's reducing members and PR_Vertex_F / PR_Vertex_Reset in the
    reference's shape (numa-PageRank.C:64-148), the loop of
    numa-PageRank.C:273-335, FP64: equal to the oracle's frontier-semantics
    PageRank to 1e-10 (dense rounds fold each row in CSC order; sparse rounds
    push with writeAdd)."""
    import torch
    L = _ref_shape_lib(pm)
    og = oracle.rmat_graph(13, 16)
    thr = {"dense": 0, "sparse": 1 << 40}[mode]
    iters = 10
    with pm.Graph.from_csr(og.off, og.idx) as g:
        pa = torch.empty(og.n, dtype=torch.float64, device="cuda")
        pb = torch.empty(og.n, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        st = L.ref_pagerank(g.handle, C.c_void_p(pa.data_ptr()), C.c_void_p(pb.data_ptr()), iters, thr)
        assert st == 0, pm.lib().pm_last_error()
        got = (pa if iters % 2 == 0 else pb).cpu().numpy()
    assert np.allclose(got, oracle.pagerank(og, iters), rtol=1e-10, atol=0)
