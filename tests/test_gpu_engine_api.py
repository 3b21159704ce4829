"""GPU test of the C++ engine API (include/polymer_b200_engine.cuh): an
application compiled outside the library with its own functors
(tests/cpp/user_max_label.cu: max-label components through edgeMapReduce,
vertexMapAll and vertexFilter) runs on a graph handle of the library and
matches the oracle in every direction regime."""
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
    L.user_max_label.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.user_max_label.restype = C.c_int
    return L


@pytest.mark.parametrize("mode", ["default", "dense", "sparse"])
def test_user_max_label_app(pm, oracle, mode):
    import torch
    L = _user_lib(pm)
    og = oracle.rmat_graph(14, 16, symmetric=True)
    comp = oracle.cc(og)                      # min id of each component
    mx = np.full(og.n, -1, np.int64)
    np.maximum.at(mx, comp, np.arange(og.n))  # max id of each component
    want = mx[comp].astype(np.int32)
    thr = {"default": og.m // 8, "dense": 0, "sparse": 1 << 40}[mode]
    with pm.Graph.from_csr(og.off, og.idx, symmetric=True) as g:
        lab = torch.empty(og.n, dtype=torch.int32, device="cuda")
        roots, rounds, dense = C.c_int64(), C.c_int(), C.c_int()
        torch.cuda.synchronize()
        st = L.user_max_label(g.handle, C.c_void_p(lab.data_ptr()), thr, C.byref(roots), C.byref(rounds),
                              C.byref(dense))
        assert st == 0, pm.lib().pm_last_error()
        got = lab.cpu().numpy()
    assert np.array_equal(got, want)
    assert roots.value == len(np.unique(comp))
    if mode == "dense":
        assert dense.value == rounds.value
    if mode == "sparse":
        assert dense.value == 0
