"""CPU tests of the C ABI library: it loads, exports every symbol declared in
include/polymer_b200.h, and fails loudly (a status, not a crash or a CPU
fallback) when no GPU is visible.  No compute call runs here."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT, have_gpu

HEADER = os.path.join(ROOT, "include", "polymer_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^PM_API\s+[\w\s\*]+?\b(pm_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("pm_graph_create", "pm_bfs", "pm_components", "pm_bellman_ford", "pm_pagerank",
              "pm_spmv", "pm_bp", "pm_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    import polymer_b200
    if not os.path.exists(polymer_b200.LIB_PATH):
        from polymer_b200 import _build
        _build.build()
    L = C.CDLL(polymer_b200.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_checked_build_exports_every_declared_symbol():
    """The bounds-checked build (PM_CHECK=1) is the same C ABI."""
    import polymer_b200
    path = os.path.join(os.path.dirname(polymer_b200.LIB_PATH), "libpolymer_b200_check.so")
    if not os.path.exists(path):
        pytest.skip("checked build not built (__graft_entry__.build())")
    L = C.CDLL(path)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_version_string():
    import polymer_b200
    assert b"sm_100a" in polymer_b200.lib().pm_version()


@pytest.mark.skipif(have_gpu(), reason="checks the no-GPU error path")
def test_no_device_is_an_error_not_a_fallback():
    import numpy as np
    import polymer_b200 as pm
    with pytest.raises(pm.PolymerError) as ei:
        pm.Graph.from_csr(np.array([0, 1, 1], np.int32), np.array([1], np.int32))
    assert ei.value.status in (3, 7)  # CUDA error or no device
    assert pm.lib().pm_last_error()


def test_null_handle_is_invalid_arg():
    import polymer_b200 as pm
    st = pm.lib().pm_bfs(None, 0, None, None, 0, -1, None)
    assert st == 1
    assert b"null graph" in pm.lib().pm_last_error()


def test_default_tunables_host_only():
    """The process-wide tunables (NULL handle) are host state: set, read back,
    range-checked and restored without a GPU."""
    import polymer_b200 as pm
    defaults = {"heavy_deg": 1024, "cta_expand": 128, "grid_expand": 256, "pull_ctas_per_sm": 0,
                "bfs_div": 20, "cc_div": 8, "bf_div": 20, "cuda_graphs": 1, "multi_div": 8, "bf_dense": 2,
                "cc_mode": 0, "bf_delta": 0, "pull_stage": 0, "push_agg": 0}
    assert {k: pm.get_default_tunable(k) for k in defaults} == defaults
    try:
        pm.set_default_tunable("heavy_deg", 4096)
        pm.set_default_tunable("bfs_div", 64)
        assert pm.get_default_tunable("heavy_deg") == 4096 and pm.get_default_tunable("bfs_div") == 64
        for name, bad in (("heavy_deg", 63), ("grid_expand", 31), ("pull_ctas_per_sm", 65),
                          ("cc_div", 0), ("cuda_graphs", -1)):
            with pytest.raises(pm.PolymerError) as ei:
                pm.set_default_tunable(name, bad)
            assert ei.value.status == 1
        assert pm.lib().pm_graph_set_tunable(None, 42, 1) == 1
        assert b"unknown tunable" in pm.lib().pm_last_error()
    finally:
        for k, v in defaults.items():
            pm.set_default_tunable(k, v)
    assert {k: pm.get_default_tunable(k) for k in defaults} == defaults


@pytest.mark.skipif(not os.path.exists(os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")),
                    reason="needs nvcc")
def test_engine_api_compiles_outside_the_library():
    """An application with its own functors (tests/cpp/user_max_label.cu)
    compiles against include/polymer_b200_engine.cuh and links with the
    library: every engine symbol it needs is exported."""
    import sys
    import polymer_b200
    if not os.path.exists(polymer_b200.LIB_PATH):
        from polymer_b200 import _build
        _build.build()
    sys.path.insert(0, os.path.join(ROOT, "tests", "cpp"))
    import build
    so = build.build()
    L = C.CDLL(so)
    assert hasattr(L, "user_max_label")


def test_tuning_table_round_trip(tmp_path):
    """A tuning table saved as JSON and loaded as process defaults (host
    state, no GPU); unknown names are refused."""
    import polymer_b200 as pm
    before = {k: pm.get_default_tunable(k) for k in pm.TUNABLES}
    path = str(tmp_path / "tuning.json")
    try:
        pm.save_tuning(path, {"heavy_deg": 512, "bfs_div": 64, "grid_expand": 256}, note="R-MAT 22 symmetric")
        assert pm.load_tuning(path) == {"heavy_deg": 512, "bfs_div": 64, "grid_expand": 256}
        assert pm.get_default_tunable("heavy_deg") == 512 and pm.get_default_tunable("bfs_div") == 64
        with pytest.raises(pm.PolymerError):
            pm.save_tuning(path, {"no_such_knob": 1})
    finally:
        for k, v in before.items():
            pm.set_default_tunable(k, v)


def test_failure_hooks_host_only():
    """The allocation-failure injection is host state (set and cleared without
    a GPU); the wait test needs a device and says so without one."""
    import polymer_b200 as pm
    pm.test_fail_alloc_after(3)
    pm.test_fail_alloc_after(0)
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        with pytest.raises(pm.PolymerError) as ei:
            pm.test_wait_timeout(10)
        assert ei.value.status == 7  # PM_ERR_NO_DEVICE


def test_memory_cache_settings_host_only():
    import polymer_b200 as pm
    pm.set_memory_cache(1 << 30)
    pm.set_memory_cache(-1)
    assert pm.memory_cached() == 0  # nothing allocated without a GPU
    pm.release_memory_cache()


def test_header_is_plain_c(tmp_path):
    """include/polymer_b200.h compiles as C99 with -pedantic: the boundary is a
    C ABI a cgo / JNI / ctypes host can bind."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("needs gcc")
    src = tmp_path / "c_abi.c"
    src.write_text('#include "polymer_b200.h"\nint main(void) { pm_graph *g = 0; (void)g; return 0; }\n')
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I" + os.path.join(ROOT, "include"),
                        "-fsyntax-only", str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
