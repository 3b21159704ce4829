"""Build of the CUDA engine: one nvcc invocation per translation unit, linked
into polymer_b200/libpolymer_b200.so (sm_100a only), in-tree so that the
shared object travels with the source tree."""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libpolymer_b200.so")
# The checked build: every vertex id the engine kernels read is bounds-tested
# (PM_CHECK=1); loaded instead of LIB when POLYMER_B200_CHECKED=1.
OBJ_CHECK = os.path.join(PKG, "_build_check")
LIB_CHECK = os.path.join(PKG, "libpolymer_b200_check.so")
SOURCES = ["pm_engine.cu", "pm_graph.cu", "pm_apps.cu", "pm_batch.cu", "pm_adjoint.cu", "pm_capi.cu",
           "pm_static.cu", "pm_tune.cu", "pm_ingest.cu", "pm_alloc.cu", "pm_async.cu",
           "pm_partition.cu", "pm_hubs.cu", "pm_dump.cu", "pm_cc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The engine's headers (the public template layer) live under include/pm.
ENGINE_INC = os.path.join(ROOT, "include", "pm")
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + ENGINE_INC, "-I" + CSRC]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False, checked: bool = False) -> str:
    obj_dir, lib = (OBJ_CHECK, LIB_CHECK) if checked else (OBJ, LIB)
    os.makedirs(obj_dir, exist_ok=True)
    headers = [os.path.join(d, f) for d in (CSRC, ENGINE_INC) for f in os.listdir(d) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "polymer_b200.h"))
    nvcc = _nvcc()
    extra = (["-Xptxas", "-v"] if ptxas_info else []) + (["-DPM_CHECK=1"] if checked else [])

    def compile_one(src):
        s = os.path.join(CSRC, src)
        o = os.path.join(obj_dir, src.replace(".cu", ".o"))
        if force or ptxas_info or _stale(o, [s] + headers):
            cmd = [nvcc, *ARCH, *FLAGS, *extra, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            p = subprocess.run(cmd, capture_output=True, text=True)
            if p.returncode != 0:
                raise RuntimeError("nvcc failed for %s:\n%s" % (src, p.stderr))
            if ptxas_info or verbose:
                sys.stderr.write(p.stderr)
        return o

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    if force or _stale(lib, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", lib, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n%s" % p.stderr)
    return lib


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
