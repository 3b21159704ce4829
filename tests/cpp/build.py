"""Builds tests/cpp/_build/lib<name>.so: applications compiled outside the
library against include/polymer_b200_engine.cuh and linked with
libpolymer_b200.so (test infrastructure): user_max_label (functors in the
engine's own shape) and ref_shape_apps (functors in the reference's shape)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def build(name: str = "user_max_label") -> str:
    out = os.path.join(HERE, "_build", "lib%s.so" % name)
    src = os.path.join(HERE, name + ".cu")
    deps = [src, os.path.join(ROOT, "include", "polymer_b200_engine.cuh"),
            os.path.join(ROOT, "include", "polymer_b200.h"),
            os.path.join(ROOT, "polymer_b200", "libpolymer_b200.so")]
    inc = os.path.join(ROOT, "include", "pm")
    deps += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".cuh")]
    if os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out) for d in deps):
        return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "include"), src, "-o", out,
           "-L" + os.path.join(ROOT, "polymer_b200"), "-lpolymer_b200",
           "-Xlinker", "-rpath," + os.path.join(ROOT, "polymer_b200")]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s" % (name, p.stderr))
    return out


if __name__ == "__main__":
    for n in ("user_max_label", "ref_shape_apps"):
        print(build(n))
