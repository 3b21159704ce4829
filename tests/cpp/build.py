"""Builds tests/cpp/_build/libuser_max_label.so: an application compiled
outside the library against include/polymer_b200_engine.cuh and linked with
libpolymer_b200.so (test infrastructure)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build", "libuser_max_label.so")


def build() -> str:
    src = os.path.join(HERE, "user_max_label.cu")
    deps = [src, os.path.join(ROOT, "include", "polymer_b200_engine.cuh"),
            os.path.join(ROOT, "polymer_b200", "libpolymer_b200.so")]
    csrc = os.path.join(ROOT, "include", "pm")
    deps += [os.path.join(csrc, f) for f in os.listdir(csrc) if f.endswith(".cuh")]
    if os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "include"), src, "-o", OUT,
           "-L" + os.path.join(ROOT, "polymer_b200"), "-lpolymer_b200",
           "-Xlinker", "-rpath," + os.path.join(ROOT, "polymer_b200")]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return OUT


if __name__ == "__main__":
    print(build())
