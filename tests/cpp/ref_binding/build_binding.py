"""Builds tests/cpp/_build/numa-PageRank-b200: the reference's numa-PageRank.C
with the body of its PageRank(graph<vertex>&, int) replaced by
pagerank_b200.inc (the binding INTEGRATION.md shows), compiled the way
oracle/Makefile compiles the reference (the single-node libnuma stand-in in
oracle/shim) and linked with libpolymer_b200.so.  Test infrastructure.

The reference source is read where it lies (the oracle's REFERENCE_DIR) and
the spliced copy is written under tests/cpp/_build, outside version control;
nothing is built when the reference sources are absent."""
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
OUT_DIR = os.path.join(ROOT, "tests", "cpp", "_build")
EXE = os.path.join(OUT_DIR, "numa-PageRank-b200")


def splice(src_text: str) -> str:
    """Replace the PageRank(graph<vertex>&, int) template (its `template`
    line through the matching closing brace) by an include of the binding."""
    m = re.search(r"template\s*<class vertex>\s*\n\s*void PageRank\(graph<vertex> &GA, int maxIter\)\s*\{", src_text)
    if not m:
        raise RuntimeError("PageRank(graph<vertex>&, int) not found")
    depth, i = 0, src_text.index("{", m.start())
    while True:
        c = src_text[i]
        if c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                break
        i += 1
    return src_text[:m.start()] + '#include "pagerank_b200.inc"\n' + src_text[i + 1:]


def build(reference_dir: str) -> str:
    src = os.path.join(reference_dir, "numa-PageRank.C")
    lib = os.path.join(ROOT, "polymer_b200", "libpolymer_b200.so")
    deps = [src, os.path.join(HERE, "pagerank_b200.inc"), os.path.join(ROOT, "include", "polymer_b200.h"), lib,
            __file__]
    if os.path.exists(EXE) and all(os.path.getmtime(d) <= os.path.getmtime(EXE) for d in deps):
        return EXE
    os.makedirs(OUT_DIR, exist_ok=True)
    spliced = os.path.join(OUT_DIR, "numa-PageRank-b200.C")
    with open(src) as f:
        text = splice(f.read())
    with open(spliced, "w") as f:
        f.write(text)
    cmd = ["g++", "-O2", "-w", "-DOPENMP", "-fopenmp", "-U_FORTIFY_SOURCE", "-D_FORTIFY_SOURCE=0",
           "-I" + os.path.join(ROOT, "oracle", "shim"), "-I" + reference_dir, "-I" + HERE,
           "-I" + os.path.join(ROOT, "include"), spliced, "-o", EXE,
           "-L" + os.path.join(ROOT, "polymer_b200"), "-lpolymer_b200",
           "-Wl,-rpath,$ORIGIN/../../../polymer_b200", "-pthread"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("g++ failed:\n" + p.stderr[-3000:])
    return EXE


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pm_oracle
    print(build(pm_oracle.REFERENCE_DIR))
