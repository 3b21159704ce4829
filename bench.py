#!/usr/bin/env python
"""Benchmark: GTEPS of the six Polymer applications on one B200.

One step runs the whole suite once on device-resident synthetic graphs:
  graph A  symmetrised R-MAT scale 22, edge factor 16, int32 weights U{1..22}:
           BFS from 16 seeded non-isolated sources, Connected Components,
           BellmanFord from the first source
  graph B  directed R-MAT scale 24, edge factor 16, float weights U(0,1]:
           PageRank 20 iterations (FP32), SpMV 10 iterations, BP 10 iterations
Edges counted (GTEPS numerator): BFS sum over sources of the out-degrees of
the reached vertices; CC and BellmanFord m; PageRank/SpMV/BP m per iteration.
value = counted edges / device time of the step (CUDA events on the graph
streams), aggregated over ranks.  `e2e` repeats the suite through the public
API from pinned host CSR arrays (graph upload + CSC build + results back).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GTEPS & %HBM peak per algo, 1 B200; batched/adjoint vs plain at FP64-tol"
SEED_GRAPH, SEED_W, SEED_X, SEED_PRIOR, SEED_SRC = (0x5EED0001, 0x5EED0002, 0x5EED0003,
                                                   0x5EED0004, 0x5EED0005)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)  # ~1.3 s timed: several clock samples
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--scale-a", type=int, default=22)
    p.add_argument("--scale-b", type=int, default=24)
    p.add_argument("--sources", type=int, default=16)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--e2e-pipeline-steps", type=int, default=6)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--no-tune", action="store_true",
                   help="keep the default tunables instead of running the autotuner at setup")
    p.add_argument("--no-cuda-graphs", action="store_true",
                   help="launch every kernel directly (the same work): for profilers that cannot see "
                        "kernels inside CUDA graphs with conditional nodes (the device-driven BFS rounds)")
    return p.parse_args()


# ---------------------------------------------------------------------------
def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def suite_config(scale_a, scale_b, n_sources, nA, mA, nB, mB, world):
    """The workload both arms run (and report under `config`): the graphs and
    applications of one step."""
    return {
        "workload": "six-application suite: BFS x%d + CC + BellmanFord on symmetrised R-MAT "
                    "scale %d ef16 (n=%d, m=%d); PageRank 20 it + SpMV 10 it + BP 10 it on "
                    "directed R-MAT scale %d ef16 (n=%d, m=%d)"
                    % (n_sources, scale_a, nA, mA, scale_b, nB, mB),
        "graphs": {"A": {"scale": scale_a, "n": nA, "m": mA}, "B": {"scale": scale_b, "n": nB, "m": mB}},
        "l2": "inputs larger than L2 (126 MB): graph A ids %d MB, graph B ids %d MB" % (mA * 4 >> 20, mB * 4 >> 20),
        "parallelism": "replicas x%d" % world,
    }


def _hash(seed, c):
    M = (1 << 64) - 1
    z = (seed + (c + 1) * 0x9E3779B97F4A7C15) & M
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
    return z ^ (z >> 31)


def pick_sources(off, k, seed):
    """k distinct seeded sources with out-edges (rank r of a replica run uses
    seed SEED_SRC + r, so ranks traverse from different sources)."""
    n = len(off) - 1
    out, seen = [], set()
    j = 0
    while len(out) < k and j < 64 * n:
        v = _hash(seed, j) % n
        j += 1
        if off[v + 1] > off[v] and v not in seen:
            seen.add(v)
            out.append(int(v))
    return out


# ---------------------------------------------------------------------------
class Suite:
    """The two device-resident graphs and the per-step application calls."""

    def __init__(self, pm, device, scale_a, scale_b, n_sources, rank):
        self.pm = pm
        t0 = time.time()
        self.A = pm.Graph.rmat(scale_a, 16, seed=SEED_GRAPH, symmetric=True, device=device)
        self.A.gen_weights_int(SEED_W, 22)
        self.B = pm.Graph.rmat(scale_b, 16, seed=SEED_GRAPH, symmetric=False, device=device)
        self.B.gen_weights_unit(SEED_W)
        self.setup_s = time.time() - t0
        offA, _ = self.A.csr()
        self.sources = self._pick_sources(offA, n_sources, SEED_SRC + rank)
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        n = self.B.n
        self.x0 = torch.from_numpy(self._uniform01(n, SEED_X)).to(self.dev)
        self.prior = torch.from_numpy(self._uniform_open(2 * n, SEED_PRIOR)).to(self.dev).view(n, 2)
        self.outA = torch.empty(self.A.n, dtype=torch.int32, device=self.dev)
        self.outB = torch.empty(self.B.n, dtype=torch.float32, device=self.dev)
        torch.cuda.synchronize(self.dev)
        self.tuning = None

    def tune(self):
        """Autotuner at setup (outside every timed region), one mix per graph
        (the applications that share its cut-offs): BFS + Components +
        BellmanFord on graph A, PageRank + SpMV + BP on graph B."""
        t0 = time.time()
        rep = {}
        for g, name, apps in ((self.A, "A", ["bfs", "cc", "bellman_ford"]),
                              (self.B, "B", ["pagerank", "spmv", "bp"])):
            r = g.tune(apps)
            rep["mix_" + name] = {"apps": apps, "trials": r["trials"],
                                  "default_ms": round(r["default_ms"], 3), "best_ms": round(r["best_ms"], 3)}
            rep["tunables_" + name] = g.tunables()
        rep["seconds"] = round(time.time() - t0, 2)
        self.tuning = rep
        return rep

    _hash = staticmethod(_hash)

    def _pick_sources(self, off, k, seed):
        return pick_sources(off, k, seed)

    def _uniform01(self, n, seed):
        return self.pm.uniform_f32(self.B, n, seed, open_interval=False).cpu().numpy()

    def _uniform_open(self, n, seed):
        return self.pm.uniform_f32(self.B, n, seed, open_interval=True).cpu().numpy()

    def step(self, per):
        """One pass of the suite; accumulates {algo: [ms, edges, algorithmic
        bytes]} into per.  Bytes per call: BFS 4 E_r + 12 n (E_r: out-degrees of
        the reached vertices); CC sum over rounds of 8 E_F + 12 n and
        BellmanFord of 12 E_F + 12 n (E_F: the round's frontier out-degrees);
        PageRank 8 m + 32 n, SpMV 12 m + 12 n, BP 4 m + 40 n per iteration."""
        pm, A, B = self.pm, self.A, self.B
        total_ms, total_edges = 0.0, 0
        nA, nB, mB = A.n, B.n, B.m

        def rec(name, ms, edges, nbytes):
            nonlocal total_ms, total_edges
            e = per.setdefault(name, [0.0, 0, 0])
            e[0] += ms
            e[1] += edges
            e[2] += nbytes
            total_ms += ms
            total_edges += edges

        for s in self.sources:
            A.timer_begin()
            _, _, st = pm.BFS(s, A, device_out=self.outA, stats=True)
            rec("bfs", A.timer_end(), st["edges_visited"], 4 * st["edges_visited"] + 12 * nA)
        A.timer_begin()
        _, st = pm.Components(A, device_out=self.outA, stats=True)
        rec("cc", A.timer_end(), A.m, 8 * st["edges_visited"] + 12 * nA * st["rounds"])
        A.timer_begin()
        _, st = pm.BellmanFord(A, self.sources[0], device_out=self.outA, stats=True)
        rec("bellman_ford", A.timer_end(), A.m, 12 * st["edges_visited"] + 12 * nA * st["rounds"])
        B.timer_begin()
        pm.PageRank(B, 20, dtype=np.float32, device_out=self.outB)
        rec("pagerank", B.timer_end(), mB * 20, (8 * mB + 32 * nB) * 20)
        B.timer_begin()
        pm.SPMV(B, self.x0, 10)
        rec("spmv", B.timer_end(), mB * 10, (12 * mB + 12 * nB) * 10)
        B.timer_begin()
        pm.BeliefPropagation(B, self.prior, 10)
        rec("bp", B.timer_end(), mB * 10, (4 * mB + 40 * nB) * 10)
        return total_ms, total_edges


def errors_block(pm, suite):
    """FP32 results of the timed suite against the same computations in FP64
    on the same graph and inputs (pm_pagerank PM_F64, pm_spmv_f64, pm_bp_f64,
    which the tests pin to the FP64 oracle): max-abs and relative-L1 error per
    result, computed on the device in FP64."""
    torch, B = suite.torch, suite.B

    def err(a32, a64):
        a = a32.reshape(-1).to(torch.float64)
        b = a64.reshape(-1)
        d = (a - b).abs()
        return {"max_abs": float(d.max()), "max_abs_fp64_value": float(b.abs().max()),
                "rel_l1": float(d.sum() / b.abs().sum().clamp_min(1e-300))}

    out = {}
    r32 = pm.PageRank(B, 20, dtype=np.float32, device_out=suite.outB)
    r64 = pm.PageRank(B, 20, dtype=np.float64, device_out=suite.outB)
    out["pagerank_20it"] = err(r32, r64)
    y32 = pm.SPMV(B, suite.x0, 10)
    y64 = pm.SPMV(B, suite.x0, 10, dtype=np.float64)
    out["spmv_10it"] = err(y32, y64)
    l32 = pm.BeliefPropagation(B, suite.prior, 10)
    l64 = pm.BeliefPropagation(B, suite.prior, 10, dtype=np.float64)
    out["bp_10it_logprod"] = err(l32, l64)
    out["reference_precision"] = ("the GPU's own FP64 path on the same graph and inputs; the FP64 oracle "
                                  "comparison at these sizes is tests/test_gpu_fullsize.py")
    return out


def use_tunables(pm, like):
    """Make `like`'s tunables the defaults of graphs created from now on (a
    user who tuned once stores the settings with the workload)."""
    for k, v in like.tunables().items():
        pm.set_default_tunable(k, v)


def e2e_run(pm, suite, steps, pipeline_steps, device=0):
    """Suite through the public API from pinned host CSR arrays, per step:
    upload + build both graphs, set weights, run, read every result back
    into preallocated pinned host buffers.

    Two schedules of the same steps.  `serial`: one host thread, each graph
    built, run and destroyed before the next is built.  The headline
    (`value`): one builder thread uploads and builds the graphs in step order
    (A, B, A, B, ...; the uploads share one host link, so one builder keeps it
    busy) up to two graphs ahead of each runner, while one runner thread per
    graph kind runs the applications on its current graph (own stream, the
    SMs) -- graph handles are independent, and the library's calls release
    the interpreter lock.  Every step's uploads and
    result reads are inside the timed region; the time is the host clock
    from the first upload to the last result, over the steps."""
    import queue
    A, B = suite.A, suite.B
    # the blocks cached by the earlier, unrelated phases (batched workloads,
    # tuning) are returned; the untimed steps below refill the cache with
    # this workload's sizes, as a serving process's earlier requests would
    suite.torch.cuda.synchronize()
    pm.release_memory_cache()
    pin = lambda c, t: pm.PinnedArray(c, t)
    hA = {"off": pin(A.n + 1, np.int32), "idx": pin(A.m, np.int32), "w": pin(A.m, np.int32)}
    hB = {"off": pin(B.n + 1, np.int32), "idx": pin(B.m, np.int32), "w": pin(B.m, np.float32),
          "x0": pin(B.n, np.float32), "prior": pin(2 * B.n, np.float32)}
    ns = len(suite.sources)
    oA = {"par": [pin(A.n, np.int32) for _ in range(ns)], "dep": [pin(A.n, np.int32) for _ in range(ns)],
          "lab": pin(A.n, np.int32), "dist": pin(A.n, np.int32)}
    oB = {"rank": pin(B.n, np.float32), "y": pin(B.n, np.float32), "lp": pin(2 * B.n, np.float32)}
    offA, idxA = A.csr()
    hA["off"].array[:] = offA
    hA["idx"].array[:] = idxA
    hA["w"].array[:] = A.weights_i32()
    offB, idxB = B.csr()
    hB["off"].array[:] = offB
    hB["idx"].array[:] = idxB
    hB["w"].array[:] = B.weights_f32()
    hB["x0"].array[:] = suite.x0.cpu().numpy()
    hB["prior"].array[:] = suite.prior.cpu().numpy().reshape(-1)
    h2d = sum(a.array.nbytes for a in hA.values()) + sum(a.array.nbytes for a in hB.values())
    d2h = sum(a.array.nbytes for a in oA["par"] + oA["dep"]) + oA["lab"].array.nbytes + \
        oA["dist"].array.nbytes + sum(a.array.nbytes for a in oB.values())

    create = threading.Lock()  # the tunable defaults are process-wide: set and used by one creation at a time

    def build(which):
        with create:
            use_tunables(pm, A if which == "A" else B)
            if which == "A":
                return pm.Graph.from_csr(hA["off"].array, hA["idx"].array, symmetric=True,
                                         weights=hA["w"].array)
            return pm.Graph.from_csr(hB["off"].array, hB["idx"].array, weights=hB["w"].array)

    def run(which, g):
        if which == "A":
            e = 0
            for k, s in enumerate(suite.sources):
                _, _, st = pm.BFS(s, g, stats=True, out=(oA["par"][k].array, oA["dep"][k].array))
                e += st["edges_visited"]
            pm.Components(g, out=oA["lab"].array)
            pm.BellmanFord(g, suite.sources[0], out=oA["dist"].array)
            return e + 2 * g.m
        pm.PageRank(g, 20, dtype=np.float32, out=oB["rank"].array)
        pm.SPMV(g, hB["x0"].array, 10, out=oB["y"].array)
        pm.BeliefPropagation(g, hB["prior"].array.reshape(-1, 2), 10, out=oB["lp"].array)
        return g.m * 40

    # serial schedule; the first step (untimed) fills the library's block
    # cache, as a serving process's earlier requests would have
    times, phases, edges = [], [], 0
    for it in range(steps + 1):
        suite.torch.cuda.synchronize()
        t0 = time.perf_counter()
        e, ph = 0, []
        for which in ("A", "B"):
            ta = time.perf_counter()
            g = build(which)
            tb = time.perf_counter()
            with g:
                e += run(which, g)
                tc = time.perf_counter()
            ph += [tb - ta, tc - tb, time.perf_counter() - tc]
        if it == 0:
            continue
        times.append(time.perf_counter() - t0)
        phases.append(ph)
        edges = e
    i = int(np.argsort(times)[len(times) // 2])
    names = ["build_A", "run_A", "free_A", "build_B", "run_B", "free_B"]
    serial = {"value": round(edges / times[i] / 1e9, 4), "seconds_per_step": round(times[i], 4),
              "phases_s": {k: round(v, 4) for k, v in zip(names, phases[i])},
              "timing": "host clock around synchronous API calls, median of %d steps after an untimed one" % steps}

    # pipelined schedule: one builder, at most two graphs of each kind ahead
    # of that kind's runner; every build and run is timed (host clock) so the
    # line can show where a slow step went
    failure, total = [], {"A": 0, "B": 0}
    spans = []  # (kind, "build" | "run", seconds)

    def timed(kind, phase, fn, *a):
        t_0 = time.perf_counter()
        r = fn(*a)
        spans.append((kind, phase, time.perf_counter() - t_0))
        return r
    queues = {"A": queue.Queue(maxsize=1), "B": queue.Queue(maxsize=1)}
    n_steps = [pipeline_steps]

    def put(q, g):  # False (and the graph closed) once any thread has failed
        while True:
            try:
                q.put(g, timeout=0.2)
                return True
            except queue.Full:
                if failure:
                    g.close()
                    return False

    def get(q):  # None once any thread has failed
        while True:
            try:
                return q.get(timeout=0.2)
            except queue.Empty:
                if failure:
                    return None

    def builder():
        try:
            for _ in range(n_steps[0]):
                for which in ("A", "B"):
                    if not put(queues[which], timed(which, "build", build, which)):
                        return
        except BaseException as exc:  # the runners stop on their next wait
            failure.append(exc)

    def runner(which):
        try:
            for _ in range(n_steps[0]):
                g = get(queues[which])
                if g is None:
                    return
                with g:
                    total[which] += timed(which, "run", run, which, g)
        except BaseException as exc:
            failure.append(exc)

    def pipelined(k):
        n_steps[0] = k
        total["A"] = total["B"] = 0
        suite.torch.cuda.synchronize()
        t0 = time.perf_counter()
        threads = [threading.Thread(target=builder, daemon=True)] + \
            [threading.Thread(target=runner, args=(w,), daemon=True) for w in ("A", "B")]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        for q in queues.values():  # graphs left after a failure
            while not q.empty():
                q.get().close()
        if failure:
            raise failure[0]
        return time.perf_counter() - t0

    # untimed: the pipeline keeps more graphs alive than the serial schedule;
    # their first builds would take their blocks from cudaMalloc
    pipelined(3)
    clocks = ClockSampler(device)
    clocks.start()
    del spans[:]
    t = pipelined(pipeline_steps)
    clk = clocks.stop()
    phases_p = {}
    for kind in ("A", "B"):
        for phase in ("build", "run"):
            d = [x[2] for x in spans if x[0] == kind and x[1] == phase]
            if d:
                phases_p["%s_%s" % (phase, kind)] = {"mean_s": round(float(np.mean(d)), 4),
                                                     "max_s": round(float(np.max(d)), 4)}
    for a in list(hA.values()) + list(hB.values()) + oA["par"] + oA["dep"] + [oA["lab"], oA["dist"]] + \
            list(oB.values()):
        a.free()
    edges = total["A"] + total["B"]
    return {"value": round(edges / t / 1e9, 4), "unit": "GTEPS", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "seconds_per_step": round(t / pipeline_steps, 4),
            "edges_per_step": int(edges // pipeline_steps), "cached_bytes_after": pm.memory_cached(),
            "timing": "host clock from the first upload to the last result read, %d steps after 3 untimed "
                      "ones; one builder thread uploads and builds the graphs in step order while one "
                      "runner thread per graph kind runs the current one" % pipeline_steps,
            "clocks": clk, "phases": phases_p, "serial": serial}


def batched_block(pm, suite, reps=3):
    """Batched workloads against plain runs on the same GPU, device time by
    CUDA events: 64-source BFS (uint64 lanes) vs 64 single-source BFS, 64-source
    BellmanFord (int32 lanes) vs 64 single-source runs, personalised PageRank
    for 32 seeds vs 32 plain runs, PageRank on 256 ER graphs in one launch vs
    256 launches."""
    A = suite.A
    offA, _ = A.csr()
    src64 = suite._pick_sources(offA, 64, SEED_SRC + 100)
    out = suite.torch.empty((64, A.n), dtype=suite.torch.int32, device=suite.dev)
    pm.BFSMulti(src64, A, device_out=out, out=out)
    ms_multi, st = [], None
    for _ in range(reps):
        A.timer_begin()
        _, st = pm.BFSMulti(src64, A, device_out=out, out=out, stats=True)
        ms_multi.append(A.timer_end())
    ms_plain = 0.0
    for s in src64:
        A.timer_begin()
        pm.BFS(s, A, device_out=suite.outA)
        ms_plain += A.timer_end()
    t = statistics.median(ms_multi)
    res = {"bfs64": {"ms": round(t, 3), "gteps": round(st["edges_visited"] / (t / 1e3) / 1e9, 2),
                     "plain_64_runs_ms": round(ms_plain, 3), "speedup_vs_plain": round(ms_plain / t, 2),
                     "graph": "symmetrised R-MAT scale %d" % int(np.log2(A.n))}}
    # asynchronous BFS (one persistent launch, reachability + parent tree) on the same sources
    pm.BFSAsync(src64[0], A, device_out=suite.outA, out=suite.outA)
    ms_async, e_async = 0.0, 0
    for s in src64[:16]:
        A.timer_begin()
        _, sta = pm.BFSAsync(s, A, device_out=suite.outA, out=suite.outA, stats=True)
        ms_async += A.timer_end()
        e_async += sta["edges_visited"]
    res["bfs_async16"] = {"ms_per_source": round(ms_async / 16, 3),
                          "gteps": round(e_async / (ms_async / 1e3) / 1e9, 2),
                          "level_synchronous_ms_per_source": round(ms_plain / 64, 3),
                          "note": "one persistent launch per source; parents form a valid tree, not a BFS tree"}
    # 64-source BellmanFord over the same graph's int32 weights (1..22)
    pm.BellmanFordMulti(src64, A, device_out=out, out=out)
    ms_multi = []
    for _ in range(reps):
        A.timer_begin()
        _, st = pm.BellmanFordMulti(src64, A, device_out=out, out=out, stats=True)
        ms_multi.append(A.timer_end())
    ms_plain, edges_plain = 0.0, 0
    for s in src64:
        A.timer_begin()
        _, st1 = pm.BellmanFord(A, s, device_out=suite.outA, stats=True)
        ms_plain += A.timer_end()
        edges_plain += st1["edges_visited"]
    t = statistics.median(ms_multi)
    res["bf64"] = {"ms": round(t, 3), "rounds": st["rounds"], "dense_rounds": st["dense_rounds"],
                   "plain_64_runs_ms": round(ms_plain, 3), "speedup_vs_plain": round(ms_plain / t, 2),
                   "plain_gteps": round(edges_plain / (ms_plain / 1e3) / 1e9, 2),
                   "gteps_equiv": round(edges_plain / (t / 1e3) / 1e9, 2),
                   "note": "gteps_equiv = edges the 64 plain runs visit / multi-source time"}
    # personalised PageRank, 32 one-hot seeds, 20 iterations, n x 32 FP32
    B = suite.B
    offB, _ = B.csr()
    seeds = suite._pick_sources(offB, 32, SEED_SRC + 200)
    outp = suite.torch.empty((B.n, 32), dtype=suite.torch.float32, device=suite.dev)
    pm.PersonalizedPageRank(B, seeds, 20, device_out=outp, out=outp)
    B.timer_begin()
    pm.PersonalizedPageRank(B, seeds, 20, device_out=outp, out=outp)
    t_ppr = B.timer_end()
    B.timer_begin()
    pm.PageRank(B, 20, dtype=np.float32, device_out=suite.outB)
    t_pr = B.timer_end()
    nB, mB = B.n, B.m
    res["ppr32"] = {"ms": round(t_ppr, 3), "gteps": round(32 * 20 * mB / (t_ppr / 1e3) / 1e9, 2),
                    "algorithmic_gbs": round(20 * (132 * mB + 264 * nB) / (t_ppr / 1e3) / 1e9, 1),
                    "algorithmic_note": "132 m + 264 n bytes per iteration; the gathered 128-byte rows "
                                        "mostly hit L2, so DRAM moves less (ncu summary in profiles/)",
                    "plain_32_vectors_ms": round(32 * t_pr, 3),
                    "speedup_vs_plain": round(32 * t_pr / t_ppr, 2),
                    "plain": "32 x one FP32 PageRank run of 20 iterations (one vector per run)"}
    # 256 Erdos-Renyi graphs, n log-uniform in [1k, 100k], avg degree 8, PageRank 20 it each
    with pm.Graph.er_batch(256, 1000, 100000, 8) as G:
        vb = G.parts()
        outg = suite.torch.empty(G.n, dtype=suite.torch.float32, device=suite.dev)
        pm.PageRankParts(G, 20, device_out=outg, out=outg)
        G.timer_begin()
        pm.PageRankParts(G, 20, device_out=outg, out=outg)
        t_parts = G.timer_end()
        off, idx = G.csr()
        t_plain = 0.0
        for i in range(len(vb) - 1):
            a, b = int(vb[i]), int(vb[i + 1])
            with pm.Graph.from_csr((off[a:b + 1] - off[a]).astype(np.int32),
                                   (idx[off[a]:off[b]] - a).astype(np.int32)) as gi:
                o = suite.torch.empty(b - a, dtype=suite.torch.float32, device=suite.dev)
                gi.timer_begin()
                pm.PageRank(gi, 20, dtype=np.float32, device_out=o, out=o)
                t_plain += gi.timer_end()
        res["er256_pagerank"] = {"ms": round(t_parts, 3), "n": int(G.n), "m": int(G.m),
                                 "gteps": round(20 * G.m / (t_parts / 1e3) / 1e9, 2),
                                 "plain_256_runs_ms": round(t_plain, 3),
                                 "speedup_vs_plain": round(t_plain / t_parts, 2),
                                 "launches": "one persistent launch (8-CTA clusters, work queue)"}
    return res


def ingest_block(pm, reps=3):
    """PBBS text ingest (pm_graph_load_pbbs): directed R-MAT scale 20 written
    as an AdjacencyGraph text file, read back with the header on the host and
    the body tokenised and parsed on the GPU, then validated and transposed
    (CSC) on the device; host clock around the synchronous call, file in the
    page cache after the first read.  Also the binary triple."""
    import tempfile
    with pm.Graph.rmat(20, 16, seed=SEED_GRAPH) as G:
        off, idx = G.csr()
    d = tempfile.mkdtemp(prefix="pm_ingest_")
    path = os.path.join(d, "rmat20.adj")
    with open(path, "w") as f:
        f.write("AdjacencyGraph\n%d\n%d\n" % (len(off) - 1, len(idx)))
    with open(path, "a") as f:
        off[:-1].tofile(f, sep="\n")
        f.write("\n")
        idx.tofile(f, sep="\n")
        f.write("\n")
    base = os.path.join(d, "rmat20b")
    with open(base + ".config", "w") as f:
        f.write("%d\n" % (len(off) - 1))
    idx.astype(np.int32).tofile(base + ".adj")
    off[:-1].astype(np.int32).tofile(base + ".idx")
    size = os.path.getsize(path)
    out = {"graph": "directed R-MAT scale 20 (n=%d, m=%d)" % (len(off) - 1, len(idx)), "text_bytes": size}
    for name, kw, p in (("text", {}, path), ("binary", {"binary": True}, base)):
        times = []
        for _ in range(reps + 1):
            t0 = time.perf_counter()
            with pm.Graph.load_pbbs(p, **kw) as g:
                assert g.m == len(idx)
            times.append(time.perf_counter() - t0)
        t = statistics.median(times[1:])
        out[name] = {"seconds": round(t, 4), "medges_per_s": round(len(idx) / t / 1e6, 1)}
        if name == "text":
            out[name]["mb_per_s"] = round(size / t / 1e6, 1)
    for fn in (path, base + ".config", base + ".adj", base + ".idx"):
        os.remove(fn)
    os.rmdir(d)
    out["timing"] = "host clock around the call (file read, parse, validation, CSC build), median of %d" % reps
    return out


def adjoint_block(pm, torch, dev, reps=3):
    """Weighted PageRank on directed R-MAT scale 20 with
    lognormal(0,1) weights normalised per source row, damping 0.85, solved to
    1e-6 relative L1; loss = sum of the ranks of 1024 seeded targets; adjoint
    (transposed iteration + per-edge gradient) vs forward solve, and the
    weighted SpMV backward vs one forward SpMV, device time."""
    with pm.Graph.rmat(20, 16, seed=SEED_GRAPH) as G:
        G.gen_weights_lognormal(0x5EED0007)
        n, m = G.n, G.m
        tgt = []
        j = 0
        while len(tgt) < 1024:
            v = Suite._hash(0x5EED0008, j) % n
            j += 1
            if v not in tgt:
                tgt.append(v)
        gp = torch.zeros(n, dtype=torch.float32, device=dev)
        gp[torch.tensor(tgt, device=dev)] = 1.0
        p = torch.empty(n, dtype=torch.float32, device=dev)
        dw = torch.empty(m, dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        fwd, adj, it_f, it_a = [], [], 0, 0
        for _ in range(reps + 1):
            G.timer_begin()
            _, it_f, _ = pm.WeightedPageRank(G, 0.85, 1e-6, 1000, device_out=p, out=p)
            fwd.append(G.timer_end())
            G.timer_begin()
            _, it_a = pm.PageRankAdjoint(G, p, gp, 0.85, 1e-6, 1000, out=dw)
            adj.append(G.timer_end())
        x = pm.uniform_f32(G, n, SEED_X)
        G.timer_begin()
        for _ in range(10):
            pm.SPMV(G, x, 1)
        t_spmv = G.timer_end() / 10
        G.timer_begin()
        for _ in range(10):
            pm.SpMVBackward(G, x, gp)
        t_spmvb = G.timer_end() / 10
        tf, ta = statistics.median(fwd[1:]), statistics.median(adj[1:])
        return {"graph": "directed R-MAT scale 20 (n=%d, m=%d), lognormal weights" % (n, m),
                "forward_ms": round(tf, 3), "forward_iters": it_f, "adjoint_ms": round(ta, 3),
                "adjoint_iters": it_a, "adjoint_over_forward": round(ta / tf, 3),
                "spmv_ms": round(t_spmv, 3), "spmv_backward_ms": round(t_spmvb, 3),
                "spmv_backward_over_forward": round(t_spmvb / t_spmv, 3),
                "tolerance": "relative L1 residual 1e-6, FP64 sums"}


def ncu_traffic():
    """DRAM bytes per PageRank pass from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "pagerank_pull_rmat24.md")
    try:
        for ln in open(path):
            if ln.strip().startswith("traffic_bytes_per_pass:"):
                return float(ln.split(":", 1)[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# CPU side: the reference binaries (oracle/_ref) or the oracle port.
# ---------------------------------------------------------------------------
def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class RefSample:
    """The reference programs (oracle/_ref, built from the unmodified sources,
    all host threads, their own nextTime timers, graph loading excluded) on
    the benchmark's own graphs: the symmetrised R-MAT A and the directed
    R-MAT B, generated by the oracle (bit-identical to the device generator)
    and written as the reference's binary graph files.

    One step is a fixed subset of the suite: one PageRank iteration on B
    (one process runs all iterations after a single load of B, 24 s at scale
    24; the per-iteration time is its timer over the iteration count) and
    one Components run or one BFS, alternating, on A (the BFS source cycles
    through the suite's 16 sources).  BP (5.9 s per iteration at scale 24 on 8
    cores, and no output), SpMV and BellmanFord (their reference inputs are
    weighted text files of 1.3-2.6 GB whose parsing outlasts the rest; the
    reference BellmanFord is also not exact) are left out."""

    def __init__(self, scale_a, scale_b, n_sources=16, b_graph=True):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pm_oracle as O
        self.O = O
        if not O.ref_available():
            raise RuntimeError("reference binaries not built (make -C oracle ref)")
        self.d = O.tempdir()
        ga = O.rmat_graph(scale_a, 16, seed=SEED_GRAPH, symmetric=True)
        self.nA, self.mA = ga.n, ga.m
        self.sources = pick_sources(ga.off, n_sources, SEED_SRC)
        self.bfs_edges = {}
        deg = np.diff(ga.off)
        for s in self.sources:
            self.bfs_edges[s] = int(deg[O.bfs(ga, s)[0] >= 0].sum())
        self.fa = O.write_binary(ga, os.path.join(self.d, "a"))
        del ga
        self.nB = self.mB = None
        if b_graph:
            gb = O.rmat_graph(scale_b, 16, seed=SEED_GRAPH)
            self.nB, self.mB = gb.n, gb.m
            self.fb = O.write_binary(gb, os.path.join(self.d, "b"))
            del gb

    def run(self, warmup, steps, threads):
        """(seconds, edges, per-application [seconds, edges]) of the timed
        steps; warm-up steps run the same programs untimed."""
        O = self.O
        per = {}
        tot_s, tot_e = 0.0, 0

        def add(k, secs, edges):
            nonlocal tot_s, tot_e
            a = per.setdefault(k, [0.0, 0])
            a[0] += secs
            a[1] += edges
            tot_s += secs
            tot_e += edges

        for i in range(warmup + steps):
            if i % 2 == 0:
                _, t = O.ref_components(self.fa, threads=threads, result=False)
                k, e = "cc", self.mA
            else:
                s = self.sources[(i // 2) % len(self.sources)]
                _, _, t = O.ref_bfs(self.fa, s, threads=threads, parents=False)
                k, e = "bfs", self.bfs_edges[s]
            if i >= warmup:
                add(k, t, e)
        if self.mB is not None:
            _, t = O.ref_pagerank(self.fb, warmup + steps, threads=threads, result=False, timeout=3600)
            add("pagerank", t * steps / (warmup + steps), self.mB * steps)
        return tot_s, tot_e, per

    def describe(self, steps):
        parts = ["per step: Components or BFS (alternating; sources cycle through the suite's 16) on "
                 "symmetrised R-MAT A"]
        if self.mB is not None:
            parts.append("one PageRank iteration on directed R-MAT B (one process, %d iterations after one "
                         "load, per-iteration time from its timer)" % steps)
        return "; ".join(parts) + ("; BP, SpMV and BellmanFord not in the sample; the reference binaries "
                                   "with their own timers (graph loading excluded)")


def cpu_baseline(suite):
    """The reference programs on graph A of the timed suite (rank 0 at N=1):
    one Components run and two BFS, their own timers, all host threads."""
    threads = cpu_threads()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pm_oracle as O
    if not O.ref_available():
        raise RuntimeError("reference binaries not built (make -C oracle ref)")
    off, idx = suite.A.csr()
    ga = O.Graph(suite.A.n, off, idx)
    f = O.write_binary(ga, os.path.join(O.tempdir(), "a"))
    deg = np.diff(off)
    per = {}
    _, t = O.ref_components(f, threads=threads, result=False)
    per["cc"] = (t, suite.A.m)
    tb, eb = 0.0, 0
    for s in suite.sources[:2]:
        _, _, t = O.ref_bfs(f, s, threads=threads, parents=False)
        tb += t
        eb += int(deg[O.bfs(ga, s)[0] >= 0].sum())
    per["bfs"] = (tb, eb)
    secs = sum(v[0] for v in per.values())
    edges = sum(v[1] for v in per.values())
    return {"value": round(edges / secs / 1e9, 5), "unit": "GTEPS", "cores": threads, "kind": "reference",
            "sample": "the reference programs (all host threads, their own timers) on graph A of the suite "
                      "(symmetrised R-MAT scale %d): one Components run and BFS from the suite's first two "
                      "sources" % int(np.log2(suite.A.n)),
            "per_algo": {k: round(v[1] / v[0] / 1e9, 5) for k, v in per.items()}}


def run_reference(args):
    """The reference arm: rank 0 alone runs the reference programs on the
    suite's own graphs (RefSample); other ranks exit without work."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    threads = cpu_threads()
    s = RefSample(args.scale_a, args.scale_b, args.sources)
    tot_s, tot_e, per = s.run(args.warmup, args.steps, threads)
    value = tot_e / tot_s / 1e9
    sample = s.describe(args.steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": "GTEPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * tot_s / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64/i32", "data": "synthetic",
        "config": suite_config(args.scale_a, args.scale_b, args.sources, s.nA, s.mA, s.nB, s.mB, world),
        "reference_sample": sample,
        "per_algo": {k: {"gteps": round(v[1] / v[0] / 1e9, 5), "ms_per_step": round(1000 * v[0] / args.steps, 3)}
                     for k, v in per.items()},
        "cpu_baseline": {"value": round(value, 5), "unit": "GTEPS", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 5), "unit": "GTEPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def aggregate_ranks(dist, ms_step, edges, device):
    """Whole-job numbers of a replica run: the slowest rank's step time (max
    over ranks) and the edges every rank counted (sum over ranks)."""
    import torch
    t = torch.tensor([ms_step, float(edges)], dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = t.clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(sm[1])


# ---------------------------------------------------------------------------
def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import polymer_b200 as pm
    suite = Suite(pm, local, args.scale_a, args.scale_b, args.sources, rank)
    if not args.no_tune:
        suite.tune()
    if args.no_cuda_graphs:
        for g in (suite.A, suite.B):
            g.set_tunable("cuda_graphs", 0)
    per = {}
    for _ in range(args.warmup):
        suite.step({})
    # roofline source: per-pass device time of the PageRank pull-reduce
    suite.B.profile(True)
    suite.B.profile_read("pagerank", reset=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = pm.kernel_launches()
    tot_ms, tot_edges = 0.0, 0
    for _ in range(args.steps):
        ms, e = suite.step(per)
        tot_ms += ms
        tot_edges += e
    torch.cuda.synchronize()
    launches = pm.kernel_launches() - launches0
    clk = clocks.stop()
    pr_ms, pr_passes = suite.B.profile_read("pagerank", reset=True)
    suite.B.profile(False)
    if dist:
        dist.barrier()
    ms_step = tot_ms / args.steps
    if dist:
        ms_step, tot_edges_all = aggregate_ranks(dist, ms_step, tot_edges, "cuda")
    else:
        tot_edges_all = float(tot_edges)
    value = tot_edges_all / args.steps / (ms_step / 1e3) / 1e9
    hbm, peak_kind = peaks()
    nB, mB = suite.B.n, suite.B.m
    pass_bytes = 8 * mB + 16 * nB
    pass_ms = pr_ms / max(pr_passes, 1)
    achieved = pass_bytes / (pass_ms / 1e3) / 1e9 if pr_passes else None
    per_algo = {}
    for k, (ms, e, nbytes) in per.items():
        gbs = nbytes / (ms / 1e3) / 1e9
        per_algo[k] = {"gteps": round(e / (ms / 1e3) / 1e9, 3), "ms_per_step": round(ms / args.steps, 3),
                       "hbm_gbs": round(gbs, 1), "hbm_frac": round(gbs / hbm, 4)}
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GTEPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/i32",
        "data": "synthetic",
        "config": suite_config(args.scale_a, args.scale_b, len(suite.sources), suite.A.n, suite.A.m, nB, mB,
                               world),
        "launch": "direct launches (--no-cuda-graphs)" if args.no_cuda_graphs else
                  "CUDA graphs: captured PageRank/SpMV/BP loops, device-driven BFS rounds",
        "per_algo": per_algo,
        "roofline": {
            "kernel": "PageRank pull-reduce pass (k_heavy_reduce + k_pull_reduce<PR_F<float>>)",
            "bound": "hbm", "achieved": round(achieved, 1) if achieved else None,
            "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
            "frac": round(achieved / hbm, 4) if achieved else None,
            "traffic": ncu_traffic(),
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the pass, from the "
                              "committed summary profiles/pagerank_pull_rmat24.md (not measured in this run)",
            "algorithmic_bytes_per_pass": pass_bytes,
            "algorithmic_bytes_rule": "8 m + 16 n: CSC id + gathered contribution per edge; offset, "
                                      "out-degree, rank write, contribution write per vertex",
            "pass_ms": round(pass_ms, 4), "passes": pr_passes,
        },
        "gpu_launches": int(launches),
        "clocks": clk,
        "tuning": suite.tuning or "default tunables (--no-tune)",
    }
    # end to end right after the timed suite: the later phases (CPU sample,
    # batched, adjoint and ingest workloads) leave host and device state that
    # a process serving this suite would not have
    if not args.no_e2e:
        e2e = e2e_run(pm, suite, args.e2e_steps, args.e2e_pipeline_steps, local)
        if dist:  # whole job: every rank's edges over the slowest rank's step
            ms_max, edges_all = aggregate_ranks(dist, 1e3 * e2e["seconds_per_step"], e2e["edges_per_step"], "cuda")
            e2e.update(value=round(edges_all / (ms_max / 1e3) / 1e9, 4), seconds_per_step=round(ms_max / 1e3, 4),
                       edges_per_step=int(edges_all), h2d_bytes_per_step=e2e["h2d_bytes_per_step"] * world,
                       d2h_bytes_per_step=e2e["d2h_bytes_per_step"] * world,
                       ranks="sum over %d ranks of edges and bytes, max over ranks of the step time" % world)
        line["e2e"] = e2e
        pm.release_memory_cache()  # the blocks of its graphs
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(suite)
        except Exception as exc:  # keep the GPU line even if the CPU sample fails
            line["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    line["errors_vs_gpu_fp64"] = errors_block(pm, suite)
    if not args.no_batched:
        line["batched"] = batched_block(pm, suite)
        line["adjoint"] = adjoint_block(pm, torch, suite.dev)
        line["ingest"] = ingest_block(pm)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
