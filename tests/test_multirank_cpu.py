"""The multi-rank path of bench.py on CPU: two `gloo` ranks (world size 2,
127.0.0.1) run the replica aggregation (max of the step times, sum of the
edges), pick their rank-specific sources, and take the reference arm's
rank > 0 exit.  No GPU is used."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import argparse
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms, edges = bench.aggregate_ranks(dist, [3.0, 5.0][rank], [100, 250][rank], "cpu")
        off = np.array([0, 2, 2, 5, 6, 6, 9, 9, 10], np.int32)  # vertices 1, 4, 6 have no out-edges
        srcs = bench.pick_sources(off, 3, bench.SEED_SRC + rank)
        got = [None] * world
        dist.all_gather_object(got, srcs)
        args = argparse.Namespace(steps=1, warmup=0, gpus=world)
        rc = bench.run_reference(args) if rank > 0 else 0
        q.put((rank, ms, edges, got, rc))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, edges, got, rc in res:
        assert ms == 5.0 and edges == 350.0        # slowest rank, all ranks' edges
        assert rc == 0                              # rank 1 of the reference arm exits without work
        assert got[0] != got[1]                     # ranks traverse from different sources
        for srcs in got:
            assert len(set(srcs)) == 3 and all(s not in (1, 4, 6) for s in srcs)
