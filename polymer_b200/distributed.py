"""Exchange functions for partition graphs (Graph.partition) over
torch.distributed.

A partition graph calls its exchange function after every pass with a vertex
array whose range [bounds[r], bounds[r+1]) rank r has just written; on
return (in the order of the library's CUDA stream) every rank's copy must
hold every rank's range: an allgather with unequal counts.  allgather_v()
builds one from torch.distributed's all_gather_into_tensor (NCCL for CUDA
tensors, gloo for host buffers) over equal-width padded slots."""
from __future__ import annotations

import contextlib
import ctypes as C


class _DeviceBytes:
    """A CUDA buffer described by the array interface torch understands."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_bytes(ptr: int, nbytes: int, device):
    """uint8 torch view of nbytes of device memory at ptr (no copy)."""
    import torch
    if nbytes == 0:
        return torch.empty(0, dtype=torch.uint8, device=device)
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device=device)


def host_bytes(ptr: int, nbytes: int):
    """uint8 torch view of nbytes of host memory at ptr (no copy)."""
    import torch
    if nbytes == 0:
        return torch.empty(0, dtype=torch.uint8)
    return torch.frombuffer((C.c_uint8 * nbytes).from_address(ptr), dtype=torch.uint8)


def partition_bounds(offsets, edges, nranks: int, row_work: int = 4):
    """The vertex ranges pm_graph_create_partition cuts for nranks ranks,
    computed on the host from the whole CSR: bound r (0 < r < nranks) is the
    first vertex v whose prefix of in-edges plus row_work * v reaches r /
    nranks of the total (in-edges + row_work * n), rounded down to a multiple
    of 32; bounds[0] = 0, bounds[nranks] = n.  row_work: the library's
    per-row work unit (polymer_b200.ROW_WORK)."""
    import numpy as np
    n = len(offsets) - 1
    indeg = np.bincount(np.asarray(edges, np.int64), minlength=n).astype(np.int64)
    key = (np.concatenate([[0], np.cumsum(indeg)]) + row_work * np.arange(n + 1)).astype(np.float64)
    total = key[-1]
    b = [0]
    for r in range(1, nranks):
        v = int(np.searchsorted(key, total * r / nranks, side="left"))
        b.append(max(v & ~31, b[-1]))
    b.append(n)
    return np.array(b, np.int64)


def allgather_v(group=None, device=None):
    """Exchange function for Graph.partition over a torch.distributed group.

    device: the CUDA device of the partition graph (torch.device or index);
    "cpu" treats buf as host memory (used by the gloo tests of the exchange
    itself).  Each rank copies its range into a slot of the widest range's
    size, all_gather_into_tensor fills every rank's slots, and the other
    ranks' ranges are copied back into place -- all on the library's stream,
    so the next pass sees them without a host synchronisation."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    on_host = device is not None and torch.device(device).type == "cpu"
    dev = torch.device("cpu") if on_host else torch.device("cuda", torch.device(device).index
                                                           if device is not None else torch.cuda.current_device())

    def exchange(buf: int, elem_bytes: int, bounds, stream) -> None:
        if len(bounds) != world + 1:
            raise ValueError("partition has %d ranks, the process group %d" % (len(bounds) - 1, world))
        lens = [(bounds[r + 1] - bounds[r]) * elem_bytes for r in range(world)]
        width = max(max(lens), 1)
        total = bounds[-1] * elem_bytes
        if on_host:
            whole = host_bytes(buf, total)
            ctx = contextlib.nullcontext()
        else:
            whole = device_bytes(buf, total, dev)
            ctx = torch.cuda.stream(torch.cuda.ExternalStream(stream, device=dev))
        with ctx:
            mine = torch.zeros(width, dtype=torch.uint8, device=dev)
            a = bounds[rank] * elem_bytes
            mine[: lens[rank]].copy_(whole[a: a + lens[rank]])
            slots = torch.empty(world * width, dtype=torch.uint8, device=dev)
            dist.all_gather_into_tensor(slots, mine, group=group)
            for r in range(world):
                if r != rank and lens[r]:
                    b = bounds[r] * elem_bytes
                    whole[b: b + lens[r]].copy_(slots[r * width: r * width + lens[r]])

    return exchange
