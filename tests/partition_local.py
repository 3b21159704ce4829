"""Test harness: the ranks of a partition graph as host threads on one GPU.

Each of P threads creates its rank's handle (Graph.partition) on device 0
and runs the same calls; the exchange function every rank's handle calls
copies the other ranks' ranges out of their buffers on the calling rank's
stream, between two host barriers (every range written before anyone reads;
every read finished before anyone writes again).  No kernel waits for
another rank on the device: only the host threads wait, with a timeout."""
import threading

import torch

from polymer_b200.distributed import device_bytes


class LocalGroup:
    def __init__(self, nranks: int, timeout: float = 120.0):
        self.nranks = nranks
        self.barrier = threading.Barrier(nranks, timeout=timeout)
        self.bufs = [None] * nranks
        self.calls = [0] * nranks

    def exchange(self, rank: int):
        dev = torch.device("cuda", 0)

        def ex(buf, elem_bytes, bounds, stream):
            s = torch.cuda.ExternalStream(stream, device=dev)
            s.synchronize()  # this rank's range is written
            self.bufs[rank] = buf
            self.calls[rank] += 1
            self.barrier.wait()
            total = bounds[-1] * elem_bytes
            mine = device_bytes(buf, total, dev)
            with torch.cuda.stream(s):
                for r in range(self.nranks):
                    a, b = bounds[r] * elem_bytes, bounds[r + 1] * elem_bytes
                    if r != rank and b > a:
                        mine[a:b].copy_(device_bytes(self.bufs[r], total, dev)[a:b])
            s.synchronize()
            self.barrier.wait()

        return ex

    def run(self, body):
        """body(rank, exchange) in one thread per rank; the per-rank results,
        or the first exception raised (the barrier is broken for the rest)."""
        out, errors = [None] * self.nranks, []

        def main(rank):
            try:
                out[rank] = body(rank, self.exchange(rank))
            except BaseException as exc:
                errors.append(exc)
                self.barrier.abort()

        ts = [threading.Thread(target=main, args=(r,)) for r in range(self.nranks)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        if errors:
            raise errors[0]
        return out
