"""Test transport for partitioned runs on ONE GPU: the parts run as threads of one process, each
driving its own solver; an exchange copies the peers' send buffers into the receive buffer
between two barriers.  Only the host synchronises the parts (no kernel waits on another part's),
and every barrier has a timeout, so a failing part ends the run with an error instead of a hang."""
from __future__ import annotations

import threading

import torch

from fooskagpu_b200 import _lib as L

TIMEOUT = 120.0


class ThreadGroup:
    def __init__(self, n_parts: int):
        self.n = n_parts
        self.barrier = threading.Barrier(n_parts, timeout=TIMEOUT)
        self.halos = [None] * n_parts
        self.values = [0.0] * n_parts


class ThreadHalo:
    def __init__(self, group: ThreadGroup, solver, mesh):
        pi = mesh.part_info
        self.g, self.p = group, pi["part"]
        maps = mesh.partition_maps()
        self.send_start = [int(x) for x in maps["send_start"]]
        self.recv_start = [int(x) for x in maps["recv_start"]]
        sb, rb = solver.halo_buffer_bytes()
        self.send = torch.empty(max(sb, 16), dtype=torch.uint8, device="cuda")
        self.recv = torch.empty(max(rb, 16), dtype=torch.uint8, device="cuda")
        group.halos[self.p] = self
        self.exchanges = 0
        solver.set_halo(self._exchange, self._allreduce, self.send.data_ptr(), self.recv.data_ptr())

    def _exchange(self, field: int, rb: int, stream) -> None:
        g = self.g
        g.barrier.wait()             # every part has packed its send buffer (its stream is synchronised)
        for q in range(g.n):
            if q == self.p:
                continue
            peer = g.halos[q]
            r0, r1 = self.recv_start[q] * rb, self.recv_start[q + 1] * rb
            s0, s1 = peer.send_start[self.p] * rb, peer.send_start[self.p + 1] * rb
            assert r1 - r0 == s1 - s0
            if r1 > r0:
                self.recv[r0:r1].copy_(peer.send[s0:s1])
        torch.cuda.synchronize()
        g.barrier.wait()             # no part packs again before every copy out of its buffer is done
        self.exchanges += 1

    def _allreduce(self, op: int, value: float) -> float:
        g = self.g
        g.values[self.p] = value
        g.barrier.wait()
        vals = list(g.values)
        g.barrier.wait()
        return min(vals) if op == L.FG_REDUCE_MIN else sum(vals)


def run_parts(fn, group: ThreadGroup):
    """Run fn(part) in one thread per part; re-raise the first failure (a failing part breaks the
    barrier so that the others stop at their next exchange)."""
    n_parts = group.n
    errors = [None] * n_parts
    out = [None] * n_parts

    def body(p):
        try:
            torch.cuda.set_device(0)
            out[p] = fn(p)
        except BaseException as e:   # noqa: BLE001 - reported to the caller
            errors[p] = e
            group.barrier.abort()

    ts = [threading.Thread(target=body, args=(p,)) for p in range(n_parts)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=4 * TIMEOUT)
    for t in ts:
        if t.is_alive():
            raise RuntimeError("a part did not finish")
    for e in errors:
        if e is not None:
            raise e
    return out
