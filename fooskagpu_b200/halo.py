"""Transport of a partitioned run over ``torch.distributed``: one process per part, one GPU each.

The reference exchanges its halo faces with MPI point-to-point messages every stage
(DP/communicate.cu) and reduces dt / the conservation sums with MPI_Allreduce.  Here each part's
solver packs the primitive records of its own cells that other parts hold as ghosts (once per
stage; each part computes its first-layer ghosts' gradients itself) into a device send buffer;
this class moves, for every neighbouring part q, the slice of records that q needs and receives
q's records into the ghost slice of the receive buffer:

- an NCCL group sends the device buffers directly (peer traffic over NVLink / NVSwitch);
- a gloo group stages them through host memory (CPU tests, or hosts without NCCL).

    mesh = Mesh.load_neu(path).partition(world, rank)
    s = Solver(mesh, case, precision="mixed", device=local_rank)
    halo = TorchHalo(s, mesh)          # after dist.init_process_group
    s.set_state(U_global[mesh.partition_maps()["cell_global"][:mesh.n_owned]])
    s.step()
"""
from __future__ import annotations

import torch
import torch.distributed as dist

from . import _lib as L


class TorchHalo:
    """Registers itself as the transport of `solver` (a solver of the part mesh `mesh`)."""

    def __init__(self, solver, mesh, group=None, device=None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        pi = mesh.part_info
        if pi["nParts"] != self.world or pi["part"] != self.rank:
            raise ValueError(f"part {pi['part']} of {pi['nParts']} does not match rank {self.rank} of {self.world}")
        maps = mesh.partition_maps()
        self.send_start = [int(x) for x in maps["send_start"]]
        self.recv_start = [int(x) for x in maps["recv_start"]]
        self.nccl = dist.get_backend(group) == "nccl"
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = torch.device(device)
        sb, rb = solver.halo_buffer_bytes()
        self.send = torch.empty(max(sb, 16), dtype=torch.uint8, device=self.device)
        self.recv = torch.empty(max(rb, 16), dtype=torch.uint8, device=self.device)
        self.exchanges = 0
        # one collective of the whole group before the first batched point-to-point call: NCCL
        # lets later batches involve only the neighbouring ranks after that (a part need not
        # touch every other part)
        self._allreduce(L.FG_REDUCE_SUM, 0.0)
        solver.set_halo(self._exchange, self._allreduce, self.send.data_ptr(), self.recv.data_ptr())

    def _sync(self):
        if self.device.type == "cuda":
            torch.cuda.synchronize(self.device)

    def _exchange(self, field: int, record_bytes: int, stream) -> None:
        # the solver has finished packing (its stream is synchronised) before calling
        stage = not self.nccl and self.device.type == "cuda"
        send = self.send.cpu() if stage else self.send
        recv = torch.empty_like(self.recv, device="cpu") if stage else self.recv
        ops = []
        for q in range(self.world):
            if q == self.rank:
                continue
            s0, s1 = self.send_start[q] * record_bytes, self.send_start[q + 1] * record_bytes
            r0, r1 = self.recv_start[q] * record_bytes, self.recv_start[q + 1] * record_bytes
            if s1 > s0:
                ops.append(dist.P2POp(dist.isend, send[s0:s1], q, self.group))
            if r1 > r0:
                ops.append(dist.P2POp(dist.irecv, recv[r0:r1], q, self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        if stage:
            n = self.recv_start[-1] * record_bytes
            self.recv[:n].copy_(recv[:n])
        # the receive buffer is complete before the solver's stream reads it
        self._sync()
        self.exchanges += 1

    def _allreduce(self, op: int, value: float) -> float:
        dev = self.device if self.nccl else torch.device("cpu")
        t = torch.tensor([value], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MIN if op == L.FG_REDUCE_MIN else dist.ReduceOp.SUM, group=self.group)
        return float(t.item())
