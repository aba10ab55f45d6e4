"""The torch.distributed transport of a partitioned run (fooskagpu_b200.halo.TorchHalo) with 2, 3
and 4 gloo ranks on the CPU (with 4, some parts have no face in common): every rank packs the records of its send cells, one exchange later each
rank holds exactly its ghosts' records (both record sizes of the mixed and FP64 paths), and the
dt / conservation reductions give the minimum / sum over the ranks.  The solver is replaced by a
stand-in that only owns the buffers (the kernels that pack and unpack them run on the GPU)."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


class _BufferOnlySolver:
    def __init__(self, n_send, n_recv, max_record_bytes):
        self.sizes = (n_send * max_record_bytes, n_recv * max_record_bytes)

    def halo_buffer_bytes(self):
        return self.sizes

    def set_halo(self, exchange, allreduce, send_ptr, recv_ptr):
        self.exchange, self.allreduce = exchange, allreduce


def _records(cells, stride, dtype):
    """A record per cell whose values identify the cell (.neu index) and the slot."""
    return (cells[:, None].astype(np.float64) * 1000.0 + np.arange(stride)[None, :]).astype(dtype)


def _rank(rank, world, port, path, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch
    import torch.distributed as dist
    from fooskagpu_b200 import _lib as L
    from fooskagpu_b200.api import Mesh
    from fooskagpu_b200.halo import TorchHalo

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        part = Mesh.load_neu(path, scale=1.0).partition(world, rank)
        mp_ = part.partition_maps()
        info = part.part_info
        fake = _BufferOnlySolver(info["nSend"], info["nRecv"], 36 * 8)
        halo = TorchHalo(fake, part, device="cpu")
        cg = mp_["cell_global"]
        ok = True
        for field, stride, dtype in ((L.FG_HALO_W, 12, np.float32), (L.FG_HALO_G, 36, np.float32),
                                     (L.FG_HALO_W, 12, np.float64), (L.FG_HALO_G, 36, np.float64)):
            rb = stride * np.dtype(dtype).itemsize
            send = _records(cg[mp_["send_cells"]], stride, dtype).view(np.uint8).ravel()
            halo.send[:send.size] = torch.from_numpy(send)
            halo.recv.fill_(0)
            fake.exchange(field, rb, None)
            got = halo.recv[:info["nRecv"] * rb].numpy().view(dtype).reshape(-1, stride)
            ok &= bool(np.array_equal(got, _records(cg[mp_["recv_cells"]], stride, dtype)))
        lo = fake.allreduce(L.FG_REDUCE_MIN, 1.5 + rank)
        tot = fake.allreduce(L.FG_REDUCE_SUM, 2.0 ** rank)
        q.put((rank, ok, lo, tot, info["nRecv"], halo.exchanges))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 4])
def test_gloo_halo_exchange(world, tmp_path):
    sys.path.insert(0, str(ROOT))
    from fooskagpu_b200 import meshgen
    path = str(tmp_path / "halo.neu")
    # 16 x 4 x 4 cells in 4 parts: parts 0 and 3 (and 1 and 2) share no face
    shape = (8, 4, 3) if world < 4 else (16, 4, 4)
    meshgen.write_neu(path, meshgen.box_tets(*shape, L=tuple(0.1 * k for k in shape), jitter=0.1, shuffle=True,
                                             side_bc={s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + (os.getpid() + 17 * world) % 1000
    ps = [ctx.Process(target=_rank, args=(r, world, port, path, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in ps), [p.exitcode for p in ps]
    res = sorted(q.get(timeout=5) for _ in range(world))
    for rank, ok, lo, tot, n_recv, n_ex in res:
        assert ok, rank
        assert n_recv > 0 and n_ex == 4
        assert lo == 1.5
        assert tot == sum(2.0 ** r for r in range(world))
