"""A partitioned run as it runs in production: one process per part, the parts' halo records
moved by fooskagpu_b200.halo.TorchHalo over torch.distributed (gloo here, host-staged; NCCL moves
the device buffers directly).  Both processes drive the real solver on cuda:0 (this machine has
one GPU): no kernel waits on another process, the host exchanges the records between the pack
and the unpack kernels, and the process group has a short timeout.  After full explicitLoop steps
(adaptive dt combined over the parts, relaxation) each part's state equals the whole-mesh run's
for its cells bit for bit, in both precisions."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent
STEPS = 4


def _part(rank, world, port, meshdir, name, prec, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    import datetime

    import torch
    import torch.distributed as dist
    from gpu_cases import make
    from fooskagpu_b200.api import Solver
    from fooskagpu_b200.halo import TorchHalo

    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        m, c, U = make(name, meshdir, prec)
        pm = m.partition(world, rank)
        s = Solver(pm, c, precision=prec, device=0)
        halo = TorchHalo(s, pm, device="cuda:0")
        cg = pm.partition_maps()["cell_global"][:pm.n_owned]
        s.set_state(U[cg])
        for _ in range(STEPS):
            s.step()
        np.savez(os.path.join(out, f"part{rank}.npz"), U=s.get_state(), cells=cg, t=s.time()[1],
                 exchanges=halo.exchanges)
        s.close()
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["tet_ref", "hex_periodic_tgv"])
def test_two_processes_match_whole_mesh(name, prec, meshdir, tmp_path):
    sys.path.insert(0, str(ROOT / "tests"))
    from gpu_cases import make
    from fooskagpu_b200.api import Solver
    m, c, U = make(name, meshdir, prec)
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    for _ in range(STEPS):
        s.step()
    Uw, tw = s.get_state(), s.time()[1]
    s.close()
    port = 29500 + (os.getpid() % 1000)
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_part, args=(r, 2, port, str(meshdir), name, prec, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0
    for r in range(2):
        d = np.load(tmp_path / f"part{r}.npz")
        assert np.array_equal(d["U"], Uw[d["cells"]]), (r, np.abs(d["U"] - Uw[d["cells"]]).max())
        assert float(d["t"]) == tw
        assert int(d["exchanges"]) == c.rkSteps * STEPS   # one exchange per stage
