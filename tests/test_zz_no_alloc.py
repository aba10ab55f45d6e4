"""The conservation integral through the entry point that allocates no device memory
(fg_cons_integral_noalloc) agrees with the solver's fg_cons_calc.

Two calls in a row on one stream: first a mesh of 287,496 cells (1,123 block partial sums, more
than the final reduction's 1,024 threads), then one of 324 cells (2 block sums), so the second
call runs with the first call's partial sums still in the shared scratch array beyond its own."""
import ctypes as C

import numpy as np
import pytest

from gpu_cases import make
from fooskagpu_b200 import cases, meshgen
from fooskagpu_b200._lib import FgError, check, lib
from fooskagpu_b200.api import Mesh, Solver

pytestmark = pytest.mark.gpu

# relative tolerance of the conservation-integral parity test
TOL = 1e-13


def _big_case(meshdir):
    path = str(meshdir / "noalloc_hex66.neu")
    meshgen.write_neu(path, meshgen.box_hexes(66, 66, 66, L=(0.003, 0.003, 0.003)))
    m = Mesh.load_neu(path, scale=1.0)
    c = cases.reference_case()
    U = cases.perturbed_two_phase_ic(c, m.arrays()["cellCenter"], seed=11, vel=10.0)
    return m, c, U


def _expected(m, c, U, ivar):
    s = Solver(m, c, precision="fp64")
    s.set_state(U)
    v = s.cons_calc(ivar)
    s.close()
    return v


def test_noalloc_matches_cons_calc(meshdir):
    import torch

    dev = torch.device("cuda:0")
    torch.cuda.set_device(0)
    cases_ = [(_big_case(meshdir), 1), (make("tet_ref", meshdir), 0)]
    want, bufs = [], []
    for (m, c, U), ivar in cases_:
        want.append(_expected(m, c, U, ivar))
        Ud = torch.from_numpy(np.ascontiguousarray(U)).to(dev)
        vd = torch.from_numpy(np.ascontiguousarray(m.arrays()["volume"], dtype=np.float64)).to(dev)
        bufs.append((Ud, vd, torch.full((1,), np.nan, dtype=torch.float64, device=dev), len(U), ivar))
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()
    for Ud, vd, out, n, ivar in bufs:
        check(lib().fg_cons_integral_noalloc(C.c_void_p(Ud.data_ptr()), C.c_void_p(vd.data_ptr()), n, ivar,
                                             C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream)))
    torch.cuda.synchronize()
    for (_, _, out, n, ivar), w in zip(bufs, want):
        got = float(out.item())
        assert abs(got - w) <= TOL * abs(w), (n, ivar, got, w)


def test_noalloc_rejects_oversize():
    nmax = 65536 * 256
    p = C.c_void_p(16)   # never dereferenced: the size check comes first
    with pytest.raises(FgError, match="static scratch limit"):
        check(lib().fg_cons_integral_noalloc(p, p, nmax + 1, 0, p, None))
