"""The reference's HLLC energy flux is discontinuous at S* = 0 (DP/starRegion.h:29 lacks the rho_K
factor), so where S* vanishes in exact arithmetic (slip and symmetry walls) round-off picks the
branch.  With the reference's default hllcTieTol = 0 the device path and the oracle therefore
differ exactly at those faces: every cell whose FP64 residual differs from the oracle's by more
than round-off touches a face with |S*| <= 1e-9 (|S_L| + |S_R|); everywhere else they agree."""
import ctypes as C

import numpy as np
import pytest

from gpu_cases import make
from oracle import oracle_py as O
from fooskagpu_b200.api import Solver

pytestmark = pytest.mark.gpu


def _pd(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(O.PD)


@pytest.mark.parametrize("name", ["tet_ref", "mixed_ref_rk3"])
def test_default_tie_rule_differs_only_at_vanishing_contact_speed(name, meshdir):
    m, c, U = make(name, meshdir, "fp64")
    c.hllcTieTol = 0.0
    o = O.Oracle(m.view(), c)
    R_o = o.residual(U).copy()
    primF = o.primF.copy()
    a = m.arrays()
    lib = O.lib()
    tie = np.zeros(m.n_fcs, dtype=bool)
    for f in range(m.n_fcs):
        n, t1, t2 = a["n"][f], a["nt1"][f], a["nt2"][f]
        sL = primF[f, 0].copy()
        sR = primF[f, 1].copy()
        bc = int(a["boundCond"][f])
        if bc != 0:
            sR = sL.copy()
            lib.orc_bc_values(C.byref(c), _pd(n), _pd(t1), _pd(t2), sR.ctypes.data_as(O.PD), bc)
        out, uL, uR = np.zeros(3), np.zeros(3), np.zeros(3)
        lib.orc_wave_speeds(C.byref(c), _pd(n), _pd(t1), _pd(t2), _pd(sL), _pd(sR), out.ctypes.data_as(O.PD),
                            uL.ctypes.data_as(O.PD), uR.ctypes.data_as(O.PD))
        tie[f] = abs(out[1]) <= 1e-9 * (abs(out[0]) + abs(out[2]))
    s = Solver(m, c, precision="fp64")
    s.set_state(U)
    s.compute_rhs()
    R_g = s.get_rhs()
    s.close()
    scale = np.maximum(np.abs(R_o).max(axis=0), 1e-6 * np.abs(R_o).max())
    err = (np.abs(R_g - R_o) / scale).max(axis=1)
    differ = np.nonzero(err > 1e-9)[0]
    touches = np.zeros(m.n_elem, dtype=bool)
    fc = a["fc2el"]
    touches[fc[tie, 0]] = True
    inner = tie & (a["boundCond"] == 0)
    touches[fc[inner, 1]] = True
    assert tie.any()
    assert np.all(touches[differ]), differ[~touches[differ]]
