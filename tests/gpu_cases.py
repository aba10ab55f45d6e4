"""Small meshes and cases shared by the GPU parity tests."""
from __future__ import annotations

import math
import os

import numpy as np

from fooskagpu_b200 import cases, meshgen
from fooskagpu_b200.api import Mesh

ALL_BC = {"x0": "inlet", "x1": "outlet", "y0": "wall", "y1": "slip", "z0": "symmetry", "z1": "slip"}
SLIP = {s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}


# The reference's energy flux is discontinuous at S* = 0 (see fg_case.hllcTieTol); the parity
# tests make both implementations take the same branch at such ties with a tolerance above the
# rounding noise of the precision under test.
TIE_TOL = {"fp64": 1e-9, "mixed": 1e-4}

# Tolerances that differ per case.  Stiffened water (p_inf = 3.43e8 Pa, 34 times the 10 MPa
# operating pressure) forms its pressure as a difference of terms of order gamma p_inf:
#  - FP32 face states leave about 1.3 decimal digits less than with the reference's fluid in a
#    single residual evaluation (mixed path, factor 20 on its residual / gradient tolerances);
#  - the collapsing bubble amplifies any perturbation of the state: in the FP64 oracle itself a
#    relative perturbation of 1e-15 of the initial state changes the state after 3 steps by
#    2e-7 relative, so round-off differences between two correct implementations (FMA
#    contraction, summation order) show up at that level after a few steps.
CASE_TOL = {"ball_bubble": {"fp64": {"state": 2e-6},
                            "mixed": {"rhs": 4e-3, "grad": 6e-3, "theta": 6e-3, "signal": 4e-5, "dt": 4e-5,
                                      "state": 1e-3}}}


def case_tol(name: str, prec: str, base: dict) -> dict:
    """`base` (tolerances by key) with the case's overrides."""
    out = dict(base)
    out.update(CASE_TOL.get(name, {}).get(prec, {}))
    return out


def make(name: str, meshdir, prec: str = "fp64") -> tuple:
    """Return (Mesh, case, U0) for a named parity case."""
    path = os.path.join(str(meshdir), name + ".neu")
    periodic = (0.0, 0.0, 0.0)
    if name == "tet_ext":
        # the extensions the configurations need: van Albada-type limiter, prescribed inlet velocity
        path = os.path.join(str(meshdir), "tet_ref.neu")
        if not os.path.exists(path):
            meshgen.write_neu(path, meshgen.box_tets(6, 3, 3, L=(0.006, 0.003, 0.003), origin=(-0.003, 0, 0),
                                                     jitter=0.1, side_bc=ALL_BC))
        c = cases.reference_case()
        c.limiter = 1
        c.inletVelFlag = 1
        c.inletVel[0], c.inletVel[1], c.inletVel[2] = 30.0, 2.0, -1.0
        c.inletStateFlag = 1
        c.inletP, c.inletT = 9.0e5, 113.0
        ic = "perturbed"
    elif name == "tet_ref":
        if not os.path.exists(path):
            meshgen.write_neu(path, meshgen.box_tets(6, 3, 3, L=(0.006, 0.003, 0.003), origin=(-0.003, 0, 0),
                                                     jitter=0.1, side_bc=ALL_BC))
        c = cases.reference_case()
        ic = "perturbed"
    elif name == "mixed_ref_rk3":
        if not os.path.exists(path):
            meshgen.write_neu(path, meshgen.box_mixed(4, 4, 3, L=(0.004, 0.004, 0.003), side_bc=SLIP))
        c = cases.reference_case()
        c.rkSteps = 3
        ic = "perturbed"
    elif name == "hex_periodic_tgv":
        L = 2 * math.pi
        if not os.path.exists(path):
            meshgen.write_neu(path, meshgen.box_hexes(8, 8, 8, L=(L, L, L), side_bc={}, shuffle=True))
        periodic = (L, L, L)
        c = cases.tgv_case()
        c.adaptDtItr = 2
        ic = "tgv"
    elif name == "tet_sod":
        if not os.path.exists(path):
            meshgen.write_neu(path, meshgen.box_tets(24, 3, 3, L=(1.0, 0.1, 0.1), jitter=0.1, side_bc=SLIP))
        c = cases.sod_case()
        c.adaptDtItr = 2
        ic = "sod"
    elif name == "ball_bubble":
        # reduced water / vapour bubble collapse: the ball generator of the 4 M-tet workload at
        # n = 8, a 2.5 mm bubble (2340 Pa) in 10 MPa water collapsing at 20 m/s, van Albada limiter
        path = os.path.join(str(meshdir), "ball8.neu")
        if not os.path.exists(path):
            meshgen.write_neu(path, meshgen.ball_tets(8))
        c = cases.water_vapour_case()
        ic = "bubble"
    else:
        raise KeyError(name)
    c.hllcTieTol = TIE_TOL[prec]
    m = Mesh.load_neu(path, scale=1.0, periodic=periodic)
    a = m.arrays()
    if ic == "perturbed":
        U = cases.perturbed_two_phase_ic(c, a["cellCenter"], seed=5, vel=25.0)
    elif ic == "bubble":
        U = cases.bubble_ic(c, a["cellCenter"], R0=2.5e-3, width=1e-3, u_wall=-20.0)
    elif ic == "tgv":
        U = cases.tgv_ic(c, a["cellCenter"])
    else:
        U = cases.sod_ic(c, a["cellCenter"])
    return m, c, U


NAMES = ["tet_ref", "mixed_ref_rk3", "hex_periodic_tgv", "tet_sod", "tet_ext", "ball_bubble"]
