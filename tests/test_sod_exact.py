"""Known-answer check: the Sod shock tube against the exact Riemann solution (Toro's exact
solver, restated in oracle/riemann_exact.py).  Pins the exact solver to the published star
state, then runs the FP64 oracle on a small jittered tet tube to t = 0.2 and bounds the L1
density error."""
import numpy as np

from fooskagpu_b200 import cases, meshgen
from fooskagpu_b200.api import Mesh
from oracle import riemann_exact as R
from oracle.oracle_py import Oracle

SLIP = {s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}
SOD = ((1.0, 0.0, 1.0), (0.125, 0.0, 0.1))


def test_exact_solver_star_state():
    # Toro, table 4.3, test 1 (the Sod problem): p* = 0.30313, u* = 0.92745,
    # rho*L = 0.42632, rho*R = 0.26557
    p, u = R.star_state(1.0, 0.0, 1.0, 0.125, 0.0, 0.1)
    assert abs(p - 0.30313) < 5e-6 and abs(u - 0.92745) < 5e-6
    rho, _, _ = R.sample(np.array([0.6, 0.75]), 0.2, 0.5, *SOD)
    assert abs(rho[0] - 0.42632) < 5e-6 and abs(rho[1] - 0.26557) < 5e-6


def sod_l1(U, centres, vol, t):
    rho = U[:, 1] + U[:, 2]
    ex, _, _ = R.sample(centres[:, 0], t, 0.5, *SOD)
    return float(np.sum(np.abs(rho - ex) * vol) / np.sum(vol))


def test_oracle_sod_l1(tmp_path):
    path = str(tmp_path / "sod.neu")
    meshgen.write_neu(path, meshgen.box_tets(60, 2, 2, L=(1.0, 0.04, 0.04), jitter=0.1, side_bc=SLIP))
    m = Mesh.load_neu(path, scale=1.0)
    a = m.arrays()
    c = cases.sod_case()
    c.adaptDt = 0
    c.dt = 0.002
    c.consCalcFlag = 0
    U = cases.sod_ic(c, a["cellCenter"])
    o = Oracle(m.view(), c)
    l1_0 = sod_l1(U, a["cellCenter"], a["volume"], 1e-9)
    for _ in range(100):   # t = 0.2
        o.step(U)
    l1 = sod_l1(U, a["cellCenter"], a["volume"], 0.2)
    assert l1_0 < 1e-3           # the initial state is the exact solution at t = 0+
    assert l1 < 0.02, l1         # coarse MUSCL + HLLC on 16 mm tets


def test_van_albada_limiter_is_less_diffusive(tmp_path):
    """The limiter extension (van Albada-type phi) against the reference's phi = r / 2 on the same
    tube: lower L1 error at t = 0.2."""
    path = str(tmp_path / "sod.neu")
    meshgen.write_neu(path, meshgen.box_tets(60, 2, 2, L=(1.0, 0.04, 0.04), jitter=0.1, side_bc=SLIP))
    m = Mesh.load_neu(path, scale=1.0)
    a = m.arrays()
    l1 = {}
    for lim in (0, 1):
        c = cases.sod_case()
        c.adaptDt = 0
        c.dt = 0.002
        c.consCalcFlag = 0
        c.limiter = lim
        U = cases.sod_ic(c, a["cellCenter"])
        o = Oracle(m.view(), c)
        for _ in range(100):
            o.step(U)
        l1[lim] = sod_l1(U, a["cellCenter"], a["volume"], 0.2)
    assert l1[1] < l1[0], l1
