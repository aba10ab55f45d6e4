"""Known-answer and statistics checks on the GPU path: the Sod shock tube against the exact
Riemann solution (FP64 and mixed precision), and the Taylor-Green kinetic-energy history of the
mixed path against the FP64 path (periodic hex cube, WALE) over its first 30 steps.  (Later the
two histories part: the thermal relaxation's 1e-2 absolute Newton tolerance turns rounding
differences into different iteration counts, and the scheme of the reference, which this path
reproduces, dissipates this coarse TGV strongly — its own CUDA build shows the same decay.)"""
import json
import math
import os

import numpy as np
import pytest

from fooskagpu_b200 import cases, meshgen
from fooskagpu_b200.api import Mesh, Solver
from oracle import riemann_exact as R

pytestmark = pytest.mark.gpu

REPORT = os.environ.get("FG_PARITY_REPORT")
SLIP = {s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}
SOD = ((1.0, 0.0, 1.0), (0.125, 0.0, 0.1))


def _report(key, val):
    if not REPORT:
        return
    d = json.load(open(REPORT)) if os.path.exists(REPORT) else {}
    d[key] = val
    json.dump(d, open(REPORT, "w"), indent=1)


def test_sod_exact_l1(meshdir):
    path = str(meshdir / "sod200.neu")
    if not os.path.exists(path):
        meshgen.write_neu(path, meshgen.box_tets(200, 4, 4, L=(1.0, 0.02, 0.02), jitter=0.1, side_bc=SLIP))
    m = Mesh.load_neu(path, scale=1.0)
    a = m.arrays()
    c = cases.sod_case()
    c.adaptDtItr = 1       # CFL 0.5 time step every step
    c.hllcTieTol = 1e-4
    # With the reference's HLLC energy star state (no rho_K factor) and the thermal relaxation,
    # the density undershoots below the right state on this mesh (the FP64 oracle shows it too);
    # the known-answer check runs the corrected star state.
    c.hllcEnergyFix = 1
    U0 = cases.sod_ic(c, a["cellCenter"])
    res = {}
    for prec in ("fp64", "mixed"):
        s = Solver(m, c, precision=prec)
        s.set_state(U0)
        t = 0.0
        for _ in range(5000):
            s.step()
            t += s.time()[0]   # the dt this step used (updated at its first stage)
            if t >= 0.2:
                break
        U = s.get_state()
        s.close()
        rho = U[:, 1] + U[:, 2]
        ex, _, _ = R.sample(a["cellCenter"][:, 0], t, 0.5, *SOD)
        res[prec] = float(np.sum(np.abs(rho - ex) * a["volume"]) / np.sum(a["volume"]))
        res[prec + "_rho"] = rho
        res[prec + "_t"] = t
    _report("physics/sod_l1", {"fp64": res["fp64"], "mixed": res["mixed"], "t": res["fp64_t"]})
    assert abs(res["fp64_t"] - res["mixed_t"]) < 1e-6 and 0.2 <= res["fp64_t"] < 0.21
    assert res["fp64"] < 8e-3 and res["mixed"] < 8e-3, res
    assert abs(res["fp64"] - res["mixed"]) < 1e-4
    assert np.abs(res["fp64_rho"] - res["mixed_rho"]).max() < 1e-3


def test_tgv_kinetic_energy_history(meshdir):
    L = 2 * math.pi
    path = str(meshdir / "tgv32.neu")
    if not os.path.exists(path):
        meshgen.write_neu(path, meshgen.box_hexes(32, 32, 32, L=(L, L, L), side_bc={}, shuffle=True))
    m = Mesh.load_neu(path, scale=1.0, periodic=(L, L, L))
    a = m.arrays()
    vol = a["volume"]
    c = cases.tgv_case()
    U0 = cases.tgv_ic(c, a["cellCenter"])

    def ke(U):
        rho = U[:, 1] + U[:, 2]
        return float(np.sum(0.5 * (U[:, 3] ** 2 + U[:, 4] ** 2 + U[:, 5] ** 2) / rho * vol) / np.sum(vol))

    hist = {}
    for prec in ("fp64", "mixed"):
        s = Solver(m, c, precision=prec)
        s.set_state(U0)
        h = [ke(U0)]
        for _ in range(6):
            for _ in range(5):
                s.step()
            h.append(ke(s.get_state()))
        hist[prec] = np.array(h)
        s.close()
    k64, k32 = hist["fp64"], hist["mixed"]
    diss64, diss32 = -np.diff(k64), -np.diff(k32)
    e_ke = float(np.abs(k32 - k64).max() / k64[0])
    e_diss = float(np.abs(diss32 - diss64).max() / np.abs(diss64).max())
    _report("physics/tgv_ke", {"ke_fp64": k64.tolist(), "ke_mixed": k32.tolist(), "max_rel_ke": e_ke,
                               "max_rel_dissipation": e_diss})
    assert np.all(diss64 > 0)            # the vortex decays
    assert e_ke < 1e-5, e_ke
    assert e_diss < 5e-3, e_diss          # per 5-step interval: a difference of small differences
