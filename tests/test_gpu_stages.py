"""Stage-by-stage parity of the device path with the oracle: one RK3 step with a fixed dt
(no relaxation), then with relaxation, then with the adaptive dt — so a divergence is pinned
to the part of the step that causes it."""
import json
import os

import numpy as np
import pytest

from conftest import rate_err, state_err
from gpu_cases import NAMES, case_tol, make
from oracle.oracle_py import Oracle
from fooskagpu_b200.api import Solver

pytestmark = pytest.mark.gpu

REPORT = os.environ.get("FG_PARITY_REPORT")
TOL = {"fp64": 1e-10, "mixed": 2e-6}


def _report(key, val):
    if not REPORT:
        return
    d = json.load(open(REPORT)) if os.path.exists(REPORT) else {}
    d[key] = val
    json.dump(d, open(REPORT, "w"), indent=1)


def _floor(U):
    # variables that are uniform in a case (alpha in the single-phase ones) are compared
    # against a floor of 1e-12 of the largest conserved magnitude instead of their own range
    return 1e-12 * np.abs(U).max()


@pytest.mark.parametrize("mode", ["fixed_dt", "relax", "adaptive"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", NAMES)
def test_one_step(name, prec, mode, meshdir):
    m, c, U = make(name, meshdir, prec)
    c.consCalcFlag = 0
    if mode in ("fixed_dt", "relax"):
        c.adaptDt = 0
        o0 = Oracle(m.view(), c)
        o0.residual(U)
        c.dt = 0.25 * c.cfl * o0.timestep_min()
        o0.close()
    c.relaxFlag = 1 if mode == "fixed_dt" else 0
    o = Oracle(m.view(), c)
    Uo = U.copy()
    o.step(Uo)
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    s.step()
    Ug = s.get_state()
    e = rate_err(Ug - U, Uo - U, U)  # the increments
    e_abs = state_err(Ug, Uo)
    _report(f"one_step/{name}/{prec}/{mode}", dict(incr=e.tolist(), state=e_abs.tolist()))
    tol = case_tol(name, prec, {"state": TOL[prec]})["state"]
    assert e_abs.max() < tol, e_abs
    s.close()
