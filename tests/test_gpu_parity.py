"""Parity of the device path (through the C ABI) with the CPU oracle.

Tolerances (per variable, max |gpu - oracle| / max |oracle|):
  FP64 path   : 1e-9 for residuals / gradients, 1e-10 for states after a few steps — the only
                differences are summation order (cell gathers vs face-order scatter), FMA
                contraction and the algebraic identities that replace the tangent frame.
  mixed path  : FP32 reconstruction / HLLC / viscous flux: 2e-4 for residuals, 3e-4 for
                limited gradients, 2e-6 for states after a few steps (FP64 update).
"""
import json
import os

import numpy as np
import pytest

from conftest import rate_err, rel_err, state_err
from gpu_cases import NAMES, case_tol, make
from oracle.oracle_py import Oracle
from fooskagpu_b200.api import Solver

pytestmark = pytest.mark.gpu

TOL = {
    "fp64": {"rhs": 1e-9, "grad": 1e-9, "theta": 1e-9, "signal": 1e-12, "dt": 1e-12, "state": 1e-10, "relax": 1e-11},
    "mixed": {"rhs": 2e-4, "grad": 3e-4, "theta": 3e-4, "signal": 2e-6, "dt": 2e-6, "state": 2e-6, "relax": 1e-11},
}
# floors relative to the case's overall scale for round-off-only quantities (e.g. the residual
# and gradient of the uniform volume fraction in the single-phase cases)
FLOOR = {"fp64": 1e-6, "mixed": 1e-3}
REPORT = os.environ.get("FG_PARITY_REPORT")


def _tol(name, prec):
    return case_tol(name, prec, TOL[prec])


def _report(key, val):
    if not REPORT:
        return
    d = {}
    if os.path.exists(REPORT):
        d = json.load(open(REPORT))
    d[key] = val
    json.dump(d, open(REPORT, "w"), indent=1)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", NAMES)
def test_residual(name, prec, meshdir):
    m, c, U = make(name, meshdir, prec)
    o = Oracle(m.view(), c)
    R_o = o.residual(U)
    smin_o = o.timestep_min()
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    s.compute_rhs(want_signal=True)
    R_g = s.get_rhs()
    g_g, th_g = s.get_limited()
    sig_g = s.get_signal()
    dt_g = s.compute_time_step()
    dt_o = min(c.cfl * smin_o, c.maxDt)
    # uniform variables (alpha in the single-phase cases) have residuals / gradients that are
    # pure round-off on both sides: normalise by a floor tied to the largest magnitude
    # below these floors a variable's value is round-off of the precision under test
    e_rhs = rate_err(R_g, R_o, U, floor=FLOOR[prec])
    gfl = FLOOR[prec] * np.abs(o.grad[:, :9]).max()
    e_grad = rel_err(g_g[:, :9].reshape(len(U), -1), o.grad[:, :9].reshape(len(U), -1), floor=gfl)
    # theta of a variable with round-off-only gradient is arbitrary in both codes (0 or 1);
    # compare the limited slopes theta * grad, which is what reconstruction uses
    sl_g = th_g[:, :9, None] * g_g[:, :9]
    sl_o = o.theta[:, :9, None] * o.grad[:, :9]
    e_th = float(rel_err(sl_g.reshape(len(U), -1), sl_o.reshape(len(U), -1), floor=gfl).max())
    e_sig = rel_err(sig_g, o.signal)
    e_dt = abs(dt_g - dt_o) / dt_o
    _report(f"residual/{name}/{prec}", dict(rhs=e_rhs.tolist(), grad=float(e_grad.max()), theta=float(e_th),
                                            signal=float(e_sig), dt=e_dt))
    t = _tol(name, prec)
    assert e_rhs.max() < t["rhs"], e_rhs
    assert e_grad.max() < t["grad"], e_grad
    assert e_th < t["theta"], e_th
    assert e_sig < t["signal"]
    assert e_dt < t["dt"]
    s.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", NAMES)
def test_steps(name, prec, meshdir):
    """Three explicitLoop steps (RK stages, adaptive dt, conservation) without relaxation:
    strict parity."""
    m, c, U = make(name, meshdir, prec)
    c.relaxFlag = 1
    o = Oracle(m.view(), c)
    Uo = U.copy()
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    nsteps = 3
    for _ in range(nsteps):
        o.step(Uo)
        s.step()
    Ug = s.get_state()
    dt_g, t_g, it_g = s.time()
    e = state_err(Ug, Uo)
    _report(f"steps/{name}/{prec}", dict(state=e.tolist(), dt=abs(dt_g - o.dt.value) / o.dt.value))
    assert it_g == nsteps
    t = _tol(name, prec)
    assert abs(dt_g - o.dt.value) <= t["dt"] * o.dt.value
    assert abs(t_g - o.time.value) <= t["dt"] * max(o.time.value, 1e-300) * nsteps
    assert e.max() < t["state"], e
    s.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", NAMES)
def test_steps_with_relaxation(name, prec, meshdir):
    """Three full explicitLoop steps including the relaxation.  The reference's thermal Newton
    stops at |p_L - p_G| < 1e-2 Pa and |T_L - T_G| < 1e-2 K (absolute), so an input difference
    at round-off level can change a cell's iteration count and move its phasic energies by up to
    ~ Cv * 1e-2 K; the bound is therefore 4e-2 / T_min relative (T_min the coldest phase)."""
    m, c, U = make(name, meshdir, prec)
    o = Oracle(m.view(), c)
    Uo = U.copy()
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    for _ in range(3):
        o.step(Uo)
        s.step()
    Ug = s.get_state()
    a = np.clip(Uo[:, 0], c.avfMin / 100, 1 - c.avfMin / 100)
    eL = Uo[:, 6] / Uo[:, 1]
    rhoL = Uo[:, 1] / a
    pL = (c.gamma[0] - 1) * rhoL * eL - c.gamma[0] * c.pInf[0] - (c.gamma[0] - 1) * c.eta[0] * rhoL
    TL = (pL + c.pInf[0]) / ((c.Cp[0] / c.gamma[0]) * (c.gamma[0] - 1) * rhoL)
    bound = max(4e-2 / max(TL.min(), 1e-300), _tol(name, prec)["state"])
    e = state_err(Ug, Uo)
    _report(f"steps_relax/{name}/{prec}", dict(state=e.tolist(), bound=bound))
    assert e.max() < bound, (e, bound)
    s.close()


@pytest.mark.parametrize("name", ["tet_ref", "mixed_ref_rk3"])
def test_relaxation(name, meshdir):
    m, c, U = make(name, meshdir)
    o = Oracle(m.view(), c)
    Uo = U.copy()
    st_o = o.relaxation(Uo)
    s = Solver(m, c, precision="fp64")
    s.set_state(U)
    st_g = s.relaxation()
    Ug = s.get_state()
    e = rel_err(Ug, Uo)
    _report(f"relax/{name}", dict(state=e.tolist(), oracle=st_o, gpu=st_g))
    assert st_g["nChem"] == st_o["nChem"] and st_g["nTherm"] == st_o["nTherm"]
    # the same Newton iteration counts and aborts cell for cell, summed
    assert st_g["nIter"] == st_o["nIter"] and st_g["nAbort"] == st_o["nAbort"], (st_g, st_o)
    assert st_o["nChem"] > 0, "fixture should exercise the chemical branch"
    assert e.max() < TOL["fp64"]["relax"], e
    s.close()


@pytest.mark.parametrize("cap", [1, 3])
def test_relaxation_iteration_caps(cap, meshdir):
    """Newton solves that hit their iteration caps (thermItrMax, chemItrMax) fall back to their
    best iterate, as the reference's do: the aborts, the iteration counts and the states agree
    with the oracle cell for cell."""
    m, c, U = make("mixed_ref_rk3", meshdir)
    c.thermItrMax = cap
    c.chemItrMax = cap
    o = Oracle(m.view(), c)
    Uo = U.copy()
    st_o = o.relaxation(Uo)
    s = Solver(m, c, precision="fp64")
    s.set_state(U)
    st_g = s.relaxation()
    Ug = s.get_state()
    e = rel_err(Ug, Uo)
    _report(f"relax_caps/{cap}", dict(state=e.tolist(), oracle=st_o, gpu=st_g))
    assert st_o["nAbort"] > 0, st_o
    assert st_g["nAbort"] == st_o["nAbort"] and st_g["nIter"] == st_o["nIter"], (st_g, st_o)
    # an unconverged Newton iterate is more sensitive to the rounding of its inputs than the
    # converged state: the FP64 state tolerance (measured 2.2e-11 with a cap of 1)
    assert e.max() < TOL["fp64"]["state"], e
    s.check_state()
    s.close()


@pytest.mark.parametrize("name", NAMES)
def test_cons_calc(name, meshdir):
    m, c, U = make(name, meshdir)
    o = Oracle(m.view(), c)
    s = Solver(m, c, precision="fp64")
    s.set_state(U)
    for iv in (0, 1, 8, 9):
        a, b = s.cons_calc(iv), o.cons_calc(iv, U)
        assert abs(a - b) <= 1e-13 * max(abs(b), 1e-300), (iv, a, b)
    s.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_deterministic(prec, meshdir):
    """No atomics on the data path: two runs give bitwise identical states."""
    m, c, U = make("tet_ref", meshdir)
    out = []
    for _ in range(2):
        s = Solver(m, c, precision=prec)
        s.set_state(U)
        for _ in range(3):
            s.step()
        out.append(s.get_state())
        s.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_periodic_conservation(prec, meshdir):
    """Periodic TGV: partial masses, total energy and vapour mass are conserved to round-off
    (both cells of a face evaluate its flux identically, so contributions cancel exactly)."""
    m, c, U = make("hex_periodic_tgv", meshdir)
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    before = [s.cons_calc(iv) for iv in (1, 2, 8)]
    for _ in range(5):
        s.step()
    after = [s.cons_calc(iv) for iv in (1, 2, 8)]
    for b, a in zip(before, after):
        assert abs(a - b) <= 1e-12 * abs(b), (a, b)
    s.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["mixed_ref_rk3", "tet_ext", "hex_periodic_tgv"])
def test_dt_step_matches_stage_api(name, prec, meshdir):
    """A step that computes a new dt (fg_step: the face kernel keeps each cell's maximum face
    signal speed, then the fused gather + RK update) equals fg_init_rk + fg_compute_rhs with the
    signal + fg_compute_time_step + fg_update for its first stage and fg_stage for the others,
    bit for bit: dt, per-cell signal and state."""
    m, c, U = make(name, meshdir, prec)
    c.adaptDt = 1
    c.adaptDtItr = 1
    c.relaxFlag = 1
    c.consCalcFlag = 0
    a = Solver(m, c, precision=prec)
    b = Solver(m, c, precision=prec)
    a.set_state(U)
    b.set_state(U)
    for _ in range(2):
        a.step()
        b.init_rk()
        b.compute_rhs(want_signal=True)
        dt = b.compute_time_step()
        b.update(0)
        for irk in range(1, c.rkSteps):
            b.stage(irk)
        assert a.time()[0] == dt
        assert np.array_equal(a.get_signal(), b.get_signal())
        assert np.array_equal(a.get_state(), b.get_state())
    a.close()
    b.close()


def test_stage_api_matches_step(meshdir):
    """fg_init_rk + fg_compute_rhs + fg_update per stage equals the fused fg_stage path."""
    m, c, U = make("mixed_ref_rk3", meshdir)
    c.adaptDt = 0
    c.dt = 1e-9
    c.relaxFlag = 1
    c.consCalcFlag = 0
    a = Solver(m, c, precision="fp64")
    b = Solver(m, c, precision="fp64")
    a.set_state(U)
    b.set_state(U)
    b.init_rk()
    for irk in range(3):
        a.stage(irk)
        b.compute_rhs()
        b.update(irk)
    Ua, Ub = a.get_state(), b.get_state()
    assert np.array_equal(Ua, Ub)
    a.close()
    b.close()
