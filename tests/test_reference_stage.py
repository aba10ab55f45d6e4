"""The oracle against the reference CUDA solver itself.

tests/golden/stage_*.npz hold what the reference binary (built from the reference sources by
oracle/build_ref.py, run on a B200 by tests/golden/make_golden.py stage) produced on small
seeded meshes: its mesh arrays, the stage-0 intermediates (primitive face states before and
after limiting, gradients, limiter, neighbour min/max, residual), the adaptive dt and the state
after a few steps.  The oracle runs the same .neu and case here on the CPU.

Tolerances: the reference sums with FP64 atomics in nondeterministic order and its device code
uses FMA contraction, so stage arrays agree to round-off (1e-11 of each variable's range); the
state after several steps includes the relaxation Newton, whose absolute tolerances make the
result sensitive at that level (see test_gpu_parity.test_steps_with_relaxation)."""
import os
from pathlib import Path

import numpy as np
import pytest

from conftest import rate_err, state_err

GOLD = Path(__file__).resolve().parent / "golden"
FIXTURES = sorted(GOLD.glob("stage_*.npz"))


def _spec(name):
    import sys
    sys.path.insert(0, str(GOLD))
    import make_golden
    return make_golden, [s for s in make_golden.stage_specs() if s["name"] == name][0]


@pytest.mark.skipif(not FIXTURES, reason="no reference stage fixtures")
@pytest.mark.parametrize("path", FIXTURES, ids=[p.stem for p in FIXTURES])
def test_oracle_matches_reference_binary(path, tmp_path):
    from fooskagpu_b200 import meshgen
    from fooskagpu_b200.api import Mesh
    from oracle.oracle_py import Oracle
    z = np.load(path)
    name = path.stem[len("stage_"):]
    mg, spec = _spec(name)
    mm, c = mg.build_spec(spec)
    neu = str(tmp_path / "sh.neu")
    meshgen.write_neu(neu, mm)
    m = Mesh.load_neu(neu, scale=c.scale)
    a = m.arrays()
    # mesh pre-processing: same face order, ownership, boundary codes and geometry
    assert np.array_equal(a["fc2el"], z["fc2el"])
    assert np.array_equal(a["boundCond"], z["bc"])
    for k, r in (("n", "n"), ("nt1", "nt1"), ("nt2", "nt2"), ("area", "area"), ("volume", "vol"),
                 ("cellCenter", "cc"), ("fcCenter", "fc")):
        d = np.abs(a[k] - z[r]).max() / np.abs(z[r]).max()
        assert d < 1e-14, (k, d)
    U0 = z["ic"]
    o = Oracle(m.view(), c)
    o.residual(U0)
    # primitive face states before limiting are computed per face without accumulation
    pf0 = o.primF  # after limiting now; recompute the unlimited ones
    from oracle import oracle_py as O
    import ctypes as C
    O.lib().orc_prim(C.byref(c), C.byref(o.view), U0.ctypes.data_as(O.PD), o.w)
    e = state_err(o.primF.reshape(-1, 10)[:, :9], z["primF0"].reshape(-1, 10)[:, :9])
    assert e.max() < 1e-13, e
    R = o.residual(U0)
    # gradients, limiter and residual
    go, gr = o.grad[:, :9].reshape(len(U0), -1), z["grad"][:, :9].reshape(len(U0), -1)
    gfl = 1e-4 * np.abs(gr).max()   # round-off floor: the alpha gradient is pure noise in single-phase cases
    eg = np.abs(go - gr).max(axis=0) / np.maximum(np.abs(gr).max(axis=0), gfl)
    assert eg.max() < 1e-10, eg
    sl_o = (o.theta[:, :9, None] * o.grad[:, :9]).reshape(len(U0), -1)
    sl_r = (z["theta"][:, :9, None] * z["grad"][:, :9]).reshape(len(U0), -1)
    assert np.abs(sl_o - sl_r).max() <= 1e-10 * max(np.abs(sl_r).max(), gfl)
    # energy flux at S* ~ 0: the reference's star energy lacks rho_K, so the flux jumps by
    # 2 |u_n p (1 - 1/rho)| A there and each code's rounding picks the branch.  Away from such
    # faces everything agrees to round-off; at them the difference is bounded by the jump.
    tie_cells, jump = _tie_faces(o, c, m.view(), len(U0))
    er = rate_err(R, z["rhs"], U0, floor=1e-6)
    other = [v for v in range(10) if v != 8]
    assert er[other].max() < 1e-10, er
    ok = ~tie_cells
    d8 = np.abs(R[:, 8] - z["rhs"][:, 8])
    assert d8[ok].max(initial=0) <= 1e-10 * np.abs(z["rhs"][:, 8]).max(), d8[ok].max()
    assert np.all(d8[tie_cells] <= jump[tie_cells] * (1 + 1e-9) + 1e-10 * np.abs(z["rhs"][:, 8]).max())
    if "dt" in z.files:
        dtmin = o.timestep_min()
        dt = min(c.cfl * dtmin, c.maxDt)
        assert abs(dt - float(z["dt"])) <= 1e-12 * float(z["dt"])
    # several full steps (relaxation included)
    U = U0.copy()
    for _ in range(int(z["steps"])):
        o.step(U)
    es = state_err(U, z["U"])
    # Sod: slip walls are exact S* = 0 ties and rho = 0.125 makes the reference's energy jump
    # 2 |u_n p (1 - 1/rho)| large (factor 7), so the reference's own multi-step result moves by
    # a few percent with its rounding; elsewhere the bound is 5e-3
    bound = 0.1 if name == "tet_sod" else 5e-3
    assert es.max() < bound, es


def _tie_faces(o, c, view, nE, tol=1e-9):
    """Cells next to faces with |S*| <= tol (|S_L| + |S_R|) and, per cell, the sum over those
    faces of the energy-flux jump 2 |u_n p (1 - 1/rho)| A of the reference's formula."""
    import ctypes as C
    from oracle import oracle_py as O
    L = O.lib()
    pf = o.primF.copy()
    nF = pf.shape[0]
    fc2el = np.ctypeslib.as_array(view.fc2el, shape=(2 * nF,)).reshape(nF, 2)
    bc = np.ctypeslib.as_array(view.boundCond, shape=(nF,))
    n = np.ctypeslib.as_array(view.n, shape=(3 * nF,)).reshape(nF, 3)
    t1 = np.ctypeslib.as_array(view.nt1, shape=(3 * nF,)).reshape(nF, 3)
    t2 = np.ctypeslib.as_array(view.nt2, shape=(3 * nF,)).reshape(nF, 3)
    area = np.ctypeslib.as_array(view.area, shape=(nF,))
    tie = np.zeros(nE, bool)
    jump = np.zeros(nE)
    P = O.PD
    for f in range(nF):
        sL = pf[f, 0].copy()
        sR = pf[f, 1].copy() if bc[f] == 0 else sL.copy()
        if bc[f] != 0:
            L.orc_bc_values(C.byref(c), n[f].copy().ctypes.data_as(P), t1[f].copy().ctypes.data_as(P),
                            t2[f].copy().ctypes.data_as(P), sR.ctypes.data_as(P), int(bc[f]))
        cs, ul, ur = np.zeros(3), np.zeros(3), np.zeros(3)
        L.orc_wave_speeds(C.byref(c), n[f].copy().ctypes.data_as(P), t1[f].copy().ctypes.data_as(P),
                          t2[f].copy().ctypes.data_as(P), sL.ctypes.data_as(P), sR.ctypes.data_as(P),
                          cs.ctypes.data_as(P), ul.ctypes.data_as(P), ur.ctypes.data_as(P))
        if abs(cs[1]) <= tol * (abs(cs[0]) + abs(cs[2])):
            j = 0.0
            for s_, u_ in ((sL, ul), (sR, ur)):
                p = s_[0] * s_[6] + (1 - s_[0]) * s_[7]
                r = s_[0] * s_[1] + (1 - s_[0]) * s_[2]
                j = max(j, 2 * abs(u_[0] * p * (1 - 1 / r)) * area[f])
            for e in (fc2el[f, 0], fc2el[f, 1] if bc[f] == 0 else -1):
                if e >= 0:
                    tie[e] = True
                    jump[e] += j
    return tie, jump
