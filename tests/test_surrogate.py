"""Learned equilibrium surrogate on the GPU: its FP32 training gradient against the FP64 oracle
network, its BF16 tensor-core forward against the oracle with BF16 rounding, training on samples
logged from the solver's own chemical Newton solves, and what it gains inside the relaxation
(fewer Newton iterations, same states within the acceptance tolerance, Newton fallback)."""
import json
import os

import numpy as np
import pytest

from fooskagpu_b200 import cases, meshgen
from fooskagpu_b200.api import Mesh, Solver, Surrogate
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu

REPORT = os.environ.get("FG_PARITY_REPORT")
SLIP = {s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}
REL_TOL = 1e-6      # acceptance: relative thermodynamic residual after the polish
POLISH = 3


def _report(key, val):
    if not REPORT:
        return
    d = json.load(open(REPORT)) if os.path.exists(REPORT) else {}
    d[key] = val
    json.dump(d, open(REPORT, "w"), indent=1)


@pytest.fixture(scope="module")
def box(meshdir):
    path = str(meshdir / "sg_box_tets.neu")
    if not os.path.exists(path):
        meshgen.write_neu(path, meshgen.box_tets(20, 10, 10, L=(0.02, 0.01, 0.01), jitter=0.1, side_bc=SLIP))
    m = Mesh.load_neu(path, scale=1.0)
    c = cases.reference_case()
    c.rkSteps = 3
    return m, c, m.arrays()["cellCenter"]


@pytest.fixture(scope="module")
def data(box):
    """Equilibrium samples logged from the FP64 solver's chemical Newton solves (2 runs)."""
    m, c, cc = box
    X, Y = [], []
    for seed in (5, 6):
        s = Solver(m, c, precision="fp64")
        s.set_state(cases.perturbed_two_phase_ic(c, cc, seed=seed, vel=25.0))
        s.relax_log(1_000_000)
        for _ in range(10):
            s.step()
        x, y = s.relax_log_read(1_000_000)
        s.close()
        X.append(x)
        Y.append(y)
    return np.concatenate(X), np.concatenate(Y)


@pytest.fixture(scope="module")
def trained(data):
    X, Y = data
    g = Surrogate(seed=1)
    g.set_data(X, Y)
    loss0 = g.loss_grad(*_standardised(g, X[:4096], Y[:4096]))[0]
    loss = g.train(25, batch=1024, lr=2e-3, seed=2)
    return g, loss0, loss


def _standardised(g, X, Y):
    v = g.norm()
    return (X - v[0:3]) / v[3:6], (Y - v[6:10]) / v[10:14]


def test_relax_log_samples(data):
    X, Y = data
    assert len(X) > 20000
    assert np.all(np.isfinite(X)) and np.all(np.isfinite(Y))
    assert np.all(X[:, 0] > 0) and np.all((X[:, 2] >= 0) & (X[:, 2] <= 1))
    assert np.all(Y[:, 0] > 0) and np.all(Y[:, 1] > 0) and np.all((Y[:, 2] > 0) & (Y[:, 2] < 1))


def test_gradient_matches_oracle(data):
    X, Y = data
    g = Surrogate(seed=7)
    g.set_data(X, Y)
    rng = np.random.default_rng(0)
    Xs = rng.normal(0, 1, (512, 3)).astype(np.float32)
    Ys = rng.normal(0, 1, (512, 4)).astype(np.float32)
    loss, grad = g.loss_grad(Xs, Ys)
    lo, go = M.loss_grad(g.params(), Xs, Ys)
    e = float(np.abs(grad - go).max() / np.abs(go).max())
    _report("surrogate/grad", dict(rel=e, loss=loss, loss_oracle=lo))
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    assert e < 1e-5, e
    g.close()


def test_tensor_core_forward_matches_oracle(trained, data):
    g, _, _ = trained
    X, _ = data
    Xb = X[:4096]
    P, hull = g.predict(Xb)
    v = g.norm()
    Z = (Xb - v[0:3]) / v[3:6]
    ob = M.forward_bf16(g.params(), Z) * v[10:14] + v[6:10]
    of = M.forward(g.params(), Z)[0] * v[10:14] + v[6:10]
    # scale per output: its spread over the batch (p, T are far from zero)
    sc = np.ptp(ob, axis=0)
    e_bf = np.abs(P - ob).max(axis=0) / sc
    e_64 = np.abs(P - of).max(axis=0) / sc
    _report("surrogate/forward", dict(vs_bf16=e_bf.tolist(), vs_fp64=e_64.tolist()))
    assert hull.all()                         # training inputs are inside the training hull
    assert e_bf.max() < 2e-2, e_bf            # BF16 rounding of activations may flip 1 ulp
    assert e_64.max() < 1e-1, e_64


def test_training_reduces_loss(trained):
    g, loss0, loss = trained
    _report("surrogate/train", dict(initial=loss0, final=loss))
    assert loss < 2e-3 * loss0 and loss < 5e-3, (loss0, loss)


def test_relaxation_gain_and_parity(box, trained):
    """A state the network was not trained on: the surrogate solves most chemical cells, with
    far fewer Newton iterations, and the relaxed state matches the Newton-only one within the
    acceptance tolerance."""
    m, c, cc = box
    g = trained[0]
    U = cases.perturbed_two_phase_ic(c, cc, seed=11, vel=25.0)
    s0 = Solver(m, c, precision="fp64")
    s0.set_state(U)
    st0 = s0.relaxation()
    U0 = s0.get_state()
    s1 = Solver(m, c, precision="fp64")
    s1.set_state(U)
    s1.set_surrogate(g, REL_TOL, POLISH)
    st1 = s1.relaxation()
    U1 = s1.get_state()
    d = np.abs(U1 - U0).max(axis=0) / np.maximum(np.abs(U0).max(axis=0), 1e-300)
    _report("surrogate/relax", dict(plain=st0, surrogate=st1, max_rel_diff=d.tolist()))
    assert st1["nChem"] == st0["nChem"] > 1000 and st1["nTherm"] == st0["nTherm"]
    assert st1["nSurrogate"] + st1["nFallback"] == st1["nChem"]
    assert st1["nSurrogate"] > 0.9 * st1["nChem"], st1          # fallback rate below 10 %
    # polish steps of the accepted cells: at least one each, at most the cap
    assert st1["nSurrogate"] <= st1["nPolish"] <= POLISH * st1["nSurrogate"], st1
    assert st1["nIter"] < 0.5 * st0["nIter"], (st0, st1)         # the gain: Newton work halved at least
    assert d.max() < 1e-4, d
    s0.close()
    s1.close()


def test_untrained_network_falls_back_to_newton(box, data):
    """With no polish steps an untrained network's predictions are never within tolerance: every
    chemical cell takes the reference Newton and the state is bitwise the Newton-only one."""
    m, c, cc = box
    X, Y = data
    g = Surrogate(seed=3)
    g.set_data(X, Y)
    U = cases.perturbed_two_phase_ic(c, cc, seed=11, vel=25.0)
    s0 = Solver(m, c, precision="fp64")
    s0.set_state(U)
    st0 = s0.relaxation()
    s1 = Solver(m, c, precision="fp64")
    s1.set_state(U)
    s1.set_surrogate(g, REL_TOL, 0)
    st1 = s1.relaxation()
    assert st1["nSurrogate"] == 0 and st1["nFallback"] == st1["nChem"] == st0["nChem"]
    assert st1["nPolish"] == 0 and st0["nPolish"] == 0
    assert st1["nIter"] == st0["nIter"]
    assert np.array_equal(s1.get_state(), s0.get_state())
    s0.close()
    s1.close()
    g.close()


def test_mixed_surrogate_steps_vs_fp64_newton(box, trained):
    """Mixed precision + surrogate against the FP64 Newton-only path over 30 explicitLoop steps:
    relative L2 error of the mixture density and the liquid pressure."""
    m, c, cc = box
    g = trained[0]
    U = cases.perturbed_two_phase_ic(c, cc, seed=12, vel=25.0)
    c = type(c).from_buffer_copy(c)
    c.hllcTieTol = 1e-4
    out = {}
    for name, prec, use in (("ref", "fp64", False), ("fast", "mixed", True)):
        s = Solver(m, c, precision=prec)
        s.set_state(U)
        if use:
            s.set_surrogate(g, REL_TOL, POLISH)
        for _ in range(30):
            s.step()
        out[name] = s.get_state()
        s.close()
    a, b = out["fast"], out["ref"]
    rho_a, rho_b = a[:, 1] + a[:, 2], b[:, 1] + b[:, 2]
    e_rho = float(np.linalg.norm(rho_a - rho_b) / np.linalg.norm(rho_b))

    def p_liq(U):
        al = np.clip(U[:, 0], c.avfMin / 100, 1 - c.avfMin / 100)
        r = U[:, 1] / al
        e = U[:, 6] / U[:, 1]
        gm = c.gamma[0]
        return (gm - 1) * r * e - gm * c.pInf[0] - (gm - 1) * c.eta[0] * r

    pa, pb = p_liq(a), p_liq(b)
    e_p = float(np.linalg.norm(pa - pb) / np.linalg.norm(pb))
    _report("surrogate/steps", dict(rho_l2=e_rho, p_l2=e_p))
    assert e_rho < 1e-3 and e_p < 1e-3, (e_rho, e_p)


def test_save_and_load(box, trained, data, tmp_path):
    """A trained network saved to .npz and loaded into a new surrogate predicts the same outputs
    bit for bit, and relaxes a state to the same result."""
    m, c, cc = box
    g = trained[0]
    X, _ = data
    path = str(tmp_path / "sg.npz")
    g.save(path)
    h = Surrogate.load(path)
    P0, h0 = g.predict(X[:2048])
    P1, h1 = h.predict(X[:2048])
    assert np.array_equal(P0, P1) and np.array_equal(h0, h1)
    U = cases.perturbed_two_phase_ic(c, cc, seed=13, vel=25.0)
    out = []
    for sg in (g, h):
        s = Solver(m, c, precision="fp64")
        s.set_state(U)
        s.set_surrogate(sg, REL_TOL, POLISH)
        s.relaxation()
        out.append(s.get_state())
        s.close()
    assert np.array_equal(out[0], out[1])
    h.close()


def test_polish_pass_forms_agree_bitwise(box, trained):
    """The surrogate's polish inside the relaxation kernel, as a pass of its own before it, and the
    automatic choice between the two give bitwise the same states and relaxation counters, in FP64
    and mixed precision, for one relaxation and over steps."""
    from fooskagpu_b200._lib import lib
    m, c, cc = box
    g = trained[0]
    U = cases.perturbed_two_phase_ic(c, cc, seed=14, vel=25.0)
    for prec in ("fp64", "mixed"):
        out = {}
        for mode in ("fused", "separate", "auto"):
            s = Solver(m, c, precision=prec)
            s.set_state(U)
            s.set_surrogate(g, REL_TOL, POLISH)
            s.set_surrogate_pass(mode)
            st = [s.relaxation()]
            for _ in range(4):
                s.step()
                st.append(s.relax_stats())
            out[mode] = (s.get_state(), st)
            if mode == "auto":
                with pytest.raises(ValueError):
                    s.set_surrogate_pass("inline")
                assert lib().fg_solver_set_surrogate_pass(s._h, 3) != 0
            s.close()
        U0, st0 = out["fused"]
        assert st0[0]["nSurrogate"] > 0.9 * st0[0]["nChem"] > 0, st0[0]
        for mode in ("separate", "auto"):
            assert out[mode][1] == st0, (prec, mode)
            assert np.array_equal(out[mode][0], U0), (prec, mode)
