"""Partitioned runs (one part per GPU in production) against the whole-mesh run, with the parts
as threads on one GPU exchanging their halo records through device copies (tests/halo_threads.py).
Each part computes its own cells' gradients, the fluxes of every face of its own cells (a face
on a part border is computed by both parts from the same records) and the updates, so the state
after full explicitLoop steps (adaptive dt combined over the parts, relaxation) must equal the
whole-mesh run's bit for bit, in both precisions, for 2 and 3 parts."""
import numpy as np
import pytest

from gpu_cases import TIE_TOL, make
from halo_threads import ThreadGroup, ThreadHalo, run_parts
from fooskagpu_b200.api import Solver

pytestmark = pytest.mark.gpu
STEPS = 5


def _whole(m, c, U, prec):
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    for _ in range(STEPS):
        s.step()
    out = s.get_state(), s.time(), s.cons_calc(1)
    s.close()
    return out


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name,P", [("tet_ref", 2), ("tet_ref", 3), ("hex_periodic_tgv", 2),
                                    ("mixed_ref_rk3", 3), ("tet_ext", 2)])
def test_partitioned_matches_whole_mesh(name, P, prec, meshdir):
    m, c, U = make(name, meshdir, prec)
    Uw, tw, cw = _whole(m, c, U, prec)
    parts = [m.partition(P, p) for p in range(P)]
    group = ThreadGroup(P)
    solvers = [Solver(pm, c, precision=prec) for pm in parts]
    halos = [ThreadHalo(group, s, pm) for s, pm in zip(solvers, parts)]
    own = [pm.partition_maps()["cell_global"][:pm.n_owned] for pm in parts]
    for s, cg in zip(solvers, own):
        s.set_state(U[cg])

    def run(p):
        for _ in range(STEPS):
            solvers[p].step()
        return solvers[p].get_state(), solvers[p].time(), solvers[p].cons_calc(1)

    res = run_parts(run, group)
    for p in range(P):
        Up, tp, cp = res[p]
        assert np.array_equal(Up, Uw[own[p]]), (p, np.abs(Up - Uw[own[p]]).max())
        assert tp == tw
        assert abs(cp - cw) <= 1e-13 * abs(cw)
        assert halos[p].exchanges == c.rkSteps * STEPS   # one exchange per stage
    for s in solvers:
        s.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_partitioned_with_surrogate_matches_whole_mesh(prec, meshdir):
    """The chemical relaxation with the learned surrogate: each part runs the tensor-core
    pre-pass over its own chemical cells; per cell the prediction and the polish are those of
    the whole-mesh run."""
    from fooskagpu_b200 import cases, meshgen
    from fooskagpu_b200.api import Mesh, Surrogate
    path = str(meshdir / "part_sg_box.neu")
    meshgen.write_neu(path, meshgen.box_tets(20, 10, 10, L=(0.02, 0.01, 0.01), jitter=0.1,
                                             side_bc={k: "slip" for k in ("x0", "x1", "y0", "y1", "z0", "z1")}))
    m = Mesh.load_neu(path, scale=1.0)
    c = cases.reference_case()
    c.rkSteps = 3
    c.hllcTieTol = TIE_TOL[prec]
    U = cases.perturbed_two_phase_ic(c, m.arrays()["cellCenter"], seed=8, vel=25.0)
    s = Solver(m, c, precision="fp64")
    s.set_state(U)
    s.relax_log(1_000_000)
    for _ in range(3):
        s.step()
    X, Y = s.relax_log_read(1_000_000)
    s.close()
    g = Surrogate(seed=4)
    g.set_data(X, Y)
    g.train(10, batch=256, lr=2e-3, seed=5)
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    s.set_surrogate(g, 1e-6, 3)
    for _ in range(STEPS):
        s.step()
    Uw = s.get_state()
    sw = s.relax_stats()
    s.close()
    P = 2
    parts = [m.partition(P, p) for p in range(P)]
    group = ThreadGroup(P)
    solvers = [Solver(pm, c, precision=prec) for pm in parts]
    halos = [ThreadHalo(group, sp, pm) for sp, pm in zip(solvers, parts)]
    own = [pm.partition_maps()["cell_global"][:pm.n_owned] for pm in parts]
    for sp, cg in zip(solvers, own):
        sp.set_state(U[cg])
        sp.set_surrogate(g, 1e-6, 3)

    def run(p):
        for _ in range(STEPS):
            solvers[p].step()
        return solvers[p].get_state(), solvers[p].relax_stats()

    res = run_parts(run, group)
    assert sw["nSurrogate"] > 0
    assert sum(r[1]["nSurrogate"] for r in res) == sw["nSurrogate"]
    assert sum(r[1]["nChem"] for r in res) == sw["nChem"]
    for p in range(P):
        assert np.array_equal(res[p][0], Uw[own[p]]), (p, np.abs(res[p][0] - Uw[own[p]]).max())
    for sp in solvers:
        sp.close()
    g.close()


def test_part_solver_needs_a_transport(meshdir):
    from fooskagpu_b200._lib import FgError
    m, c, U = make("tet_ref", meshdir, "fp64")
    pm = m.partition(2, 0)
    s = Solver(pm, c, precision="fp64")
    s.set_state(U[pm.partition_maps()["cell_global"][:pm.n_owned]])
    with pytest.raises(FgError, match="fg_solver_set_halo"):
        s.step()
    s.close()


def test_transport_only_for_parts(meshdir):
    """A solver of a whole mesh has no halo: no buffers, and a transport is refused."""
    from fooskagpu_b200._lib import FgError
    m, c, U = make("tet_ref", meshdir, "fp64")
    s = Solver(m, c, precision="fp64")
    assert s.halo_buffer_bytes() == (0, 0)
    with pytest.raises(FgError, match="not a part"):
        s.set_halo(lambda f, rb, st: None, lambda op, v: v, 0, 0)
    s.close()
