"""Edge sizes on the device path against the oracle: a mesh of one hex cell whose six faces carry
the six boundary kinds (inlet, outlet, wall, slip, symmetry, slip), and a mesh whose last
gradient block holds a single cell (129 cells: 128 + 1), over three full explicitLoop steps."""
import numpy as np
import pytest

from fooskagpu_b200 import cases, meshgen
from fooskagpu_b200.api import Mesh, Solver
from oracle.oracle_py import Oracle

pytestmark = pytest.mark.gpu
ALL_BC = {"x0": "inlet", "x1": "outlet", "y0": "wall", "y1": "slip", "z0": "symmetry", "z1": "slip"}
TOL = {"fp64": (1e-10, 1e-9), "mixed": (2e-6, 1e-4)}   # state tolerance, HLLC tie tolerance


def _compare(path, prec, steps=3):
    m = Mesh.load_neu(path, scale=1.0)
    c = cases.reference_case()
    c.rkSteps = 3
    tol, tie = TOL[prec]
    c.hllcTieTol = tie
    U = cases.perturbed_two_phase_ic(c, m.arrays()["cellCenter"], seed=9, vel=25.0)
    o = Oracle(m.view(), c)
    Uo = U.copy()
    for _ in range(steps):
        o.step(Uo)
    o.close()
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    for _ in range(steps):
        s.step()
    Ug = s.get_state()
    s.close()
    scale = np.maximum(np.abs(Uo).max(axis=0), 1e-300)
    err = (np.abs(Ug - Uo).max(axis=0) / scale)
    err[scale < 1e-200] = 0.0
    assert err.max() < tol, err


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_single_cell_every_boundary(prec, meshdir):
    path = str(meshdir / "edge_one_cell.neu")
    meshgen.write_neu(path, meshgen.box_hexes(1, 1, 1, L=(0.001, 0.001, 0.001), side_bc=ALL_BC))
    _compare(path, prec)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_last_block_single_cell(prec, meshdir):
    path = str(meshdir / "edge_129.neu")
    # a row of 129 hexes: the gradient blocks hold 128 (FP32) or 64 (FP64) cells, so the last
    # block holds one cell in either precision, and so does the last gather block
    meshgen.write_neu(path, meshgen.box_hexes(129, 1, 1, L=(0.0129, 0.0001, 0.0001),
                                              side_bc={k: "slip" for k in ALL_BC}))
    _compare(path, prec)
