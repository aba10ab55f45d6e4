"""The pressure datum (fg_case.pressureDatum) on the liquid-jet case at rest (gas with a trace of
liquid at 5 MPa everywhere, meshgen.jet_cylinder reduced):

- the momentum residual of interior cells: the FP32 face momentum flux A p_F n of the reference's
  form rounds the ambient pressure (eps p A per face); with the datum at the ambient pressure the
  residual falls by orders of magnitude in the mixed path, and the FP64 path is unchanged to
  rounding;
- the thermal relaxation after one step: the spurious velocities of that rounding perturb the
  stiff trace liquid's density by about 1e-10, which is 0.05-0.5 Pa of its pressure, above the
  reference Newton's absolute tolerance of 1e-2 Pa; with the datum the mixed path's Newton takes
  the FP64 path's iteration count."""
import numpy as np
import pytest

from fooskagpu_b200 import cases, meshgen
from fooskagpu_b200.api import Mesh, Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def jet():
    nm = meshgen.jet_cylinder(n=32, nz_prism=4, nz_tet=4)
    m = Mesh.build(nm.nodes, nm.elems, nm.bcs)
    cc = m.arrays()["cellCenter"]
    r = np.hypot(cc[:, 0], cc[:, 1])
    inner = (cc[:, 2] > 0.3 * cc[:, 2].max()) & (cc[:, 2] < 0.7 * cc[:, 2].max()) & (r < 0.7 * r.max())
    yield m, cc, inner
    m.close()


def _case(datum):
    c = cases.jet_case()
    c.pressureDatum = datum
    return c


def _momentum_residual(m, c, U, prec, inner):
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    s.compute_rhs()
    R = s.get_rhs()
    s.close()
    return np.abs(R[inner, 3:6]).max()


def test_datum_removes_ambient_pressure_rounding(jet):
    m, cc, inner = jet
    c0, c1 = _case(0.0), _case(5e6)
    U = cases.jet_ic(c0, cc)
    assert inner.sum() > 100
    mixed0 = _momentum_residual(m, c0, U, "mixed", inner)
    mixed1 = _momentum_residual(m, c1, U, "mixed", inner)
    fp0 = _momentum_residual(m, c0, U, "fp64", inner)
    fp1 = _momentum_residual(m, c1, U, "fp64", inner)
    print("momentum residual max (N): mixed", mixed0, "->", mixed1, " fp64", fp0, "->", fp1)
    assert mixed0 > 0 and mixed1 < 1e-3 * mixed0
    # the FP64 path: rounding-level either way, far below the mixed path's reference form
    assert max(fp0, fp1) < 1e-6 * mixed0


def test_datum_keeps_thermal_newton_at_fp64_iterations(jet):
    m, cc, _ = jet
    its = {}
    for prec, datum in (("fp64", 5e6), ("mixed", 5e6), ("mixed", 0.0)):
        c = _case(datum)
        s = Solver(m, c, precision=prec)
        s.set_state(cases.jet_ic(c, cc))
        s.step()
        st = s.relax_stats()
        its[(prec, datum)] = st["nIter"] / max(1, st["nTherm"] + st["nChem"])
        s.close()
    print("Newton iterations per relaxed cell:", its)
    assert its[("mixed", 5e6)] < 1.2 * its[("fp64", 5e6)]
    assert its[("mixed", 0.0)] > its[("mixed", 5e6)]
