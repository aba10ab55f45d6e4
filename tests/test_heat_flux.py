"""Heat-conduction extension (fg_case.heatFlux) in the FP64 oracle: for a quadratic temperature
profile at rest and uniform pressure, the energy residual of interior cells is div(k grad T) V
= 2 a k V; with heatFlux = 0 it vanishes."""
import numpy as np

from fooskagpu_b200 import cases, meshgen
from fooskagpu_b200.api import Mesh
from oracle.oracle_py import Oracle

SLIP = {s: "slip" for s in ("x0", "x1", "y0", "y1", "z0", "z1")}


def test_quadratic_temperature_conduction(tmp_path):
    path = str(tmp_path / "box.neu")
    meshgen.write_neu(path, meshgen.box_hexes(24, 3, 3, L=(1.0, 0.125, 0.125), side_bc=SLIP))
    m = Mesh.load_neu(path, scale=1.0)
    a = m.arrays()
    x = a["cellCenter"][:, 0]
    c = cases.ideal_gas_case(mu=0.05)
    c.heatFlux = 1
    c.Pr[0] = c.Pr[1] = 0.7
    c.turbulence = 0
    p = 1.0
    aq = 0.4
    T = 1.0 + aq * x * x
    rho = p / ((c.Cp[0] / c.gamma[0]) * (c.gamma[0] - 1) * T)
    z = np.zeros_like(x)
    U = cases.prim_to_cons(c, 0.5, rho, rho, z, z, z, p)
    o = Oracle(m.view(), c)
    R = o.residual(U)
    k = c.Cp[0] * c.dynVisc[0] / c.Pr[0]
    inner = (x > 0.1) & (x < 0.9)
    want = 2 * aq * k * a["volume"][inner]
    got = R[inner, 8]
    assert np.allclose(got, want, rtol=0.05), (got[:4], want[:4])
    c.heatFlux = 0
    R0 = Oracle(m.view(), c).residual(U)
    assert np.abs(R0[:, 8]).max() < 1e-12 * np.abs(got).max() + 1e-15
