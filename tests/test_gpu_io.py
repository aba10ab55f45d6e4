"""Checkpoint / restart and the binary field dump on the GPU path."""
import numpy as np
import pytest

from gpu_cases import make
from fooskagpu_b200.api import Solver, read_field_dump

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_restart_is_bitwise(prec, meshdir, tmp_path):
    """3 steps + checkpoint + restart in a new solver + 2 steps == 5 uninterrupted steps."""
    m, c, U = make("tet_ref", meshdir, prec)
    c.adaptDtItr = 2          # a dt update falls after the restart
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    for _ in range(5):
        s.step()
    U5, t5 = s.get_state(), s.time()
    s.close()
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    for _ in range(3):
        s.step()
    ck = tmp_path / "ck.bin"
    s.checkpoint_write(str(ck))
    s.close()
    r = Solver(m, c, precision=prec)
    r.checkpoint_read(str(ck))
    assert r.time()[2] == 3
    for _ in range(2):
        r.step()
    assert np.array_equal(r.get_state(), U5)
    assert r.time() == t5
    r.close()


def test_checkpoint_rejects_other_mesh(meshdir, tmp_path):
    m, c, U = make("tet_ref", meshdir)
    s = Solver(m, c, precision="fp64")
    s.set_state(U)
    ck = tmp_path / "ck.bin"
    s.checkpoint_write(str(ck))
    m2, c2, _ = make("tet_sod", meshdir)
    r = Solver(m2, c2, precision="fp64")
    with pytest.raises(Exception, match="cells"):
        r.checkpoint_read(str(ck))
    s.close()
    r.close()


def test_field_dump_matches_state(meshdir, tmp_path):
    m, c, U0 = make("tet_ref", meshdir)
    s = Solver(m, c, precision="fp64")
    s.set_state(U0)
    for _ in range(2):
        s.step()
    f = tmp_path / "field.bin"
    s.field_dump(str(f))
    U = s.get_state()
    d = read_field_dump(str(f))
    v = d["data"]
    assert d["iStep"] == 2 and d["time"] == s.time()[1]
    a = m.arrays()
    aL, aG = U[:, 0], 1 - U[:, 0]
    rL, rG = U[:, 1] / aL, U[:, 2] / aG
    rho = aL * rL + aG * rG

    def p_of(k, r, e):
        g = c.gamma[k]
        return (g - 1) * r * e - g * c.pInf[k] - (g - 1) * c.eta[k] * r

    pL, pG = p_of(0, rL, U[:, 6] / U[:, 1]), p_of(1, rG, U[:, 7] / U[:, 2])
    want = {"x": a["cellCenter"][:, 0], "avfL": aL, "avfG": aG, "rho": rho, "U": U[:, 3] / rho,
            "W": U[:, 5] / rho, "pressure": aL * pL + aG * pG, "vaporMass": U[:, 9]}
    for k, w in want.items():
        col = v[:, d["names"].index(k)]
        assert np.allclose(col, w, rtol=1e-12, atol=1e-12 * np.abs(w).max()), k
    T = v[:, d["names"].index("temperature")]
    assert np.all(T > 50) and np.all(T < 300)
    g = v[:, d["names"].index("gradRho")]
    assert np.all(np.isfinite(g)) and np.all(g >= 0) and g.max() > 0
    s.close()
