"""Failure detection on the GPU path without any GPU fault: invalid states are rejected on
upload, and a run driven unstable (time step far above the CFL limit) reports FG_ERR_NAN from
fg_step / fg_check_state instead of carrying on; uploading a good state clears it."""
import numpy as np
import pytest

from gpu_cases import make
from fooskagpu_b200._lib import FG_ERR_NAN, FgError
from fooskagpu_b200.api import Solver

pytestmark = pytest.mark.gpu


def test_set_state_rejects_bad_states(meshdir):
    m, c, U = make("tet_ref", meshdir)
    s = Solver(m, c, precision="fp64")
    for bad in ("nan", "alpha", "density"):
        V = U.copy()
        if bad == "nan":
            V[7, 4] = np.nan
        elif bad == "alpha":
            V[3, 0] = 1.5
        else:
            V[5, 2] = -1.0
        with pytest.raises(FgError) as e:
            s.set_state(V)
        assert e.value.code == FG_ERR_NAN
    s.set_state(U)
    assert s.check_state() == -1
    # the first unusable cell in the caller's order is named, and a rejected upload leaves the
    # state as it was
    V = U.copy()
    V[9, 1] = -2.0
    V[4, 5] = np.inf
    with pytest.raises(FgError, match="cell 4 "):
        s.set_state(V)
    assert np.array_equal(s.get_state(), U)
    s.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_unstable_run_is_reported(prec, meshdir):
    m, c, U = make("tet_sod", meshdir, prec)
    c.adaptDt = 0
    c.dt = 2.0                      # hundreds of times the CFL limit
    s = Solver(m, c, precision=prec)
    s.set_state(U)
    caught = None
    for _ in range(60):
        try:
            s.step()
        except FgError as e:
            caught = e
            break
    if caught is None:
        with pytest.raises(FgError) as e:
            s.check_state()
        caught = e.value
    assert caught.code == FG_ERR_NAN
    # a good state clears the flag; a stable dt then steps normally
    s.set_state(U)
    s.set_dt(1e-5)
    s.step()
    assert s.check_state() == -1
    s.close()
