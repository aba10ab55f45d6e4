"""Asynchronous state transfer and the state probe through the C ABI.

- fg_set_state_async + fg_step equals fg_set_state + fg_step bit for bit, and so does
  fg_get_state_async after fg_state_join and a stream synchronisation, over several back-to-back
  steps; downloads queued back to back (more than the two staging buffers) each land intact;
- a rejected asynchronous upload leaves the state as it was and is reported by fg_check_state
  and every fg_step until a good upload; the synchronous upload reports it at once;
- fg_probe equals the oracle's conservation integral of variable 0 and numpy's extrema of the
  downloaded state."""
import numpy as np
import pytest
import torch

from gpu_cases import make
from oracle.oracle_py import Oracle
from fooskagpu_b200 import cases
from fooskagpu_b200._lib import FgError
from fooskagpu_b200.api import Solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_async_transfer_equals_sync(prec, meshdir):
    m, c, U = make("tet_ref", meshdir, prec)
    st = torch.cuda.Stream()
    a = Solver(m, c, precision=prec)
    b = Solver(m, c, precision=prec)
    Uin = torch.empty(U.shape, dtype=torch.float64, pin_memory=True)
    Uin.numpy()[:] = U
    Uout = torch.empty(U.shape, dtype=torch.float64, pin_memory=True)
    for k in range(3):
        a.set_state(U)
        a.step()
        Ua = a.get_state()
        b.set_state_async(Uin.numpy(), stream=st.cuda_stream)
        b.step(stream=st.cuda_stream)
        b.get_state_async(Uout.numpy(), stream=st.cuda_stream)
        b.state_join(stream=st.cuda_stream)
        st.synchronize()
        assert np.array_equal(Ua, Uout.numpy()), k
    a.close()
    b.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_back_to_back_downloads(prec, meshdir):
    m, c, U = make("tet_ref", meshdir, prec)
    st = torch.cuda.Stream()
    a = Solver(m, c, precision=prec)
    b = Solver(m, c, precision=prec)
    a.set_state(U)
    b.set_state(U)
    want, outs = [], []
    for k in range(5):
        a.step()
        want.append(a.get_state())
        b.step(stream=st.cuda_stream)
        o = torch.empty(U.shape, dtype=torch.float64, pin_memory=True)
        b.get_state_async(o.numpy(), stream=st.cuda_stream)
        outs.append(o)
    b.state_join(stream=st.cuda_stream)
    st.synchronize()
    for k in range(5):
        assert np.array_equal(want[k], outs[k].numpy()), k
    a.close()
    b.close()


def test_rejected_async_upload_keeps_the_state(meshdir):
    m, c, U = make("tet_ref", meshdir, "fp64")
    s = Solver(m, c, precision="fp64")
    s.set_state(U)
    s.step()
    good = s.get_state()
    bad = U.copy()
    bad[7, 3] = np.nan
    bad[11, 1] = -1.0
    s.set_state_async(np.ascontiguousarray(bad))
    with pytest.raises(FgError, match="cell 7") as e:
        s.check_state()
    assert e.value.code == 5
    with pytest.raises(FgError, match="not replaced"):
        s.step()
    assert np.array_equal(s.get_state(), good)
    s.set_state_async(np.ascontiguousarray(U))
    s.step()
    assert s.check_state() == -1
    with pytest.raises(FgError, match="cell 7"):
        s.set_state(bad)
    s.step()                          # a synchronous rejection is reported once, the state stays usable
    s.close()


def test_probe_matches_host(meshdir):
    m, c, U = make("ball_bubble", meshdir, "fp64")
    o = Oracle(m.view(), c)
    s = Solver(m, c, precision="fp64")
    s.set_state(U)
    for _ in range(2):
        s.step()
    pr = s.probe()
    Ug = s.get_state()
    vol = m.arrays()["volume"]
    assert abs(pr["vapourVolume"] - o.cons_calc(0, Ug)) <= 1e-12 * abs(pr["vapourVolume"])
    p = cases.mixture_pressure(c, Ug)
    assert abs(pr["maxPressure"] - p.max()) <= 1e-12 * abs(p.max())
    assert abs(pr["minPressure"] - p.min()) <= 1e-9 * abs(p).max()
    rho = Ug[:, 1] + Ug[:, 2]
    speed = np.sqrt((Ug[:, 3] ** 2 + Ug[:, 4] ** 2 + Ug[:, 5] ** 2)) / rho
    assert abs(pr["maxSpeed"] - speed.max()) <= 1e-9 * max(speed.max(), 1e-300)
    assert abs(pr["vapourVolume"] - ((1 - Ug[:, 0]) * vol).sum()) <= 1e-9 * pr["vapourVolume"]
    s.close()
