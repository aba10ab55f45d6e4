"""CPU checks of the FP64 restatement of the surrogate network (the oracle its device
forward / backward kernels are compared with): analytic gradient vs central differences, and
the BF16 rounding emulation."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.3, M.NPARAM)
    X = rng.normal(0, 1, (16, 3))
    T = rng.normal(0, 1, (16, 4))
    _, g = M.loss_grad(p, X, T)
    idx = rng.choice(M.NPARAM, 40, replace=False)
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_grad(pp, X, T)[0] - M.loss_grad(pm, X, T)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, -2.5, 3.0e38, 1e-40], dtype=np.float32)
    r = M.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0); 1 + 3*2^-8 rounds up
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2**-6 and r[3] == -2.5
    assert np.all(np.isfinite(r[:5]))
    assert abs(r[5] - 1e-40) <= 2.0**-133   # subnormal: quantum 2^-133


def test_layout():
    assert M.NPARAM == 8836
