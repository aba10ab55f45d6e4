"""TEST INFRASTRUCTURE ONLY — exact solution of the Riemann problem for the ideal-gas Euler
equations (the exact Riemann solver of E. F. Toro, "Riemann Solvers and Numerical Methods for
Fluid Dynamics", chapter 4: pressure function with shock / rarefaction branches, Newton
iteration for the star pressure, sampling of the self-similar solution).  Known-answer check of
the Sod shock tube computed by the solver (the two-phase model with both phases the same ideal
gas reduces to these equations).
"""
from __future__ import annotations

import math

import numpy as np


def _f(p, rho, pk, ck, g):
    """Pressure function f_K(p) and its derivative for side K."""
    if p > pk:   # shock
        A = 2.0 / ((g + 1.0) * rho)
        B = (g - 1.0) / (g + 1.0) * pk
        q = math.sqrt(A / (p + B))
        return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (p + B))
    # rarefaction
    r = (p / pk) ** ((g - 1.0) / (2.0 * g))
    return 2.0 * ck / (g - 1.0) * (r - 1.0), (p / pk) ** (-(g + 1.0) / (2.0 * g)) / (rho * ck)


def star_state(rl, ul, pl, rr, ur, pr, g=1.4, tol=1e-14, itmax=100):
    """Star-region pressure and velocity (Newton iteration from the two-rarefaction guess)."""
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    z = (g - 1.0) / (2.0 * g)
    p = ((cl + cr - 0.5 * (g - 1.0) * (ur - ul)) / (cl / pl ** z + cr / pr ** z)) ** (1.0 / z)
    for _ in range(itmax):
        fl, dl = _f(p, rl, pl, cl, g)
        fr, dr = _f(p, rr, pr, cr, g)
        pn = p - (fl + fr + ur - ul) / (dl + dr)
        pn = max(pn, 1e-14)
        if abs(pn - p) <= tol * 0.5 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    return p, u


def sample(x, t, x0, left, right, g=1.4):
    """Density, velocity, pressure of the exact solution at positions x and time t > 0."""
    rl, ul, pl = left
    rr, ur, pr = right
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    gm = (g - 1.0) / (g + 1.0)
    s = (np.asarray(x, dtype=np.float64) - x0) / t
    rho, u, p = np.empty_like(s), np.empty_like(s), np.empty_like(s)
    for i, si in enumerate(s):
        if si <= us:   # left of the contact
            if ps > pl:   # left shock
                sl = ul - cl * math.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if si <= sl:
                    rho[i], u[i], p[i] = rl, ul, pl
                else:
                    rho[i] = rl * ((ps / pl + gm) / (gm * ps / pl + 1.0))
                    u[i], p[i] = us, ps
            else:         # left rarefaction
                shl = ul - cl
                csl = cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - csl
                if si <= shl:
                    rho[i], u[i], p[i] = rl, ul, pl
                elif si >= stl:
                    rho[i] = rl * (ps / pl) ** (1.0 / g)
                    u[i], p[i] = us, ps
                else:
                    c = 2.0 / (g + 1) * (cl + (g - 1) / 2 * (ul - si))
                    u[i] = 2.0 / (g + 1) * (cl + (g - 1) / 2 * ul + si)
                    rho[i] = rl * (c / cl) ** (2.0 / (g - 1))
                    p[i] = pl * (c / cl) ** (2.0 * g / (g - 1))
        else:          # right of the contact
            if ps > pr:   # right shock
                sr = ur + cr * math.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if si >= sr:
                    rho[i], u[i], p[i] = rr, ur, pr
                else:
                    rho[i] = rr * ((ps / pr + gm) / (gm * ps / pr + 1.0))
                    u[i], p[i] = us, ps
            else:         # right rarefaction
                shr = ur + cr
                csr = cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + csr
                if si >= shr:
                    rho[i], u[i], p[i] = rr, ur, pr
                elif si <= str_:
                    rho[i] = rr * (ps / pr) ** (1.0 / g)
                    u[i], p[i] = us, ps
                else:
                    c = 2.0 / (g + 1) * (cr - (g - 1) / 2 * (ur - si))
                    u[i] = 2.0 / (g + 1) * (-cr + (g - 1) / 2 * ur + si)
                    rho[i] = rr * (c / cr) ** (2.0 / (g - 1))
                    p[i] = pr * (c / cr) ** (2.0 * g / (g - 1))
    return rho, u, p
