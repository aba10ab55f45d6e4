"""Case parameters (``fg_case`` = the reference's INPUT fields) and initial conditions.

Initial states are built like the reference's initVec (DP/initialize.cu:18-59): phasic
densities from (p, T) or given directly, phasic internal energies from the stiffened-gas
e(p, rho), and U = [alpha, alpha rhoL, (1-alpha) rhoG, rho u, rho v, rho w,
alpha rhoL eL, (1-alpha) rhoG eG, rho E, m_v].
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .api import default_case
from ._lib import FgCase


def _e(case: FgCase, m: int, p, rho):
    g, pinf, eta = case.gamma[m], case.pInf[m], case.eta[m]
    return (p + g * pinf + (g - 1) * eta * rho) / (rho * (g - 1))


def rho_of_pT(case: FgCase, m: int, p, T):
    g, pinf, cp = case.gamma[m], case.pInf[m], case.Cp[m]
    return (p + pinf) / ((cp / g) * T * (g - 1))


def prim_to_cons(case: FgCase, alpha, rhoL, rhoG, u, v, w, pL, pG=None, mv=0.0) -> np.ndarray:
    alpha, rhoL, rhoG, u, v, w, pL = np.broadcast_arrays(*map(np.asarray, (alpha, rhoL, rhoG, u, v, w, pL)))
    pG = pL if pG is None else np.broadcast_to(np.asarray(pG), pL.shape)
    mv = np.broadcast_to(np.asarray(mv, dtype=np.float64), pL.shape)
    n = pL.shape[0]
    U = np.empty((n, 10))
    ar = alpha * rhoL
    ag = (1 - alpha) * rhoG
    rho = ar + ag
    eL = _e(case, 0, pL, rhoL)
    eG = _e(case, 1, pG, rhoG)
    U[:, 0] = alpha
    U[:, 1] = ar
    U[:, 2] = ag
    U[:, 3] = rho * u
    U[:, 4] = rho * v
    U[:, 5] = rho * w
    U[:, 6] = ar * eL
    U[:, 7] = ag * eG
    U[:, 8] = ar * eL + ag * eG + 0.5 * rho * (u * u + v * v + w * w)
    U[:, 9] = mv
    return U


# ---------------------------------------------------------------- single-phase ideal gas
def _start(base) -> FgCase:
    """A copy of `base`, or the reference's defaults (fg_case_default) when base is None."""
    if base is None:
        return default_case()
    c = FgCase()
    C.pointer(c)[0] = base
    return c


def ideal_gas_case(gamma=1.4, cp=3.5, mu=0.0, rk=3, cfl=0.5, adapt_itr=100, base=None) -> FgCase:
    """Both phases the same ideal gas (p_inf = 0, eta = 0, equal Cp), no phase change:
    the two-phase model then reduces to single-phase Euler/Navier-Stokes for any alpha.
    base: the case to start from (default: the reference's values, fg_case_default)."""
    c = _start(base)
    for m in range(2):
        c.gamma[m] = gamma
        c.pInf[m] = 0.0
        c.Cp[m] = cp
        c.eta[m] = 0.0
        c.dynVisc[m] = mu
        c.satConst[m] = 0.0
    c.chemFlag = 0
    c.woodsFlag = 0
    c.viscFlag = 1 if mu > 0 else 0
    c.turbulence = 1 if mu > 0 else 0
    c.rkSteps = rk
    c.cfl = cfl
    c.maxDt = 1e30
    c.adaptDt = 1
    c.adaptDtItr = adapt_itr
    c.scale = 1.0
    c.consCalcIvar = 1
    return c


def sod_case() -> FgCase:
    """Sod shock tube (inviscid HLLC + MUSCL, SSP-RK3, CFL 0.5)."""
    return ideal_gas_case(gamma=1.4, cp=3.5, mu=0.0, rk=3, cfl=0.5, adapt_itr=10)


def sod_ic(case: FgCase, centres: np.ndarray, x0: float = 0.5, alpha: float = 0.5) -> np.ndarray:
    left = centres[:, 0] < x0
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    z = np.zeros_like(rho)
    return prim_to_cons(case, alpha, rho, rho, z, z, z, p)


def tgv_case(mach=0.1, re=1600.0, rk=3, cfl=0.5, pr=0.71, base=None) -> FgCase:
    """Taylor-Green vortex, rho0 = V0 = L = 1, mu = rho0 V0 L / Re, WALE LES, heat conduction at
    Prandtl number pr (the heat-flux extension; pr = 0 turns it off)."""
    c = ideal_gas_case(gamma=1.4, cp=3.5, mu=1.0 / re, rk=rk, cfl=cfl, adapt_itr=100, base=base)
    if pr > 0:
        c.heatFlux = 1
        c.Pr[0] = c.Pr[1] = pr
    return c


def tgv_ic(case: FgCase, centres: np.ndarray, mach=0.1, alpha: float = 0.5) -> np.ndarray:
    x, y, z = centres[:, 0], centres[:, 1], centres[:, 2]
    g = case.gamma[0]
    p0 = 1.0 / (g * mach * mach)
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(x)
    p = p0 + (1.0 / 16.0) * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    rho = p / p0                     # isothermal start
    return prim_to_cons(case, alpha, rho, rho, u, v, w, p)


# ---------------------------------------------------------------- the reference's own case
def reference_case() -> FgCase:
    """The parameters hard-coded in DP/buildInput.cu:10-69 with mesh coordinates in metres."""
    c = default_case()
    c.scale = 1.0
    return c


def reference_ic(case: FgCase, centres: np.ndarray) -> np.ndarray:
    """Two regions split at x < 0 (DP/initialize.cu:4-8, 26): liquid at 11.4e5 Pa / 115.3 K on
    the left, vapour at 2.6e5 Pa / 115.3 K on the right."""
    left = centres[:, 0] < 0.0
    alpha = np.where(left, 1.0 - case.avfMin, case.avfMin)
    p = np.where(left, 11.4e5, 2.6e5)
    T = 115.3
    rl = rho_of_pT(case, 0, p, T)
    rg = rho_of_pT(case, 1, p, T)
    z = np.zeros_like(p)
    return prim_to_cons(case, alpha, rl, rg, z, z, z, p)


def perturbed_two_phase_ic(case: FgCase, centres: np.ndarray, seed: int = 7, vel=20.0) -> np.ndarray:
    """Smoothly varying two-phase state around the reference's operating point: volume
    fraction, pressures and temperatures vary in space, velocities of O(vel), some cells
    above saturation and some with vapour mass above chemLimit (exercises Wood's sound
    speed, star states of both signs and the chemical relaxation branch)."""
    rng = np.random.default_rng(seed)
    x = centres
    span = np.ptp(x, axis=0) + 1e-30
    xi = (x - x.min(axis=0)) / span
    k = rng.uniform(1.0, 3.0, size=(6, 3))
    ph = rng.uniform(0, 2 * np.pi, size=6)
    f = [np.sin(2 * np.pi * (xi @ k[i]) + ph[i]) for i in range(6)]
    alpha = 0.5 + 0.45 * f[0]
    p = 7e5 + 4e5 * f[1]
    T = 115.3 + 3.0 * f[2]
    rl = rho_of_pT(case, 0, p, T)
    rg = rho_of_pT(case, 1, p, T)
    u = vel * f[3]
    v = vel * f[4]
    w = vel * 0.5 * f[5]
    mv = (1 - alpha) * rg * np.clip(0.5 + 0.5 * f[0], 0, 1)
    return prim_to_cons(case, alpha, rl, rg, u, v, w, p, p, mv)


# ---------------------------------------------------------------- water / vapour bubble collapse
# Saturated water at 293.15 K (IAPWS-IF97 steam tables): the reference state of the fit below.
WATER_SAT_293 = dict(T=293.15, p=2339.2, rho_l=998.16, rho_v=0.017314, h_l=83.91e3, h_v=2537.4e3)


def water_vapour_constants(gamma_l=6.12, pinf_l=3.43e8, gamma_v=1.33, pinf_v=0.0, ref=WATER_SAT_293) -> dict:
    """Stiffened-gas water / vapour constants in the reference's model for the given (gamma, p_inf)
    of each phase, fitted on one saturation state the way Le Metayer, Massoni & Saurel (2004,
    "Elaborating equations of state of a liquid and its vapor for two-phase flow models") fit
    theirs:
      - C_v of each phase from its density on the saturation line, rho = (p + p_inf) / ((gamma - 1) C_v T);
      - the energy offset eta (their q) from the phase enthalpy, h = C_p T + eta;
      - the vapour entropy constant (their q'; the reference's satConst[1], with satConst[0] = 0)
        so that the two Gibbs energies are equal at the reference state.
    The entropy keeps the reference's log10 form, s = C_v log10(T^gamma / (p + p_inf)^(gamma - 1)) + q'
    (DP/chemRlx.cu:38-50), so the saturation line of the model passes through (ref T, ref p).
    The liquid (gamma, p_inf) = (6.12, 3.43e8 Pa) is an acoustic fit: the model's sound speed and
    density are water's, its heat capacity is not."""
    T, p = ref["T"], ref["p"]
    cvl = (p + pinf_l) / ((gamma_l - 1) * ref["rho_l"] * T)
    cvv = (p + pinf_v) / ((gamma_v - 1) * ref["rho_v"] * T)
    cpl, cpv = gamma_l * cvl, gamma_v * cvv
    etal = ref["h_l"] - cpl * T
    etav = ref["h_v"] - cpv * T
    sl = cvl * np.log10(T ** gamma_l / (p + pinf_l) ** (gamma_l - 1))
    sv = cvv * np.log10(T ** gamma_v / (p + pinf_v) ** (gamma_v - 1))
    qv = (ref["h_v"] - ref["h_l"]) / T + sl - sv
    return dict(gamma=(gamma_l, gamma_v), pInf=(pinf_l, pinf_v), Cp=(cpl, cpv), eta=(etal, etav), satConst=(0.0, qv))


def water_vapour_case(rk=3, cfl=0.5, adapt_itr=10, limiter=1, viscous=True, base=None, p_datum=1e7) -> FgCase:
    """Water / vapour homogeneous mixture with Gibbs-equilibrium mass transfer (per-cell Newton),
    HLLC + MUSCL with the van Albada-type limiter (limiter = 1), SSP-RK3; laminar viscosity of
    water (1.0e-3 Pa s) and vapour (9.7e-6 Pa s) at 20 C, no turbulence model.  The wave speeds
    use the frozen mixture sound speed (woodsFlag = 0): Wood's equilibrium sound speed of a
    water / vapour mixture is a few m/s, and with it as the HLLC wave-speed estimate and in the
    CFL bound the reference scheme blows up in the first steps of the bubble collapse.  The
    other INPUT fields keep the reference's values (DP/buildInput.cu:10-69); dt adapts every
    adapt_itr steps.  The pressure datum (fg_case.pressureDatum) is p_datum, the ambient pressure
    (10 MPa for the bubble's liquid): the reduced-precision face momentum flux then carries no
    rounding of the ambient pressure, whose spurious velocities would make the reference's
    absolute-tolerance thermal Newton iterate on the stiff minor phase (0 = the reference's form)."""
    c = _start(base)
    c.woodsFlag = 0
    c.pressureDatum = p_datum
    k = water_vapour_constants()
    for m in range(2):
        c.gamma[m] = k["gamma"][m]
        c.pInf[m] = k["pInf"][m]
        c.Cp[m] = k["Cp"][m]
        c.eta[m] = k["eta"][m]
        c.satConst[m] = k["satConst"][m]
    c.dynVisc[0], c.dynVisc[1] = 1.0e-3, 9.7e-6
    c.viscFlag = 1 if viscous else 0
    c.turbulence = 0
    c.rkSteps = rk
    c.cfl = cfl
    c.adaptDt = 1
    c.adaptDtItr = adapt_itr
    c.maxDt = 1e-6
    c.limiter = limiter
    c.scale = 1.0
    c.consCalcIvar = 0       # vapour volume: the integral of 1 - alpha
    return c


def bubble_ic(case: FgCase, centres: np.ndarray, R0=1e-3, p_bubble=2340.0, p_liquid=1e7, T=298.15,
              width=1e-4, u_wall=0.0) -> np.ndarray:
    """Rayleigh bubble: vapour (liquid volume fraction avfMin) inside radius R0 at p_bubble, liquid
    (1 - avfMin) outside with the Rayleigh-Plesset pressure field p = p_liquid + (p_bubble -
    p_liquid) R0 / r (continuous at R0, p_liquid far away), uniform temperature T; the volume
    fraction changes over a tanh profile of the given width.  At rest by default; u_wall != 0
    gives the radial flow of a bubble wall moving at u_wall, u = u_wall (R0 / r)^2 outside and
    u_wall r / R0 inside.  At T = 298.15 K the saturation pressure of the model is above
    p_bubble, so the liquid of the interface cells is superheated and the Gibbs relaxation acts
    there."""
    r = np.linalg.norm(centres, axis=1)
    amin = case.avfMin
    alpha = amin + (1 - 2 * amin) * 0.5 * (1 + np.tanh((r - R0) / width))
    p = np.where(r <= R0, p_bubble, p_liquid + (p_bubble - p_liquid) * R0 / np.maximum(r, 1e-30))
    rl = rho_of_pT(case, 0, p, T)
    rg = rho_of_pT(case, 1, p, T)
    ur = np.where(r <= R0, u_wall * r / R0, u_wall * (R0 / np.maximum(r, 1e-30)) ** 2)
    rhat = centres / np.maximum(r, 1e-30)[:, None]
    vel = ur[:, None] * rhat
    mv = (1 - alpha) * rg
    return prim_to_cons(case, alpha, rl, rg, vel[:, 0], vel[:, 1], vel[:, 2], p, p, mv)


def mixture_pressure(case: FgCase, U: np.ndarray) -> np.ndarray:
    """Volume-fraction weighted pressure alpha p_L + (1 - alpha) p_G of a state (reference order),
    with alpha clamped as cons2prim does (DP/cons2prim.h:6)."""
    a = np.clip(U[:, 0], case.avfMin / 100, 1 - case.avfMin / 100)
    out = np.zeros(len(U))
    for m, (vol, part, en) in enumerate(((a, U[:, 1], U[:, 6]), (1 - a, U[:, 2], U[:, 7]))):
        rho = part / vol
        e = en / part
        g = case.gamma[m]
        pm = (g - 1) * rho * e - g * case.pInf[m] - (g - 1) * case.eta[m] * rho
        out += vol * pm
    return out


# ---------------------------------------------------------------- liquid jet into pressurised gas
def jet_case(u_jet=200.0, p_gas=5e6, T=298.15, rk=3, cfl=0.3, base=None) -> FgCase:
    """Water jet at u_jet through the inlet (bc 3) into gas at p_gas: the water / vapour constants
    of water_vapour_case with the WALE eddy viscosity (turbulence = 1; Re_D = rho u D / mu = 4e4
    for D = 0.2 mm), the reference's limiter, and the inlet extensions: prescribed inlet velocity
    (0, 0, u_jet) and the inlet state (p_gas, T) instead of the reference's fixed one.  The time
    step adapts every step at CFL 0.3: the CFL bound sees the gas until the liquid (four times
    the sound speed) has entered a cell, and a dt held over ten steps blows up at the inlet."""
    c = water_vapour_case(rk=rk, cfl=cfl, adapt_itr=1, limiter=0, viscous=True, base=base, p_datum=p_gas)
    c.turbulence = 1
    c.inletVelFlag = 1
    c.inletVel[0], c.inletVel[1], c.inletVel[2] = 0.0, 0.0, u_jet
    c.inletStateFlag = 1
    c.inletP, c.inletT = p_gas, T
    return c


def jet_ic(case: FgCase, centres: np.ndarray, p_gas=5e6, T=298.15) -> np.ndarray:
    """Gas (liquid volume fraction avfMin) at p_gas and T, at rest, everywhere."""
    n = len(centres)
    p = np.full(n, p_gas)
    rl = rho_of_pT(case, 0, p, T)
    rg = rho_of_pT(case, 1, p, T)
    z = np.zeros(n)
    return prim_to_cons(case, np.full(n, case.avfMin), rl, rg, z, z, z, p, p, (1 - case.avfMin) * rg)
