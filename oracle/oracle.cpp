/*
 * oracle.cpp — TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * FP64 CPU restatement of the reference FooskaGPU double-precision solver's explicit
 * residual path.  Each function cites the reference file:line it restates (paths relative to
 * "mulitphase Solver/doublePrecision/", written DP/ below).  Arithmetic is written in the
 * reference's evaluation order so that the scalar functions agree bit for bit with the
 * reference headers compiled for the host (the known-answer tests check exactly that).
 *
 * Build: g++ -O2 -fopenmp -ffp-contract=off (no FMA contraction, as the host reference build).
 */
#include "oracle.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

int g_threads = 1;

inline double clamp_avf(const fg_case *c, double a) {
    /* fmin(fmax(avfMin/100, a), 1.0 - avfMin/100)  (DP/cons2prim.h:6) */
    return fmin(fmax(c->avfMin / 100, a), 1.0 - c->avfMin / 100);
}

/* Stiffened gas with energy offset eta (DP/eqos.h:1-23). */
inline double eqos(const fg_case *c, int m, int id, double v1, double v2) {
    const double g = c->gamma[m], pinf = c->pInf[m], cp = c->Cp[m], eta = c->eta[m];
    double r = 0;
    switch (id) {
    case 0: /* p(rho, e) */
        r = (g - 1) * v1 * v2 - g * pinf - (g - 1) * eta * v1;
        break;
    case 1: /* T(rho, e) */
        r = (g - 1) * v1 * v2 - g * pinf - (g - 1) * eta * v1;
        r = (r + pinf) / ((cp / g) * (g - 1) * v1);
        break;
    case 2: /* rho(p, T) */
        r = (v1 + pinf) / ((cp / g) * v2 * (g - 1));
        break;
    case 3: /* e(p, rho) */
        r = (v1 + g * pinf + (g - 1) * eta * v2) / (v2 * (g - 1));
        break;
    case 4: /* sound speed c(rho, p) */
        r = sqrt((g * (v2 + pinf)) / v1);
        break;
    }
    return r;
}

/* DP/cons2prim.h:2-24 — prim = [alpha, rhoL, rhoG, u, v, w, pL, pG, m_v, rho]. */
inline void cons2prim(const fg_case *c, const double *U, double *s) {
    s[0] = clamp_avf(c, U[0]);
    s[1] = U[1] / s[0];
    s[2] = U[2] / (1 - s[0]);
    const double rho = s[0] * s[1] + (1 - s[0]) * s[2];
    s[3] = U[3] / rho;
    s[4] = U[4] / rho;
    s[5] = U[5] / rho;
    const double eL = U[6] / (s[0] * s[1]);
    const double eG = U[7] / ((1 - s[0]) * s[2]);
    s[6] = eqos(c, 0, 0, s[1], eL);
    s[7] = eqos(c, 1, 0, s[2], eG);
    s[8] = U[9];
    s[9] = rho;
}

/* DP/prim2cons.h:2-21 */
inline void prim2cons(const fg_case *c, const double *p, double *u) {
    u[0] = p[0];
    u[1] = p[0] * p[1];
    u[2] = (1 - p[0]) * p[2];
    const double rho = u[1] + u[2];
    u[3] = rho * p[3];
    u[4] = rho * p[4];
    u[5] = rho * p[5];
    u[6] = u[1] * eqos(c, 0, 3, p[6], p[1]);
    u[7] = u[2] * eqos(c, 1, 3, p[7], p[2]);
    u[8] = u[6] + u[7] + 0.5 * rho * (p[3] * p[3] + p[4] * p[4] + p[5] * p[5]);
    u[9] = p[8];
}

/* DP/rotateVector.h:2-14 */
inline void to_local(const double *g, double *l, const double *n, const double *t1, const double *t2) {
    l[0] = g[0] * n[0] + g[1] * n[1] + g[2] * n[2];
    l[1] = g[0] * t1[0] + g[1] * t1[1] + g[2] * t1[2];
    l[2] = g[0] * t2[0] + g[1] * t2[1] + g[2] * t2[2];
}
inline void to_global(const double *l, double *g, const double *n, const double *t1, const double *t2) {
    g[0] = l[0] * n[0] + l[1] * t1[0] + l[2] * t2[0];
    g[1] = l[0] * n[1] + l[1] * t1[1] + l[2] * t2[1];
    g[2] = l[0] * n[2] + l[1] * t1[2] + l[2] * t2[2];
}

/* DP/waveSpeeds.h:2-46 — cOut = [S_L, S_star, S_R]. */
void wave_speeds(const fg_case *c, const double *n, const double *t1, const double *t2,
                 const double *sL, const double *sR, double *cOut, double *uL, double *uR) {
    double vL[3] = {sL[3], sL[4], sL[5]}, vR[3] = {sR[3], sR[4], sR[5]};
    to_local(vL, uL, n, t1, t2);
    to_local(vR, uR, n, t1, t2);
    double cL, cR;
    if ((sL[8] + sR[8]) / 2 > c->chemLimit && c->woodsFlag == 1) {
        /* Wood's mixture sound speed */
        double rm = sL[0] * sL[1] + (1 - sL[0]) * sL[2];
        double cl = eqos(c, 0, 4, sL[1], sL[6]);
        double cg = eqos(c, 1, 4, sL[2], sL[7]);
        cL = 1 / sqrt(rm * (sL[0] / (sL[1] * cl * cl) + (1 - sL[0]) / (sL[2] * cg * cg)));
        rm = sR[0] * sR[1] + (1 - sR[0]) * sR[2];
        cl = eqos(c, 0, 4, sR[1], sR[6]);
        cg = eqos(c, 1, 4, sR[2], sR[7]);
        cR = 1 / sqrt(rm * (sR[0] / (sR[1] * cl * cl) + (1 - sR[0]) / (sR[2] * cg * cg)));
    } else {
        /* mass-fraction weighted frozen sound speed */
        double yl = sL[0] * sL[1] / (sL[0] * sL[1] + (1 - sL[0]) * sL[2]);
        double yg = (1 - sL[0]) * sL[2] / (sL[0] * sL[1] + (1 - sL[0]) * sL[2]);
        cL = sqrt(yl * pow(eqos(c, 0, 4, sL[1], sL[6]), 2) + yg * pow(eqos(c, 1, 4, sL[2], sL[7]), 2));
        yl = sR[0] * sR[1] / (sR[0] * sR[1] + (1 - sR[0]) * sR[2]);
        yg = (1 - sR[0]) * sR[2] / (sR[0] * sR[1] + (1 - sR[0]) * sR[2]);
        cR = sqrt(yl * pow(eqos(c, 0, 4, sR[1], sR[6]), 2) + yg * pow(eqos(c, 1, 4, sR[2], sR[7]), 2));
    }
    cOut[0] = fmin(uL[0] - cL, uR[0] - cR);
    cOut[2] = fmax(uL[0] + cL, uR[0] + cR);
    const double pL = sL[0] * sL[6] + (1 - sL[0]) * sL[7];
    const double pR = sR[0] * sR[6] + (1 - sR[0]) * sR[7];
    const double rL = sL[0] * sL[1] + (1 - sL[0]) * sL[2];
    const double rR = sR[0] * sR[1] + (1 - sR[0]) * sR[2];
    cOut[1] = (pR - pL + rL * uL[0] * (cOut[0] - uL[0]) - rR * uR[0] * (cOut[2] - uR[0])) /
              (rL * (cOut[0] - uL[0]) - rR * (cOut[2] - uR[0]));
}

/* Boundary ghost states (DP/bc.h:2-84): 1 symmetry, 2 outlet, 3 inlet, 4 slip, 5 wall. */
void bc_values(const fg_case *c, const double *n, const double *t1, const double *t2, double *s, int bc) {
    if (bc == 1 || bc == 4 || bc == 5) {
        double v[3] = {s[3], s[4], s[5]}, l[3], r[3];
        to_local(v, l, n, t1, t2);
        r[0] = -l[0];
        r[1] = (bc == 5) ? -l[1] : l[1];
        r[2] = (bc == 5) ? -l[2] : l[2];
        to_global(r, v, n, t1, t2);
        s[3] = v[0];
        s[4] = v[1];
        s[5] = v[2];
    } else if (bc == 3) {
        /* Dirichlet inlet with the reference's fixed p = 11.4e5 Pa, T = 115.3 K (DP/bc.h:2-25), or
         * the case's prescribed inlet state (extension) */
        const int own = (c->inletStateFlag == 1);
        const double pIn = own ? c->inletP : 11.4e5, tIn = own ? c->inletT : 115.3;
        s[0] = 1.0 - c->avfMin;
        s[1] = eqos(c, 0, 2, pIn, tIn);
        s[2] = eqos(c, 1, 2, pIn, tIn);
        s[6] = pIn;
        s[7] = pIn;
        s[8] = 0;
        s[9] = 0;
        if (c->inletVelFlag == 1) {   /* prescribed inlet velocity (extension) */
            s[3] = c->inletVel[0];
            s[4] = c->inletVel[1];
            s[5] = c->inletVel[2];
        }
    }
    /* bc == 2 (outlet): zero gradient, ghost = interior */
}

/* HLLC star state (DP/starRegion.h:3-35); consF[6], consF[7] are replaced by the star
 * phasic energies, consF[8] is read. */
void star_region(const fg_case *c, const double *s, const double *ul, double SK, double SS,
                 const double *n, const double *t1, const double *t2, double *uNC, double *vS,
                 double *consF) {
    double u[3] = {SS, ul[1], ul[2]};
    to_global(u, uNC, n, t1, t2);
    const double rSL = s[1] * (SK - ul[0]) / (SK - SS);
    const double rSG = s[2] * (SK - ul[0]) / (SK - SS);
    vS[0] = s[0];
    vS[1] = s[0] * rSL;
    vS[2] = (1 - s[0]) * rSG;
    const double rS = vS[1] + vS[2];
    vS[3] = rS * uNC[0];
    vS[4] = rS * uNC[1];
    vS[5] = rS * uNC[2];
    const double g0 = c->gamma[0], g1 = c->gamma[1];
    const double pSL = (s[6] + c->pInf[0]) * ((g0 - 1) * s[1] - (g0 + 1) * rSL) /
                           ((g0 - 1) * rSL - (g0 + 1) * s[1]) - c->pInf[0];
    const double pSG = (s[7] + c->pInf[1]) * ((g1 - 1) * s[2] - (g1 + 1) * rSG) /
                           ((g1 - 1) * rSG - (g1 + 1) * s[2]) - c->pInf[1];
    consF[6] = vS[1] * eqos(c, 0, 3, pSL, rSL);
    consF[7] = vS[2] * eqos(c, 1, 3, pSG, rSG);
    const double p = s[0] * s[6] + (1 - s[0]) * s[7];
    const double r = s[0] * s[1] + (1 - s[0]) * s[2];
    if (c->hllcEnergyFix == 1)   /* standard HLLC energy star state (extension) */
        vS[8] = ((SK - ul[0]) / (SK - SS)) * (consF[8] + r * (SS - ul[0]) * (SS + p / (r * (SK - ul[0]))));
    else
        vS[8] = ((SK - ul[0]) / (SK - SS)) * (consF[8] + (SS - ul[0]) * (SS + p / (r * (SK - ul[0]))));
    vS[9] = s[8] * (SK - ul[0]) / (SK - SS);
}

/* Advective flux (DP/flux.h:32-91). */
void adv_flux(const fg_case *c, const double *p, double *F, const double *n, const double *uNC,
              double areL, double areG) {
    const double rho = p[0] * p[1] + (1 - p[0]) * p[2];
    const double prs = p[0] * p[6] + (1 - p[0]) * p[7];
    const double rE = p[0] * p[1] * eqos(c, 0, 3, p[6], p[1]) +
                      (1 - p[0]) * p[2] * eqos(c, 1, 3, p[7], p[2]) +
                      0.5 * rho * (p[3] * p[3] + p[4] * p[4] + p[5] * p[5]);
    double f;
    f = uNC[0] * p[0] * n[0]; f += uNC[1] * p[0] * n[1]; f += uNC[2] * p[0] * n[2]; F[0] = f;
    f = p[3] * p[0] * p[1] * n[0]; f += p[4] * p[0] * p[1] * n[1]; f += p[5] * p[0] * p[1] * n[2]; F[1] = f;
    f = p[3] * (1 - p[0]) * p[2] * n[0]; f += p[4] * (1 - p[0]) * p[2] * n[1]; f += p[5] * (1 - p[0]) * p[2] * n[2]; F[2] = f;
    f = rho * p[3] * p[3] * n[0]; f += rho * p[3] * p[4] * n[1]; f += rho * p[3] * p[5] * n[2]; F[3] = f;
    f = rho * p[4] * p[3] * n[0]; f += rho * p[4] * p[4] * n[1]; f += rho * p[4] * p[5] * n[2]; F[4] = f;
    f = rho * p[5] * p[3] * n[0]; f += rho * p[5] * p[4] * n[1]; f += rho * p[5] * p[5] * n[2]; F[5] = f;
    f = uNC[0] * areL * n[0]; f += uNC[1] * areL * n[1]; f += uNC[2] * areL * n[2]; F[6] = f;
    f = uNC[0] * areG * n[0]; f += uNC[1] * areG * n[1]; f += uNC[2] * areG * n[2]; F[7] = f;
    f = p[3] * (rE + prs) * n[0]; f += p[4] * (rE + prs) * n[1]; f += p[5] * (rE + prs) * n[2]; F[8] = f;
    f = p[3] * p[8] * n[0]; f += p[4] * p[8] * n[1]; f += p[5] * p[8] * n[2]; F[9] = f;
}

/* Non-conservative terms from cell-centre states (DP/flux.h:1-30); fnc[k*2+side]. */
void flux_source(const fg_case *c, const double *uNC, const double *UL, const double *UR,
                 const double *n, double *fnc) {
    const double *Us[2] = {UL, UR};
    for (int s = 0; s < 2; s++) {
        const double *U = Us[s];
        const double a = fmin(fmax(c->avfMin / 100, U[0]), 1 - c->avfMin / 100);
        const double rl = U[1] / a, rg = U[2] / (1 - a);
        const double el = U[6] / (a * rl), eg = U[7] / ((1 - a) * rg);
        const double pl = eqos(c, 0, 0, rl, el), pg = eqos(c, 1, 0, rg, eg);
        fnc[0 * 2 + s] = a * uNC[0] * n[0] + a * uNC[1] * n[1] + a * uNC[2] * n[2];
        fnc[1 * 2 + s] = a * pl * uNC[0] * n[0] + a * pl * uNC[1] * n[1] + a * pl * uNC[2] * n[2];
        fnc[2 * 2 + s] = (1 - a) * pg * uNC[0] * n[0] + (1 - a) * pg * uNC[1] * n[1] + (1 - a) * pg * uNC[2] * n[2];
    }
}

/* Cell-centre mixture pressure (DP/computeRHS.cu:38-52). */
double centre_pressure(const fg_case *c, const double *U) {
    const double a = fmin(fmax(c->avfMin / 100, U[0]), 1.0 - c->avfMin / 100);
    const double rl = U[1] / a, rg = U[2] / (1 - a);
    const double el = U[6] / (a * rl), eg = U[7] / ((1 - a) * rg);
    return a * eqos(c, 0, 0, rl, el) + (1 - a) * eqos(c, 1, 0, rg, eg);
}

/* Contribution of one face to one side (DP/computeRHS.cu:61-75), written to out[10]. */
void side_contrib(int id, const double *fa, const double *fh, const double *fnc, double pt,
                  const double *n, double A, double *out) {
    const double sg = (id == 0) ? -1.0 : 1.0;
    out[0] = sg * (fa[0] - fnc[0 * 2 + id]) * A;
    out[1] = sg * (fa[1] + fh[1]) * A;
    out[2] = sg * (fa[2] + fh[2]) * A;
    out[3] = sg * (fa[3] + fh[3] + pt * n[0]) * A;
    out[4] = sg * (fa[4] + fh[4] + pt * n[1]) * A;
    out[5] = sg * (fa[5] + fh[5] + pt * n[2]) * A;
    out[6] = sg * (fa[6] + fnc[1 * 2 + id]) * A;
    out[7] = sg * (fa[7] + fnc[2 * 2 + id]) * A;
    out[8] = sg * (fa[8] + fh[8]) * A;
    out[9] = sg * (fa[9] + fh[9]) * A;
}

/* computeFlux body for one face (DP/computeRHS.cu:78-146).  solL/solR are the reconstructed
 * face states (solR already the ghost for boundary faces), UL/UR cell-centre conserved states.
 * out[0..9] owner, out[10..19] neighbour. */
void face_flux(const fg_case *c, const double *n, const double *t1, const double *t2, double A,
               int bc, const double *solL, const double *solR, const double *UL, const double *UR,
               double *out) {
    double cs[3], uL[3], uR[3];
    wave_speeds(c, n, t1, t2, solL, solR, cs, uL, uR);
    int isLeft = (cs[1] >= 0);
    if (c->hllcTieTol > 0 && fabs(cs[1]) <= c->hllcTieTol * (fabs(cs[0]) + fabs(cs[2]))) isLeft = 1;
    const int isStar = (cs[0] < 0 && cs[2] >= 0);
    const double *s = isLeft ? solL : solR;
    const double *vl = isLeft ? uL : uR;
    const double cK = isLeft ? cs[0] : cs[2];
    double uNC[3] = {s[3], s[4], s[5]};
    double consF[10], vS[10] = {0}, fh[10] = {0}, fa[10], fnc[6];
    prim2cons(c, s, consF);
    if (isStar) {
        star_region(c, s, vl, cK, cs[1], n, t1, t2, uNC, vS, consF);
        const int idx[7] = {1, 2, 3, 4, 5, 8, 9};
        for (int k = 0; k < 7; k++) fh[idx[k]] = cK * (vS[idx[k]] - consF[idx[k]]);
    }
    adv_flux(c, s, fa, n, uNC, consF[6], consF[7]);
    flux_source(c, uNC, UL, UR, n, fnc);
    const double pF = s[0] * s[6] + (1 - s[0]) * s[7];
    const double pc0 = pF - centre_pressure(c, UL);
    side_contrib(0, fa, fh, fnc, pc0, n, A, out);
    if (bc == 0) {
        const double pc1 = pF - centre_pressure(c, UR);
        side_contrib(1, fa, fh, fnc, pc1, n, A, out + 10);
    } else {
        for (int v = 0; v < 10; v++) out[10 + v] = 0;
    }
}

/* WALE eddy viscosity (DP/computeViscousStresses.cu:3-60). */
double eddy_visc(double ux, double uy, double uz, double vx, double vy, double vz, double wx,
                 double wy, double wz, double vol) {
    double g[3][3] = {{ux, uy, uz}, {vx, vy, vz}, {wx, wy, wz}};
    double sq[3][3], sd[3][3], st[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            sq[i][j] = 0.0;
            for (int k = 0; k < 3; k++) sq[i][j] += g[i][k] * g[k][j];
        }
    double T = 0.0;
    for (int i = 0; i < 3; i++) T += sq[i][i];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            const int kr = (i == j);
            sd[i][j] = 0.5 * (sq[i][j] + sq[j][i]) - (1.0 / 3.0) * kr * T;
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) st[i][j] = 0.5 * (g[i][j] + g[j][i]);
    double s1 = 0, s2 = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            s1 += sd[i][j] * sd[i][j];
            s2 += st[i][j] * st[i][j];
        }
    double num = pow(s1, 1.5);
    const double den = pow(s1, 1.25) + pow(s2, 2.5) + 1e-12;
    if (den < 1e-10) num = 0;
    const double Ls = 0.325 * pow(vol, 0.3333333333333);
    return Ls * Ls * num / den;
}

/* Gradient of the liquid-phase temperature T = (pL + pInf) / (cv (gamma - 1) rhoL) of a cell
 * (chain rule on the gradients of rhoL and pL), for the heat-conduction extension. */
static void cell_grad_t(const fg_case *c, const double *U, const double *g, double *out) {
    double s[10];
    cons2prim(c, U, s);
    const double rl = s[1], pl = s[6];
    const double cvgm1 = (c->Cp[0] / c->gamma[0]) * (c->gamma[0] - 1);
    const double k = (pl + c->pInf[0]) / rl;
    for (int d = 0; d < 3; d++) out[d] = (g[6 * 3 + d] - k * g[1 * 3 + d]) / (cvgm1 * rl);
}

/* Viscous face flux (DP/computeViscousStresses.cu:66-174) — out[0..9] owner, [10..19] nb.
 * Uo / Un: cell-centre states of owner and neighbour (heat-conduction extension only). */
void viscous_face(const fg_case *c, const double *gO, const double *gN, double volAvg,
                  const double *pf0, const double *pf1, const double *n, double A, int bc,
                  const double *Uo, const double *Un, double *out) {
    const double ux = (gO[9 + 0] + gN[9 + 0]) / 2, uy = (gO[9 + 1] + gN[9 + 1]) / 2, uz = (gO[9 + 2] + gN[9 + 2]) / 2;
    const double vx = (gO[12 + 0] + gN[12 + 0]) / 2, vy = (gO[12 + 1] + gN[12 + 1]) / 2, vz = (gO[12 + 2] + gN[12 + 2]) / 2;
    const double wx = (gO[15 + 0] + gN[15 + 0]) / 2, wy = (gO[15 + 1] + gN[15 + 1]) / 2, wz = (gO[15 + 2] + gN[15 + 2]) / 2;
    double nu_t = 0;
    if (c->turbulence == 1) nu_t = eddy_visc(ux, uy, uz, vx, vy, vz, wx, wy, wz, volAvg);
    double tau[3][3];
    tau[0][0] = (2.0 * ux - (2.0 / 3.0) * (ux + vy + wz));
    tau[1][1] = (2.0 * vy - (2.0 / 3.0) * (ux + vy + wz));
    tau[2][2] = (2.0 * wz - (2.0 / 3.0) * (ux + vy + wz));
    tau[0][1] = (uy + vx);
    tau[0][2] = (uz + wx);
    tau[1][2] = (vz + wy);
    tau[1][0] = tau[0][1];
    tau[2][1] = tau[1][2];
    tau[2][0] = tau[0][2];
    const double a1 = pf0[0], r1 = a1 * pf0[1] + (1 - a1) * pf0[2];
    const double a2 = pf1[0], r2 = a2 * pf1[1] + (1 - a2) * pf1[2];
    const double rF = (r1 + r2) / 2, aF = (a1 + a2) / 2;
    const double mu = aF * c->dynVisc[0] + (1 - aF) * c->dynVisc[1] + rF * nu_t;
    double vs[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) vs[i][j] = mu * tau[i][j];
    double fm[3];
    for (int i = 0; i < 3; i++) fm[i] = vs[i][0] * n[0] + vs[i][1] * n[1] + vs[i][2] * n[2];
    for (int v = 0; v < 20; v++) out[v] = 0;
    for (int i = 0; i < 3; i++) {
        out[3 + i] = (fm[i]) * A;
        if (bc == 0) out[13 + i] = -(fm[i]) * A;
    }
    const double vf[3] = {(pf0[3] + pf1[3]) / 2, (pf0[4] + pf1[4]) / 2, (pf0[5] + pf1[5]) / 2};
    double fe[3];
    for (int i = 0; i < 3; i++) {
        double stv = 0;
        for (int j = 0; j < 3; j++) stv += tau[i][j] * vf[j];
        fe[i] = (mu * stv) * n[i];
    }
    out[8] = (fe[0] + fe[1] + fe[2]) * A;
    if (bc == 0) out[18] = -(fe[0] + fe[1] + fe[2]) * A;
    if (c->heatFlux == 1 && bc == 0) {
        /* Fourier conduction (extension): k = cp mu / Pr at the face, mean of the two cells'
         * temperature gradients; boundary faces adiabatic */
        double tO[3], tN[3];
        cell_grad_t(c, Uo, gO, tO);
        cell_grad_t(c, Un, gN, tN);
        const double cpF = aF * c->Cp[0] + (1 - aF) * c->Cp[1];
        const double prF = aF * c->Pr[0] + (1 - aF) * c->Pr[1];
        const double kF = mu * cpF / prF;
        double q = 0;
        for (int d = 0; d < 3; d++) q += 0.5 * (tO[d] + tN[d]) * n[d];
        out[8] += kF * q * A;
        out[18] -= kF * q * A;
    }
}

/* Max signal speed of a face state (DP/computeTimeStep.cu:15-46). */
double face_max_signal(const fg_case *c, const double *pv, const double *n, const double *t1,
                       const double *t2) {
    const double a = pv[0], rl = pv[1], rg = pv[2];
    const double vg[3] = {pv[3], pv[4], pv[5]};
    const double pl = pv[6], pg = pv[7];
    const double rm = a * rl + (1 - a) * rg;
    const double cl = eqos(c, 0, 4, rl, pl), cg = eqos(c, 1, 4, rg, pg);
    double cm;
    if (pv[8] > c->chemLimit && c->woodsFlag == 1) {
        cm = 1 / sqrt(rm * (a / (rl * cl * cl) + (1 - a) / (rg * cg * cg)));
    } else {
        const double yl = a * rl / rm, yg = (1 - a) * rg / rm;
        cm = sqrt(yl * cl * cl + yg * cg * cg);
    }
    double vl[3];
    to_local(vg, vl, n, t1, t2);
    return fabs(vl[0]) + cm;
}

/* ---------------- relaxation ---------------- */

/* Saturation temperature Newton (DP/relaxation.cu:4-38). */
double saturation_temp(const fg_case *c, double P, double temp, double urf) {
    const double Pinf = c->pInf[0];
    const double g1 = c->gamma[0], g2 = c->gamma[1];
    const double Cp1 = c->Cp[0], Cp2 = c->Cp[1];
    const double Cv1 = Cp1 / g1, Cv2 = Cp2 / g2;
    const double eta1 = c->eta[0], eta2 = c->eta[1];
    const double etaT1 = 0;
    const double etaT2 = c->satConst[0] * log10(P) + c->satConst[1];
    const double As = (Cp1 - Cp2 + etaT2 - etaT1) / (Cp2 - Cv2);
    const double Bs = (eta1 - eta2) / (Cp2 - Cv2);
    const double Cs = (Cp2 - Cp1) / (Cp2 - Cv2);
    const double Ds = (Cp1 - Cv1) / (Cp2 - Cv2);
    const double dT = 1.e-3;
    double fun = 1, T = temp;
    int itr = 0;
    while (fabs(fun) > 1.e-2 && itr < 50) {
        fun = As + Bs / T + Cs * log10(T) + Ds * log10(P + Pinf) - log10(P);
        const double fdt = As + Bs / (T + dT) + Cs * log10(T + dT) + Ds * log10(P + Pinf) - log10(P);
        const double gr = (fdt - fun) / dT;
        T = T - urf * fun / gr;
        itr++;
    }
    return T;
}

/* thermal residual (DP/thermRlx.cu:70-90); writes the primary phase's entries of x. */
void therm_residual(const fg_case *c, int pm, double *x, const double *ar, const double *enr,
                    float dP, float dT, double *r0, double *r1) {
    double s1 = 0, s2 = 0;
    for (int m = 0; m < 2; m++)
        if (m != pm) {
            s1 = ar[m] / x[m];
            s2 = ar[m] * (x[2 + m] - enr[m]);
        }
    x[pm] = (1 / (1 - s1)) * ar[pm];
    x[2 + pm] = enr[pm] - (1 / ar[pm]) * s2;
    double p[2], T[2];
    for (int m = 0; m < 2; m++) {
        p[m] = eqos(c, m, 0, x[m], x[m + 2]);
        T[m] = eqos(c, m, 1, x[m], x[m + 2]);
    }
    *r0 = p[0] - p[1] - dP;
    *r1 = T[0] - T[1] - dT;
}

int therm_relax_cell(const fg_case *c, double *U, int *itrOut) {
    /* initialisation (DP/thermRlx.cu:4-40) */
    double avf[2], rho[2], ar[2], enr[2], vel[3], Y[2], x[4], ax[4];
    avf[0] = fmin(fmax(c->avfMin / 100, U[0]), 1 - c->avfMin / 100);
    avf[1] = 1 - avf[0];
    rho[0] = U[1] / avf[0];
    rho[1] = U[2] / avf[1];
    ar[0] = avf[0] * rho[0];
    ar[1] = avf[1] * rho[1];
    enr[0] = U[6] / ar[0];
    enr[1] = U[7] / ar[1];
    const double rm = ar[0] + ar[1];
    vel[0] = U[3] / rm;
    vel[1] = U[4] / rm;
    vel[2] = U[5] / rm;
    Y[0] = ar[0] / rm;
    Y[1] = ar[1] / rm;
    const double rE = U[8];
    x[0] = rho[0]; x[1] = rho[1]; x[2] = enr[0]; x[3] = enr[1];
    for (int i = 0; i < 4; i++) ax[i] = x[i];
    int pm = 0;
    {
        double mx = -1.0;
        for (int m = 0; m < 2; m++)
            if (avf[m] > mx) { mx = avf[m]; pm = m; }
    }
    /* energy redistribution (DP/thermRlx.cu:208-210) */
    const double de = rE / rm - Y[0] * enr[0] - Y[1] * enr[1] - 0.5 * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
    enr[0] += de;
    enr[1] += de;
    const float dP = 0.0f, dT = 0.0f; /* finite-rate branch (thermFntRlxFlag) is not supported */
    float minRes = 1e9f;
    int abortFlag = 0, itr = 0, aborted = 0;
    bool conv = false;
    double res[2], jac[2][2], inv[2][2];
    while (!conv) {
        itr++;
        therm_residual(c, pm, x, ar, enr, dP, dT, &res[0], &res[1]);
        /* finite-difference Jacobian (DP/thermRlx.cu:92-115) */
        double e[2], rdf[2][2];
        int iv = 0;
        for (int j = 0; j < 4; j++)
            if (j != pm && j != pm + 2) {
                e[iv] = 1e-4 * x[j];
                x[j] += e[iv];
                therm_residual(c, pm, x, ar, enr, dP, dT, &rdf[0][iv], &rdf[1][iv]);
                x[j] -= e[iv];
                iv++;
            }
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) {
                jac[i][j] = (rdf[i][j] - res[i]) / e[j];
                if (std::isnan(jac[i][j])) abortFlag = 1;
            }
        /* 2x2 inverse (DP/thermRlx.cu:117-126) */
        const double det = jac[0][0] * jac[1][1] - jac[1][0] * jac[0][1];
        inv[0][0] = jac[1][1] / det;
        inv[1][1] = jac[0][0] / det;
        inv[1][0] = -jac[1][0] / det;
        inv[0][1] = -jac[0][1] / det;
        if (det == 0) abortFlag = 1;
        /* best-iterate bookkeeping (DP/thermRlx.cu:128-140) */
        if (abortFlag == 0 && x[0] > 0.0 && x[1] > 0.0) {
            const float chk = sqrt(res[0] * res[0] + res[1] * res[1]);
            if (chk < minRes) {
                minRes = chk;
                for (int i = 0; i < 4; i++) ax[i] = x[i];
            }
        }
        /* Newton update (DP/thermRlx.cu:142-170) */
        iv = 0;
        for (int i = 0; i < 4; i++)
            if (i != pm && i != pm + 2) {
                double dx = 0;
                for (int j = 0; j < 2; j++) dx += inv[iv][j] * res[j];
                x[i] = x[i] - c->thermUrf * dx;
                iv++;
            }
        int chk = 0;
        for (int j = 0; j < 2; j++)
            if (fabs(res[j]) > 1.e-2) chk += 1;
        if (chk == 0) conv = true;
        if (abortFlag == 1 || itr > c->thermItrMax) {
            for (int i = 0; i < 4; i++) x[i] = ax[i];
            conv = true;
            aborted = 1;
        }
    }
    /* write back (DP/thermRlx.cu:172-187) */
    double s1 = 0, s2 = 0;
    for (int m = 0; m < 2; m++)
        if (m != pm) {
            s1 = ar[m] / x[m];
            s2 = ar[m] * (x[2 + m] - enr[m]);
        }
    x[pm] = (1 / (1 - s1)) * ar[pm];
    x[2 + pm] = enr[pm] - (1 / ar[pm]) * s2;
    U[0] = fmin(fmax(c->avfMin / 100, ar[0] / x[0]), 1 - c->avfMin / 100);
    U[6] = ar[0] * x[2];
    U[7] = ar[1] * x[3];
    if (itrOut) *itrOut = itr;
    return aborted;
}

/* Gibbs free energy (DP/chemRlx.cu:38-50). */
double gibbs(const fg_case *c, int m, double P, double T) {
    double et[2];
    et[0] = 0;
    et[1] = c->satConst[0] * log10(P) + c->satConst[1];
    const double h = c->Cp[m] * T + c->eta[m];
    const double s = (c->Cp[m] / c->gamma[m]) * log10(pow(T, c->gamma[m]) / pow(P + c->pInf[m], c->gamma[m] - 1)) + et[m];
    return h - T * s;
}

/* chemical residual (DP/chemRlx.cu:52-76). */
void chem_residual(const fg_case *c, int pm, double *x, double rm, double re, double *r0,
                   double *r1, double *r2) {
    double s1 = 0, s2 = 0, s3 = 0;
    for (int m = 0; m < 2; m++)
        if (m != pm) {
            s1 = x[m];
            s2 = x[m] * x[m + 2];
            s3 = x[m] * x[m + 2] * x[m + 4];
        }
    x[pm] = 1 - s1;
    x[pm + 2] = (rm - s2) / x[pm];
    x[pm + 4] = (re - s3) / (x[pm] * x[pm + 2]);
    double p[2], T[2], g[2];
    for (int m = 0; m < 2; m++) {
        p[m] = eqos(c, m, 0, x[m + 2], x[m + 4]);
        T[m] = eqos(c, m, 1, x[m + 2], x[m + 4]);
        g[m] = gibbs(c, m, p[m], T[m]);
    }
    *r0 = p[0] - p[1];
    *r1 = T[0] - T[1];
    *r2 = g[0] - g[1];
}

/* step-halving safeguard (DP/chemRlx.cu:139-162); urf arrives as float as in the reference. */
void chem_check_update(const fg_case *c, double xOld, double *x, double dx, int i, float urf,
                       int *abortFlag, double rho) {
    if (i == 0 || i == 1) {
        if (x[i] < 0) { while (x[i] < c->chemLimit && urf > 0.0005) { urf = urf / 2; x[i] = xOld - urf * dx; } }
        if (x[i] > 1) { while (x[i] > 1.0 - c->chemLimit && urf > 0.0005) { urf = urf / 2; x[i] = xOld - urf * dx; } }
        if (x[i] < 0) *abortFlag = 1;
        if (x[i] > 1) *abortFlag = 1;
    } else if (i == 2 || i == 3) {
        double ar = x[i - 2] * x[i];
        if (x[i] < 0) { while (x[i] < 0 && urf > 0.0005) { urf = urf / 2; x[i] = xOld - urf * dx; } }
        if (ar > rho) { while (ar > rho && urf > 0.0005) { urf = urf / 2; x[i] = xOld - urf * dx; ar = x[i - 2] * x[i]; } }
        if (x[i] < 0) *abortFlag = 1;
        if (ar > rho) *abortFlag = 1;
    }
}

int chem_relax_cell(const fg_case *c, double *U, int *itrOut) {
    /* initialisation (DP/chemRlx.cu:4-36) */
    double x[6], ax[6];
    x[0] = fmin(fmax(c->avfMin / 100, U[0]), 1 - c->avfMin / 100);
    x[1] = 1 - x[0];
    x[2] = U[1] / x[0];
    x[3] = U[2] / x[1];
    x[4] = U[6] / (x[0] * x[2]);
    x[5] = U[7] / (x[1] * x[3]);
    for (int i = 0; i < 6; i++) ax[i] = x[i];
    const double rm = x[0] * x[2] + x[1] * x[3];
    const double u = U[3] / rm, v = U[4] / rm, w = U[5] / rm;
    const double re = U[8] - 0.5 * rm * (u * u + v * v + w * w);
    int pm = 0;
    {
        double mx = -1.0;
        for (int m = 0; m < 2; m++)
            if (x[m] > mx) { mx = x[m]; pm = m; }
    }
    float minRes = 1e9f;
    int abortFlag = 0, itr = 0, aborted = 0;
    bool conv = false;
    double res[3], jac[3][3], inv[3][3];
    while (!conv) {
        itr++;
        chem_residual(c, pm, x, rm, re, &res[0], &res[1], &res[2]);
        /* finite-difference Jacobian (DP/chemRlx.cu:78-101) */
        double e[3], rdf[3][3];
        int iv = 0;
        for (int j = 0; j < 6; j++)
            if (j != pm && j != pm + 2 && j != pm + 4) {
                e[iv] = fabs(x[j]) < 1e-9 ? 1e-10 : 1.e-5 * x[j];
                x[j] += e[iv];
                chem_residual(c, pm, x, rm, re, &rdf[0][iv], &rdf[1][iv], &rdf[2][iv]);
                x[j] -= e[iv];
                iv++;
            }
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                jac[i][j] = (rdf[i][j] - res[i]) / e[j];
                if (std::isnan(jac[i][j])) abortFlag = 1;
            }
        /* 3x3 inverse (DP/chemRlx.cu:103-123) */
        const double det = jac[0][0] * (jac[1][1] * jac[2][2] - jac[1][2] * jac[2][1]) -
                           jac[0][1] * (jac[1][0] * jac[2][2] - jac[1][2] * jac[2][0]) +
                           jac[0][2] * (jac[1][0] * jac[2][1] - jac[1][1] * jac[2][0]);
        if (det == 0) abortFlag = 1;
        const double id = 1.0 / det;
        inv[0][0] = id * (jac[1][1] * jac[2][2] - jac[1][2] * jac[2][1]);
        inv[0][1] = -id * (jac[0][1] * jac[2][2] - jac[0][2] * jac[2][1]);
        inv[0][2] = id * (jac[0][1] * jac[1][2] - jac[0][2] * jac[1][1]);
        inv[1][0] = -id * (jac[1][0] * jac[2][2] - jac[1][2] * jac[2][0]);
        inv[1][1] = id * (jac[0][0] * jac[2][2] - jac[0][2] * jac[2][0]);
        inv[1][2] = -id * (jac[0][0] * jac[1][2] - jac[0][2] * jac[1][0]);
        inv[2][0] = id * (jac[1][0] * jac[2][1] - jac[1][1] * jac[2][0]);
        inv[2][1] = -id * (jac[0][0] * jac[2][1] - jac[0][1] * jac[2][0]);
        inv[2][2] = id * (jac[0][0] * jac[1][1] - jac[0][1] * jac[1][0]);
        /* best-iterate bookkeeping (DP/chemRlx.cu:125-137) */
        if (abortFlag == 0 && x[0] > 0.0 && x[0] < 1.0 && x[1] > 0.0 && x[1] < 1.0 && x[2] > 0.0 && x[3] > 0.0) {
            const float chk = sqrt(res[0] * res[0] + res[1] * res[1] + res[2] * res[2]);
            if (chk < minRes) {
                minRes = chk;
                for (int i = 0; i < 6; i++) ax[i] = x[i];
            }
        }
        /* Newton update with safeguards (DP/chemRlx.cu:164-193); the safeguard's abort flag
         * is local to this update, as in the reference (passed by value there). */
        int abortLocal = abortFlag;
        iv = 0;
        for (int i = 0; i < 6; i++)
            if (i != pm && i != pm + 2 && i != pm + 4) {
                double dx = 0;
                for (int j = 0; j < 3; j++) dx += inv[iv][j] * res[j];
                x[i] = x[i] - c->chemUrf * dx;
                chem_check_update(c, x[i] + c->chemUrf * dx, x, dx, i, (float)c->chemUrf, &abortLocal, rm);
                iv++;
            }
        int chk = 0;
        for (int j = 0; j < 3; j++)
            if (fabs(res[j]) > 1.e-1) chk += 1;
        if (chk == 0) conv = true;
        if (abortLocal == 1 || itr > c->chemItrMax) {
            for (int i = 0; i < 6; i++) x[i] = ax[i];
            conv = true;
            aborted = 1;
        }
    }
    /* write back (DP/chemRlx.cu:195-215) */
    double s1 = 0, s2 = 0, s3 = 0;
    for (int m = 0; m < 2; m++)
        if (m != pm) {
            s1 = x[m];
            s2 = x[m] * x[m + 2];
            s3 = x[m] * x[m + 2] * x[m + 4];
        }
    x[pm] = 1 - s1;
    x[pm + 2] = (rm - s2) / x[pm];
    x[pm + 4] = (re - s3) / (x[pm] * x[pm + 2]);
    U[0] = fmin(fmax(c->avfMin / 100, x[0]), 1 - c->avfMin / 100);
    U[1] = x[0] * x[2];
    U[2] = x[1] * x[3];
    U[6] = x[0] * x[2] * x[4];
    U[7] = x[1] * x[3] * x[5];
    U[9] = x[1] * x[3];
    if (itrOut) *itrOut = itr;
    return aborted;
}

/* ---------------- mesh helpers: per-cell face lists in increasing face order ---------------- */

struct CellFaces {
    std::vector<int> start, face, side;
};

void build_cell_faces(const fg_mesh_view *m, CellFaces &cf) {
    const int nE = m->nElem, nF = m->nFcs;
    cf.start.assign(nE + 1, 0);
    for (int f = 0; f < nF; f++) {
        cf.start[m->fc2el[2 * f] + 1]++;
        if (m->boundCond[f] == 0) cf.start[m->fc2el[2 * f + 1] + 1]++;
    }
    for (int i = 0; i < nE; i++) cf.start[i + 1] += cf.start[i];
    cf.face.resize(cf.start[nE]);
    cf.side.resize(cf.start[nE]);
    std::vector<int> pos(cf.start.begin(), cf.start.end() - 1);
    for (int f = 0; f < nF; f++) {
        int o = m->fc2el[2 * f];
        cf.face[pos[o]] = f; cf.side[pos[o]] = 0; pos[o]++;
        if (m->boundCond[f] == 0) {
            int nb = m->fc2el[2 * f + 1];
            cf.face[pos[nb]] = f; cf.side[pos[nb]] = 1; pos[nb]++;
        }
    }
}

} // namespace

/* ======================================================================= C ABI */

struct orc_work_ext {
    orc_work w;
    int nElem, nFcs;
    const void *meshKey;
    CellFaces cf;
    std::vector<double> fbuf;   /* per-face side contributions, nFcs*20 */
};

extern "C" {

int orc_set_threads(int n) {
    int old = g_threads;
    g_threads = n < 1 ? 1 : n;
    return old;
}

orc_work *orc_work_new(int nElem, int nFcs) {
    orc_work_ext *e = new orc_work_ext();
    e->nElem = nElem;
    e->nFcs = nFcs;
    e->meshKey = nullptr;
    orc_work &w = e->w;
    w.U0 = (double *)calloc((size_t)nElem * 10, sizeof(double));
    w.primF = (double *)calloc((size_t)nFcs * 20, sizeof(double));
    w.grad = (double *)calloc((size_t)nElem * 30, sizeof(double));
    w.wMin = (double *)calloc((size_t)nElem * 10, sizeof(double));
    w.wMax = (double *)calloc((size_t)nElem * 10, sizeof(double));
    w.ext = (double *)calloc((size_t)nFcs * 20, sizeof(double));
    w.theta = (double *)calloc((size_t)nElem * 10, sizeof(double));
    w.RHS = (double *)calloc((size_t)nElem * 10, sizeof(double));
    w.signal = (double *)calloc((size_t)nElem, sizeof(double));
    return &e->w;
}

void orc_work_free(orc_work *w) {
    if (!w) return;
    free(w->U0); free(w->primF); free(w->grad); free(w->wMin); free(w->wMax);
    free(w->ext); free(w->theta); free(w->RHS); free(w->signal);
    delete reinterpret_cast<orc_work_ext *>(w);
}

static orc_work_ext *ext_of(orc_work *w, const fg_mesh_view *m) {
    orc_work_ext *e = reinterpret_cast<orc_work_ext *>(w);
    if (e->meshKey != (const void *)m->fc2el) {
        build_cell_faces(m, e->cf);
        e->fbuf.assign((size_t)m->nFcs * 20, 0.0);
        e->meshKey = (const void *)m->fc2el;
    }
    return e;
}

double orc_eqos(const fg_case *c, int imat, int id, double v1, double v2) { return eqos(c, imat, id, v1, v2); }
void orc_cons2prim(const fg_case *c, const double *U, double *sol) { cons2prim(c, U, sol); }
void orc_prim2cons(const fg_case *c, const double *prim, double *cons) { prim2cons(c, prim, cons); }
void orc_wave_speeds(const fg_case *c, const double *n, const double *t1, const double *t2,
                     const double *solL, const double *solR, double *cOut, double *uL, double *uR) {
    wave_speeds(c, n, t1, t2, solL, solR, cOut, uL, uR);
}
void orc_bc_values(const fg_case *c, const double *n, const double *t1, const double *t2, double *sol, int bc) {
    bc_values(c, n, t1, t2, sol, bc);
}
void orc_face_flux(const fg_case *c, const double *n, const double *t1, const double *t2, double area,
                   int bc, const double *solL, const double *solR, const double *UL, const double *UR,
                   double *out) {
    double sR[10];
    for (int v = 0; v < 10; v++) sR[v] = (bc == 0) ? solR[v] : solL[v];
    if (bc != 0) bc_values(c, n, t1, t2, sR, bc);
    face_flux(c, n, t1, t2, area, bc, solL, sR, UL, (bc == 0) ? UR : UL, out);
}
void orc_star_region(const fg_case *c, const double *sol, const double *uLcl, double SK, double SS,
                     const double *n, const double *t1, const double *t2, const double *consF_in, double *out) {
    double unc[3], vS[10] = {0}, cf[10];
    for (int v = 0; v < 10; v++) cf[v] = consF_in[v];
    star_region(c, sol, uLcl, SK, SS, n, t1, t2, unc, vS, cf);
    vS[6] = 0;
    vS[7] = 0;
    for (int d = 0; d < 3; d++) out[d] = unc[d];
    for (int v = 0; v < 10; v++) out[3 + v] = vS[v];
    for (int v = 0; v < 10; v++) out[13 + v] = cf[v];
}
void orc_adv_flux(const fg_case *c, const double *prim, const double *n, const double *uNC, double areL,
                  double areG, double *out) {
    adv_flux(c, prim, out, n, uNC, areL, areG);
}
void orc_flux_source(const fg_case *c, const double *uNC, const double *UL, const double *UR, const double *n,
                     double *out) {
    flux_source(c, uNC, UL, UR, n, out);
}
double orc_eddy_visc(const double *g, double volume) {
    return eddy_visc(g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], g[8], volume);
}
double orc_saturation_temp(const fg_case *c, double P, double T, double urf) { return saturation_temp(c, P, T, urf); }
int orc_therm_relax_cell(const fg_case *c, double *U, int *itrOut) { return therm_relax_cell(c, U, itrOut); }
int orc_chem_relax_cell(const fg_case *c, double *U, int *itrOut) { return chem_relax_cell(c, U, itrOut); }

/* convert2PrimVec (DP/computePrimVec.cu:38-80) */
void orc_prim(const fg_case *c, const fg_mesh_view *m, const double *U, orc_work *w) {
    const int nF = m->nFcs;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int f = 0; f < nF; f++) {
        const int bc = m->boundCond[f];
        const int id = (bc == 0);
        double *s0 = w->primF + (size_t)f * 20, *s1 = s0 + 10;
        cons2prim(c, U + (size_t)m->fc2el[2 * f] * 10, s0);
        cons2prim(c, U + (size_t)m->fc2el[2 * f + id] * 10, s1);
        if (bc != 0) bc_values(c, m->n + 3 * f, m->nt1 + 3 * f, m->nt2 + 3 * f, s1, bc);
    }
}

/* initializeLimiters + initializeGrad + greenGauss (DP/computeGrad.cu:3-91) */
void orc_grad(const fg_case *, const fg_mesh_view *m, orc_work *w) {
    orc_work_ext *e = ext_of(w, m);
    const int nE = m->nElem;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int cI = 0; cI < nE; cI++) {
        double *g = w->grad + (size_t)cI * 30;
        double *mn = w->wMin + (size_t)cI * 10, *mx = w->wMax + (size_t)cI * 10;
        for (int k = 0; k < 30; k++) g[k] = 0.0;
        for (int v = 0; v < 10; v++) { mn[v] = 1e12; mx[v] = -1e12; }
        for (int q = e->cf.start[cI]; q < e->cf.start[cI + 1]; q++) {
            const int f = e->cf.face[q], side = e->cf.side[q];
            const double *pL = w->primF + (size_t)f * 20, *pR = pL + 10;
            const double *nv = m->n + 3 * f;
            const double A = m->area[f], V = m->volume[cI];
            for (int v = 0; v < 10; v++) {
                const double sL = pL[v], sR = pR[v];
                const double other = (side == 0) ? sR : sL;
                if (mx[v] < other) mx[v] = other;     /* atomic max / min keep the extreme */
                if (mn[v] > other) mn[v] = other;
                for (int d = 0; d < 3; d++) {
                    if (side == 0) g[v * 3 + d] += ((sL + sR) / 2) * nv[d] * A / V;
                    else g[v * 3 + d] += -((sL + sR) / 2) * nv[d] * A / V;
                }
            }
        }
    }
}

/* initializeTheta + computeLimiter + updateFaces (DP/computeFaceValues.cu:4-113) */
void orc_limiter(const fg_case *c, const fg_mesh_view *m, orc_work *w) {
    orc_work_ext *e = ext_of(w, m);
    const int nE = m->nElem, nF = m->nFcs;
    /* extension and per-side limiter value, face-parallel */
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int f = 0; f < nF; f++) {
        const int bc = m->boundCond[f];
        for (int id = 0; id < 2; id++) {
            if (!(id != 1 || bc == 0)) continue;
            const int cI = m->fc2el[2 * f + id];
            const double *sh = (id == 1 && m->nbShift) ? m->nbShift + 3 * f : nullptr;
            const double xf = m->fcCenter[3 * f + 0] + (sh ? sh[0] : 0.0);
            const double yf = m->fcCenter[3 * f + 1] + (sh ? sh[1] : 0.0);
            const double zf = m->fcCenter[3 * f + 2] + (sh ? sh[2] : 0.0);
            const double xc = m->cellCenter[3 * cI + 0], yc = m->cellCenter[3 * cI + 1], zc = m->cellCenter[3 * cI + 2];
            for (int v = 0; v < 10; v++) {
                const double sol = w->primF[(size_t)f * 20 + id * 10 + v];
                const double *g = w->grad + (size_t)cI * 30 + v * 3;
                const double wun = sol + (xf - xc) * g[0] + (yf - yc) * g[1] + (zf - zc) * g[2];
                w->ext[(size_t)f * 20 + id * 10 + v] = (xf - xc) * g[0] + (yf - yc) * g[1] + (zf - zc) * g[2];
                (void)wun;
            }
        }
    }
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int cI = 0; cI < nE; cI++) {
        double *th = w->theta + (size_t)cI * 10;
        for (int v = 0; v < 10; v++) th[v] = 1e9;
        for (int q = e->cf.start[cI]; q < e->cf.start[cI + 1]; q++) {
            const int f = e->cf.face[q], id = e->cf.side[q];
            const double *sh = (id == 1 && m->nbShift) ? m->nbShift + 3 * f : nullptr;
            const double xf = m->fcCenter[3 * f + 0] + (sh ? sh[0] : 0.0);
            const double yf = m->fcCenter[3 * f + 1] + (sh ? sh[1] : 0.0);
            const double zf = m->fcCenter[3 * f + 2] + (sh ? sh[2] : 0.0);
            const double xc = m->cellCenter[3 * cI + 0], yc = m->cellCenter[3 * cI + 1], zc = m->cellCenter[3 * cI + 2];
            for (int v = 0; v < 10; v++) {
                const double sol = w->primF[(size_t)f * 20 + id * 10 + v];
                const double *g = w->grad + (size_t)cI * 30 + v * 3;
                const double wun = sol + (xf - xc) * g[0] + (yf - yc) * g[1] + (zf - zc) * g[2];
                const double wmax = w->wMax[(size_t)cI * 10 + v], wmin = w->wMin[(size_t)cI * 10 + v];
                double phi;
                if (wun - sol != 0) {
                    if (c->limiter == 1) {   /* van Albada-type limiter function (extension) */
                        const double r = (wun > sol) ? (wmax - sol) / (wun - sol) : (wmin - sol) / (wun - sol);
                        phi = (r * r + r) / (r * r + 1);
                    } else {
                        phi = (wun > sol) ? (wmax - sol) / (2 * (wun - sol)) : (wmin - sol) / (2 * (wun - sol));
                    }
                } else {
                    phi = 1;
                }
                const double tt = fmax(0, fmin(phi, 1));
                if (th[v] > tt) th[v] = tt;   /* atomic min */
            }
        }
    }
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int f = 0; f < nF; f++) {
        const int bc = m->boundCond[f];
        for (int id = 0; id < 2; id++) {
            if (!(id != 1 || bc == 0)) continue;
            const int cI = m->fc2el[2 * f + id];
            for (int v = 0; v < 10; v++)
                w->primF[(size_t)f * 20 + id * 10 + v] += w->theta[(size_t)cI * 10 + v] * w->ext[(size_t)f * 20 + id * 10 + v];
        }
    }
}

/* initializeRHS + computeFlux + computeViscousStresses (DP/computeRHS.cu:12-146,
 * DP/computeViscousStresses.cu:66-174), accumulated per cell in face order. */
void orc_rhs(const fg_case *c, const fg_mesh_view *m, const double *U, orc_work *w) {
    orc_work_ext *e = ext_of(w, m);
    const int nE = m->nElem, nF = m->nFcs;
    double *fb = e->fbuf.data();
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1 && c->viscFlag != 1) break;
#pragma omp parallel for num_threads(g_threads) schedule(static)
        for (int f = 0; f < nF; f++) {
            const int bc = m->boundCond[f];
            const int id = (bc == 0);
            const int o = m->fc2el[2 * f], nb = m->fc2el[2 * f + id];
            const double *n = m->n + 3 * f, *t1 = m->nt1 + 3 * f, *t2 = m->nt2 + 3 * f;
            const double *pf = w->primF + (size_t)f * 20;
            if (pass == 0) {
                double sL[10], sR[10];
                for (int v = 0; v < 10; v++) { sL[v] = pf[v]; sR[v] = pf[id * 10 + v]; }
                if (bc != 0) bc_values(c, n, t1, t2, sR, bc);
                face_flux(c, n, t1, t2, m->area[f], bc, sL, sR, U + (size_t)o * 10, U + (size_t)nb * 10, fb + (size_t)f * 20);
            } else {
                const double vavg = (m->volume[o] + m->volume[nb]) / 2;
                viscous_face(c, w->grad + (size_t)o * 30, w->grad + (size_t)nb * 30, vavg, pf, pf + 10, n,
                             m->area[f], bc, U + (size_t)o * 10, U + (size_t)nb * 10, fb + (size_t)f * 20);
            }
        }
#pragma omp parallel for num_threads(g_threads) schedule(static)
        for (int cI = 0; cI < nE; cI++) {
            double *R = w->RHS + (size_t)cI * 10;
            if (pass == 0)
                for (int v = 0; v < 10; v++) R[v] = 0.0;
            for (int q = e->cf.start[cI]; q < e->cf.start[cI + 1]; q++) {
                const double *src = fb + (size_t)e->cf.face[q] * 20 + e->cf.side[q] * 10;
                if (pass == 0) {
                    for (int v = 0; v < 10; v++) R[v] += src[v];
                } else {
                    /* the viscous kernel only touches momentum and energy */
                    R[3] += src[3]; R[4] += src[4]; R[5] += src[5]; R[8] += src[8];
                }
            }
        }
    }
}

void orc_residual(const fg_case *c, const fg_mesh_view *m, const double *U, orc_work *w) {
    orc_prim(c, m, U, w);
    orc_grad(c, m, w);
    orc_limiter(c, m, w);
    orc_rhs(c, m, U, w);
}

/* computeLocalSignalSum + computeLocalCFL (DP/computeTimeStep.cu:97-159): returns the
 * minimum over cells of pow(V, 0.3333)/s; w->signal holds s per cell. */
double orc_timestep_min(const fg_case *c, const fg_mesh_view *m, orc_work *w) {
    orc_work_ext *e = ext_of(w, m);
    const int nE = m->nElem, nF = m->nFcs;
    double *fb = e->fbuf.data();
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int f = 0; f < nF; f++) {
        const double *n = m->n + 3 * f, *t1 = m->nt1 + 3 * f, *t2 = m->nt2 + 3 * f;
        const double cl = face_max_signal(c, w->primF + (size_t)f * 20, n, t1, t2);
        double cr = 0;
        if (m->boundCond[f] == 0) cr = face_max_signal(c, w->primF + (size_t)f * 20 + 10, n, t1, t2);
        fb[f] = fmax(cl, cr);
    }
    double gmin = 1e12;
#pragma omp parallel for num_threads(g_threads) schedule(static) reduction(min : gmin)
    for (int cI = 0; cI < nE; cI++) {
        double s = -1e9;
        for (int q = e->cf.start[cI]; q < e->cf.start[cI + 1]; q++) {
            const double v = fb[e->cf.face[q]];
            if (s < v) s = v;
        }
        w->signal[cI] = s;
        const double val = pow(m->volume[cI], 0.3333) / s;
        gmin = fmin(gmin, val);
    }
    return gmin;
}

void orc_init_rk(const fg_mesh_view *m, const double *U, orc_work *w) {
    memcpy(w->U0, U, sizeof(double) * 10 * (size_t)m->nElem);
}

/* rk3stage1/2/3 and rungeKutta (DP/update.cu:19-103) */
void orc_update(const fg_case *c, const fg_mesh_view *m, int irk, double dt, double *U, orc_work *w) {
    const int nE = m->nElem;
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int cI = 0; cI < nE; cI++) {
        const double V = m->volume[cI];
        for (int v = 0; v < 10; v++) {
            /* only the last of the three neglect assignments survives (DP/update.cu:26-28) */
            const int neglect = (v == 5 && c->neglectZ == 1);
            const size_t k = (size_t)cI * 10 + v;
            const double R = w->RHS[k];
            if (c->rkSteps == 1) {
                U[k] = (1 - neglect) * (U[k] + dt * (1.0 / V) * R);
            } else if (irk == 0) {
                U[k] = (1 - neglect) * (w->U0[k] + dt * (1.0 / V) * R);
            } else if (irk == 1) {
                U[k] = (1 - neglect) * ((3.0 / 4.0) * w->U0[k] + (1.0 / 4.0) * U[k] + (1.0 / 4.0) * dt * (1.0 / V) * R);
            } else {
                U[k] = (1 - neglect) * ((1.0 / 3.0) * w->U0[k] + (2.0 / 3.0) * U[k] + (2.0 / 3.0) * dt * (1.0 / V) * R);
            }
        }
    }
}

/* relaxation (DP/relaxation.cu:46-114) */
void orc_relaxation(const fg_case *c, const fg_mesh_view *m, double *U, fg_relax_stats *st) {
    const int nE = m->nElem;
    int nT = 0, nC = 0, nA = 0, nI = 0;
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 256) reduction(+ : nT, nC, nA, nI)
    for (int cI = 0; cI < nE; cI++) {
        double *u = U + (size_t)cI * 10;
        int chem = 0;
        if (c->chemFlag == 1) {
            const double avf = fmin(fmax(c->avfMin / 100, u[0]), 1 - c->avfMin / 100);
            const double rho = u[1] / avf;
            const double enr = u[6] / (avf * rho);
            const double tl = eqos(c, 0, 1, rho, enr);
            const double pl = eqos(c, 0, 0, rho, enr);
            const double ts = saturation_temp(c, pl, tl, c->satTempUrf);
            chem = (tl > ts && avf > c->chemLimit);
        }
        /* the reference runs thermalRlx on the therm list, then chemRlx on the chem list;
         * each cell is in exactly one list and cells are independent */
        int it = 0;
        if (chem) { nA += chem_relax_cell(c, u, &it); nC++; }
        else { nA += therm_relax_cell(c, u, &it); nT++; }
        nI += it;
    }
    if (st) { st->nTherm = nT; st->nChem = nC; st->nAbort = nA; st->nIter = nI; st->nSurrogate = 0; st->nFallback = 0; st->nPolish = 0; }
}

/* integrateConsVar + consCalc (DP/consCalc.cu:3-60); fixed 4096-cell chunks so the result
 * does not depend on the thread count. */
double orc_cons_calc(const fg_mesh_view *m, int ivar, const double *U) {
    const int nE = m->nElem, CH = 4096, nCh = (nE + CH - 1) / CH;
    std::vector<double> part(nCh, 0.0);
#pragma omp parallel for num_threads(g_threads) schedule(static)
    for (int k = 0; k < nCh; k++) {
        double s = 0.0;
        for (int cI = k * CH; cI < std::min(nE, (k + 1) * CH); cI++) {
            const double var = (ivar == 0) ? 1.0 - U[(size_t)cI * 10 + ivar] : U[(size_t)cI * 10 + ivar];
            s += var * m->volume[cI];
        }
        part[k] = s;
    }
    double t = 0.0;
    for (int k = 0; k < nCh; k++) t += part[k];
    return t;
}

/* explicitLoop body (DP/explicitLoop.cu:28-64) */
void orc_step(const fg_case *c, const fg_mesh_view *m, double *U, orc_work *w, double *dt,
              double *time, int *iStep, double *consOut, fg_relax_stats *rs) {
    *time += *dt;
    if (c->rkSteps > 1) orc_init_rk(m, U, w);
    for (int irk = 0; irk < c->rkSteps; irk++) {
        orc_residual(c, m, U, w);
        if (c->adaptDt == 1 && irk == 0 && (*iStep) % c->adaptDtItr == 0) {
            const double mn = orc_timestep_min(c, m, w);
            *dt = fmin(c->cfl * mn, c->maxDt);
        }
        orc_update(c, m, irk, *dt, U, w);
    }
    if (c->relaxFlag == 0) orc_relaxation(c, m, U, rs);
    if (c->consCalcFlag == 1 && (*iStep) % c->adaptDtItr == 0 && consOut)
        *consOut = orc_cons_calc(m, c->consCalcIvar, U);
    (*iStep)++;
}

} /* extern "C" */
