/*
 * ref_kat.cpp — TEST INFRASTRUCTURE ONLY.
 *
 * Host harness around the reference's own device code, compiled by g++ from the reference
 * sources where they lie (the physics headers of mulitphase Solver/doublePrecision/ and the
 * kernel-only files thermRlx.cu, chemRlx.cu, computeViscousStresses.cu) with the stubs in
 * refshim/.  Built by oracle/build_ref.py into oracle/_ref/libref_host.so; it exists only
 * where the reference tree is present.  Each entry point runs one reference function on the
 * given inputs so that tests and tests/golden/make_golden.py can compare the oracle's
 * restatement against the reference bit for bit (same host compiler, same libm).
 */
#include "strdata.h"
#include "eqos.h"
#include "rotateVector.h"
#include "bc.h"
#include "cons2prim.h"
#include "waveSpeeds.h"
#include "flux.h"
#include "starRegion.h"
#include "prim2cons.h"

#include "../include/fooskagpu.h"

uint3 threadIdx, blockIdx;
dim3 blockDim, gridDim;

__global__ void thermalRlx(INPUT *d_input, int nElem, int itrMax, double urf, int *idTherm2iel, double *consVec);
__global__ void chemRlx(INPUT *d_input, int nElem, int itrMax, double urf, int *idiChem2iel, double *consVec);

static void to_input(const fg_case *c, INPUT *in) {
    memset(in, 0, sizeof(*in));
#define CP(f) in->f = c->f
    CP(dt); CP(cfl); CP(adaptDt); CP(adaptDtItr); CP(maxDt); CP(avfMin); CP(rkSteps); CP(finalTime);
    CP(exportTime); CP(restartStep); CP(restartFlag); CP(neglectX); CP(neglectY); CP(neglectZ);
    CP(nMaterials); CP(NEQ); CP(scale); CP(viscFlag); CP(turbulence); CP(woodsFlag);
    CP(thermFntRlxFlag); CP(thermRlxRate); CP(thermUrf); CP(thermItrMax); CP(chemFlag);
    CP(chemFntRlxFlag); CP(chemRlxRate); CP(chemUrf); CP(chemItrMax); CP(chemCondesation);
    CP(chemLimit); CP(consCalcFlag); CP(consCalcIvar); CP(satTempUrf);
#undef CP
    for (int k = 0; k < 2; k++) {
        in->pInf[k] = c->pInf[k];
        in->gamma[k] = c->gamma[k];
        in->Cp[k] = c->Cp[k];
        in->eta[k] = c->eta[k];
        in->satConst[k] = c->satConst[k];
        in->dynVisc[k] = c->dynVisc[k];
        in->heatCoef[k] = c->heatCoef[k];
        in->Pr[k] = c->Pr[k];
    }
}

static void one_thread() {
    threadIdx.x = threadIdx.y = threadIdx.z = 0;
    blockIdx.x = blockIdx.y = blockIdx.z = 0;
    blockDim.x = 1; blockDim.y = 1; blockDim.z = 1;
    gridDim.x = 1; gridDim.y = 1; gridDim.z = 1;
}

extern "C" {

double refkat_eqos(const fg_case *c, int imat, int id, double v1, double v2) {
    INPUT in;
    to_input(c, &in);
    return eqos(&in, imat, id, v1, v2);
}

void refkat_cons2prim(const fg_case *c, const double *U, double *sol) {
    INPUT in;
    to_input(c, &in);
    double u[10], s[10];
    for (int i = 0; i < 10; i++) u[i] = U[i];
    cons2prim(&in, u, s);
    for (int i = 0; i < 10; i++) sol[i] = s[i];
}

void refkat_prim2cons(const fg_case *c, const double *prim, double *cons) {
    INPUT in;
    to_input(c, &in);
    double p[10];
    for (int i = 0; i < 10; i++) p[i] = prim[i];
    prim2cons(&in, p, cons);
}

void refkat_wave_speeds(const fg_case *c, const double *n, const double *t1, const double *t2, const double *sL,
                        const double *sR, double *cOut, double *uL, double *uR) {
    INPUT in;
    to_input(c, &in);
    double N[3], T1[3], T2[3], L[10], R[10], cc[3], ul[3], ur[3];
    for (int d = 0; d < 3; d++) { N[d] = n[d]; T1[d] = t1[d]; T2[d] = t2[d]; }
    for (int v = 0; v < 10; v++) { L[v] = sL[v]; R[v] = sR[v]; }
    waveSpeeds(&in, N, T1, T2, L, R, cc, ul, ur);
    for (int d = 0; d < 3; d++) { cOut[d] = cc[d]; uL[d] = ul[d]; uR[d] = ur[d]; }
}

void refkat_bc_values(const fg_case *c, const double *n, const double *t1, const double *t2, double *sol, int bc) {
    INPUT in;
    to_input(c, &in);
    double N[3], T1[3], T2[3], S[10];
    for (int d = 0; d < 3; d++) { N[d] = n[d]; T1[d] = t1[d]; T2[d] = t2[d]; }
    for (int v = 0; v < 10; v++) S[v] = sol[v];
    bcValues(&in, N, T1, T2, S, bc);
    for (int v = 0; v < 10; v++) sol[v] = S[v];
}

/* starRegion (DP/starRegion.h): out = [uNonCons(3), vecS(10) with 6,7 zeroed, consF(10)] */
void refkat_star_region(const fg_case *c, const double *sol, const double *uLcl, double SK, double SS,
                        const double *n, const double *t1, const double *t2, const double *consF_in, double *out) {
    INPUT in;
    to_input(c, &in);
    double S[10], ul[3], N[3], T1[3], T2[3], unc[3], vS[10] = {0}, cf[10];
    for (int v = 0; v < 10; v++) { S[v] = sol[v]; cf[v] = consF_in[v]; }
    for (int d = 0; d < 3; d++) { ul[d] = uLcl[d]; N[d] = n[d]; T1[d] = t1[d]; T2[d] = t2[d]; }
    starRegion(&in, S, ul, SK, SS, N, T1, T2, unc, vS, cf);
    vS[6] = 0; vS[7] = 0;
    for (int d = 0; d < 3; d++) out[d] = unc[d];
    for (int v = 0; v < 10; v++) out[3 + v] = vS[v];
    for (int v = 0; v < 10; v++) out[13 + v] = cf[v];
}

/* flux (DP/flux.h:32-91): fluxAdv[10] */
void refkat_flux(const fg_case *c, const double *prim, const double *n, const double *uNC, double areL,
                 double areG, double *out) {
    INPUT in;
    to_input(c, &in);
    double P[10], N[3], U[3], F[15] = {0};
    for (int v = 0; v < 10; v++) P[v] = prim[v];
    for (int d = 0; d < 3; d++) { N[d] = n[d]; U[d] = uNC[d]; }
    flux(&in, 0, P, F, N, U, areL, areG);
    for (int v = 0; v < 10; v++) out[v] = F[v];
}

/* fluxSource (DP/flux.h:1-30): fnc[6] */
void refkat_flux_source(const fg_case *c, const double *uNC, const double *UL, const double *UR, const double *n,
                        double *out) {
    INPUT in;
    to_input(c, &in);
    double ul[10], ur[10], N[3], fnc[6];
    for (int v = 0; v < 10; v++) { ul[v] = UL[v]; ur[v] = UR[v]; }
    for (int d = 0; d < 3; d++) N[d] = n[d];
    fluxSource(&in, (double *)uNC, ul, ur, N, fnc);
    for (int k = 0; k < 6; k++) out[k] = fnc[k];
}

/* computeViscousStresses (DP/computeViscousStresses.cu:66) run on a single face.
 * primF[20] (slots 0,1), gradO[30], gradN[30], vol[2], bc; RHS[20] = owner, neighbour. */
void refkat_viscous_face(const fg_case *c, const double *primF, const double *gradO, const double *gradN,
                         const double *n, double area, const double *vol, int bc, double *RHS) {
    INPUT in;
    to_input(c, &in);
    int fc2el[2] = {0, bc == 0 ? 1 : -1};
    int bcs[1] = {bc};
    double pf[20], grad[60], N[3], A[1] = {area}, V[2] = {vol[0], vol[1]};
    for (int i = 0; i < 20; i++) { pf[i] = primF[i]; RHS[i] = 0.0; }
    for (int i = 0; i < 30; i++) { grad[i] = gradO[i]; grad[30 + i] = gradN[i]; }
    for (int d = 0; d < 3; d++) N[d] = n[d];
    one_thread();
    computeViscousStresses(&in, 1, fc2el, bcs, pf, grad, N, A, V, RHS);
}

void refkat_therm_cell(const fg_case *c, double *U) {
    INPUT in;
    to_input(c, &in);
    int id[1] = {0};
    one_thread();
    thermalRlx(&in, 1, in.thermItrMax, in.thermUrf, id, U);
}

void refkat_chem_cell(const fg_case *c, double *U) {
    INPUT in;
    to_input(c, &in);
    int id[1] = {0};
    one_thread();
    chemRlx(&in, 1, in.chemItrMax, in.chemUrf, id, U);
}

}  /* extern "C" */
