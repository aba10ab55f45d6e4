/*
 * oracle.h — TEST INFRASTRUCTURE ONLY.  CPU FP64 restatement of the reference FooskaGPU
 * double-precision solver's per-stage residual path (mulitphase Solver/doublePrecision/).
 *
 * The oracle is the checker: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference leg call it.  The product path never does.
 *
 * Semantics follow the reference kernels run by one thread: every face loop visits faces in
 * increasing index order and accumulates into cells in that order (the reference accumulates
 * with atomics in nondeterministic order; this is one admissible serialisation of it).  The
 * OpenMP build reproduces that order exactly (per-face work in parallel, per-cell gathers over
 * faces sorted by index), so results are bitwise independent of the thread count.
 *
 * Arrays use the reference layout (DP/startDevice.cu:25-50):
 *   U[c*10+v], primF[(f*2+s)*10+v], grad[(c*10+v)*3+d], wMin/wMax/theta[c*10+v],
 *   ext[(f*2+s)*10+v], RHS[c*10+v].
 */
#ifndef FG_ORACLE_H
#define FG_ORACLE_H

#include "../include/fooskagpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_work {
    double *U0;      /* nElem*10  */
    double *primF;   /* nFcs*20   */
    double *grad;    /* nElem*30  */
    double *wMin;    /* nElem*10  */
    double *wMax;    /* nElem*10  */
    double *ext;     /* nFcs*20   */
    double *theta;   /* nElem*10  */
    double *RHS;     /* nElem*10  */
    double *signal;  /* nElem     */
} orc_work;

/* Allocate / free a work set for a mesh. */
orc_work *orc_work_new(int nElem, int nFcs);
void      orc_work_free(orc_work *w);
/* Threads used by the oracle's OpenMP loops (1 = serial).  Returns the previous value. */
int       orc_set_threads(int n);

/* --- scalar physics (for known-answer tests against the reference headers) --- */
double orc_eqos(const fg_case *c, int imat, int id, double v1, double v2);   /* DP/eqos.h:1 */
void   orc_cons2prim(const fg_case *c, const double *U, double *sol);          /* DP/cons2prim.h:2 */
void   orc_prim2cons(const fg_case *c, const double *prim, double *cons);      /* DP/prim2cons.h:2 */
void   orc_wave_speeds(const fg_case *c, const double *n, const double *t1, const double *t2,
                       const double *solL, const double *solR, double *cOut,
                       double *uL, double *uR);                                 /* DP/waveSpeeds.h:2 */
void   orc_bc_values(const fg_case *c, const double *n, const double *t1, const double *t2,
                     double *sol, int bc);                                      /* DP/bc.h:78 */
/* Flux of one face (computeFlux body, DP/computeRHS.cu:78-146) for given left/right primitive
 * states and the two cell-centre conserved states; out[0..9] owner contribution, out[10..19]
 * neighbour contribution (both already multiplied by area and sign). */
void   orc_face_flux(const fg_case *c, const double *n, const double *t1, const double *t2,
                     double area, int bc, const double *solL, const double *solR,
                     const double *UL, const double *UR, double *out);
/* Star state, advective flux and non-conservative terms (DP/starRegion.h:3-35, DP/flux.h:1-91).
 * star out[23] = uNonCons(3), vecS(10, entries 6 and 7 zero), consF(10). */
void   orc_star_region(const fg_case *c, const double *sol, const double *uLcl, double SK, double SS,
                       const double *n, const double *t1, const double *t2, const double *consF_in, double *out);
void   orc_adv_flux(const fg_case *c, const double *prim, const double *n, const double *uNC, double areL,
                    double areG, double *out);
void   orc_flux_source(const fg_case *c, const double *uNC, const double *UL, const double *UR,
                       const double *n, double *out);
double orc_eddy_visc(const double *g9, double volume);                         /* DP/computeViscousStresses.cu:3 */
double orc_saturation_temp(const fg_case *c, double P, double T, double urf);  /* DP/relaxation.cu:4 */
/* Thermal / chemical relaxation of one cell's U in place; returns 1 if the solve fell back to
 * the best iterate (abort path), 0 otherwise.  itrOut receives the iteration count. */
int    orc_therm_relax_cell(const fg_case *c, double *U, int *itrOut);          /* DP/thermRlx.cu:189 */
int    orc_chem_relax_cell(const fg_case *c, double *U, int *itrOut);           /* DP/chemRlx.cu:217 */

/* --- stage functions on a whole mesh (reference layout) --- */
void orc_prim(const fg_case *c, const fg_mesh_view *m, const double *U, orc_work *w);      /* convert2PrimVec */
void orc_grad(const fg_case *c, const fg_mesh_view *m, orc_work *w);                       /* greenGauss      */
void orc_limiter(const fg_case *c, const fg_mesh_view *m, orc_work *w);                    /* computeLimiter + updateFaces */
void orc_rhs(const fg_case *c, const fg_mesh_view *m, const double *U, orc_work *w);       /* initRHS + computeFlux + viscous */
double orc_timestep_min(const fg_case *c, const fg_mesh_view *m, orc_work *w);            /* min_c V^0.3333/s_c */
void orc_update(const fg_case *c, const fg_mesh_view *m, int irk, double dt, double *U, orc_work *w);
void orc_init_rk(const fg_mesh_view *m, const double *U, orc_work *w);
/* relaxation: returns counts in stats (nTherm, nChem, nAbort). */
void orc_relaxation(const fg_case *c, const fg_mesh_view *m, double *U, fg_relax_stats *stats);
double orc_cons_calc(const fg_mesh_view *m, int ivar, const double *U);

/* Residual of U into w->RHS (prim, grad, limiter, flux, viscous), i.e. one computeRHS. */
void orc_residual(const fg_case *c, const fg_mesh_view *m, const double *U, orc_work *w);

/* One explicitLoop step (DP/explicitLoop.cu:28-64) with the same dt / time bookkeeping.
 * *dt, *time and *iStep are read and updated.  consOut (may be NULL) receives the
 * conservation integral of consCalcIvar when it is computed this step (else unchanged). */
void orc_step(const fg_case *c, const fg_mesh_view *m, double *U, orc_work *w,
              double *dt, double *time, int *iStep, double *consOut, fg_relax_stats *rs);

#ifdef __cplusplus
}
#endif
#endif
