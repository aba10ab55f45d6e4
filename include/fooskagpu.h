/*
 * fooskagpu.h — C ABI of the B200-native explicit residual path of the FooskaGPU
 * two-phase finite-volume solver (one GPU, sm_100a).
 *
 * The reference has no plugin API: its boundary is the set of host stage functions that
 * `explicitLoop` calls (mulitphase Solver/doublePrecision/strdata.h:206-247), operating on
 * MESH / FIELD structs filled by `mainStart`.  Every entry point below replaces one of those
 * functions (cited per declaration) with an opaque handle, plain pointers and sizes, and an
 * integer status instead of `void` + printed CUDA errors.  No entry point aborts the process.
 *
 * Layout conventions at the boundary (what callers pass in and get back) are the reference's:
 *   - conserved state U: AoS double, U[cell*10 + v], cells in .neu element order,
 *     v = [alpha, alpha*rhoL, (1-alpha)*rhoG, rho*u, rho*v, rho*w,
 *          alpha*rhoL*eL, (1-alpha)*rhoG*eG, rho*E, vapour mass]   (DP/initialize.cu:45-54)
 *   - the device keeps its own renumbered SoA copy; conversion happens in fg_set_state /
 *     fg_get_state.
 */
#ifndef FOOSKAGPU_H
#define FOOSKAGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
enum fg_status_code {
    FG_OK              = 0,
    FG_ERR_ARG         = 1,  /* null pointer, out-of-range argument, size mismatch        */
    FG_ERR_IO          = 2,  /* mesh / case file missing or unreadable                     */
    FG_ERR_MESH        = 3,  /* malformed .neu, untagged open boundary, unmatched periodic */
    FG_ERR_CUDA        = 4,  /* CUDA runtime error (message via fg_last_error)             */
    FG_ERR_NAN         = 5,  /* non-finite value or non-positive density in the state      */
    FG_ERR_UNSUPPORTED = 6,  /* option the build does not implement                        */
    FG_ERR_NOMEM       = 7   /* device or host allocation failed                           */
};

/* Text of the last error raised on the calling thread (never NULL). */
const char *fg_last_error(void);

/* ---------------------------------------------------------------- case parameters
 * Field-for-field the reference's `struct INPUT` (DP/strdata.h:49-98), same names, same
 * meaning, same order.  Values are set by the caller (the reference hard-codes them in
 * DP/buildInput.cu:10-69); fg_case_default() returns those hard-coded values.
 * The trailing block holds options the reference lacks; zero selects reference behaviour. */
typedef struct fg_case {
    double  dt;
    double  cfl;
    int32_t adaptDt;
    int32_t adaptDtItr;
    double  maxDt;
    double  avfMin;

    int32_t rkSteps;
    double  finalTime;
    double  exportTime;
    int32_t restartStep;
    int32_t restartFlag;
    int32_t neglectX;
    int32_t neglectY;
    int32_t neglectZ;
    int32_t nMaterials;
    int32_t NEQ;
    double  scale;
    int32_t viscFlag;
    int32_t turbulence;
    int32_t woodsFlag;

    int32_t thermFntRlxFlag;
    double  thermRlxRate;
    double  thermUrf;
    int32_t thermItrMax;

    int32_t chemFlag;
    int32_t chemFntRlxFlag;
    double  chemRlxRate;
    double  chemUrf;
    int32_t chemItrMax;
    int32_t chemCondesation;
    double  chemLimit;

    int32_t consCalcFlag;
    int32_t consCalcIvar;

    double  satTempUrf;

    double  pInf[2];
    double  gamma[2];
    double  Cp[2];
    double  eta[2];
    double  satConst[2];
    double  dynVisc[2];
    double  heatCoef[2];
    double  Pr[2];

    /* ---- extensions (not in the reference; 0 = reference behaviour) ---- */
    int32_t relaxFlag;      /* 0: relaxation every step as the reference; 1: skip relaxation */
    /* The reference's HLLC energy star state (DP/starRegion.h:29) lacks the rho_K factor on its
     * second term, so the energy flux jumps at S* = 0 (left branch: u_L p_L (1 - 1/rho_L),
     * right branch: its mirror).  Where S* = 0 in exact arithmetic (slip walls, symmetry planes)
     * round-off picks the branch, in the reference as well.
     *   hllcEnergyFix = 1 uses the standard HLLC energy star state (continuous at S* = 0);
     *   hllcTieTol > 0 treats |S*| <= hllcTieTol * (|S_L| + |S_R|) as S* = 0 (left state), which
     *   makes two implementations with different rounding take the same branch. */
    int32_t hllcEnergyFix;
    double  hllcTieTol;
    /* heatFlux = 1 (with viscFlag = 1): Fourier heat conduction in the viscous energy flux,
     * k = cp mu / Pr with cp, Pr volume-fraction weighted at the face and mu the viscous flux's
     * (laminar + WALE), temperature gradient = mean of the two cells' liquid-phase
     * T = (p + pInf) / (cv (gamma - 1) rho) gradients; adiabatic boundary faces.  The reference
     * declares Pr and heatCoef (DP/strdata.h:96-97) but never uses them. */
    int32_t heatFlux;
    /* limiter = 1: van Albada-type limiter function phi(r) = min(1, (r^2 + r) / (r^2 + 1)) with
     * r = (w_max - w) / Delta (or w_min), in place of the reference's phi = r / 2
     * (DP/computeFaceValues.cu:73-79), the minimum over the cell's faces as before. */
    int32_t limiter;
    /* inletVelFlag = 1: the inlet ghost (bc 3) takes the velocity inletVel instead of the
     * interior velocity (the reference's inlet copies it, DP/bc.h:8-18). */
    int32_t inletVelFlag;
    /* inletStateFlag = 1: the inlet ghost's phase densities and pressures come from inletP, inletT
     * instead of the reference's fixed 11.4e5 Pa and 115.3 K (DP/bc.h:2-25). */
    int32_t inletStateFlag;
    int32_t reserved[2];
    double  inletVel[3];
    double  inletP;
    double  inletT;
    /* pressureDatum (Pa, 0 = the reference's form): the face momentum flux carries A (p_F - P0) n
     * and the cell-centre pressure term (p_C - P0) times the cell's sum of outward n A, the same
     * residual in exact arithmetic.  With P0 near the ambient pressure the reduced-precision face
     * math carries no rounding of the ambient pressure into the momentum residual (at rest:
     * none at all), where it would otherwise raise spurious velocities of order eps p / (rho c). */
    double  pressureDatum;
} fg_case;

/* Fill *c with the values the reference hard-codes in DP/buildInput.cu:10-69. */
void fg_case_default(fg_case *c);

/* ---------------------------------------------------------------- mesh
 * Replaces translator_ptw + meshConnectivity + decompose(size 1) + buildLocalMesh +
 * meshProperties (DP/translator.cu:3, DP/meshConnectivity.cu:175, DP/buildLocalMesh.cu:460,
 * DP/meshProperties.cu:139).  Reads a Gambit neutral file with the reference's grammar,
 * matches faces, computes the reference's geometry in FP64, builds the reference face order
 * (owner = lower element index) and a locality-preserving renumbering for the device. */
typedef struct fg_mesh fg_mesh;

enum fg_renumber { FG_RENUMBER_NONE = 0, FG_RENUMBER_MORTON = 1, FG_RENUMBER_RCM = 2 };

typedef struct fg_mesh_opts {
    double  scale;        /* coordinates are multiplied by this (reference: input.scale)   */
    double  periodic[3];  /* >0: box length of a periodic axis (extension; 0 = none)       */
    int32_t renumber;     /* enum fg_renumber for the device ordering                      */
    int32_t gpu;          /* 1: match faces, order them, compute the geometry and the Morton
                             order on GPU `device` (same arrays as the host path; Morton or none) */
    int32_t device;
    int32_t reserved[1];
} fg_mesh_opts;

typedef struct fg_mesh_info {
    int32_t nElem;        /* cells                                                          */
    int32_t nNodes;
    int32_t nFcs;         /* faces (interior + boundary), reference face order              */
    int32_t nBoundary;    /* faces with boundCond != 0                                      */
    int32_t nPeriodic;    /* interior faces formed by periodic matching                     */
    int32_t maxFaces;     /* max faces per cell (4 tet, 5 prism/pyramid, 6 hex)             */
    int32_t nTet, nPyr, nPrism, nHex;
} fg_mesh_info;

/* Read-only views of the reference-layout host arrays (valid until fg_mesh_free).
 * fc2el[f*2+s], boundCond[f], cellCenter[c*3+d], fcCenter[f*3+d], n/nt1/nt2[f*3+d],
 * area[f], volume[c]  — the arrays of the reference's MESH struct (DP/strdata.h:100-115).
 * nbShift[f*3+d] is the periodic image offset of face f seen from its neighbour (0 if none). */
typedef struct fg_mesh_view {
    int32_t nElem, nFcs;
    const int32_t *fc2el;
    const int32_t *boundCond;
    const double  *cellCenter;
    const double  *fcCenter;
    const double  *n, *nt1, *nt2;
    const double  *area;
    const double  *volume;
    const double  *nbShift;
} fg_mesh_view;

int  fg_mesh_load_neu(const char *path, const fg_mesh_opts *opts, fg_mesh **out);
/* The same pipeline for element lists already in memory (a generator, another reader), without
 * the text: what translator_ptw fills from the file (DP/translator.cu:24-349) handed over as
 * arrays in .neu element order.  nodes[nNodes*3] (multiplied by opts->scale); elNN[nElem] nodes
 * per element (4 tet, 5 pyramid, 6 prism, 8 hex); elNodes[nElem*8] 0-based node ids in Gambit
 * order (entries past elNN ignored); elBc[nElem*6] boundary code of each local face
 * (0 interior / untagged, 1 symmetry, 2 outlet, 3 inlet, 4 slip, 5 wall: the codes the reader
 * maps 45/26/13/42/51 to).  The arrays are copied. */
int  fg_mesh_build(int32_t nNodes, const double *nodes, int32_t nElem, const int32_t *elNN, const int32_t *elNodes,
                   const int32_t *elBc, const fg_mesh_opts *opts, fg_mesh **out);
int  fg_mesh_info_get(const fg_mesh *m, fg_mesh_info *info);
int  fg_mesh_view_get(const fg_mesh *m, fg_mesh_view *view);
/* new2old[i] = reference (.neu) index of device cell i. */
int  fg_mesh_permutation(const fg_mesh *m, int32_t *new2old, int32_t n);
void fg_mesh_free(fg_mesh *m);

/* ---------------------------------------------------------------- partitioned runs
 * Replace the reference's METIS decomposition, local-mesh build and per-stage halo
 * communication (DP/decompose.cu:52, DP/buildLocalMesh.cu, DP/communicate.cu) for runs with one
 * GPU per part.  Part p of P owns the cells of the contiguous range [n p / P, n (p+1) / P) of the
 * mesh's device order (the Morton order of the cell centres: a compact region) and holds two
 * layers of ghost cells: its face neighbours in other parts, and their face neighbours outside
 * both.  The part mesh keeps every face that touches an own or a first-layer cell with the whole
 * mesh's orientation, geometry and boundary code, so the part computes the gradients of its
 * first-layer ghosts itself and only primitive records cross between parts.
 *
 * fg_mesh_partition: part `part` of `nParts` of a loaded mesh, as a new mesh handle whose cells
 * are the own cells (device order) followed by the ghosts.  A solver created on it takes and
 * returns the state of the own cells only (fg_set_state / fg_get_state: nOwned rows, in that
 * order), and needs a transport (fg_solver_set_halo) before its first stage. */
int fg_mesh_partition(const fg_mesh *m, int32_t nParts, int32_t part, fg_mesh **out);
typedef struct fg_partition_info {
    int32_t nParts, part;   /* 1, 0 for a mesh that is not a part                     */
    int32_t nOwned;         /* own cells: the first nOwned cells of the part mesh      */
    int32_t nGhost;         /* ghost cells of both layers, after the own ones          */
    int32_t nSend, nRecv;   /* entries of the send / receive lists over all parts      */
    int32_t nGhost1;        /* first-layer ghosts: cells [nOwned, nOwned + nGhost1)    */
} fg_partition_info;
int fg_mesh_partition_info(const fg_mesh *m, fg_partition_info *info);
/* cellGlobal[nOwned + nGhost]: .neu index in the whole mesh of each cell of the part;
 * sendStart[nParts + 1], sendCells[nSend]: the own cells whose records go to part q (those
 * within two face hops of q's cells) are sendCells[sendStart[q] .. sendStart[q+1]); recvStart /
 * recvCells the same for the ghosts whose records come from part q.  Both lists follow the whole
 * mesh's device order, so the k-th record part p sends to q is q's k-th ghost from p.  Any
 * pointer may be NULL. */
int fg_mesh_partition_maps(const fg_mesh *m, int32_t *cellGlobal, int32_t *sendStart, int32_t *sendCells,
                           int32_t *recvStart, int32_t *recvCells);

/* Transport of a partitioned run (the caller's NCCL / MPI / shared memory).  Per RK stage the
 * solver exchanges the primitive records (FG_HALO_W) of the ghost cells once, before the gradient
 * pass (FG_HALO_G, the gradient records, is not exchanged: each part computes its first-layer
 * ghosts' gradients); the dt (every adaptDtItr steps) and the conservation integral are combined
 * with allreduce.
 *   exchange(ctx, field, recordBytes, stream): when called, sendBuf holds the nSend records of
 *     `field` (recordBytes each, in send-list order) and every earlier kernel on `stream` has
 *     finished.  The callee sends records [sendStart[q], sendStart[q+1]) to part q, receives part
 *     q's into records [recvStart[q], recvStart[q+1]) of recvBuf for every q, and returns 0 once
 *     recvBuf is complete (readable by work enqueued on `stream` afterwards).
 *   allreduce(ctx, op, value): combine *value over the parts (op FG_REDUCE_MIN / FG_REDUCE_SUM) in
 *     place; 0 on success.
 * sendBuf / recvBuf: device buffers of at least the sizes fg_halo_buffer_bytes gives. */
enum fg_halo_field { FG_HALO_W = 0, FG_HALO_G = 1 };
enum fg_reduce_op { FG_REDUCE_MIN = 0, FG_REDUCE_SUM = 1 };
typedef struct fg_halo_ops {
    void *ctx;
    int (*exchange)(void *ctx, int32_t field, int64_t recordBytes, void *stream);
    int (*allreduce)(void *ctx, int32_t op, double *value);
} fg_halo_ops;

/* ---------------------------------------------------------------- solver context
 * Replaces startDevice (DP/startDevice.cu:14): allocates every device array once. */
typedef struct fg_solver fg_solver;

enum fg_precision {
    FG_PREC_FP64  = 0,   /* FP64 everywhere ("plain" path)                                       */
    FG_PREC_MIXED = 1    /* FP32 reconstruction / HLLC / WALE / viscous; FP64 state, RK, dt, Newton */
};

int fg_solver_create(const fg_mesh *m, const fg_case *c, int32_t precision, int32_t device,
                     fg_solver **out);
int fg_solver_destroy(fg_solver *s);
/* Device bytes held by the solver (mesh + field arrays). */
int fg_solver_memory(const fg_solver *s, uint64_t *bytes);
/* Partitioned runs: device bytes the send / receive buffers of fg_solver_set_halo need (0 on a
 * solver of a whole mesh), and the transport with those buffers. */
int fg_halo_buffer_bytes(const fg_solver *s, int64_t *sendBytes, int64_t *recvBytes);
int fg_solver_set_halo(fg_solver *s, const fg_halo_ops *ops, void *sendBuf, void *recvBuf);

/* Replaces initialize / readField (DP/initialize.cu:61, DP/restart.cu:424): upload U
 * (nElem*10 doubles, reference order; the own cells of a part mesh) from host memory.  The
 * upload is checked on the device before it replaces the state: FG_ERR_NAN names the first cell
 * that is not finite, has alpha outside [0, 1] or a negative partial density, and the state is
 * left as it was.  Synchronises `stream` (may be NULL). */
int fg_set_state(fg_solver *s, const double *U, void *stream);
/* fg_set_state without the synchronisation, for pipelines that upload every step: the call
 * returns at once.  The copy runs on the solver's own copy stream into its own staging buffer
 * (so it overlaps the work already queued on `stream`, such as the previous step and its
 * download); the check and the replacement are queued on `stream` after it.  From pinned host
 * memory the copy is asynchronous: keep U unchanged until `stream` has passed the replacement.
 * A rejected upload leaves the state as it was and is reported by fg_check_state and by every
 * fg_step (FG_ERR_NAN, naming the cell) until a state is uploaded successfully. */
int fg_set_state_async(fg_solver *s, const double *U, void *stream);
/* Download U (nElem*10 doubles, reference order).  Synchronises `stream`. */
int fg_get_state(fg_solver *s, double *U, void *stream);
/* fg_get_state without the synchronisation: the gather kernel is queued on `stream`, the copy
 * into U (pinned host memory) on the solver's own download stream, so it overlaps the work the
 * caller queues on `stream` next (two staging buffers: the third download in a row waits for
 * the first to finish).  U is complete once a stream that waited through fg_state_join has passed
 * that point, or after a device synchronisation. */
int fg_get_state_async(fg_solver *s, double *U, void *stream);
/* Make `stream` wait, on the device (no host wait), for every fg_get_state_async issued so far. */
int fg_state_join(fg_solver *s, void *stream);

/* ---------------------------------------------------------------- stage functions */

/* computePrimVec + computeGrad + computeFaceValues(limiter) + computeRHS (+ viscous)
 * (DP/computePrimVec.cu:82, DP/computeGrad.cu:263, DP/computeFaceValues.cu:138,
 *  DP/computeRHS.cu:384): residual of the current state into the device RHS buffer.
 * With want_signal != 0 also the per-cell max signal speed used by computeTimeStep. */
int fg_compute_rhs(fg_solver *s, int32_t want_signal, void *stream);

/* computeTimeStep (DP/computeTimeStep.cu:172): after fg_compute_rhs(want_signal=1),
 * dt = min(cfl * min_c V^0.3333 / s_c, maxDt), kept on the device; *dt_out (may be NULL)
 * receives it (synchronises the stream when non-NULL). */
int fg_compute_time_step(fg_solver *s, double *dt_out, void *stream);

/* initRk (DP/update.cu:141): U0 = U. */
int fg_init_rk(fg_solver *s, void *stream);

/* update (DP/update.cu:105): Runge-Kutta stage irk from the RHS buffer with the device dt. */
int fg_update(fg_solver *s, int32_t irk, void *stream);

/* One full RK stage irk with the fused residual + update kernel (no RHS buffer round trip). */
int fg_stage(fg_solver *s, int32_t irk, void *stream);

/* relaxation (DP/relaxation.cu:77): partition + thermal + chemical equilibrium (FP64 Newton). */
typedef struct fg_relax_stats {
    int32_t nTherm;       /* cells relaxed thermally          */
    int32_t nChem;        /* cells relaxed chemically         */
    int32_t nAbort;       /* Newton solves that fell back to the best iterate */
    int32_t nIter;        /* Newton iterations summed over all cells (surrogate polish steps included) */
    int32_t nSurrogate;   /* chemical cells solved from the surrogate's prediction            */
    int32_t nFallback;    /* chemical cells that took the reference Newton with a surrogate attached
                             (outside the training hull, or polish residual above tolerance)   */
    int32_t nPolish;      /* polish Newton steps of the cells counted in nSurrogate            */
} fg_relax_stats;
int fg_relaxation(fg_solver *s, fg_relax_stats *stats, void *stream);
/* counts of the most recent relaxation, including the one inside fg_step (synchronises) */
int fg_relax_stats_read(fg_solver *s, fg_relax_stats *stats);

/* ---------------------------------------------------------------- learned equilibrium surrogate
 * No counterpart in the reference (whose chemical relaxation is the per-cell Newton of
 * DP/chemRlx.cu:4-267).  An MLP 3 -> 64 -> 64 -> 64 -> 4 (GELU) maps a chemical cell's
 * (rho, e, Y) — mixture density, mixture internal energy per unit mass, vapour mass fraction
 * before the solve — to the equilibrium (p, T, alpha, Y_eq).  Trained on the GPU (FP32, Adam)
 * on samples logged from the solver's own Newton solves; evaluated in the relaxation kernel on
 * the BF16 tensor cores (FP32 accumulation).  The prediction seeds at most polishIters full
 * Newton steps on the reference's residuals; a cell is accepted when |p_L - p_G| <= relTol |p|,
 * |T_L - T_G| <= relTol T and |g_L - g_G| <= relTol Cp_L T, else (and for inputs outside the
 * training hull: per-feature box plus a Mahalanobis bound) it takes the reference Newton. */
typedef struct fg_surrogate fg_surrogate;
#define FG_SG_NPARAM 8836   /* W1[3][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64][4] b4[4] */
#define FG_SG_NNORM 30      /* xMean[3] xStd[3] yMean[4] yStd[4] boxLo[3] boxHi[3] covInv[9] d2Max */
int fg_surrogate_create(int32_t device, uint64_t seed, fg_surrogate **out);   /* seeded random init */
int fg_surrogate_destroy(fg_surrogate *g);
/* X [n][3] = (rho, e, Y), Y [n][4] = (p, T, alpha, Y_eq), host FP32; sets the standardisation and
 * the training hull from these samples and keeps them on the device for training */
int fg_surrogate_set_data(fg_surrogate *g, const float *X, const float *Y, int64_t n);
/* epochs of shuffled mini-batches (Adam, cosine-decayed lr); *final_loss = loss of the last batch */
int fg_surrogate_train(fg_surrogate *g, int32_t epochs, int32_t batch, float lr, uint64_t seed, float *final_loss);
/* mean squared error over the 4 outputs of n standardised samples and its gradient [FG_SG_NPARAM]
 * (FP32 forward/backward kernels, no update); host arrays */
int fg_surrogate_loss_grad(fg_surrogate *g, const float *Xs, const float *Ys, int32_t n, float *loss, float *grad);
int fg_surrogate_get_params(fg_surrogate *g, float *params);
int fg_surrogate_set_params(fg_surrogate *g, const float *params);
int fg_surrogate_get_norm(fg_surrogate *g, float *norm);
int fg_surrogate_set_norm(fg_surrogate *g, const float *norm);
/* tensor-core forward of n raw inputs (host arrays): Y [n][4] raw outputs, in_hull [n] (may be NULL) */
int fg_surrogate_predict(fg_surrogate *g, const float *X, int32_t n, float *Y, int32_t *in_hull);
/* attach (g != NULL) or detach the surrogate used by fg_relaxation / fg_step; g must outlive the
 * attachment and live on the solver's device */
int fg_solver_set_surrogate(fg_solver *s, const fg_surrogate *g, double relTol, int32_t polishIters);
/* where the attached surrogate's polish runs (no counterpart in the reference; a tuning knob):
 * FG_SG_PASS_FUSED inside the relaxation kernel (faster when many cells are chemical),
 * FG_SG_PASS_SEPARATE as a pass of its own before it (faster when few are), FG_SG_PASS_AUTO
 * (default) chooses per relaxation from the chemical cells of an earlier one (separate below
 * 10 %; it queries an event and copies 32 bytes of counters back behind each relaxation, so set
 * _FUSED or _SEPARATE before capturing a relaxation into a CUDA graph).  The relaxed states and
 * counters are bitwise the same for all three. */
#define FG_SG_PASS_AUTO 0
#define FG_SG_PASS_FUSED 1
#define FG_SG_PASS_SEPARATE 2
int fg_solver_set_surrogate_pass(fg_solver *s, int32_t mode);
/* log of chemical Newton solves as surrogate training samples: capacity 0 turns it off;
 * fg_relax_log_read copies min(logged, cap) samples (X [][3], Y [][4], order not defined) */
int fg_relax_log(fg_solver *s, int64_t capacity);
int fg_relax_log_read(fg_solver *s, float *X, float *Y, int64_t cap, int64_t *count);

/* consCalc (DP/consCalc.cu:40): FP64 integral of variable ivar over the domain
 * (ivar 0 integrates 1-alpha).  Deterministic two-level reduction. */
int fg_cons_calc(fg_solver *s, int32_t ivar, double *out, void *stream);

/* Conservation integral without device allocation.  No counterpart in the reference: it is
 * for callers that cannot call cudaMalloc when they need the integral (an application whose
 * pool allocator owns all device memory, a monitor between the steps of a latency-critical
 * loop where cudaMalloc / cudaFree may synchronise the device).
 * U: device, reference layout U[cell*10 + v]; vol: device, nCells volumes; out: device, one
 * double, receives the integral of variable ivar (ivar 0 integrates 1-alpha).  The result is
 * deterministic for a given nCells and cell order; it agrees with fg_cons_calc (which sums the
 * cells in the solver's own device order) to rounding, not bit for bit.
 * Runs on the calling thread's current device, asynchronously on `stream`.
 * The block partial sums go to a static device array of FG_NOALLOC_MAX_CELLS/256 doubles
 * (512 KiB, held on every device that loads the library until exit); nCells above
 * FG_NOALLOC_MAX_CELLS is rejected with FG_ERR_ARG.  The first call on a device looks the
 * array's address up (cudaGetSymbolAddress) and keeps it for the life of the process: make that
 * first call before any stream capture, and do not call it on a device that was reset
 * (cudaDeviceReset) after its first call there.
 * All calls on a device share the array: calls that overlap on the GPU race. */
#define FG_NOALLOC_MAX_CELLS (65536 * 256)
int fg_cons_integral_noalloc(const double *U, const double *vol, int32_t nCells, int32_t ivar, double *out,
                             void *stream);

/* State probe for monitoring a run (no counterpart in the reference, whose consCalc gives the
 * integral of one variable, DP/consCalc.cu:40): vapour volume = integral of 1 - alpha (consCalc
 * of variable 0), maximum and minimum of the mixture pressure alpha p_L + (1 - alpha) p_G and the
 * maximum speed |u|, from the current state, by deterministic device reductions.  Synchronises
 * `stream`.  Not available on a part of a partitioned mesh. */
typedef struct fg_probe_out {
    double vapourVolume;
    double maxPressure;
    double minPressure;
    double maxSpeed;
} fg_probe_out;
int fg_probe(fg_solver *s, fg_probe_out *out, void *stream);

/* dt and physical time held by the solver. */
int fg_get_time(fg_solver *s, double *dt, double *physicalTime, int32_t *iStep);
int fg_set_dt(fg_solver *s, double dt);

/* Checkpoint / restart (DP/restart.cu:113-152 writeFieldRestart, :424-497 readField, which store
 * consVec as 11-digit ASCII).  Binary and exact: header (magic "FGCKPT01", nElem, NEQ, iStep,
 * precision, physicalTime, dt) + U[nElem*10] in .neu element order.  fg_checkpoint_read restores
 * the state, dt, physical time and step counter; restarting reproduces an uninterrupted run
 * bit for bit. */
int fg_checkpoint_write(fg_solver *s, const char *path);
int fg_checkpoint_read(fg_solver *s, const char *path);

/* Field dump replacing the Tecplot ASCII export (DP/export_plt.cu:95-174): binary, per cell in
 * .neu element order (not averaged to the nodes): magic "FGFIELD1", int32 {nElem, 13, iStep, 0},
 * double physicalTime, then double[nElem][13] = x y z avfL avfG rho U V W pressure temperature
 * vaporMass |grad rho| (pressure and temperature volume-fraction weighted as the reference's
 * export; |grad rho| from the most recent gradient pass). */
int fg_field_dump(fg_solver *s, const char *path);

/* Failure detection (the reference prints CUDA errors and continues).  fg_set_state rejects a
 * state that is not finite, has alpha outside [0, 1] or a negative partial density
 * (FG_ERR_NAN).  The RK kernels flag a state they produce that is not finite or has a
 * non-positive mixture density (alpha may leave [0, 1] by rounding; cons2prim clamps it, as in
 * the reference); the flag lives in mapped
 * host memory, so fg_step checks it at entry without synchronising and returns FG_ERR_NAN from
 * then on (the flag is seen once the flagged kernel has run: at most a few steps late).
 * fg_check_state synchronises and reports it; *badStep = the step that produced it, or -1.
 * fg_set_state / fg_checkpoint_read clear it. */
int fg_check_state(fg_solver *s, int32_t *badStep);

/* One explicitLoop iteration (DP/explicitLoop.cu:28-64): time advance, RK stages with the
 * adaptive dt at stage 0 every adaptDtItr steps, relaxation, conservation every adaptDtItr. */
int fg_step(fg_solver *s, void *stream);

/* ---------------------------------------------------------------- instrumentation
 * (the reference has per-phase cudaEvent timers commented out, e.g. DP/computeRHS.cu:221-235)
 * With profiling enabled every kernel launch of the solver is bracketed by CUDA events on the
 * stream it is launched on; fg_profile_read synchronises and returns per-kind totals.
 * Kinds: 0 gradient+limiter, 1 face flux, 2 RK update from the residual buffer, 3 relaxation,
 *        4 dt reduction, 5 conservation, 6 other (state copies, time advance),
 *        7 owner-side gather (+ RK combination in a fused stage). */
enum { FG_K_GRAD = 0, FG_K_FLUX = 1, FG_K_UPDATE = 2, FG_K_RELAX = 3, FG_K_DT = 4, FG_K_CONS = 5, FG_K_OTHER = 6,
       FG_K_GATHER = 7, FG_K_NKINDS = 8 };
typedef struct fg_kernel_times {
    double  ms[FG_K_NKINDS];
    int64_t launches[FG_K_NKINDS];
} fg_kernel_times;
int fg_profile(fg_solver *s, int32_t enable);                 /* enable (1) / disable (0); resets */
int fg_profile_read(fg_solver *s, fg_kernel_times *out);
/* Number of kernels the solver has launched since creation. */
int fg_launch_count(fg_solver *s, uint64_t *count);

/* ---------------------------------------------------------------- parity hooks
 * Copies of intermediate device buffers in reference order, for tests.
 *   fg_get_rhs:    RHS[nElem*10]            (after fg_compute_rhs)
 *   fg_get_limited: grad[nElem*10*3] and theta[nElem*10] of the last residual (vars 0..8;
 *                   var 9, the mixture density the reference also limits but never uses,
 *                   is returned as 0)
 *   fg_get_signal: per-cell max signal speed of the last fg_compute_rhs(want_signal=1) or of the
 *                   last dt step of fg_step (which computes it in the face kernel instead) */
int fg_get_rhs(fg_solver *s, double *rhs);
int fg_get_limited(fg_solver *s, double *grad, double *theta);
int fg_get_signal(fg_solver *s, double *signal);

#ifdef __cplusplus
}
#endif
#endif /* FOOSKAGPU_H */
