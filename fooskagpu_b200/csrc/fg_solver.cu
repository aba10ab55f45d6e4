// C ABI of the device residual path: solver lifetime, state transfer, stage functions and the
// explicitLoop step (host side).  See include/fooskagpu.h for the reference function each
// entry point replaces.
#include "../../include/fooskagpu.h"
#include "fg_kernels.cuh"
#include "fg_mesh.h"
#include "fg_surrogate.cuh"

#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err = "";

int set_err(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

#define FG_CUDA_TRY(expr)                                                                         \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return set_err(e_ == cudaErrorMemoryAllocation ? FG_ERR_NOMEM : FG_ERR_CUDA,          \
                           std::string(#expr) + ": " + cudaGetErrorString(e_));                   \
    } while (0)

#define FG_LAUNCH_CHECK(what)                                                                     \
    do {                                                                                          \
        cudaError_t e_ = cudaGetLastError();                                                      \
        if (e_ != cudaSuccess) return set_err(FG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t b) {
        release();
        bytes = b;
        return cudaMalloc(&p, b ? b : 16);
    }
    template <typename X>
    X *as() const { return reinterpret_cast<X *>(p); }
};

}  // namespace

namespace fg {
int surrogate_view(const fg_surrogate *g, SurrogateDev *out);
int surrogate_device(const fg_surrogate *g);
}  // namespace fg

// ------------------------------------------------------------------ solver base
struct fg_solver {
    virtual ~fg_solver() {
        for (cudaEvent_t e : evPool) cudaEventDestroy(e);
        if (hBad) cudaFreeHost((void *)hBad);
        if (evInFree) cudaEventDestroy(evInFree);
        if (evCopied) cudaEventDestroy(evCopied);
        if (copyStream) cudaStreamDestroy(copyStream);
        for (cudaEvent_t e : evOutFree)
            if (e) cudaEventDestroy(e);
        if (evGathered) cudaEventDestroy(evGathered);
        if (downStream) cudaStreamDestroy(downStream);
        if (hCntPrev) cudaFreeHost(hCntPrev);
        if (evCnt) cudaEventDestroy(evCnt);
    }
    // where the surrogate's polish runs (FG_SG_PASS_*).  Automatic: the relaxation counters of a
    // surrogate relaxation are copied to pinned host memory behind it (buffer and event created
    // on the first one), one copy in flight at a time; once a copy has arrived, its chemical
    // cells choose the form (sgAutoPass) that the following relaxations use until the next one
    // arrives.  The host may run many steps ahead of the device: a copy still in flight keeps the
    // form chosen before.
    int sgPass = FG_SG_PASS_AUTO;
    int sgAutoPass = 0;
    int32_t *hCntPrev = nullptr;
    cudaEvent_t evCnt = nullptr;
    bool cntPending = false;
    // asynchronous uploads copy on their own stream into their own staging buffer, so the copy of
    // the next state overlaps the work queued before it (created on the first asynchronous upload)
    cudaStream_t copyStream = nullptr;
    cudaEvent_t evInFree = nullptr;   // the last scatter has read the upload staging buffer
    cudaEvent_t evCopied = nullptr;   // the upload copy has landed
    // asynchronous downloads: the gather kernel on the caller's stream into one of two staging
    // buffers, the copy to the host on the solver's download stream (created on first use)
    cudaStream_t downStream = nullptr;
    cudaEvent_t evOutFree[2] = {nullptr, nullptr};   // the download from staging buffer b has finished
    cudaEvent_t evGathered = nullptr;                // the gather into the current buffer is done
    int outNext = 0;                                 // staging buffer of the next download
    int state_join(cudaStream_t s) {
        // the download stream runs its copies in order: waiting for the last one covers all
        if (downStream) FG_CUDA_TRY(cudaStreamWaitEvent(s, evOutFree[outNext ^ 1], 0));
        return FG_OK;
    }
    int init_flag() {
        void *h = nullptr;
        FG_CUDA_TRY(cudaHostAlloc(&h, 2 * sizeof(int32_t), cudaHostAllocMapped));
        hBad = static_cast<volatile int32_t *>(h);
        hBad[0] = 0;
        hBad[1] = 0;
        FG_CUDA_TRY(cudaHostGetDevicePointer((void **)&dBad, h, 0));
        return FG_OK;
    }
    int upload_error() const {
        return set_err(FG_ERR_NAN, "fg_set_state: cell " + std::to_string(hBad[1] - 1) +
                                       " is not finite or has alpha outside [0, 1] or a negative partial density"
                                       " (the state was not replaced)");
    }
    // a flagged state (RK kernels) or a rejected upload, in that order of precedence
    int flag_error() const { return hBad[1] ? upload_error() : bad_state_error(); }
    int bad_state_error() const {
        return set_err(FG_ERR_NAN, "the state became non-finite or its density non-positive in step " +
                                       std::to_string(*hBad - 1) + " (reset it with fg_set_state / fg_checkpoint_read)");
    }
    int device = 0;
    // ---- instrumentation: events around every launch when enabled
    bool prof = false;
    std::vector<cudaEvent_t> evPool;
    size_t evUsed = 0;
    std::vector<int> recKind;
    uint64_t launches = 0;
    cudaEvent_t ev_next() {
        if (evUsed == evPool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            evPool.push_back(e);
        }
        return evPool[evUsed++];
    }
    void prof_begin(int kind, cudaStream_t s) {
        launches++;
        if (!prof) return;
        recKind.push_back(kind);
        cudaEventRecord(ev_next(), s);
    }
    void prof_end(cudaStream_t s) {
        if (!prof) return;
        cudaEventRecord(ev_next(), s);
    }
    int prof_read(fg_kernel_times *out) {
        memset(out, 0, sizeof(*out));
        if (cudaDeviceSynchronize() != cudaSuccess) return set_err(FG_ERR_CUDA, "profile read: device error");
        for (size_t i = 0; i < recKind.size(); i++) {
            float ms = 0;
            cudaEventElapsedTime(&ms, evPool[2 * i], evPool[2 * i + 1]);
            out->ms[recKind[i]] += ms;
            out->launches[recKind[i]]++;
        }
        return FG_OK;
    }
    void prof_reset(bool en) {
        prof = en;
        evUsed = 0;
        recKind.clear();
    }
    fg_case cs{};
    int precision = FG_PREC_FP64;
    // failure flags (mapped host memory: read without a stream sync): [0] step + 1 of a state the
    // RK kernels found unusable, [1] first unusable cell + 1 of a rejected upload
    volatile int32_t *hBad = nullptr;
    int32_t *dBad = nullptr;
    std::vector<double> cellCenter;   // reference order, for the field dump
    // attached equilibrium surrogate (not owned) and the optional chemical-solve log
    const fg_surrogate *sg = nullptr;
    double sgTol = 1e-6;
    int sgIters = 3;
    DevBuf logX, logY, logCnt;
    long long logCap = 0;
    int n = 0, nSlots = 0;
    int nU = 0;               // own cells: the state rows (n - nU ghosts on a partitioned mesh)
    int nG = 0;               // cells with gradients: own and first-layer ghost cells
    int nFEval = 0;           // faces touching an own cell: the first nFEval of the GPU face order
    bool parted = false;      // built from one part of a partitioned mesh
    fg_halo_ops halo{};       // the partitioned run's transport (fg_solver_set_halo)
    void *haloSend = nullptr, *haloRecv = nullptr;
    int iStep = 0;
    uint64_t bytes = 0;
    virtual int init(const fg::Mesh &m) = 0;
    // gradient pass only; face fluxes + gather (+ RK unless mode is the residual) only
    virtual int gradients(cudaStream_t s) = 0;
    virtual int flux(int mode, int wantSignal, int irk, int writeU0, cudaStream_t s) = 0;
    // partitioned runs: send the own halo cells' records of `field` and receive the ghosts'
    virtual int halo_exchange(int field, cudaStream_t s) = 0;
    virtual void halo_bytes(int64_t *send, int64_t *recv) const = 0;
    // gradient pass with the record exchanges a partitioned run needs around it: the ghosts'
    // primitive records before (they changed in the last update / relaxation), their gradient
    // records after (the face fluxes read both sides')
    int gradients_halo(cudaStream_t s) {
        // one exchange per stage: the ghosts' primitive records; the gradient pass covers the own
        // and first-layer cells, whose faces the part mesh holds
        int rc;
        if (parted && (rc = halo_exchange(FG_HALO_W, s))) return rc;
        return gradients(s);
    }
    // combine a per-part scalar over the parts (no-op on an unpartitioned mesh)
    int reduce(int op, double *v) {
        if (!parted) return FG_OK;
        if (!halo.allreduce)
            return set_err(FG_ERR_ARG, "partitioned mesh: set the transport with fg_solver_set_halo first");
        if (halo.allreduce(halo.ctx, op, v) != 0) return set_err(FG_ERR_CUDA, "partitioned run: allreduce failed");
        return FG_OK;
    }
    // upload U; wait = true synchronises and reports a rejected upload, false leaves the report to
    // the flags (fg_step / fg_check_state)
    virtual int set_state(const double *U, cudaStream_t s, bool wait) = 0;
    // download U; wait = false leaves the copy queued on the stream
    virtual int get_state(double *U, cudaStream_t s, bool wait) = 0;
    virtual int compute_rhs(int wantSignal, cudaStream_t s) = 0;
    // stage irk with a new dt first (the dt step of explicitLoop), fused
    virtual int dt_stage(int irk, int writeU0, cudaStream_t s) = 0;
    virtual int time_step(double *dtOut, cudaStream_t s) = 0;
    virtual int init_rk(cudaStream_t s) = 0;
    virtual int update(int irk, int writeU0, cudaStream_t s) = 0;
    virtual int stage(int irk, int writeU0, cudaStream_t s) = 0;
    virtual int relax(fg_relax_stats *st, cudaStream_t s) = 0;
    virtual int relax_counts(fg_relax_stats *st) = 0;
    virtual int cons(int ivar, double *out, cudaStream_t s) = 0;
    virtual int probe(double *out4, cudaStream_t s) = 0;
    virtual int advance_time(cudaStream_t s) = 0;
    virtual int get_time(double *dt, double *t) = 0;
    virtual int set_dt(double dt) = 0;
    virtual int set_time(double t) = 0;
    // 13 export variables per cell in .neu element order (host array nElem * 13)
    virtual int field_vars(double *out) = 0;
    virtual int get_rhs(double *rhs) = 0;
    virtual int get_limited(double *grad, double *theta) = 0;
    virtual int get_signal(double *sig) = 0;
};

namespace fg {

__global__ void k_advance_time(const double *dt, double *t) { *t += *dt; }

// export variables of DP/export_plt.cu:42-80 per cell (not averaged to the nodes): x y z avfL avfG
// rho U V W pressure temperature vaporMass |grad rho|, the last from the most recent gradient
// pass; written to out[old * 13 + k] (the .neu element order)
template <typename T>
__global__ void k_field_vars(int n, const double *__restrict__ U, const T *__restrict__ G, size_t gStride,
                             const int32_t *new2old, const PhysD D, const double *cp, double *out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double u[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) u[v] = U[(size_t)v * n + c];
    const double aL = u[0], aG = 1 - aL;
    const double rL = u[1] / aL, rG = u[2] / aG;
    const double rho = aL * rL + aG * rG;
    const double eL = u[6] / (aL * rL), eG = u[7] / (aG * rG);
    const double pL = D.gm1[0] * rL * eL - D.gpinf[0] - D.gm1eta[0] * rL;
    const double pG = D.gm1[1] * rG * eG - D.gpinf[1] - D.gm1eta[1] * rG;
    const double tL = (pL + D.pinf[0]) / ((cp[0] / D.gam[0]) * D.gm1[0] * rL);
    const double tG = (pG + D.pinf[1]) / ((cp[1] / D.gam[1]) * D.gm1[1] * rG);
    // grad rho = (rhoL - rhoG) grad alpha + alpha grad rhoL + (1 - alpha) grad rhoG
    // gradients of W: component d of var v is value NP + 3 v + d of the record
    auto g = [&](int q) { return (double)G[grec_index<T>(gStride, (size_t)c, NP + q)]; };
    double gr[3];
#pragma unroll
    for (int d = 0; d < 3; d++) gr[d] = (rL - rG) * g(d) + aL * g(3 + d) + aG * g(6 + d);
    double *o = out + (size_t)new2old[c] * 13;
    o[3] = aL;
    o[4] = aG;
    o[5] = rho;
    o[6] = u[3] / rho;
    o[7] = u[4] / rho;
    o[8] = u[5] / rho;
    o[9] = aL * pL + aG * pG;
    o[10] = aL * tL + aG * tG;
    o[11] = u[9];
    o[12] = sqrt(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
}

// automatic surrogate polish pass: a separate pass when fewer than one cell in kSparseChemInv of
// the previous surrogate relaxation was chemical
constexpr int kSparseChemInv = 10;

template <typename T>
struct SolverT : public fg_solver {
    DevBuf dNbr, dFlags, dGeo, dVol, dVolP, dNew2Old, dHaloStart, dHaloIds, dSlotLocal;
    DevBuf dU, dU0, dRHS, dW[2], dG, dSig, dCellSig, dBlockMin, dScal, dCnt, dCons, dStage;
    DevBuf dStageIn;   // staging buffer of the asynchronous uploads (on first use)
    DevBuf dStageOut[2];   // staging buffers of the asynchronous downloads (on first use)
    DevBuf dFIdx, dFGeo, dSlotFace, dClosure, dFB;
    DevBuf dOrdFlag, dOrdCnt, dOrdOff, dOrder, dOrdTotal;   // relaxation cell ordering
    DevBuf dPred, dHullOk, dTcErr;                          // surrogate predictions
    DevBuf dSendCells, dRecvCells;                          // halo lists of a partitioned mesh
    DevBuf dChk;                                            // set_state: first unusable cell
    DevBuf dProbe;                                          // fg_probe block results (on first use)
    std::vector<int32_t> sendStart, recvStart;
    int cur = 0;
    DevMesh<T> dm{};
    PhysT<T> P{};
    PhysD D{};
    RelaxParams R{};

    Fields<T> fields(int wIn) {
        Fields<T> f;
        f.FB = dFB.as<T>();
        f.U = dU.as<double>();
        f.U0 = dU0.as<double>();
        f.RHS = dRHS.as<double>();
        f.Win = dW[wIn].as<T>();
        f.Wout = dW[1 - wIn].as<T>();
        f.G = dG.as<T>();
        f.signal = dSig.as<double>();
        f.cellSig = dCellSig.as<T>();
        f.blockMin = dBlockMin.as<double>();
        f.dt = dScal.as<double>();
        f.bad = dBad;
        f.step = iStep;
        return f;
    }

    int init(const fg::Mesh &m) override {
        n = m.nElem;
        nU = m.owned();
        nG = m.gradient_cells();
        parted = m.nOwned >= 0;
        nSlots = m.maxFaces;
        cellCenter.assign(m.cellCenter.begin(), m.cellCenter.end());
        FG_CUDA_TRY(cudaSetDevice(device));
        if (init_flag() != FG_OK) return FG_ERR_CUDA;
        // physics constants in T and FP64
        for (int k = 0; k < 2; k++) {
            const double g = cs.gamma[k];
            P.gam[k] = (T)g;
            P.gm1[k] = (T)(g - 1);
            P.gp1[k] = (T)(g + 1);
            P.pinf[k] = (T)cs.pInf[k];
            P.gpinf[k] = (T)(g * cs.pInf[k]);
            P.cvgm1[k] = (T)((cs.Cp[k] / g) * (g - 1));
            P.gm1eta[k] = (T)((g - 1) * cs.eta[k]);
            P.mu[k] = (T)cs.dynVisc[k];
            P.cp[k] = (T)cs.Cp[k];
            P.prn[k] = (T)cs.Pr[k];
            D.gam[k] = g;
            D.gm1[k] = g - 1;
            D.pinf[k] = cs.pInf[k];
            D.gpinf[k] = g * cs.pInf[k];
            D.cvgm1[k] = (cs.Cp[k] / g) * (g - 1);
            D.gm1eta[k] = (g - 1) * cs.eta[k];
            R.gam[k] = g;
            R.pinf[k] = cs.pInf[k];
            R.cp[k] = cs.Cp[k];
            R.eta[k] = cs.eta[k];
            R.satConst[k] = cs.satConst[k];
        }
        D.avfLo = cs.avfMin / 100;
        D.avfHi = 1.0 - cs.avfMin / 100;
        P.chemLimit = (T)cs.chemLimit;
        P.woods = (cs.woodsFlag == 1);
        P.visc = (cs.viscFlag == 1);
        P.heat = (cs.viscFlag == 1 && cs.heatFlux == 1);
        P.limiter = cs.limiter;
        P.inVelFlag = (cs.inletVelFlag == 1);
        for (int d = 0; d < 3; d++) P.inVel[d] = (T)cs.inletVel[d];
        P.pDatum = (T)cs.pressureDatum;
        D.pDatum = (double)P.pDatum;   // the face and cell terms use the same datum value
        if (cs.limiter != 0 && cs.limiter != 1) return set_err(FG_ERR_UNSUPPORTED, "limiter must be 0 or 1");
        if (P.heat && !(cs.Pr[0] > 0 && cs.Pr[1] > 0))
            return set_err(FG_ERR_ARG, "heatFlux needs Pr[0] > 0 and Pr[1] > 0");
        P.turb = (cs.turbulence == 1);
        P.energyFix = (cs.hllcEnergyFix == 1);
        P.tieTol = (T)cs.hllcTieTol;
        {
            // inlet ghost (DP/bc.h:2-25): rho from p = 11.4e5 Pa, T = 115.3 K, or the case's
            // prescribed inlet state (extension)
            const bool own = (cs.inletStateFlag == 1);
            const double pIn = own ? cs.inletP : 11.4e5, tIn = own ? cs.inletT : 115.3;
            P.inAlpha = (T)(1.0 - cs.avfMin);
            P.inRhoL = (T)((pIn + cs.pInf[0]) / ((cs.Cp[0] / cs.gamma[0]) * tIn * (cs.gamma[0] - 1)));
            P.inRhoG = (T)((pIn + cs.pInf[1]) / ((cs.Cp[1] / cs.gamma[1]) * tIn * (cs.gamma[1] - 1)));
            P.inP = (T)pIn;
        }
        R.avfMin = cs.avfMin;
        R.chemLimit = cs.chemLimit;
        R.thermUrf = cs.thermUrf;
        R.chemUrf = cs.chemUrf;
        R.satTempUrf = cs.satTempUrf;
        R.thermItrMax = cs.thermItrMax;
        R.chemItrMax = cs.chemItrMax;
        R.chemFlag = cs.chemFlag;

        // ---- device mesh (ELL slots in element-local face order) ----
        const int nF = m.nFcs;
        std::vector<int32_t> elFc2fc((size_t)m.nElem * 6, -1), elFcSide((size_t)m.nElem * 6, 0);
        for (int f = 0; f < nF; f++) {
            elFc2fc[(size_t)m.fc2el[2 * f] * 6 + m.fc2elFc[2 * f]] = f;
            elFcSide[(size_t)m.fc2el[2 * f] * 6 + m.fc2elFc[2 * f]] = 0;
            if (m.boundCond[f] == 0) {
                elFc2fc[(size_t)m.fc2el[2 * f + 1] * 6 + m.fc2elFc[2 * f + 1]] = f;
                elFcSide[(size_t)m.fc2el[2 * f + 1] * 6 + m.fc2elFc[2 * f + 1]] = 1;
            }
        }
        const size_t S = (size_t)nSlots * n;
        // component stride of the geometry arrays: padded to 16 bytes (see DevMesh::geoStride)
        const size_t GS = (S * sizeof(T) + 15) / 16 * 16 / sizeof(T);
        std::vector<int32_t> nbr(S, INT32_MIN), flags(n, 0);
        std::vector<T> geo(6 * GS, (T)0);
        std::vector<double> volP(n), vol(n);
        for (int i = 0; i < n; i++) {
            const int o = m.new2old[i];
            const fg::ElemType *et = fg::elem_type_for_nodes(m.elNN[o]);
            vol[i] = m.volume[o];
            volP[i] = pow(m.volume[o], 0.3333);
            if (i >= nG) continue;   // a second-layer ghost: records only, no faces of its own
            int fl = et->nFaces;
            for (int k = 0; k < et->nFaces; k++) {
                const int f = elFc2fc[(size_t)o * 6 + k];
                const int side = elFcSide[(size_t)o * 6 + k];
                if (f < 0) return set_err(FG_ERR_MESH, "internal: element face without a face record");
                const size_t q = (size_t)i * nSlots + k;   // cell-major: the lanes of a cell read contiguously
                const int bc = m.boundCond[f];
                const int own = m.fc2el[2 * f], nbo = m.fc2el[2 * f + 1];
                const double *fc = &m.fcCenter[(size_t)f * 3];
                const double *sh = &m.nbShift[(size_t)f * 3];
                double xOwnSide[3], xNbSide[3];
                for (int d = 0; d < 3; d++) {
                    xOwnSide[d] = fc[d];
                    xNbSide[d] = fc[d] + sh[d];
                }
                if (side == 0) {
                    fl |= 1 << (3 + k);
                    nbr[q] = (bc == 0) ? m.old2new[nbo] : -bc;
                } else {
                    nbr[q] = m.old2new[own];
                }
                // outward n A in T arithmetic: (+-1) * n * A, the gradient's operand order
                const T sg = (side == 0) ? (T)1 : (T)-1;
                for (int d = 0; d < 3; d++) geo[(size_t)d * GS + q] = sg * (T)m.n[(size_t)f * 3 + d] * (T)m.area[f];
                // face centre (the periodic image on the neighbour's side) - own cell centre
                for (int d = 0; d < 3; d++) {
                    const double dcv = (side == 0) ? xOwnSide[d] - m.cellCenter[(size_t)o * 3 + d]
                                                   : xNbSide[d] - m.cellCenter[(size_t)o * 3 + d];
                    geo[(size_t)(3 + d) * GS + q] = (T)dcv;
                }
            }
            flags[i] = fl;
        }
        // faces in GPU order: tiles of kFaceTile consecutive owner cells (renumbered); within a
        // tile by the owner's element-local face (slot), then by owner.  The lanes of a gather warp
        // then read the records of the same local face of nearby cells from nearby positions, and
        // the face kernel's lanes take nearby owners whose neighbours lie in one direction of a hex
        // brick.  A ghost owns the faces it shares with own cells where the whole mesh makes it the
        // owner.  On a part the faces touching an own cell come first (the face kernel evaluates
        // those only); the faces among ghosts, kept for the first-layer ghosts' gradients, follow.
        std::vector<int32_t> gFace(nF, -1), slotFace(S, -1), fIdx(2 * (size_t)nF);
        int nFo = 0;
        auto touches_own = [&](int f) {
            return m.old2new[m.fc2el[2 * f]] < nU || (m.boundCond[f] == 0 && m.old2new[m.fc2el[2 * f + 1]] < nU);
        };
        for (int pass = 0; pass < 2; pass++) {
            for (int t0 = 0; t0 < n; t0 += kFaceTile) {
                const int t1 = std::min(n, t0 + kFaceTile);
                for (int k = 0; k < MAXSLOT; k++)
                    for (int i = t0; i < t1; i++) {
                        const int o = m.new2old[i];
                        if (k >= fg::elem_type_for_nodes(m.elNN[o])->nFaces) continue;
                        const int f = elFc2fc[(size_t)o * 6 + k];
                        if (f >= 0 && elFcSide[(size_t)o * 6 + k] == 0 && touches_own(f) == (pass == 0))
                            gFace[f] = nFo++;
                    }
            }
            if (pass == 0) nFEval = nFo;
        }
        if (nFo != nF) return set_err(FG_ERR_MESH, "internal: face ownership does not cover every face");
        // face geometry: 11 components (n[3], A, x_f - x_owner [3], x_f - x_nb [3], WALE Ls^2)
        const size_t FS = ((size_t)nF * sizeof(T) + 15) / 16 * 16 / sizeof(T);
        std::vector<T> fgeo(11 * FS, (T)0);
        for (int f = 0; f < nF; f++) {
            const int g = gFace[f];
            const int own = m.fc2el[2 * f], nbo = m.fc2el[2 * f + 1];
            const int bc = m.boundCond[f];
            fIdx[g] = m.old2new[own];
            fIdx[(size_t)nF + g] = (bc == 0) ? m.old2new[nbo] : -bc;
            for (int d = 0; d < 3; d++) fgeo[(size_t)d * FS + g] = (T)m.n[(size_t)f * 3 + d];
            fgeo[3 * FS + g] = (T)m.area[f];
            for (int d = 0; d < 3; d++) {
                const double xf = m.fcCenter[(size_t)f * 3 + d];
                fgeo[(size_t)(4 + d) * FS + g] = (T)(xf - m.cellCenter[(size_t)own * 3 + d]);
                if (bc == 0)
                    fgeo[(size_t)(7 + d) * FS + g] =
                        (T)((xf + m.nbShift[(size_t)f * 3 + d]) - m.cellCenter[(size_t)nbo * 3 + d]);
            }
            // WALE length scale squared of the face (DP/computeViscousStresses.cu:54-56)
            const double vAvg = (bc == 0) ? (m.volume[own] + m.volume[nbo]) * 0.5 : m.volume[own];
            const double ls = 0.325 * pow(vAvg, 0.3333333333333);
            fgeo[10 * FS + g] = (T)(ls * ls);
        }
        // slot -> face, and each cell's sum of outward n A (closes to rounding on a closed cell)
        std::vector<double> clo(3 * (size_t)n, 0.0);
        for (int i = 0; i < n; i++) {
            const int o = m.new2old[i];
            const int nfc = flags[i] & 7;
            for (int k = 0; k < nfc; k++) {
                const int f = elFc2fc[(size_t)o * 6 + k];
                slotFace[(size_t)i * nSlots + k] = gFace[f];
                const double sg = ((flags[i] >> (3 + k)) & 1) ? 1.0 : -1.0;
                for (int d = 0; d < 3; d++) clo[(size_t)d * n + i] += sg * m.n[(size_t)f * 3 + d] * m.area[f];
            }
        }
        std::vector<T> closure(3 * (size_t)n);
        for (size_t q = 0; q < closure.size(); q++) closure[q] = (T)clo[q];
        // shared-memory staging plan: per block of B consecutive cells, the list of face
        // neighbours outside the block and each slot's index among the staged records
        const int B = StageCells<T>::value;
        const int nBlk = (n + B - 1) / B;
        std::vector<int32_t> haloStart(nBlk + 1, 0), haloIds;
        std::vector<int16_t> slotLocal(S, -1);
        haloIds.reserve((size_t)n * 2);
        int maxHalo = 0;
        {
            std::vector<int32_t> stamp(n, -1), pos(n, 0);
            for (int b = 0; b < nBlk; b++) {
                const int lo = b * B, hi = std::min(n, lo + B);
                int H = 0;
                for (int i = lo; i < hi; i++) {
                    const int nfc = flags[i] & 7;
                    for (int k = 0; k < nfc; k++) {
                        const size_t q = (size_t)i * nSlots + k;
                        const int nb = nbr[q];
                        if (nb < 0) {
                            slotLocal[q] = (int16_t)nb;   // -bc
                            continue;
                        }
                        if (nb >= lo && nb < hi) {
                            slotLocal[q] = (int16_t)(nb - lo);
                        } else {
                            if (stamp[nb] != b) {
                                stamp[nb] = b;
                                pos[nb] = H++;
                                haloIds.push_back(nb);
                            }
                            if (B + pos[nb] > 32767) return set_err(FG_ERR_MESH, "staging halo too large");
                            slotLocal[q] = (int16_t)(B + pos[nb]);
                        }
                    }
                }
                haloStart[b + 1] = (int32_t)haloIds.size();
                maxHalo = std::max(maxHalo, H);
            }
        }
        FG_CUDA_TRY(cudaSetDevice(device));
        FG_CUDA_TRY(dHaloStart.alloc((size_t)(nBlk + 1) * sizeof(int32_t)));
        FG_CUDA_TRY(dHaloIds.alloc(std::max<size_t>(haloIds.size(), 1) * sizeof(int32_t)));
        FG_CUDA_TRY(dSlotLocal.alloc(S * sizeof(int16_t)));
        FG_CUDA_TRY(cudaMemcpy(dHaloStart.p, haloStart.data(), haloStart.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
        if (!haloIds.empty())
            FG_CUDA_TRY(cudaMemcpy(dHaloIds.p, haloIds.data(), haloIds.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
        FG_CUDA_TRY(cudaMemcpy(dSlotLocal.p, slotLocal.data(), S * sizeof(int16_t), cudaMemcpyHostToDevice));
        dm.blockCells = B;
        dm.maxHalo = maxHalo;
        dm.haloStart = dHaloStart.as<int32_t>();
        dm.haloIds = dHaloIds.as<int32_t>();
        dm.slotLocal = dSlotLocal.as<int16_t>();
        FG_CUDA_TRY(dNbr.alloc(S * sizeof(int32_t)));
        FG_CUDA_TRY(dFlags.alloc((size_t)n * sizeof(int32_t)));
        FG_CUDA_TRY(dGeo.alloc(6 * GS * sizeof(T)));
        FG_CUDA_TRY(dVol.alloc((size_t)n * sizeof(double)));
        FG_CUDA_TRY(dVolP.alloc((size_t)n * sizeof(double)));
        FG_CUDA_TRY(dNew2Old.alloc((size_t)n * sizeof(int32_t)));
        FG_CUDA_TRY(cudaMemcpy(dNbr.p, nbr.data(), S * sizeof(int32_t), cudaMemcpyHostToDevice));
        FG_CUDA_TRY(cudaMemcpy(dFlags.p, flags.data(), (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice));
        FG_CUDA_TRY(cudaMemcpy(dGeo.p, geo.data(), 6 * GS * sizeof(T), cudaMemcpyHostToDevice));
        FG_CUDA_TRY(cudaMemcpy(dVol.p, vol.data(), (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
        FG_CUDA_TRY(cudaMemcpy(dVolP.p, volP.data(), (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
        FG_CUDA_TRY(cudaMemcpy(dNew2Old.p, m.new2old.data(), (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice));
        FG_CUDA_TRY(dFIdx.alloc(2 * (size_t)nF * sizeof(int32_t)));
        FG_CUDA_TRY(dFGeo.alloc(11 * FS * sizeof(T)));
        FG_CUDA_TRY(dSlotFace.alloc(S * sizeof(int32_t)));
        FG_CUDA_TRY(dClosure.alloc(3 * (size_t)n * sizeof(T)));
        FG_CUDA_TRY(dFB.alloc((size_t)nF * FREC * sizeof(T)));
        FG_CUDA_TRY(cudaMemcpy(dFIdx.p, fIdx.data(), 2 * (size_t)nF * sizeof(int32_t), cudaMemcpyHostToDevice));
        FG_CUDA_TRY(cudaMemcpy(dFGeo.p, fgeo.data(), 11 * FS * sizeof(T), cudaMemcpyHostToDevice));
        FG_CUDA_TRY(cudaMemcpy(dSlotFace.p, slotFace.data(), S * sizeof(int32_t), cudaMemcpyHostToDevice));
        FG_CUDA_TRY(cudaMemcpy(dClosure.p, closure.data(), 3 * (size_t)n * sizeof(T), cudaMemcpyHostToDevice));
        FG_CUDA_TRY(cudaMemset(dFB.p, 0, (size_t)nF * FREC * sizeof(T)));
        const size_t u = (size_t)nU * NV * sizeof(double);
        FG_CUDA_TRY(dU.alloc(u));
        FG_CUDA_TRY(dU0.alloc(u));
        FG_CUDA_TRY(dRHS.alloc(u));
        FG_CUDA_TRY(dStage.alloc(u));
        FG_CUDA_TRY(dW[0].alloc((size_t)n * WREC * sizeof(T)));
        FG_CUDA_TRY(dW[1].alloc((size_t)n * WREC * sizeof(T)));
        FG_CUDA_TRY(dG.alloc((size_t)n * grec_alloc<T>() * sizeof(T)));
        FG_CUDA_TRY(dSig.alloc((size_t)n * sizeof(double)));
        FG_CUDA_TRY(dCellSig.alloc((size_t)n * sizeof(T)));
        FG_CUDA_TRY(dBlockMin.alloc((size_t)std::max(flux_blocks(n), cons_blocks(n)) * sizeof(double)));
        FG_CUDA_TRY(dScal.alloc(4 * sizeof(double)));   // dt, time, cons
        FG_CUDA_TRY(dCnt.alloc(8 * sizeof(int32_t)));
        FG_CUDA_TRY(dChk.alloc(sizeof(int32_t)));
        FG_CUDA_TRY(dOrdFlag.alloc((size_t)n));
        FG_CUDA_TRY(dOrdCnt.alloc((size_t)relax_order_blocks(n) * sizeof(int32_t)));
        FG_CUDA_TRY(dOrdOff.alloc((size_t)relax_order_blocks(n) * sizeof(int32_t)));
        FG_CUDA_TRY(dOrder.alloc((size_t)n * sizeof(int32_t)));
        FG_CUDA_TRY(dOrdTotal.alloc(sizeof(int32_t)));
        FG_CUDA_TRY(dPred.alloc((size_t)n * sizeof(float4)));
        FG_CUDA_TRY(dHullOk.alloc((size_t)n * sizeof(int32_t)));
        FG_CUDA_TRY(dTcErr.alloc(sizeof(int32_t)));
        FG_CUDA_TRY(cudaMemset(dTcErr.p, 0, sizeof(int32_t)));
        FG_CUDA_TRY(cudaMemset(dU.p, 0, u));
        FG_CUDA_TRY(cudaMemset(dU0.p, 0, u));
        FG_CUDA_TRY(cudaMemset(dRHS.p, 0, u));
        FG_CUDA_TRY(cudaMemset(dW[0].p, 0, (size_t)n * WREC * sizeof(T)));
        FG_CUDA_TRY(cudaMemset(dW[1].p, 0, (size_t)n * WREC * sizeof(T)));
        FG_CUDA_TRY(cudaMemset(dG.p, 0, (size_t)n * grec_alloc<T>() * sizeof(T)));
        const double scal[4] = {cs.dt, 0.0, 0.0, 0.0};
        FG_CUDA_TRY(cudaMemcpy(dScal.p, scal, sizeof(scal), cudaMemcpyHostToDevice));
        bytes = 0;
        for (DevBuf *b : {&dNbr, &dFlags, &dGeo, &dVol, &dVolP, &dNew2Old, &dU, &dU0, &dRHS, &dStage, &dW[0], &dW[1], &dG,
                          &dSig, &dCellSig, &dBlockMin, &dScal, &dCnt, &dHaloStart, &dHaloIds, &dSlotLocal, &dFIdx, &dFGeo,
                          &dSlotFace, &dClosure, &dFB, &dOrdFlag, &dOrdCnt, &dOrdOff, &dOrder, &dOrdTotal,
                          &dPred, &dHullOk, &dTcErr})
            bytes += b->bytes;
        dm.n = n;
        dm.nU = nU;
        dm.nG = nG;
        dm.nFEval = nFEval;
        dm.nSlots = nSlots;
        dm.nbr = dNbr.as<int32_t>();
        dm.flags = dFlags.as<int32_t>();
        T *g = dGeo.as<T>();
        dm.geoStride = GS;
        dm.aox = g + 0 * GS; dm.aoy = g + 1 * GS; dm.aoz = g + 2 * GS;
        dm.dcx = g + 3 * GS; dm.dcy = g + 4 * GS; dm.dcz = g + 5 * GS;
        dm.vol = dVol.as<double>();
        dm.volP = dVolP.as<double>();
        dm.nF = nF;
        dm.fStride = FS;
        dm.fOwn = dFIdx.as<int32_t>();
        dm.fNb = dFIdx.as<int32_t>() + nF;
        {
            const T *fg = dFGeo.as<T>();
            dm.fnx = fg; dm.fny = fg + FS; dm.fnz = fg + 2 * FS; dm.fA = fg + 3 * FS;
            for (int d = 0; d < 3; d++) {
                dm.fdo[d] = fg + (4 + d) * FS;
                dm.fdn[d] = fg + (7 + d) * FS;
            }
            dm.fLsSq = fg + 10 * FS;
        }
        dm.slotFace = dSlotFace.as<int32_t>();
        dm.closure = dClosure.as<T>();
        if (parted) {
            sendStart = m.sendStart;
            recvStart = m.recvStart;
            FG_CUDA_TRY(dSendCells.alloc(std::max<size_t>(m.sendCells.size(), 1) * sizeof(int32_t)));
            FG_CUDA_TRY(dRecvCells.alloc(std::max<size_t>(m.recvCells.size(), 1) * sizeof(int32_t)));
            if (!m.sendCells.empty())
                FG_CUDA_TRY(cudaMemcpy(dSendCells.p, m.sendCells.data(), m.sendCells.size() * sizeof(int32_t),
                                       cudaMemcpyHostToDevice));
            if (!m.recvCells.empty())
                FG_CUDA_TRY(cudaMemcpy(dRecvCells.p, m.recvCells.data(), m.recvCells.size() * sizeof(int32_t),
                                       cudaMemcpyHostToDevice));
            bytes += dSendCells.bytes + dRecvCells.bytes;
        }
        if (stage_kernels_setup<T>(dm) != 0)
            return set_err(FG_ERR_CUDA, "stage kernels need more shared memory than the device allows (halo " +
                                            std::to_string(maxHalo) + " cells)");
        return FG_OK;
    }

    int set_state(const double *U, cudaStream_t s, bool wait) override {
        const size_t ub = (size_t)nU * NV * sizeof(double);
        double *stage = dStage.as<double>();
        if (wait) {
            FG_CUDA_TRY(cudaMemcpyAsync(dStage.p, U, ub, cudaMemcpyHostToDevice, s));
        } else {
            if (!copyStream) {
                FG_CUDA_TRY(dStageIn.alloc(ub));
                bytes += dStageIn.bytes;
                FG_CUDA_TRY(cudaStreamCreateWithFlags(&copyStream, cudaStreamNonBlocking));
                FG_CUDA_TRY(cudaEventCreateWithFlags(&evInFree, cudaEventDisableTiming));
                FG_CUDA_TRY(cudaEventCreateWithFlags(&evCopied, cudaEventDisableTiming));
                FG_CUDA_TRY(cudaEventRecord(evInFree, s));
            }
            // the copy waits only until the previous asynchronous upload has been scattered; the
            // check and the scatter wait for the copy and follow the work queued on `s`
            FG_CUDA_TRY(cudaStreamWaitEvent(copyStream, evInFree, 0));
            FG_CUDA_TRY(cudaMemcpyAsync(dStageIn.p, U, ub, cudaMemcpyHostToDevice, copyStream));
            FG_CUDA_TRY(cudaEventRecord(evCopied, copyStream));
            FG_CUDA_TRY(cudaStreamWaitEvent(s, evCopied, 0));
            stage = dStageIn.as<double>();
        }
        // checked on the device; the scatter replaces the state only if every cell is usable
        prof_begin(FG_K_OTHER, s);
        launch_check_state(nU, stage, dChk.as<int32_t>(), s);
        prof_end(s);
        FG_LAUNCH_CHECK("set_state check");
        prof_begin(FG_K_OTHER, s);
        launch_scatter_state(nU, stage, dNew2Old.as<int32_t>(), dU.as<double>(), dChk.as<int32_t>(), dBad, s);
        prof_end(s);
        if (!wait) FG_CUDA_TRY(cudaEventRecord(evInFree, s));
        prof_begin(FG_K_OTHER, s);
        launch_prim<T>(nU, dU.as<double>(), dW[cur].as<T>(), (size_t)n, D, s);
        prof_end(s);
        FG_LAUNCH_CHECK("set_state");
        if (!wait) return FG_OK;
        FG_CUDA_TRY(cudaStreamSynchronize(s));
        if (hBad[1]) {
            const int rc = upload_error();
            hBad[1] = 0;   // reported here: the old state stays usable
            return rc;
        }
        return FG_OK;
    }
    int get_state(double *U, cudaStream_t s, bool wait) override {
        const size_t ub = (size_t)nU * NV * sizeof(double);
        if (wait) {
            prof_begin(FG_K_OTHER, s);
            launch_gather_state(nU, dU.as<double>(), dNew2Old.as<int32_t>(), dStage.as<double>(), s);
            prof_end(s);
            FG_LAUNCH_CHECK("get_state");
            FG_CUDA_TRY(cudaMemcpyAsync(U, dStage.p, ub, cudaMemcpyDeviceToHost, s));
            FG_CUDA_TRY(cudaStreamSynchronize(s));
            return FG_OK;
        }
        if (!downStream) {
            for (DevBuf &b : dStageOut) {
                FG_CUDA_TRY(b.alloc(ub));
                bytes += b.bytes;
            }
            FG_CUDA_TRY(cudaStreamCreateWithFlags(&downStream, cudaStreamNonBlocking));
            for (cudaEvent_t &e : evOutFree) {
                FG_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                FG_CUDA_TRY(cudaEventRecord(e, s));
            }
            FG_CUDA_TRY(cudaEventCreateWithFlags(&evGathered, cudaEventDisableTiming));
        }
        // the gather waits until the download two calls back has read this buffer; the copy
        // overlaps whatever the caller queues on `s` next
        const int b = outNext;
        outNext ^= 1;
        FG_CUDA_TRY(cudaStreamWaitEvent(s, evOutFree[b], 0));
        prof_begin(FG_K_OTHER, s);
        launch_gather_state(nU, dU.as<double>(), dNew2Old.as<int32_t>(), dStageOut[b].as<double>(), s);
        prof_end(s);
        FG_LAUNCH_CHECK("get_state");
        FG_CUDA_TRY(cudaEventRecord(evGathered, s));
        FG_CUDA_TRY(cudaStreamWaitEvent(downStream, evGathered, 0));
        FG_CUDA_TRY(cudaMemcpyAsync(U, dStageOut[b].p, ub, cudaMemcpyDeviceToHost, downStream));
        FG_CUDA_TRY(cudaEventRecord(evOutFree[b], downStream));
        return FG_OK;
    }
    StageCoef coef(int irk, int writeU0) const {
        StageCoef sc;
        sc.rk = (cs.rkSteps == 3) ? 3 : 1;
        sc.irk = irk;
        sc.writeU0 = writeU0;
        sc.neglectZ = (cs.neglectZ == 1);
        return sc;
    }
    int gradients(cudaStream_t s) override {
        Fields<T> f = fields(cur);
        prof_begin(FG_K_GRAD, s);
        launch_grad<T>(dm, f, P, s);
        prof_end(s);
        FG_LAUNCH_CHECK("gradients");
        return FG_OK;
    }
    int flux(int mode, int wantSignal, int irk, int writeU0, cudaStream_t s) override {
        Fields<T> f = fields(cur);
        prof_begin(FG_K_FLUX, s);
        launch_face<T>(dm, f, P, wantSignal, s);
        prof_end(s);
        prof_begin(FG_K_GATHER, s);
        launch_gather<T>(dm, f, D, mode, wantSignal, mode == FLUX_RHS ? coef(0, 0) : coef(irk, writeU0), s);
        prof_end(s);
        FG_LAUNCH_CHECK("flux");
        if (mode != FLUX_RHS) cur ^= 1;
        return FG_OK;
    }
    int halo_exchange(int field, cudaStream_t s) override {
        if (!halo.exchange)
            return set_err(FG_ERR_ARG, "partitioned mesh: set the transport with fg_solver_set_halo first");
        if (field != FG_HALO_W) return set_err(FG_ERR_ARG, "partitioned run: only primitive records are exchanged");
        T *rec = dW[cur].as<T>();
        const int stride = WREC;
        const int vpvRec = vpv<T>();
        const int nSend = sendStart.back(), nRecv = recvStart.back();
        prof_begin(FG_K_OTHER, s);
        launch_halo_pack<T>(rec, (size_t)n, stride, vpvRec, dSendCells.as<int32_t>(), nSend, static_cast<T *>(haloSend), s);
        prof_end(s);
        FG_LAUNCH_CHECK("halo pack");
        FG_CUDA_TRY(cudaStreamSynchronize(s));
        if (halo.exchange(halo.ctx, field, (int64_t)stride * (int64_t)sizeof(T), s) != 0)
            return set_err(FG_ERR_CUDA, "partitioned run: halo exchange failed");
        prof_begin(FG_K_OTHER, s);
        launch_halo_unpack<T>(rec, (size_t)n, stride, vpvRec, dRecvCells.as<int32_t>(), nRecv,
                            static_cast<const T *>(haloRecv), s);
        prof_end(s);
        FG_LAUNCH_CHECK("halo unpack");
        return FG_OK;
    }
    void halo_bytes(int64_t *send, int64_t *recv) const override {
        const int64_t rb = (int64_t)WREC * (int64_t)sizeof(T);   // primitive records only
        *send = parted ? rb * sendStart.back() : 0;
        *recv = parted ? rb * recvStart.back() : 0;
    }
    int compute_rhs(int wantSignal, cudaStream_t s) override {
        int rc;
        if ((rc = gradients_halo(s))) return rc;
        return flux(FLUX_RHS, wantSignal, 0, 0, s);
    }
    int time_step(double *dtOut, cudaStream_t s) override {
        prof_begin(FG_K_DT, s);
        launch_dt_finalize(dBlockMin.as<double>(), flux_blocks(nU), cs.cfl, cs.maxDt, dScal.as<double>(), s);
        prof_end(s);
        FG_LAUNCH_CHECK("time_step");
        if (parted) {
            // the whole mesh's dt: the minimum over the parts
            double dt = 0;
            FG_CUDA_TRY(cudaMemcpyAsync(&dt, dScal.p, sizeof(double), cudaMemcpyDeviceToHost, s));
            FG_CUDA_TRY(cudaStreamSynchronize(s));
            int rc = reduce(FG_REDUCE_MIN, &dt);
            if (rc) return rc;
            FG_CUDA_TRY(cudaMemcpyAsync(dScal.p, &dt, sizeof(double), cudaMemcpyHostToDevice, s));
            FG_CUDA_TRY(cudaStreamSynchronize(s));
            if (dtOut) *dtOut = dt;
            return FG_OK;
        }
        if (dtOut) {
            FG_CUDA_TRY(cudaMemcpyAsync(dtOut, dScal.p, sizeof(double), cudaMemcpyDeviceToHost, s));
            FG_CUDA_TRY(cudaStreamSynchronize(s));
        }
        return FG_OK;
    }
    int init_rk(cudaStream_t s) override {
        prof_begin(FG_K_OTHER, s);
        launch_copy_u0(nU, dU.as<double>(), dU0.as<double>(), s);
        prof_end(s);
        FG_LAUNCH_CHECK("init_rk");
        return FG_OK;
    }
    int update(int irk, int writeU0, cudaStream_t s) override {
        Fields<T> f = fields(cur);
        prof_begin(FG_K_UPDATE, s);
        launch_update<T>(dm, f, D, coef(irk, writeU0), s);
        prof_end(s);
        FG_LAUNCH_CHECK("update");
        cur ^= 1;
        return FG_OK;
    }
    int dt_stage(int irk, int writeU0, cudaStream_t s) override {
        // the face kernel also keeps each cell's maximum face signal, so the new dt is known before
        // the fused gather + RK update of this stage (no residual buffer, no separate update pass);
        // dt, signal and the updated state equal those of compute_rhs + time_step + update
        int rc;
        if ((rc = gradients_halo(s))) return rc;
        Fields<T> f = fields(cur);
        FG_CUDA_TRY(cudaMemsetAsync(dCellSig.p, 0, (size_t)n * sizeof(T), s));
        prof_begin(FG_K_FLUX, s);
        launch_face<T>(dm, f, P, 2, s);
        prof_end(s);
        prof_begin(FG_K_DT, s);
        launch_cell_cfl<T>(dm, f, s);
        prof_end(s);
        FG_LAUNCH_CHECK("cell cfl");
        if ((rc = time_step(nullptr, s))) return rc;
        prof_begin(FG_K_GATHER, s);
        launch_gather<T>(dm, f, D, FLUX_FUSED, 0, coef(irk, writeU0), s);
        prof_end(s);
        FG_LAUNCH_CHECK("dt stage");
        cur ^= 1;
        return FG_OK;
    }
    int stage(int irk, int writeU0, cudaStream_t s) override {
        int rc;
        if ((rc = gradients_halo(s))) return rc;
        return flux(FLUX_FUSED, 0, irk, writeU0, s);
    }
    int relax(fg_relax_stats *st, cudaStream_t s) override {
        FG_CUDA_TRY(cudaMemsetAsync(dCnt.p, 0, 8 * sizeof(int32_t), s));
        SurrogateDev S{};
        if (sg) {
            const int rc = surrogate_view(sg, &S);
            if (rc != FG_OK) return rc;
            S.relTol = sgTol;
            S.polishIters = sgIters;
        }
        RelaxLog L{logX.as<float>(), logY.as<float>(), logCap > 0 ? logCnt.as<unsigned long long>() : nullptr, logCap};
        // with the surrogate, where its polish runs: inside the relaxation kernel, which then
        // needs the polish's register budget (4 resident blocks), or as a pass of its own before
        // it, which costs a launch and a second read of the chemical cells' states but leaves the
        // relaxation kernel the thermal Newton's budget (6 blocks).  Measured: the separate pass
        // is faster when few cells are chemical (4 M-tet bubble, about 1,000 chemical cells: 2.51e9
        // -> 2.60e9 cell-updates/s), the polish inside when many are (96^3 box, 39 % chemical:
        // 0.61 against 0.75 ms per relaxation).  The results are bitwise the same either way, so
        // the automatic choice may use whatever counters have reached the host.
        int pass = sgPass == FG_SG_PASS_SEPARATE;
        const bool autoPass = sg && sgPass == FG_SG_PASS_AUTO;
        if (autoPass) {
            if (!hCntPrev) {
                FG_CUDA_TRY(cudaHostAlloc((void **)&hCntPrev, 8 * sizeof(int32_t), cudaHostAllocDefault));
                FG_CUDA_TRY(cudaEventCreateWithFlags(&evCnt, cudaEventDisableTiming));
            } else if (cntPending && cudaPeekAtLastError() == cudaSuccess) {
                const cudaError_t q = cudaEventQuery(evCnt);
                if (q == cudaSuccess) {
                    sgAutoPass = (int64_t)hCntPrev[1] * kSparseChemInv < (int64_t)nU;
                    cntPending = false;
                } else if (q == cudaErrorNotReady) {
                    // not an error: clear it where the query itself left it as the last error
                    if (cudaPeekAtLastError() == cudaErrorNotReady) (void)cudaGetLastError();
                } else {
                    return set_err(FG_ERR_CUDA, std::string("relaxation counters: ") + cudaGetErrorString(q));
                }
            }
            pass = sgAutoPass;
        }
        const RelaxOrder O{dOrdFlag.as<uint8_t>(), dOrdCnt.as<int32_t>(), dOrdOff.as<int32_t>(), dOrder.as<int32_t>(),
                           dOrdTotal.as<int32_t>(), dPred.as<float4>(), dHullOk.as<int32_t>(), dTcErr.as<int32_t>(),
                           pass};
        prof_begin(FG_K_RELAX, s);
        const int k = launch_relax<T>(nU, dU.as<double>(), dW[cur].as<T>(), (size_t)n, D, R, dCnt.as<int32_t>(), S, L, O, s);
        prof_end(s);
        launches += k - 1;
        FG_LAUNCH_CHECK("relaxation");
        if (autoPass && !cntPending) {
            FG_CUDA_TRY(cudaMemcpyAsync(hCntPrev, dCnt.p, 8 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            FG_CUDA_TRY(cudaEventRecord(evCnt, s));
            cntPending = true;
        }
        if (st) {
            FG_CUDA_TRY(cudaStreamSynchronize(s));
            return relax_counts(st);
        }
        return FG_OK;
    }
    int relax_counts(fg_relax_stats *st) override {
        int32_t h[8];
        FG_CUDA_TRY(cudaDeviceSynchronize());
        FG_CUDA_TRY(cudaMemcpy(h, dCnt.p, sizeof(h), cudaMemcpyDeviceToHost));
        st->nTherm = h[0];
        st->nChem = h[1];
        st->nAbort = h[2];
        st->nIter = h[3];
        st->nSurrogate = h[4];
        st->nFallback = h[5];
        st->nPolish = h[6];
        return FG_OK;
    }
    int probe(double *out4, cudaStream_t s) override {
        if (parted) return set_err(FG_ERR_UNSUPPORTED, "fg_probe: not available on a part of a partitioned mesh");
        if (!dProbe.p) {
            FG_CUDA_TRY(dProbe.alloc(((size_t)4 * cons_blocks(nU) + 4) * sizeof(double)));
            bytes += dProbe.bytes;
        }
        double *o = dProbe.as<double>() + (size_t)4 * cons_blocks(nU);
        prof_begin(FG_K_OTHER, s);
        launch_probe(nU, dU.as<double>(), dVol.as<double>(), D, dProbe.as<double>(), o, s);
        prof_end(s);
        launches++;  // two kernels
        FG_LAUNCH_CHECK("probe");
        FG_CUDA_TRY(cudaMemcpyAsync(out4, o, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
        FG_CUDA_TRY(cudaStreamSynchronize(s));
        return FG_OK;
    }
    int cons(int ivar, double *out, cudaStream_t s) override {
        double *o = dScal.as<double>() + 2;
        prof_begin(FG_K_CONS, s);
        launch_cons(nU, ivar, dU.as<double>(), dVol.as<double>(), dBlockMin.as<double>(), o, s);
        prof_end(s);
        launches++;  // two kernels
        FG_LAUNCH_CHECK("cons_calc");
        if (parted) {
            // the whole mesh's integral: the sum over the parts
            double v = 0;
            FG_CUDA_TRY(cudaMemcpyAsync(&v, o, sizeof(double), cudaMemcpyDeviceToHost, s));
            FG_CUDA_TRY(cudaStreamSynchronize(s));
            int rc = reduce(FG_REDUCE_SUM, &v);
            if (rc) return rc;
            FG_CUDA_TRY(cudaMemcpyAsync(o, &v, sizeof(double), cudaMemcpyHostToDevice, s));
            FG_CUDA_TRY(cudaStreamSynchronize(s));
            if (out) *out = v;
            return FG_OK;
        }
        if (out) {
            FG_CUDA_TRY(cudaMemcpyAsync(out, o, sizeof(double), cudaMemcpyDeviceToHost, s));
            FG_CUDA_TRY(cudaStreamSynchronize(s));
        }
        return FG_OK;
    }
    int advance_time(cudaStream_t s) override {
        prof_begin(FG_K_OTHER, s);
        k_advance_time<<<1, 1, 0, s>>>(dScal.as<double>(), dScal.as<double>() + 1);
        prof_end(s);
        FG_LAUNCH_CHECK("advance_time");
        return FG_OK;
    }
    int get_time(double *dt, double *t) override {
        double h[2];
        FG_CUDA_TRY(cudaDeviceSynchronize());
        FG_CUDA_TRY(cudaMemcpy(h, dScal.p, sizeof(h), cudaMemcpyDeviceToHost));
        if (dt) *dt = h[0];
        if (t) *t = h[1];
        return FG_OK;
    }
    int set_dt(double dt) override {
        FG_CUDA_TRY(cudaDeviceSynchronize());
        FG_CUDA_TRY(cudaMemcpy(dScal.p, &dt, sizeof(double), cudaMemcpyHostToDevice));
        return FG_OK;
    }
    int set_time(double t) override {
        FG_CUDA_TRY(cudaDeviceSynchronize());
        FG_CUDA_TRY(cudaMemcpy(dScal.as<double>() + 1, &t, sizeof(double), cudaMemcpyHostToDevice));
        return FG_OK;
    }
    int field_vars(double *out) override {
        DevBuf dOut, dCp;
        FG_CUDA_TRY(dOut.alloc((size_t)nU * 13 * sizeof(double)));
        FG_CUDA_TRY(dCp.alloc(2 * sizeof(double)));
        FG_CUDA_TRY(cudaMemcpy(dCp.p, cs.Cp, 2 * sizeof(double), cudaMemcpyHostToDevice));
        k_field_vars<T><<<(nU + 255) / 256, 256>>>(nU, dU.as<double>(), dG.as<T>(), (size_t)n, dNew2Old.as<int32_t>(), D,
                                                  dCp.as<double>(), dOut.as<double>());
        FG_LAUNCH_CHECK("field_vars");
        launches++;
        FG_CUDA_TRY(cudaDeviceSynchronize());
        FG_CUDA_TRY(cudaMemcpy(out, dOut.p, (size_t)nU * 13 * sizeof(double), cudaMemcpyDeviceToHost));
        return FG_OK;
    }
    int get_rhs(double *rhs) override {
        launch_gather_state(nU, dRHS.as<double>(), dNew2Old.as<int32_t>(), dStage.as<double>(), 0);
        FG_LAUNCH_CHECK("get_rhs");
        FG_CUDA_TRY(cudaMemcpy(rhs, dStage.p, (size_t)nU * NV * sizeof(double), cudaMemcpyDeviceToHost));
        return FG_OK;
    }
    int get_limited(double *grad, double *theta) override {
        FG_CUDA_TRY(cudaDeviceSynchronize());
        std::vector<T> g((size_t)n * grec_alloc<T>());
        std::vector<int32_t> n2o(nU);
        FG_CUDA_TRY(cudaMemcpy(g.data(), dG.p, g.size() * sizeof(T), cudaMemcpyDeviceToHost));
        FG_CUDA_TRY(cudaMemcpy(n2o.data(), dNew2Old.p, (size_t)nU * sizeof(int32_t), cudaMemcpyDeviceToHost));
        for (int i = 0; i < nU; i++) {
            const size_t o = (size_t)n2o[i];
            for (int v = 0; v < NV; v++) {
                if (theta) theta[o * NV + v] = (v < NP) ? (double)g[grec_index<T>((size_t)n, i, v)] : 0.0;
                for (int d = 0; d < 3; d++)
                    if (grad) grad[(o * NV + v) * 3 + d] = (v < NP) ? (double)g[grec_index<T>((size_t)n, i, NP + 3 * v + d)] : 0.0;
            }
        }
        return FG_OK;
    }
    int get_signal(double *sig) override {
        FG_CUDA_TRY(cudaDeviceSynchronize());
        std::vector<double> h(nU);
        std::vector<int32_t> n2o(nU);
        FG_CUDA_TRY(cudaMemcpy(h.data(), dSig.p, (size_t)nU * sizeof(double), cudaMemcpyDeviceToHost));
        FG_CUDA_TRY(cudaMemcpy(n2o.data(), dNew2Old.p, (size_t)nU * sizeof(int32_t), cudaMemcpyDeviceToHost));
        for (int i = 0; i < nU; i++) sig[n2o[i]] = h[i];
        return FG_OK;
    }
};

}  // namespace fg

// ------------------------------------------------------------------ C ABI
namespace fg {
// error message setter for the other translation units of the C ABI
int set_error(int code, const std::string &msg) { return set_err(code, msg); }
}  // namespace fg

extern "C" {

const char *fg_last_error(void) { return g_err.c_str(); }

void fg_case_default(fg_case *c) {
    // values hard-coded in DP/buildInput.cu:10-69
    if (!c) return;
    memset(c, 0, sizeof(*c));
    c->dt = 0.0;
    c->adaptDt = 1;
    c->adaptDtItr = 100;
    c->maxDt = 1e-8;
    c->cfl = 0.1;
    c->avfMin = 1e-4;
    c->rkSteps = 1;
    c->finalTime = 3.5e-3;
    c->exportTime = 2.0e-5;
    c->restartStep = 100000;
    c->restartFlag = 0;
    c->neglectX = 0;
    c->neglectY = 0;
    c->neglectZ = 0;
    c->nMaterials = 2;
    c->NEQ = 10;
    c->scale = 0.001;
    c->viscFlag = 1;
    c->turbulence = 1;
    c->woodsFlag = 1;
    c->thermFntRlxFlag = 0;
    c->thermRlxRate = 0.5;
    c->thermUrf = 0.8;
    c->thermItrMax = 25;
    c->chemFlag = 1;
    c->chemFntRlxFlag = 0;
    c->chemRlxRate = 0;
    c->chemUrf = 0.5;
    c->chemItrMax = 40;
    c->chemCondesation = 0;
    c->chemLimit = 20e-4;
    c->consCalcFlag = 1;
    c->consCalcIvar = 9;
    c->satTempUrf = 0.8;
    c->gamma[0] = 2.17290;
    c->pInf[0] = 114907765;
    c->Cp[0] = 1854.4;
    c->eta[0] = -302568.5557;
    c->satConst[0] = -488.9933492;
    c->dynVisc[0] = 1.8e-4;
    c->gamma[1] = 1.4588;
    c->pInf[1] = 0.0;
    c->Cp[1] = 965.98;
    c->eta[1] = 9741.04362;
    c->satConst[1] = 297.63826;
    c->dynVisc[1] = 1.99e-5;
}

int fg_mesh_load_neu(const char *path, const fg_mesh_opts *opts, fg_mesh **out) {
    if (!path || !out) return set_err(FG_ERR_ARG, "fg_mesh_load_neu: null argument");
    *out = nullptr;
    fg_mesh_opts o{};
    o.scale = 1.0;
    o.renumber = FG_RENUMBER_MORTON;
    if (opts) o = *opts;
    if (!(o.scale > 0)) return set_err(FG_ERR_ARG, "fg_mesh_load_neu: scale must be > 0");
    std::unique_ptr<fg_mesh> m(new fg_mesh());
    std::string err;
    int rc = fg::read_neu(path, o.scale, m->m, err);
    if (rc != FG_OK) return set_err(rc, err);
    rc = o.gpu ? fg::finish_mesh_gpu(m->m, o, err) : fg::finish_mesh(m->m, o, err);
    if (rc != FG_OK) return set_err(rc, err);
    *out = m.release();
    return FG_OK;
}

int fg_mesh_build(int32_t nNodes, const double *nodes, int32_t nElem, const int32_t *elNN, const int32_t *elNodes,
                  const int32_t *elBc, const fg_mesh_opts *opts, fg_mesh **out) {
    if (!nodes || !elNN || !elNodes || !elBc || !out) return set_err(FG_ERR_ARG, "fg_mesh_build: null argument");
    *out = nullptr;
    fg_mesh_opts o{};
    o.scale = 1.0;
    o.renumber = FG_RENUMBER_MORTON;
    if (opts) o = *opts;
    if (!(o.scale > 0)) return set_err(FG_ERR_ARG, "fg_mesh_build: scale must be > 0");
    std::unique_ptr<fg_mesh> m(new fg_mesh());
    std::string err;
    int rc = fg::mesh_from_arrays(nNodes, nodes, nElem, elNN, elNodes, elBc, o.scale, m->m, err);
    if (rc != FG_OK) return set_err(rc, err);
    rc = o.gpu ? fg::finish_mesh_gpu(m->m, o, err) : fg::finish_mesh(m->m, o, err);
    if (rc != FG_OK) return set_err(rc, err);
    *out = m.release();
    return FG_OK;
}

int fg_mesh_info_get(const fg_mesh *mm, fg_mesh_info *info) {
    if (!mm || !info) return set_err(FG_ERR_ARG, "fg_mesh_info_get: null argument");
    const fg::Mesh &m = mm->m;
    info->nElem = m.nElem;
    info->nNodes = m.nNodes;
    info->nFcs = m.nFcs;
    info->nBoundary = m.nBoundary;
    info->nPeriodic = m.nPeriodic;
    info->maxFaces = m.maxFaces;
    info->nTet = m.nTet;
    info->nPyr = m.nPyr;
    info->nPrism = m.nPrism;
    info->nHex = m.nHex;
    return FG_OK;
}

int fg_mesh_view_get(const fg_mesh *mm, fg_mesh_view *v) {
    if (!mm || !v) return set_err(FG_ERR_ARG, "fg_mesh_view_get: null argument");
    const fg::Mesh &m = mm->m;
    v->nElem = m.nElem;
    v->nFcs = m.nFcs;
    v->fc2el = m.fc2el.data();
    v->boundCond = m.boundCond.data();
    v->cellCenter = m.cellCenter.data();
    v->fcCenter = m.fcCenter.data();
    v->n = m.n.data();
    v->nt1 = m.nt1.data();
    v->nt2 = m.nt2.data();
    v->area = m.area.data();
    v->volume = m.volume.data();
    v->nbShift = m.nbShift.data();
    return FG_OK;
}

int fg_mesh_permutation(const fg_mesh *mm, int32_t *new2old, int32_t n) {
    if (!mm || !new2old) return set_err(FG_ERR_ARG, "fg_mesh_permutation: null argument");
    if (n != mm->m.nElem) return set_err(FG_ERR_ARG, "fg_mesh_permutation: size mismatch");
    memcpy(new2old, mm->m.new2old.data(), sizeof(int32_t) * (size_t)n);
    return FG_OK;
}

void fg_mesh_free(fg_mesh *m) { delete m; }

int fg_mesh_partition(const fg_mesh *mm, int32_t nParts, int32_t part, fg_mesh **out) {
    if (!mm || !out) return set_err(FG_ERR_ARG, "fg_mesh_partition: null argument");
    *out = nullptr;
    std::unique_ptr<fg_mesh> l(new fg_mesh());
    std::string err;
    const int rc = fg::partition_mesh(mm->m, nParts, part, l->m, err);
    if (rc != FG_OK) return set_err(rc, err);
    *out = l.release();
    return FG_OK;
}
int fg_mesh_partition_info(const fg_mesh *mm, fg_partition_info *info) {
    if (!mm || !info) return set_err(FG_ERR_ARG, "fg_mesh_partition_info: null argument");
    const fg::Mesh &m = mm->m;
    info->nParts = m.nParts;
    info->part = m.part;
    info->nOwned = m.owned();
    info->nGhost = m.nElem - m.owned();
    info->nSend = m.sendStart.empty() ? 0 : m.sendStart.back();
    info->nRecv = m.recvStart.empty() ? 0 : m.recvStart.back();
    info->nGhost1 = m.nOwned < 0 ? 0 : m.nGhost1;
    return FG_OK;
}
int fg_mesh_partition_maps(const fg_mesh *mm, int32_t *cellGlobal, int32_t *sendStart, int32_t *sendCells,
                           int32_t *recvStart, int32_t *recvCells) {
    if (!mm) return set_err(FG_ERR_ARG, "fg_mesh_partition_maps: null mesh");
    const fg::Mesh &m = mm->m;
    if (m.nOwned < 0) {
        // a whole mesh: one part owning every cell, no halo
        if (cellGlobal) std::iota(cellGlobal, cellGlobal + m.nElem, 0);
        if (sendStart) sendStart[0] = sendStart[1] = 0;
        if (recvStart) recvStart[0] = recvStart[1] = 0;
        return FG_OK;
    }
    if (cellGlobal) std::copy(m.cellGlobal.begin(), m.cellGlobal.end(), cellGlobal);
    if (sendStart) std::copy(m.sendStart.begin(), m.sendStart.end(), sendStart);
    if (sendCells) std::copy(m.sendCells.begin(), m.sendCells.end(), sendCells);
    if (recvStart) std::copy(m.recvStart.begin(), m.recvStart.end(), recvStart);
    if (recvCells) std::copy(m.recvCells.begin(), m.recvCells.end(), recvCells);
    return FG_OK;
}

int fg_solver_create(const fg_mesh *m, const fg_case *c, int32_t precision, int32_t device, fg_solver **out) {
    if (!m || !c || !out) return set_err(FG_ERR_ARG, "fg_solver_create: null argument");
    *out = nullptr;
    if (c->rkSteps != 1 && c->rkSteps != 3) return set_err(FG_ERR_UNSUPPORTED, "rkSteps must be 1 or 3");
    if (c->thermFntRlxFlag != 0 || c->chemFntRlxFlag != 0)
        return set_err(FG_ERR_UNSUPPORTED, "finite-rate relaxation (thermFntRlxFlag/chemFntRlxFlag) is not supported");
    if (c->adaptDt == 1 && c->adaptDtItr <= 0) return set_err(FG_ERR_ARG, "adaptDtItr must be > 0");
    if (m->m.maxFaces > fg::MAXSLOT) return set_err(FG_ERR_MESH, "cell with more than 6 faces");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_err(FG_ERR_CUDA, "no CUDA device available (the device path has no CPU fallback)");
    if (device < 0 || device >= ndev) return set_err(FG_ERR_ARG, "device index out of range");
    std::unique_ptr<fg_solver> s;
    if (precision == FG_PREC_FP64) s.reset(new fg::SolverT<double>());
    else if (precision == FG_PREC_MIXED) s.reset(new fg::SolverT<float>());
    if (s) s->precision = precision;
    else return set_err(FG_ERR_ARG, "unknown precision");
    s->device = device;
    s->cs = *c;
    int rc = s->init(m->m);
    if (rc != FG_OK) return rc;
    *out = s.release();
    return FG_OK;
}

int fg_solver_destroy(fg_solver *s) {
    if (!s) return FG_OK;
    cudaSetDevice(s->device);
    cudaDeviceSynchronize();
    delete s;
    return FG_OK;
}

int fg_solver_memory(const fg_solver *s, uint64_t *bytes) {
    if (!s || !bytes) return set_err(FG_ERR_ARG, "fg_solver_memory: null argument");
    *bytes = s->bytes;
    return FG_OK;
}
int fg_halo_buffer_bytes(const fg_solver *s, int64_t *sendBytes, int64_t *recvBytes) {
    if (!s || !sendBytes || !recvBytes) return set_err(FG_ERR_ARG, "fg_halo_buffer_bytes: null argument");
    s->halo_bytes(sendBytes, recvBytes);
    return FG_OK;
}
int fg_solver_set_halo(fg_solver *s, const fg_halo_ops *ops, void *sendBuf, void *recvBuf) {
    if (!s || !ops || !ops->exchange || !ops->allreduce) return set_err(FG_ERR_ARG, "fg_solver_set_halo: null argument");
    if (!s->parted) return set_err(FG_ERR_ARG, "fg_solver_set_halo: the solver's mesh is not a part (fg_mesh_partition)");
    int64_t sb = 0, rb = 0;
    s->halo_bytes(&sb, &rb);
    if ((sb > 0 && !sendBuf) || (rb > 0 && !recvBuf)) return set_err(FG_ERR_ARG, "fg_solver_set_halo: null buffer");
    s->halo = *ops;
    s->haloSend = sendBuf;
    s->haloRecv = recvBuf;
    return FG_OK;
}

#define FG_ENTER(s)                                                                   \
    do {                                                                              \
        if (!(s)) return set_err(FG_ERR_ARG, "null solver");                          \
        if (cudaSetDevice((s)->device) != cudaSuccess) return set_err(FG_ERR_CUDA, "cudaSetDevice failed"); \
    } while (0)

int fg_set_state(fg_solver *s, const double *U, void *stream) {
    FG_ENTER(s);
    if (!U) return set_err(FG_ERR_ARG, "fg_set_state: null U");
    return s->set_state(U, (cudaStream_t)stream, true);
}
int fg_set_state_async(fg_solver *s, const double *U, void *stream) {
    FG_ENTER(s);
    if (!U) return set_err(FG_ERR_ARG, "fg_set_state_async: null U");
    return s->set_state(U, (cudaStream_t)stream, false);
}
int fg_get_state(fg_solver *s, double *U, void *stream) {
    FG_ENTER(s);
    if (!U) return set_err(FG_ERR_ARG, "fg_get_state: null U");
    return s->get_state(U, (cudaStream_t)stream, true);
}
int fg_get_state_async(fg_solver *s, double *U, void *stream) {
    FG_ENTER(s);
    if (!U) return set_err(FG_ERR_ARG, "fg_get_state_async: null U");
    return s->get_state(U, (cudaStream_t)stream, false);
}
int fg_state_join(fg_solver *s, void *stream) {
    FG_ENTER(s);
    return s->state_join((cudaStream_t)stream);
}
int fg_compute_rhs(fg_solver *s, int32_t want_signal, void *stream) {
    FG_ENTER(s);
    return s->compute_rhs(want_signal ? 1 : 0, (cudaStream_t)stream);
}
int fg_compute_time_step(fg_solver *s, double *dt_out, void *stream) {
    FG_ENTER(s);
    return s->time_step(dt_out, (cudaStream_t)stream);
}
int fg_init_rk(fg_solver *s, void *stream) {
    FG_ENTER(s);
    return s->init_rk((cudaStream_t)stream);
}
int fg_update(fg_solver *s, int32_t irk, void *stream) {
    FG_ENTER(s);
    if (irk < 0 || irk >= s->cs.rkSteps) return set_err(FG_ERR_ARG, "irk out of range");
    return s->update(irk, 0, (cudaStream_t)stream);
}
int fg_stage(fg_solver *s, int32_t irk, void *stream) {
    FG_ENTER(s);
    if (irk < 0 || irk >= s->cs.rkSteps) return set_err(FG_ERR_ARG, "irk out of range");
    return s->stage(irk, (s->cs.rkSteps == 3 && irk == 0) ? 1 : 0, (cudaStream_t)stream);
}
int fg_relaxation(fg_solver *s, fg_relax_stats *stats, void *stream) {
    FG_ENTER(s);
    return s->relax(stats, (cudaStream_t)stream);
}
int fg_solver_set_surrogate(fg_solver *s, const fg_surrogate *g, double relTol, int32_t polishIters) {
    FG_ENTER(s);
    if (g) {
        if (!(relTol > 0) || polishIters < 0 || polishIters > 20)
            return set_err(FG_ERR_ARG, "fg_solver_set_surrogate: relTol > 0 and 0 <= polishIters <= 20");
        if (fg::surrogate_device(g) != s->device)
            return set_err(FG_ERR_ARG, "fg_solver_set_surrogate: surrogate lives on another device");
        fg::SurrogateDev tmp{};
        const int rc = fg::surrogate_view(g, &tmp);
        if (rc != FG_OK) return rc;
    }
    s->sg = g;
    s->sgTol = relTol;
    s->sgIters = polishIters;
    return FG_OK;
}
int fg_solver_set_surrogate_pass(fg_solver *s, int32_t mode) {
    FG_ENTER(s);
    if (mode != FG_SG_PASS_AUTO && mode != FG_SG_PASS_FUSED && mode != FG_SG_PASS_SEPARATE)
        return set_err(FG_ERR_ARG, "fg_solver_set_surrogate_pass: mode is FG_SG_PASS_AUTO, _FUSED or _SEPARATE");
    s->sgPass = mode;
    return FG_OK;
}
int fg_relax_stats_read(fg_solver *s, fg_relax_stats *stats) {
    FG_ENTER(s);
    if (!stats) return set_err(FG_ERR_ARG, "fg_relax_stats_read: null argument");
    return s->relax_counts(stats);
}
int fg_relax_log(fg_solver *s, int64_t capacity) {
    FG_ENTER(s);
    if (capacity < 0 || capacity > ((int64_t)1 << 31)) return set_err(FG_ERR_ARG, "fg_relax_log: 0 <= capacity <= 2^31");
    s->logX.release();
    s->logY.release();
    s->logCnt.release();
    s->logCap = 0;
    if (capacity == 0) return FG_OK;
    FG_CUDA_TRY(s->logX.alloc((size_t)capacity * 3 * sizeof(float)));
    FG_CUDA_TRY(s->logY.alloc((size_t)capacity * 4 * sizeof(float)));
    FG_CUDA_TRY(s->logCnt.alloc(sizeof(unsigned long long)));
    FG_CUDA_TRY(cudaMemset(s->logCnt.p, 0, sizeof(unsigned long long)));
    s->logCap = capacity;
    return FG_OK;
}
int fg_relax_log_read(fg_solver *s, float *X, float *Y, int64_t cap, int64_t *count) {
    FG_ENTER(s);
    if (!count) return set_err(FG_ERR_ARG, "fg_relax_log_read: null count");
    *count = 0;
    if (s->logCap == 0) return FG_OK;
    unsigned long long c = 0;
    FG_CUDA_TRY(cudaDeviceSynchronize());
    FG_CUDA_TRY(cudaMemcpy(&c, s->logCnt.p, sizeof(c), cudaMemcpyDeviceToHost));
    const int64_t have = std::min<int64_t>((int64_t)c, s->logCap);
    const int64_t k = std::min<int64_t>(have, cap);
    if (k > 0) {
        if (!X || !Y) return set_err(FG_ERR_ARG, "fg_relax_log_read: null buffer");
        FG_CUDA_TRY(cudaMemcpy(X, s->logX.p, (size_t)k * 3 * sizeof(float), cudaMemcpyDeviceToHost));
        FG_CUDA_TRY(cudaMemcpy(Y, s->logY.p, (size_t)k * 4 * sizeof(float), cudaMemcpyDeviceToHost));
    }
    *count = k;
    return FG_OK;
}
int fg_cons_calc(fg_solver *s, int32_t ivar, double *out, void *stream) {
    FG_ENTER(s);
    if (ivar < 0 || ivar >= 10) return set_err(FG_ERR_ARG, "ivar out of range");
    return s->cons(ivar, out, (cudaStream_t)stream);
}
int fg_probe(fg_solver *s, fg_probe_out *out, void *stream) {
    FG_ENTER(s);
    if (!out) return set_err(FG_ERR_ARG, "fg_probe: null output");
    double v[4];
    const int rc = s->probe(v, (cudaStream_t)stream);
    if (rc != FG_OK) return rc;
    out->vapourVolume = v[0];
    out->maxPressure = v[1];
    out->minPressure = v[2];
    out->maxSpeed = v[3];
    return FG_OK;
}

int fg_get_time(fg_solver *s, double *dt, double *physicalTime, int32_t *iStep) {
    FG_ENTER(s);
    if (iStep) *iStep = s->iStep;
    return s->get_time(dt, physicalTime);
}
int fg_set_dt(fg_solver *s, double dt) {
    FG_ENTER(s);
    return s->set_dt(dt);
}

// ---- checkpoint / restart and field dump (binary; the reference writes ASCII with 11 digits,
// DP/restart.cu:113-152, and node-averaged Tecplot text, DP/export_plt.cu:95-174)
namespace {
const char kCkMagic[8] = {'F', 'G', 'C', 'K', 'P', 'T', '0', '1'};
const char kFdMagic[8] = {'F', 'G', 'F', 'I', 'E', 'L', 'D', '1'};
struct CkHeader {
    char magic[8];
    int32_t nElem, neq, iStep, precision;
    double physicalTime, dt;
};
}  // namespace

int fg_checkpoint_write(fg_solver *s, const char *path) {
    FG_ENTER(s);
    if (!path) return set_err(FG_ERR_ARG, "fg_checkpoint_write: null path");
    std::vector<double> U((size_t)s->nU * fg::NV);
    int rc = s->get_state(U.data(), 0, true);
    if (rc != FG_OK) return rc;
    CkHeader h{};
    std::memcpy(h.magic, kCkMagic, 8);
    h.nElem = s->nU;
    h.neq = fg::NV;
    h.iStep = s->iStep;
    h.precision = s->precision;
    rc = s->get_time(&h.dt, &h.physicalTime);
    if (rc != FG_OK) return rc;
    FILE *fp = fopen(path, "wb");
    if (!fp) return set_err(FG_ERR_IO, std::string("fg_checkpoint_write: cannot open ") + path);
    const bool ok = fwrite(&h, sizeof(h), 1, fp) == 1 && fwrite(U.data(), sizeof(double), U.size(), fp) == U.size();
    if (fclose(fp) != 0 || !ok) return set_err(FG_ERR_IO, std::string("fg_checkpoint_write: write failed: ") + path);
    return FG_OK;
}

int fg_checkpoint_read(fg_solver *s, const char *path) {
    FG_ENTER(s);
    if (!path) return set_err(FG_ERR_ARG, "fg_checkpoint_read: null path");
    FILE *fp = fopen(path, "rb");
    if (!fp) return set_err(FG_ERR_IO, std::string("fg_checkpoint_read: cannot open ") + path);
    CkHeader h{};
    std::vector<double> U((size_t)s->nU * fg::NV);
    bool ok = fread(&h, sizeof(h), 1, fp) == 1 && std::memcmp(h.magic, kCkMagic, 8) == 0;
    if (ok && (h.nElem != s->nU || h.neq != fg::NV)) {
        fclose(fp);
        return set_err(FG_ERR_ARG, "fg_checkpoint_read: checkpoint is for " + std::to_string(h.nElem) +
                                       " cells, the solver has " + std::to_string(s->nU));
    }
    ok = ok && fread(U.data(), sizeof(double), U.size(), fp) == U.size();
    fclose(fp);
    if (!ok) return set_err(FG_ERR_IO, std::string("fg_checkpoint_read: not a checkpoint or truncated: ") + path);
    int rc = s->set_state(U.data(), 0, true);
    if (rc == FG_OK) rc = s->set_dt(h.dt);
    if (rc == FG_OK) rc = s->set_time(h.physicalTime);
    if (rc != FG_OK) return rc;
    s->iStep = h.iStep;
    return FG_OK;
}

int fg_field_dump(fg_solver *s, const char *path) {
    FG_ENTER(s);
    if (!path) return set_err(FG_ERR_ARG, "fg_field_dump: null path");
    const double *cellCenter = s->cellCenter.data();
    std::vector<double> v((size_t)s->nU * 13);
    int rc = s->field_vars(v.data());
    if (rc != FG_OK) return rc;
    for (int i = 0; i < s->nU; i++)
        for (int d = 0; d < 3; d++) v[(size_t)i * 13 + d] = cellCenter[(size_t)i * 3 + d];
    double t = 0, dt = 0;
    rc = s->get_time(&dt, &t);
    if (rc != FG_OK) return rc;
    FILE *fp = fopen(path, "wb");
    if (!fp) return set_err(FG_ERR_IO, std::string("fg_field_dump: cannot open ") + path);
    const int32_t hdr[4] = {s->nU, 13, s->iStep, 0};
    const bool ok = fwrite(kFdMagic, 1, 8, fp) == 8 && fwrite(hdr, sizeof(hdr), 1, fp) == 1 &&
                    fwrite(&t, sizeof(double), 1, fp) == 1 && fwrite(v.data(), sizeof(double), v.size(), fp) == v.size();
    if (fclose(fp) != 0 || !ok) return set_err(FG_ERR_IO, std::string("fg_field_dump: write failed: ") + path);
    return FG_OK;
}

int fg_check_state(fg_solver *s, int32_t *badStep) {
    FG_ENTER(s);
    FG_CUDA_TRY(cudaDeviceSynchronize());
    if (badStep) *badStep = s->hBad[0] ? s->hBad[0] - 1 : -1;
    return (s->hBad[0] || s->hBad[1]) ? s->flag_error() : FG_OK;
}

int fg_step(fg_solver *s, void *stream) {
    FG_ENTER(s);
    if (s->hBad[0] || s->hBad[1]) return s->flag_error();
    cudaStream_t st = (cudaStream_t)stream;
    const fg_case &c = s->cs;
    int rc = s->advance_time(st);   // physicalTime += dt (previous dt, DP/explicitLoop.cu:29)
    if (rc) return rc;
    const int rk = c.rkSteps;
    for (int irk = 0; irk < rk; irk++) {
        const int writeU0 = (rk == 3 && irk == 0);
        if (c.adaptDt == 1 && irk == 0 && s->iStep % c.adaptDtItr == 0) {
            // residual with the signal speeds, new dt, then the stage update (DP/explicitLoop.cu:45-47)
            if ((rc = s->dt_stage(irk, writeU0, st))) return rc;
        } else {
            if ((rc = s->stage(irk, writeU0, st))) return rc;
        }
    }
    if (c.relaxFlag == 0)
        if ((rc = s->relax(nullptr, st))) return rc;
    if (c.consCalcFlag == 1 && s->iStep % c.adaptDtItr == 0)
        if ((rc = s->cons(c.consCalcIvar, nullptr, st))) return rc;
    s->iStep++;
    return FG_OK;
}

int fg_profile(fg_solver *s, int32_t enable) {
    FG_ENTER(s);
    if (cudaDeviceSynchronize() != cudaSuccess) return set_err(FG_ERR_CUDA, "fg_profile: device error");
    s->prof_reset(enable != 0);
    return FG_OK;
}
int fg_profile_read(fg_solver *s, fg_kernel_times *out) {
    FG_ENTER(s);
    if (!out) return set_err(FG_ERR_ARG, "null output");
    return s->prof_read(out);
}
int fg_launch_count(fg_solver *s, uint64_t *count) {
    FG_ENTER(s);
    if (!count) return set_err(FG_ERR_ARG, "null output");
    *count = s->launches;
    return FG_OK;
}

int fg_get_rhs(fg_solver *s, double *rhs) {
    FG_ENTER(s);
    if (!rhs) return set_err(FG_ERR_ARG, "null rhs");
    return s->get_rhs(rhs);
}
int fg_get_limited(fg_solver *s, double *grad, double *theta) {
    FG_ENTER(s);
    return s->get_limited(grad, theta);
}
int fg_get_signal(fg_solver *s, double *signal) {
    FG_ENTER(s);
    if (!signal) return set_err(FG_ERR_ARG, "null signal");
    return s->get_signal(signal);
}

}  // extern "C"
