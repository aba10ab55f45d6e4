// Kernels of the per-stage residual path (sm_100a).
//
// Dataflow per Runge-Kutta stage (no atomics):
//   k_grad   : cell-centric.  Primitive states of the cell and its face neighbours (or boundary
//              ghosts) -> Green-Gauss gradient, neighbour min/max, limiter theta.
//              Replaces convert2PrimVec + greenGauss + computeLimiter
//              (DP/computePrimVec.cu:38, DP/computeGrad.cu:158, DP/computeFaceValues.cu:29).
//   k_face   : one thread per face.  MUSCL face states of both sides, HLLC flux with the
//              non-conservative and pressure terms, WALE + viscous flux, written once as a
//              12-word face record.  Replaces updateFaces + computeFlux + computeViscousStresses
//              (DP/computeFaceValues.cu:91, DP/computeRHS.cu:78, DP/computeViscousStresses.cu:66).
//   k_gather : one thread per cell.  Sums the records of the cell's faces with its orientation
//              sign in FP64 in slot order (deterministic owner-side gather), adds the cell-centre
//              terms, then the FP64 Runge-Kutta combination and the new primitive record
//              (DP/update.cu:19-103), or stores the residual.
#include "fg_kernels.cuh"

#include <climits>

namespace fg {


template <typename T>
__device__ __forceinline__ void store_frec(T *FB, int f, const T *r) {
    T *p = FB + (size_t)f * FREC;
#pragma unroll
    for (int v = 0; v < FREC; v++) p[v] = r[v];
}
template <>
__device__ __forceinline__ void store_frec<float>(float *FB, int f, const float *r) {
    float4 *p = reinterpret_cast<float4 *>(FB + (size_t)f * FREC);
    p[0] = make_float4(r[0], r[1], r[2], r[3]);
    p[1] = make_float4(r[4], r[5], r[6], r[7]);
    p[2] = make_float4(r[8], r[9], r[10], r[11]);
}
template <typename T>
__device__ __forceinline__ void load_frec(const T *__restrict__ FB, int f, T *r) {
    const T *p = FB + (size_t)f * FREC;
#pragma unroll
    for (int v = 0; v < FREC; v++) r[v] = __ldg(p + v);
}
template <>
__device__ __forceinline__ void load_frec<float>(const float *__restrict__ FB, int f, float *r) {
    const float4 *p = reinterpret_cast<const float4 *>(FB + (size_t)f * FREC);
    const float4 a = __ldg(p), b = __ldg(p + 1), d = __ldg(p + 2);
    r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w;
    r[4] = b.x; r[5] = b.y; r[6] = b.z; r[7] = b.w;
    r[8] = d.x; r[9] = d.y; r[10] = d.z; r[11] = d.w;
}

// ------------------------------------------------------------------ shared-memory staging
// A block handles `blockCells` consecutive (Morton-ordered, hence spatially compact) cells.  It
// first copies into shared memory
//   - the records of its own cells and of its halo (face neighbours outside the block),
//   - the per-slot face geometry of its own cells (contiguous in the cell-major layout),
// then each thread computes its cell's faces from shared memory only.  Strides are odd numbers
// of words so that threads of a warp reading the same field of consecutive cells hit distinct
// banks.  slotLocal holds the neighbour's staged-record index, or -bc on a boundary slot.
constexpr int kGeoComp = 6;    // aox aoy aoz dcx dcy dcz

// record area rounded up to 16 bytes so the staged geometry arrays start aligned
template <typename T>
__host__ __device__ inline size_t rec_area(const DevMesh<T> &m, int stride) {
    return (((size_t)(m.blockCells + m.maxHalo) * stride * sizeof(T)) + 15) / 16 * 16;
}

template <typename T> struct Stage;
template <> struct Stage<float> {
    static constexpr int WS = 13;   // W(9) + volume + pad, odd
};
template <> struct Stage<double> {
    static constexpr int WS = 11;
};
__host__ __device__ constexpr int slot_stride(int nSlots) { return nSlots | 1; }

// per-slot geometry of a cell: staged in shared memory, or read from global memory
template <typename T>
struct SlotGeo {
    const T *sg;
    const int *sl;
    int GS;         // component stride of the staged arrays
    int d0;         // t * slot stride
    const DevMesh<T> *m;
    size_t g0;      // c * nSlots
    __device__ __forceinline__ T get(int comp, int k) const {
#if FG_STAGE_GEOMETRY
        return sg[comp * GS + d0 + k];   // d0 = t * nSlots
#else
        const size_t g = g0 + k;
        switch (comp) {
        case 0: return m->aox[g];
        case 1: return m->aoy[g];
        case 2: return m->aoz[g];
        case 3: return m->dcx[g];
        case 4: return m->dcy[g];
        default: return m->dcz[g];
        }
#endif
    }
    __device__ __forceinline__ int local(int k) const {
#if FG_STAGE_GEOMETRY
        return sl[d0 + k];
#else
        return m->slotLocal[g0 + k];
#endif
    }
};

template <typename T>
__device__ __forceinline__ int staged_source(const DevMesh<T> &m, int b, int r, int lo, int nOwn) {
    return (r < m.blockCells) ? ((r < nOwn) ? lo + r : -1) : m.haloIds[m.haloStart[b] + (r - m.blockCells)];
}

// copy the per-slot geometry and local indices of the block's own cells: the block's slots are a
// contiguous range of each cell-major array, copied with 16-byte loads in the global layout
template <typename T>
__device__ __forceinline__ void stage_geometry(const DevMesh<T> &m, int lo, int nOwn, T *sg, int *sl) {
#if !FG_STAGE_GEOMETRY
    return;
#endif
    using V = typename Vec16<T>::type;
    constexpr int TPV = 16 / sizeof(T);
    const int S = m.nSlots;
    const int B = m.blockCells;
    const int nV = (nOwn * S + TPV - 1) / TPV;          // vectors per component actually used
    const int stride = B * S;                            // component stride in shared memory
    const size_t cstride = m.geoStride;
    const size_t g0 = (size_t)lo * S;                    // 16-byte aligned: B * S * sizeof(T) % 16 == 0
    for (int i = threadIdx.x; i < kGeoComp * nV; i += blockDim.x) {
        const int cpt = i / nV, j = i % nV;
        const V x = __ldg(reinterpret_cast<const V *>(m.aox + cpt * cstride + g0) + j);
        reinterpret_cast<V *>(sg + (size_t)cpt * stride)[j] = x;
    }
    for (int i = threadIdx.x; i < nOwn * S; i += blockDim.x) sl[i] = m.slotLocal[g0 + i];
}

// ------------------------------------------------------------------ gradient + limiter
// limiter function of a face increment diff with num = w_max - w or w_min - w: the reference's
// phi = num / (2 diff), or the van Albada-type extension phi(r) = (r^2 + r) / (r^2 + 1), r = num / diff
template <typename T, int kLim>
__device__ __forceinline__ T limiter_phi(T num, T diff) {
    if (kLim == 1) {
        const T r = num / diff;
        return (r * r + r) / (r * r + 1);
    }
    return num / (2 * diff);
}

// slot loops of the gradient kernel: unrolled to the largest face count (the loads of every slot
// can then be issued early), or a plain loop to the cell's face count
#ifndef FG_GRAD_UNROLL
#define FG_GRAD_UNROLL 1
#endif
#if FG_GRAD_UNROLL
#define FG_GRAD_SLOT_LOOP(k, nf) _Pragma("unroll") for (int k = 0; k < MAXSLOT; k++) if (k < (nf))
#else
#define FG_GRAD_SLOT_LOOP(k, nf) for (int k = 0; k < (nf); k++)
#endif

// kLim: 0 the reference's limiter function, 1 the van Albada-type extension (fg_case.limiter)
template <typename T, int kLim>
__global__ void __launch_bounds__(StageCells<T>::value, MinBlocks<T>::grad) k_grad(const DevMesh<T> m, const T *__restrict__ W,
                                                                T *__restrict__ G, const PhysT<T> P) {
    constexpr int WS = Stage<T>::WS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int b = blockIdx.x;
    const int B = m.blockCells;
    const int lo = b * B;
    const int nOwn = min(B, m.nG - lo);      // cells whose gradients this block computes
    const int nBlockRecs = min(B, m.n - lo);  // cells of the block range with records (ghosts of a part too)
    const int nRec = B + (m.haloStart[b + 1] - m.haloStart[b]);
    const int SS = slot_stride(m.nSlots);
    T *rec = reinterpret_cast<T *>(smem_raw);                       // nRecMax * WS
    T *sg = reinterpret_cast<T *>(smem_raw + rec_area<T>(m, WS));   // kGeoComp * B * nSlots
    int *sl = reinterpret_cast<int *>(sg + (size_t)kGeoComp * B * m.nSlots);
    {
        // each lane copies one 16-byte vector of a W record; consecutive lanes take the same
        // vector of consecutive staged cells (contiguous for the block's own cells)
        using V = typename Vec16<T>::type;
        constexpr int TPV = vpv<T>();
        constexpr int WV = (NP + TPV - 1) / TPV;   // vectors holding the NP used values
        const V *Wv = reinterpret_cast<const V *>(W);
        for (int r = threadIdx.x; r < nRec; r += blockDim.x) {
            const int src = staged_source(m, b, r, lo, nBlockRecs);
            if (src < 0) continue;
#pragma unroll
            for (int q = 0; q < WV; q++) {
                const V x = __ldg(Wv + (size_t)q * m.n + src);
#pragma unroll
                for (int j = 0; j < TPV; j++)
                    if (q * TPV + j < NP) rec[r * WS + q * TPV + j] = vlane(x, j);
            }
        }
    }
    stage_geometry(m, lo, nOwn, sg, sl);
    __syncthreads();
    const int t = threadIdx.x;
    const int c = lo + t;
    if (t >= nOwn) return;
    const SlotGeo<T> geo{sg, sl, B * m.nSlots, t * m.nSlots, &m, (size_t)c * m.nSlots};
    T w[NP], gs[NP * 3], mn[NP], mx[NP];
#pragma unroll
    for (int v = 0; v < NP; v++) {
        w[v] = rec[t * WS + v];
        gs[3 * v] = gs[3 * v + 1] = gs[3 * v + 2] = 0;
        mn[v] = (T)1e12;
        mx[v] = (T)-1e12;
    }
    const int fl = m.flags[c];
    const int nf = fl & 7;
    FG_GRAD_SLOT_LOOP(k, nf) {
        const int li = geo.local(k);
        // outward n A of the face (the host computed (+-1) n A in T arithmetic, as the reference's
        // sign times normal times area)
        const T ax = geo.get(0, k), ay = geo.get(1, k), az = geo.get(2, k);
        T ot[NP];
        if (li >= 0) {
#pragma unroll
            for (int v = 0; v < NP; v++) ot[v] = rec[li * WS + v];
        } else {
            // boundary slot: the cell owns the face, so its canonical normal points outward
            const int fi = m.slotFace[(size_t)c * m.nSlots + k];
#pragma unroll
            for (int v = 0; v < NP; v++) ot[v] = w[v];
            ghost_state(P, -li, m.fnx[fi], m.fny[fi], m.fnz[fi], ot);
        }
#pragma unroll
        for (int v = 0; v < NP; v++) {
            mx[v] = fmax(mx[v], ot[v]);
            mn[v] = fmin(mn[v], ot[v]);
            const T h = (w[v] + ot[v]) * (T)0.5;
            gs[3 * v + 0] += h * ax;
            gs[3 * v + 1] += h * ay;
            gs[3 * v + 2] += h * az;
        }
    }
    const T iv = (T)(1.0 / m.vol[c]);
#pragma unroll
    for (int q = 0; q < NP * 3; q++) gs[q] *= iv;
    // limiter (DP/computeFaceValues.cu:66-81): theta = min over the faces of clamp(phi, 0, 1), phi
    // of the face's increment diff = (w + (x_f - x_c) . grad w) - w and of num = w_max - w (diff
    // > 0) or w_min - w (diff < 0).  clamp(phi) does not increase with |diff| on either side
    // (for both limiter functions and either sign of num), so the minimum over the faces is that
    // of the largest positive and of the most negative increment: two divisions per variable
    // instead of one per face, the same result.
    T dpos[NP], dneg[NP];
#pragma unroll
    for (int v = 0; v < NP; v++) dpos[v] = dneg[v] = 0;
    FG_GRAD_SLOT_LOOP(k, nf) {
        const T dx = geo.get(3, k), dy = geo.get(4, k), dz = geo.get(5, k);
#pragma unroll
        for (int v = 0; v < NP; v++) {
            const T ext = dx * gs[3 * v] + dy * gs[3 * v + 1] + dz * gs[3 * v + 2];
            const T diff = (w[v] + ext) - w[v];
            dpos[v] = fmax(dpos[v], diff);
            dneg[v] = fmin(dneg[v], diff);
        }
    }
    T th[NP];
#pragma unroll
    for (int v = 0; v < NP; v++) {
        T t = 1;
        if (dpos[v] > 0) t = fmin(t, limiter_phi<T, kLim>(mx[v] - w[v], dpos[v]));
        if (dneg[v] < 0) t = fmin(t, limiter_phi<T, kLim>(mn[v] - w[v], dneg[v]));
        th[v] = fmax((T)0, t);
    }
    T out[GREC];
#pragma unroll
    for (int v = 0; v < NP; v++) out[v] = th[v];
#pragma unroll
    for (int q = 0; q < NP * 3; q++) out[NP + q] = gs[q];
    grec_store<T, GREC>(G, m.n, c, out);
}

// MUSCL face state of a cell: w + theta * ((x_f - x_c) . grad w)  (DP/computeFaceValues.cu:66-105)
template <typename T>
__device__ __forceinline__ void face_state(const T *w, const T *g, T dx, T dy, T dz, T *s) {
#pragma unroll
    for (int v = 0; v < NP; v++) {
        const T ext = fma(dx, g[NP + 3 * v], fma(dy, g[NP + 3 * v + 1], dz * g[NP + 3 * v + 2]));
        s[v] = fma(g[v], ext, w[v]);
    }
}

// gradient of the liquid-phase temperature T = (p_L + pInf) / (cv (gamma - 1) rho_L) of a cell from
// its record and gradients (chain rule), added to acc
template <typename T>
__device__ __forceinline__ void cell_grad_t(const PhysT<T> &P, const T *w, const T *g, T *acc) {
    const T rl = w[1], pl = w[6];
    const T c = (pl + P.pinf[0]) / rl;
    const T inv = (T)1 / (P.cvgm1[0] * rl);
#pragma unroll
    for (int d = 0; d < 3; d++) acc[d] += (g[NP + 3 * 6 + d] - c * g[NP + 3 * 1 + d]) * inv;
}

// Flux part of a face, shared by the face kernels: HLLC + pressure + viscous (+ heat) flux of the
// reconstructed states sL (owner) and sR (neighbour or ghost), written as the face record of fi.
// p1: neighbour state for the viscous flux (the cell-centre ghost on a boundary face);
// gO / gN: the two cells' velocity gradients; gT: sum of their temperature gradients.
template <typename T>
__device__ __forceinline__ T face_tail(const PhysT<T> &P, const T *sL, const T *sR, const T *p1, const T *gO,
                                          const T *gN, const T *gT, int nb, T nx, T ny, T nz, T A, T lsSq,
                                          int wantSignal, T *__restrict__ FB, int fi) {
    T F[NV], unc, pF;
    hllc_flux(P, sL, sR, nx, ny, nz, F, unc, pF);
    T H[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) H[v] = A * F[v];
    // the face pressure relative to the datum P0; the gather adds (p_C - P0) times the cell's
    // sum of outward n A, so the residual is the same for every P0 in exact arithmetic
    const T pd = pF - P.pDatum;
    H[3] += A * pd * nx;
    H[4] += A * pd * ny;
    H[5] += A * pd * nz;
    if (P.visc) {
        T gv[9];
#pragma unroll
        for (int q = 0; q < 9; q++) gv[q] = (gO[q] + gN[q]) * (T)0.5;
        const T nut = P.turb ? wale_nu(gv, lsSq) : (T)0;
        const T dv = (gv[0] + gv[4] + gv[8]) * ((T)2 / 3);
        const T t00 = 2 * gv[0] - dv, t11 = 2 * gv[4] - dv, t22 = 2 * gv[8] - dv;
        const T t01 = gv[1] + gv[3], t02 = gv[2] + gv[6], t12 = gv[5] + gv[7];
        const T a1 = sL[0], r1 = sL[0] * sL[1] + (1 - sL[0]) * sL[2];
        const T a2 = p1[0], r2 = p1[0] * p1[1] + (1 - p1[0]) * p1[2];
        const T mu = (a1 + a2) * (T)0.5 * P.mu[0] + (1 - (a1 + a2) * (T)0.5) * P.mu[1] + (r1 + r2) * (T)0.5 * nut;
        const T vx = (sL[3] + p1[3]) * (T)0.5, vy = (sL[4] + p1[4]) * (T)0.5, vz = (sL[5] + p1[5]) * (T)0.5;
        const T muA = mu * A;
        H[3] -= muA * (t00 * nx + t01 * ny + t02 * nz);
        H[4] -= muA * (t01 * nx + t11 * ny + t12 * nz);
        H[5] -= muA * (t02 * nx + t12 * ny + t22 * nz);
        H[8] -= muA * ((t00 * vx + t01 * vy + t02 * vz) * nx + (t01 * vx + t11 * vy + t12 * vz) * ny +
                       (t02 * vx + t12 * vy + t22 * vz) * nz);
        if (P.heat && nb >= 0) {
            // Fourier conduction k grad T . n (extension); adiabatic boundary faces
            const T aF = (a1 + a2) * (T)0.5;
            const T kF = mu * (aF * P.cp[0] + (1 - aF) * P.cp[1]) / (aF * P.prn[0] + (1 - aF) * P.prn[1]);
            H[8] -= A * kF * (T)0.5 * (gT[0] * nx + gT[1] * ny + gT[2] * nz);
        }
    }
    T sig = 0;
    if (wantSignal) {
        // DP/computeTimeStep.cu:97-129: both reconstructed sides of an interior face, the owner
        // side only on a boundary
        sig = face_signal(P, sL, nx, ny, nz);
        if (nb >= 0) sig = fmax(sig, face_signal(P, sR, nx, ny, nz));
    }
    T rec[FREC];
#pragma unroll
    for (int v = 0; v < NV; v++) rec[v] = H[v];
    rec[NV] = A * unc;
    rec[NV + 1] = sig;
    store_frec(FB, fi, rec);
    return sig;
}

// running maximum of a cell's face signal speeds: signal speeds are non-negative, and the integer
// order of non-negative IEEE values is their numeric order, so the maximum is exact and independent
// of the order of the updates.  A NaN signal is skipped, as fmax skips it.
__device__ __forceinline__ void signal_max(float *a, float v) {
    if (v >= 0.0f) atomicMax(reinterpret_cast<int *>(a), __float_as_int(v));
}
__device__ __forceinline__ void signal_max(double *a, double v) {
    if (v >= 0.0) atomicMax(reinterpret_cast<long long *>(a), __double_as_longlong(v));
}

// ------------------------------------------------------------------ face flux (once per face)
// Record of face f with canonical normal n (owner -> neighbour), area A:
//   H[v] = A (F[v] - Visc[v]) + A pF n (momentum),  u = A (u* . n),  signal
// where F is the HLLC + advective flux (DP/computeRHS.cu:117-131), Visc the WALE viscous flux
// (DP/computeViscousStresses.cu:87-170) and pF the upwind mixture pressure.  A cell with
// orientation s (-1 owner, +1 neighbour, the reference's sign) receives s * H[v] plus its
// cell-centre terms, which k_gather adds from sums over its faces:
//   var 0: -alpha_c s u,  vars 6/7: +alpha_c pL_c s u, +(1-alpha_c) pG_c s u,
//   momentum: -pC_c s A n summed = pC_c * (sum of outward n A)  (DP/flux.h:1-30, DP/computeRHS.cu:38-75)
template <typename T>
__global__ void __launch_bounds__(FG_FACE_THREADS, MinBlocks<T>::face) k_face(const DevMesh<T> m, const T *__restrict__ W, const T *__restrict__ G,
                                              T *__restrict__ FB, T *cellSig, const PhysT<T> P, int wantSignal) {
    const int fi = blockIdx.x * blockDim.x + threadIdx.x;
    if (fi >= m.nFEval) return;
    const int o = m.fOwn[fi];
    const int nb = m.fNb[fi];
    const T nx = m.fnx[fi], ny = m.fny[fi], nz = m.fnz[fi], A = m.fA[fi];
    T wo[NP], sL[NP], sR[NP], p1[NP], gO[9], gN[9];
    T gT[3] = {0, 0, 0};   // sum of the two cells' temperature gradients (heat conduction)
    {
        T g[GREC];
        rec_load<T, NP>(W, m.n, o, wo);
        grec_load<T, GREC>(G, m.n, o, g);
        face_state(wo, g, m.fdo[0][fi], m.fdo[1][fi], m.fdo[2][fi], sL);
#pragma unroll
        for (int q = 0; q < 9; q++) gO[q] = g[NP + 9 + q];
        if (P.heat && nb >= 0) cell_grad_t(P, wo, g, gT);
    }
    if (nb >= 0) {
        T wn[NP], g[GREC];
        rec_load<T, NP>(W, m.n, nb, wn);
        grec_load<T, GREC>(G, m.n, nb, g);
        face_state(wn, g, m.fdn[0][fi], m.fdn[1][fi], m.fdn[2][fi], sR);
#pragma unroll
        for (int q = 0; q < 9; q++) gN[q] = g[NP + 9 + q];
        if (P.heat) cell_grad_t(P, wn, g, gT);
#pragma unroll
        for (int v = 0; v < NP; v++) p1[v] = sR[v];
    } else {
        // ghost of the reconstructed state for the flux (DP/computeRHS.cu:113); the viscous flux
        // reads the ghost of the cell-centre state (DP/computePrimVec.cu:61-76) and the owner's
        // gradient twice
#pragma unroll
        for (int v = 0; v < NP; v++) {
            sR[v] = sL[v];
            p1[v] = wo[v];
        }
        ghost_state(P, -nb, nx, ny, nz, sR);
        ghost_state(P, -nb, nx, ny, nz, p1);
#pragma unroll
        for (int q = 0; q < 9; q++) gN[q] = gO[q];
    }
    const T sig = face_tail(P, sL, sR, p1, gO, gN, gT, nb, nx, ny, nz, A, m.fLsSq[fi], wantSignal, FB, fi);
    if (wantSignal == 2) {
        // own cells only: a ghost's dt bound belongs to its own part
        if (o < m.nU) signal_max(cellSig + o, sig);
        if (nb >= 0 && nb < m.nU) signal_max(cellSig + nb, sig);
    }
}

// ------------------------------------------------------------------ owner-side gather + RK
template <typename T>
__global__ void __launch_bounds__(FG_GATHER_THREADS, MinBlocks<T>::gather) k_gather(const DevMesh<T> m, Fields<T> f, const PhysD D, int mode,
                                                int wantSignal, StageCoef sc) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = m.nU;   // state rows (U, U0, RHS stride)
    double cfl = 1e12;
    if (c < n) {
        const int fl = m.flags[c];
        const int nf = fl & 7;
        double acc[NV], su = 0.0;
#pragma unroll
        for (int v = 0; v < NV; v++) acc[v] = 0.0;
        T sig = (T)-1e9;
        const size_t base = (size_t)c * m.nSlots;
        for (int k = 0; k < nf; k++) {
            const int fi = m.slotFace[base + k];
            const double s = ((fl >> (3 + k)) & 1) ? -1.0 : 1.0;
            T rec[FREC];
            load_frec(f.FB, fi, rec);
#pragma unroll
            for (int v = 0; v < NV; v++) acc[v] += s * (double)rec[v];
            su += s * (double)rec[NV];
            sig = fmax(sig, rec[NV + 1]);
        }
        T w[NP];
        rec_load<T, NP>(f.Win, m.n, c, w);
        const double a = w[0], pl = w[6], pg = w[7];
        const double pc = (double)(w[0] * w[6] + (1 - w[0]) * w[7]) - D.pDatum;
        acc[0] -= a * su;
        acc[6] += a * pl * su;
        acc[7] += (1.0 - a) * pg * su;
        acc[3] += pc * (double)m.closure[c];
        acc[4] += pc * (double)m.closure[(size_t)m.n + c];
        acc[5] += pc * (double)m.closure[2 * (size_t)m.n + c];
        const double vc = m.vol[c];
        if (wantSignal) {
            f.signal[c] = (double)sig;
            cfl = m.volP[c] / (double)sig;
        }
        if (mode == FLUX_RHS) {
#pragma unroll
            for (int v = 0; v < NV; v++) f.RHS[(size_t)v * n + c] = acc[v];
        } else {
            // FP64 Runge-Kutta combination (DP/update.cu:19-103)
            const double dt = *f.dt;
            const double dtv = dt * (1.0 / vc);
            double u[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const size_t q = (size_t)v * n + c;
                const double uc = f.U[q];
                double r;
                if (sc.rk == 1) {
                    r = uc + dtv * acc[v];
                } else if (sc.irk == 0) {
                    if (sc.writeU0) f.U0[q] = uc;
                    const double u0 = sc.writeU0 ? uc : f.U0[q];
                    r = u0 + dtv * acc[v];
                } else if (sc.irk == 1) {
                    r = 0.75 * f.U0[q] + 0.25 * uc + (0.25 * dt) * (1.0 / vc) * acc[v];
                } else {
                    r = (1.0 / 3.0) * f.U0[q] + (2.0 / 3.0) * uc + ((2.0 / 3.0) * dt) * (1.0 / vc) * acc[v];
                }
                if (v == 5 && sc.neglectZ) r = 0.0;
                u[v] = r;
                f.U[q] = r;
            }
            if (!state_ok(u)) *f.bad = f.step + 1;
            T wo[NP];
            cons2prim_d(D, u, wo);
            rec_store<T, NP>(f.Wout, m.n, c, wo);
        }
    }
    if (wantSignal) {
        // deterministic block minimum of the CFL bound
        __shared__ double red[32];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) cfl = fmin(cfl, __shfl_down_sync(0xffffffffu, cfl, off));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cfl;
        __syncthreads();
        if (threadIdx.x == 0) {
            double bm = red[0];
            for (int i = 1; i < (int)(blockDim.x >> 5); i++) bm = fmin(bm, red[i]);
            f.blockMin[blockIdx.x] = bm;
        }
    }
}

// CFL bound of the own cells from their maximum face signal speed (k_face with wantSignal 2), as
// the gather kernel computes it on the residual path: signal[c], then the deterministic block
// minimum of volP / signal over blocks of the gather kernel's size
template <typename T>
__global__ void k_cell_cfl(const DevMesh<T> m, const T *__restrict__ cellSig, double *signal, double *blockMin) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double cfl = 1e12;
    if (c < m.nU) {
        const T sig = cellSig[c];
        signal[c] = (double)sig;
        cfl = m.volP[c] / (double)sig;
    }
    __shared__ double red[32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) cfl = fmin(cfl, __shfl_down_sync(0xffffffffu, cfl, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cfl;
    __syncthreads();
    if (threadIdx.x == 0) {
        double bm = red[0];
        for (int i = 1; i < (int)(blockDim.x >> 5); i++) bm = fmin(bm, red[i]);
        blockMin[blockIdx.x] = bm;
    }
}

// RK stage from the RHS buffer (DP/update.cu:19-103)
template <typename T>
__global__ void k_update(const DevMesh<T> m, Fields<T> f, const PhysD D, StageCoef sc) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = m.nU;
    if (c >= n) return;
    const double dt = *f.dt;
    const double vc = m.vol[c];
    double u[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) {
        const size_t q = (size_t)v * n + c;
        const double uc = f.U[q], R = f.RHS[q];
        double r;
        if (sc.rk == 1) r = uc + dt * (1.0 / vc) * R;
        else if (sc.irk == 0) {
            if (sc.writeU0) f.U0[q] = uc;
            r = (sc.writeU0 ? uc : f.U0[q]) + dt * (1.0 / vc) * R;
        } else if (sc.irk == 1) r = 0.75 * f.U0[q] + 0.25 * uc + (0.25 * dt) * (1.0 / vc) * R;
        else r = (1.0 / 3.0) * f.U0[q] + (2.0 / 3.0) * uc + ((2.0 / 3.0) * dt) * (1.0 / vc) * R;
        if (v == 5 && sc.neglectZ) r = 0.0;
        u[v] = r;
        f.U[q] = r;
    }
    if (!state_ok(u)) *f.bad = f.step + 1;
    T wo[NP];
    cons2prim_d(D, u, wo);
    rec_store<T, NP>(f.Wout, m.n, c, wo);
}

template <typename T>
__global__ void k_prim(int n, const double *__restrict__ U, T *W, size_t wStride, const PhysD D) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double u[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) u[v] = U[(size_t)v * n + c];
    T w[NP];
    cons2prim_d(D, u, w);
    rec_store<T, NP>(W, wStride, c, w);
}

__global__ void k_dt_finalize(const double *blockMin, int nb, double cfl, double maxDt, double *dt) {
    __shared__ double red[32];
    double v = 1e12;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) v = fmin(v, blockMin[i]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = red[0];
        for (int i = 1; i < (int)(blockDim.x >> 5); i++) b = fmin(b, red[i]);
        *dt = fmin(cfl * b, maxDt);
    }
}

// ------------------------------------------------------------------ conservation (DP/consCalc.cu:3-34)
constexpr int kConsThreads = 256;
__global__ void k_cons_blocks(int n, int ivar, const double *__restrict__ U, const double *__restrict__ vol,
                              double *blockSum) {
    __shared__ double sh[kConsThreads];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (c < n) {
        const double x = U[(size_t)ivar * n + c];
        v = ((ivar == 0) ? 1.0 - x : x) * vol[c];
    }
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = kConsThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) blockSum[blockIdx.x] = sh[0];
}
__global__ void k_cons_final(const double *blockSum, int nb, double *out) {
    // fixed-shape tree over per-thread strided partial sums: deterministic for a given nb
    __shared__ double sh[1024];
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) v += blockSum[i];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// ------------------------------------------------------------------ state probe
// Per block of kConsThreads cells: [0] sum of (1 - alpha) V (the vapour volume, the reference's
// consCalc of variable 0), [1] max and [2] min of the mixture pressure alpha p_L + (1 - alpha) p_G,
// [3] max speed |u|; then one block combines the block results in block order.  Deterministic.
__global__ void k_probe_blocks(int n, const double *__restrict__ U, const double *__restrict__ vol, const PhysD D,
                               double *blockOut) {
    __shared__ double sh[4][kConsThreads];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double vv = 0.0, pmax = -1e300, pmin = 1e300, umax = 0.0;
    if (c < n) {
        double u[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) u[v] = U[(size_t)v * n + c];
        double w[NP];
        cons2prim_d(D, u, w);
        const double p = w[0] * w[6] + (1 - w[0]) * w[7];
        vv = (1.0 - u[0]) * vol[c];
        pmax = pmin = p;
        umax = sqrt(w[3] * w[3] + w[4] * w[4] + w[5] * w[5]);
    }
    sh[0][threadIdx.x] = vv;
    sh[1][threadIdx.x] = pmax;
    sh[2][threadIdx.x] = pmin;
    sh[3][threadIdx.x] = umax;
    __syncthreads();
    for (int st = kConsThreads / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) {
            const int o = threadIdx.x + st;
            sh[0][threadIdx.x] += sh[0][o];
            sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][o]);
            sh[2][threadIdx.x] = fmin(sh[2][threadIdx.x], sh[2][o]);
            sh[3][threadIdx.x] = fmax(sh[3][threadIdx.x], sh[3][o]);
        }
        __syncthreads();
    }
    if (threadIdx.x < 4) blockOut[(size_t)blockIdx.x * 4 + threadIdx.x] = sh[threadIdx.x][0];
}
__global__ void k_probe_final(const double *blockOut, int nb, double *out) {
    __shared__ double sh[4][1024];
    double vv = 0.0, pmax = -1e300, pmin = 1e300, umax = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        vv += blockOut[(size_t)i * 4 + 0];
        pmax = fmax(pmax, blockOut[(size_t)i * 4 + 1]);
        pmin = fmin(pmin, blockOut[(size_t)i * 4 + 2]);
        umax = fmax(umax, blockOut[(size_t)i * 4 + 3]);
    }
    sh[0][threadIdx.x] = vv;
    sh[1][threadIdx.x] = pmax;
    sh[2][threadIdx.x] = pmin;
    sh[3][threadIdx.x] = umax;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) {
            const int o = threadIdx.x + st;
            sh[0][threadIdx.x] += sh[0][o];
            sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][o]);
            sh[2][threadIdx.x] = fmin(sh[2][threadIdx.x], sh[2][o]);
            sh[3][threadIdx.x] = fmax(sh[3][threadIdx.x], sh[3][o]);
        }
        __syncthreads();
    }
    if (threadIdx.x < 4) out[threadIdx.x] = sh[threadIdx.x][0];
}

// ------------------------------------------------------------------ uploaded state check
// firstBad = min over cells c of an AoS state Ua[c * 10 + v] that is not usable: a non-finite
// sum, alpha outside [0, 1] (beyond 1e-9) or a negative partial density (the order-independent
// minimum reports the first such cell in the caller's order)
__global__ void k_check_state(int n, const double *__restrict__ Ua, int32_t *firstBad) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double *u = Ua + (size_t)c * NV;
    double sum = 0;
#pragma unroll
    for (int v = 0; v < NV; v++) sum += u[v];
    const bool ok = isfinite(sum) && u[0] >= -1e-9 && u[0] <= 1.0 + 1e-9 && u[1] >= 0.0 && u[2] >= 0.0 &&
                    u[1] + u[2] > 0.0;
    if (!ok) atomicMin(firstBad, c);
}

// ------------------------------------------------------------------ state layout conversion
// U (renumbered SoA) = the uploaded AoS state, unless the check found an unusable cell: then U is
// left as it was and flags[1] = that cell + 1.  A state that replaces U clears both flags (the
// RK kernels' flags[0] and a previous rejection).
__global__ void k_scatter_state(int n, const double *__restrict__ Ua, const int32_t *__restrict__ new2old, double *U,
                                const int32_t *firstBad, int32_t *flags) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int fb = *firstBad;
    if (fb < n) {
        if (c == 0) flags[1] = fb + 1;
        return;
    }
    if (c == 0) {
        flags[0] = 0;
        flags[1] = 0;
    }
    if (c >= n) return;
    const size_t o = (size_t)new2old[c] * NV;
#pragma unroll
    for (int v = 0; v < NV; v++) U[(size_t)v * n + c] = Ua[o + v];
}
__global__ void k_gather_state(int n, const double *__restrict__ U, const int32_t *__restrict__ new2old, double *Ua) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const size_t o = (size_t)new2old[c] * NV;
#pragma unroll
    for (int v = 0; v < NV; v++) Ua[o + v] = U[(size_t)v * n + c];
}
__global__ void k_copy(size_t cnt, const double *__restrict__ a, double *b) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t st = (size_t)gridDim.x * blockDim.x;
    for (; i < cnt; i += st) b[i] = a[i];
}

// ------------------------------------------------------------------ halo records (partitioned runs)
// out[k * nval + v] = value v of the record of cells[k] (records of nRec cells, nval values each):
// the records of the cells another part needs, packed whole
template <typename T>
__global__ void k_halo_pack(const T *__restrict__ rec, size_t nRec, int nval, int vpv, const int32_t *__restrict__ cells,
                            int cnt, T *__restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)cnt * nval) return;
    const size_t k = i / nval;
    const int v = (int)(i - k * nval);
    out[i] = rec[((size_t)(v / vpv) * nRec + (size_t)cells[k]) * vpv + (size_t)(v % vpv)];
}
// value v of the record of cells[k] = in[k * nval + v]: the ghosts' records received from their parts
template <typename T>
__global__ void k_halo_unpack(T *__restrict__ rec, size_t nRec, int nval, int vpv, const int32_t *__restrict__ cells,
                              int cnt, const T *__restrict__ in) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)cnt * nval) return;
    const size_t k = i / nval;
    const int v = (int)(i - k * nval);
    rec[((size_t)(v / vpv) * nRec + (size_t)cells[k]) * vpv + (size_t)(v % vpv)] = in[i];
}

// ------------------------------------------------------------------ launchers
constexpr int kGatherThreads = FG_GATHER_THREADS;
int flux_blocks(int n) { return (n + kGatherThreads - 1) / kGatherThreads; }
int cons_blocks(int n) { return (n + kConsThreads - 1) / kConsThreads; }

template <typename T>
static size_t geo_smem(const DevMesh<T> &m) {
    if (!FG_STAGE_GEOMETRY) return 0;
    const size_t slots = (size_t)m.blockCells * m.nSlots;
    return slots * kGeoComp * sizeof(T) + slots * sizeof(int);
}
template <typename T>
static size_t grad_smem(const DevMesh<T> &m) {
    return rec_area<T>(m, Stage<T>::WS) + geo_smem(m);
}
// raise (never lower) a kernel's dynamic shared-memory limit on the current device: solvers of
// different meshes launch the same kernels with different amounts
static int raise_smem(const void *fn, size_t bytes) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, fn) != cudaSuccess) return 1;
    if ((size_t)a.maxDynamicSharedSizeBytes >= bytes) return 0;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess;
}
template <typename T>
int stage_kernels_setup(const DevMesh<T> &m) {
    return raise_smem((const void *)k_grad<T, 0>, grad_smem(m)) | raise_smem((const void *)k_grad<T, 1>, grad_smem(m));
}
template <typename T>
void launch_grad(const DevMesh<T> &m, const Fields<T> &f, const PhysT<T> &P, cudaStream_t s) {
    const int nb = (m.nG + m.blockCells - 1) / m.blockCells;
    if (P.limiter == 1)
        k_grad<T, 1><<<nb, m.blockCells, grad_smem(m), s>>>(m, f.Win, f.G, P);
    else
        k_grad<T, 0><<<nb, m.blockCells, grad_smem(m), s>>>(m, f.Win, f.G, P);
}
template <typename T>
void launch_face(const DevMesh<T> &m, const Fields<T> &f, const PhysT<T> &P, int wantSignal, cudaStream_t s) {
    if (m.nFEval == 0) return;
    k_face<T><<<(m.nFEval + FG_FACE_THREADS - 1) / FG_FACE_THREADS, FG_FACE_THREADS, 0, s>>>(m, f.Win, f.G, f.FB, f.cellSig, P,
                                                                                      wantSignal);
}
template <typename T>
void launch_cell_cfl(const DevMesh<T> &m, const Fields<T> &f, cudaStream_t s) {
    k_cell_cfl<T><<<flux_blocks(m.nU), kGatherThreads, 0, s>>>(m, f.cellSig, f.signal, f.blockMin);
}
template <typename T>
void launch_gather(const DevMesh<T> &m, const Fields<T> &f, const PhysD &D, int mode, int wantSignal,
                   StageCoef sc, cudaStream_t s) {
    k_gather<T><<<flux_blocks(m.nU), kGatherThreads, 0, s>>>(m, f, D, mode, wantSignal, sc);
}
template int stage_kernels_setup<float>(const DevMesh<float> &);
template int stage_kernels_setup<double>(const DevMesh<double> &);
template <typename T>
void launch_update(const DevMesh<T> &m, const Fields<T> &f, const PhysD &D, StageCoef sc, cudaStream_t s) {
    k_update<T><<<(m.nU + 255) / 256, 256, 0, s>>>(m, f, D, sc);
}
template <typename T>
void launch_halo_pack(const T *rec, size_t nRec, int nval, int vpv, const int32_t *cells, int cnt, T *out,
                      cudaStream_t s) {
    const size_t tot = (size_t)cnt * nval;
    if (tot) k_halo_pack<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(rec, nRec, nval, vpv, cells, cnt, out);
}
template <typename T>
void launch_halo_unpack(T *rec, size_t nRec, int nval, int vpv, const int32_t *cells, int cnt, const T *in,
                        cudaStream_t s) {
    const size_t tot = (size_t)cnt * nval;
    if (tot) k_halo_unpack<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(rec, nRec, nval, vpv, cells, cnt, in);
}
template void launch_halo_pack<float>(const float *, size_t, int, int, const int32_t *, int, float *, cudaStream_t);
template void launch_halo_pack<double>(const double *, size_t, int, int, const int32_t *, int, double *, cudaStream_t);
template void launch_halo_unpack<float>(float *, size_t, int, int, const int32_t *, int, const float *, cudaStream_t);
template void launch_halo_unpack<double>(double *, size_t, int, int, const int32_t *, int, const double *, cudaStream_t);
template <typename T>
void launch_prim(int n, const double *U, T *W, size_t wStride, const PhysD &D, cudaStream_t s) {
    k_prim<T><<<(n + 255) / 256, 256, 0, s>>>(n, U, W, wStride, D);
}
void launch_dt_finalize(const double *blockMin, int nBlocks, double cfl, double maxDt, double *dt, cudaStream_t s) {
    k_dt_finalize<<<1, 1024, 0, s>>>(blockMin, nBlocks, cfl, maxDt, dt);
}
void launch_cons(int n, int ivar, const double *U, const double *vol, double *blockSum, double *out, cudaStream_t s) {
    const int nb = cons_blocks(n);
    k_cons_blocks<<<nb, kConsThreads, 0, s>>>(n, ivar, U, vol, blockSum);
    k_cons_final<<<1, 1024, 0, s>>>(blockSum, nb, out);
}
void launch_probe(int n, const double *U, const double *vol, const PhysD &D, double *blockOut, double *out,
                  cudaStream_t s) {
    const int nb = cons_blocks(n);
    k_probe_blocks<<<nb, kConsThreads, 0, s>>>(n, U, vol, D, blockOut);
    k_probe_final<<<1, 1024, 0, s>>>(blockOut, nb, out);
}
void launch_check_state(int n, const double *Ua, int32_t *firstBad, cudaStream_t s) {
    // "none" = 0x7f7f7f7f, above any cell count
    cudaMemsetAsync(firstBad, 0x7f, sizeof(int32_t), s);
    if (n > 0) k_check_state<<<(n + 255) / 256, 256, 0, s>>>(n, Ua, firstBad);
}
void launch_scatter_state(int n, const double *Ua, const int32_t *new2old, double *U, const int32_t *firstBad,
                          int32_t *flags, cudaStream_t s) {
    k_scatter_state<<<(n + 255) / 256, 256, 0, s>>>(n, Ua, new2old, U, firstBad, flags);
}
void launch_gather_state(int n, const double *U, const int32_t *new2old, double *Ua, cudaStream_t s) {
    k_gather_state<<<(n + 255) / 256, 256, 0, s>>>(n, U, new2old, Ua);
}
void launch_copy_u0(int n, const double *U, double *U0, cudaStream_t s) {
    const size_t cnt = (size_t)n * NV;
    k_copy<<<(int)std::min<size_t>((cnt + 255) / 256, 148 * 16), 256, 0, s>>>(cnt, U, U0);
}

template void launch_grad<float>(const DevMesh<float> &, const Fields<float> &, const PhysT<float> &, cudaStream_t);
template void launch_grad<double>(const DevMesh<double> &, const Fields<double> &, const PhysT<double> &, cudaStream_t);
template void launch_face<float>(const DevMesh<float> &, const Fields<float> &, const PhysT<float> &, int, cudaStream_t);
template void launch_face<double>(const DevMesh<double> &, const Fields<double> &, const PhysT<double> &, int, cudaStream_t);
template void launch_cell_cfl<float>(const DevMesh<float> &, const Fields<float> &, cudaStream_t);
template void launch_cell_cfl<double>(const DevMesh<double> &, const Fields<double> &, cudaStream_t);
template void launch_gather<float>(const DevMesh<float> &, const Fields<float> &, const PhysD &, int, int, StageCoef, cudaStream_t);
template void launch_gather<double>(const DevMesh<double> &, const Fields<double> &, const PhysD &, int, int, StageCoef, cudaStream_t);
template void launch_update<float>(const DevMesh<float> &, const Fields<float> &, const PhysD &, StageCoef, cudaStream_t);
template void launch_update<double>(const DevMesh<double> &, const Fields<double> &, const PhysD &, StageCoef, cudaStream_t);
template void launch_prim<float>(int, const double *, float *, size_t, const PhysD &, cudaStream_t);
template void launch_prim<double>(int, const double *, double *, size_t, const PhysD &, cudaStream_t);

}  // namespace fg
