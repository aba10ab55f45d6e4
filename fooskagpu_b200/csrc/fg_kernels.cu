// Kernels of the per-stage residual path (sm_100a).
//
// Dataflow per Runge-Kutta stage (no atomics, no face buffers):
//   k_grad : cell-centric.  Primitive states of the cell and its face neighbours (or boundary
//            ghosts) -> Green-Gauss gradient, neighbour min/max, limiter theta.
//            Replaces convert2PrimVec + greenGauss + computeLimiter
//            (DP/computePrimVec.cu:38, DP/computeGrad.cu:158, DP/computeFaceValues.cu:29).
//   k_flux : cell-centric.  For every face of the cell: MUSCL face states of both sides,
//            HLLC + non-conservative terms + pressure correction, WALE + viscous flux;
//            the cell's residual is summed in registers (deterministic owner-side gather),
//            then the FP64 Runge-Kutta combination and the new primitive record.
//            Replaces updateFaces + computeFlux + computeViscousStresses + rk3stage*/rungeKutta
//            (DP/computeFaceValues.cu:91, DP/computeRHS.cu:78, DP/computeViscousStresses.cu:66,
//            DP/update.cu:19-103).
// Both cells of an interior face evaluate its flux from identical inputs in the canonical
// (owner -> neighbour) orientation, so owner and neighbour contributions cancel exactly.
#include "fg_kernels.cuh"

#include <climits>

namespace fg {


template <typename T>
__device__ __forceinline__ void load_rec(const T *__restrict__ W, int c, T *w) {
    const T *p = W + (size_t)c * WREC;
#pragma unroll
    for (int v = 0; v < NP; v++) w[v] = __ldg(p + v);
}
template <>
__device__ __forceinline__ void load_rec<float>(const float *__restrict__ W, int c, float *w) {
    const float4 *p = reinterpret_cast<const float4 *>(W + (size_t)c * WREC);
    const float4 a = __ldg(p), b = __ldg(p + 1), d = __ldg(p + 2);
    w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
    w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
    w[8] = d.x;
}
template <typename T>
__device__ __forceinline__ void store_rec(T *W, int c, const T *w) {
    T *p = W + (size_t)c * WREC;
#pragma unroll
    for (int v = 0; v < NP; v++) p[v] = w[v];
#pragma unroll
    for (int v = NP; v < WREC; v++) p[v] = 0;
}
template <>
__device__ __forceinline__ void store_rec<float>(float *W, int c, const float *w) {
    float4 *p = reinterpret_cast<float4 *>(W + (size_t)c * WREC);
    p[0] = make_float4(w[0], w[1], w[2], w[3]);
    p[1] = make_float4(w[4], w[5], w[6], w[7]);
    p[2] = make_float4(w[8], 0.f, 0.f, 0.f);
}
template <typename T>
__device__ __forceinline__ void load_g(const T *__restrict__ G, int c, T *g) {
    const T *p = G + (size_t)c * GREC;
#pragma unroll
    for (int v = 0; v < GREC; v++) g[v] = __ldg(p + v);
}
template <>
__device__ __forceinline__ void load_g<float>(const float *__restrict__ G, int c, float *g) {
    const float4 *p = reinterpret_cast<const float4 *>(G + (size_t)c * GREC);
#pragma unroll
    for (int q = 0; q < GREC / 4; q++) {
        const float4 t = __ldg(p + q);
        g[4 * q + 0] = t.x; g[4 * q + 1] = t.y; g[4 * q + 2] = t.z; g[4 * q + 3] = t.w;
    }
}
template <typename T>
__device__ __forceinline__ void store_g(T *G, int c, const T *g) {
    T *p = G + (size_t)c * GREC;
#pragma unroll
    for (int v = 0; v < GREC; v++) p[v] = g[v];
}
template <>
__device__ __forceinline__ void store_g<float>(float *G, int c, const float *g) {
    float4 *p = reinterpret_cast<float4 *>(G + (size_t)c * GREC);
#pragma unroll
    for (int q = 0; q < GREC / 4; q++) p[q] = make_float4(g[4 * q], g[4 * q + 1], g[4 * q + 2], g[4 * q + 3]);
}

// ------------------------------------------------------------------ shared-memory staging
// A block handles `blockCells` consecutive (Morton-ordered, hence spatially compact) cells.  It
// first copies into shared memory
//   - the records of its own cells and of its halo (face neighbours outside the block),
//   - the per-slot face geometry of its own cells (contiguous in the cell-major layout),
// then each thread computes its cell's faces from shared memory only.  Strides are odd numbers
// of words so that threads of a warp reading the same field of consecutive cells hit distinct
// banks.  slotLocal holds the neighbour's staged-record index, or -bc on a boundary slot.
constexpr int kGeoComp = 10;   // nx ny nz A dcx dcy dcz dnx dny dnz

template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; };
template <> struct Vec16<double> { using type = double2; };

// record area rounded up to 16 bytes so the staged geometry arrays start aligned
template <typename T>
__host__ __device__ inline size_t rec_area(const DevMesh<T> &m, int stride) {
    return (((size_t)(m.blockCells + m.maxHalo) * stride * sizeof(T)) + 15) / 16 * 16;
}

template <typename T> struct Stage;
template <> struct Stage<float> {
    static constexpr int WS = 13;   // W(9) + volume + pad, odd
    static constexpr int RS = 47;   // W(9) theta(9) grad(27) volume + pad, odd
};
template <> struct Stage<double> {
    static constexpr int WS = 11;
    static constexpr int RS = 47;
};
// staged record layout (in T): [0..8] W, [9] volume, then (flux records) [10..18] theta,
// [19..45] grad
constexpr int kRecVol = 9;
constexpr int kRecTh = 10;
constexpr int kRecGrad = 19;
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
        case 0: return m->nx[g];
        case 1: return m->ny[g];
        case 2: return m->nz[g];
        case 3: return m->A[g];
        case 4: return m->dcx[g];
        case 5: return m->dcy[g];
        case 6: return m->dcz[g];
        case 7: return m->dnx[g];
        case 8: return m->dny[g];
        default: return m->dnz[g];
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
        const V x = __ldg(reinterpret_cast<const V *>(m.nx + cpt * cstride + g0) + j);
        reinterpret_cast<V *>(sg + (size_t)cpt * stride)[j] = x;
    }
    for (int i = threadIdx.x; i < nOwn * S; i += blockDim.x) sl[i] = m.slotLocal[g0 + i];
}

// ------------------------------------------------------------------ gradient + limiter
template <typename T>
__global__ void __launch_bounds__(StageCells<T>::value) k_grad(const DevMesh<T> m, const T *__restrict__ W,
                                                                T *__restrict__ G, const PhysT<T> P) {
    constexpr int WS = Stage<T>::WS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int b = blockIdx.x;
    const int B = m.blockCells;
    const int lo = b * B;
    const int nOwn = min(B, m.n - lo);
    const int nRec = B + (m.haloStart[b + 1] - m.haloStart[b]);
    const int SS = slot_stride(m.nSlots);
    T *rec = reinterpret_cast<T *>(smem_raw);                       // nRecMax * WS
    T *sg = reinterpret_cast<T *>(smem_raw + rec_area<T>(m, WS));   // kGeoComp * B * nSlots
    int *sl = reinterpret_cast<int *>(sg + (size_t)kGeoComp * B * m.nSlots);
    {
        // each lane copies one 16-byte vector of a W record (WREC / TPV vectors per record)
        using V = typename Vec16<T>::type;
        constexpr int TPV = 16 / sizeof(T);
        constexpr int WV = WREC / TPV;
        const V *Wv = reinterpret_cast<const V *>(W);
        for (int i = threadIdx.x; i < nRec * WV; i += blockDim.x) {
            const int r = i / WV, q = i - (i / WV) * WV;
            const int src = staged_source(m, b, r, lo, nOwn);
            if (src < 0) continue;
            const V x = __ldg(Wv + (size_t)src * WV + q);
            const T *xs = reinterpret_cast<const T *>(&x);
#pragma unroll
            for (int j = 0; j < TPV; j++)
                if (q * TPV + j < NP) rec[r * WS + q * TPV + j] = xs[j];
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
    for (int k = 0; k < nf; k++) {
        const int li = geo.local(k);
        const T nx = geo.get(0, k), ny = geo.get(1, k), nz = geo.get(2, k), A = geo.get(3, k);
        const T sgn = ((fl >> (3 + k)) & 1) ? (T)1 : (T)-1;   // outward orientation of this cell
        T ot[NP];
        if (li >= 0) {
#pragma unroll
            for (int v = 0; v < NP; v++) ot[v] = rec[li * WS + v];
        } else {
#pragma unroll
            for (int v = 0; v < NP; v++) ot[v] = w[v];
            ghost_state(P, -li, nx, ny, nz, ot);
        }
        const T ax = sgn * nx * A, ay = sgn * ny * A, az = sgn * nz * A;
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
    // limiter (DP/computeFaceValues.cu:66-81): theta = min over faces of clamp(phi, 0, 1)
    T th[NP];
#pragma unroll
    for (int v = 0; v < NP; v++) th[v] = (T)1e9;
    for (int k = 0; k < nf; k++) {
        const T dx = geo.get(4, k), dy = geo.get(5, k), dz = geo.get(6, k);
#pragma unroll
        for (int v = 0; v < NP; v++) {
            const T ext = dx * gs[3 * v] + dy * gs[3 * v + 1] + dz * gs[3 * v + 2];
            const T wun = w[v] + ext;
            const T diff = wun - w[v];
            T phi = 1;
            if (diff != 0) phi = ((wun > w[v]) ? (mx[v] - w[v]) : (mn[v] - w[v])) / (2 * diff);
            th[v] = fmin(th[v], fmax((T)0, fmin(phi, (T)1)));
        }
    }
    T out[GREC];
#pragma unroll
    for (int v = 0; v < NP; v++) out[v] = th[v];
#pragma unroll
    for (int q = 0; q < NP * 3; q++) out[NP + q] = gs[q];
    store_g(G, c, out);
}

// MUSCL face state of a cell: w + theta * ((x_f - x_c) . grad w)  (DP/computeFaceValues.cu:66-105);
// r points at a staged record
template <typename T>
__device__ __forceinline__ void face_state(const T *r, T dx, T dy, T dz, T *s) {
#pragma unroll
    for (int v = 0; v < NP; v++) {
        const T *g = r + kRecGrad + 3 * v;
        const T ext = fma(dx, g[0], fma(dy, g[1], dz * g[2]));
        s[v] = fma(r[kRecTh + v], ext, r[v]);
    }
}

// ------------------------------------------------------------------ flux + gather + RK
template <typename T>
__global__ void __launch_bounds__(StageCells<T>::value) k_flux(const DevMesh<T> m, Fields<T> f, const PhysT<T> P,
                                                                const PhysD D, int mode, int wantSignal, StageCoef sc) {
    constexpr int RS = Stage<T>::RS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int b = blockIdx.x;
    const int B = m.blockCells;
    const int lo = b * B;
    const int n = m.n;
    const int nOwn = min(B, n - lo);
    const int nRec = B + (m.haloStart[b + 1] - m.haloStart[b]);
    const int SS = slot_stride(m.nSlots);
    T *rec = reinterpret_cast<T *>(smem_raw);
    T *sg = reinterpret_cast<T *>(smem_raw + rec_area<T>(m, RS));
    int *sl = reinterpret_cast<int *>(sg + (size_t)kGeoComp * B * m.nSlots);
    // records: W(9) | volume | theta(9) grad(27): 16-byte vectors of the W and G records, the
    // volume taken by the lane that copies the W vector holding W[8]
    {
        using V = typename Vec16<T>::type;
        constexpr int TPV = 16 / sizeof(T);
        constexpr int WV = WREC / TPV, GV = GREC / TPV, NVR = WV + GV;
        const V *Wv = reinterpret_cast<const V *>(f.Win);
        const V *Gv = reinterpret_cast<const V *>(f.G);
        for (int i = threadIdx.x; i < nRec * NVR; i += blockDim.x) {
            const int r = i / NVR, q = i - (i / NVR) * NVR;
            const int src = staged_source(m, b, r, lo, nOwn);
            if (src < 0) continue;
            T *dst = rec + r * RS;
            if (q < WV) {
                const V x = __ldg(Wv + (size_t)src * WV + q);
                const T *xs = reinterpret_cast<const T *>(&x);
#pragma unroll
                for (int j = 0; j < TPV; j++)
                    if (q * TPV + j < NP) dst[q * TPV + j] = xs[j];
                if (q * TPV <= NP - 1 && NP - 1 < (q + 1) * TPV) dst[kRecVol] = (T)m.vol[src];
            } else {
                const V x = __ldg(Gv + (size_t)src * GV + (q - WV));
                const T *xs = reinterpret_cast<const T *>(&x);
#pragma unroll
                for (int j = 0; j < TPV; j++) dst[kRecTh + (q - WV) * TPV + j] = xs[j];
            }
        }
    }
    stage_geometry(m, lo, nOwn, sg, sl);
    __syncthreads();
    const int t = threadIdx.x;
    const int c = lo + t;
    const bool cell = t < nOwn;
    const SlotGeo<T> geo{sg, sl, B * m.nSlots, t * m.nSlots, &m, (size_t)c * m.nSlots};
    double cfl = 1e12;   // per-cell CFL bound for the block minimum
    if (cell) {
        const T *me = rec + t * RS;
        T w[NP];
#pragma unroll
        for (int v = 0; v < NP; v++) w[v] = me[v];
        const T pc = w[0] * w[6] + (1 - w[0]) * w[7];
        double acc[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) acc[v] = 0.0;
        T sig = (T)-1e9;
        const int fl = m.flags[c];
        const int nf = fl & 7;
        const double vc = m.vol[c];
        for (int k = 0; k < nf; k++) {
            const int li = geo.local(k);
            const bool own = (fl >> (3 + k)) & 1;
            const T nx = geo.get(0, k), ny = geo.get(1, k), nz = geo.get(2, k), A = geo.get(3, k);
            T sc_[NP], so[NP];   // own and other reconstructed face states
            face_state(me, geo.get(4, k), geo.get(5, k), geo.get(6, k), sc_);
            const T *gme = me + kRecGrad + 9;    // own velocity gradient
            const T *gO, *gN;                    // velocity gradients of owner / neighbour (viscous)
            T p1[NP];                            // slot-1 state as the viscous kernel reads it
            T vAvg;
            if (li >= 0) {
                const T *ot = rec + li * RS;
                face_state(ot, geo.get(7, k), geo.get(8, k), geo.get(9, k), so);
                const T *gnb = ot + kRecGrad + 9;
                gO = own ? gme : gnb;
                gN = own ? gnb : gme;
                const T vn = ot[kRecVol], vm = me[kRecVol];
                vAvg = (own ? (vm + vn) : (vn + vm)) * (T)0.5;
            } else {
                // ghost of the reconstructed state for the flux (DP/computeRHS.cu:113)
#pragma unroll
                for (int v = 0; v < NP; v++) so[v] = sc_[v];
                ghost_state(P, -li, nx, ny, nz, so);
                // the viscous flux reads the ghost of the cell-centre state (DP/computePrimVec.cu:61-76)
#pragma unroll
                for (int v = 0; v < NP; v++) p1[v] = w[v];
                ghost_state(P, -li, nx, ny, nz, p1);
                gO = gN = gme;
                vAvg = me[kRecVol];
            }
            const T *L = own ? sc_ : so;
            const T *R = own ? so : sc_;
            if (li >= 0) {
#pragma unroll
                for (int v = 0; v < NP; v++) p1[v] = R[v];
            }
            T F[NV], unc, pF;
            hllc_flux(P, L, R, nx, ny, nz, F, unc, pF);
            // side terms with this cell's centre state (DP/flux.h:1-30, DP/computeRHS.cu:38-75)
            const T sgn = own ? (T)-1 : (T)1;
            const T dp = pF - pc;
            T cb[NV];
            cb[0] = sgn * (F[0] - w[0] * unc) * A;
            cb[1] = sgn * F[1] * A;
            cb[2] = sgn * F[2] * A;
            cb[3] = sgn * (F[3] + dp * nx) * A;
            cb[4] = sgn * (F[4] + dp * ny) * A;
            cb[5] = sgn * (F[5] + dp * nz) * A;
            cb[6] = sgn * (F[6] + w[0] * w[6] * unc) * A;
            cb[7] = sgn * (F[7] + (1 - w[0]) * w[7] * unc) * A;
            cb[8] = sgn * F[8] * A;
            cb[9] = sgn * F[9] * A;
            if (P.visc) {
                // DP/computeViscousStresses.cu:87-170 with slot 0 = owner face state (L)
                T gv[9];
#pragma unroll
                for (int q = 0; q < 9; q++) gv[q] = (gO[q] + gN[q]) * (T)0.5;
                const T nut = P.turb ? wale_nu(gv, vAvg) : (T)0;
                const T dv = (gv[0] + gv[4] + gv[8]) * ((T)2 / 3);
                const T t00 = 2 * gv[0] - dv, t11 = 2 * gv[4] - dv, t22 = 2 * gv[8] - dv;
                const T t01 = gv[1] + gv[3], t02 = gv[2] + gv[6], t12 = gv[5] + gv[7];
                const T a1 = L[0], r1 = L[0] * L[1] + (1 - L[0]) * L[2];
                const T a2 = p1[0], r2 = p1[0] * p1[1] + (1 - p1[0]) * p1[2];
                const T mu = (a1 + a2) * (T)0.5 * P.mu[0] + (1 - (a1 + a2) * (T)0.5) * P.mu[1] + (r1 + r2) * (T)0.5 * nut;
                const T fmx = mu * (t00 * nx + t01 * ny + t02 * nz);
                const T fmy = mu * (t01 * nx + t11 * ny + t12 * nz);
                const T fmz = mu * (t02 * nx + t12 * ny + t22 * nz);
                const T vx = (L[3] + p1[3]) * (T)0.5, vy = (L[4] + p1[4]) * (T)0.5, vz = (L[5] + p1[5]) * (T)0.5;
                const T fe = mu * ((t00 * vx + t01 * vy + t02 * vz) * nx + (t01 * vx + t11 * vy + t12 * vz) * ny +
                                   (t02 * vx + t12 * vy + t22 * vz) * nz);
                const T vs = own ? A : -A;
                cb[3] += fmx * vs;
                cb[4] += fmy * vs;
                cb[5] += fmz * vs;
                cb[8] += fe * vs;
            }
#pragma unroll
            for (int v = 0; v < NV; v++) acc[v] += (double)cb[v];
            if (wantSignal) {
                T s = face_signal(P, sc_, nx, ny, nz);
                if (li >= 0) s = fmax(s, face_signal(P, so, nx, ny, nz));
                sig = fmax(sig, s);
            }
        }
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
            T wo[NP];
            cons2prim_d(D, u, wo);
            store_rec(f.Wout, c, wo);
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

// RK stage from the RHS buffer (DP/update.cu:19-103)
template <typename T>
__global__ void k_update(const DevMesh<T> m, Fields<T> f, const PhysD D, StageCoef sc) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = m.n;
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
    T wo[NP];
    cons2prim_d(D, u, wo);
    store_rec(f.Wout, c, wo);
}

template <typename T>
__global__ void k_prim(int n, const double *__restrict__ U, T *W, const PhysD D) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double u[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) u[v] = U[(size_t)v * n + c];
    T w[NP];
    cons2prim_d(D, u, w);
    store_rec(W, c, w);
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

// ------------------------------------------------------------------ state layout conversion
__global__ void k_scatter_state(int n, const double *__restrict__ Ua, const int32_t *__restrict__ new2old, double *U) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
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

// ------------------------------------------------------------------ launchers
int flux_blocks(int n, int blockCells) { return (n + blockCells - 1) / blockCells; }
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
template <typename T>
static size_t flux_smem(const DevMesh<T> &m) {
    return rec_area<T>(m, Stage<T>::RS) + geo_smem(m);
}
template <typename T>
int stage_kernels_setup(const DevMesh<T> &m) {
    if (cudaFuncSetAttribute(k_grad<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_smem(m)) != cudaSuccess)
        return 1;
    if (cudaFuncSetAttribute(k_flux<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)flux_smem(m)) != cudaSuccess)
        return 1;
    return 0;
}
template <typename T>
void launch_grad(const DevMesh<T> &m, const Fields<T> &f, const PhysT<T> &P, cudaStream_t s) {
    const int nb = (m.n + m.blockCells - 1) / m.blockCells;
    k_grad<T><<<nb, m.blockCells, grad_smem(m), s>>>(m, f.Win, f.G, P);
}
template <typename T>
void launch_flux(const DevMesh<T> &m, const Fields<T> &f, const PhysT<T> &P, const PhysD &D, int mode,
                 int wantSignal, StageCoef sc, cudaStream_t s) {
    const int nb = (m.n + m.blockCells - 1) / m.blockCells;
    k_flux<T><<<nb, m.blockCells, flux_smem(m), s>>>(m, f, P, D, mode, wantSignal, sc);
}
template int stage_kernels_setup<float>(const DevMesh<float> &);
template int stage_kernels_setup<double>(const DevMesh<double> &);
template <typename T>
void launch_update(const DevMesh<T> &m, const Fields<T> &f, const PhysD &D, StageCoef sc, cudaStream_t s) {
    k_update<T><<<(m.n + 255) / 256, 256, 0, s>>>(m, f, D, sc);
}
template <typename T>
void launch_prim(int n, const double *U, T *W, const PhysD &D, cudaStream_t s) {
    k_prim<T><<<(n + 255) / 256, 256, 0, s>>>(n, U, W, D);
}
void launch_dt_finalize(const double *blockMin, int nBlocks, double cfl, double maxDt, double *dt, cudaStream_t s) {
    k_dt_finalize<<<1, 1024, 0, s>>>(blockMin, nBlocks, cfl, maxDt, dt);
}
void launch_cons(int n, int ivar, const double *U, const double *vol, double *blockSum, double *out, cudaStream_t s) {
    const int nb = cons_blocks(n);
    k_cons_blocks<<<nb, kConsThreads, 0, s>>>(n, ivar, U, vol, blockSum);
    k_cons_final<<<1, 1024, 0, s>>>(blockSum, nb, out);
}
void launch_scatter_state(int n, const double *Ua, const int32_t *new2old, double *U, cudaStream_t s) {
    k_scatter_state<<<(n + 255) / 256, 256, 0, s>>>(n, Ua, new2old, U);
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
template void launch_flux<float>(const DevMesh<float> &, const Fields<float> &, const PhysT<float> &, const PhysD &, int, int, StageCoef, cudaStream_t);
template void launch_flux<double>(const DevMesh<double> &, const Fields<double> &, const PhysT<double> &, const PhysD &, int, int, StageCoef, cudaStream_t);
template void launch_update<float>(const DevMesh<float> &, const Fields<float> &, const PhysD &, StageCoef, cudaStream_t);
template void launch_update<double>(const DevMesh<double> &, const Fields<double> &, const PhysD &, StageCoef, cudaStream_t);
template void launch_prim<float>(int, const double *, float *, const PhysD &, cudaStream_t);
template void launch_prim<double>(int, const double *, double *, const PhysD &, cudaStream_t);

}  // namespace fg
