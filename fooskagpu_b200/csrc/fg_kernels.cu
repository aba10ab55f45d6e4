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

constexpr int kGradThreads = 128;
constexpr int kFluxThreads = 128;

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

// ------------------------------------------------------------------ lane groups
// A cell is handled by a group of G lanes (G = 4 for tetrahedra, 8 when a cell can have 5 or 6
// faces); lane k of the group works on the face in slot k.  Partial results are combined with
// a butterfly of warp shuffles inside the group, whose order is fixed — so results are
// deterministic — and every lane ends with the cell total.
template <int G, typename X>
__device__ __forceinline__ X group_sum(X v) {
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off, G);
    return v;
}
template <int G, typename X>
__device__ __forceinline__ X group_min(X v) {
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, off, G));
    return v;
}
template <int G, typename X>
__device__ __forceinline__ X group_max(X v) {
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off, G));
    return v;
}

// ------------------------------------------------------------------ gradient + limiter
template <typename T, int G>
__global__ void __launch_bounds__(kGradThreads) k_grad(const DevMesh<T> m, const T *__restrict__ W,
                                                       T *__restrict__ G_, const PhysT<T> P) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = gid / G;
    const int k = gid % G;
    const bool cell = c < m.n;     // uniform across the group
    const int cc = cell ? c : m.n - 1;
    T w[NP];
    load_rec(W, cc, w);
    const int fl = m.flags[cc];
    const int nf = fl & 7;
    const bool act = cell && k < nf;
    const size_t o = (size_t)cc * m.nSlots + (act ? k : 0);
    T gs[NP * 3], mn[NP], mx[NP];
#pragma unroll
    for (int v = 0; v < NP; v++) {
        gs[3 * v] = gs[3 * v + 1] = gs[3 * v + 2] = 0;
        mn[v] = (T)1e12;
        mx[v] = (T)-1e12;
    }
    if (act) {
        const int nb = m.nbr[o];
        const T nx = m.nx[o], ny = m.ny[o], nz = m.nz[o], A = m.A[o];
        const T sg = ((fl >> (3 + k)) & 1) ? (T)1 : (T)-1;   // outward orientation of this cell
        T ot[NP];
        if (nb >= 0) {
            load_rec(W, nb, ot);
        } else {
#pragma unroll
            for (int v = 0; v < NP; v++) ot[v] = w[v];
            ghost_state(P, -nb, nx, ny, nz, ot);
        }
        const T ax = sg * nx * A, ay = sg * ny * A, az = sg * nz * A;
#pragma unroll
        for (int v = 0; v < NP; v++) {
            mx[v] = ot[v];
            mn[v] = ot[v];
            const T h = (w[v] + ot[v]) * (T)0.5;
            gs[3 * v + 0] = h * ax;
            gs[3 * v + 1] = h * ay;
            gs[3 * v + 2] = h * az;
        }
    }
    const T iv = (T)(1.0 / m.vol[cc]);
#pragma unroll
    for (int q = 0; q < NP * 3; q++) gs[q] = group_sum<G>(gs[q]) * iv;
#pragma unroll
    for (int v = 0; v < NP; v++) {
        mn[v] = group_min<G>(mn[v]);
        mx[v] = group_max<G>(mx[v]);
    }
    // limiter (DP/computeFaceValues.cu:66-81): theta = min over faces of clamp(phi, 0, 1)
    T th[NP];
#pragma unroll
    for (int v = 0; v < NP; v++) th[v] = (T)1e9;
    if (act) {
        const T dx = m.dcx[o], dy = m.dcy[o], dz = m.dcz[o];
#pragma unroll
        for (int v = 0; v < NP; v++) {
            const T ext = dx * gs[3 * v] + dy * gs[3 * v + 1] + dz * gs[3 * v + 2];
            const T wun = w[v] + ext;
            const T diff = wun - w[v];
            T phi = 1;
            if (diff != 0) phi = ((wun > w[v]) ? (mx[v] - w[v]) : (mn[v] - w[v])) / (2 * diff);
            th[v] = fmax((T)0, fmin(phi, (T)1));
        }
    }
#pragma unroll
    for (int v = 0; v < NP; v++) th[v] = group_min<G>(th[v]);
    if (cell) {
        // the record [theta(9), grad(27)] is written by the lanes of the group in 4-word pieces
        T rec[GREC];
#pragma unroll
        for (int v = 0; v < NP; v++) rec[v] = th[v];
#pragma unroll
        for (int q = 0; q < NP * 3; q++) rec[NP + q] = gs[q];
        T *dst = G_ + (size_t)c * GREC;
#pragma unroll
        for (int piece = 0; piece < GREC / 4; piece++)
            if (piece % G == k) {
#pragma unroll
                for (int j = 0; j < 4; j++) dst[4 * piece + j] = rec[4 * piece + j];
            }
    }
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

// ------------------------------------------------------------------ flux + gather + RK
template <typename T, int G>
__global__ void __launch_bounds__(kFluxThreads) k_flux(const DevMesh<T> m, Fields<T> f, const PhysT<T> P,
                                                       const PhysD D, int mode, int wantSignal, StageCoef sc) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = gid / G;
    const int k = gid % G;
    const int n = m.n;
    const bool cell = c < n;
    const int cc = cell ? c : n - 1;
    const int fl = m.flags[cc];
    const int nf = fl & 7;
    const bool act = cell && k < nf;
    T w[NP];
    load_rec(f.Win, cc, w);
    T cb[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) cb[v] = 0;
    T sig = (T)-1e9;
    const double vc = m.vol[cc];
    if (act) {
        const size_t o = (size_t)cc * m.nSlots + k;
        const int nb = m.nbr[o];
        const bool own = (fl >> (3 + k)) & 1;
        const T nx = m.nx[o], ny = m.ny[o], nz = m.nz[o], A = m.A[o];
        T sc_[NP], so[NP];   // own and other reconstructed face states
        T gO[9], gN[9];      // velocity gradients of owner / neighbour (viscous)
        T p1[NP];            // slot-1 state as the viscous kernel reads it
        T vAvg;
        {
            T g[GREC];
            load_g(f.G, cc, g);
            face_state(w, g, m.dcx[o], m.dcy[o], m.dcz[o], sc_);
#pragma unroll
            for (int q = 0; q < 9; q++) gO[q] = g[NP + 9 + q];
        }
        if (nb >= 0) {
            T wn[NP], gn[GREC];
            load_rec(f.Win, nb, wn);
            load_g(f.G, nb, gn);
            face_state(wn, gn, m.dnx[o], m.dny[o], m.dnz[o], so);
#pragma unroll
            for (int q = 0; q < 9; q++) {
                const T gc = gO[q];
                gO[q] = own ? gc : gn[NP + 9 + q];
                gN[q] = own ? gn[NP + 9 + q] : gc;
            }
            const double vn = m.vol[nb];
            vAvg = (T)((own ? (vc + vn) : (vn + vc)) * 0.5);
        } else {
            // ghost of the reconstructed state for the flux (DP/computeRHS.cu:113)
#pragma unroll
            for (int v = 0; v < NP; v++) so[v] = sc_[v];
            ghost_state(P, -nb, nx, ny, nz, so);
            // the viscous flux reads the ghost of the cell-centre state (DP/computePrimVec.cu:61-76)
#pragma unroll
            for (int v = 0; v < NP; v++) p1[v] = w[v];
            ghost_state(P, -nb, nx, ny, nz, p1);
#pragma unroll
            for (int q = 0; q < 9; q++) gN[q] = gO[q];
            vAvg = (T)vc;
        }
        const T *L = own ? sc_ : so;
        const T *R = own ? so : sc_;
        if (nb >= 0) {
#pragma unroll
            for (int v = 0; v < NP; v++) p1[v] = R[v];
        }
        T F[NV], unc, pF;
        hllc_flux(P, L, R, nx, ny, nz, F, unc, pF);
        // side terms with this cell's centre state (DP/flux.h:1-30, DP/computeRHS.cu:38-75)
        const T pc = w[0] * w[6] + (1 - w[0]) * w[7];
        const T sgn = own ? (T)-1 : (T)1;
        const T dp = pF - pc;
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
        if (wantSignal) {
            sig = face_signal(P, sc_, nx, ny, nz);
            if (nb >= 0) sig = fmax(sig, face_signal(P, so, nx, ny, nz));
        }
    }
    // cell residual: FP64 butterfly over the group's faces
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) acc[v] = group_sum<G>((double)cb[v]);
    double cfl = 1e12;   // per-cell CFL bound for the block minimum
    if (wantSignal) {
        sig = group_max<G>(sig);
        if (cell) {
            if (k == 0) f.signal[c] = (double)sig;
            cfl = m.volP[c] / (double)sig;
        }
    }
    if (mode == FLUX_RHS) {
        // lane j stores variables j, j + G, ...
        if (cell) {
#pragma unroll
            for (int v = 0; v < NV; v++)
                if (v % G == k) f.RHS[(size_t)v * n + c] = acc[v];
        }
    } else {
        // FP64 Runge-Kutta combination (DP/update.cu:19-103): lane j updates variables j, j + G,
        // ...; the new state is then shuffled to every lane and lane 0 writes the primitive record
        double rl[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) rl[v] = 0.0;
        if (cell) {
            const double dt = *f.dt;
            const double dtv = dt * (1.0 / vc);
#pragma unroll
            for (int v = 0; v < NV; v++) {
                if (v % G != k) continue;
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
                f.U[q] = r;
                rl[v] = r;
            }
        }
        double un[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) un[v] = __shfl_sync(0xffffffffu, rl[v], v % G, G);
        if (cell && k == 0) {
            T wo[NP];
            cons2prim_d(D, un, wo);
            store_rec(f.Wout, c, wo);
        }
    }
    if (wantSignal) {
        // deterministic block minimum of the CFL bound
        __shared__ double red[kFluxThreads / 32];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) cfl = fmin(cfl, __shfl_down_sync(0xffffffffu, cfl, off));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cfl;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = red[0];
            for (int i = 1; i < kFluxThreads / 32; i++) b = fmin(b, red[i]);
            f.blockMin[blockIdx.x] = b;
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
int lane_group(int nSlots) { return nSlots <= 4 ? 4 : 8; }
int flux_blocks(int n, int nSlots) {
    return (int)(((size_t)n * lane_group(nSlots) + kFluxThreads - 1) / kFluxThreads);
}
int cons_blocks(int n) { return (n + kConsThreads - 1) / kConsThreads; }

template <typename T>
void launch_grad(const DevMesh<T> &m, const Fields<T> &f, const PhysT<T> &P, cudaStream_t s) {
    const int nb = (int)(((size_t)m.n * lane_group(m.nSlots) + kGradThreads - 1) / kGradThreads);
    if (lane_group(m.nSlots) == 4) k_grad<T, 4><<<nb, kGradThreads, 0, s>>>(m, f.Win, f.G, P);
    else k_grad<T, 8><<<nb, kGradThreads, 0, s>>>(m, f.Win, f.G, P);
}
template <typename T>
void launch_flux(const DevMesh<T> &m, const Fields<T> &f, const PhysT<T> &P, const PhysD &D, int mode,
                 int wantSignal, StageCoef sc, cudaStream_t s) {
    const int nb = flux_blocks(m.n, m.nSlots);
    if (lane_group(m.nSlots) == 4) k_flux<T, 4><<<nb, kFluxThreads, 0, s>>>(m, f, P, D, mode, wantSignal, sc);
    else k_flux<T, 8><<<nb, kFluxThreads, 0, s>>>(m, f, P, D, mode, wantSignal, sc);
}
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
