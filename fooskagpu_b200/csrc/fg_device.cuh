// Device-side physics of the residual path, templated on the face-math type T
// (float for the mixed path, double for the FP64 path).  Cell-centre conversions,
// the Runge-Kutta combination and the Newton solves are always FP64.
//
// The formulas are those of the reference (DP/eqos.h, DP/cons2prim.h, DP/prim2cons.h,
// DP/waveSpeeds.h, DP/starRegion.h, DP/flux.h, DP/bc.h, DP/computeRHS.cu,
// DP/computeViscousStresses.cu, DP/computeTimeStep.cu).  Two algebraic identities replace
// the reference's explicit tangent frame (n, t1, t2 orthonormal):
//   lcl2glb([S*, u.t1, u.t2]) = u + (S* - u.n) n       (star velocity, DP/starRegion.h:7-8)
//   lcl2glb([-u.n, u.t1, u.t2]) = u - 2 (u.n) n         (slip / symmetry ghost, DP/bc.h:47-84)
// so the device needs only the unit normal per face.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fg {

// Primitive record: [alpha, rhoL, rhoG, u, v, w, pL, pG, m_v]; stored padded to WREC.
constexpr int NP = 9;
constexpr int WREC = 12;
// Per-cell limited-gradient record: theta[9] then grad[9][3].
constexpr int GREC = 36;
constexpr int NV = 10;
constexpr int MAXSLOT = 6;

// ---------------------------------------------------------------- record layout
// The per-cell records (W: WREC values, G: GREC values) are stored component-major in 16-byte
// vectors: vector q of cell c (values q * VPV .. q * VPV + VPV - 1, VPV = 16 / sizeof(T)) sits at
// base + (q * stride + c) * VPV, stride = the number of cells with records.  A warp that reads
// one vector of consecutive or nearby cells (the owners of consecutive faces, the Morton-ordered
// neighbours) touches a few cache lines instead of one line per lane as with whole records.
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; };
template <> struct Vec16<double> { using type = double2; };
template <typename T>
__host__ __device__ constexpr int vpv() { return 16 / (int)sizeof(T); }
// index of value v of cell c
template <typename T>
__host__ __device__ inline size_t rec_index(size_t stride, size_t c, int v) {
    return ((size_t)(v / vpv<T>()) * stride + c) * vpv<T>() + (size_t)(v % vpv<T>());
}
// lane j of a 16-byte vector (no address of a vector is taken, so the vectors stay in registers)
__device__ __forceinline__ float vlane(const float4 &x, int j) { return j == 0 ? x.x : j == 1 ? x.y : j == 2 ? x.z : x.w; }
__device__ __forceinline__ double vlane(const double2 &x, int j) { return j == 0 ? x.x : x.y; }
// the first NVAL values of the record of cell c
template <typename T, int NVAL>
__device__ __forceinline__ void rec_load(const T *__restrict__ base, size_t stride, int c, T *out) {
    using V = typename Vec16<T>::type;
    constexpr int P = vpv<T>();
    const V *b = reinterpret_cast<const V *>(base);
#pragma unroll
    for (int q = 0; q < (NVAL + P - 1) / P; q++) {
        const V x = __ldg(b + (size_t)q * stride + c);
#pragma unroll
        for (int j = 0; j < P; j++)
            if (q * P + j < NVAL) out[q * P + j] = vlane(x, j);
    }
}
// store NVAL values as the record of cell c (the rest of the last vector is zero)
template <typename T, int NVAL>
__device__ __forceinline__ void rec_store(T *base, size_t stride, int c, const T *in) {
    using V = typename Vec16<T>::type;
    constexpr int P = vpv<T>();
    V *b = reinterpret_cast<V *>(base);
    auto val = [&](int i) { return i < NVAL ? in[i] : (T)0; };
#pragma unroll
    for (int q = 0; q < (NVAL + P - 1) / P; q++) {
        V x;
        if constexpr (P == 4) x = make_float4(val(4 * q), val(4 * q + 1), val(4 * q + 2), val(4 * q + 3));
        else x = make_double2(val(2 * q), val(2 * q + 1));
        b[(size_t)q * stride + c] = x;
    }
}

// The gradient records G use the same component-major layout with vectors of 16 or 32 bytes per
// precision: 32-byte vectors halve the vector loads of the face kernel (256-bit
// ld.global.nc.v4.f64 / v8.f32).  FP64 records (36 values = 9 vectors of 4) take them: the FP64
// face kernel measured 1-2 % faster; FP32 records would need padding to 40 values, and the FP32
// face kernel measured 5 % slower with them.  grec_alloc<T>() values per cell are allocated.
#ifndef FG_G_VEC_BYTES_F
#define FG_G_VEC_BYTES_F 16
#endif
#ifndef FG_G_VEC_BYTES_D
#define FG_G_VEC_BYTES_D 32
#endif
template <typename T>
__host__ __device__ constexpr int gvec_bytes() { return sizeof(T) == 4 ? FG_G_VEC_BYTES_F : FG_G_VEC_BYTES_D; }
template <typename T>
__host__ __device__ constexpr int gvec() { return gvec_bytes<T>() / (int)sizeof(T); }
template <typename T>
__host__ __device__ constexpr int grec_alloc() { return (GREC + gvec<T>() - 1) / gvec<T>() * gvec<T>(); }
template <typename T>
__host__ __device__ inline size_t grec_index(size_t stride, size_t c, int v) {
    return ((size_t)(v / gvec<T>()) * stride + c) * gvec<T>() + (size_t)(v % gvec<T>());
}
// one 32-byte vector: the loads read data that is not written during the kernel (non-coherent
// path), the stores are ordinary
__device__ __forceinline__ void ld32(const float *p, float *r) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7])
        : "l"(p));
}
__device__ __forceinline__ void ld32(const double *p, double *r) {
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(r[0]), "=d"(r[1]), "=d"(r[2]), "=d"(r[3]) : "l"(p));
}
__device__ __forceinline__ void st32(float *p, const float *r) {
    asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(r[0]), "f"(r[1]), "f"(r[2]),
                 "f"(r[3]), "f"(r[4]), "f"(r[5]), "f"(r[6]), "f"(r[7])
                 : "memory");
}
__device__ __forceinline__ void st32(double *p, const double *r) {
    asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(r[0]), "d"(r[1]), "d"(r[2]), "d"(r[3])
                 : "memory");
}
// the first NVAL values of the G record of cell c
template <typename T, int NVAL>
__device__ __forceinline__ void grec_load(const T *__restrict__ base, size_t stride, int c, T *out) {
    if constexpr (gvec_bytes<T>() == 16) {
        rec_load<T, NVAL>(base, stride, c, out);
    } else {
        constexpr int P = gvec<T>();
#pragma unroll
        for (int q = 0; q < (NVAL + P - 1) / P; q++) {
            T x[P];
            ld32(base + ((size_t)q * stride + c) * P, x);
#pragma unroll
            for (int j = 0; j < P; j++)
                if (q * P + j < NVAL) out[q * P + j] = x[j];
        }
    }
}
// store NVAL values as the G record of cell c (the rest of the last vector is zero)
template <typename T, int NVAL>
__device__ __forceinline__ void grec_store(T *base, size_t stride, int c, const T *in) {
    if constexpr (gvec_bytes<T>() == 16) {
        rec_store<T, NVAL>(base, stride, c, in);
    } else {
        constexpr int P = gvec<T>();
#pragma unroll
        for (int q = 0; q < (NVAL + P - 1) / P; q++) {
            T x[P];
#pragma unroll
            for (int j = 0; j < P; j++) x[j] = (q * P + j < NVAL) ? in[q * P + j] : (T)0;
            st32(base + ((size_t)q * stride + c) * P, x);
        }
    }
}

template <typename T>
struct PhysT {
    T gam[2], gm1[2], gp1[2], pinf[2], gpinf[2], cvgm1[2], gm1eta[2], mu[2];
    T chemLimit;
    // inlet ghost state (DP/bc.h:2-25), precomputed in FP64 on the host
    T inAlpha, inRhoL, inRhoG, inP;
    T tieTol;      // |S*| <= tieTol (|S_L| + |S_R|) counts as S* = 0 (extension; 0 = reference)
    T cp[2], prn[2];   // heat conduction (extension): k = cp mu / Pr
    T inVel[3];        // prescribed inlet velocity (extension, inVelFlag)
    T pDatum;          // pressure datum of the face momentum flux (extension, 0 = reference)
    int woods, visc, turb, energyFix, heat, limiter, inVelFlag;
};

struct PhysD {
    double gam[2], gm1[2], pinf[2], gpinf[2], cvgm1[2], gm1eta[2];
    double avfLo, avfHi;
    double pDatum;     // pressure datum of the cell-centre pressure term (PhysT::pDatum)
};

// ---------------------------------------------------------------- equation of state
template <typename T>
__device__ __forceinline__ T eos_p(const PhysT<T> &P, int m, T rho, T e) {
    return P.gm1[m] * rho * e - P.gpinf[m] - P.gm1eta[m] * rho;
}
template <typename T>
__device__ __forceinline__ T eos_e(const PhysT<T> &P, int m, T p, T rho) {
    return (p + P.gpinf[m] + P.gm1eta[m] * rho) / (rho * P.gm1[m]);
}
template <typename T>
__device__ __forceinline__ T eos_c2(const PhysT<T> &P, int m, T rho, T p) {
    return (P.gam[m] * (p + P.pinf[m])) / rho;
}

// FP64 cons -> prim at the cell centre (DP/cons2prim.h:2-24), rounded to T for storage.
template <typename S>
__device__ __forceinline__ void cons2prim_d(const PhysD &D, const double *U, S *w) {
    const double a = fmin(fmax(D.avfLo, U[0]), D.avfHi);
    const double rl = U[1] / a;
    const double rg = U[2] / (1 - a);
    const double rho = a * rl + (1 - a) * rg;
    const double el = U[6] / (a * rl);
    const double eg = U[7] / ((1 - a) * rg);
    w[0] = (S)a;
    w[1] = (S)rl;
    w[2] = (S)rg;
    w[3] = (S)(U[3] / rho);
    w[4] = (S)(U[4] / rho);
    w[5] = (S)(U[5] / rho);
    w[6] = (S)(D.gm1[0] * rl * el - D.gpinf[0] - D.gm1eta[0] * rl);
    w[7] = (S)(D.gm1[1] * rg * eg - D.gpinf[1] - D.gm1eta[1] * rg);
    w[8] = (S)U[9];
}

// Boundary ghost of a primitive state (DP/bc.h:78-84).  bc: 1 symmetry, 2 outlet, 3 inlet,
// 4 slip, 5 wall.
template <typename T>
__device__ __forceinline__ void ghost_state(const PhysT<T> &P, int bc, T nx, T ny, T nz, T *s) {
    if (bc == 1 || bc == 4) {
        const T un = s[3] * nx + s[4] * ny + s[5] * nz;
        s[3] = s[3] - 2 * un * nx;
        s[4] = s[4] - 2 * un * ny;
        s[5] = s[5] - 2 * un * nz;
    } else if (bc == 5) {
        s[3] = -s[3];
        s[4] = -s[4];
        s[5] = -s[5];
    } else if (bc == 3) {
        s[0] = P.inAlpha;
        s[1] = P.inRhoL;
        s[2] = P.inRhoG;
        s[6] = P.inP;
        s[7] = P.inP;
        s[8] = 0;
        if (P.inVelFlag) {
            s[3] = P.inVel[0];
            s[4] = P.inVel[1];
            s[5] = P.inVel[2];
        }
    }
}

// Mixture sound speed of one state (DP/waveSpeeds.h:14-34, DP/computeTimeStep.cu:34-40).
template <typename T>
__device__ __forceinline__ T mix_sound(const PhysT<T> &P, const T *s, bool wood) {
    const T c2l = eos_c2(P, 0, s[1], s[6]);
    const T c2g = eos_c2(P, 1, s[2], s[7]);
    const T al = s[0], ag = 1 - s[0];
    const T rho = al * s[1] + ag * s[2];
    if (wood) return 1 / sqrt(rho * (al / (s[1] * c2l) + ag / (s[2] * c2g)));
    return sqrt((al * s[1] * c2l + ag * s[2] * c2g) / rho);
}

// Max signal speed |u.n| + c of one face state (DP/computeTimeStep.cu:15-46).
template <typename T>
__device__ __forceinline__ T face_signal(const PhysT<T> &P, const T *s, T nx, T ny, T nz) {
    const bool wood = (s[8] > P.chemLimit) && P.woods;
    const T un = s[3] * nx + s[4] * ny + s[5] * nz;
    return fabs(un) + mix_sound(P, s, wood);
}

// HLLC face flux (DP/waveSpeeds.h, DP/starRegion.h, DP/flux.h, DP/computeRHS.cu:24-36,
// 117-131).  Output: F[10] = advective + HLLC correction (side-independent part),
// unc = star/upwind velocity . n (for the non-conservative terms), pF = upwind mixture p.
template <typename T>
__device__ __forceinline__ void hllc_flux(const PhysT<T> &P, const T *L, const T *R, T nx, T ny, T nz,
                                          T *F, T &unc, T &pF) {
    const T uL = L[3] * nx + L[4] * ny + L[5] * nz;
    const T uR = R[3] * nx + R[4] * ny + R[5] * nz;
    const bool wood = ((L[8] + R[8]) / 2 > P.chemLimit) && P.woods;
    const T cL = mix_sound(P, L, wood);
    const T cR = mix_sound(P, R, wood);
    const T SL = fmin(uL - cL, uR - cR);
    const T SR = fmax(uL + cL, uR + cR);
    const T pmL = L[0] * L[6] + (1 - L[0]) * L[7];
    const T pmR = R[0] * R[6] + (1 - R[0]) * R[7];
    const T rL = L[0] * L[1] + (1 - L[0]) * L[2];
    const T rR = R[0] * R[1] + (1 - R[0]) * R[2];
    const T Ss = (pmR - pmL + rL * uL * (SL - uL) - rR * uR * (SR - uR)) / (rL * (SL - uL) - rR * (SR - uR));
    const bool left = (Ss >= 0) || (P.tieTol > 0 && fabs(Ss) <= P.tieTol * (fabs(SL) + fabs(SR)));
    const bool star = (SL < 0) && (SR >= 0);
    T s[NP];
#pragma unroll
    for (int v = 0; v < NP; v++) s[v] = left ? L[v] : R[v];
    const T un = left ? uL : uR;
    const T cK = left ? SL : SR;
    const T pm = left ? pmL : pmR;
    const T rho = left ? rL : rR;
    // prim2cons (DP/prim2cons.h:2-21)
    const T c1 = s[0] * s[1];
    const T c2 = (1 - s[0]) * s[2];
    const T el = eos_e(P, 0, s[6], s[1]);
    const T eg = eos_e(P, 1, s[7], s[2]);
    const T ke = (T)0.5 * rho * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
    const T c6 = c1 * el, c7 = c2 * eg;
    const T c8 = c6 + c7 + ke;
    T ux = s[3], uy = s[4], uz = s[5];
    T ar6 = c6, ar7 = c7;
    T h1 = 0, h2 = 0, h3 = 0, h4 = 0, h5 = 0, h8 = 0, h9 = 0;
    if (star) {
        const T du = Ss - un;
        ux = s[3] + du * nx;
        uy = s[4] + du * ny;
        uz = s[5] + du * nz;
        const T fac = (cK - un) / (cK - Ss);
        const T rSL = s[1] * fac;
        const T rSG = s[2] * fac;
        const T v1 = s[0] * rSL;
        const T v2 = (1 - s[0]) * rSG;
        const T rS = v1 + v2;
        const T pSL = (s[6] + P.pinf[0]) * (P.gm1[0] * s[1] - P.gp1[0] * rSL) / (P.gm1[0] * rSL - P.gp1[0] * s[1]) - P.pinf[0];
        const T pSG = (s[7] + P.pinf[1]) * (P.gm1[1] * s[2] - P.gp1[1] * rSG) / (P.gm1[1] * rSG - P.gp1[1] * s[2]) - P.pinf[1];
        ar6 = v1 * eos_e(P, 0, pSL, rSL);
        ar7 = v2 * eos_e(P, 1, pSG, rSG);
        // reference energy star state (DP/starRegion.h:29); energyFix restores the rho_K factor
        const T v8 = fac * (c8 + (P.energyFix ? rho : (T)1) * du * (Ss + pm / (rho * (cK - un))));
        const T v9 = s[8] * fac;
        h1 = cK * (v1 - c1);
        h2 = cK * (v2 - c2);
        h3 = cK * (rS * ux - rho * s[3]);
        h4 = cK * (rS * uy - rho * s[4]);
        h5 = cK * (rS * uz - rho * s[5]);
        h8 = cK * (v8 - c8);
        h9 = cK * (v9 - s[8]);
    }
    const T uncn = ux * nx + uy * ny + uz * nz;
    F[0] = s[0] * uncn;
    F[1] = c1 * un + h1;
    F[2] = c2 * un + h2;
    F[3] = rho * s[3] * un + h3;
    F[4] = rho * s[4] * un + h4;
    F[5] = rho * s[5] * un + h5;
    F[6] = ar6 * uncn;
    F[7] = ar7 * uncn;
    F[8] = un * (c8 + pm) + h8;
    F[9] = s[8] * un + h9;
    unc = uncn;
    pF = pm;
}

// WALE eddy viscosity (DP/computeViscousStresses.cu:3-60) for g = grad u (row i = component);
// lsSq = Ls^2 = (0.325 Vavg^0.3333333333333)^2, precomputed per face on the host in FP64.
// Without the constants 1e-12 and 1e-10 the formula is homogeneous of degree 1 in g, and
// (S_d:S_d)^1.5 grows as |g|^6: in FP32 it overflows for gradients above about 1e6 1/s (a 200 m/s
// jet over a 10 um cell).  For |g|max = lam > 1 the FP32 path therefore evaluates it on g / lam
// with the constants divided by lam^5 and multiplies the result by lam: the same value in exact
// arithmetic.  The FP64 path evaluates the reference's expression as written.
template <typename T>
__device__ __forceinline__ T wale_nu_scaled(const T *g, T lsSq, T eps, T zeroBelow) {
    T sq[9];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) sq[i * 3 + j] = g[i * 3 + 0] * g[0 * 3 + j] + g[i * 3 + 1] * g[1 * 3 + j] + g[i * 3 + 2] * g[2 * 3 + j];
    const T tr = sq[0] + sq[4] + sq[8];
    T s1 = 0, s2 = 0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const T sd = (T)0.5 * (sq[i * 3 + j] + sq[j * 3 + i]) - ((i == j) ? tr / 3 : (T)0);
            const T st = (T)0.5 * (g[i * 3 + j] + g[j * 3 + i]);
            s1 += sd * sd;
            s2 += st * st;
        }
    const T r1 = sqrt(s1), r2 = sqrt(s2);
    T num = s1 * r1;                       // s1^1.5
    const T den = s1 * sqrt(r1) + s2 * s2 * r2 + eps;  // s1^1.25 + s2^2.5 + 1e-12
    if (den < zeroBelow) num = 0;
    return lsSq * num / den;
}
template <typename T>
__device__ __forceinline__ T wale_nu(const T *g, T lsSq) {
    return wale_nu_scaled(g, lsSq, (T)1e-12, (T)1e-10);
}
template <>
__device__ __forceinline__ float wale_nu<float>(const float *g, float lsSq) {
    float lam = 0.f;
#pragma unroll
    for (int q = 0; q < 9; q++) lam = fmaxf(lam, fabsf(g[q]));
    if (!(lam > 1.f)) return wale_nu_scaled(g, lsSq, 1e-12f, 1e-10f);
    const float inv = 1.f / lam;
    float gs[9];
#pragma unroll
    for (int q = 0; q < 9; q++) gs[q] = g[q] * inv;
    const float l2 = lam * lam, l5 = l2 * l2 * lam;   // inf above ~5e7: the constants vanish
    return lam * wale_nu_scaled(gs, lsSq, 1e-12f / l5, 1e-10f / l5);
}

}  // namespace fg
