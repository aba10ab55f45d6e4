// Phase relaxation (FP64): partition by saturation temperature, thermal (p, T) equilibrium
// Newton and chemical (p, T, Gibbs) equilibrium Newton, one thread per cell.
// Restates DP/relaxation.cu:4-75, DP/thermRlx.cu:4-235, DP/chemRlx.cu:4-267 on the device;
// the partition is decided per cell in the same kernel instead of atomic-append lists
// (cells are independent, so the result is identical and deterministic).
// Every Newton loop is bounded by the reference's iteration caps (thermItrMax, chemItrMax,
// 50 for the saturation temperature, urf > 0.0005 for step halving).
//
// With a surrogate attached, a chemical cell inside the network's training hull starts from the
// network's equilibrium prediction and takes at most `polishIters` full Newton steps on the
// reference's residuals; it is accepted when every relative residual is within `relTol`,
// otherwise (and outside the hull) the cell takes the reference Newton unchanged.
#include "fg_kernels.cuh"
#include "fg_sg_tc.cuh"

namespace fg {

namespace {

struct Ph {
    double g, pinf, cp, eta;
};

__device__ __forceinline__ double p_of(const Ph &h, double r, double e) {
    return (h.g - 1) * r * e - h.g * h.pinf - (h.g - 1) * h.eta * r;
}
__device__ __forceinline__ double t_of(const Ph &h, double r, double e) {
    const double p = (h.g - 1) * r * e - h.g * h.pinf - (h.g - 1) * h.eta * r;
    return (p + h.pinf) / ((h.cp / h.g) * (h.g - 1) * r);
}

__device__ double sat_temp(const RelaxParams &R, double P, double temp, double urf) {
    const double Pinf = R.pinf[0];
    const double g1 = R.gam[0], g2 = R.gam[1];
    const double Cp1 = R.cp[0], Cp2 = R.cp[1];
    const double Cv1 = Cp1 / g1, Cv2 = Cp2 / g2;
    const double etaT2 = R.satConst[0] * log10(P) + R.satConst[1];
    const double As = (Cp1 - Cp2 + etaT2 - 0.0) / (Cp2 - Cv2);
    const double Bs = (R.eta[0] - R.eta[1]) / (Cp2 - Cv2);
    const double Cs = (Cp2 - Cp1) / (Cp2 - Cv2);
    const double Ds = (Cp1 - Cv1) / (Cp2 - Cv2);
    const double dT = 1.e-3;
    const double lpp = Ds * log10(P + Pinf), lp = log10(P);
    double fun = 1, T = temp;
    for (int itr = 0; fabs(fun) > 1.e-2 && itr < 50; itr++) {
        fun = As + Bs / T + Cs * log10(T) + lpp - lp;
        const double fdt = As + Bs / (T + dT) + Cs * log10(T + dT) + lpp - lp;
        T = T - urf * fun / ((fdt - fun) / dT);
    }
    return T;
}

__device__ __forceinline__ void therm_res(const Ph *h, int pm, double *x, const double *ar, const double *enr,
                                          double *r0, double *r1) {
    const int mm = 1 - pm;
    const double s1 = ar[mm] / x[mm];
    const double s2 = ar[mm] * (x[2 + mm] - enr[mm]);
    x[pm] = (1 / (1 - s1)) * ar[pm];
    x[2 + pm] = enr[pm] - (1 / ar[pm]) * s2;
    *r0 = p_of(h[0], x[0], x[2]) - p_of(h[1], x[1], x[3]);
    *r1 = t_of(h[0], x[0], x[2]) - t_of(h[1], x[1], x[3]);
}

__device__ int therm_cell(const RelaxParams &R, const Ph *h, double *U, int *iters) {
    double ar[2], enr[2], x[4], ax[4];
    const double a0 = fmin(fmax(R.avfMin / 100, U[0]), 1 - R.avfMin / 100);
    const double a1 = 1 - a0;
    const double rho0 = U[1] / a0, rho1 = U[2] / a1;
    ar[0] = a0 * rho0;
    ar[1] = a1 * rho1;
    enr[0] = U[6] / ar[0];
    enr[1] = U[7] / ar[1];
    const double rm = ar[0] + ar[1];
    const double u = U[3] / rm, v = U[4] / rm, w = U[5] / rm;
    x[0] = rho0; x[1] = rho1; x[2] = enr[0]; x[3] = enr[1];
#pragma unroll
    for (int i = 0; i < 4; i++) ax[i] = x[i];
    const int pm = (a1 > a0) ? 1 : 0;
    const double de = U[8] / rm - (ar[0] / rm) * enr[0] - (ar[1] / rm) * enr[1] - 0.5 * (u * u + v * v + w * w);
    enr[0] += de;
    enr[1] += de;
    const int mm = 1 - pm;
    float minRes = 1e9f;
    int abortFlag = 0, aborted = 0;
    for (int itr = 1;; itr++) {
        *iters = itr;
        double res[2], rdf[2][2], e[2];
        therm_res(h, pm, x, ar, enr, &res[0], &res[1]);
        // finite-difference Jacobian over the minor phase's (rho, e)
        const int js[2] = {mm, mm + 2};
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int j = js[q];
            e[q] = 1e-4 * x[j];
            x[j] += e[q];
            therm_res(h, pm, x, ar, enr, &rdf[0][q], &rdf[1][q]);
            x[j] -= e[q];
        }
        double jac[2][2];
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 2; j++) {
                jac[i][j] = (rdf[i][j] - res[i]) / e[j];
                if (isnan(jac[i][j])) abortFlag = 1;
            }
        const double det = jac[0][0] * jac[1][1] - jac[1][0] * jac[0][1];
        const double i00 = jac[1][1] / det, i11 = jac[0][0] / det, i10 = -jac[1][0] / det, i01 = -jac[0][1] / det;
        if (det == 0) abortFlag = 1;
        if (abortFlag == 0 && x[0] > 0.0 && x[1] > 0.0) {
            const float chk = sqrt(res[0] * res[0] + res[1] * res[1]);
            if (chk < minRes) {
                minRes = chk;
#pragma unroll
                for (int i = 0; i < 4; i++) ax[i] = x[i];
            }
        }
        x[mm] = x[mm] - R.thermUrf * (i00 * res[0] + i01 * res[1]);
        x[mm + 2] = x[mm + 2] - R.thermUrf * (i10 * res[0] + i11 * res[1]);
        const bool conv = !(fabs(res[0]) > 1.e-2) && !(fabs(res[1]) > 1.e-2);
        if (abortFlag == 1 || itr > R.thermItrMax) {
#pragma unroll
            for (int i = 0; i < 4; i++) x[i] = ax[i];
            aborted = 1;
            break;
        }
        if (conv) break;
    }
    const double s1 = ar[mm] / x[mm];
    const double s2 = ar[mm] * (x[2 + mm] - enr[mm]);
    x[pm] = (1 / (1 - s1)) * ar[pm];
    x[2 + pm] = enr[pm] - (1 / ar[pm]) * s2;
    U[0] = fmin(fmax(R.avfMin / 100, ar[0] / x[0]), 1 - R.avfMin / 100);
    U[6] = ar[0] * x[2];
    U[7] = ar[1] * x[3];
    return aborted;
}

__device__ __forceinline__ double gibbs_of(const RelaxParams &R, int m, double P, double T) {
    const double et = (m == 1) ? R.satConst[0] * log10(P) + R.satConst[1] : 0.0;
    const double hh = R.cp[m] * T + R.eta[m];
    const double s = (R.cp[m] / R.gam[m]) * log10(pow(T, R.gam[m]) / pow(P + R.pinf[m], R.gam[m] - 1)) + et;
    return hh - T * s;
}

__device__ void chem_res(const RelaxParams &R, const Ph *h, int pm, double *x, double rm, double re, double *r) {
    const int mm = 1 - pm;
    const double s1 = x[mm], s2 = x[mm] * x[mm + 2], s3 = x[mm] * x[mm + 2] * x[mm + 4];
    x[pm] = 1 - s1;
    x[pm + 2] = (rm - s2) / x[pm];
    x[pm + 4] = (re - s3) / (x[pm] * x[pm + 2]);
    double p[2], T[2];
#pragma unroll
    for (int m = 0; m < 2; m++) {
        p[m] = p_of(h[m], x[m + 2], x[m + 4]);
        T[m] = t_of(h[m], x[m + 2], x[m + 4]);
    }
    r[0] = p[0] - p[1];
    r[1] = T[0] - T[1];
    r[2] = gibbs_of(R, 0, p[0], T[0]) - gibbs_of(R, 1, p[1], T[1]);
}

__device__ void chem_check(const RelaxParams &R, double xOld, double *x, double dx, int i, float urf, int *ab, double rho) {
    if (i == 0 || i == 1) {
        if (x[i] < 0) { while (x[i] < R.chemLimit && urf > 0.0005f) { urf = urf / 2; x[i] = xOld - urf * dx; } }
        if (x[i] > 1) { while (x[i] > 1.0 - R.chemLimit && urf > 0.0005f) { urf = urf / 2; x[i] = xOld - urf * dx; } }
        if (x[i] < 0) *ab = 1;
        if (x[i] > 1) *ab = 1;
    } else if (i == 2 || i == 3) {
        double ar = x[i - 2] * x[i];
        if (x[i] < 0) { while (x[i] < 0 && urf > 0.0005f) { urf = urf / 2; x[i] = xOld - urf * dx; } }
        if (ar > rho) { while (ar > rho && urf > 0.0005f) { urf = urf / 2; x[i] = xOld - urf * dx; ar = x[i - 2] * x[i]; } }
        if (x[i] < 0) *ab = 1;
        if (ar > rho) *ab = 1;
    }
}

__device__ int chem_cell(const RelaxParams &R, const Ph *h, double *U, int *iters) {
    double x[6], ax[6];
    x[0] = fmin(fmax(R.avfMin / 100, U[0]), 1 - R.avfMin / 100);
    x[1] = 1 - x[0];
    x[2] = U[1] / x[0];
    x[3] = U[2] / x[1];
    x[4] = U[6] / (x[0] * x[2]);
    x[5] = U[7] / (x[1] * x[3]);
#pragma unroll
    for (int i = 0; i < 6; i++) ax[i] = x[i];
    const double rm = x[0] * x[2] + x[1] * x[3];
    const double u = U[3] / rm, v = U[4] / rm, w = U[5] / rm;
    const double re = U[8] - 0.5 * rm * (u * u + v * v + w * w);
    const int pm = (x[1] > x[0]) ? 1 : 0;
    const int mm = 1 - pm;
    float minRes = 1e9f;
    int abortFlag = 0, aborted = 0;
    for (int itr = 1;; itr++) {
        *iters = itr;
        double res[3], rdf[3][3], e[3];
        chem_res(R, h, pm, x, rm, re, res);
        const int js[3] = {mm, mm + 2, mm + 4};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int j = js[q];
            e[q] = fabs(x[j]) < 1e-9 ? 1e-10 : 1.e-5 * x[j];
            x[j] += e[q];
            double rr[3];
            chem_res(R, h, pm, x, rm, re, rr);
            rdf[0][q] = rr[0]; rdf[1][q] = rr[1]; rdf[2][q] = rr[2];
            x[j] -= e[q];
        }
        double j_[3][3];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                j_[i][j] = (rdf[i][j] - res[i]) / e[j];
                if (isnan(j_[i][j])) abortFlag = 1;
            }
        const double det = j_[0][0] * (j_[1][1] * j_[2][2] - j_[1][2] * j_[2][1]) -
                           j_[0][1] * (j_[1][0] * j_[2][2] - j_[1][2] * j_[2][0]) +
                           j_[0][2] * (j_[1][0] * j_[2][1] - j_[1][1] * j_[2][0]);
        if (det == 0) abortFlag = 1;
        const double id = 1.0 / det;
        double inv[3][3];
        inv[0][0] = id * (j_[1][1] * j_[2][2] - j_[1][2] * j_[2][1]);
        inv[0][1] = -id * (j_[0][1] * j_[2][2] - j_[0][2] * j_[2][1]);
        inv[0][2] = id * (j_[0][1] * j_[1][2] - j_[0][2] * j_[1][1]);
        inv[1][0] = -id * (j_[1][0] * j_[2][2] - j_[1][2] * j_[2][0]);
        inv[1][1] = id * (j_[0][0] * j_[2][2] - j_[0][2] * j_[2][0]);
        inv[1][2] = -id * (j_[0][0] * j_[1][2] - j_[0][2] * j_[1][0]);
        inv[2][0] = id * (j_[1][0] * j_[2][1] - j_[1][1] * j_[2][0]);
        inv[2][1] = -id * (j_[0][0] * j_[2][1] - j_[0][1] * j_[2][0]);
        inv[2][2] = id * (j_[0][0] * j_[1][1] - j_[0][1] * j_[1][0]);
        if (abortFlag == 0 && x[0] > 0.0 && x[0] < 1.0 && x[1] > 0.0 && x[1] < 1.0 && x[2] > 0.0 && x[3] > 0.0) {
            const float chk = sqrt(res[0] * res[0] + res[1] * res[1] + res[2] * res[2]);
            if (chk < minRes) {
                minRes = chk;
#pragma unroll
                for (int i = 0; i < 6; i++) ax[i] = x[i];
            }
        }
        int abLocal = abortFlag;
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int i = js[q];
            const double dx = inv[q][0] * res[0] + inv[q][1] * res[1] + inv[q][2] * res[2];
            x[i] = x[i] - R.chemUrf * dx;
            chem_check(R, x[i] + R.chemUrf * dx, x, dx, i, (float)R.chemUrf, &abLocal, rm);
        }
        const bool conv = !(fabs(res[0]) > 1.e-1) && !(fabs(res[1]) > 1.e-1) && !(fabs(res[2]) > 1.e-1);
        if (abLocal == 1 || itr > R.chemItrMax) {
#pragma unroll
            for (int i = 0; i < 6; i++) x[i] = ax[i];
            aborted = 1;
            break;
        }
        if (conv) break;
    }
    const double s1 = x[mm], s2 = x[mm] * x[mm + 2], s3 = x[mm] * x[mm + 2] * x[mm + 4];
    x[pm] = 1 - s1;
    x[pm + 2] = (rm - s2) / x[pm];
    x[pm + 4] = (re - s3) / (x[pm] * x[pm + 2]);
    U[0] = fmin(fmax(R.avfMin / 100, x[0]), 1 - R.avfMin / 100);
    U[1] = x[0] * x[2];
    U[2] = x[1] * x[3];
    U[6] = x[0] * x[2] * x[4];
    U[7] = x[1] * x[3] * x[5];
    U[9] = x[1] * x[3];
    return aborted;
}

// mixture density and internal energy per unit volume exactly as chem_cell forms them
__device__ __forceinline__ void chem_mixture(const RelaxParams &R, const double *U, double *rm, double *re, double *ag) {
    const double a0 = fmin(fmax(R.avfMin / 100, U[0]), 1 - R.avfMin / 100);
    const double a1 = 1 - a0;
    const double r0 = U[1] / a0, r1 = U[2] / a1;
    const double m = a0 * r0 + a1 * r1;
    const double u = U[3] / m, v = U[4] / m, w = U[5] / m;
    *rm = m;
    *re = U[8] - 0.5 * m * (u * u + v * v + w * w);
    *ag = a1 * r1;
}

// Full-step Newton from the surrogate's equilibrium (p, T, alpha) on the residuals of chem_res.
// Returns 1 and writes U when every relative residual is within relTol.
__device__ int chem_polish(const RelaxParams &R, const Ph *h, double *U, const float *y, double rm, double re,
                           double relTol, int maxIt, int *iters) {
    const double p = y[0], T = y[1];
    if (!(T > 0) || !(p > -h[0].pinf) || !(p > -h[1].pinf)) return 0;
    double x[6];
    const double rL = (p + h[0].pinf) / ((h[0].cp / h[0].g) * (h[0].g - 1) * T);
    const double rG = (p + h[1].pinf) / ((h[1].cp / h[1].g) * (h[1].g - 1) * T);
    double a = (rm - rG) / (rL - rG);   // mass balance at (p, T)
    if (!(a > 0 && a < 1)) a = y[2];
    if (!(a > 0 && a < 1)) return 0;
    x[0] = a;
    x[1] = 1 - a;
    x[2] = rL;
    x[3] = rG;
    x[4] = (p + h[0].g * h[0].pinf) / ((h[0].g - 1) * rL) + h[0].eta;
    x[5] = (p + h[1].g * h[1].pinf) / ((h[1].g - 1) * rG) + h[1].eta;
    const int pm = (x[1] > x[0]) ? 1 : 0, mm = 1 - pm;
    const double sp = fmax(fabs(p), 1.0), sT = T, sg = h[0].cp * T;
    int ok = 0;
    for (int itr = 0; itr <= maxIt; itr++) {
        double res[3];
        chem_res(R, h, pm, x, rm, re, res);
        if (!(x[0] > 0 && x[0] < 1 && x[2] > 0 && x[3] > 0)) break;
        if (fabs(res[0]) <= relTol * sp && fabs(res[1]) <= relTol * sT && fabs(res[2]) <= relTol * sg) {
            ok = 1;
            break;
        }
        if (itr == maxIt) break;
        *iters = itr + 1;
        const int js[3] = {mm, mm + 2, mm + 4};
        double jac[3][3], e[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const int j = js[q];
            e[q] = fabs(x[j]) < 1e-9 ? 1e-10 : 1.e-5 * x[j];
            x[j] += e[q];
            double rr[3];
            chem_res(R, h, pm, x, rm, re, rr);
            x[j] -= e[q];
#pragma unroll
            for (int i = 0; i < 3; i++) jac[i][q] = (rr[i] - res[i]) / e[q];
        }
        const double det = jac[0][0] * (jac[1][1] * jac[2][2] - jac[1][2] * jac[2][1]) -
                           jac[0][1] * (jac[1][0] * jac[2][2] - jac[1][2] * jac[2][0]) +
                           jac[0][2] * (jac[1][0] * jac[2][1] - jac[1][1] * jac[2][0]);
        if (!(fabs(det) > 0) || !isfinite(det)) break;
        const double id = 1.0 / det;
        double inv[3][3];
        inv[0][0] = id * (jac[1][1] * jac[2][2] - jac[1][2] * jac[2][1]);
        inv[0][1] = -id * (jac[0][1] * jac[2][2] - jac[0][2] * jac[2][1]);
        inv[0][2] = id * (jac[0][1] * jac[1][2] - jac[0][2] * jac[1][1]);
        inv[1][0] = -id * (jac[1][0] * jac[2][2] - jac[1][2] * jac[2][0]);
        inv[1][1] = id * (jac[0][0] * jac[2][2] - jac[0][2] * jac[2][0]);
        inv[1][2] = -id * (jac[0][0] * jac[1][2] - jac[0][2] * jac[1][0]);
        inv[2][0] = id * (jac[1][0] * jac[2][1] - jac[1][1] * jac[2][0]);
        inv[2][1] = -id * (jac[0][0] * jac[2][1] - jac[0][1] * jac[2][0]);
        inv[2][2] = id * (jac[0][0] * jac[1][1] - jac[0][1] * jac[1][0]);
#pragma unroll
        for (int q = 0; q < 3; q++) x[js[q]] -= inv[q][0] * res[0] + inv[q][1] * res[1] + inv[q][2] * res[2];
    }
    if (!ok) return 0;
    U[0] = fmin(fmax(R.avfMin / 100, x[0]), 1 - R.avfMin / 100);
    U[1] = x[0] * x[2];
    U[2] = x[1] * x[3];
    U[6] = x[0] * x[2] * x[4];
    U[7] = x[1] * x[3] * x[5];
    U[9] = x[1] * x[3];
    return 1;
}

// partitionRelaxation (DP/relaxation.cu:4-75): the cell needs the chemical (Gibbs) solve when its
// liquid temperature is above the saturation temperature at its liquid pressure and its
// volume fraction above chemLimit
__device__ __forceinline__ int needs_chem(const RelaxParams &R, const Ph *h, const double *u) {
    const double avf = fmin(fmax(R.avfMin / 100, u[0]), 1 - R.avfMin / 100);
    const double rho = u[1] / avf;
    const double enr = u[6] / (avf * rho);
    const double tl = t_of(h[0], rho, enr);
    const double pl = p_of(h[0], rho, enr);
    const double ts = sat_temp(R, pl, tl, R.satTempUrf);
    return (tl > ts && avf > R.chemLimit);
}

}  // namespace

// ---- ordering of the cells for the relaxation: chemical cells first, then thermal cells, each
// in cell order (a deterministic block prefix sum; no atomics), so that every warp of the
// relaxation kernel but one runs a single branch
constexpr int kOrdThreads = 256;

__global__ void k_relax_partition(int n, const double *__restrict__ U, const RelaxParams R, uint8_t *isChem,
                                  int32_t *blockChem) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    int chem = 0;
    if (c < n) {
        const Ph h[2] = {{R.gam[0], R.pinf[0], R.cp[0], R.eta[0]}, {R.gam[1], R.pinf[1], R.cp[1], R.eta[1]}};
        double u[NV];
        u[0] = U[c];
        u[1] = U[(size_t)n + c];
        u[6] = U[(size_t)6 * n + c];
        chem = needs_chem(R, h, u);
        isChem[c] = (uint8_t)chem;
    }
    const int cnt = __syncthreads_count(chem);
    if (threadIdx.x == 0) blockChem[blockIdx.x] = cnt;
}

// exclusive scan of the per-block counts (one block of 1024 threads), total into *total
__global__ void k_relax_scan(const int32_t *cnt, int nb, int32_t *off, int32_t *total) {
    __shared__ int32_t sh[1024];
    const int t = threadIdx.x;
    const int per = (nb + 1023) / 1024;
    const int lo = min(nb, t * per), hi = min(nb, lo + per);
    int s = 0;
    for (int i = lo; i < hi; i++) s += cnt[i];
    sh[t] = s;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
        const int v = (t >= d) ? sh[t - d] : 0;
        __syncthreads();
        sh[t] += v;
        __syncthreads();
    }
    int base = t ? sh[t - 1] : 0;
    for (int i = lo; i < hi; i++) {
        off[i] = base;
        base += cnt[i];
    }
    if (t == 1023) *total = sh[1023];
}

__global__ void k_relax_order(int n, const uint8_t *isChem, const int32_t *blockOff, const int32_t *total,
                              int32_t *order) {
    __shared__ int32_t warpChem[kOrdThreads / 32];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int chem = (c < n) ? isChem[c] : 0;
    const unsigned bal = __ballot_sync(0xffffffffu, chem);
    if (lane == 0) warpChem[wid] = __popc(bal);
    __syncthreads();
    int before = 0;   // chemical cells of this block before this warp
    for (int w = 0; w < wid; w++) before += warpChem[w];
    if (c >= n) return;
    const int rankC = before + __popc(bal & ((1u << lane) - 1u));    // chemical cells before c in the block
    const int rankT = (int)threadIdx.x - rankC;                       // thermal cells before c in the block
    const int b = blockIdx.x;
    if (chem) order[blockOff[b] + rankC] = c;
    else order[*total + (b * kOrdThreads - blockOff[b]) + rankT] = c;
}


// kSG / kLog: instantiated with the surrogate path / the solve log; the plain instantiation
// carries none of their code (and none of their registers).  kPass (with kSG): the surrogate's
// polish ran before, in k_relax_polish, and the cells it accepted are skipped; otherwise the
// polish runs here.  kOrd: thread i relaxes cell order[i], chemical when i < *nChem
// (k_relax_order); otherwise thread i relaxes cell i and decides the branch itself.
// surrogate input of the relaxation: chemical cell order[i], i < *nChem
struct InRelax {
    const double *U;
    int n;
    const int32_t *order;
    const int32_t *nChem;
    RelaxParams R;
    __device__ int count() const { return *nChem; }
    __device__ void features(int i, const SurrogateNorm &N, float (&z)[3]) const {
        const int c = order[i];
        double u[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) u[v] = U[(size_t)v * n + c];
        double rm, re, ag;
        chem_mixture(R, u, &rm, &re, &ag);
        const float f[3] = {(float)rm, (float)(re / rm), (float)(ag / rm)};
#pragma unroll
        for (int k = 0; k < 3; k++) z[k] = (f[k] - N.xMean[k]) / N.xStd[k];
    }
};

// resident blocks asked of the compiler for the thermal-only instantiation (kOrd false): its
// FP64 Newton is latency-bound; 6 blocks of 128 threads (80 registers, a few spilled) measured
// 0.180 -> 0.150 ms early and 0.461 -> 0.400 ms later in the 128^3 TGV against 4 blocks
#ifndef FG_THERM_MINBLOCKS
#define FG_THERM_MINBLOCKS 6
#endif
// the same for the chemical-first instantiations (kOrd true: Gibbs and thermal Newton).  Without
// the surrogate 6 blocks (85 registers) measured 0.770 -> 0.730 ms per relaxation on a 64^3
// two-phase box (39 % chemical cells) and 1.321 -> 1.157 ms on the 4 M-tet bubble (almost all
// thermal) against 4 blocks (5 and 7 were slower on the box); uncapped (156-196 registers) was
// 2.81 ms against 1.99 at 4 blocks on the 96^3 box.  With the surrogate's polish path 4 blocks
// (128 registers) measured 0.81 -> 0.66 ms against uncapped on that box.  The same budget serves
// k_relax_polish, the surrogate's polish as a pass of its own.
#ifndef FG_CHEM_MINBLOCKS
#define FG_CHEM_MINBLOCKS 6
#endif
#ifndef FG_CHEM_SG_MINBLOCKS
#define FG_CHEM_SG_MINBLOCKS 4
#endif

// hullOk[i] of a chemical cell whose polished surrogate solution k_relax_polish accepted
constexpr int32_t kPolished = 2;

// Surrogate pass over the chemical cells (order[0 .. *nChem)), before k_relax: each cell whose
// network input lies inside the training hull (hullOk[i] = 1, k_sg_tc) is polished from the
// network's prediction pred[i]; an accepted cell gets its relaxed state (U and its W record) and
// hullOk[i] = kPolished, and k_relax leaves it alone.  Running the polish in its own kernel keeps
// its register budget off the thermal Newton's.  Grid-stride over the resident blocks.  Counts
// the polish steps (accepted or not) as Newton iterations, the accepted cells and their polish
// steps.  Its results are bitwise those of the polish inside k_relax (same arithmetic per cell).
template <typename T>
__global__ void __launch_bounds__(128, FG_CHEM_SG_MINBLOCKS) k_relax_polish(int n, double *U, T *W, size_t wStride,
                                               const PhysD D, const RelaxParams R, int32_t *counters,
                                               const SurrogateDev S, const int32_t *order, const int32_t *nChem,
                                               const float4 *pred, int32_t *hullOk) {
    const int m = *nChem;
    const Ph h[2] = {{R.gam[0], R.pinf[0], R.cp[0], R.eta[0]}, {R.gam[1], R.pinf[1], R.cp[1], R.eta[1]}};
    // base is the same for every thread of the block: the warp collectives below see full warps
    for (int base = blockIdx.x * blockDim.x; base < m; base += gridDim.x * blockDim.x) {
        const int i = base + threadIdx.x;
        int used = 0, pits = 0;
        if (i < m && hullOk[i]) {
            const int c = order[i];
            double u[NV];
#pragma unroll
            for (int v = 0; v < NV; v++) u[v] = U[(size_t)v * n + c];
            double rm, re, ag;
            chem_mixture(R, u, &rm, &re, &ag);
            const float4 p4 = pred[i];
            const float pr[4] = {p4.x, p4.y, p4.z, p4.w};
            used = chem_polish(R, h, u, pr, rm, re, S.relTol, S.polishIters, &pits);
            if (used) {
                U[(size_t)0 * n + c] = u[0];
                U[(size_t)1 * n + c] = u[1];
                U[(size_t)2 * n + c] = u[2];
                U[(size_t)6 * n + c] = u[6];
                U[(size_t)7 * n + c] = u[7];
                U[(size_t)9 * n + c] = u[9];
                T w[NP];
                cons2prim_d(D, u, w);
                rec_store<T, NP>(W, wStride, c, w);
                hullOk[i] = kPolished;
            }
        }
        const unsigned maskS = __ballot_sync(0xffffffffu, used);
        const int itsW = __reduce_add_sync(0xffffffffu, pits);
        const int polW = __reduce_add_sync(0xffffffffu, used ? pits : 0);
        if ((threadIdx.x & 31) == 0) {
            if (itsW) atomicAdd(&counters[3], itsW);
            if (maskS) atomicAdd(&counters[4], __popc(maskS));
            if (polW) atomicAdd(&counters[6], polW);
        }
    }
}

template <typename T, bool kSG, bool kLog, bool kOrd, bool kPass = false>
__global__ void __launch_bounds__(128, kOrd ? ((kSG && !kPass) ? FG_CHEM_SG_MINBLOCKS : FG_CHEM_MINBLOCKS)
                                            : FG_THERM_MINBLOCKS) k_relax(int n, double *U, T *W, size_t wStride, const PhysD D, const RelaxParams R,
                                               int32_t *counters, const SurrogateDev S, const RelaxLog Lg,
                                               const int32_t *order, const int32_t *nChem, const float4 *pred,
                                               const int32_t *hullOk) {
    constexpr bool kPolish = kSG && !kPass;   // the polish runs in this kernel
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool act = i < n;
    const int c = (kOrd && act) ? order[i] : i;
    int chem = 0, ab = 0, its = 0, used = 0, pits = 0;
    const Ph h[2] = {{R.gam[0], R.pinf[0], R.cp[0], R.eta[0]}, {R.gam[1], R.pinf[1], R.cp[1], R.eta[1]}};
    double u[NV];
    double rm = 0, re = 0, ag = 0;
    if (act) {
        // kOrd: cells ordered chemical-first (chemFlag == 1); otherwise every cell is thermal
        // (chemFlag != 1), and the chemical solver is compiled out of this instantiation
        if (kOrd) chem = i < *nChem;
        // relaxed already by the surrogate pass
        if (kSG && kPass && chem) used = hullOk[i] == kPolished;
    }
    if (act && !used) {
#pragma unroll
        for (int v = 0; v < NV; v++) u[v] = U[(size_t)v * n + c];
        if (chem && (kPolish || kLog)) chem_mixture(R, u, &rm, &re, &ag);
        // the network's prediction for this cell (k_sg_tc over the chemical cells) if its input
        // is inside the training hull
        if (kPolish && chem && hullOk[i] != 0) {
            const float4 p4 = pred[i];
            const float pr[4] = {p4.x, p4.y, p4.z, p4.w};
            used = chem_polish(R, h, u, pr, rm, re, S.relTol, S.polishIters, &pits);
        }
        if (!used) {
            ab = (kOrd && chem) ? chem_cell(R, h, u, &its) : therm_cell(R, h, u, &its);
        }
        if (kLog && chem && !used && !ab) {
            // training sample: (rho, e, Y) before the solve -> (p, T, alpha, Y_eq) after it
            const unsigned long long k = atomicAdd(Lg.count, 1ULL);
            if (k < (unsigned long long)Lg.cap) {
                const double a0 = fmin(fmax(R.avfMin / 100, u[0]), 1 - R.avfMin / 100);
                const double rL = u[1] / a0, eL = u[6] / u[1];
                float *x = Lg.X + k * 3, *y = Lg.Y + k * 4;
                x[0] = (float)rm;
                x[1] = (float)(re / rm);
                x[2] = (float)(ag / rm);
                y[0] = (float)p_of(h[0], rL, eL);
                y[1] = (float)t_of(h[0], rL, eL);
                y[2] = (float)a0;
                y[3] = (float)(u[9] / rm);
            }
        }
        its += pits;   // polish steps count as Newton iterations (accepted or not)
        U[(size_t)0 * n + c] = u[0];
        U[(size_t)1 * n + c] = u[1];
        U[(size_t)2 * n + c] = u[2];
        U[(size_t)6 * n + c] = u[6];
        U[(size_t)7 * n + c] = u[7];
        U[(size_t)9 * n + c] = u[9];
        T w[NP];
        cons2prim_d(D, u, w);
        rec_store<T, NP>(W, wStride, c, w);
    }
    // warp-aggregated counters (sums of integers: order does not matter)
    const unsigned mask = __ballot_sync(0xffffffffu, act && chem);
    const unsigned maskT = __ballot_sync(0xffffffffu, act && !chem);
    const unsigned maskA = __ballot_sync(0xffffffffu, act && ab);
    // accepted cells and their polish steps: counted here when the polish ran here
    const unsigned maskS = kPolish ? __ballot_sync(0xffffffffu, act && used) : 0u;
    const unsigned maskF = __ballot_sync(0xffffffffu, act && chem && kSG && !used);
    const int itsW = __reduce_add_sync(0xffffffffu, its);
    const int polW = kPolish ? __reduce_add_sync(0xffffffffu, used ? pits : 0) : 0;
    if ((threadIdx.x & 31) == 0) {
        if (maskT) atomicAdd(&counters[0], __popc(maskT));
        if (mask) atomicAdd(&counters[1], __popc(mask));
        if (maskA) atomicAdd(&counters[2], __popc(maskA));
        if (itsW) atomicAdd(&counters[3], itsW);
        if (maskS) atomicAdd(&counters[4], __popc(maskS));
        if (maskF) atomicAdd(&counters[5], __popc(maskF));
        if (polW) atomicAdd(&counters[6], polW);
    }
}

int relax_order_blocks(int n) { return (n + kOrdThreads - 1) / kOrdThreads; }

template <typename T, bool kOrd>
static void launch_relax_k(int n, double *U, T *W, size_t wStride, const PhysD &D, const RelaxParams &R, int32_t *counters,
                           const SurrogateDev &S, const RelaxLog &L, const RelaxOrder *O, cudaStream_t s) {
    const int nb = (n + 127) / 128;
    const bool lg = L.count != nullptr;
    const int32_t *order = O ? O->order : nullptr, *nChem = O ? O->total : nullptr;
    const float4 *pred = O ? O->pred : nullptr;
    const int32_t *hull = O ? O->hullOk : nullptr;
    if constexpr (kOrd) {
        // the surrogate runs only with the chemical-first order; the logged instantiation keeps
        // the polish inside (launch_relax runs no separate pass with the log on)
        if (S.enabled) {
            if (lg)
                k_relax<T, true, true, kOrd><<<nb, 128, 0, s>>>(n, U, W, wStride, D, R, counters, S, L, order, nChem, pred, hull);
            else if (O->polishPass)
                k_relax<T, true, false, kOrd, true><<<nb, 128, 0, s>>>(n, U, W, wStride, D, R, counters, S, L, order, nChem, pred, hull);
            else
                k_relax<T, true, false, kOrd><<<nb, 128, 0, s>>>(n, U, W, wStride, D, R, counters, S, L, order, nChem, pred, hull);
            return;
        }
    }
    if (lg)
        k_relax<T, false, true, kOrd><<<nb, 128, 0, s>>>(n, U, W, wStride, D, R, counters, S, L, order, nChem, pred, hull);
    else
        k_relax<T, false, false, kOrd><<<nb, 128, 0, s>>>(n, U, W, wStride, D, R, counters, S, L, order, nChem, pred, hull);
}

template <typename T>
int launch_relax(int n, double *U, T *W, size_t wStride, const PhysD &D, const RelaxParams &R, int32_t *counters,
                 const SurrogateDev &S, const RelaxLog &L, const RelaxOrder &O, cudaStream_t s) {
    if (R.chemFlag != 1) {
        // every cell is thermal: no ordering needed (and no surrogate)
        launch_relax_k<T, false>(n, U, W, wStride, D, R, counters, SurrogateDev{}, L, nullptr, s);
        return 1;
    }
    const int nb = relax_order_blocks(n);
    k_relax_partition<<<nb, kOrdThreads, 0, s>>>(n, U, R, O.isChem, O.blockCnt);
    k_relax_scan<<<1, 1024, 0, s>>>(O.blockCnt, nb, O.blockOff, O.total);
    k_relax_order<<<nb, kOrdThreads, 0, s>>>(n, O.isChem, O.blockOff, O.total, O.order);
    int k = 4;
    if (S.enabled) {
        // the network on the tensor cores for the chemical cells (order[0 .. nChem)), tiles of 128
        const int tiles = (n + TC_M - 1) / TC_M;
        k_sg_tc<InRelax><<<std::min(tiles, 148 * 4), 128, TC_SMEM, s>>>(S, S.pack, InRelax{U, n, O.order, O.total, R},
                                                                        O.pred, O.hullOk, O.tcErr);
        k++;
        if (O.polishPass && L.count == nullptr) {
            k_relax_polish<T><<<std::min((n + 127) / 128, 148 * FG_CHEM_SG_MINBLOCKS), 128, 0, s>>>(
                n, U, W, wStride, D, R, counters, S, O.order, O.total, O.pred, O.hullOk);
            k++;
        }
    }
    launch_relax_k<T, true>(n, U, W, wStride, D, R, counters, S, L, &O, s);
    return k;
}

template int launch_relax<float>(int, double *, float *, size_t, const PhysD &, const RelaxParams &, int32_t *,
                                 const SurrogateDev &, const RelaxLog &, const RelaxOrder &, cudaStream_t);
template int launch_relax<double>(int, double *, double *, size_t, const PhysD &, const RelaxParams &, int32_t *,
                                  const SurrogateDev &, const RelaxLog &, const RelaxOrder &, cudaStream_t);

}  // namespace fg
