// Learned equilibrium surrogate: training (forward / backward / Adam on the GPU, FP32), batch
// prediction through the BF16 tensor-core forward the relaxation kernel uses, and the C ABI
// (fg_surrogate_*).  It has no counterpart in the reference, whose chemical relaxation is the
// per-cell Newton of DP/chemRlx.cu:4-267; the network only supplies that Newton's starting point.
//
// Training: inputs (rho, e, Y) and targets (p, T, alpha, Y_eq) are standardised with the
// statistics of the training set; loss = mean squared error over the 4 standardised outputs;
// parameters are FP32 with Adam.  Every reduction over samples (weight gradients, loss) sums
// fixed chunks in a fixed order, so training is deterministic for a given seed.
#include "../../include/fooskagpu.h"
#include "fg_sg_tc.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace fg {
int set_error(int code, const std::string &msg);
}
static_assert(fg::SG_NPARAM == FG_SG_NPARAM, "parameter count of the C header");
static_assert(sizeof(fg::SurrogateNorm) == FG_SG_NNORM * sizeof(float), "normalisation record of the C header");

using namespace fg;

namespace {

struct Buf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaError_t alloc(size_t b) {
        release();
        bytes = b;
        return cudaMalloc(&p, b ? b : 16);
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    ~Buf() { release(); }
    template <typename X> X *as() const { return static_cast<X *>(p); }
};

#define SG_TRY(expr)                                                                                  \
    do {                                                                                              \
        cudaError_t e_ = (expr);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fg::set_error(e_ == cudaErrorMemoryAllocation ? FG_ERR_NOMEM : FG_ERR_CUDA,        \
                                 std::string(#expr) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

constexpr int kChunks = 64;   // sample chunks of the weight-gradient reduction

// GELU (tanh form) and its derivative in training: with u = c (z + a z^3), th = tanh(u),
//   gelu = z / 2 (1 + th),  gelu' = (1 + th) / 2 + z / 2 (1 - th^2) c (1 + 3 a z^2)
__device__ __forceinline__ float gelu_f(float z) {
    return 0.5f * z * (1.0f + tanhf(SG_GELU_C * fmaf(SG_GELU_A * z, z * z, z)));
}
__device__ __forceinline__ float gelu_d(float z) {
    const float th = tanhf(SG_GELU_C * fmaf(SG_GELU_A * z, z * z, z));
    return 0.5f * (1.0f + th) + 0.5f * z * (1.0f - th * th) * SG_GELU_C * fmaf(3.0f * SG_GELU_A * z, z, 1.0f);
}

// rows of X and Y selected by perm[start .. start+B)
__global__ void k_sg_gather(const int32_t *perm, int start, int B, const float *X, const float *Y, float *bx,
                            float *by) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B) return;
    const int s = perm[start + i];
#pragma unroll
    for (int k = 0; k < SG_IN; k++) bx[(size_t)i * SG_IN + k] = X[(size_t)s * SG_IN + k];
#pragma unroll
    for (int k = 0; k < SG_OUT; k++) by[(size_t)i * SG_OUT + k] = Y[(size_t)s * SG_OUT + k];
}

// Z = X W + b (X: B x K, W: K x N row-major), A = gelu(Z) (act) or Z
__global__ void k_dense_fwd(const float *X, int K, const float *W, const float *b, int N, int B, float *Z, float *A,
                            int act) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * N) return;
    const int r = i / N, n = i - r * N;
    float z = b[n];
    for (int k = 0; k < K; k++) z = fmaf(X[(size_t)r * K + k], W[k * N + n], z);
    if (Z) Z[i] = z;
    A[i] = act ? gelu_f(z) : z;
}

// dY = 2 (Y - T) / (B * 4); per-block partial sums of the squared error
__global__ void k_sg_loss(const float *Yp, const float *Tt, int cnt, float scale, float *dY, float *part) {
    __shared__ float sh[256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float e = 0.f;
    if (i < cnt) {
        const float d = Yp[i] - Tt[i];
        dY[i] = 2.f * d * scale;
        e = d * d;
    }
    sh[threadIdx.x] = e;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// dX = (dZ W^T) * gelu'(Zprev)  (dZ: B x N, W: K x N, Zprev: B x K)
__global__ void k_dense_bwd_data(const float *dZ, const float *W, int N, int K, const float *Zprev, int B,
                                 float *dX) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * K) return;
    const int r = i / K, k = i - r * K;
    float s = 0.f;
    for (int n = 0; n < N; n++) s = fmaf(dZ[(size_t)r * N + n], W[k * N + n], s);
    dX[i] = s * gelu_d(Zprev[i]);
}

// partial weight / bias gradients over one chunk of samples:
// part[chunk][k*N+n] = sum_r A[r][k] dZ[r][n],  part[chunk][K*N+n] = sum_r dZ[r][n]
__global__ void k_dense_bwd_w(const float *A, const float *dZ, int B, int K, int N, int chunk, float *part) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int nq = K * N + N;
    if (q >= nq) return;
    const int c = blockIdx.y;
    const int r0 = c * chunk, r1 = min(B, r0 + chunk);
    float s = 0.f;
    if (q < K * N) {
        const int k = q / N, n = q - k * N;
        for (int r = r0; r < r1; r++) s = fmaf(A[(size_t)r * K + k], dZ[(size_t)r * N + n], s);
    } else {
        const int n = q - K * N;
        for (int r = r0; r < r1; r++) s += dZ[(size_t)r * N + n];
    }
    part[(size_t)c * nq + q] = s;
}

// g[wOff + k*N+n] / g[bOff + n] = sum over chunks in order
__global__ void k_reduce_chunks(const float *part, int chunks, int K, int N, float *g, int wOff, int bOff) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int nq = K * N + N;
    if (q >= nq) return;
    float s = 0.f;
    for (int c = 0; c < chunks; c++) s += part[(size_t)c * nq + q];
    if (q < K * N) g[wOff + q] = s;
    else g[bOff + (q - K * N)] = s;
}

__global__ void k_adam(float *P, const float *G, float *M, float *V, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = G[i];
    const float m = b1 * M[i] + (1.f - b1) * g;
    const float v = b2 * V[i] + (1.f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

// batch prediction input: raw samples X[n][3]
struct InPredict {
    const float *X;
    int n;
    __device__ int count() const { return n; }
    __device__ void features(int i, const SurrogateNorm &N, float (&z)[3]) const {
#pragma unroll
        for (int k = 0; k < 3; k++) z[k] = (X[(size_t)i * 3 + k] - N.xMean[k]) / N.xStd[k];
    }
};

// ---------------------------------------------------------------- host helpers
uint16_t bf16_rne(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) return (uint16_t)((u >> 16) | 0x40u);   // NaN
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return (uint16_t)(u >> 16);
}

// one layer W[K][N] (row-major, in x out) as the B operand of the tensor-core layer: N rows of
// K (K-major), K padded to 16 * kSlabs and N to nPad with zeros, in the canonical layout
void pack_layer_tc(const float *W, int K, int N, int kSlabs, int nPad, unsigned char *out) {
    for (int n = 0; n < nPad; n++)
        for (int k = 0; k < 16 * kSlabs; k++) {
            const uint16_t v = (k < K && n < N) ? bf16_rne(W[k * N + n]) : (uint16_t)0;
            std::memcpy(out + tc_smem_off_host(n, k, nPad), &v, 2);
        }
}

bool invert3(const double *a, double *inv) {
    const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                       a[2] * (a[3] * a[7] - a[4] * a[6]);
    if (!(std::fabs(det) > 0)) return false;
    const double id = 1.0 / det;
    inv[0] = (a[4] * a[8] - a[5] * a[7]) * id;
    inv[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    inv[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    inv[3] = (a[5] * a[6] - a[3] * a[8]) * id;
    inv[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    inv[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    inv[6] = (a[3] * a[7] - a[4] * a[6]) * id;
    inv[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    inv[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    return true;
}

}  // namespace

struct fg_surrogate {
    int device = 0;
    Buf P, G, M, V, pack;           // parameters, gradient, Adam moments, packed BF16 fragments
    Buf X, Y;                       // standardised training data (n x 3, n x 4)
    Buf perm;
    int64_t n = 0;
    int64_t adamStep = 0;
    SurrogateNorm norm{};
    bool hasNorm = false;
    // batch work buffers (capacity cap rows)
    int cap = 0;
    Buf bx, by, z1, a1, z2, a2, z3, a3, yp, dy, d3, d2, d1, part, lossPart;

    int ensure_batch(int B) {
        if (B <= cap) return FG_OK;
        cap = B;
        const size_t h = (size_t)B * SG_H * sizeof(float);
        SG_TRY(bx.alloc((size_t)B * SG_IN * sizeof(float)));
        SG_TRY(by.alloc((size_t)B * SG_OUT * sizeof(float)));
        for (Buf *b : {&z1, &a1, &z2, &a2, &z3, &a3, &d3, &d2, &d1}) SG_TRY(b->alloc(h));
        SG_TRY(yp.alloc((size_t)B * SG_OUT * sizeof(float)));
        SG_TRY(dy.alloc((size_t)B * SG_OUT * sizeof(float)));
        SG_TRY(part.alloc((size_t)kChunks * (SG_H * SG_H + SG_H) * sizeof(float)));
        SG_TRY(lossPart.alloc((size_t)((B * SG_OUT + 255) / 256) * sizeof(float)));
        return FG_OK;
    }

    int repack() {
        std::vector<float> p(SG_NPARAM);
        SG_TRY(cudaMemcpy(p.data(), P.p, SG_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
        std::vector<unsigned char> pk(TC_WBYTES, 0);
        pack_layer_tc(p.data() + SG_OFF_W1, SG_IN, SG_H, 1, 64, pk.data() + TC_W1);
        pack_layer_tc(p.data() + SG_OFF_W2, SG_H, SG_H, 4, 64, pk.data() + TC_W2);
        pack_layer_tc(p.data() + SG_OFF_W3, SG_H, SG_H, 4, 64, pk.data() + TC_W3);
        pack_layer_tc(p.data() + SG_OFF_W4, SG_H, SG_OUT, 4, 16, pk.data() + TC_W4);
        SG_TRY(cudaMemcpy(pack.p, pk.data(), TC_WBYTES, cudaMemcpyHostToDevice));
        return FG_OK;
    }

    // forward + loss + backward over the batch in bx / by (standardised); grad into G
    int fwd_bwd(int B, float *lossOut, cudaStream_t s) {
        const float *Pp = P.as<float>();
        float *Gp = G.as<float>();
        const int T = 256;
        auto grid = [&](long long c) { return (int)((c + T - 1) / T); };
        k_dense_fwd<<<grid((long long)B * SG_H), T, 0, s>>>(bx.as<float>(), SG_IN, Pp + SG_OFF_W1, Pp + SG_OFF_B1, SG_H, B,
                                                           z1.as<float>(), a1.as<float>(), 1);
        k_dense_fwd<<<grid((long long)B * SG_H), T, 0, s>>>(a1.as<float>(), SG_H, Pp + SG_OFF_W2, Pp + SG_OFF_B2, SG_H, B,
                                                           z2.as<float>(), a2.as<float>(), 1);
        k_dense_fwd<<<grid((long long)B * SG_H), T, 0, s>>>(a2.as<float>(), SG_H, Pp + SG_OFF_W3, Pp + SG_OFF_B3, SG_H, B,
                                                           z3.as<float>(), a3.as<float>(), 1);
        k_dense_fwd<<<grid((long long)B * SG_OUT), T, 0, s>>>(a3.as<float>(), SG_H, Pp + SG_OFF_W4, Pp + SG_OFF_B4, SG_OUT,
                                                             B, nullptr, yp.as<float>(), 0);
        const int cnt = B * SG_OUT;
        const int nLoss = grid(cnt);
        k_sg_loss<<<nLoss, T, 0, s>>>(yp.as<float>(), by.as<float>(), cnt, 1.0f / (float)cnt, dy.as<float>(),
                                      lossPart.as<float>());
        const int chunk = (B + kChunks - 1) / kChunks;
        auto wgrad = [&](const float *A, const float *dZ, int K, int N, int wOff, int bOff) {
            dim3 g2(grid((long long)K * N + N), kChunks);
            k_dense_bwd_w<<<g2, T, 0, s>>>(A, dZ, B, K, N, chunk, part.as<float>());
            k_reduce_chunks<<<grid((long long)K * N + N), T, 0, s>>>(part.as<float>(), kChunks, K, N, Gp, wOff, bOff);
        };
        // layer 4 (linear): dZ4 = dy
        wgrad(a3.as<float>(), dy.as<float>(), SG_H, SG_OUT, SG_OFF_W4, SG_OFF_B4);
        k_dense_bwd_data<<<grid((long long)B * SG_H), T, 0, s>>>(dy.as<float>(), Pp + SG_OFF_W4, SG_OUT, SG_H,
                                                                z3.as<float>(), B, d3.as<float>());
        wgrad(a2.as<float>(), d3.as<float>(), SG_H, SG_H, SG_OFF_W3, SG_OFF_B3);
        k_dense_bwd_data<<<grid((long long)B * SG_H), T, 0, s>>>(d3.as<float>(), Pp + SG_OFF_W3, SG_H, SG_H,
                                                                z2.as<float>(), B, d2.as<float>());
        wgrad(a1.as<float>(), d2.as<float>(), SG_H, SG_H, SG_OFF_W2, SG_OFF_B2);
        k_dense_bwd_data<<<grid((long long)B * SG_H), T, 0, s>>>(d2.as<float>(), Pp + SG_OFF_W2, SG_H, SG_H,
                                                                z1.as<float>(), B, d1.as<float>());
        wgrad(bx.as<float>(), d1.as<float>(), SG_IN, SG_H, SG_OFF_W1, SG_OFF_B1);
        SG_TRY(cudaGetLastError());
        if (lossOut) {
            std::vector<float> lp(nLoss);
            SG_TRY(cudaMemcpyAsync(lp.data(), lossPart.p, nLoss * sizeof(float), cudaMemcpyDeviceToHost, s));
            SG_TRY(cudaStreamSynchronize(s));
            double sum = 0;
            for (float v : lp) sum += v;
            *lossOut = (float)(sum / cnt);
        }
        return FG_OK;
    }
};

namespace fg {
// device view of a surrogate for the relaxation kernel
int surrogate_view(const fg_surrogate *g, SurrogateDev *out) {
    if (!g || !g->hasNorm) return fg::set_error(FG_ERR_ARG, "surrogate has no training data statistics");
    out->pack = g->pack.as<unsigned char>();
    out->params = g->P.as<float>();
    out->norm = g->norm;
    out->enabled = 1;
    return FG_OK;
}
int surrogate_device(const fg_surrogate *g) { return g ? g->device : -1; }
}  // namespace fg

extern "C" {

int fg_surrogate_create(int32_t device, uint64_t seed, fg_surrogate **out) {
    if (!out) return fg::set_error(FG_ERR_ARG, "fg_surrogate_create: null argument");
    *out = nullptr;
    SG_TRY(cudaSetDevice(device));
    fg_surrogate *g = new fg_surrogate();
    g->device = device;
    int rc = FG_OK;
    auto fail = [&](int code) { delete g; return code; };
    if (cudaSuccess != g->P.alloc(SG_NPARAM * sizeof(float)) || cudaSuccess != g->G.alloc(SG_NPARAM * sizeof(float)) ||
        cudaSuccess != g->M.alloc(SG_NPARAM * sizeof(float)) || cudaSuccess != g->V.alloc(SG_NPARAM * sizeof(float)) ||
        cudaSuccess != g->pack.alloc(TC_WBYTES))
        return fail(fg::set_error(FG_ERR_NOMEM, "fg_surrogate_create: device allocation failed"));
    // He-style initialisation: W ~ N(0, 2 / fan_in), b = 0 (seeded, reproducible)
    std::vector<float> p(SG_NPARAM, 0.f);
    std::mt19937_64 rng(seed);
    auto init = [&](int off, int K, int N) {
        std::normal_distribution<double> nd(0.0, std::sqrt(2.0 / K));
        for (int i = 0; i < K * N; i++) p[off + i] = (float)nd(rng);
    };
    init(SG_OFF_W1, SG_IN, SG_H);
    init(SG_OFF_W2, SG_H, SG_H);
    init(SG_OFF_W3, SG_H, SG_H);
    init(SG_OFF_W4, SG_H, SG_OUT);
    if (cudaMemcpy(g->P.p, p.data(), SG_NPARAM * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(g->M.p, 0, SG_NPARAM * sizeof(float)) != cudaSuccess ||
        cudaMemset(g->V.p, 0, SG_NPARAM * sizeof(float)) != cudaSuccess ||
        cudaMemset(g->G.p, 0, SG_NPARAM * sizeof(float)) != cudaSuccess)
        return fail(fg::set_error(FG_ERR_CUDA, "fg_surrogate_create: initialisation copy failed"));
    rc = g->repack();
    if (rc != FG_OK) return fail(rc);
    *out = g;
    return FG_OK;
}

int fg_surrogate_destroy(fg_surrogate *g) {
    if (!g) return FG_OK;
    cudaSetDevice(g->device);
    delete g;
    return FG_OK;
}

int fg_surrogate_set_data(fg_surrogate *g, const float *X, const float *Y, int64_t n) {
    if (!g || !X || !Y) return fg::set_error(FG_ERR_ARG, "fg_surrogate_set_data: null argument");
    if (n < 16 || n > (int64_t)INT32_MAX) return fg::set_error(FG_ERR_ARG, "fg_surrogate_set_data: need 16 .. 2^31-1 samples");
    SG_TRY(cudaSetDevice(g->device));
    // statistics of the run's samples (FP64 accumulation)
    double mx[3] = {0, 0, 0}, my[4] = {0, 0, 0, 0}, sx[3] = {0, 0, 0}, sy[4] = {0, 0, 0, 0};
    for (int64_t i = 0; i < n; i++) {
        for (int k = 0; k < 3; k++) mx[k] += X[i * 3 + k];
        for (int k = 0; k < 4; k++) my[k] += Y[i * 4 + k];
    }
    for (int k = 0; k < 3; k++) mx[k] /= (double)n;
    for (int k = 0; k < 4; k++) my[k] /= (double)n;
    for (int64_t i = 0; i < n; i++) {
        for (int k = 0; k < 3; k++) sx[k] += (X[i * 3 + k] - mx[k]) * (X[i * 3 + k] - mx[k]);
        for (int k = 0; k < 4; k++) sy[k] += (Y[i * 4 + k] - my[k]) * (Y[i * 4 + k] - my[k]);
    }
    SurrogateNorm N{};
    for (int k = 0; k < 3; k++) {
        N.xMean[k] = (float)mx[k];
        N.xStd[k] = (float)std::max(std::sqrt(sx[k] / (double)n), 1e-30);
    }
    for (int k = 0; k < 4; k++) {
        N.yMean[k] = (float)my[k];
        N.yStd[k] = (float)std::max(std::sqrt(sy[k] / (double)n), 1e-30);
    }
    std::vector<float> xs((size_t)n * 3), ys((size_t)n * 4);
    double cov[9] = {0};
    for (int k = 0; k < 3; k++) {
        N.boxLo[k] = 1e30f;
        N.boxHi[k] = -1e30f;
    }
    for (int64_t i = 0; i < n; i++) {
        float z[3];
        for (int k = 0; k < 3; k++) {
            z[k] = (X[i * 3 + k] - N.xMean[k]) / N.xStd[k];
            xs[i * 3 + k] = z[k];
            N.boxLo[k] = std::min(N.boxLo[k], z[k]);
            N.boxHi[k] = std::max(N.boxHi[k], z[k]);
        }
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) cov[3 * a + b] += (double)z[a] * z[b];
        for (int k = 0; k < 4; k++) ys[i * 4 + k] = (Y[i * 4 + k] - N.yMean[k]) / N.yStd[k];
    }
    for (double &c : cov) c /= (double)n;
    double ci[9];
    if (!invert3(cov, ci)) return fg::set_error(FG_ERR_ARG, "fg_surrogate_set_data: degenerate input covariance");
    for (int k = 0; k < 9; k++) N.covInv[k] = (float)ci[k];
    double d2m = 0;
    for (int64_t i = 0; i < n; i++) {
        double d2 = 0;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) d2 += (double)xs[i * 3 + a] * N.covInv[3 * a + b] * xs[i * 3 + b];
        d2m = std::max(d2m, d2);
    }
    N.d2Max = (float)d2m;
    SG_TRY(g->X.alloc(xs.size() * sizeof(float)));
    SG_TRY(g->Y.alloc(ys.size() * sizeof(float)));
    SG_TRY(g->perm.alloc((size_t)n * sizeof(int32_t)));
    SG_TRY(cudaMemcpy(g->X.p, xs.data(), xs.size() * sizeof(float), cudaMemcpyHostToDevice));
    SG_TRY(cudaMemcpy(g->Y.p, ys.data(), ys.size() * sizeof(float), cudaMemcpyHostToDevice));
    g->n = n;
    g->norm = N;
    g->hasNorm = true;
    return FG_OK;
}

int fg_surrogate_train(fg_surrogate *g, int32_t epochs, int32_t batch, float lr, uint64_t seed, float *finalLoss) {
    if (!g) return fg::set_error(FG_ERR_ARG, "fg_surrogate_train: null argument");
    if (g->n == 0) return fg::set_error(FG_ERR_ARG, "fg_surrogate_train: no training data (fg_surrogate_set_data)");
    if (epochs < 0 || batch < 32 || batch > (1 << 20) || !(lr > 0))
        return fg::set_error(FG_ERR_ARG, "fg_surrogate_train: epochs >= 0, 32 <= batch <= 2^20, lr > 0");
    SG_TRY(cudaSetDevice(g->device));
    int rc = g->ensure_batch(batch);
    if (rc != FG_OK) return rc;
    cudaStream_t s = 0;
    std::mt19937_64 rng(seed);
    std::vector<int32_t> perm((size_t)g->n);
    for (int64_t i = 0; i < g->n; i++) perm[i] = (int32_t)i;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    double epochLoss = 0;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(perm.begin(), perm.end(), rng);
        SG_TRY(cudaMemcpy(g->perm.p, perm.data(), perm.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
        const int64_t nb = g->n / batch;   // full batches only
        double sum = 0;
        // cosine decay of the learning rate over the whole run
        for (int64_t b = 0; b < nb; b++) {
            k_sg_gather<<<(batch + 255) / 256, 256, 0, s>>>(g->perm.as<int32_t>(), (int)(b * batch), batch,
                                                            g->X.as<float>(), g->Y.as<float>(), g->bx.as<float>(),
                                                            g->by.as<float>());
            const bool last = (b == nb - 1);
            float l = 0;
            rc = g->fwd_bwd(batch, last ? &l : nullptr, s);
            if (rc != FG_OK) return rc;
            if (last) sum = l;
            g->adamStep++;
            const double prog = ((double)ep * nb + b) / std::max<double>(1.0, (double)epochs * nb);
            const float lrt = (float)(lr * 0.5 * (1.0 + std::cos(3.14159265358979 * prog)));
            const float c1 = 1.f - std::pow(b1, (float)g->adamStep), c2 = 1.f - std::pow(b2, (float)g->adamStep);
            k_adam<<<(SG_NPARAM + 255) / 256, 256, 0, s>>>(g->P.as<float>(), g->G.as<float>(), g->M.as<float>(),
                                                          g->V.as<float>(), SG_NPARAM, lrt, b1, b2, eps, c1, c2);
        }
        SG_TRY(cudaGetLastError());
        epochLoss = sum;
    }
    SG_TRY(cudaDeviceSynchronize());
    rc = g->repack();
    if (rc != FG_OK) return rc;
    if (finalLoss) *finalLoss = (float)epochLoss;
    return FG_OK;
}

int fg_surrogate_loss_grad(fg_surrogate *g, const float *X, const float *Y, int32_t n, float *loss, float *grad) {
    if (!g || !X || !Y || !grad) return fg::set_error(FG_ERR_ARG, "fg_surrogate_loss_grad: null argument");
    if (n < 1 || n > (1 << 20)) return fg::set_error(FG_ERR_ARG, "fg_surrogate_loss_grad: 1 <= n <= 2^20");
    SG_TRY(cudaSetDevice(g->device));
    int rc = g->ensure_batch(n);
    if (rc != FG_OK) return rc;
    SG_TRY(cudaMemcpy(g->bx.p, X, (size_t)n * SG_IN * sizeof(float), cudaMemcpyHostToDevice));
    SG_TRY(cudaMemcpy(g->by.p, Y, (size_t)n * SG_OUT * sizeof(float), cudaMemcpyHostToDevice));
    float l = 0;
    rc = g->fwd_bwd(n, &l, 0);
    if (rc != FG_OK) return rc;
    SG_TRY(cudaMemcpy(grad, g->G.p, SG_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
    return FG_OK;
}

int fg_surrogate_get_params(fg_surrogate *g, float *params) {
    if (!g || !params) return fg::set_error(FG_ERR_ARG, "fg_surrogate_get_params: null argument");
    SG_TRY(cudaSetDevice(g->device));
    SG_TRY(cudaMemcpy(params, g->P.p, SG_NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    return FG_OK;
}

int fg_surrogate_set_params(fg_surrogate *g, const float *params) {
    if (!g || !params) return fg::set_error(FG_ERR_ARG, "fg_surrogate_set_params: null argument");
    SG_TRY(cudaSetDevice(g->device));
    SG_TRY(cudaMemcpy(g->P.p, params, SG_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
    return g->repack();
}

int fg_surrogate_get_norm(fg_surrogate *g, float *norm) {
    if (!g || !norm) return fg::set_error(FG_ERR_ARG, "fg_surrogate_get_norm: null argument");
    if (!g->hasNorm) return fg::set_error(FG_ERR_ARG, "fg_surrogate_get_norm: no training data statistics");
    std::memcpy(norm, &g->norm, sizeof(SurrogateNorm));
    return FG_OK;
}

int fg_surrogate_set_norm(fg_surrogate *g, const float *norm) {
    if (!g || !norm) return fg::set_error(FG_ERR_ARG, "fg_surrogate_set_norm: null argument");
    std::memcpy(&g->norm, norm, sizeof(SurrogateNorm));
    g->hasNorm = true;
    return FG_OK;
}

int fg_surrogate_predict(fg_surrogate *g, const float *X, int32_t n, float *Y, int32_t *inHull) {
    if (!g || !X || !Y) return fg::set_error(FG_ERR_ARG, "fg_surrogate_predict: null argument");
    if (n < 1 || n > (1 << 24)) return fg::set_error(FG_ERR_ARG, "fg_surrogate_predict: 1 <= n <= 2^24");
    SG_TRY(cudaSetDevice(g->device));
    SurrogateDev S{};
    int rc = surrogate_view(g, &S);
    if (rc != FG_OK) return rc;
    Buf dx, dy, dh, de;
    SG_TRY(dx.alloc((size_t)n * 3 * sizeof(float)));
    SG_TRY(dy.alloc((size_t)n * 4 * sizeof(float)));
    SG_TRY(dh.alloc((size_t)n * sizeof(int32_t)));
    SG_TRY(de.alloc(sizeof(int32_t)));
    SG_TRY(cudaMemset(de.p, 0, sizeof(int32_t)));
    SG_TRY(cudaMemcpy(dx.p, X, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice));
    const int tiles = (n + TC_M - 1) / TC_M;
    k_sg_tc<InPredict><<<std::min(tiles, 148 * 4), 128, TC_SMEM>>>(S, S.pack, InPredict{dx.as<float>(), n},
                                                                   dy.as<float4>(), dh.as<int32_t>(), de.as<int32_t>());
    SG_TRY(cudaGetLastError());
    int32_t terr = 0;
    SG_TRY(cudaMemcpy(&terr, de.p, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (terr) return fg::set_error(FG_ERR_CUDA, "fg_surrogate_predict: tensor-core completion wait timed out");
    SG_TRY(cudaMemcpy(Y, dy.p, (size_t)n * 4 * sizeof(float), cudaMemcpyDeviceToHost));
    if (inHull) SG_TRY(cudaMemcpy(inHull, dh.p, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    return FG_OK;
}

}  // extern "C"
