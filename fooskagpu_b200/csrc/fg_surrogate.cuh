// Learned equilibrium surrogate: a 3 -> 64 -> 64 -> 64 -> 4 GELU MLP evaluated by one warp for
// 32 cells at a time on the BF16 tensor cores (mma.sync m16n8k16, FP32 accumulation), with the
// activations kept in registers between layers.
//
// It maps the state of a cell that needs the chemical (Gibbs) equilibrium solve
// (DP/chemRlx.cu) — mixture density rho, mixture internal energy per unit mass e, vapour mass
// fraction before the solve Y — to the equilibrium (p, T, alpha, Y_eq).  The relaxation kernel
// uses the prediction as the starting point of a short full-step Newton polish on the
// reference's residuals; cells outside the training hull or whose polished residual stays
// above tolerance take the reference Newton from its usual starting point.
//
// Fragment layouts (PTX ISA, mma.m16n8k16 with .bf16 A/B and .f32 C/D), lane = 4 g + t:
//   A (16x16, row): a0 = A[g][2t..2t+1], a1 = A[g+8][2t..2t+1], a2 = A[g][2t+8..], a3 = A[g+8][2t+8..]
//   B (16x8, col) : b0 = B[2t..2t+1][g],  b1 = B[2t+8..2t+9][g]
//   C (16x8)      : c0,c1 = C[g][2t..2t+1], c2,c3 = C[g+8][2t..2t+1]
// so the C fragments of n-tiles 2kk and 2kk+1 of one layer are exactly the A fragment of k-tile
// kk of the next layer.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace fg {

constexpr int SG_IN = 3, SG_H = 64, SG_OUT = 4;
// flat FP32 parameter vector: W1[3][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64][4] b4[4]
constexpr int SG_OFF_W1 = 0, SG_OFF_B1 = SG_OFF_W1 + SG_IN * SG_H, SG_OFF_W2 = SG_OFF_B1 + SG_H,
              SG_OFF_B2 = SG_OFF_W2 + SG_H * SG_H, SG_OFF_W3 = SG_OFF_B2 + SG_H,
              SG_OFF_B3 = SG_OFF_W3 + SG_H * SG_H, SG_OFF_W4 = SG_OFF_B3 + SG_H,
              SG_OFF_B4 = SG_OFF_W4 + SG_H * SG_OUT, SG_NPARAM = SG_OFF_B4 + SG_OUT;
// packed BF16 B fragments (uint32 = 2 x bf16) per layer: [k-tile][n-tile][lane][2]
constexpr int SG_PK_L1 = 0;                          // 1 k-tile x 8 n-tiles
constexpr int SG_PK_L2 = SG_PK_L1 + 1 * 8 * 64;      // 4 x 8
constexpr int SG_PK_L3 = SG_PK_L2 + 4 * 8 * 64;      // 4 x 8
constexpr int SG_PK_L4 = SG_PK_L3 + 4 * 8 * 64;      // 4 x 1
constexpr int SG_PK_TOTAL = SG_PK_L4 + 4 * 1 * 64;

// normalisation and training hull (all FP32, in this order in SurrogateDev::norm)
struct SurrogateNorm {
    float xMean[3], xStd[3], yMean[4], yStd[4];
    float boxLo[3], boxHi[3];   // per-feature range of the normalised training inputs
    float covInv[9];            // inverse covariance of the normalised training inputs
    float d2Max;                // largest squared Mahalanobis distance seen in training
};

struct SurrogateDev {
    const uint32_t *pack;   // SG_PK_TOTAL packed B fragments
    const float *params;    // SG_NPARAM FP32 parameters (biases read from here)
    SurrogateNorm norm;
    double relTol;          // accepted when every relative residual <= relTol after the polish
    int polishIters;        // full Newton steps allowed from the prediction
    int enabled;
};

__device__ __forceinline__ uint32_t sg_pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ void sg_mma(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                       uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float sg_gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

// One 16-row tile through the network.  x0..x2 / y0..y2: normalised inputs of rows g and g+8
// of the tile as this lane's A fragment needs them (only lanes with t = 0, 1 use them).
// Returns this lane's C fragment of the output layer (columns 2t, 2t+1 of rows g and g+8;
// columns >= 4 are padding).
__device__ __forceinline__ void sg_tile(const SurrogateDev &S, int lane, float rg0, float rg1, float rg2, float rh0,
                                        float rh1, float rh2, float (&out)[4]) {
    const int t = lane & 3;
    const float *P = S.params;
    // layer 1: K = 3 padded to 16 (a2 = a3 = 0: columns 8..15)
    uint32_t a0 = 0, a1 = 0;
    if (t == 0) {
        a0 = sg_pack_bf16(rg0, rg1);
        a1 = sg_pack_bf16(rh0, rh1);
    } else if (t == 1) {
        a0 = sg_pack_bf16(rg2, 0.f);
        a1 = sg_pack_bf16(rh2, 0.f);
    }
    float h[8][4];
    {
        const uint2 *B = reinterpret_cast<const uint2 *>(S.pack + SG_PK_L1);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const float b0 = __ldg(P + SG_OFF_B1 + 8 * j + 2 * t), b1 = __ldg(P + SG_OFF_B1 + 8 * j + 2 * t + 1);
            h[j][0] = b0; h[j][1] = b1; h[j][2] = b0; h[j][3] = b1;
            const uint2 w = __ldg(B + j * 32 + lane);
            sg_mma(h[j], a0, a1, 0u, 0u, w.x, w.y);
#pragma unroll
            for (int q = 0; q < 4; q++) h[j][q] = sg_gelu(h[j][q]);
        }
    }
    // layers 2 and 3: 64 -> 64
#pragma unroll
    for (int L = 0; L < 2; L++) {
        const uint2 *B = reinterpret_cast<const uint2 *>(S.pack + (L == 0 ? SG_PK_L2 : SG_PK_L3));
        const float *bias = P + (L == 0 ? SG_OFF_B2 : SG_OFF_B3);
        uint32_t A[4][4];
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            A[kk][0] = sg_pack_bf16(h[2 * kk][0], h[2 * kk][1]);
            A[kk][1] = sg_pack_bf16(h[2 * kk][2], h[2 * kk][3]);
            A[kk][2] = sg_pack_bf16(h[2 * kk + 1][0], h[2 * kk + 1][1]);
            A[kk][3] = sg_pack_bf16(h[2 * kk + 1][2], h[2 * kk + 1][3]);
        }
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const float b0 = __ldg(bias + 8 * j + 2 * t), b1 = __ldg(bias + 8 * j + 2 * t + 1);
            float acc[4] = {b0, b1, b0, b1};
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                const uint2 w = __ldg(B + (kk * 8 + j) * 32 + lane);
                sg_mma(acc, A[kk][0], A[kk][1], A[kk][2], A[kk][3], w.x, w.y);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) h[j][q] = sg_gelu(acc[q]);
        }
    }
    // layer 4: 64 -> 4 (N padded to 8), linear
    {
        const uint2 *B = reinterpret_cast<const uint2 *>(S.pack + SG_PK_L4);
        const float b0 = (2 * t < SG_OUT) ? __ldg(P + SG_OFF_B4 + 2 * t) : 0.f;
        const float b1 = (2 * t + 1 < SG_OUT) ? __ldg(P + SG_OFF_B4 + 2 * t + 1) : 0.f;
        out[0] = b0; out[1] = b1; out[2] = b0; out[3] = b1;
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            const uint32_t x0 = sg_pack_bf16(h[2 * kk][0], h[2 * kk][1]);
            const uint32_t x1 = sg_pack_bf16(h[2 * kk][2], h[2 * kk][3]);
            const uint32_t x2 = sg_pack_bf16(h[2 * kk + 1][0], h[2 * kk + 1][1]);
            const uint32_t x3 = sg_pack_bf16(h[2 * kk + 1][2], h[2 * kk + 1][3]);
            const uint2 w = __ldg(B + kk * 32 + lane);
            sg_mma(out, x0, x1, x2, x3, w.x, w.y);
        }
    }
}

// Whole warp (all 32 lanes must call it, converged): lane l supplies the normalised inputs of
// its own row (ignored when !valid) and receives its 4 normalised outputs.
__device__ __forceinline__ void sg_warp_forward(const SurrogateDev &S, const float (&xin)[3], float (&yout)[4]) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2;
    float res[2][4];
#pragma unroll
    for (int T = 0; T < 2; T++) {
        // inputs of rows g and g+8 of tile T (cells of lanes 16 T + g and 16 T + g + 8)
        const int sg = 16 * T + g, sh = sg + 8;
        const float g0 = __shfl_sync(0xffffffffu, xin[0], sg), g1 = __shfl_sync(0xffffffffu, xin[1], sg),
                    g2 = __shfl_sync(0xffffffffu, xin[2], sg);
        const float h0 = __shfl_sync(0xffffffffu, xin[0], sh), h1 = __shfl_sync(0xffffffffu, xin[1], sh),
                    h2 = __shfl_sync(0xffffffffu, xin[2], sh);
        sg_tile(S, lane, g0, g1, g2, h0, h1, h2, res[T]);
    }
    // row r of tile T (lane 16 T + r): columns 0,1 sit in lane 4 (r mod 8) + 0, columns 2,3 in
    // lane 4 (r mod 8) + 1, as c0,c1 for r < 8 and c2,c3 for r >= 8
    const int T = lane >> 4, r = lane & 15, gr = r & 7;
    const bool hi = r >= 8;
#pragma unroll
    for (int TT = 0; TT < 2; TT++) {
        float v[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int src = 4 * gr + (q >> 1);
            const float lo = __shfl_sync(0xffffffffu, res[TT][q & 1], src);
            const float up = __shfl_sync(0xffffffffu, res[TT][2 + (q & 1)], src);
            v[q] = hi ? up : lo;
        }
        if (TT == T) {
#pragma unroll
            for (int q = 0; q < 4; q++) yout[q] = v[q];
        }
    }
}

// Inside the training hull: per-feature box and Mahalanobis bound on the normalised inputs.
__device__ __forceinline__ bool sg_in_hull(const SurrogateNorm &N, const float (&z)[3]) {
#pragma unroll
    for (int i = 0; i < 3; i++)
        if (!(z[i] >= N.boxLo[i] && z[i] <= N.boxHi[i])) return false;
    float d2 = 0.f;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) d2 += z[i] * N.covInv[3 * i + j] * z[j];
    return d2 <= N.d2Max;
}

}  // namespace fg
