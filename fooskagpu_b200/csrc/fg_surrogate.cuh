// Learned equilibrium surrogate: a 3 -> 64 -> 64 -> 64 -> 4 GELU MLP evaluated on the BF16
// tensor cores (tcgen05, fg_sg_tc.cuh) with FP32 accumulation.
//
// It maps the state of a cell that needs the chemical (Gibbs) equilibrium solve
// (DP/chemRlx.cu) — mixture density rho, mixture internal energy per unit mass e, vapour mass
// fraction before the solve Y — to the equilibrium (p, T, alpha, Y_eq).  The relaxation kernel
// uses the prediction as the starting point of a short full-step Newton polish on the
// reference's residuals; cells outside the training hull or whose polished residual stays
// above tolerance take the reference Newton from its usual starting point.
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

// normalisation and training hull (all FP32, in this order in SurrogateDev::norm)
struct SurrogateNorm {
    float xMean[3], xStd[3], yMean[4], yStd[4];
    float boxLo[3], boxHi[3];   // per-feature range of the normalised training inputs
    float covInv[9];            // inverse covariance of the normalised training inputs
    float d2Max;                // largest squared Mahalanobis distance seen in training
};

struct SurrogateDev {
    const unsigned char *pack;   // BF16 weights in the tensor-core operand layout (TC_WBYTES)
    const float *params;         // SG_NPARAM FP32 parameters (biases read from here)
    SurrogateNorm norm;
    double relTol;          // accepted when every relative residual <= relTol after the polish
    int polishIters;        // full Newton steps allowed from the prediction
    int enabled;
};

// GELU in its tanh form (Hendrycks & Gimpel, "Gaussian Error Linear Units", 2016):
//   gelu(x) = x / 2 (1 + tanh(sqrt(2 / pi) (x + 0.044715 x^3)))
// the network's activation in training (FP32, tanhf) and in the tensor-core inference, where the
// hardware tanh.approx.f32 (relative error about 2^-11, below the BF16 rounding of the
// activations that follows) keeps the epilogue short.
constexpr float SG_GELU_C = 0.79788456080286536f, SG_GELU_A = 0.044715f;
__device__ __forceinline__ float sg_gelu(float x) {
    float th;
    const float u = SG_GELU_C * fmaf(SG_GELU_A * x, x * x, x);
    asm("tanh.approx.f32 %0, %1;" : "=f"(th) : "f"(u));
    return 0.5f * x * (1.0f + th);
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
