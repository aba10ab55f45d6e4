// Surrogate network on the 5th-generation tensor cores (tcgen05, sm_100a): one CTA of 128
// threads evaluates tiles of 128 samples; every layer is a 128 x N x K BF16 GEMM with FP32
// accumulators in tensor memory (TMEM), issued by one thread; the activations go back to shared
// memory as the next layer's A operand after bias + GELU in registers.
//
// Shared-memory operands use the K-major, no-swizzle canonical layout of the UMMA descriptors:
// for a 16-wide K slab, element (row, k) of an R-row operand sits at byte
//   (row / 8) * 256 + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2
// (8-row x 16-byte core matrices; leading-dimension offset 128 B between the two K halves,
// stride offset 256 B between 8-row groups), slabs one after the other.
//
// Every wait on the MMA-completion mbarrier is bounded; on time-out the tile is marked failed,
// the CTA still waits (bounded) for its MMAs, frees its TMEM and leaves.
#pragma once
#include "fg_surrogate.cuh"

namespace fg {

constexpr int TC_M = 128;                      // samples per tile (TMEM lanes)
constexpr int TC_W1 = 0;                       // W1: N 64 x K 16 (3 used)          2 KB
constexpr int TC_W2 = TC_W1 + 64 * 16 * 2;     // W2: N 64 x K 64                    8 KB
constexpr int TC_W3 = TC_W2 + 64 * 64 * 2;     // W3: N 64 x K 64                    8 KB
constexpr int TC_W4 = TC_W3 + 64 * 64 * 2;     // W4: N 16 x K 64 (4 used)           2 KB
constexpr int TC_WBYTES = TC_W4 + 16 * 64 * 2; // packed weights (bytes)
constexpr int TC_A = TC_WBYTES;                // activations: 128 x K 64            16 KB
constexpr int TC_BIAS = TC_A + TC_M * 64 * 2;  // hidden-layer biases, FP32 3 x 64    768 B
constexpr int TC_BAR = TC_BIAS + 3 * 64 * 4;   // mbarrier (8 B) + TMEM address (4 B)
constexpr int TC_SMEM = TC_BAR + 16;
constexpr uint32_t TC_TMEM_COLS = 64;

__device__ __forceinline__ uint32_t tc_smem_off(int row, int k, int rows) {
    // byte offset of (row, k) in a K-major canonical operand of `rows` rows, 16-wide K slabs
    return (uint32_t)((k >> 4) * rows * 32 + (row >> 3) * 256 + ((k >> 3) & 1) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// UMMA shared-memory descriptor: no swizzle, LBO 128 B (K halves), SBO 256 B (8-row groups),
// version 1 (sm100)
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
           (1ull << 46);
}

// instruction descriptor, kind::f16: D f32, A and B bf16, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ uint32_t tc_smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// bounded wait for the mbarrier phase of `parity`; false on time-out
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
    for (int it = 0; it < (1 << 22); it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// row `row`, columns k0 .. k0 + 7 (k0 a multiple of 8) of the A operand: 8 consecutive BF16 of
// one core-matrix row, one 16-byte store
__device__ __forceinline__ void tc_store8_bf16(unsigned char *smA, int row, int k0, const float *x) {
    __nv_bfloat162 p[4];
#pragma unroll
    for (int q = 0; q < 4; q++) p[q] = __floats2bfloat162_rn(x[2 * q], x[2 * q + 1]);   // x[2q] in the low half
    *reinterpret_cast<uint4 *>(smA + tc_smem_off(row, k0, TC_M)) = *reinterpret_cast<const uint4 *>(p);
}

// One layer on the tensor cores: D[128 x n] = A[128 x 16 kSlabs] * W^T, into TMEM; returns false
// if the completion wait timed out.  Called by all 128 threads.
__device__ __forceinline__ bool tc_layer(unsigned char *sm, uint32_t tmem, int wOff, int n, int kSlabs,
                                         uint32_t &phase) {
    const uint32_t bar = tc_smem_addr(sm + TC_BAR);
    tc_proxy_fence();          // generic-proxy writes of A visible to the tensor cores
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc_fence_after();
        const uint32_t aBase = tc_smem_addr(sm + TC_A), wBase = tc_smem_addr(sm + wOff);
        const uint32_t idesc = tc_idesc(n);
        for (int kk = 0; kk < kSlabs; kk++)
            tc_mma(tmem, tc_desc(aBase + kk * TC_M * 32), tc_desc(wBase + kk * n * 32), idesc, kk > 0 ? 1u : 0u);
        tc_commit(bar);
    }
    const bool ok = tc_wait(bar, phase);
    phase ^= 1u;
    tc_fence_after();
    return ok;
}

// byte offset of (row, k) as above, for host-side packing
inline uint32_t tc_smem_off_host(int row, int k, int rows) {
    return (uint32_t)((k >> 4) * rows * 32 + (row >> 3) * 256 + ((k >> 3) & 1) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Evaluate the network for the samples of `in` (tiles of 128, persistent CTAs): out[i] = raw
// outputs (p, T, alpha, Y_eq), hull[i] = inside the training hull.  `wpack` holds the four
// layers' weights in the canonical layout (TC_WBYTES bytes); *err = 1 if an MMA completion wait
// timed out.  128 threads per CTA, TC_SMEM bytes of dynamic shared memory.
template <class In>
__global__ void __launch_bounds__(128) k_sg_tc(const SurrogateDev S, const unsigned char *__restrict__ wpack, In in,
                                               float4 *__restrict__ out, int32_t *__restrict__ hull, int32_t *err) {
    extern __shared__ __align__(128) unsigned char sm[];
    const int t = threadIdx.x;
    for (int q = t; q < TC_WBYTES / 16; q += blockDim.x)
        reinterpret_cast<uint4 *>(sm)[q] = reinterpret_cast<const uint4 *>(wpack)[q];
    {
        // the three hidden layers' biases, read by every thread of a tile (broadcast)
        float *b = reinterpret_cast<float *>(sm + TC_BIAS);
        for (int q = t; q < 3 * 64; q += blockDim.x)
            b[q] = __ldg(S.params + (q < 64 ? SG_OFF_B1 + q : (q < 128 ? SG_OFF_B2 + q - 64 : SG_OFF_B3 + q - 128)));
    }
    const uint32_t bar = tc_smem_addr(sm + TC_BAR);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + TC_BAR + 8);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");   // visible to the async proxy
    }
    if (t < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(tslot)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t tw = tmem + ((uint32_t)(t & ~31) << 16);   // this warp's 32 TMEM lanes
    const float *P = S.params;
    const int n = in.count();
    const int tiles = (n + TC_M - 1) / TC_M;
    uint32_t phase = 0;
    bool ok = true;
    unsigned char *A = sm + TC_A;
    for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const int i = tile * TC_M + t;
        float z[3] = {0.f, 0.f, 0.f};
        bool h = false;
        if (i < n) {
            in.features(i, S.norm, z);
            h = sg_in_hull(S.norm, z);
        }
        {
            const float x[8] = {z[0], z[1], z[2], 0.f, 0.f, 0.f, 0.f, 0.f}, zero[8] = {};
            tc_store8_bf16(A, t, 0, x);
            tc_store8_bf16(A, t, 8, zero);
        }
        float v[64];
        // hidden layers: 3 -> 64 -> 64 -> 64, GELU
#pragma unroll 1
        for (int L = 0; L < 3 && ok; L++) {
            const int wOff = L == 0 ? TC_W1 : (L == 1 ? TC_W2 : TC_W3);
            const float4 *bias = reinterpret_cast<const float4 *>(sm + TC_BIAS) + L * 16;
            ok = __syncthreads_and(tc_layer(sm, tmem, wOff, 64, L == 0 ? 1 : 4, phase));
            if (!ok) break;
#pragma unroll
            for (int c = 0; c < 4; c++) tc_ld16(tw + 16 * c, v + 16 * c);
#pragma unroll
            for (int j8 = 0; j8 < 8; j8++) {
                const float4 ba = bias[2 * j8], bb = bias[2 * j8 + 1];
                const float b8[8] = {ba.x, ba.y, ba.z, ba.w, bb.x, bb.y, bb.z, bb.w};
                float x[8];
#pragma unroll
                for (int q = 0; q < 8; q++) x[q] = sg_gelu(v[8 * j8 + q] + b8[q]);
                tc_store8_bf16(A, t, 8 * j8, x);
            }
        }
        if (!ok) break;
        // output layer: 64 -> 4 (N padded to 16), linear
        ok = __syncthreads_and(tc_layer(sm, tmem, TC_W4, 16, 4, phase));
        if (!ok) break;
        tc_ld16(tw, v);
        if (i < n) {
            float o[4];
#pragma unroll
            for (int q = 0; q < 4; q++) o[q] = S.norm.yMean[q] + S.norm.yStd[q] * (v[q] + __ldg(P + SG_OFF_B4 + q));
            out[i] = make_float4(o[0], o[1], o[2], o[3]);
            if (hull) hull[i] = h ? 1 : 0;
        }
    }
    if (!ok) {
        // a completion wait timed out: wait (bounded) for the phase still open (the parity before
        // the flip in tc_layer) before freeing TMEM
        tc_wait(bar, phase ^ 1u);
        if (t == 0) atomicExch(err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (t < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
}

}  // namespace fg
