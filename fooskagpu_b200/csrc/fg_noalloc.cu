// Conservation integral over caller-owned device arrays that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc when they want the integral.  A host
// application that gives all device memory to its own pool allocator at start-up and permits no
// other allocation, or a monitor that samples the integral between the time steps of a
// latency-critical loop, where cudaMalloc / cudaFree may synchronise the device and stall the
// pipeline.  The solver's fg_cons_calc keeps its block partial sums in a buffer that
// fg_solver_create allocates; this entry point keeps them in a fixed array of the library's own
// device memory instead, so the caller only passes the state, the volumes and the output.
//
// The scratch array holds FG_NOALLOC_MAX_CELLS / 256 doubles (512 KiB).  Every device on which
// the library's module is loaded holds it until the process exits.  All calls on a device share
// it: two calls whose kernels overlap on the GPU (different streams without an ordering between
// them) race on it and give wrong sums; calls on one stream, or ordered by events, are safe.
// Nothing in it needs to start at zero: each call writes every entry it reads before reading
// it, and entries left over from an earlier, larger call are never read.
#include "../../include/fooskagpu.h"

#include <cuda_runtime.h>

#include <mutex>
#include <string>

namespace fg {
int set_error(int code, const std::string &msg);   // sets the message of fg_last_error
}

namespace {

constexpr int kThreads = 256;                               // cells per block partial sum
constexpr int kMaxBlocks = FG_NOALLOC_MAX_CELLS / kThreads; // entries of the scratch array
constexpr int kMaxDevices = 64;

// Block partial sums.  In host code this name is only a stand-in for the symbol: the device
// address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) double g_consScratch[kMaxBlocks];

// partial sums of (ivar == 0 ? 1 - U : U) * vol over blocks of kThreads cells, state in the
// reference layout U[cell * 10 + v]
__global__ void k_cons_blocks_aos(int n, int ivar, const double *__restrict__ U, const double *__restrict__ vol,
                                  double *blockSum) {
    __shared__ double sh[kThreads];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (c < n) {
        const double x = U[(size_t)c * 10 + ivar];
        v = ((ivar == 0) ? 1.0 - x : x) * vol[c];
    }
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) blockSum[blockIdx.x] = sh[0];
}

// fixed-shape tree over strided partial sums of the nb block sums: deterministic for a given n
__global__ void k_cons_final_static(const double *blockSum, int nb, double *out) {
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

std::mutex g_mu;
double *g_scratch[kMaxDevices] = {};

// device address of the scratch array on the current device (looked up on first use)
int scratch_on(int dev, double **p) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[dev]) {
        void *q = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&q, g_consScratch);
        if (e != cudaSuccess)
            return fg::set_error(FG_ERR_CUDA, std::string("fg_cons_integral_noalloc: cudaGetSymbolAddress: ") +
                                                  cudaGetErrorString(e));
        g_scratch[dev] = static_cast<double *>(q);
    }
    *p = g_scratch[dev];
    return FG_OK;
}

}  // namespace

extern "C" int fg_cons_integral_noalloc(const double *U, const double *vol, int32_t nCells, int32_t ivar,
                                        double *out, void *stream) {
    if (!U || !vol || !out) return fg::set_error(FG_ERR_ARG, "fg_cons_integral_noalloc: null argument");
    if (ivar < 0 || ivar > 9) return fg::set_error(FG_ERR_ARG, "fg_cons_integral_noalloc: ivar must be 0..9");
    if (nCells < 0) return fg::set_error(FG_ERR_ARG, "fg_cons_integral_noalloc: negative cell count");
    if (nCells > FG_NOALLOC_MAX_CELLS)
        return fg::set_error(FG_ERR_ARG, "fg_cons_integral_noalloc: " + std::to_string(nCells) +
                                             " cells exceed the static scratch limit of " +
                                             std::to_string(FG_NOALLOC_MAX_CELLS) + " cells");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return fg::set_error(FG_ERR_CUDA, std::string("fg_cons_integral_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return fg::set_error(FG_ERR_UNSUPPORTED, "fg_cons_integral_noalloc: device index above 63");
    double *scratch = nullptr;
    const int rc = scratch_on(dev, &scratch);
    if (rc != FG_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nb = (nCells + kThreads - 1) / kThreads;
    if (nb > 0) k_cons_blocks_aos<<<nb, kThreads, 0, s>>>(nCells, ivar, U, vol, scratch);
    k_cons_final_static<<<1, 1024, 0, s>>>(scratch, nb, out);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return fg::set_error(FG_ERR_CUDA, std::string("fg_cons_integral_noalloc: launch: ") + cudaGetErrorString(e));
    return FG_OK;
}
