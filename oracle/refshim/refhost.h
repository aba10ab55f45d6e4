/* Host emulation of the few CUDA built-ins the reference's kernel-only files use, so that
 * their device functions can be compiled by g++ and run serially as known-answer checks.
 * TEST INFRASTRUCTURE ONLY.  A "launch" is a plain call with one thread in one block, which
 * makes every grid-stride loop visit its items in order. */
#ifndef FG_REFSHIM_REFHOST_H
#define FG_REFSHIM_REFHOST_H
#include <cuda_runtime.h>
#include <cmath>
#ifndef __noinline__
#define __noinline__ __attribute__((noinline))
#endif
extern uint3 threadIdx, blockIdx;
extern dim3 blockDim, gridDim;
static inline double atomicAdd(double *a, double v) { double o = *a; *a = o + v; return o; }
static inline int atomicAdd(int *a, int v) { int o = *a; *a = o + v; return o; }
using std::isnan;
#endif
