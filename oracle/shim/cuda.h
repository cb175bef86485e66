/*
 * Host stand-in for <cuda.h> used ONLY by oracle/ref_host_harness.cpp, which
 * compiles the reference's device functions with g++ so that they run on the
 * CPU as a checker.  The CUDA execution-space qualifiers become nothing, the
 * built-in thread coordinates become harness-owned globals, and the few
 * device intrinsics the reference calls get sequential host definitions.
 */
#ifndef LMB_HOST_SHIM_CUDA_H
#define LMB_HOST_SHIM_CUDA_H

#include <stdint.h>
#include <stdlib.h>

#define __device__
#define __global__
#define __host__
#define __shared__ static
#define __constant__
#define __forceinline__ inline
#define __launch_bounds__(a, b)

struct lmb_shim_dim3 {
    unsigned int x, y, z;
};

/* Thread and block coordinates are set by the harness before each call. */
extern lmb_shim_dim3 threadIdx, blockIdx, blockDim, gridDim;

/* The harness drives a block's threads phase by phase, so the barrier itself
 * has nothing left to do. */
static inline void __syncthreads() {}

/* The harness is single-threaded per lattice, so a plain read-modify-write
 * is atomic. */
static inline unsigned int atomicAdd(unsigned int *p, unsigned int v)
{
    unsigned int old = *p;
    *p = old + v;
    return old;
}

template <typename T>
static inline T __ldg(const T *p) { return *p; }

#endif
