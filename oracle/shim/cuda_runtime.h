/* Host stand-in for <cuda_runtime.h>: see shim/cuda.h. */
#ifndef LMB_HOST_SHIM_CUDA_RUNTIME_H
#define LMB_HOST_SHIM_CUDA_RUNTIME_H
#include "cuda.h"
#endif
