// Test of the grid barrier's bounded wait (lmb::grid_barrier,
// lattice_microbes_b200/csrc/lmb_device.cuh), the one spin-wait of the
// library's kernels.  Test infrastructure only: built into
// tests/cpp/_build/libgrid_selftest.so and called by
// tests/test_gpu_failure.py.
//
// lmb_selftest_grid_barrier(blocks, target, status, elapsed_ms): one
// cooperative launch of `blocks` blocks that each pass one grid barrier
// expecting `target` arrivals.  With target <= blocks every wait ends at once;
// with target > blocks no block can ever be released (nothing else arrives),
// so every wait must give up by itself.  A block whose wait gave up sets the
// status to LMB_E_TIMEOUT, as the grid-resident kernel does.  Returns the
// CUDA error of the launch and of the synchronisation (0 when the context is
// still usable); *status is the device status, *elapsed_ms the kernel's
// duration by CUDA events.
#include <cuda_runtime.h>
#include <stdint.h>

#include "lmb.h"
#include "lmb_device.cuh"

namespace {

struct BarrierState {
    unsigned long long bar;
    int32_t status;
};

__global__ void barrier_selftest_kernel(BarrierState *st, unsigned long long target)
{
    if (!lmb::grid_barrier(&st->bar, target) && threadIdx.x == 0)
        atomicCAS(&st->status, (int32_t)LMB_OK, (int32_t)LMB_E_TIMEOUT);
}

}  // namespace

extern "C" int lmb_selftest_grid_barrier(uint32_t blocks, uint32_t target, int32_t *status, float *elapsed_ms)
{
    BarrierState *st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&st, sizeof(BarrierState));
    if (e == cudaSuccess) e = cudaMemset(st, 0, sizeof(BarrierState));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(blocks);
        cfg.blockDim = dim3(128);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaEventRecord(e0, 0);
        e = cudaLaunchKernelEx(&cfg, barrier_selftest_kernel, st, (unsigned long long)target);
        cudaEventRecord(e1, 0);
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) {
        BarrierState h = {};
        e = cudaMemcpy(&h, st, sizeof(h), cudaMemcpyDeviceToHost);
        *status = h.status;
        cudaEventElapsedTime(elapsed_ms, e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaFree(st);
    return (int)e;
}
