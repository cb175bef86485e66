// lmb_noalloc.cu -- species counts without any device allocation.
//
// Some callers cannot allocate device memory at the moment they want a
// count: a host application that hands all device memory to its own pool
// allocator and forbids other allocations, a process that counts from inside
// a callback or hook where cudaMalloc would synchronize the device or fail
// under a memory cap, or a serving loop that must not grow its footprint
// between requests.  lmb_lattice_species_counts allocates a device buffer
// for the per-species totals on first use; this variant keeps those totals in
// a fixed, file-scope device array instead and needs nothing from the caller
// but the lattice in device memory and a host array for the result.
//
// The array holds LMB_NOALLOC_MAX_SPECIES + 1 64-bit counters (32 KiB).  It
// exists once per device for the whole process, from the first use of the
// library on that device until exit.  The first call on a device looks up the
// array's device address (cudaGetSymbolAddress), so that call should come
// before any stream capture on that device.  The address is kept until exit; a
// cudaDeviceReset reloads the module, possibly elsewhere, so the entry point is
// not usable on a device after it has been reset (as no lmb handle on that
// device is).  Every call zeroes it on the stream
// before counting, so a call never sees the previous call's totals; two calls
// whose work overlaps on the GPU (different streams, no ordering between
// them) write the same array and race.
#include <cuda_runtime.h>

#include <mutex>

#include "lmb.h"
#include "lmb_internal.h"

namespace {

// Device scratch of the no-allocation entry point.  In host code this name
// stands for the symbol, not for a device address: the address comes from
// cudaGetSymbolAddress, once per device, below.
static __device__ __align__(256) unsigned long long g_noalloc_counts[LMB_NOALLOC_MAX_SPECIES + 1];

constexpr int MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
unsigned long long *g_noalloc_ptr[MAX_DEVICES] = {nullptr};

// The device address of the scratch array on the current device, looked up
// on the first call for that device.
int noalloc_scratch(int device, unsigned long long **out)
{
    if (device < 0 || device >= MAX_DEVICES) return LMB_E_ARG;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_counts) != cudaSuccess || !p) return LMB_E_CUDA;
        g_noalloc_ptr[device] = (unsigned long long *)p;
    }
    *out = g_noalloc_ptr[device];
    return LMB_OK;
}

}  // namespace

extern "C" int lmb_species_counts_noalloc(const uint32_t *particles, uint32_t X, uint32_t Y, uint32_t Z,
                                          uint32_t particles_per_site, uint32_t bytes_per_particle,
                                          uint32_t number_species, uint64_t *counts, void *cuda_stream)
{
    if (!particles || !counts || X == 0 || Y == 0 || Z == 0) return LMB_E_ARG;
    if (number_species > LMB_NOALLOC_MAX_SPECIES) return LMB_E_UNSUPPORTED;
    if (!lmb::slots_supported((int)bytes_per_particle, (int)particles_per_site)) return LMB_E_UNSUPPORTED;
    const unsigned long long N = (unsigned long long)X * Y * Z;
    if (N > 0xFFFFFFFFull) return LMB_E_UNSUPPORTED;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return LMB_E_CUDA;
    unsigned long long *scratch = nullptr;
    int rc = noalloc_scratch(device, &scratch);
    if (rc != LMB_OK) return rc;
    cudaStream_t stream = (cudaStream_t)cuda_stream;
    lmb::Geometry g;
    g.X = X;
    g.Y = Y;
    g.Z = Z;
    g.XY = X * Y;
    g.N = (uint32_t)N;
    const size_t bytes = sizeof(unsigned long long) * (number_species + 1);
    if (cudaMemsetAsync(scratch, 0, bytes, stream) != cudaSuccess) return LMB_E_CUDA;
    if (lmb::launch_counts((int)bytes_per_particle, (int)particles_per_site, particles, g, number_species, scratch,
                           stream) != cudaSuccess)
        return LMB_E_CUDA;
    if (cudaMemcpyAsync(counts, scratch, bytes, cudaMemcpyDeviceToHost, stream) != cudaSuccess) return LMB_E_CUDA;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return LMB_E_CUDA;
    counts[0] = 0;
    return LMB_OK;
}
