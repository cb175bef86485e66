// lmb_device.cuh -- device building blocks of the MPD-RDME timestep.
//
// Arithmetic that decides a particle's fate is written so that the compiler
// cannot fuse a multiply into a following add (__fmul_rn / __fsub_rn): every
// product and sum is rounded on its own, as the restatement of the
// reference's rules requires.
#pragma once

#include <stdint.h>

#include "lmb_internal.h"

namespace lmb {

// Programmatic dependent launch between the kernels of a timestep.  Every
// kernel of the chain starts with chain_enter(): it waits until the kernel
// before it in the stream has finished and its writes are visible (at once
// when that kernel was not launched as part of a chain), then lets the next
// kernel of the chain be launched, so that its blocks are scheduled while
// this kernel's last blocks run instead of after them.  Nothing is read or
// written before the wait.
__device__ __forceinline__ void chain_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Grid barrier of a cooperative launch (all blocks resident at once).  Each
// block adds one arrival to `bar` (zeroed before the launch) and waits, in
// thread 0, until the count reaches `target` = (barriers passed + 1) x
// blocks.  The wait is bounded: it gives up after GRID_WAIT_NS of
// %globaltimer time (or GRID_SPIN_LIMIT polls, whichever comes first) and
// returns false, so a block that never arrives ends the run with an error
// status instead of holding the GPU.
constexpr unsigned long long GRID_WAIT_NS = 1000000000ull;  // 1 s
constexpr uint32_t GRID_SPIN_LIMIT = 1u << 24;

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool grid_barrier(unsigned long long *bar, unsigned long long target)
{
    __shared__ uint32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1ull);
        const unsigned long long t0 = globaltimer_ns();
        uint32_t ok = 0;
        for (uint32_t it = 0; it < GRID_SPIN_LIMIT; it++) {
            unsigned long long v;
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(bar) : "memory");
            if (v >= target) {
                ok = 1;
                break;
            }
            if ((it & 63u) == 63u && globaltimer_ns() - t0 > GRID_WAIT_NS) break;
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Model-table read.  The tables live in global memory, or in shared memory
// when a kernel stages them there, so the load is a generic one.
template <typename T>
__device__ __forceinline__ T tload(const T *p)
{
    return *p;
}

// Counter hash of (key ^ timestep hash), upper 32 bits
// (rdme/dev/xor_random_dev.cu:46-53).
__device__ __forceinline__ uint32_t mix_hash(unsigned long long v, unsigned long long th)
{
    v ^= th;
    v = v * 3935559000370003845ULL + 2691343689449507681ULL;
    v ^= v >> 21;
    v ^= v << 37;
    v ^= v >> 4;
    v *= 2685821657736338717ULL;
    return (uint32_t)(v >> 32);
}

// [0,1) float: (float)r rounded to nearest, times 2^-32 (xor_random_dev.cu:44,66-70).
__device__ __forceinline__ float hash_float(unsigned long long key, unsigned long long th)
{
    return __fmul_rn(__uint2float_rn(mix_hash(key, th)), 2.32830643654e-10f);
}

// Per-launch seed mixing (MpdRdmeSolver.cu:987-994), evaluated on the device
// from the run state so that captured launches replay with the right step.
__host__ __device__ __forceinline__ unsigned long long timestep_hash(uint32_t seed, uint32_t step,
                                                                     uint32_t substep)
{
    unsigned long long h = ((((unsigned long long)seed << 30) + step) << 2) + substep;
    h = h * 3202034522624059733ULL + 4354685564936845319ULL;
    h ^= h >> 20;
    h ^= h << 41;
    h ^= h >> 5;
    h *= 7664345821815920749ULL;
    return h;
}

// Sets rs->step and the four sub-step hashes that go with it.
__device__ __forceinline__ void set_step(RunState *rs, uint32_t seed, uint32_t step)
{
    rs->step = step;
#pragma unroll
    for (uint32_t k = 0; k < 4; k++) rs->th[k] = timestep_hash(seed, step, k);
}

// Hash-key slot bits (byte_diffusion_1d_dev.cu:51-60).
template <int S>
struct CountBits {
    static constexpr int value = S <= 4 ? 2 : (S <= 8 ? 3 : 4);
};

// A site's S slots held in W registers (4 uint8 slots per word for byte
// lattices, one uint32 slot per word for int lattices).
template <int BPS, int S>
struct SiteWords {
    static constexpr int W = (BPS == 1) ? S / 4 : S;
    uint32_t w[W];

    __device__ __forceinline__ void load(const uint32_t *__restrict__ lat, uint32_t N, uint32_t i)
    {
#pragma unroll
        for (int k = 0; k < W; k++) w[k] = __ldg(lat + (size_t)k * N + i);
    }
    __device__ __forceinline__ void store(uint32_t *lat, uint32_t N, uint32_t i) const
    {
#pragma unroll
        for (int k = 0; k < W; k++) lat[(size_t)k * N + i] = w[k];
    }
    // Loads a packed site (occupied slots first, as every sweep writes them)
    // touching only the word planes that hold particles: plane k + 1 is read
    // only when plane k is full (every slot of a byte word, or the one slot
    // of an int word, occupied); the other planes are zero.
    __device__ __forceinline__ void load_packed(const uint32_t *lat, uint32_t N, uint32_t i)
    {
        clear();
        bool more = true;
#pragma unroll
        for (int k = 0; k < W; k++) {
            if (more) {
                w[k] = lat[(size_t)k * N + i];
                more = BPS == 1 ? (w[k] >> 24) != 0u : w[k] != 0u;
            }
        }
    }
    // Loads words 0 .. nw - 1 through the read-only path and clears the
    // rest: a site whose words from nw on are known to be zero (a plane
    // bound), in a buffer nothing writes during the kernel.
    __device__ __forceinline__ void load_planes(const uint32_t *__restrict__ lat, uint32_t N, uint32_t i,
                                                uint32_t nw)
    {
#pragma unroll
        for (int k = 0; k < W; k++) w[k] = (uint32_t)k < nw ? __ldg(lat + (size_t)k * N + i) : 0u;
    }
    // Stores words 0 .. nw - 1.
    __device__ __forceinline__ void store_first(uint32_t *lat, uint32_t N, uint32_t i, uint32_t nw) const
    {
#pragma unroll
        for (int k = 0; k < W; k++)
            if ((uint32_t)k < nw) lat[(size_t)k * N + i] = w[k];
    }
    // Loads words 0 .. nw - 1 (independent loads) and clears the rest: a
    // packed site whose particle count is known.
    __device__ __forceinline__ void load_first(const uint32_t *lat, uint32_t N, uint32_t i, uint32_t nw)
    {
#pragma unroll
        for (int k = 0; k < W; k++) w[k] = (uint32_t)k < nw ? lat[(size_t)k * N + i] : 0u;
    }
    __device__ __forceinline__ uint32_t slot(int k) const
    {
        if (BPS == 1) return (w[k >> 2] >> (8 * (k & 3))) & 0xFFu;
        return w[k];
    }
    __device__ __forceinline__ bool empty() const
    {
        uint32_t o = 0;
#pragma unroll
        for (int k = 0; k < W; k++) o |= w[k];
        return o == 0;
    }
    __device__ __forceinline__ void clear()
    {
#pragma unroll
        for (int k = 0; k < W; k++) w[k] = 0;
    }
    // Writes slot n (n < S) without dynamic register indexing.
    __device__ __forceinline__ void put(int n, uint32_t p)
    {
        if (BPS == 1) {
#pragma unroll
            for (int k = 0; k < W; k++)
                if ((n >> 2) == k) w[k] |= (p & 0xFFu) << (8 * (n & 3));
        } else {
#pragma unroll
            for (int k = 0; k < W; k++)
                if (n == k) w[k] = p;
        }
    }
};

// T[src][dst][species], 0 for out-of-range ids (byte_diffusion_1d_dev.cu:70-78).
__device__ __forceinline__ float lookup_T(const DevTables &m, uint32_t p, uint32_t src, uint32_t dst)
{
    if ((uint32_t)(p - 1u) >= m.ns || dst >= m.nst || src >= m.nst) return 0.0f;
    return tload(m.T + ((size_t)src * m.nst + dst) * m.ns + (p - 1u));
}

// One row T[src][dst][*] of the transition table, held in registers: the
// lookups of a site's particles need no access to the table set itself.
struct TRow {
    const float *row;  // null when src or dst is out of range
    uint32_t ns;
    __device__ __forceinline__ TRow(const float *T, uint32_t ns_, uint32_t nst, uint32_t src, uint32_t dst)
        : row(src < nst && dst < nst ? T + ((size_t)src * nst + dst) * ns_ : nullptr), ns(ns_)
    {
    }
    // lookup_T for particle p, the same value.
    __device__ __forceinline__ float operator()(uint32_t p) const
    {
        return (row && (uint32_t)(p - 1u) < ns) ? tload(row + (p - 1u)) : 0.0f;
    }
};

// Queues one overflowed particle; the list index comes from an atomic, the
// sort key restores a deterministic order later.
__device__ __forceinline__ void push_overflow(RunState *rs, OverflowEntry *list, uint32_t cap,
                                              uint32_t phase, uint32_t site, uint32_t seq, uint32_t particle)
{
    uint32_t idx = atomicAdd(&rs->ovf_count, 1u);
    if (idx < cap) {
        OverflowEntry e;
        e.key = ((unsigned long long)phase << KEY_PHASE_SHIFT) |
                ((unsigned long long)site << KEY_SITE_SHIFT) | (unsigned long long)seq;
        e.site = site;
        e.particle = particle;
        list[idx] = e;
    }
}

}  // namespace lmb
