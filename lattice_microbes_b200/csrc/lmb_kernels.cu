// lmb_kernels.cu -- per-phase MPD-RDME kernels for sm_100a.
//
// One timestep is x, y and z hop sweeps (ping-pong buffers), the reaction
// step in place, then on-device overflow resolution
// (MpdRdmeSolver.cu:996-1193).  Every kernel reads the run state first and
// does nothing once a run has failed, so a queued run stops cleanly at the
// failing timestep.
//
// Sweep design: one thread per site.  A thread loads its own site and its two
// neighbours along the sweep axis (coalesced word-planar loads; the neighbour
// rows are L1/L2 hits for the neighbouring warps), recomputes the neighbours'
// hop decisions from the counter hash, and assembles its new site in
// registers.  Because every decision is a pure function of (seed, step, site,
// slot, site types), recomputing a neighbour's choice gives the same answer
// the neighbour's own thread gets, so no shared-memory exchange or barrier is
// needed.  Empty neighbourhoods take a store-only fast path.
#include <cuda_runtime.h>
#include <stdint.h>

#include "lmb.h"
#include "lmb_device.cuh"
#include "lmb_internal.h"

namespace lmb {

// ---------------------------------------------------------------------------
// Diffusion sweep
// ---------------------------------------------------------------------------

// Appends particles to a new site in order; the (S+1)-th and later ones
// overflow with seq = position - S (byte_diffusion_1d_dev.cu:199-269).
template <int BPS, int S>
struct SiteBuilder {
    SiteWords<BPS, S> out;
    int n;
    __device__ __forceinline__ void init()
    {
        out.clear();
        n = 0;
    }
    __device__ __forceinline__ void push(uint32_t p, RunState *rs, OverflowEntry *list, uint32_t cap,
                                         uint32_t phase, uint32_t site)
    {
        if (n < S) out.put(n, p);
        else push_overflow(rs, list, cap, phase, site, (uint32_t)(n - S), p);
        n++;
    }
};

template <int BPS, int S, int DIM>
__global__ void __launch_bounds__(256) sweep_kernel(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst,
                                                    const uint8_t *__restrict__ sites, Geometry g, DevTables m,
                                                    RunState *__restrict__ rs, OverflowEntry *__restrict__ list,
                                                    uint32_t cap)
{
    if (rs->status != LMB_OK) return;
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    const uint32_t z = blockIdx.z;
    if (x >= g.X || y >= g.Y) return;
    const uint32_t i = x + y * g.X + z * g.XY;
    uint32_t im, ip;
    if (DIM == 0) {
        im = i - x + (x == 0 ? g.X - 1 : x - 1);
        ip = i - x + (x == g.X - 1 ? 0 : x + 1);
    } else if (DIM == 1) {
        const uint32_t base = i - y * g.X;
        im = base + (y == 0 ? g.Y - 1 : y - 1) * g.X;
        ip = base + (y == g.Y - 1 ? 0 : y + 1) * g.X;
    } else {
        const uint32_t base = i - z * g.XY;
        im = base + (z == 0 ? g.Z - 1 : z - 1) * g.XY;
        ip = base + (z == g.Z - 1 ? 0 : z + 1) * g.XY;
    }
    SiteWords<BPS, S> own, mn, pl;
    own.load(src, g.N, i);
    mn.load(src, g.N, im);
    pl.load(src, g.N, ip);
    SiteBuilder<BPS, S> b;
    b.init();
    if (own.empty() && mn.empty() && pl.empty()) {
        b.out.store(dst, g.N, i);
        return;
    }
    const unsigned long long th = timestep_hash(rs->seed, rs->step, DIM);
    const uint32_t t = __ldg(sites + i), tm = __ldg(sites + im), tp = __ldg(sites + ip);
    constexpr int CB = CountBits<S>::value;
    const uint32_t phase = DIM + 1;
    // Stayers of this site, slot order.
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p = own.slot(k);
        if (p) {
            const float r = hash_float(((unsigned long long)i << CB) | (unsigned)k, th);
            const float qm = lookup_T(m, p, t, tm);
            const float qp = lookup_T(m, p, t, tp);
            const bool plus = (r >= 0.5f) && (r < __fadd_rn(qp, 0.5f));
            if (!plus && !(r < qm)) b.push(p, rs, list, cap, phase, i);
        }
    }
    // PLUS movers of the minus neighbour.
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p = mn.slot(k);
        if (p) {
            const float r = hash_float(((unsigned long long)im << CB) | (unsigned)k, th);
            const float qp = lookup_T(m, p, tm, t);
            if ((r >= 0.5f) && (r < __fadd_rn(qp, 0.5f))) b.push(p, rs, list, cap, phase, i);
        }
    }
    // MINUS movers of the plus neighbour.
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p = pl.slot(k);
        if (p) {
            const float r = hash_float(((unsigned long long)ip << CB) | (unsigned)k, th);
            const float qm = lookup_T(m, p, tp, t);
            if (r < qm) b.push(p, rs, list, cap, phase, i);
        }
    }
    b.out.store(dst, g.N, i);
}

// ---------------------------------------------------------------------------
// Reaction
// ---------------------------------------------------------------------------

// Per-reaction propensity from FP32 counts (byte_reaction_dev.cu:62-102,
// MPD_GLOBAL_R_MATRIX branch: the self reaction is rate*n*(n-1)).
template <int BPS, int S>
__device__ __forceinline__ float reaction_propensity(const DevTables &m, uint32_t t, const SiteWords<BPS, S> &s,
                                                     uint32_t rx)
{
    if (!__ldg(m.RL + (size_t)rx * m.nst + t)) return 0.0f;
    const uint32_t d1 = __ldg(m.D1 + rx), d2 = __ldg(m.D2 + rx);
    float n1 = 0.0f, n2 = 0.0f;
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p = s.slot(k);
        if (p > 0) {
            n1 = __fadd_rn(n1, p == d1 ? 1.0f : 0.0f);
            n2 = __fadd_rn(n2, p == d2 ? 1.0f : 0.0f);
        }
    }
    const float rate = __ldg(m.rate + rx);
    switch (__ldg(m.order + rx)) {
    case 1: return rate;
    case 2: return __fmul_rn(rate, n1);
    case 3: return __fmul_rn(__fmul_rn(rate, n1), n2);
    case 4: return __fmul_rn(__fmul_rn(rate, n1), __fsub_rn(n1, 1.0f));
    default: return 0.0f;
    }
}

constexpr int MAX_STOICH = 32;

// precomp_reaction_kernel (MpdRdmeSolver.cu:1590-1675) with
// byte_reaction_dev.cu:121-258: table propensity sum in slot order, double
// precision probability, one reaction at most, in-place update.
template <int BPS, int S>
__global__ void __launch_bounds__(256) reaction_kernel(uint32_t *__restrict__ lat, const uint8_t *__restrict__ sites,
                                                       Geometry g, DevTables m, RunState *__restrict__ rs,
                                                       OverflowEntry *__restrict__ list, uint32_t cap)
{
    if (rs->status != LMB_OK) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    const uint32_t t = __ldg(sites + i);
    SiteWords<BPS, S> s;
    s.load_plain(lat, g.N, i);
    float a = __ldg(m.qp0 + t);
    if (s.empty() && a == 0.0f) return;
    const size_t o1 = (size_t)t * m.ns, o2 = (size_t)t * m.ns * m.ns;
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t p1 = s.slot(k);
        if (p1 > 0) {
            a = __fadd_rn(a, __ldg(m.qp1 + o1 + (p1 - 1)));
#pragma unroll
            for (int j = k + 1; j < S; j++) {
                const uint32_t p2 = s.slot(j);
                if (p2 > 0) a = __fadd_rn(a, __ldg(m.qp2 + o2 + (size_t)(p1 - 1) * m.ns + (p2 - 1)));
            }
        }
    }
    if (a == 0.0f) return;
    const float prob = (float)(1.0 - exp(-(double)a));
    const unsigned long long th = timestep_hash(rs->seed, rs->step, 3);
    const float r0 = hash_float(((unsigned long long)i << 1) | 0ull, th);
    if (!(prob > 0.0f && r0 <= prob)) return;

    float rp = __fmul_rn(hash_float(((unsigned long long)i << 1) | 1ull, th), a);
    uint32_t idx = 0;
    for (uint32_t rx = 0; rx < m.nr; rx++) {
        const float prop = reaction_propensity<BPS, S>(m, t, s, rx);
        if (prop > 0.0f) {
            if (rp > 0.0f) idx = rx;
            rp = __fsub_rn(rp, prop);
        }
    }
    atomicAdd(&rs->reactions, 1ull);

    // Stoichiometry of the chosen reaction, ascending species.
    const uint32_t e0 = __ldg(m.stoich_off + idx), e1 = __ldg(m.stoich_off + idx + 1);
    const int ne = (int)(e1 - e0) < MAX_STOICH ? (int)(e1 - e0) : MAX_STOICH;
    uint32_t sp[MAX_STOICH];
    int dlt[MAX_STOICH];
    for (int e = 0; e < ne; e++) {
        sp[e] = __ldg(m.stoich_sp + e0 + e);
        dlt[e] = __ldg(m.stoich_d + e0 + e);
    }
    // Survivors in slot order; a consumed reactant bumps its count.
    SiteWords<BPS, S> out;
    out.clear();
    int n = 0;
#pragma unroll
    for (int k = 0; k < S; k++) {
        const uint32_t q = s.slot(k);
        if (q > 0) {
            bool consumed = false;
            for (int e = 0; e < ne; e++) {
                if (sp[e] == q - 1) {
                    if (dlt[e] < 0) {
                        dlt[e]++;
                        consumed = true;
                    }
                    break;
                }
            }
            if (!consumed) out.put(n++, q);
        }
    }
    // Products by ascending species id; extra ones overflow.
    uint32_t seq = 0;
    for (int e = 0; e < ne; e++) {
        for (int j = 0; j < dlt[e]; j++) {
            const uint32_t p = sp[e] + 1;
            if (n < S) out.put(n++, p);
            else push_overflow(rs, list, cap, 4u, i, seq++, p);
        }
    }
    out.store(lat, g.N, i);
}

// ---------------------------------------------------------------------------
// Overflow resolution (one block)
// ---------------------------------------------------------------------------

template <int BPS, int S>
__device__ uint32_t occupancy_at(const uint32_t *lat, uint32_t N, uint32_t i)
{
    SiteWords<BPS, S> s;
    s.load_plain(lat, N, i);
    uint32_t k = 0;
#pragma unroll
    for (int j = 0; j < S; j++)
        if (k == (uint32_t)j && s.slot(j) != 0) k++;
    return k;
}

// First empty slot of site i gets p (ByteLattice.cpp:265-289); false if full.
template <int BPS, int S>
__device__ bool add_particle(uint32_t *lat, uint32_t N, uint32_t i, uint32_t p)
{
    SiteWords<BPS, S> s;
    s.load_plain(lat, N, i);
#pragma unroll
    for (int j = 0; j < S; j++) {
        if (s.slot(j) == 0) {
            s.put(j, p);
            s.store(lat, N, i);
            return true;
        }
    }
    return false;
}

// Classic reinsertion (MpdRdmeSolver.cu:1103-1189): shells of radius 0..4
// from Lattice::getNearbySites (Lattice.cpp:106-128: clamped to the lattice,
// x outer, y, z inner), first site of the same type with a free slot.
template <int BPS, int S>
__device__ bool reinsert_classic(uint32_t *lat, const uint8_t *sites, const Geometry &g, uint32_t idx, uint32_t p)
{
    const uint32_t xc = idx % g.X, yc = (idx / g.X) % g.Y, zc = idx / g.XY;
    const uint8_t tc = sites[idx];
    for (uint32_t radius = 0; radius <= 4; radius++) {
        const uint32_t mind = radius > 0 ? radius - 1 : 0, maxd = radius;
        const double min2 = (double)(mind * mind), max2 = (double)(maxd * maxd);
        const uint32_t x0 = xc >= maxd ? xc - maxd : 0, x1 = (xc + maxd < g.X) ? xc + maxd : g.X - 1;
        const uint32_t y0 = yc >= maxd ? yc - maxd : 0, y1 = (yc + maxd < g.Y) ? yc + maxd : g.Y - 1;
        const uint32_t z0 = zc >= maxd ? zc - maxd : 0, z1 = (zc + maxd < g.Z) ? zc + maxd : g.Z - 1;
        for (uint32_t x = x0; x <= x1; x++)
            for (uint32_t y = y0; y <= y1; y++)
                for (uint32_t z = z0; z <= z1; z++) {
                    const double dx = (double)x - xc, dy = (double)y - yc, dz = (double)z - zc;
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    if (!(r2 <= max2 && (r2 > min2 || mind == maxd))) continue;
                    const uint32_t j = x + y * g.X + z * g.XY;
                    if (sites[j] == tc && occupancy_at<BPS, S>(lat, g.N, j) < (uint32_t)S)
                        if (add_particle<BPS, S>(lat, g.N, j, p)) return true;
                }
    }
    return false;
}

constexpr int RESOLVE_THREADS = 512;

// Sorts the step's overflow entries by key (carried entries first, then
// (phase, site, seq)) and reinserts them in that order; advances the step.
template <int BPS, int S>
__global__ void __launch_bounds__(RESOLVE_THREADS) resolve_kernel(uint32_t *__restrict__ lat,
                                                                  const uint8_t *__restrict__ sites, Geometry g,
                                                                  RunState *__restrict__ rs,
                                                                  OverflowEntry *__restrict__ list, uint32_t cap)
{
    extern __shared__ OverflowEntry sh[];
    if (rs->status != LMB_OK) return;
    const uint32_t n = rs->ovf_count;
    const uint32_t carried = rs->carried;
    if (n == 0) {
        if (threadIdx.x == 0) rs->step++;
        return;
    }
    if (n > cap) {
        if (threadIdx.x == 0) {
            rs->overflows += (unsigned long long)(n - carried);
            rs->status = LMB_E_OVERFLOW_EXHAUSTED;
            rs->failed_step = rs->step;
        }
        return;
    }
    uint32_t pow2 = 1;
    while (pow2 < n) pow2 <<= 1;
    for (uint32_t e = threadIdx.x; e < pow2; e += blockDim.x) {
        if (e < n) sh[e] = list[e];
        else {
            sh[e].key = ~0ull;
            sh[e].site = 0;
            sh[e].particle = 0;
        }
    }
    __syncthreads();
    // Bitonic sort of pow2 entries by key.
    for (uint32_t k = 2; k <= pow2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t e = threadIdx.x; e < pow2; e += blockDim.x) {
                const uint32_t o = e ^ j;
                if (o > e) {
                    const bool up = (e & k) == 0;
                    const OverflowEntry a = sh[e], b = sh[o];
                    if ((a.key > b.key) == up) {
                        sh[e] = b;
                        sh[o] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x != 0) return;
    rs->overflows += (unsigned long long)(n - carried);
    if (rs->mode == LMB_OVERFLOW_CLASSIC) {
        for (uint32_t e = 0; e < n; e++) {
            if (!reinsert_classic<BPS, S>(lat, sites, g, sh[e].site, sh[e].particle)) {
                rs->status = LMB_E_OVERFLOW_UNRESOLVED;
                rs->failed_step = rs->step;
                return;
            }
        }
        rs->ovf_count = 0;
        rs->carried = 0;
    } else {
        // Relaxed (MpdRdmeSolver.cu:1677-1761): own site only; the rest stay
        // queued, in order, for the next timestep.
        uint32_t kept = 0;
        for (uint32_t e = 0; e < n; e++) {
            if (!add_particle<BPS, S>(lat, g.N, sh[e].site, sh[e].particle)) {
                OverflowEntry o = sh[e];
                o.key = (unsigned long long)kept;  // phase 0, list order
                list[kept++] = o;
            }
        }
        rs->ovf_count = kept;
        rs->carried = kept;
    }
    __threadfence();
    rs->step++;
}

// Sets the run state for a new run without a host round trip.  The relaxed
// handler's queue survives across runs; the classic one starts empty.
__global__ void begin_run_kernel(RunState *rs, uint32_t seed, uint32_t first, uint32_t n, uint32_t mode)
{
    rs->seed = seed;
    rs->step = first;
    rs->end_step = first + n;
    rs->status = LMB_OK;
    rs->failed_step = 0;
    rs->mode = mode;
    rs->overflows = 0;
    rs->reactions = 0;
    if (mode == LMB_OVERFLOW_CLASSIC) {
        rs->ovf_count = 0;
        rs->carried = 0;
    }
}

cudaError_t launch_begin_run(RunState *rs, uint32_t seed, uint32_t first, uint32_t n, uint32_t mode,
                             cudaStream_t stream)
{
    count_launch();
    begin_run_kernel<<<1, 1, 0, stream>>>(rs, seed, first, n, mode);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Counts, validation, layout conversion
// ---------------------------------------------------------------------------

template <int BPS, int S>
__global__ void counts_kernel(const uint32_t *__restrict__ lat, Geometry g, uint32_t ns,
                              unsigned long long *__restrict__ counts)
{
    extern __shared__ unsigned int hist[];
    const bool use_shared = ns + 1 <= 8192;
    if (use_shared)
        for (uint32_t s = threadIdx.x; s <= ns; s += blockDim.x) hist[s] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g.N; i += gridDim.x * blockDim.x) {
        SiteWords<BPS, S> s;
        s.load(lat, g.N, i);
        if (s.empty()) continue;
#pragma unroll
        for (int k = 0; k < S; k++) {
            const uint32_t p = s.slot(k);
            if (p && p <= ns) {
                if (use_shared) atomicAdd(&hist[p], 1u);
                else atomicAdd(&counts[p], 1ull);
            }
        }
    }
    __syncthreads();
    if (use_shared)
        for (uint32_t s = threadIdx.x; s <= ns; s += blockDim.x)
            if (hist[s]) atomicAdd(&counts[s], (unsigned long long)hist[s]);
}

template <int BPS, int S>
__global__ void validate_kernel(const uint32_t *__restrict__ lat, const uint8_t *__restrict__ sites, Geometry g,
                                RunState *rs)
{
    uint32_t ms = 0, mt = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g.N; i += gridDim.x * blockDim.x) {
        SiteWords<BPS, S> s;
        s.load(lat, g.N, i);
#pragma unroll
        for (int k = 0; k < S; k++) ms = max(ms, s.slot(k));
        mt = max(mt, (uint32_t)sites[i]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        ms = max(ms, __shfl_xor_sync(0xffffffffu, ms, o));
        mt = max(mt, __shfl_xor_sync(0xffffffffu, mt, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&rs->max_species, ms);
        atomicMax(&rs->max_site_type, mt);
    }
}

// Row-major [x][y][z][p] -> native packed sites (RDMESolver.cpp:144-189: each
// nonzero entry goes to the first free slot, in row-major order).
template <int BPS, int S>
__global__ void row_major_to_native_kernel(const void *__restrict__ rm, const uint8_t *__restrict__ rm_sites,
                                           uint32_t *__restrict__ native, uint8_t *__restrict__ sites, Geometry g,
                                           RunState *rs)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    const uint32_t x = i % g.X, y = (i / g.X) % g.Y, z = i / g.XY;
    const size_t r = ((size_t)x * g.Y + y) * g.Z + z;
    SiteWords<BPS, S> s;
    s.clear();
    int n = 0;
    uint32_t ms = 0;
    for (int k = 0; k < S; k++) {
        const uint32_t p = BPS == 1 ? (uint32_t)((const uint8_t *)rm)[r * S + k] : ((const uint32_t *)rm)[r * S + k];
        if (p) {
            s.put(n++, p);
            ms = max(ms, p);
        }
    }
    s.store(native, g.N, i);
    const uint8_t st = rm_sites[r];
    sites[i] = st;
    atomicMax(&rs->max_species, ms);
    atomicMax(&rs->max_site_type, (uint32_t)st);
}

template <int BPS, int S>
__global__ void native_to_row_major_kernel(const uint32_t *__restrict__ native, const uint8_t *__restrict__ sites,
                                           void *__restrict__ rm, uint8_t *__restrict__ rm_sites, Geometry g)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N) return;
    const uint32_t x = i % g.X, y = (i / g.X) % g.Y, z = i / g.XY;
    const size_t r = ((size_t)x * g.Y + y) * g.Z + z;
    SiteWords<BPS, S> s;
    s.load(native, g.N, i);
#pragma unroll
    for (int k = 0; k < S; k++) {
        if (BPS == 1) ((uint8_t *)rm)[r * S + k] = (uint8_t)s.slot(k);
        else ((uint32_t *)rm)[r * S + k] = s.slot(k);
    }
    if (rm_sites) rm_sites[r] = sites[i];
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------

static void sweep_shape(const Geometry &g, dim3 &grid, dim3 &block)
{
    uint32_t bx = ((g.X + 31) / 32) * 32;
    if (bx > 128) bx = 128;
    uint32_t by = 256 / bx;
    if (by > g.Y) by = g.Y;
    block = dim3(bx, by, 1);
    grid = dim3((g.X + bx - 1) / bx, (g.Y + by - 1) / by, g.Z);
}

#define LMB_DISPATCH(BPS_, S_, ...)                                                   \
    if (bps == BPS_ && slots == S_) {                                                 \
        constexpr int BPS = BPS_;                                                     \
        constexpr int S = S_;                                                         \
        __VA_ARGS__;                                                                  \
        return cudaGetLastError();                                                    \
    }

#define LMB_DISPATCH_ALL(...)                \
    LMB_DISPATCH(1, 4, __VA_ARGS__)          \
    LMB_DISPATCH(1, 8, __VA_ARGS__)          \
    LMB_DISPATCH(1, 16, __VA_ARGS__)         \
    LMB_DISPATCH(1, 32, __VA_ARGS__)         \
    LMB_DISPATCH(4, 4, __VA_ARGS__)          \
    LMB_DISPATCH(4, 8, __VA_ARGS__)          \
    LMB_DISPATCH(4, 16, __VA_ARGS__)         \
    return cudaErrorInvalidValue;

bool slots_supported(int bps, int slots)
{
    if (bps == 1) return slots == 4 || slots == 8 || slots == 16 || slots == 32;
    if (bps == 4) return slots == 4 || slots == 8 || slots == 16;
    return false;
}

cudaError_t launch_sweep(int bps, int slots, int dim, const uint32_t *src, uint32_t *dst, const uint8_t *sites,
                         const Geometry &g, const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                         cudaStream_t stream)
{
    dim3 grid, block;
    sweep_shape(g, grid, block);
    count_launch();
    LMB_DISPATCH_ALL({
        if (dim == 0) sweep_kernel<BPS, S, 0><<<grid, block, 0, stream>>>(src, dst, sites, g, m, rs, list, cap);
        else if (dim == 1) sweep_kernel<BPS, S, 1><<<grid, block, 0, stream>>>(src, dst, sites, g, m, rs, list, cap);
        else sweep_kernel<BPS, S, 2><<<grid, block, 0, stream>>>(src, dst, sites, g, m, rs, list, cap);
    })
}

cudaError_t launch_reaction(int bps, int slots, uint32_t *lat, const uint8_t *sites, const Geometry &g,
                            const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap, cudaStream_t stream)
{
    const uint32_t threads = 256, blocks = (g.N + threads - 1) / threads;
    count_launch();
    LMB_DISPATCH_ALL(reaction_kernel<BPS, S><<<blocks, threads, 0, stream>>>(lat, sites, g, m, rs, list, cap))
}

cudaError_t launch_resolve(int bps, int slots, uint32_t *lat, const uint8_t *sites, const Geometry &g, RunState *rs,
                           OverflowEntry *list, uint32_t cap, cudaStream_t stream)
{
    uint32_t pow2 = 1;
    while (pow2 < cap) pow2 <<= 1;
    const size_t smem = (size_t)pow2 * sizeof(OverflowEntry);
    count_launch();
    LMB_DISPATCH_ALL({
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(resolve_kernel<BPS, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        resolve_kernel<BPS, S><<<1, RESOLVE_THREADS, smem, stream>>>(lat, sites, g, rs, list, cap);
    })
}

cudaError_t launch_counts(int bps, int slots, const uint32_t *lat, const Geometry &g, uint32_t ns,
                          unsigned long long *counts, cudaStream_t stream)
{
    const uint32_t threads = 256;
    uint32_t blocks = (g.N + threads - 1) / threads;
    if (blocks > 148 * 8) blocks = 148 * 8;
    const size_t smem = ns + 1 <= 8192 ? (ns + 1) * sizeof(unsigned int) : 0;
    count_launch();
    LMB_DISPATCH_ALL(counts_kernel<BPS, S><<<blocks, threads, smem, stream>>>(lat, g, ns, counts))
}

cudaError_t launch_validate(int bps, int slots, const uint32_t *lat, const uint8_t *sites, const Geometry &g,
                            RunState *rs, cudaStream_t stream)
{
    const uint32_t threads = 256;
    uint32_t blocks = (g.N + threads - 1) / threads;
    if (blocks > 148 * 8) blocks = 148 * 8;
    count_launch();
    LMB_DISPATCH_ALL(validate_kernel<BPS, S><<<blocks, threads, 0, stream>>>(lat, sites, g, rs))
}

cudaError_t launch_row_major_to_native(int bps, int slots, const void *rm, const uint8_t *rm_sites, uint32_t *native,
                                       uint8_t *sites, const Geometry &g, RunState *rs, cudaStream_t stream)
{
    const uint32_t threads = 256, blocks = (g.N + threads - 1) / threads;
    count_launch();
    LMB_DISPATCH_ALL(
        row_major_to_native_kernel<BPS, S><<<blocks, threads, 0, stream>>>(rm, rm_sites, native, sites, g, rs))
}

cudaError_t launch_native_to_row_major(int bps, int slots, const uint32_t *native, const uint8_t *sites, void *rm,
                                       uint8_t *rm_sites, const Geometry &g, cudaStream_t stream)
{
    const uint32_t threads = 256, blocks = (g.N + threads - 1) / threads;
    count_launch();
    LMB_DISPATCH_ALL(
        native_to_row_major_kernel<BPS, S><<<blocks, threads, 0, stream>>>(native, sites, rm, rm_sites, g))
}

}  // namespace lmb
