// lmb_overflow.cuh -- on-device overflow resolution, shared by the per-phase
// resolve kernel and the last block of the fused timestep kernel.
//
// The reference copies the whole lattice to the host when any particle
// overflowed and reinserts there (MpdRdmeSolver.cu:1103-1189).  Here one
// block sorts the step's queue by (phase, site, seq) -- one of the orders the
// reference's atomicAdd list can take -- and reinserts in that order with the
// same search, on the device.  Lattice words are read through L2 (ld.cg):
// other blocks of the same launch may have just written them.
#pragma once

#include "lmb.h"
#include "lmb_device.cuh"
#include "lmb_internal.h"

namespace lmb {

template <int BPS, int S>
__device__ __forceinline__ void load_site_cg(const uint32_t *lat, uint32_t N, uint32_t i, SiteWords<BPS, S> &s)
{
#pragma unroll
    for (int k = 0; k < SiteWords<BPS, S>::W; k++) s.w[k] = __ldcg(lat + (size_t)k * N + i);
}

// Slots up to the first empty one (ByteLattice.cpp:187-206).
template <int BPS, int S>
__device__ uint32_t occupancy_at(const uint32_t *lat, uint32_t N, uint32_t i)
{
    SiteWords<BPS, S> s;
    load_site_cg<BPS, S>(lat, N, i, s);
    uint32_t k = 0;
#pragma unroll
    for (int j = 0; j < S; j++)
        if (k == (uint32_t)j && s.slot(j) != 0) k++;
    return k;
}

// Raises the plane bound of site i's segment to cover slot k (pb may be
// null: the lattice keeps no plane bounds).
template <int BPS>
__device__ __forceinline__ void cover_slot(uint32_t *pb, uint32_t i, uint32_t k)
{
    if (pb) {
        const uint32_t planes = (BPS == 1 ? k >> 2 : k) + 1u;
        if (__ldcg(pb + (i >> PB_SHIFT)) < planes) atomicMax(pb + (i >> PB_SHIFT), planes);
    }
}

// First empty slot of site i gets p (ByteLattice.cpp:265-289); false if full.
template <int BPS, int S>
__device__ bool add_particle(uint32_t *lat, uint32_t N, uint32_t i, uint32_t p, uint32_t *pb)
{
    SiteWords<BPS, S> s;
    load_site_cg<BPS, S>(lat, N, i, s);
#pragma unroll
    for (int j = 0; j < S; j++) {
        if (s.slot(j) == 0) {
            s.put(j, p);
            s.store(lat, N, i);
            cover_slot<BPS>(pb, i, (uint32_t)j);
            return true;
        }
    }
    return false;
}

// Classic reinsertion (MpdRdmeSolver.cu:1113-1156): shells of radius 0..4
// from Lattice::getNearbySites (Lattice.cpp:106-128: clamped to the lattice,
// x outer, y, z inner), first site of the same type with a free slot.
template <int BPS, int S>
__device__ bool reinsert_classic(uint32_t *lat, const uint8_t *sites, const Geometry &g, uint32_t idx, uint32_t p,
                                 uint32_t *pb)
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
                        if (add_particle<BPS, S>(lat, g.N, j, p, pb)) return true;
                }
    }
    return false;
}

// Smallest power of two >= n (n >= 1).
__host__ __device__ __forceinline__ uint32_t pow2_at_least(uint32_t n)
{
    uint32_t p = 1;
    while (p < n) p <<= 1;
    return p;
}

// Resolves the step's overflow queue with the whole block (thread `tid` of
// `nthreads`); `sh` holds pow2_at_least(cap) entries.  On success the step
// counter advances.  pb: the lattice's plane bounds, raised for every slot
// filled here (null when it keeps none).  counts (when not null): species
// counts of the lattice being taken, to which every particle put back is
// added.
template <int BPS, int S>
__device__ void resolve_block_flat(uint32_t *lat, const uint8_t *sites, const Geometry &g, RunState *rs,
                                   OverflowEntry *list, uint32_t cap, OverflowEntry *sh, uint32_t tid,
                                   uint32_t nthreads, uint32_t *pb, unsigned long long *counts = nullptr)
{
    const uint32_t n = *(volatile uint32_t *)&rs->ovf_count;
    const uint32_t carried = rs->carried;
    if (n == 0) {
        if (tid == 0) set_step(rs, rs->seed, rs->step + 1);
        return;
    }
    if (n > cap) {
        if (tid == 0) {
            rs->overflows += (unsigned long long)(n - carried);
            rs->status = LMB_E_OVERFLOW_EXHAUSTED;
            rs->failed_step = rs->step;
        }
        return;
    }
    const uint32_t p2 = pow2_at_least(n);
    for (uint32_t e = tid; e < p2; e += nthreads) {
        if (e < n) {
            OverflowEntry v;
            v.key = __ldcg(&list[e].key);
            v.site = __ldcg(&list[e].site);
            v.particle = __ldcg(&list[e].particle);
            sh[e] = v;
        } else {
            sh[e].key = ~0ull;
            sh[e].site = 0;
            sh[e].particle = 0;
        }
    }
    __syncthreads();
    // Bitonic sort by key.
    for (uint32_t k = 2; k <= p2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t e = tid; e < p2; e += nthreads) {
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
    if (tid != 0) return;
    rs->overflows += (unsigned long long)(n - carried);
    if (rs->mode == LMB_OVERFLOW_CLASSIC) {
        for (uint32_t e = 0; e < n; e++) {
            if (!reinsert_classic<BPS, S>(lat, sites, g, sh[e].site, sh[e].particle, pb)) {
                rs->status = LMB_E_OVERFLOW_UNRESOLVED;
                rs->failed_step = rs->step;
                return;
            }
            if (counts) atomicAdd(counts + sh[e].particle, 1ull);
        }
        rs->ovf_count = 0;
        rs->carried = 0;
    } else {
        // Relaxed (MpdRdmeSolver.cu:1677-1761): own site only; the rest stay
        // queued, in order, for the next timestep.
        uint32_t kept = 0;
        for (uint32_t e = 0; e < n; e++) {
            if (!add_particle<BPS, S>(lat, g.N, sh[e].site, sh[e].particle, pb)) {
                OverflowEntry o = sh[e];
                o.key = (unsigned long long)kept;  // phase 0, list order
                list[kept++] = o;
            } else if (counts) {
                atomicAdd(counts + sh[e].particle, 1ull);
            }
        }
        rs->ovf_count = kept;
        rs->carried = kept;
    }
    __threadfence();
    set_step(rs, rs->seed, rs->step + 1);
}

template <int BPS, int S>
__device__ void resolve_block(uint32_t *lat, const uint8_t *sites, const Geometry &g, RunState *rs,
                              OverflowEntry *list, uint32_t cap, OverflowEntry *sh, uint32_t *pb)
{
    resolve_block_flat<BPS, S>(lat, sites, g, rs, list, cap, sh, threadIdx.x, blockDim.x, pb);
}

}  // namespace lmb
