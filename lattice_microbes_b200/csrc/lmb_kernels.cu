// lmb_kernels.cu -- per-phase MPD-RDME kernels for sm_100a.
//
// One timestep is x, y and z hop sweeps (ping-pong buffers), the reaction
// step in place, then on-device overflow resolution
// (MpdRdmeSolver.cu:996-1193).  Every kernel reads the run state first and
// does nothing once a run has failed, so a queued run stops cleanly at the
// failing timestep.
//
// Sweep design: one thread per site; a block covers a tile of sites that is
// long along the sweep axis (x rows for the x sweep, 8 y rows or 8 z planes
// for the y and z sweeps, plus a halo row of threads on either side that
// only reads).  Each thread draws its own site's hop choices once (one hash
// per particle, balanced over the warp), publishes the site and its choices
// in shared memory, and the tile's threads assemble their new sites from
// their own and their two neighbours' entries.  Halo rows and the ends of x
// rows longer than 256 sites draw a neighbour's choices a second time; every
// decision is a pure function of (seed, step, site, slot, site types), so the
// copies agree.
#include <cuda_runtime.h>
#include <stdint.h>

#include "lmb.h"
#include "lmb_device.cuh"
#include "lmb_internal.h"
#include "lmb_overflow.cuh"
#include "lmb_site.cuh"

namespace lmb {

// ---------------------------------------------------------------------------
// Diffusion sweep
// ---------------------------------------------------------------------------

// Sites written by one block, and threads of a y or z block: its tile plus
// one halo row of threads on either side along the sweep axis.
constexpr int SWEEP_THREADS = 256;
constexpr int SWEEP_MAX_THREADS = 320;

// Lattice coordinates of the thread's site.  x tiles are whole x rows (or
// 256-site pieces of longer rows); y and z tiles carry a halo row on either
// side, so thread row r of a tile starting at a0 holds axis coordinate
// a0 - 1 + r, wrapped periodically.  Rows past the wrap point (a0 - 1 + r >
// extent) hold no site; a row at exactly the extent holds coordinate 0 and is
// read but not written.
template <int DIM>
__device__ __forceinline__ void sweep_site_of(const Geometry &g, uint32_t &x, uint32_t &y, uint32_t &z, bool &in,
                                              bool &out)
{
    x = blockIdx.x * blockDim.x + threadIdx.x;
    y = blockIdx.y * blockDim.y + threadIdx.y;
    z = blockIdx.z * blockDim.z + threadIdx.z;
    if (DIM == 0) {
        in = out = x < g.X && y < g.Y && z < g.Z;
        return;
    }
    const uint32_t A = DIM == 1 ? g.Y : g.Z;
    const uint32_t r = DIM == 1 ? threadIdx.y : threadIdx.z;
    const uint32_t L = (DIM == 1 ? blockDim.y : blockDim.z) - 2u;
    const int64_t u = (int64_t)(DIM == 1 ? blockIdx.y : blockIdx.z) * L - 1 + r;
    const uint32_t a = u < 0 ? A - 1u : (u >= (int64_t)A ? 0u : (uint32_t)u);
    if (DIM == 1) y = a;
    else z = a;
    in = x < g.X && (DIM == 1 ? z < g.Z : y < g.Y) && u <= (int64_t)A;
    out = in && r >= 1u && r <= L && u < (int64_t)A;
}

// Lattice indices of the site and its two neighbours along axis DIM
// (periodic); for the x sweep also where the neighbours sit in the block's
// tile (-1: outside).  In y and z tiles they are the thread rows either side.
template <int DIM>
__device__ __forceinline__ void sweep_neighbours(const Geometry &g, uint32_t x, uint32_t y, uint32_t z, int lid,
                                                 uint32_t &i, uint32_t &im, uint32_t &ip, int &lm, int &lp)
{
    i = x + y * g.X + z * g.XY;
    if (DIM == 0) {
        const uint32_t xm = x == 0 ? g.X - 1 : x - 1, xp = x == g.X - 1 ? 0 : x + 1;
        im = i - x + xm;
        ip = i - x + xp;
        const uint32_t x0 = blockIdx.x * blockDim.x;
        lm = (xm >= x0 && xm < x0 + blockDim.x) ? lid - (int)x + (int)xm : -1;
        lp = (xp >= x0 && xp < x0 + blockDim.x) ? lid - (int)x + (int)xp : -1;
    } else if (DIM == 1) {
        const uint32_t ym = y == 0 ? g.Y - 1 : y - 1, yp = y == g.Y - 1 ? 0 : y + 1;
        im = i - y * g.X + ym * g.X;
        ip = i - y * g.X + yp * g.X;
        lm = lid - (int)blockDim.x;
        lp = lid + (int)blockDim.x;
    } else {
        const uint32_t zm = z == 0 ? g.Z - 1 : z - 1, zp = z == g.Z - 1 ? 0 : z + 1;
        im = i - z * g.XY + zm * g.XY;
        ip = i - z * g.XY + zp * g.XY;
        lm = lid - (int)(blockDim.x * blockDim.y);
        lp = lid + (int)(blockDim.x * blockDim.y);
    }
}

// Appends site i (type t, n particles after the z sweep) to the reaction
// list when its reaction step could change it (reaction_may_fire), one
// atomic per group of converged lanes.  An entry is the pair (i, t << 8 |
// n).  Entries past rx_cap are dropped but counted, which sends the reaction
// step over every site.
// rb: the bound's inputs for type t; th: the reaction sub-step's hash.
__device__ __forceinline__ void list_for_reaction(uint32_t n, uint32_t t, uint32_t i, int lid, const ReactBound &rb,
                                                  unsigned long long th, RunState *rs, uint32_t *rx_sites,
                                                  uint32_t rx_cap)
{
    bool need = false;
    if (n != 0 || rb.a0 != 0.0f) need = reaction_may_fire(n, rb, hash_float((unsigned long long)i << 1, th));
    const uint32_t act = __activemask();
    const uint32_t want = __ballot_sync(act, need);
    if (!need) return;
    const uint32_t lane = (uint32_t)lid & 31u, leader = __ffs(want) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&rs->rx_count, (uint32_t)__popc(want));
    base = __shfl_sync(want, base, leader);
    const uint32_t idx = base + __popc(want & ((1u << lane) - 1u));
    if (idx < rx_cap) reinterpret_cast<uint2 *>(rx_sites)[idx] = make_uint2(i, (t << 8) | n);
}

// Planes of site i's segment that may hold particles (all W without plane
// bounds).
template <int W>
__device__ __forceinline__ uint32_t planes_at(const uint32_t *__restrict__ pb, uint32_t i)
{
    if (!pb) return (uint32_t)W;
    const uint32_t b = __ldg(pb + (i >> PB_SHIFT));
    return b < (uint32_t)W ? b : (uint32_t)W;
}

// Writes the warp's new sites with plane bounds: every lane of the warp holds
// one site of the same segment (nw: words its new content uses; `word(k)`:
// word k of it).  Planes below the larger of the warp's new bound and the
// destination's old one are written (zeros above a site's content), then the
// new bound replaces the old.
template <int W, typename WordFn>
__device__ __forceinline__ void store_bounded(uint32_t *__restrict__ dst, uint32_t *__restrict__ pb_dst,
                                              uint32_t N, uint32_t i, uint32_t nw, WordFn word)
{
    const uint32_t wmax = __reduce_max_sync(0xffffffffu, nw);
    const uint32_t seg = i >> PB_SHIFT;
    const uint32_t old = pb_dst[seg];
    const uint32_t lim = wmax > old ? wmax : (old < (uint32_t)W ? old : (uint32_t)W);
#pragma unroll
    for (int k = 0; k < W; k++)
        if ((uint32_t)k < lim) dst[(size_t)k * N + i] = word(k);
    __syncwarp();
    if ((threadIdx.x & 31u) == 0) pb_dst[seg] = wmax;
}

template <int BPS, int S, int DIM>
__global__ void __launch_bounds__(SWEEP_MAX_THREADS) sweep_kernel(const uint32_t *__restrict__ src,
                                                                  uint32_t *__restrict__ dst,
                                                                  const uint8_t *__restrict__ sites, Geometry g,
                                                                  DevTables m, RunState *__restrict__ rs,
                                                                  OverflowEntry *__restrict__ list, uint32_t cap,
                                                                  uint32_t *__restrict__ rx_sites, uint32_t rx_cap,
                                                                  const uint32_t *__restrict__ pb_src,
                                                                  uint32_t *__restrict__ pb_dst)
{
    using Code = typename ChoiceCode<S>::type;
    constexpr int W = SiteWords<BPS, S>::W;
    constexpr int NT = DIM == 0 ? SWEEP_THREADS : SWEEP_MAX_THREADS;
    __shared__ uint32_t sw[W][NT];
    __shared__ Code sc[NT];
    chain_enter();
    // The run state's status is loaded with everything else and checked
    // before the first write (a failed run's kernels do nothing), so that
    // its round trip does not come first.
    const int32_t status = rs->status;
    // The z sweep lists reaction sites unless the list overflowed recently.
    const bool listing = DIM == 2 && rs->rx_skip == 0;
    uint32_t x, y, z;
    bool in, out;
    sweep_site_of<DIM>(g, x, y, z, in, out);
    const int lid = (int)(threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z));
    uint32_t i = 0, im = 0, ip = 0;
    int lm = -1, lp = -1;
    SiteWords<BPS, S> own;
    own.clear();
    uint32_t t = 0, tm = 0, tp = 0;
    Code c_own = 0;
    const unsigned long long th = rs->th[DIM];
    uint32_t occ = 0;
    if (in) {
        sweep_neighbours<DIM>(g, x, y, z, lid, i, im, ip, lm, lp);
        own.load_planes(src, g.N, i, planes_at<W>(pb_src, i));
        t = __ldg(sites + i);
        tm = __ldg(sites + im);
        tp = __ldg(sites + ip);
        occ = occupied_slots<BPS, S>(own);
        if constexpr (BPS == 4) {
            // Only a site's occupied slots are ever read from the tile (by
            // the hashing, its own stayers and its neighbours' arrivals).
#pragma unroll
            for (int k = 0; k < W; k++)
                if ((occ >> k) & 1u) sw[k][lid] = own.w[k];
        } else {
#pragma unroll
            for (int k = 0; k < W; k++) sw[k][lid] = own.w[k];
        }
    }
    if (status != LMB_OK) return;  // the same for the whole block
    sc[lid] = 0;
    __syncwarp();
    // The warp's particles drawn together: particle q of the warp (in site,
    // then slot order) goes to lane q % 32, so every lane hashes about the
    // same number of particles however unevenly the sites are filled.
    {
        constexpr int CB = CountBits<S>::value;
        const uint32_t lane = (uint32_t)lid & 31u, wbase = (uint32_t)lid & ~31u;
        const uint32_t n = __popc(occ);
        uint32_t incl = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += v;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31), excl = incl - n;
        for (uint32_t base = 0; base < total; base += 32) {
            const uint32_t q = base + lane;
            // Owner lane: the last lane whose first particle index is <= q.
            uint32_t o = 0;
#pragma unroll
            for (uint32_t step = 16; step >= 1; step >>= 1) {
                const uint32_t e = __shfl_sync(0xffffffffu, excl, (o + step) & 31u);
                if (o + step < 32 && e <= q) o += step;
            }
            const uint32_t occ_o = __shfl_sync(0xffffffffu, occ, o);
            const uint32_t j = q - __shfl_sync(0xffffffffu, excl, o);
            const uint32_t t_o = __shfl_sync(0xffffffffu, t, o), tm_o = __shfl_sync(0xffffffffu, tm, o);
            const uint32_t tp_o = __shfl_sync(0xffffffffu, tp, o), gi_o = __shfl_sync(0xffffffffu, i, o);
            if (q < total) {
                uint32_t mbits = occ_o;
                for (uint32_t r = 0; r < j; r++) mbits &= mbits - 1;
                const uint32_t k = __ffs(mbits) - 1;
                const uint32_t so = wbase + o;
                const uint32_t p = BPS == 1 ? (sw[k >> 2][so] >> (8 * (k & 3u))) & 0xFFu : sw[k][so];
                const float rv = hash_float(((unsigned long long)gi_o << CB) | k, th);
                const float qp = lookup_T(m, p, t_o, tp_o);
                Code bit = 0;
                if ((rv >= 0.5f) && (rv < __fadd_rn(qp, 0.5f))) bit = (Code)1 << (S + k);
                else if (rv < lookup_T(m, p, t_o, tm_o)) bit = (Code)1 << k;
                if (bit) atomicOr(&sc[so], bit);
            }
        }
    }
    __syncthreads();
    if (!out) return;
    c_own = sc[lid];
    // Lattice index of the neighbour's own outer neighbour along the axis.
    auto outer_minus = [&]() {
        if (DIM == 0) {
            const uint32_t xm = x == 0 ? g.X - 1 : x - 1;
            return i - x + (xm == 0 ? g.X - 1 : xm - 1);
        } else if (DIM == 1) {
            const uint32_t ym = y == 0 ? g.Y - 1 : y - 1;
            return i - y * g.X + (ym == 0 ? g.Y - 1 : ym - 1) * g.X;
        }
        const uint32_t zm = z == 0 ? g.Z - 1 : z - 1;
        return i - z * g.XY + (zm == 0 ? g.Z - 1 : zm - 1) * g.XY;
    };
    auto outer_plus = [&]() {
        if (DIM == 0) {
            const uint32_t xp = x == g.X - 1 ? 0 : x + 1;
            return i - x + (xp == g.X - 1 ? 0 : xp + 1);
        } else if (DIM == 1) {
            const uint32_t yp = y == g.Y - 1 ? 0 : y + 1;
            return i - y * g.X + (yp == g.Y - 1 ? 0 : yp + 1) * g.X;
        }
        const uint32_t zp = z == g.Z - 1 ? 0 : z + 1;
        return i - z * g.XY + (zp == g.Z - 1 ? 0 : zp + 1) * g.XY;
    };
    if constexpr (BPS == 4) {
        // IntLattice: a slot is a whole word, read by index from shared or
        // global memory rather than selected among S registers; the new site
        // is gathered in shared memory and written plane by plane.
        __shared__ uint32_t so[S][SWEEP_THREADS];
        // Index among the block's written sites (the halo row of a y or z
        // tile comes first).
        const int oid = DIM == 0 ? lid : lid - (DIM == 1 ? (int)blockDim.x : (int)(blockDim.x * blockDim.y));
        constexpr int CB = CountBits<S>::value;
        constexpr uint32_t LOW = (1u << S) - 1u;
        auto choices_mem = [&](uint32_t idx, uint32_t occ_n, uint32_t t_n, uint32_t tm_n, uint32_t tp_n) {
            Code c = 0;
            while (occ_n) {
                const uint32_t k = __ffs(occ_n) - 1;
                occ_n &= occ_n - 1;
                const uint32_t p = __ldg(src + (size_t)k * g.N + idx);
                const float r = hash_float(((unsigned long long)idx << CB) | k, th);
                if ((r >= 0.5f) && (r < __fadd_rn(lookup_T(m, p, t_n, tp_n), 0.5f))) c |= (Code)1 << (S + k);
                else if (r < lookup_T(m, p, t_n, tm_n)) c |= (Code)1 << k;
            }
            return c;
        };
        Code c_mn = 0, c_pl = 0;
        if (DIM != 0 || lm >= 0) {
            c_mn = sc[lm];
        } else {
            SiteWords<BPS, S> mn;
            mn.load_planes(src, g.N, im, planes_at<W>(pb_src, im));
            const uint32_t o = occupied_slots<BPS, S>(mn);
            if (o) c_mn = choices_mem(im, o, tm, __ldg(sites + outer_minus()), t);
        }
        if (DIM != 0 || lp >= 0) {
            c_pl = sc[lp];
        } else {
            SiteWords<BPS, S> pl;
            pl.load_planes(src, g.N, ip, planes_at<W>(pb_src, ip));
            const uint32_t o = occupied_slots<BPS, S>(pl);
            if (o) c_pl = choices_mem(ip, o, tp, t, __ldg(sites + outer_plus()));
        }
        uint32_t n = 0;
        auto push = [&](uint32_t p) {
            if (n < (uint32_t)S) so[n][oid] = p;
            else push_overflow(rs, list, cap, (uint32_t)DIM + 1, i, n - (uint32_t)S, p);
            n++;
        };
        uint32_t stay = occ & ~((uint32_t)c_own | (uint32_t)(c_own >> S)) & LOW;
        while (stay) {
            const uint32_t k = __ffs(stay) - 1;
            stay &= stay - 1;
            push(sw[k][lid]);
        }
        uint32_t in_m = (uint32_t)(c_mn >> S) & LOW;
        while (in_m) {
            const uint32_t k = __ffs(in_m) - 1;
            in_m &= in_m - 1;
            push(DIM != 0 || lm >= 0 ? sw[k][lm] : __ldg(src + (size_t)k * g.N + im));
        }
        uint32_t in_p = (uint32_t)c_pl & LOW;
        while (in_p) {
            const uint32_t k = __ffs(in_p) - 1;
            in_p &= in_p - 1;
            push(DIM != 0 || lp >= 0 ? sw[k][lp] : __ldg(src + (size_t)k * g.N + ip));
        }
        if (pb_dst) {
            store_bounded<W>(dst, pb_dst, g.N, i, n < (uint32_t)S ? n : (uint32_t)S,
                             [&](int k) { return (uint32_t)k < n ? so[k][oid] : 0u; });
        } else {
#pragma unroll
            for (int k = 0; k < S; k++) dst[(size_t)k * g.N + i] = (uint32_t)k < n ? so[k][oid] : 0u;
        }
        if (DIM == 2 && rx_sites && listing)
            list_for_reaction(n < (uint32_t)S ? n : (uint32_t)S, t, i, lid, react_bound(t, m), rs->th[3], rs,
                              rx_sites, rx_cap);
    } else {
        // The neighbours: from the tile, or loaded with their choices drawn here.
        SiteWords<BPS, S> mn, pl;
        Code c_mn = 0, c_pl = 0;
        if (DIM != 0 || lm >= 0) {
#pragma unroll
            for (int k = 0; k < W; k++) mn.w[k] = sw[k][lm];
            c_mn = sc[lm];
        } else {
            mn.load_planes(src, g.N, im, planes_at<W>(pb_src, im));
            if (!mn.empty()) c_mn = site_choices<BPS, S>(mn, tm, __ldg(sites + outer_minus()), t, im, th, m);
        }
        if (DIM != 0 || lp >= 0) {
#pragma unroll
            for (int k = 0; k < W; k++) pl.w[k] = sw[k][lp];
            c_pl = sc[lp];
        } else {
            pl.load_planes(src, g.N, ip, planes_at<W>(pb_src, ip));
            if (!pl.empty()) c_pl = site_choices<BPS, S>(pl, tp, t, __ldg(sites + outer_plus()), ip, th, m);
        }
        const SiteWords<BPS, S> out = assemble_site<BPS, S>(own, c_own, mn, c_mn, pl, c_pl, i, true,
                                                            (uint32_t)DIM + 1, rs, list, cap);
        const uint32_t n_out = (uint32_t)__popc(occupied_slots<BPS, S>(out));
        if (pb_dst) store_bounded<W>(dst, pb_dst, g.N, i, (n_out + 3u) >> 2, [&](int k) { return out.w[k]; });
        else out.store(dst, g.N, i);
        if (DIM == 2 && rx_sites && listing)
            list_for_reaction(n_out, t, i, lid, react_bound(t, m), rs->th[3], rs, rx_sites, rx_cap);
    }
}

// ---------------------------------------------------------------------------
// IntLattice sweep with plane bounds
// ---------------------------------------------------------------------------

// y and z tiles of the plane-bounded sweep: 16 sites along the axis plus a
// halo row on either side, 32 sites (one segment) across.
constexpr int SWEEP_PB_TILE = 16;
constexpr int SWEEP_PB_YZ_THREADS = 32 * (SWEEP_PB_TILE + 2);

// The sweep rule by particle, for lattices that keep plane bounds and whose
// x rows fit one block (X a multiple of 32, at most 256: every warp holds
// the 32 sites of one segment of one x row, and an x tile is whole rows);
// IntLattices and ByteLattices of up to 16 slots.  The warp's particles are
// spread over its lanes (particle q of the warp, in site then slot order, on
// lane q % 32) once to draw their choices and once more, after the block has
// every choice, to place them.  A particle's place in its new site follows
// from the choice masks alone: a stayer comes after the site's stayers of
// lower slots; a particle arriving from the minus neighbour after every
// stayer and that neighbour's PLUS movers of lower slots; one arriving from
// the plus neighbour after those and the minus neighbour's PLUS movers and
// its own site's MINUS movers of lower slots (byte_diffusion_1d_dev.cu:
// 199-269 builds the same order site by site).  Each particle is placed by
// the block that owns its new site (halo rows place what moves into the
// tile): an IntLattice particle straight into the destination word, a
// ByteLattice particle into its byte of the site's words assembled in shared
// memory and stored whole after a barrier.  Places past the last slot
// overflow with the same sequence numbers.  Each site clears its words from
// its new content up to the larger of the warp's new bound and the
// destination's old one, and the warp stores its new bound.
template <int BPS, int S, int DIM, int NT>
__global__ void __launch_bounds__(NT, DIM == 0 ? 4 : 3)
    sweep_pp_kernel(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst, const uint8_t *__restrict__ sites,
                    Geometry g, DevTables m, RunState *__restrict__ rs, OverflowEntry *__restrict__ list,
                    uint32_t cap, uint32_t *__restrict__ rx_sites, uint32_t rx_cap,
                    const uint32_t *__restrict__ pb_src, uint32_t *__restrict__ pb_dst)
{
    static_assert(S <= 16, "slot masks and list entries hold 16 slots");
    constexpr int W = SiteWords<BPS, S>::W;
    constexpr int CB = CountBits<S>::value;
    constexpr uint32_t LOW = (1u << S) - 1u;
    constexpr uint32_t OUT = 1u << 16;  // occupancy word flag: the block writes this site
    // Dynamic shared memory (sweep_pp_smem bytes):
    //   sw[W][NT]  words of the tile's sites, planes below the bound
    //   sc[NT]     choices: bit k MINUS, bit S + k PLUS for slot k
    //   so[NT]     occupied slots, | OUT for written sites
    //   pl[NT * S] each warp's particles in site, then slot order: lane << 4 | slot
    //   ow[W][NT]  (ByteLattices) the written sites' new words
    extern __shared__ uint32_t smem_pp[];
    uint32_t(*sw)[NT] = reinterpret_cast<uint32_t(*)[NT]>(smem_pp);
    uint32_t *sc = smem_pp + W * NT;
    uint32_t *so = sc + NT;
    uint16_t *pl = reinterpret_cast<uint16_t *>(so + NT);
    uint32_t(*ow)[NT] = reinterpret_cast<uint32_t(*)[NT]>(pl + NT * S);
    chain_enter();
    // Checked before the first write, loaded with everything else (as in
    // sweep_kernel).
    const int32_t status = rs->status;
    const bool listing = DIM == 2 && rx_sites && rs->rx_skip == 0;
    uint32_t x, y, z;
    bool in, out;
    sweep_site_of<DIM>(g, x, y, z, in, out);
    const int lid = (int)(threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z));
    const uint32_t lane = (uint32_t)lid & 31u;
    uint32_t i = 0, im = 0, ip = 0;
    int lm = -1, lp = -1;
    uint32_t t = 0, tm = 0, tp = 0, occ = 0;
    const unsigned long long th = rs->th[DIM];
    // The destination's old plane bound, loaded here rather than where it is
    // used, so that its round trip to L2 (the previous sweep wrote it from
    // another SM) is not on the critical path of the warp's tail; no other
    // warp writes it.
    uint32_t old_pb = 0;
    // Occupied slots of word k of a site.
    auto word_slots = [](uint32_t v, uint32_t k) -> uint32_t {
        if (BPS == 4) return (v != 0u ? 1u : 0u) << k;
        const uint32_t hi = (v | ((v & 0x7F7F7F7Fu) + 0x7F7F7F7Fu)) & 0x80808080u;
        return ((((hi >> 7) * 0x10204080u) >> 28) & 0xFu) << (4 * k);
    };
    if (in) {
        sweep_neighbours<DIM>(g, x, y, z, lid, i, im, ip, lm, lp);
        // Planes 0 and 1 are read with the bound rather than after it (a
        // plane at or above the bound reads as zero, so the early read is
        // harmless): nearly every segment needs plane 0 and most plane 1,
        // and the bound's round trip no longer comes first.
        constexpr uint32_t EARLY = W < 2 ? W : 2;
        const uint32_t npl = planes_at<W>(pb_src, i);
        uint32_t v[EARLY];
#pragma unroll
        for (uint32_t k = 0; k < EARLY; k++) v[k] = __ldg(src + (size_t)k * g.N + i);
        t = __ldg(sites + i);
        tm = __ldg(sites + im);
        tp = __ldg(sites + ip);
        if (out) old_pb = pb_dst[i >> PB_SHIFT];
#pragma unroll
        for (uint32_t k = 0; k < EARLY; k++) {
            sw[k][lid] = v[k];
            occ |= word_slots(v[k], k);
        }
        for (uint32_t k = EARLY; k < npl; k++) {
            const uint32_t vk = __ldg(src + (size_t)k * g.N + i);
            sw[k][lid] = vk;
            occ |= word_slots(vk, k);
        }
    }
    if (status != LMB_OK) return;  // the same for the whole block
    so[lid] = occ | (out ? OUT : 0u);
    sc[lid] = 0;
    if (BPS == 1) {
#pragma unroll
        for (int k = 0; k < W; k++) ow[k][lid] = 0u;
    }
    __syncwarp();
    // The warp's particles: prefix counts over the lanes' sites.
    const uint32_t wbase = (uint32_t)lid & ~31u;
    const uint32_t cnt = __popc(occ);
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t vv = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += vv;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31), excl = incl - cnt;
    uint16_t *wpl = pl + wbase * S;
    {
        uint32_t q = excl;
        for (uint32_t mb = occ; mb; mb &= mb - 1) wpl[q++] = (uint16_t)((lane << 4) | (__ffs(mb) - 1));
    }
    __syncwarp();
    // Particle q of the warp: its site's lane and its slot (lane 0, slot 0
    // past the last particle).
    auto particle = [&](uint32_t q, uint32_t &o, uint32_t &k) {
        const uint32_t e = q < total ? wpl[q] : 0u;
        o = e >> 4;
        k = e & 15u;
    };
    // The particle in slot k of tile site sl.
    auto slot_value = [&](uint32_t sl, uint32_t k) -> uint32_t {
        if (BPS == 4) return sw[k][sl];
        return (sw[k >> 2][sl] >> (8u * (k & 3u))) & 0xFFu;
    };
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t q = base + lane;
        uint32_t o, k;
        particle(q, o, k);
        const uint32_t t_o = __shfl_sync(0xffffffffu, t, o), tm_o = __shfl_sync(0xffffffffu, tm, o);
        const uint32_t tp_o = __shfl_sync(0xffffffffu, tp, o), gi_o = __shfl_sync(0xffffffffu, i, o);
        if (q < total) {
            const uint32_t sl = wbase + o;
            const uint32_t p = slot_value(sl, k);
            const float rv = hash_float(((unsigned long long)gi_o << CB) | k, th);
            // PLUS when 0.5 <= r < q(t -> tp) + 0.5, else MINUS when r <
            // q(t -> tm).  Every q is at most 0.5 (larger ones are refused
            // when a model is built), so a draw of 0.5 or more cannot move
            // MINUS and each particle needs one table entry.
            const bool hi = rv >= 0.5f;
            const float qv = lookup_T(m, p, t_o, hi ? tp_o : tm_o);
            uint32_t bit = 0;
            if (hi) {
                if (rv < __fadd_rn(qv, 0.5f)) bit = 1u << (S + k);
            } else if (rv < qv) {
                bit = 1u << k;
            }
            if (bit) atomicOr(&sc[sl], bit);
        }
    }
    __syncthreads();
    // Tile neighbours of tile site l at x coordinate xl (x tiles are whole
    // rows, periodic; y and z tiles are 32 sites wide).
    auto xminus = [&](uint32_t xl) { return xl == 0 ? g.X - 1 : xl - 1; };
    auto xplus = [&](uint32_t xl) { return xl == g.X - 1 ? 0 : xl + 1; };
    auto tile_minus = [&](uint32_t l, uint32_t xl) -> uint32_t {
        if (DIM == 0) return l - xl + xminus(xl);
        return l - 32u;
    };
    auto tile_plus = [&](uint32_t l, uint32_t xl) -> uint32_t {
        if (DIM == 0) return l - xl + xplus(xl);
        return l + 32u;
    };
    auto stays = [&](uint32_t l) { return so[l] & ~(sc[l] | (sc[l] >> S)) & LOW; };
    // Place every particle whose new site this block writes.
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t q = base + lane;
        uint32_t o, k;
        particle(q, o, k);
        const uint32_t gi_o = __shfl_sync(0xffffffffu, i, o), im_o = __shfl_sync(0xffffffffu, im, o);
        const uint32_t ip_o = __shfl_sync(0xffffffffu, ip, o);
        const uint32_t x_o = DIM == 0 ? __shfl_sync(0xffffffffu, x, o) : 0u;
        if (q < total) {
            const uint32_t sl = wbase + o;
            const uint32_t c = sc[sl];
            const uint32_t below = (1u << k) - 1u;
            const uint32_t plus = (c >> (S + k)) & 1u, minus = (c >> k) & 1u;
            // New site in the tile; a y or z tile's halo rows move particles
            // out of the tile as well, which other blocks place.
            const uint32_t row = sl >> 5, rows = DIM == 1 ? blockDim.y : blockDim.z;
            const bool inside = DIM == 0 || !((plus && row + 1u >= rows) || (minus && row == 0));
            const uint32_t d = plus ? tile_plus(sl, x_o) : (minus ? tile_minus(sl, x_o) : sl);
            if (inside && (so[d] & OUT)) {
                uint32_t gd, pos;
                if (plus) {  // after the new site's stayers
                    gd = ip_o;
                    pos = __popc(stays(d)) + __popc((c >> S) & below);
                } else if (minus) {  // after its stayers and the PLUS arrivals from its minus side
                    gd = im_o;
                    pos = __popc(stays(d)) + __popc((sc[tile_minus(d, xminus(x_o))] >> S) & LOW) +
                          __popc(c & below);
                } else {
                    gd = gi_o;
                    pos = __popc(stays(sl) & below);
                }
                const uint32_t p = slot_value(sl, k);
                if (pos >= (uint32_t)S) push_overflow(rs, list, cap, (uint32_t)DIM + 1, gd, pos - (uint32_t)S, p);
                else if (BPS == 4) dst[(size_t)pos * g.N + gd] = p;
                else reinterpret_cast<uint8_t *>(&ow[pos >> 2][d])[pos & 3u] = (uint8_t)p;
            }
        }
    }
    if (BPS == 1) __syncthreads();  // every byte of the written sites placed
    if (!out) return;
    // The site's new count: its stayers and both neighbours' arrivals.
    const uint32_t n = __popc(stays((uint32_t)lid)) + __popc((sc[tile_minus((uint32_t)lid, x)] >> S) & LOW) +
                       __popc(sc[tile_plus((uint32_t)lid, x)] & LOW);
    const uint32_t held = n < (uint32_t)S ? n : (uint32_t)S;  // particles the site holds
    const uint32_t nw = BPS == 4 ? held : (held + 3u) >> 2;    // words they fill
    const uint32_t wmax = __reduce_max_sync(0xffffffffu, nw);
    const uint32_t seg = i >> PB_SHIFT;
    const uint32_t lim = wmax > old_pb ? wmax : (old_pb < (uint32_t)W ? old_pb : (uint32_t)W);
    if (BPS == 4) {
        for (uint32_t k = nw; k < lim; k++) dst[(size_t)k * g.N + i] = 0u;
    } else {
        for (uint32_t k = 0; k < lim; k++) dst[(size_t)k * g.N + i] = k < nw ? ow[k][lid] : 0u;
    }
    __syncwarp();
    if (lane == 0) pb_dst[seg] = wmax;
    if (listing) list_for_reaction(held, t, i, lid, react_bound(t, m), rs->th[3], rs, rx_sites, rx_cap);
}

// ---------------------------------------------------------------------------
// Reaction
// ---------------------------------------------------------------------------

template <int BPS, int S>
__global__ void __launch_bounds__(256) reaction_kernel(uint32_t *__restrict__ lat, const uint8_t *__restrict__ sites,
                                                       Geometry g, DevTables m, RunState *__restrict__ rs,
                                                       OverflowEntry *__restrict__ list, uint32_t cap,
                                                       const uint32_t *__restrict__ rx_sites, uint32_t rx_cap,
                                                       uint32_t *__restrict__ pb)
{
    constexpr int W = SiteWords<BPS, S>::W;
    chain_enter();
    // The status, the list's state and the hash in one round trip.
    const int32_t status = rs->status;
    const uint32_t rx_skip = rs->rx_skip, rx_count = rs->rx_count;
    if (status != LMB_OK) return;
    // The sites the z sweep listed, or every site when it listed none or
    // more than the list holds.
    const uint32_t listed = rx_sites && rx_skip == 0 ? rx_count : 0xFFFFFFFFu;
    const bool all = listed > rx_cap;
    const uint32_t n = all ? g.N : listed;
    const unsigned long long th = rs->th[3];
    // Listed sites go round the blocks (entry j to block j % gridDim.x), so
    // that the few thousand entries spread over every SM; a pass over every
    // site keeps neighbouring sites on neighbouring lanes.
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t j0 = all ? blockIdx.x * blockDim.x + threadIdx.x : threadIdx.x * gridDim.x + blockIdx.x;
    for (uint32_t j = j0; j < n; j += stride) {
        // The z sweep wrote this buffer, so its sites are packed (occupied
        // slots first, whatever the input had): only the planes holding
        // particles are read.
        uint32_t i, t;
        SiteWords<BPS, S> s;
        if (all) {
            i = j;
            t = __ldg(sites + i);
            if (pb) s.load_first(lat, g.N, i, planes_at<W>(pb, i));
            else s.load_packed(lat, g.N, i);
        } else {
            const uint2 e = reinterpret_cast<const uint2 *>(rx_sites)[j];
            const uint32_t np = e.y & 0xFFu;
            i = e.x;
            t = e.y >> 8;
            s.load_first(lat, g.N, i, BPS == 1 ? (np + 3u) / 4u : np);
        }
        if (react_site<BPS, S, 0>(s, t, i, th, m, rs, list, cap)) {
            s.store(lat, g.N, i);
            if (pb) {
                // Products may fill slots above the segment's bound.
                const uint32_t n = (uint32_t)__popc(occupied_slots<BPS, S>(s));
                if (n) cover_slot<BPS>(pb, i, n - 1u);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Overflow resolution (one block; the logic is in lmb_overflow.cuh)
// ---------------------------------------------------------------------------

constexpr int RESOLVE_THREADS = 512;

template <int BPS, int S>
__global__ void __launch_bounds__(RESOLVE_THREADS) resolve_kernel(uint32_t *__restrict__ lat,
                                                                  const uint8_t *__restrict__ sites, Geometry g,
                                                                  RunState *__restrict__ rs,
                                                                  OverflowEntry *__restrict__ list, uint32_t cap,
                                                                  uint32_t rx_cap, uint32_t *__restrict__ pb)
{
    extern __shared__ OverflowEntry sh[];
    chain_enter();
    if (rs->status != LMB_OK) return;
    // The reaction step of this timestep has read its site list.  A list
    // that overflowed is not built for the next 31 timesteps (the reaction
    // step visits every site meanwhile; either way the result is the same).
    if (threadIdx.x == 0) {
        if (rs->rx_skip) rs->rx_skip--;
        else if (rs->rx_count > rx_cap) rs->rx_skip = 31;
        rs->rx_count = 0;
    }
    resolve_block<BPS, S>(lat, sites, g, rs, list, cap, sh, pb);
}

// Sets the run state for a new run without a host round trip.  The relaxed
// handler's queue survives across runs; the classic one starts empty.
__global__ void begin_run_kernel(RunState *rs, uint32_t seed, uint32_t first, uint32_t n, uint32_t mode,
                                 uint32_t count_step, uint32_t count_ns, unsigned long long *counts)
{
    rs->count_step = count_step;
    rs->count_ns = count_ns;
    rs->counts = counts;
    rs->seed = seed;
    set_step(rs, seed, first);
    rs->end_step = first + n;
    rs->status = LMB_OK;
    rs->failed_step = 0;
    rs->mode = mode;
    rs->overflows = 0;
    rs->reactions = 0;
    rs->tiles_done = 0;
    rs->rx_count = 0;
    rs->rx_skip = 0;
    if (mode == LMB_OVERFLOW_CLASSIC) {
        rs->ovf_count = 0;
        rs->carried = 0;
    }
}

// A run whose lattice holds a species id above ns or a site type of nst or
// more (validate_kernel's maxima) fails before its first timestep with
// LMB_E_ARG, as the host check of a synchronous run refuses it.
__global__ void check_contents_kernel(RunState *rs, uint32_t ns, uint32_t nst)
{
    if (rs->max_species > ns || rs->max_site_type >= nst) {
        rs->status = LMB_E_ARG;
        rs->failed_step = rs->step;
    }
}

cudaError_t launch_check_contents(RunState *rs, uint32_t ns, uint32_t nst, cudaStream_t stream)
{
    count_launch();
    check_contents_kernel<<<1, 1, 0, stream>>>(rs, ns, nst);
    return cudaGetLastError();
}

__global__ void fill_bounds_kernel(uint32_t *pb, uint32_t count, uint32_t planes)
{
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) pb[j] = planes;
}

// Batch forms: run state j lives at *rs_ptrs[j]; seeds[j] is its seed.
// Run state of every lattice of a batch: timesteps first .. first + n - 1, or
// per-lattice ranges firsts[j] / counts[j] when those arrays are given.
__global__ void begin_batch_kernel(RunState *const *rs_ptrs, const uint32_t *seeds, uint32_t count, uint32_t first,
                                   uint32_t n, const uint32_t *firsts, const uint32_t *counts, uint32_t mode)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    RunState *rs = rs_ptrs[j];
    const uint32_t f = firsts ? firsts[j] : first;
    rs->count_step = ~0u;
    rs->seed = seeds[j];
    set_step(rs, seeds[j], f);
    rs->end_step = f + (counts ? counts[j] : n);
    rs->status = LMB_OK;
    rs->failed_step = 0;
    rs->mode = mode;
    rs->overflows = 0;
    rs->reactions = 0;
    rs->tiles_done = 0;
    rs->rx_count = 0;
    rs->rx_skip = 0;
    if (mode == LMB_OVERFLOW_CLASSIC) {
        rs->ovf_count = 0;
        rs->carried = 0;
    }
}

__global__ void gather_states_kernel(RunState *const *rs_ptrs, uint32_t count, RunState *out)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < count) out[j] = *rs_ptrs[j];
}

cudaError_t launch_begin_batch(RunState *const *rs_ptrs, const uint32_t *seeds, uint32_t count, uint32_t first,
                               uint32_t n, const uint32_t *firsts, const uint32_t *counts, uint32_t mode,
                               cudaStream_t stream)
{
    count_launch();
    begin_batch_kernel<<<(count + 127) / 128, 128, 0, stream>>>(rs_ptrs, seeds, count, first, n, firsts, counts,
                                                                mode);
    return cudaGetLastError();
}

cudaError_t launch_gather_states(RunState *const *rs_ptrs, uint32_t count, RunState *out, cudaStream_t stream)
{
    count_launch();
    gather_states_kernel<<<(count + 127) / 128, 128, 0, stream>>>(rs_ptrs, count, out);
    return cudaGetLastError();
}

cudaError_t launch_fill_bounds(uint32_t *pb, uint32_t count, uint32_t planes, cudaStream_t stream)
{
    uint32_t blocks = (count + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    if (blocks == 0) return cudaSuccess;
    count_launch();
    fill_bounds_kernel<<<blocks, 256, 0, stream>>>(pb, count, planes);
    return cudaGetLastError();
}

cudaError_t launch_begin_run(RunState *rs, uint32_t seed, uint32_t first, uint32_t n, uint32_t mode,
                             cudaStream_t stream, uint32_t count_step, uint32_t count_ns, unsigned long long *counts)
{
    count_launch();
    begin_run_kernel<<<1, 1, 0, stream>>>(rs, seed, first, n, mode, count_step, count_ns, counts);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Counts, validation, layout conversion
// ---------------------------------------------------------------------------

template <int BPS, int S>
__global__ void counts_kernel(const uint32_t *__restrict__ lat, Geometry g, uint32_t ns,
                              unsigned long long *__restrict__ counts, const uint32_t *__restrict__ pb)
{
    constexpr int W = SiteWords<BPS, S>::W;
    extern __shared__ unsigned int hist[];
    const bool use_shared = ns + 1 <= 8192;
    if (use_shared)
        for (uint32_t s = threadIdx.x; s <= ns; s += blockDim.x) hist[s] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g.N; i += gridDim.x * blockDim.x) {
        SiteWords<BPS, S> s;
        s.load_planes(lat, g.N, i, planes_at<W>(pb, i));
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
    if (rm) {
        SiteWords<BPS, S> s;
        s.load(native, g.N, i);
#pragma unroll
        for (int k = 0; k < S; k++) {
            if (BPS == 1) ((uint8_t *)rm)[r * S + k] = (uint8_t)s.slot(k);
            else ((uint32_t *)rm)[r * S + k] = s.slot(k);
        }
    }
    if (rm_sites) rm_sites[r] = sites[i];
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------

// Tiles long along the sweep axis: whole x rows (up to 256 sites) for x; for
// y and z, 32 x 8 sites in the x-y or x-z plane (wider when the axis is
// shorter than 8) launched with one halo row of threads on either side.
// Every block is a whole number of warps.
static void sweep_shape(const Geometry &g, int dim, dim3 &grid, dim3 &block)
{
    const uint32_t xw = ((g.X + 31) / 32) * 32;
    if (dim == 0) {
        const uint32_t bx = xw > 256 ? 256 : xw;
        uint32_t by = 256 / bx;
        if (by > g.Y) by = g.Y;
        block = dim3(bx, by, 1);
        grid = dim3((g.X + bx - 1) / bx, (g.Y + by - 1) / by, g.Z);
        return;
    }
    const uint32_t A = dim == 1 ? g.Y : g.Z;
    const uint32_t L = A < 8 ? A : 8;
    uint32_t bx = (SWEEP_MAX_THREADS / (L + 2)) & ~31u;
    if (bx > xw) bx = xw;
    if (dim == 1) {
        block = dim3(bx, L + 2, 1);
        grid = dim3((g.X + bx - 1) / bx, (g.Y + L - 1) / L, g.Z);
    } else {
        block = dim3(bx, 1, L + 2);
        grid = dim3((g.X + bx - 1) / bx, g.Y, (g.Z + L - 1) / L);
    }
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

// Dynamic shared memory of sweep_pp_kernel<BPS, S, *, NT>.
static size_t sweep_pp_smem(int BPS, int S, int NT)
{
    const size_t W = BPS == 1 ? (size_t)S / 4 : (size_t)S;
    return (size_t)NT * (W * 4 + 8 + (size_t)S * 2 + (BPS == 1 ? W * 4 : 0));
}

// Raises kernel K's dynamic shared-memory limit once per device to the
// largest size asked for so far (setting it on every launch costs host time).
// One cache per kernel: instantiations share a function type, not a limit.
template <auto K>
static cudaError_t raise_smem_limit(size_t bytes)
{
    static size_t granted[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (bytes <= 48 * 1024 || bytes <= granted[dev]) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    // The whole unified L1 / shared array as shared memory, so that as many
    // blocks fit as the registers allow.
    if (e == cudaSuccess) e = cudaFuncSetAttribute(K, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e == cudaSuccess) granted[dev] = bytes;
    return e;
}

cudaError_t launch_sweep(int bps, int slots, int dim, const uint32_t *src, uint32_t *dst, const uint8_t *sites,
                         const Geometry &g, const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                         uint32_t *rx_sites, uint32_t rx_cap, const uint32_t *pb_src, uint32_t *pb_dst,
                         cudaStream_t stream)
{
    dim3 grid, block;
    sweep_shape(g, dim, grid, block);
    // Plane bounds need each warp on one whole segment of 32 sites.
    if (g.X % 32u != 0) pb_src = pb_dst = nullptr;
    if (!pb_src || !pb_dst) pb_src = pb_dst = nullptr;
    if (pb_src && g.X <= (uint32_t)SWEEP_THREADS && slots <= 16 && (bps == 4 || slots >= 4)) {
        // Plane-bounded lattices whose rows fit a block: by particle, y and z
        // tiles of SWEEP_PB_TILE sites along the axis, one segment across.
        if (dim != 0) {
            const uint32_t A = dim == 1 ? g.Y : g.Z;
            const uint32_t L = A < (uint32_t)SWEEP_PB_TILE ? A : (uint32_t)SWEEP_PB_TILE;
            if (dim == 1) {
                block = dim3(32, L + 2, 1);
                grid = dim3(g.X / 32, (g.Y + L - 1) / L, g.Z);
            } else {
                block = dim3(32, 1, L + 2);
                grid = dim3(g.X / 32, g.Y, (g.Z + L - 1) / L);
            }
        }
        count_launch();
        constexpr int YZ = SWEEP_PB_YZ_THREADS;
        cudaError_t e;
#define LMB_PP_SWEEP(BPS_, S_)                                                                                     \
    if (bps == BPS_ && slots == S_) {                                                                             \
        if (dim == 0) {                                                                                           \
            const size_t sm = sweep_pp_smem(BPS_, S_, SWEEP_THREADS);                                             \
            if ((e = raise_smem_limit<sweep_pp_kernel<BPS_, S_, 0, SWEEP_THREADS>>(sm)) != cudaSuccess) return e;  \
            e = launch_chain(sweep_pp_kernel<BPS_, S_, 0, SWEEP_THREADS>, grid, block, sm, stream, src, dst, sites, \
                             g, m, rs, list, cap, nullptr, 0u, pb_src, pb_dst);                                   \
        } else if (dim == 1) {                                                                                    \
            const size_t sm = sweep_pp_smem(BPS_, S_, YZ);                                                        \
            if ((e = raise_smem_limit<sweep_pp_kernel<BPS_, S_, 1, YZ>>(sm)) != cudaSuccess) return e;            \
            e = launch_chain(sweep_pp_kernel<BPS_, S_, 1, YZ>, grid, block, sm, stream, src, dst, sites, g, m, rs, \
                             list, cap, nullptr, 0u, pb_src, pb_dst);                                             \
        } else {                                                                                                  \
            const size_t sm = sweep_pp_smem(BPS_, S_, YZ);                                                        \
            if ((e = raise_smem_limit<sweep_pp_kernel<BPS_, S_, 2, YZ>>(sm)) != cudaSuccess) return e;            \
            e = launch_chain(sweep_pp_kernel<BPS_, S_, 2, YZ>, grid, block, sm, stream, src, dst, sites, g, m, rs, \
                             list, cap, rx_sites, rx_cap, pb_src, pb_dst);                                        \
        }                                                                                                         \
        return e;                                                                                                 \
    }
        LMB_PP_SWEEP(4, 4)
        LMB_PP_SWEEP(4, 8)
        LMB_PP_SWEEP(4, 16)
        LMB_PP_SWEEP(1, 4)
        LMB_PP_SWEEP(1, 8)
        LMB_PP_SWEEP(1, 16)
#undef LMB_PP_SWEEP
        return cudaErrorInvalidValue;
    }
    count_launch();
    LMB_DISPATCH_ALL({
        if (dim == 0)
            return launch_chain(sweep_kernel<BPS, S, 0>, grid, block, 0, stream, src, dst, sites, g, m, rs, list, cap,
                                nullptr, 0u, pb_src, pb_dst);
        else if (dim == 1)
            return launch_chain(sweep_kernel<BPS, S, 1>, grid, block, 0, stream, src, dst, sites, g, m, rs, list, cap,
                                nullptr, 0u, pb_src, pb_dst);
        else
            return launch_chain(sweep_kernel<BPS, S, 2>, grid, block, 0, stream, src, dst, sites, g, m, rs, list, cap,
                                rx_sites, rx_cap, pb_src, pb_dst);
    })
}

// A grid of at most 8 blocks per SM strides over the listed sites (or every
// site); the full pass keeps as many threads resident as one thread per site
// would.
cudaError_t launch_reaction(int bps, int slots, uint32_t *lat, const uint8_t *sites, const Geometry &g,
                            const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                            const uint32_t *rx_sites, uint32_t rx_cap, uint32_t *pb, cudaStream_t stream)
{
    // One wave: four blocks per SM fit every instantiation's registers.
    const uint32_t threads = 256;
    uint32_t blocks = (g.N + threads - 1) / threads;
    if (blocks > 148 * 4) blocks = 148 * 4;
    if (g.X % 32u != 0) pb = nullptr;
    count_launch();
    LMB_DISPATCH_ALL(return launch_chain(reaction_kernel<BPS, S>, dim3(blocks), dim3(threads), 0, stream, lat, sites,
                                         g, m, rs, list, cap, rx_sites, rx_cap, pb))
}

cudaError_t launch_resolve(int bps, int slots, uint32_t *lat, const uint8_t *sites, const Geometry &g, RunState *rs,
                           OverflowEntry *list, uint32_t cap, uint32_t rx_cap, uint32_t *pb, cudaStream_t stream)
{
    if (g.X % 32u != 0) pb = nullptr;
    uint32_t pow2 = 1;
    while (pow2 < cap) pow2 <<= 1;
    const size_t smem = (size_t)pow2 * sizeof(OverflowEntry);
    count_launch();
    LMB_DISPATCH_ALL({
        static bool raised[64] = {false};
        int dev = 0;
        cudaGetDevice(&dev);
        if (smem > 48 * 1024 && dev >= 0 && dev < 64 && !raised[dev]) {
            cudaFuncSetAttribute(resolve_kernel<BPS, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            raised[dev] = true;
        }
        return launch_chain(resolve_kernel<BPS, S>, dim3(1), dim3(RESOLVE_THREADS), smem, stream, lat, sites, g, rs,
                            list, cap, rx_cap, pb);
    })
}

cudaError_t launch_counts(int bps, int slots, const uint32_t *lat, const Geometry &g, uint32_t ns,
                          unsigned long long *counts, cudaStream_t stream, const uint32_t *pb)
{
    const uint32_t threads = 256;
    uint32_t blocks = (g.N + threads - 1) / threads;
    if (blocks > 148 * 8) blocks = 148 * 8;
    const size_t smem = ns + 1 <= 8192 ? (ns + 1) * sizeof(unsigned int) : 0;
    count_launch();
    LMB_DISPATCH_ALL(counts_kernel<BPS, S><<<blocks, threads, smem, stream>>>(lat, g, ns, counts, pb))
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
