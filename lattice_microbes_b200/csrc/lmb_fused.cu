// lmb_fused.cu -- one launch per MPD timestep: x, y, z sweeps and the
// reaction of a tile of full x-rows, staged in shared memory.
//
// A block owns Ty x Tz full rows (all x) of the lattice.  It loads the owned
// rows plus one halo row on each side in y and z (periodic wrap) into shared
// memory once, then
//   x sweep over every loaded row (x neighbours are in the same row),
//   y sweep over the owned y rows of every loaded z plane,
//   z sweep over the owned rows, followed in registers by the reaction,
// and writes the owned rows once.  Versus the reference schedule (three
// sweep kernels and a reaction kernel, each reading and writing the whole
// lattice) this reads the lattice once (plus halo rows, which neighbouring
// blocks also read and L2 serves) and writes it once per timestep.
//
// Halo rows are recomputed by several blocks; every decision is a pure
// function of (seed, step, site, slot, site types), so the copies agree, and
// only the owner of a site queues its overflows.  The last block of a launch
// to finish resolves the overflow queue (lmb_overflow.cuh), so a timestep is a
// single launch.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "lmb.h"
#include "lmb_device.cuh"
#include "lmb_fused.h"
#include "lmb_internal.h"
#include "lmb_overflow.cuh"
#include "lmb_site.cuh"

namespace lmb {

template <int BPS, int S>
__device__ __forceinline__ void load_smem(const uint32_t *buf, uint32_t R, uint32_t l, SiteWords<BPS, S> &s)
{
#pragma unroll
    for (int k = 0; k < SiteWords<BPS, S>::W; k++) s.w[k] = buf[(size_t)k * R + l];
}

template <int BPS, int S>
__device__ __forceinline__ void store_smem(uint32_t *buf, uint32_t R, uint32_t l, const SiteWords<BPS, S> &s)
{
#pragma unroll
    for (int k = 0; k < SiteWords<BPS, S>::W; k++) buf[(size_t)k * R + l] = s.w[k];
}

// Copies the model tables into shared memory at `dst` (16-byte aligned;
// stage_bytes long, each table at a 16-byte boundary) and returns a table set
// pointing there.  The device tables sit at 256-byte boundaries of one block
// (zero padded), so the copy moves whole 16-byte granules, every thread's
// loads independent of each other.
constexpr int NTABLES = 15;
__device__ __forceinline__ DevTables stage_tables(const DevTables &m, uint8_t *dst, uint32_t tid, uint32_t nthr)
{
    DevTables s = m;
    const void *srcs[NTABLES] = {m.T, m.qp0, m.qp1, m.qp2, m.order, m.D1, m.D2, m.rate, m.RL, m.stoich_off,
                                 m.stoich_sp, m.stoich_d, m.qpmax, m.rx_off, m.rx_list};
    const uint32_t sizes[NTABLES] = {m.nst * m.nst * m.ns * 4, m.nst * 4, m.nst * m.ns * 4,
                                     m.nst * m.ns * m.ns * 4, m.nr * 4, m.nr * 4, m.nr * 4, m.nr * 4,
                                     m.nr * m.nst, (m.nr + 1) * 4, m.nnz * 4, m.nnz * 4, 2 * m.nst * 4,
                                     (m.ns + 2) * 4, m.nr * 4};
    uint32_t first[NTABLES + 1];
    first[0] = 0;
#pragma unroll
    for (int k = 0; k < NTABLES; k++) first[k + 1] = first[k] + (sizes[k] + 15u) / 16u;
    uint4 *out = (uint4 *)dst;
    for (uint32_t gr = tid; gr < first[NTABLES]; gr += nthr) {
        const uint4 *src = (const uint4 *)srcs[0];
        uint32_t f = 0;
#pragma unroll
        for (int j = 1; j < NTABLES; j++)
            if (gr >= first[j]) {
                src = (const uint4 *)srcs[j];
                f = first[j];
            }
        out[gr] = __ldg(src + (gr - f));
    }
    const void *outs[NTABLES];
#pragma unroll
    for (int k = 0; k < NTABLES; k++) outs[k] = dst + 16u * first[k];
    s.T = (const float *)outs[0];
    s.qp0 = (const float *)outs[1];
    s.qp1 = (const float *)outs[2];
    s.qp2 = (const float *)outs[3];
    s.order = (const uint32_t *)outs[4];
    s.D1 = (const uint32_t *)outs[5];
    s.D2 = (const uint32_t *)outs[6];
    s.rate = (const float *)outs[7];
    s.RL = (const uint8_t *)outs[8];
    s.stoich_off = (const uint32_t *)outs[9];
    s.stoich_sp = (const uint32_t *)outs[10];
    s.stoich_d = (const int32_t *)outs[11];
    s.qpmax = (const float *)outs[12];
    s.rx_off = (const uint32_t *)outs[13];
    s.rx_list = (const uint32_t *)outs[14];
    return s;
}

template <int BPS, int S>
__device__ __noinline__ SiteWords<BPS, S> react_site_ool(SiteWords<BPS, S> s, uint32_t t, uint32_t gi,
                                                         unsigned long long th, const DevTables &m, RunState *rs,
                                                         OverflowEntry *list, uint32_t cap)
{
    react_site<BPS, S, 8>(s, t, gi, th, m, rs, list, cap);
    return s;
}

// Row flags of the loaded region.
constexpr uint8_t ROW_OWNED = 1;

// Bit x of the result is set when site x or one of its x neighbours (periodic
// in the row of X sites) is occupied; `row` holds the row's MW mask words.
__device__ __forceinline__ uint32_t x_neighbourhood(const uint32_t *row, uint32_t w, uint32_t MW, uint32_t X)
{
    const uint32_t cur = row[w];
    const uint32_t prev = w > 0 ? row[w - 1] : 0u, next = w + 1 < MW ? row[w + 1] : 0u;
    uint32_t a = cur | (cur << 1) | (cur >> 1) | (prev >> 31) | (next << 31);
    // Periodic ends: x = 0 sees x = X - 1 and the other way round.
    const uint32_t last_bit = (X - 1) & 31u, last_word = (X - 1) >> 5;
    if (w == 0 && ((row[last_word] >> last_bit) & 1u)) a |= 1u;
    if (w == last_word && (row[0] & 1u)) a |= 1u << last_bit;
    const uint32_t valid = (w == last_word && (X & 31u)) ? ((1u << (X & 31u)) - 1u) : 0xffffffffu;
    return a & valid;
}

// Warp-cooperative list append: every lane of the warp calls this with its
// mask word (0 if none); entries (row << 16 | x) land contiguously in `work`
// with one shared atomic per warp.
__device__ __forceinline__ void warp_append(uint32_t b, uint32_t r, uint32_t w, uint32_t *work, uint32_t *count)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n = __popc(b);
    uint32_t incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    if (total == 0) return;
    uint32_t base = 0;
    if (lane == 31) base = atomicAdd(count, total);
    base = __shfl_sync(0xffffffffu, base, 31) + incl - n;
    while (b) {
        const uint32_t k = __ffs(b) - 1;
        b &= b - 1;
        work[base++] = (r << 16) | (w * 32 + k);
    }
}

// Shared-memory layout of a tile: A[W][R], B[W][R] particle words (valid
// where the occupancy bit is set), work[R] site list, T[R] site types, then
// occA / occB [rows * MW] occupancy bit masks and the staged model tables;
// per region row its lattice index of x = 0 and flags, and the region rows
// the y and z sweeps produce.  Filled once: no sweep divides.
struct TileSmem {
    uint32_t *A, *B, *work;
    uint8_t *T;
    uint32_t *occA, *occB;
    uint8_t *tables;
    uint32_t *rowbase;
    uint16_t *yrow, *zrow;
    uint8_t *rowflag;
    uint32_t *cnt;
};

template <int BPS, int S>
__device__ __forceinline__ TileSmem tile_smem(uint32_t *smem, const TileShape &ts, uint32_t *rowbase, uint16_t *yrow,
                                              uint16_t *zrow, uint8_t *rowflag, uint32_t *cnt)
{
    constexpr int W = SiteWords<BPS, S>::W;
    const uint32_t R = ts.R, rows = ts.Ry * ts.Rz, MW = ts.MW;
    TileSmem t;
    t.A = smem;
    t.B = t.A + W * R;
    t.work = t.B + W * R;
    t.T = (uint8_t *)(t.work + R);
    t.occA = (uint32_t *)(t.T + ((R + 15u) & ~15u));
    t.occB = t.occA + rows * MW;
    t.tables = (uint8_t *)(((uintptr_t)(t.occB + rows * MW) + 15u) & ~(uintptr_t)15u);
    t.rowbase = rowbase;
    t.yrow = yrow;
    t.zrow = zrow;
    t.rowflag = rowflag;
    t.cnt = cnt;
    return t;
}

// Row tables of tile `tile` (no barrier).
__device__ __forceinline__ void tile_rows(const Geometry &g, const TileShape &ts, uint32_t tile, const TileSmem &t)
{
    const uint32_t X = g.X, Ry = ts.Ry, Ty = ts.Ty, Tz = ts.Tz, tid = threadIdx.x, nthr = blockDim.x;
    const uint32_t y0 = (tile % ts.tiles_y) * Ty, z0 = (tile / ts.tiles_y) * Tz;
    const uint32_t rows = Ry * ts.Rz, yrows = Ty * ts.Rz, orows = Ty * Tz;
    for (uint32_t r = tid; r < rows; r += nthr) {
        const uint32_t ly = r % Ry, lz = r / Ry;
        t.rowbase[r] = ((y0 + ly + g.Y - 1) % g.Y) * X + ((z0 + lz + g.Z - 1) % g.Z) * g.XY;
        t.rowflag[r] = ly >= 1 && ly <= Ty && lz >= 1 && lz <= Tz ? ROW_OWNED : 0;
    }
    for (uint32_t q = tid; q < yrows; q += nthr) t.yrow[q] = (uint16_t)((q / Ty) * Ry + 1 + q % Ty);
    for (uint32_t q = tid; q < orows; q += nthr) t.zrow[q] = (uint16_t)((1 + q / Ty) * Ry + 1 + q % Ty);
    if (tid < 4) t.cnt[tid] = 0;
}

template <bool CG>
__device__ __forceinline__ uint4 load16(const uint32_t *p)
{
    return CG ? __ldcg((const uint4 *)p) : __ldg((const uint4 *)p);
}

template <bool CG>
__device__ __forceinline__ uint32_t load4(const uint32_t *p)
{
    return CG ? __ldcg(p) : __ldg(p);
}

// Loads region rows of `src` into `w` with their occupancy masks in `occ`:
// every row, or (halo_only) the rows the tile does not own; the site types
// too when `types`.  CG: read through L2 (the rows were written by other
// blocks of the same launch).  Ends with a block barrier.
template <int BPS, int S, bool CG>
__device__ __forceinline__ void tile_load(const uint32_t *__restrict__ src, const uint8_t *__restrict__ sites,
                                          const Geometry &g, const TileShape &ts, const TileSmem &t, uint32_t *w,
                                          uint32_t *occ, bool halo_only, bool types)
{
    constexpr int W = SiteWords<BPS, S>::W;
    const uint32_t X = g.X, R = ts.R, MW = ts.MW, rows = ts.Ry * ts.Rz, tid = threadIdx.x, nthr = blockDim.x;
    if (ts.vec) {
        // 16-byte loads: an item is 4 consecutive sites of one row, read from
        // every word plane (W 16-byte loads), with its 4 occupancy bits OR-ed
        // into the row's mask word.  Up to four items in flight per thread.
        for (uint32_t i = tid; i < rows * MW; i += nthr)
            if (!halo_only || !(t.rowflag[i / MW] & ROW_OWNED)) occ[i] = 0u;
        const uint32_t q4 = X / 4, nq = rows * q4;
        constexpr int U = W >= 4 ? 2 : 8 / W;
        __syncthreads();
        for (uint32_t i0 = tid; i0 < nq; i0 += U * nthr) {
            uint4 v[U][W];
            uint32_t rr[U], cc[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const uint32_t i = i0 + u * nthr;
                rr[u] = ~0u;
                if (i < nq) {
                    const uint32_t r = i / q4, c = i - r * q4;
                    if (halo_only && (t.rowflag[r] & ROW_OWNED)) continue;
                    rr[u] = r;
                    cc[u] = c;
#pragma unroll
                    for (int k = 0; k < W; k++) v[u][k] = load16<CG>(src + (size_t)k * g.N + t.rowbase[r] + 4 * c);
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (rr[u] == ~0u) continue;
                const uint32_t r = rr[u], x = 4 * cc[u];
                uint4 o = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
                for (int k = 0; k < W; k++) {
                    *(uint4 *)(w + k * R + r * X + x) = v[u][k];
                    o.x |= v[u][k].x;
                    o.y |= v[u][k].y;
                    o.z |= v[u][k].z;
                    o.w |= v[u][k].w;
                }
                const uint32_t bits = (o.x ? 1u : 0u) | (o.y ? 2u : 0u) | (o.z ? 4u : 0u) | (o.w ? 8u : 0u);
                if (bits) atomicOr(&occ[r * MW + (x >> 5)], bits << (x & 31u));
            }
        }
        if (types) {
            const uint32_t q16 = X / 16, nt = rows * q16;
            for (uint32_t i = tid; i < nt; i += nthr) {
                const uint32_t r = i / q16, c = i - r * q16;
                *((uint4 *)(t.T + r * X) + c) = __ldg((const uint4 *)(sites + t.rowbase[r]) + c);
            }
        }
    } else {
        // Rows not 16-byte aligned: one word per thread.
        const uint32_t bx = ts.bx, by = nthr / bx, tx = tid % bx, ty = tid / bx;
        for (uint32_t r = ty; r < rows; r += by) {
            if (halo_only && (t.rowflag[r] & ROW_OWNED)) continue;
            const uint32_t gbase = t.rowbase[r];
            for (uint32_t xb = 0; xb < X; xb += bx) {
                const uint32_t x = xb + tx;
                bool o_site = false;
                if (x < X) {
                    const uint32_t l = r * X + x, gi = gbase + x;
                    uint32_t o = 0;
#pragma unroll
                    for (int k = 0; k < W; k++) {
                        const uint32_t v = load4<CG>(src + (size_t)k * g.N + gi);
                        w[k * R + l] = v;
                        o |= v;
                    }
                    if (types) t.T[l] = __ldg(sites + gi);
                    o_site = o != 0;
                }
                const uint32_t mask = __ballot_sync(0xffffffffu, o_site);
                if ((tx & 31u) == 0 && (x >> 5) < MW) occ[r * MW + (x >> 5)] = mask;
            }
        }
    }
    __syncthreads();
}

// One timestep of the tile in shared memory, from (w, o) = the region at the
// start of the timestep; on return (w, o) hold the owned rows after the x,
// y and z sweeps and the reaction (the other rows are stale).  Ends with a
// block barrier.  ROWS: transition-table lookups through rows held in
// registers (TTable) rather than through the table set (TableSet); the two
// give the same values and differ only in register use.
template <int BPS, int S, bool ROWS>
__device__ __forceinline__ void tile_timestep(const Geometry &g, const DevTables &mt, RunState *__restrict__ rs,
                                              OverflowEntry *__restrict__ list, uint32_t cap, const TileShape &ts,
                                              const TileSmem &t, uint32_t *&src_w, uint32_t *&dst_w,
                                              uint32_t *&src_o, uint32_t *&dst_o, uint32_t seed, uint32_t step,
                                              int with_reaction)
{
    const uint32_t X = g.X, R = ts.R, Ry = ts.Ry, Ty = ts.Ty, Tz = ts.Tz, MW = ts.MW;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const uint32_t rows = Ry * ts.Rz, yrows = Ty * ts.Rz, orows = Ty * Tz;
    uint32_t *work = t.work;
    const uint8_t *T = t.T;
    const uint32_t *rowbase = t.rowbase;
    // Models without zeroth-order reactions react only on occupied sites:
    // the reaction then runs in the z sweep's pass, without a pass of its own.
    bool zeroth = false;
    for (uint32_t q = 0; q < mt.nst; q++) zeroth |= mt.qp0[q] != 0.0f;
    const bool react_inline = with_reaction && !zeroth;
    const unsigned long long th_rx = timestep_hash(seed, step, 3);
    using Tables = typename std::conditional<ROWS, TTable, TableSet>::type;
    Tables tabs;
    if constexpr (ROWS) tabs = TTable{mt.T, mt.ns, mt.nst};
    else tabs = TableSet{&mt};
    if (tid < 4) t.cnt[tid] = 0;
    __syncthreads();
#pragma unroll 1
    for (int phase = 0; phase < 3; phase++) {
        const unsigned long long th = timestep_hash(seed, step, (uint32_t)phase);
        const uint16_t *orow = phase == 0 ? nullptr : (phase == 1 ? t.yrow : t.zrow);
        const uint32_t nout = phase == 0 ? rows : (phase == 1 ? yrows : orows);
        const uint32_t d = phase == 1 ? 1u : Ry;  // row step of the y / z neighbours
        uint32_t *cnt = &t.cnt[phase];

        // 1. Active outputs: occupied or next to an occupied site on the axis.
        for (uint32_t i0 = 0; i0 < nout * MW; i0 += nthr) {
            const uint32_t i = i0 + tid;
            uint32_t a = 0, r = 0, w = 0;
            if (i < nout * MW) {
                const uint32_t q = i / MW;
                w = i - q * MW;
                r = orow ? orow[q] : q;
                if (phase == 0) a = x_neighbourhood(src_o + r * MW, w, MW, X);
                else a = src_o[r * MW + w] | src_o[(r - d) * MW + w] | src_o[(r + d) * MW + w];
                dst_o[r * MW + w] = 0u;
            }
            warp_append(a, r, w, work, cnt);
        }
        __syncthreads();

        // 2. The sweep rule for each active output.
        const uint32_t nact = *cnt;
        for (uint32_t j = tid; j < nact; j += nthr) {
            const uint32_t e = work[j], r = e >> 16, x = e & 0xFFFFu, l = r * X + x;
            uint32_t rm = r, rp = r, xm = x, xp = x;
            if (phase == 0) {
                xm = x == 0 ? X - 1 : x - 1;
                xp = x == X - 1 ? 0 : x + 1;
            } else {
                rm = r - d;
                rp = r + d;
            }
            const uint32_t lm = rm * X + xm, lp = rp * X + xp;
            SiteWords<BPS, S> own, mn, pl;
            own.clear();
            mn.clear();
            pl.clear();
            if ((src_o[r * MW + (x >> 5)] >> (x & 31u)) & 1u) load_smem<BPS, S>(src_w, R, l, own);
            if ((src_o[rm * MW + (xm >> 5)] >> (xm & 31u)) & 1u) load_smem<BPS, S>(src_w, R, lm, mn);
            if ((src_o[rp * MW + (xp >> 5)] >> (xp & 31u)) & 1u) load_smem<BPS, S>(src_w, R, lp, pl);
            const bool record = phase == 2 || (t.rowflag[r] & ROW_OWNED);
            own = sweep_site<BPS, S>(own, mn, pl, T[l], T[lm], T[lp], rowbase[r] + x, rowbase[rm] + xm,
                                     rowbase[rp] + xp, th, tabs, record, (uint32_t)phase + 1, rs, list, cap);
            // After the z sweep an owned site reacts right away in
            // registers, when only occupied sites can react.  Its exact
            // early exit is taken here; only a site whose draw may react
            // makes the call.
            if (phase == 2 && react_inline && !own.empty()) {
                const uint32_t gi = rowbase[r] + x, ts = T[l];
                const float r0 = hash_float((unsigned long long)gi << 1, th_rx);
                if (reaction_may_fire((uint32_t)__popc(occupied_slots<BPS, S>(own)), tload(mt.qp0 + ts), ts, r0, mt))
                    own = react_site_ool<BPS, S>(own, ts, gi, th_rx, mt, rs, list, cap);
            }
            if (!own.empty()) {
                store_smem<BPS, S>(dst_w, R, l, own);
                atomicOr(&dst_o[r * MW + (x >> 5)], 1u << (x & 31u));
            }
        }
        __syncthreads();
        uint32_t *t0 = src_w;
        src_w = dst_w;
        dst_w = t0;
        t0 = src_o;
        src_o = dst_o;
        dst_o = t0;
    }
    // After three sweeps the owned rows are in src_w / src_o.

    // Reaction on the owned sites that can react: the occupied ones, or every
    // site when the model has zeroth-order reactions.
    if (with_reaction && !react_inline) {
        const unsigned long long th = th_rx;
        for (uint32_t i0 = 0; i0 < orows * MW; i0 += nthr) {
            const uint32_t i = i0 + tid;
            uint32_t a = 0, r = 0, w = 0;
            if (i < orows * MW) {
                const uint32_t q = i / MW;
                w = i - q * MW;
                r = t.zrow[q];
                const uint32_t all = (w + 1 < MW || !(X & 31u)) ? 0xffffffffu : ((1u << (X & 31u)) - 1u);
                a = zeroth ? all : src_o[r * MW + w];
            }
            warp_append(a, r, w, work, &t.cnt[3]);
        }
        __syncthreads();
        const uint32_t n = t.cnt[3];
        for (uint32_t j = tid; j < n; j += nthr) {
            const uint32_t e = work[j], r = e >> 16, x = e & 0xFFFFu, l = r * X + x;
            const bool occ = (src_o[r * MW + (x >> 5)] >> (x & 31u)) & 1u;
            SiteWords<BPS, S> s;
            s.clear();
            if (occ) load_smem<BPS, S>(src_w, R, l, s);
            else if (mt.qp0[T[l]] == 0.0f) continue;
            s = react_site_ool<BPS, S>(s, T[l], rowbase[r] + x, th, mt, rs, list, cap);
            store_smem<BPS, S>(src_w, R, l, s);
            if (s.empty()) atomicAnd(&src_o[r * MW + (x >> 5)], ~(1u << (x & 31u)));
            else atomicOr(&src_o[r * MW + (x >> 5)], 1u << (x & 31u));
        }
        __syncthreads();
    }
}

// Dense write of the owned rows (empty sites as zeros) from (w, o).
template <int BPS, int S>
__device__ __forceinline__ void tile_store(uint32_t *__restrict__ dst, const Geometry &g, const TileShape &ts,
                                           const TileSmem &t, const uint32_t *w, const uint32_t *o)
{
    constexpr int W = SiteWords<BPS, S>::W;
    const uint32_t X = g.X, R = ts.R, MW = ts.MW, orows = ts.Ty * ts.Tz, tid = threadIdx.x, nthr = blockDim.x;
    if (ts.vec) {
        // Four sites per thread: a 16-byte store per word plane.
        const uint32_t q4 = X / 4, n4 = orows * q4;
        for (uint32_t i = tid; i < n4; i += nthr) {
            const uint32_t q = i / q4, c = i - q * q4, r = t.zrow[q], x = 4 * c;
            const uint32_t bits = (o[r * MW + (x >> 5)] >> (x & 31u)) & 0xFu;
#pragma unroll
            for (int k = 0; k < W; k++) {
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (bits) {
                    const uint32_t *a = w + k * R + r * X + x;
                    v.x = (bits & 1u) ? a[0] : 0u;
                    v.y = (bits & 2u) ? a[1] : 0u;
                    v.z = (bits & 4u) ? a[2] : 0u;
                    v.w = (bits & 8u) ? a[3] : 0u;
                }
                *((uint4 *)(dst + (size_t)k * g.N + t.rowbase[r]) + c) = v;
            }
        }
    } else {
        const uint32_t bx = ts.bx, by = nthr / bx, tx = tid % bx, ty = tid / bx;
        for (uint32_t q = ty; q < orows; q += by) {
            const uint32_t r = t.zrow[q];
            const uint32_t gb = t.rowbase[r];
            for (uint32_t x = tx; x < X; x += bx) {
                SiteWords<BPS, S> s;
                s.clear();
                if ((o[r * MW + (x >> 5)] >> (x & 31u)) & 1u) load_smem<BPS, S>(w, R, r * X + x, s);
                s.store(dst, g.N, gb + x);
            }
        }
    }
}

// Species counts of the tile's owned rows from (w, o), added to counts[0..ns]
// (a species id above ns goes to entry 0): a shared-memory histogram in the
// work list (R >= ns + 1 entries, free after the timestep), then one global
// atomic per species the tile holds.
template <int BPS, int S>
__device__ __forceinline__ void tile_count(const Geometry &g, const TileShape &ts, const TileSmem &t,
                                           const uint32_t *w, const uint32_t *o, uint32_t ns,
                                           unsigned long long *counts)
{
    const uint32_t X = g.X, R = ts.R, MW = ts.MW, orows = ts.Ty * ts.Tz, tid = threadIdx.x, nthr = blockDim.x;
    uint32_t *hist = t.work;
    for (uint32_t b = tid; b <= ns; b += nthr) hist[b] = 0;
    __syncthreads();
    for (uint32_t i = tid; i < orows * X; i += nthr) {
        const uint32_t q = i / X, x = i - q * X, r = t.zrow[q];
        if (!((o[r * MW + (x >> 5)] >> (x & 31u)) & 1u)) continue;
        SiteWords<BPS, S> s;
        load_smem<BPS, S>(w, R, r * X + x, s);
#pragma unroll
        for (int k = 0; k < S; k++) {
            const uint32_t p = s.slot(k);
            if (p) atomicAdd(&hist[p <= ns ? p : 0u], 1u);
        }
    }
    __syncthreads();
    for (uint32_t b = tid; b <= ns; b += nthr)
        if (hist[b]) atomicAdd(counts + b, (unsigned long long)hist[b]);
}

// One timestep of one tile (`tile` of the lattice's `ntiles`), run by the
// whole block.  The block is flat (FUSED_THREADS threads); the tile's
// logical bx x by layout (bx a multiple of 32, so a warp is 32 consecutive x
// of one row) comes from the tile shape.
template <int BPS, int S, bool ROWS>
__device__ __forceinline__ void fused_tile(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst,
                                           const uint8_t *__restrict__ sites, const Geometry &g, const DevTables &m,
                                           RunState *__restrict__ rs, OverflowEntry *__restrict__ list, uint32_t cap,
                                           const TileShape &ts, int with_reaction, uint32_t tile, uint32_t ntiles)
{
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ uint32_t s_last;
    __shared__ uint32_t s_cnt[4];
    __shared__ uint32_t rowbase[FUSED_MAX_ROWS];
    __shared__ uint16_t yrow[FUSED_MAX_ROWS], zrow[FUSED_MAX_ROWS];
    __shared__ uint8_t rowflag[FUSED_MAX_ROWS];
    // A failed run stops; in a batch, a lattice whose own timestep range is
    // done sits out the remaining launches.  The run state is loaded now and
    // checked after the region load (before the first write), so that its
    // round trip overlaps the loads.
    const int32_t status = rs->status;
    const uint32_t seed = rs->seed, step = rs->step, end_step = rs->end_step;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const TileSmem t = tile_smem<BPS, S>(smem, ts, rowbase, yrow, zrow, rowflag, s_cnt);
    // The model tables, from shared memory when they are small; the table set
    // itself is kept in shared memory so that calls take it by reference
    // without a per-thread copy.
    __shared__ DevTables s_mt;
    {
        const DevTables staged = m.stage_bytes ? stage_tables(m, t.tables, tid, nthr) : m;
        if (tid == 0) s_mt = staged;
    }
    tile_rows(g, ts, tile, t);
    __syncthreads();
    tile_load<BPS, S, false>(src, sites, g, ts, t, t.A, t.occA, false, true);
    if (status != LMB_OK || step >= end_step) return;  // the same for the whole block

    uint32_t *src_w = t.A, *dst_w = t.B, *src_o = t.occA, *dst_o = t.occB;
    tile_timestep<BPS, S, ROWS>(g, s_mt, rs, list, cap, ts, t, src_w, dst_w, src_o, dst_o, seed, step,
                                with_reaction);
    tile_store<BPS, S>(dst, g, ts, t, src_w, src_o);
    // The run's species count, at the timestep it was asked for.
    const bool counting = step == rs->count_step;
    if (counting) tile_count<BPS, S>(g, ts, t, src_w, src_o, rs->count_ns, rs->counts);

    // The last block to finish resolves the overflow queue and advances the
    // step counter.
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        const uint32_t prev = atomicAdd(&rs->tiles_done, 1u);
        s_last = prev == ntiles - 1;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        if (tid == 0) rs->tiles_done = 0;
        resolve_block_flat<BPS, S>(dst, sites, g, rs, list, cap, (OverflowEntry *)smem, tid, nthr, nullptr,
                                   counting ? rs->counts : nullptr);
    }
}

// MINB: blocks per SM the launch bounds promise, the number the tile's
// shared memory lets an SM hold (2, 3 or 4): the compiler then keeps as much
// of the tile's state in registers as that occupancy allows.
template <int BPS, int S, int MINB>
__global__ void __launch_bounds__(FUSED_THREADS, MINB) fused_step_kernel(const uint32_t *__restrict__ src,
                                                                   uint32_t *__restrict__ dst,
                                                                   const uint8_t *__restrict__ sites, Geometry g,
                                                                   const __grid_constant__ DevTables m,
                                                                   RunState *__restrict__ rs,
                                                                   OverflowEntry *__restrict__ list, uint32_t cap,
                                                                   const __grid_constant__ TileShape ts,
                                                                   int with_reaction)
{
    chain_enter();
    fused_tile<BPS, S, true>(src, dst, sites, g, m, rs, list, cap, ts, with_reaction, blockIdx.x, gridDim.x);
}

// A batch of lattices advanced together: block b runs the tile of the job
// whose tile range holds b.  The buffers a job reads and writes alternate
// with `parity` (flipped every timestep), from the job's buffer index at the
// start of the run.
// Two blocks per SM: the batch plan picks tiles of at most 100 KB of shared
// memory for that (the bound also lets the compiler keep the tile's state in
// registers rather than spill it).
template <int BPS, int S>
__global__ void __launch_bounds__(FUSED_THREADS, 2) fused_batch_kernel(const FusedJob *__restrict__ jobs,
                                                                    uint32_t njobs, uint32_t parity)
{
    chain_enter();
    uint32_t lo = 0, hi = njobs;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (jobs[mid].tile_begin <= blockIdx.x) lo = mid;
        else hi = mid;
    }
    const FusedJob &j = jobs[lo];
    const uint32_t c = j.cur0 ^ parity;
    fused_tile<BPS, S, false>(j.buf[c], j.buf[c ^ 1], j.sites, j.g, j.m, j.rs, j.list, j.cap, j.ts,
                              j.with_reaction, blockIdx.x - j.tile_begin, j.ts.tiles_y * j.ts.tiles_z);
}

// ---------------------------------------------------------------------------
// Planning and launch
// ---------------------------------------------------------------------------

static size_t region_bytes(uint32_t X, uint32_t Ty, uint32_t Tz, uint32_t W)
{
    const size_t rows = (size_t)(Ty + 2) * (Tz + 2), R = (size_t)X * rows, MW = (X + 31) / 32;
    return 2 * (size_t)W * R * 4 + R * 4 + ((R + 15) & ~(size_t)15) + 2 * rows * MW * 4;
}

size_t fused_smem_bytes(const TileShape &ts, uint32_t X, uint32_t W, uint32_t cap, uint32_t stage_bytes)
{
    const size_t tile = region_bytes(X, ts.Ty, ts.Tz, W) + 16 + stage_bytes;
    const size_t sort = (size_t)pow2_at_least(cap) * sizeof(OverflowEntry);
    return tile > sort ? tile : sort;
}

bool fused_make_shape(const Geometry &g, int bps, int slots, uint32_t Ty, uint32_t Tz, TileShape &ts)
{
    if (!slots_supported(bps, slots) || slots > 16) return false;  // 2-bit codes of 16 slots per word
    if (Ty == 0 || Tz == 0 || Ty > g.Y || Tz > g.Z || g.Y % Ty || g.Z % Tz) return false;
    const uint32_t W = bps == 1 ? slots / 4 : slots;
    if (g.X > 1024) return false;
    if ((Ty + 2) * (Tz + 2) > FUSED_MAX_ROWS) return false;
    if (region_bytes(g.X, Ty, Tz, W) > FUSED_MAX_SMEM) return false;
    ts.Ty = Ty;
    ts.Tz = Tz;
    ts.Ry = Ty + 2;
    ts.Rz = Tz + 2;
    ts.tiles_y = g.Y / Ty;
    ts.tiles_z = g.Z / Tz;
    ts.R = g.X * ts.Ry * ts.Rz;
    ts.MW = (g.X + 31) / 32;
    // 16-byte row loads need 16-byte aligned rows: X words and X type bytes.
    ts.vec = (g.X % 16u) == 0;
    uint32_t bx = ((g.X + 31) / 32) * 32;
    if (bx > 128) bx = 128;
    ts.bx = bx;
    ts.by = FUSED_THREADS / bx;
    return true;
}

// Default plan: the least halo overhead among shapes that fit in shared
// memory and still give every SM two blocks; failing that, the most blocks.
bool fused_default_shape(const Geometry &g, int bps, int slots, TileShape &ts)
{
    const uint32_t cands[] = {1, 2, 4, 8, 16};
    bool found = false;
    double best = 1e30;
    for (uint32_t Ty : cands)
        for (uint32_t Tz : cands) {
            TileShape t;
            if (!fused_make_shape(g, bps, slots, Ty, Tz, t)) continue;
            const uint32_t W = bps == 1 ? slots / 4 : slots;
            if (region_bytes(g.X, Ty, Tz, W) > FUSED_PREFERRED_SMEM) continue;
            const double tiles = (double)t.tiles_y * t.tiles_z;
            const double halo = (double)(Ty + 2) * (Tz + 2) / ((double)Ty * Tz);
            const double score = tiles >= 2 * 148 ? halo : 1e6 / tiles;
            if (score < best) {
                best = score;
                ts = t;
                found = true;
            }
        }
    return found;
}

// The dynamic shared-memory limit is raised once per instantiation (per
// device) to the largest size any launch needs; setting it on every launch
// costs host time comparable to the kernel itself.
template <int BPS, int S, int MINB>
static cudaError_t ensure_smem_limit(size_t smem)
{
    static size_t granted[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    // The kernel's static shared memory counts against the default 48 KB
    // too, so the limit is raised for any size not granted yet.
    if (smem <= granted[dev]) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(fused_step_kernel<BPS, S, MINB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) granted[dev] = smem;
    return e;
}

// A tile a batch may use: it fits, and its region leaves room for the two
// blocks per SM the batch kernel is built for.
bool fused_batch_shape_ok(const Geometry &g, int bps, int slots, uint32_t Ty, uint32_t Tz, TileShape &ts)
{
    if (!fused_make_shape(g, bps, slots, Ty, Tz, ts)) return false;
    const uint32_t W = bps == 1 ? slots / 4 : slots;
    return region_bytes(g.X, Ty, Tz, W) <= FUSED_PREFERRED_SMEM;
}

// Batch plan: the batch already fills the GPU with many lattices, so each
// lattice takes the tile with the least halo overhead that still lets two
// blocks share an SM.
bool fused_batch_shape(const Geometry &g, int bps, int slots, TileShape &ts)
{
    const uint32_t cands[] = {1, 2, 4, 8, 16};
    bool found = false;
    double best = 1e30;
    for (uint32_t Ty : cands)
        for (uint32_t Tz : cands) {
            TileShape t;
            if (!fused_make_shape(g, bps, slots, Ty, Tz, t)) continue;
            const uint32_t W = bps == 1 ? slots / 4 : slots;
            if (region_bytes(g.X, Ty, Tz, W) > FUSED_PREFERRED_SMEM) continue;
            const double halo = (double)(Ty + 2) * (Tz + 2) / ((double)Ty * Tz);
            const double score = halo - 1e-6 * Ty * Tz;
            if (score < best) {
                best = score;
                ts = t;
                found = true;
            }
        }
    return found;
}

template <int BPS, int S, int MINB>
static cudaError_t fused_launch(dim3 grid, dim3 block, size_t smem, cudaStream_t stream, const uint32_t *src,
                                uint32_t *dst, const uint8_t *sites, const Geometry &g, const DevTables &m,
                                RunState *rs, OverflowEntry *list, uint32_t cap, const TileShape &ts,
                                int with_reaction)
{
    cudaError_t e = ensure_smem_limit<BPS, S, MINB>(smem);
    if (e != cudaSuccess) return e;
    return launch_chain(fused_step_kernel<BPS, S, MINB>, grid, block, smem, stream, src, dst, sites, g, m, rs, list,
                        cap, ts, with_reaction);
}

#define FUSED_DISPATCH(BPS_, S_)                                                                            \
    if (bps == BPS_ && slots == S_) {                                                                       \
        if (per_sm >= 4)                                                                                    \
            return fused_launch<BPS_, S_, 4>(grid, block, smem, stream, src, dst, sites, g, m, rs, list, cap, ts, \
                                             with_reaction);                                                \
        if (per_sm == 3)                                                                                    \
            return fused_launch<BPS_, S_, 3>(grid, block, smem, stream, src, dst, sites, g, m, rs, list, cap, ts, \
                                             with_reaction);                                                \
        return fused_launch<BPS_, S_, 2>(grid, block, smem, stream, src, dst, sites, g, m, rs, list, cap, ts,    \
                                         with_reaction);                                                    \
    }

cudaError_t launch_fused(int bps, int slots, const uint32_t *src, uint32_t *dst, const uint8_t *sites,
                         const Geometry &g, const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                         const TileShape &ts, int with_reaction, cudaStream_t stream)
{
    const uint32_t W = bps == 1 ? slots / 4 : slots;
    const size_t smem = fused_smem_bytes(ts, g.X, W, cap, m.stage_bytes);
    const dim3 grid(ts.tiles_y * ts.tiles_z), block(FUSED_THREADS);
    // Blocks of this size an SM's 228 KB of shared memory holds (the static
    // part and 1 KB reserved per block included).
    const uint32_t per_sm = (uint32_t)((228u * 1024u) / (smem + 3088u + 1024u));
    count_launch();
    FUSED_DISPATCH(1, 4)
    FUSED_DISPATCH(1, 8)
    FUSED_DISPATCH(1, 16)
    FUSED_DISPATCH(4, 4)
    FUSED_DISPATCH(4, 8)
    FUSED_DISPATCH(4, 16)
    return cudaErrorInvalidValue;
}

template <int BPS, int S>
static cudaError_t ensure_batch_smem_limit(size_t smem)
{
    static size_t granted[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    // The kernel's static shared memory counts against the default 48 KB
    // too, so the limit is raised for any size not granted yet.
    if (smem <= granted[dev]) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(fused_batch_kernel<BPS, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess) granted[dev] = smem;
    return e;
}

#define BATCH_DISPATCH(BPS_, S_)                                                                      \
    if (bps == BPS_ && slots == S_) {                                                                 \
        cudaError_t e = ensure_batch_smem_limit<BPS_, S_>(smem);                                      \
        if (e != cudaSuccess) return e;                                                               \
        return launch_chain(fused_batch_kernel<BPS_, S_>, dim3(total_tiles), dim3(FUSED_THREADS), smem, stream, \
                            jobs, njobs, parity);                                                     \
    }

cudaError_t launch_fused_batch(int bps, int slots, const FusedJob *jobs, uint32_t njobs, uint32_t total_tiles,
                               size_t smem, uint32_t parity, cudaStream_t stream)
{
    count_launch();
    BATCH_DISPATCH(1, 4)
    BATCH_DISPATCH(1, 8)
    BATCH_DISPATCH(1, 16)
    BATCH_DISPATCH(4, 4)
    BATCH_DISPATCH(4, 8)
    BATCH_DISPATCH(4, 16)
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// Cluster-resident runs of small lattices
// ---------------------------------------------------------------------------
//
// A lattice whose two buffers fit in the shared memory of one thread-block
// cluster runs a whole run in one launch.  CTA `rank` of the C in the cluster
// holds z planes rank * P .. rank * P + P - 1 (both buffers and the site
// types), so the x and y sweeps read only its own shared memory and the z
// sweep reads the neighbouring CTA's edge plane through distributed shared
// memory.  Hardware cluster barriers replace the launches between phases:
// one before the z sweep (the other CTAs' y output complete) and one after
// it (their z reads done before the next x sweep overwrites that buffer).
// Every site belongs to exactly one CTA, so sweep_site records its
// overflows once; the reaction runs on each site right after its z sweep.
// A timestep in which any site of the cluster ended full may have queued
// overflows: then the state goes to global memory, CTA 0 resolves the queue
// there (the same resolve_block_flat, step counter included), and every
// CTA reloads its planes.  The sweep rules, hashes and orders are those of
// the fused and per-phase kernels, so the result is theirs bit for bit.
//
// All CTAs run the same number of timesteps and take every branch that
// holds a cluster barrier together: the loop bounds come from the run state
// written before the launch, and the two decisions inside the loop (a full
// site somewhere, a failed resolution) are read by all CTAs from the same
// place after a barrier.
constexpr uint32_t CLUSTER_THREADS = 1024;

template <int BPS, int S>
__device__ __forceinline__ bool site_full(const SiteWords<BPS, S> &s)
{
    return __popc(occupied_slots<BPS, S>(s)) == S;
}

template <int BPS, int S>
__global__ void __launch_bounds__(CLUSTER_THREADS, 1)
    cluster_run_kernel(uint32_t *__restrict__ buf0, uint32_t *__restrict__ buf1, const uint8_t *__restrict__ sites,
                       Geometry g, const __grid_constant__ DevTables m, RunState *__restrict__ rs,
                       OverflowEntry *__restrict__ list, uint32_t cap, uint32_t P, uint32_t words_at,
                       uint32_t tables_at)
{
    namespace cg = cooperative_groups;
    constexpr int W = SiteWords<BPS, S>::W;
    cg::cluster_group cl = cg::this_cluster();
    const uint32_t rank = cl.block_rank(), C = cl.num_blocks();
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const uint32_t X = g.X, Y = g.Y, XY = g.XY, n = P * XY, z0 = rank * P;
    // Dynamic shared memory: the site types T[n]; at words_at the two
    // buffers' words A[W][n], B[W][n], a region that CTA 0's overflow sort
    // reuses (the state is in global memory then) and that is sized for it;
    // the staged model tables at tables_at.
    extern __shared__ __align__(16) uint32_t smem[];
    uint8_t *T = reinterpret_cast<uint8_t *>(smem);
    uint32_t *A = reinterpret_cast<uint32_t *>(reinterpret_cast<uint8_t *>(smem) + words_at);
    uint32_t *B = A + (size_t)W * n;
    OverflowEntry *sort = reinterpret_cast<OverflowEntry *>(A);
    uint8_t *tab = reinterpret_cast<uint8_t *>(smem) + tables_at;
    __shared__ uint32_t s_flag[2];  // CTA 0's: a site of the cluster ended full, by timestep parity
    __shared__ uint32_t s_full, s_go;
    __shared__ DevTables s_mt;
    const uint32_t seed = rs->seed, first = rs->step, end = rs->end_step;
    if (rs->status != LMB_OK || first >= end) return;  // the same for every CTA
    {
        const DevTables staged = m.stage_bytes ? stage_tables(m, tab, tid, nthr) : m;
        if (tid == 0) {
            s_mt = staged;
            s_flag[0] = s_flag[1] = 0;
            s_full = 0;
        }
    }
    for (uint32_t k = 0; k < (uint32_t)W; k++)
        for (uint32_t l = tid; l < n; l += nthr) A[k * n + l] = __ldcg(buf0 + (size_t)k * g.N + (size_t)z0 * XY + l);
    for (uint32_t l = tid; l < n; l += nthr) T[l] = sites[(size_t)z0 * XY + l];
    bool zeroth = false;
    for (uint32_t q = 0; q < m.nst; q++) zeroth |= m.qp0[q] != 0.0f;
    const bool reacting = m.nr > 0;
    cl.sync();  // every CTA's planes and flags in place before any remote access
    const DevTables &mt = s_mt;
    const TableSet tabs{&mt};
    const uint32_t rm = rank == 0 ? C - 1 : rank - 1, rp = rank == C - 1 ? 0 : rank + 1;
    uint32_t parity = 0;  // the global buffer a copy of the current state belongs in: buf0 or buf1
    for (uint32_t step = first; step < end; step++) {
        uint32_t full = 0;
        // x sweep, A -> B.
        {
            const unsigned long long th = timestep_hash(seed, step, 0);
            for (uint32_t l = tid; l < n; l += nthr) {
                const uint32_t x = l % X, xm = x == 0 ? X - 1 : x - 1, xp = x == X - 1 ? 0 : x + 1;
                const uint32_t lm = l - x + xm, lp = l - x + xp, gi = z0 * XY + l;
                SiteWords<BPS, S> own, mn, pl;
                load_smem<BPS, S>(A, n, l, own);
                load_smem<BPS, S>(A, n, lm, mn);
                load_smem<BPS, S>(A, n, lp, pl);
                own = sweep_site<BPS, S>(own, mn, pl, T[l], T[lm], T[lp], gi, gi - x + xm, gi - x + xp, th, tabs,
                                         true, 1u, rs, list, cap);
                store_smem<BPS, S>(B, n, l, own);
                full |= site_full<BPS, S>(own) ? 1u : 0u;
            }
        }
        __syncthreads();
        // y sweep, B -> A.
        {
            const unsigned long long th = timestep_hash(seed, step, 1);
            for (uint32_t l = tid; l < n; l += nthr) {
                const uint32_t p = l / XY, r = l - p * XY, y = r / X;
                const uint32_t ym = y == 0 ? Y - 1 : y - 1, yp = y == Y - 1 ? 0 : y + 1;
                const uint32_t lm = l - y * X + ym * X, lp = l - y * X + yp * X, gi = z0 * XY + l;
                SiteWords<BPS, S> own, mn, pl;
                load_smem<BPS, S>(B, n, l, own);
                load_smem<BPS, S>(B, n, lm, mn);
                load_smem<BPS, S>(B, n, lp, pl);
                own = sweep_site<BPS, S>(own, mn, pl, T[l], T[lm], T[lp], gi, gi - y * X + ym * X,
                                         gi - y * X + yp * X, th, tabs, true, 2u, rs, list, cap);
                store_smem<BPS, S>(A, n, l, own);
                full |= site_full<BPS, S>(own) ? 1u : 0u;
            }
        }
        cl.sync();  // every CTA's y output in place before the z sweep reads edge planes
        // z sweep, A -> B, and the reaction of each site right after it.
        {
            const unsigned long long th = timestep_hash(seed, step, 2), th_rx = timestep_hash(seed, step, 3);
            const uint32_t *Am = cl.map_shared_rank(A, rm), *Ap = cl.map_shared_rank(A, rp);
            const uint8_t *Tm = cl.map_shared_rank(T, rm), *Tp = cl.map_shared_rank(T, rp);
            for (uint32_t l = tid; l < n; l += nthr) {
                const uint32_t p = l / XY, r = l - p * XY, z = z0 + p;
                const uint32_t zm = z == 0 ? g.Z - 1 : z - 1, zp = z == g.Z - 1 ? 0 : z + 1;
                const uint32_t gi = z * XY + r;
                SiteWords<BPS, S> own, mn, pl;
                load_smem<BPS, S>(A, n, l, own);
                uint32_t tm, tp;
                if (p > 0) {
                    load_smem<BPS, S>(A, n, l - XY, mn);
                    tm = T[l - XY];
                } else {  // plane P - 1 of the CTA before (periodic)
                    load_smem<BPS, S>(Am, n, (P - 1) * XY + r, mn);
                    tm = Tm[(P - 1) * XY + r];
                }
                if (p + 1 < P) {
                    load_smem<BPS, S>(A, n, l + XY, pl);
                    tp = T[l + XY];
                } else {  // plane 0 of the CTA after
                    load_smem<BPS, S>(Ap, n, r, pl);
                    tp = Tp[r];
                }
                own = sweep_site<BPS, S>(own, mn, pl, T[l], tm, tp, gi, zm * XY + r, zp * XY + r, th, tabs, true,
                                         3u, rs, list, cap);
                if (reacting && (zeroth || !own.empty())) {
                    const uint32_t ts = T[l];
                    const float a0 = tload(mt.qp0 + ts);
                    if (!own.empty() || a0 != 0.0f) {
                        const float r0 = hash_float((unsigned long long)gi << 1, th_rx);
                        if (reaction_may_fire((uint32_t)__popc(occupied_slots<BPS, S>(own)), a0, ts, r0, mt))
                            own = react_site_ool<BPS, S>(own, ts, gi, th_rx, mt, rs, list, cap);
                    }
                }
                store_smem<BPS, S>(B, n, l, own);
                full |= site_full<BPS, S>(own) ? 1u : 0u;
            }
        }
        if (full) atomicOr(&s_full, 1u);
        __syncthreads();
        if (tid == 0 && s_full) atomicOr(cl.map_shared_rank(&s_flag[step & 1u], 0), 1u);
        cl.sync();  // every z output and every flag in place
        if (tid == 0) {
            s_go = *cl.map_shared_rank(&s_flag[step & 1u], 0);
            s_full = 0;
            if (rank == 0) s_flag[(step + 1u) & 1u] = 0;  // the next timestep's flag, unused until then
        }
        __syncthreads();
        parity ^= 1u;
        if (s_go) {
            // Overflows may be queued: resolve them in global memory as the
            // per-phase and fused schedules do.
            uint32_t *gb = parity ? buf1 : buf0;
            for (uint32_t k = 0; k < (uint32_t)W; k++)
                for (uint32_t l = tid; l < n; l += nthr) gb[(size_t)k * g.N + (size_t)z0 * XY + l] = B[k * n + l];
            __threadfence();
            cl.sync();  // the whole state in gb; no remote reads of shared memory remain
            if (rank == 0) {
                if (tid == 0) rs->step = step;
                __syncthreads();
                resolve_block_flat<BPS, S>(gb, sites, g, rs, list, cap, sort, tid, nthr, nullptr);
                __threadfence();
            }
            cl.sync();  // the resolution (or its failure) visible to every CTA
            if (*(volatile int32_t *)&rs->status != LMB_OK) return;  // the partial lattice is in gb
            for (uint32_t k = 0; k < (uint32_t)W; k++)
                for (uint32_t l = tid; l < n; l += nthr) B[k * n + l] = __ldcg(gb + (size_t)k * g.N + (size_t)z0 * XY + l);
            __syncthreads();
        }
        uint32_t *t0 = A;
        A = B;
        B = t0;
    }
    // The final state, in the buffer the timestep count's parity gives.
    uint32_t *gb = parity ? buf1 : buf0;
    for (uint32_t k = 0; k < (uint32_t)W; k++)
        for (uint32_t l = tid; l < n; l += nthr) gb[(size_t)k * g.N + (size_t)z0 * XY + l] = A[k * n + l];
    if (rank == 0 && tid == 0) set_step(rs, seed, end);
    cl.sync();  // no CTA leaves while another may still read its shared memory
}

// Plan of a cluster-resident run: C CTAs (the largest of 16, 8, 4, 2, 1 that
// divides Z and that the device can place) of P = Z / C planes each, and the
// dynamic shared memory of a CTA.  False when the lattice does not fit.
// Byte offsets in a CTA's dynamic shared memory: the buffers' words (and the
// overflow sort) at words_at, after the site types; the tables at tables_at.
static void cluster_layout(const Geometry &g, uint32_t W, uint32_t P, uint32_t cap, size_t &words_at,
                           size_t &tables_at)
{
    const size_t n = (size_t)P * g.XY;
    words_at = (n + 15) & ~(size_t)15;
    const size_t words = 2 * (size_t)W * n * 4;
    const size_t sort = (size_t)pow2_at_least(cap) * sizeof(OverflowEntry);
    tables_at = words_at + ((words > sort ? words : sort) + 15 & ~(size_t)15);
}

template <int BPS, int S>
static bool cluster_plan_t(const Geometry &g, uint32_t cap, uint32_t stage_bytes, uint32_t &C, uint32_t &P,
                           size_t &words_at, size_t &tables_at, size_t &smem)
{
    const uint32_t W = SiteWords<BPS, S>::W;
    for (uint32_t c = 16; c >= 1; c >>= 1) {
        if (g.Z % c) continue;
        const uint32_t p = g.Z / c;
        size_t wa = 0, ta = 0;
        cluster_layout(g, W, p, cap, wa, ta);
        const size_t sm = ta + stage_bytes;
        if (sm > 200 * 1024) continue;
        if (cudaFuncSetAttribute(cluster_run_kernel<BPS, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) !=
                cudaSuccess ||
            cudaFuncSetAttribute(cluster_run_kernel<BPS, S>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(c);
        cfg.blockDim = dim3(CLUSTER_THREADS);
        cfg.dynamicSmemBytes = sm;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = c;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, cluster_run_kernel<BPS, S>, &cfg) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        if (clusters < 1) continue;
        C = c;
        P = p;
        words_at = wa;
        tables_at = ta;
        smem = sm;
        return true;
    }
    return false;
}

#define CLUSTER_DISPATCH(BPS_, S_, ...) \
    if (bps == BPS_ && slots == S_) {   \
        __VA_ARGS__;                    \
    }

bool cluster_plan(const Geometry &g, int bps, int slots, uint32_t cap, uint32_t stage_bytes, uint32_t &C,
                  uint32_t &P)
{
    size_t words_at = 0, tables_at = 0, smem = 0;
    if (slots > 16) return false;
    CLUSTER_DISPATCH(1, 4, return cluster_plan_t<1, 4>(g, cap, stage_bytes, C, P, words_at, tables_at, smem))
    CLUSTER_DISPATCH(1, 8, return cluster_plan_t<1, 8>(g, cap, stage_bytes, C, P, words_at, tables_at, smem))
    CLUSTER_DISPATCH(1, 16, return cluster_plan_t<1, 16>(g, cap, stage_bytes, C, P, words_at, tables_at, smem))
    CLUSTER_DISPATCH(4, 4, return cluster_plan_t<4, 4>(g, cap, stage_bytes, C, P, words_at, tables_at, smem))
    CLUSTER_DISPATCH(4, 8, return cluster_plan_t<4, 8>(g, cap, stage_bytes, C, P, words_at, tables_at, smem))
    CLUSTER_DISPATCH(4, 16, return cluster_plan_t<4, 16>(g, cap, stage_bytes, C, P, words_at, tables_at, smem))
    return false;
}

template <int BPS, int S>
static cudaError_t cluster_launch_t(uint32_t *buf0, uint32_t *buf1, const uint8_t *sites, const Geometry &g,
                                    const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                                    cudaStream_t stream)
{
    uint32_t C = 0, P = 0;
    size_t words_at = 0, tables_at = 0, smem = 0;
    if (!cluster_plan_t<BPS, S>(g, cap, m.stage_bytes, C, P, words_at, tables_at, smem))
        return cudaErrorInvalidConfiguration;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(CLUSTER_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    count_launch();
    return cudaLaunchKernelEx(&cfg, cluster_run_kernel<BPS, S>, buf0, buf1, sites, g, m, rs, list, cap, P,
                              (uint32_t)words_at, (uint32_t)tables_at);
}

cudaError_t launch_cluster_run(int bps, int slots, uint32_t *buf0, uint32_t *buf1, const uint8_t *sites,
                               const Geometry &g, const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                               cudaStream_t stream)
{
    CLUSTER_DISPATCH(1, 4, return cluster_launch_t<1, 4>(buf0, buf1, sites, g, m, rs, list, cap, stream))
    CLUSTER_DISPATCH(1, 8, return cluster_launch_t<1, 8>(buf0, buf1, sites, g, m, rs, list, cap, stream))
    CLUSTER_DISPATCH(1, 16, return cluster_launch_t<1, 16>(buf0, buf1, sites, g, m, rs, list, cap, stream))
    CLUSTER_DISPATCH(4, 4, return cluster_launch_t<4, 4>(buf0, buf1, sites, g, m, rs, list, cap, stream))
    CLUSTER_DISPATCH(4, 8, return cluster_launch_t<4, 8>(buf0, buf1, sites, g, m, rs, list, cap, stream))
    CLUSTER_DISPATCH(4, 16, return cluster_launch_t<4, 16>(buf0, buf1, sites, g, m, rs, list, cap, stream))
    return cudaErrorInvalidValue;
}


// ---------------------------------------------------------------------------
// Grid-resident fused tiles: every tile of a fused plan resident at once
// ---------------------------------------------------------------------------
//
// When the plan's tiles fit on the device together (a cooperative launch of
// one block per tile), one launch runs every timestep of a run.  A block
// keeps its region in shared memory from one timestep to the next: after
// tile_timestep it stores its owned rows into the global buffer of that
// timestep (buf1, buf0, buf1, ... : the buffers alternate as they do between
// fused launches), and after a grid barrier it reloads only its halo rows
// from there, which the neighbouring tiles stored.  The site types and the
// staged model tables are loaded once per run.
//
// Overflows: a block that queued one sees the queue count non-zero after its
// own timestep (its atomics precede that read), and raises the timestep's flag
// (RunState::grid_full, by timestep index modulo 3) before the barrier; after
// it every block reads the same flag.  When it is up, block 0 resolves the
// queue in the timestep's buffer (which then holds the whole lattice), and
// after a second barrier every block reloads its whole region.  Block 0 clears
// the flag of timestep + 2 after the barrier of timestep: every block read
// that flag (as timestep - 1's) before this barrier, and raises it only after
// the next one, which block 0 reaches after the clearing store.
//
// Hazards on the buffers: a buffer is written at timestep k + 2 only after the
// barrier of timestep k + 1, which every block reaches after its halo reads of
// timestep k; the input (buf0) is first written at the second timestep, after
// every block has loaded its region.  So a run gives, bit for bit, what the
// same number of fused launches gives.
//
// The barrier (grid_barrier, lmb_device.cuh) is bounded: a wait that gives up
// sets LMB_E_TIMEOUT and ends the block; the others give up at their next
// barrier.
template <int BPS, int S>
__global__ void __launch_bounds__(FUSED_THREADS, 2)
    fused_grid_kernel(uint32_t *__restrict__ buf0, uint32_t *__restrict__ buf1, const uint8_t *__restrict__ sites,
                      Geometry g, const __grid_constant__ DevTables m, RunState *__restrict__ rs,
                      OverflowEntry *__restrict__ list, uint32_t cap, const __grid_constant__ TileShape ts,
                      int with_reaction)
{
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ uint32_t s_cnt[4];
    __shared__ uint32_t rowbase[FUSED_MAX_ROWS];
    __shared__ uint16_t yrow[FUSED_MAX_ROWS], zrow[FUSED_MAX_ROWS];
    __shared__ uint8_t rowflag[FUSED_MAX_ROWS];
    __shared__ uint32_t s_go;
    __shared__ DevTables s_mt;
    const int32_t status = rs->status;
    const uint32_t seed = rs->seed, first = rs->step, end = rs->end_step;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x, nblocks = gridDim.x;
    const TileSmem t = tile_smem<BPS, S>(smem, ts, rowbase, yrow, zrow, rowflag, s_cnt);
    {
        const DevTables staged = m.stage_bytes ? stage_tables(m, t.tables, tid, nthr) : m;
        if (tid == 0) s_mt = staged;
    }
    tile_rows(g, ts, blockIdx.x, t);
    __syncthreads();
    tile_load<BPS, S, true>(buf0, sites, g, ts, t, t.A, t.occA, false, true);
    if (status != LMB_OK || first >= end) return;  // the same for every block

    uint32_t *src_w = t.A, *dst_w = t.B, *src_o = t.occA, *dst_o = t.occB;
    unsigned long long passed = 0;  // arrivals the barriers passed so far have counted
    uint32_t k = 0;
    for (uint32_t step = first; step < end; step++, k++) {
        tile_timestep<BPS, S, true>(g, s_mt, rs, list, cap, ts, t, src_w, dst_w, src_o, dst_o, seed, step,
                                    with_reaction);
        uint32_t *out = (k & 1u) ? buf0 : buf1;
        tile_store<BPS, S>(out, g, ts, t, src_w, src_o);
        // tile_timestep ended with a block barrier: this block's overflows
        // are in the queue count.
        if (tid == 0 && __ldcg(&rs->ovf_count) != 0) atomicOr(&rs->grid_full[step % 3u], 1u);
        passed += nblocks;
        if (!grid_barrier(&rs->grid_bar, passed)) {
            if (tid == 0) atomicCAS(&rs->status, (int32_t)LMB_OK, (int32_t)LMB_E_TIMEOUT);
            return;
        }
        if (tid == 0) {
            s_go = __ldcg(&rs->grid_full[step % 3u]);
            if (blockIdx.x == 0) rs->grid_full[(step + 2u) % 3u] = 0;
        }
        __syncthreads();
        if (s_go) {
            // Overflows are queued: block 0 resolves them in `out`, as the
            // last block of a fused launch does, then every block reloads.
            if (blockIdx.x == 0) {
                if (tid == 0) rs->step = step;
                __syncthreads();
                resolve_block_flat<BPS, S>(out, sites, g, rs, list, cap, (OverflowEntry *)smem, tid, nthr, nullptr);
                __threadfence();
            }
            passed += nblocks;
            if (!grid_barrier(&rs->grid_bar, passed)) {
                if (tid == 0) atomicCAS(&rs->status, (int32_t)LMB_OK, (int32_t)LMB_E_TIMEOUT);
                return;
            }
            if (*(volatile int32_t *)&rs->status != LMB_OK) return;  // the partial lattice is in `out`
            // Block 0's sort area covered its whole dynamic shared memory:
            // the staged tables (same place, same contents) and the site
            // types come back with the region.
            if (blockIdx.x == 0 && m.stage_bytes) stage_tables(m, t.tables, tid, nthr);
            tile_load<BPS, S, true>(out, sites, g, ts, t, src_w, src_o, false, blockIdx.x == 0);
        } else {
            tile_load<BPS, S, true>(out, sites, g, ts, t, src_w, src_o, true, false);
        }
    }
    if (blockIdx.x == 0 && tid == 0) set_step(rs, seed, end);
}

// Blocks of fused_grid_kernel with `smem` bytes an SM holds at once (0 when
// the kernel's attributes cannot be set).
template <int BPS, int S>
static uint32_t grid_blocks_per_sm(size_t smem)
{
    // The limit only grows (per device), as for the fused kernel, so that a
    // smaller plan checked later never lowers it under a larger one's launch.
    static size_t granted[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 0;
    }
    if (smem > granted[dev]) {
        if (cudaFuncSetAttribute(fused_grid_kernel<BPS, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        granted[dev] = smem;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused_grid_kernel<BPS, S>, FUSED_THREADS, smem) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (uint32_t)per_sm;
}

#define GRID_DISPATCH(BPS_, S_, ...) \
    if (bps == BPS_ && slots == S_) { \
        __VA_ARGS__;                  \
    }

static uint32_t grid_capacity(int bps, int slots, size_t smem)
{
    int dev = 0, sms = 0, coop = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) {
        cudaGetLastError();
        return 0;
    }
    uint32_t per_sm = 0;
    GRID_DISPATCH(1, 4, per_sm = grid_blocks_per_sm<1, 4>(smem))
    GRID_DISPATCH(1, 8, per_sm = grid_blocks_per_sm<1, 8>(smem))
    GRID_DISPATCH(1, 16, per_sm = grid_blocks_per_sm<1, 16>(smem))
    GRID_DISPATCH(4, 4, per_sm = grid_blocks_per_sm<4, 4>(smem))
    GRID_DISPATCH(4, 8, per_sm = grid_blocks_per_sm<4, 8>(smem))
    GRID_DISPATCH(4, 16, per_sm = grid_blocks_per_sm<4, 16>(smem))
    return per_sm * (uint32_t)sms;
}

bool fused_grid_fits(const Geometry &g, int bps, int slots, uint32_t cap, uint32_t stage_bytes, const TileShape &ts)
{
    const uint32_t W = bps == 1 ? slots / 4 : slots;
    const size_t smem = fused_smem_bytes(ts, g.X, W, cap, stage_bytes);
    if (smem > FUSED_MAX_SMEM) return false;
    return ts.tiles_y * ts.tiles_z <= grid_capacity(bps, slots, smem);
}

bool fused_grid_default_shape(const Geometry &g, int bps, int slots, uint32_t cap, uint32_t stage_bytes,
                              TileShape &ts)
{
    // The most tiles among the shapes whose tiles fit together (a timestep
    // is the slowest tile's chain, shorter for smaller tiles), then the least
    // halo overhead.  On the rod cell this picks 4 x 8 (256 tiles), the
    // fastest plan measured; 8 x 8 (128 tiles, the least halo) is 7 % slower.
    const uint32_t cands[] = {1, 2, 4, 8, 16};
    bool found = false;
    uint32_t best_tiles = 0;
    double best_halo = 1e30;
    for (uint32_t Ty : cands)
        for (uint32_t Tz : cands) {
            TileShape t;
            if (!fused_make_shape(g, bps, slots, Ty, Tz, t) || !fused_grid_fits(g, bps, slots, cap, stage_bytes, t))
                continue;
            const uint32_t tiles = t.tiles_y * t.tiles_z;
            const double halo = (double)(Ty + 2) * (Tz + 2) / ((double)Ty * Tz);
            if (tiles > best_tiles || (tiles == best_tiles && halo < best_halo)) {
                best_tiles = tiles;
                best_halo = halo;
                ts = t;
                found = true;
            }
        }
    return found;
}

template <int BPS, int S>
static cudaError_t fused_grid_launch_t(uint32_t *buf0, uint32_t *buf1, const uint8_t *sites, const Geometry &g,
                                       const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                                       const TileShape &ts, int with_reaction, size_t smem, cudaStream_t stream)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ts.tiles_y * ts.tiles_z);
    cfg.blockDim = dim3(FUSED_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // every block resident at once, or no launch
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    count_launch();
    return cudaLaunchKernelEx(&cfg, fused_grid_kernel<BPS, S>, buf0, buf1, sites, g, m, rs, list, cap, ts,
                              with_reaction);
}

cudaError_t launch_fused_grid(int bps, int slots, uint32_t *buf0, uint32_t *buf1, const uint8_t *sites,
                              const Geometry &g, const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                              const TileShape &ts, int with_reaction, cudaStream_t stream)
{
    if (!fused_grid_fits(g, bps, slots, cap, m.stage_bytes, ts)) return cudaErrorInvalidConfiguration;
    const uint32_t W = bps == 1 ? slots / 4 : slots;
    const size_t smem = fused_smem_bytes(ts, g.X, W, cap, m.stage_bytes);
    // The barrier count and the three overflow flags, contiguous in the run state.
    cudaError_t e = cudaMemsetAsync(&rs->grid_bar, 0, sizeof(unsigned long long) + 3 * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    GRID_DISPATCH(1, 4, return fused_grid_launch_t<1, 4>(buf0, buf1, sites, g, m, rs, list, cap, ts, with_reaction, smem, stream))
    GRID_DISPATCH(1, 8, return fused_grid_launch_t<1, 8>(buf0, buf1, sites, g, m, rs, list, cap, ts, with_reaction, smem, stream))
    GRID_DISPATCH(1, 16, return fused_grid_launch_t<1, 16>(buf0, buf1, sites, g, m, rs, list, cap, ts, with_reaction, smem, stream))
    GRID_DISPATCH(4, 4, return fused_grid_launch_t<4, 4>(buf0, buf1, sites, g, m, rs, list, cap, ts, with_reaction, smem, stream))
    GRID_DISPATCH(4, 8, return fused_grid_launch_t<4, 8>(buf0, buf1, sites, g, m, rs, list, cap, ts, with_reaction, smem, stream))
    GRID_DISPATCH(4, 16, return fused_grid_launch_t<4, 16>(buf0, buf1, sites, g, m, rs, list, cap, ts, with_reaction, smem, stream))
    return cudaErrorInvalidValue;
}

}  // namespace lmb
