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
#include <cuda_runtime.h>
#include <stdint.h>

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

template <int BPS, int S>
__global__ void __launch_bounds__(FUSED_THREADS) fused_step_kernel(const uint32_t *__restrict__ src,
                                                                   uint32_t *__restrict__ dst,
                                                                   const uint8_t *__restrict__ sites, Geometry g,
                                                                   DevTables m, RunState *__restrict__ rs,
                                                                   OverflowEntry *__restrict__ list, uint32_t cap,
                                                                   TileShape ts, int with_reaction)
{
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ uint32_t s_last;
    constexpr int W = SiteWords<BPS, S>::W;
    if (rs->status != LMB_OK) return;
    const uint32_t X = g.X, Y = g.Y, Z = g.Z, R = ts.R, Ry = ts.Ry, Ty = ts.Ty, Tz = ts.Tz;
    uint32_t *A = smem;
    uint32_t *B = smem + (size_t)W * R;
    uint8_t *T = (uint8_t *)(smem + (size_t)2 * W * R);
    const uint32_t tyi = blockIdx.x % ts.tiles_y, tzi = blockIdx.x / ts.tiles_y;
    const uint32_t y0 = tyi * Ty, z0 = tzi * Tz;
    const uint32_t seed = rs->seed, step = rs->step;
    const uint32_t tx = threadIdx.x, ty = threadIdx.y, bx = blockDim.x, by = blockDim.y;
    // Region row r = lz * Ry + ly maps to lattice row (y0 - 1 + ly, z0 - 1 + lz), periodic.
#define GY(ly) ((y0 + (ly) + Y - 1) % Y)
#define GZ(lz) ((z0 + (lz) + Z - 1) % Z)

    // Load the region.
    const uint32_t rows = Ry * ts.Rz;
    for (uint32_t r = ty; r < rows; r += by) {
        const uint32_t ly = r % Ry, lz = r / Ry;
        const uint32_t gbase = GY(ly) * X + GZ(lz) * g.XY;
        for (uint32_t x = tx; x < X; x += bx) {
            const uint32_t l = r * X + x, gi = gbase + x;
#pragma unroll
            for (int k = 0; k < W; k++) A[(size_t)k * R + l] = __ldg(src + (size_t)k * g.N + gi);
            T[l] = __ldg(sites + gi);
        }
    }
    __syncthreads();

    // x sweep of every loaded row: A -> B.
    {
        const unsigned long long th = timestep_hash(seed, step, 0);
        for (uint32_t r = ty; r < rows; r += by) {
            const uint32_t ly = r % Ry, lz = r / Ry;
            const bool owned_row = ly >= 1 && ly <= Ty && lz >= 1 && lz <= Tz;
            const uint32_t gbase = GY(ly) * X + GZ(lz) * g.XY;
            for (uint32_t x = tx; x < X; x += bx) {
                const uint32_t xm = x == 0 ? X - 1 : x - 1, xp = x == X - 1 ? 0 : x + 1;
                const uint32_t l = r * X + x, lm = r * X + xm, lp = r * X + xp;
                SiteWords<BPS, S> own, mn, pl;
                load_smem<BPS, S>(A, R, l, own);
                load_smem<BPS, S>(A, R, lm, mn);
                load_smem<BPS, S>(A, R, lp, pl);
                if (!(own.empty() && mn.empty() && pl.empty()))
                    own = sweep_site<BPS, S>(own, mn, pl, T[l], T[lm], T[lp], gbase + x, gbase + xm, gbase + xp, th,
                                             m, owned_row, 1u, rs, list, cap);
                store_smem<BPS, S>(B, R, l, own);
            }
        }
    }
    __syncthreads();

    // y sweep of the owned y rows of every loaded z plane: B -> A.
    {
        const unsigned long long th = timestep_hash(seed, step, 1);
        const uint32_t yrows = Ty * ts.Rz;
        for (uint32_t q = ty; q < yrows; q += by) {
            const uint32_t ly = 1 + q % Ty, lz = q / Ty;
            const uint32_t r = lz * Ry + ly;
            const bool owned_row = lz >= 1 && lz <= Tz;
            const uint32_t gz = GZ(lz) * g.XY;
            const uint32_t gb = GY(ly) * X + gz, gbm = GY(ly - 1) * X + gz, gbp = GY(ly + 1) * X + gz;
            for (uint32_t x = tx; x < X; x += bx) {
                const uint32_t l = r * X + x, lm = l - X, lp = l + X;
                SiteWords<BPS, S> own, mn, pl;
                load_smem<BPS, S>(B, R, l, own);
                load_smem<BPS, S>(B, R, lm, mn);
                load_smem<BPS, S>(B, R, lp, pl);
                if (!(own.empty() && mn.empty() && pl.empty()))
                    own = sweep_site<BPS, S>(own, mn, pl, T[l], T[lm], T[lp], gb + x, gbm + x, gbp + x, th, m,
                                             owned_row, 2u, rs, list, cap);
                store_smem<BPS, S>(A, R, l, own);
            }
        }
    }
    __syncthreads();

    // z sweep of the owned rows (A), then the reaction in registers, then the
    // single write of the owned rows.
    {
        const unsigned long long thz = timestep_hash(seed, step, 2);
        const unsigned long long thr = timestep_hash(seed, step, 3);
        const uint32_t orows = Ty * Tz;
        for (uint32_t q = ty; q < orows; q += by) {
            const uint32_t ly = 1 + q % Ty, lz = 1 + q / Ty;
            const uint32_t r = lz * Ry + ly;
            const uint32_t gyx = GY(ly) * X;
            const uint32_t gb = gyx + GZ(lz) * g.XY, gbm = gyx + GZ(lz - 1) * g.XY, gbp = gyx + GZ(lz + 1) * g.XY;
            const uint32_t RX = Ry * X;
            for (uint32_t x = tx; x < X; x += bx) {
                const uint32_t l = r * X + x, lm = l - RX, lp = l + RX;
                SiteWords<BPS, S> own, mn, pl;
                load_smem<BPS, S>(A, R, l, own);
                load_smem<BPS, S>(A, R, lm, mn);
                load_smem<BPS, S>(A, R, lp, pl);
                if (!(own.empty() && mn.empty() && pl.empty()))
                    own = sweep_site<BPS, S>(own, mn, pl, T[l], T[lm], T[lp], gb + x, gbm + x, gbp + x, thz, m,
                                             true, 3u, rs, list, cap);
                if (with_reaction) react_site<BPS, S>(own, T[l], gb + x, thr, m, rs, list, cap);
                own.store(dst, g.N, gb + x);
            }
        }
    }
#undef GY
#undef GZ

    // The last block to finish resolves the overflow queue and advances the
    // step counter.
    __syncthreads();
    if (tx == 0 && ty == 0) {
        __threadfence();
        const uint32_t prev = atomicAdd(&rs->tiles_done, 1u);
        s_last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        if (tx == 0 && ty == 0) rs->tiles_done = 0;
        // Flatten the 2-D block for the shared resolver.
        resolve_block_flat<BPS, S>(dst, sites, g, rs, list, cap, (OverflowEntry *)smem, tx + ty * bx, bx * by);
    }
}

// ---------------------------------------------------------------------------
// Planning and launch
// ---------------------------------------------------------------------------

static size_t region_bytes(uint32_t X, uint32_t Ty, uint32_t Tz, uint32_t W)
{
    const size_t R = (size_t)X * (Ty + 2) * (Tz + 2);
    return ((2 * (size_t)W * R * 4 + R) + 15) & ~(size_t)15;
}

size_t fused_smem_bytes(const TileShape &ts, uint32_t X, uint32_t W, uint32_t cap)
{
    const size_t tile = region_bytes(X, ts.Ty, ts.Tz, W);
    const size_t sort = (size_t)pow2_at_least(cap) * sizeof(OverflowEntry);
    return tile > sort ? tile : sort;
}

bool fused_make_shape(const Geometry &g, int bps, int slots, uint32_t Ty, uint32_t Tz, TileShape &ts)
{
    if (!slots_supported(bps, slots)) return false;
    if (Ty == 0 || Tz == 0 || Ty > g.Y || Tz > g.Z || g.Y % Ty || g.Z % Tz) return false;
    const uint32_t W = bps == 1 ? slots / 4 : slots;
    if (g.X > 1024) return false;
    if (region_bytes(g.X, Ty, Tz, W) > FUSED_MAX_SMEM) return false;
    ts.Ty = Ty;
    ts.Tz = Tz;
    ts.Ry = Ty + 2;
    ts.Rz = Tz + 2;
    ts.tiles_y = g.Y / Ty;
    ts.tiles_z = g.Z / Tz;
    ts.R = g.X * ts.Ry * ts.Rz;
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

#define FUSED_DISPATCH(BPS_, S_)                                                                                   \
    if (bps == BPS_ && slots == S_) {                                                                              \
        auto kern = fused_step_kernel<BPS_, S_>;                                                                   \
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        kern<<<grid, block, smem, stream>>>(src, dst, sites, g, m, rs, list, cap, ts, with_reaction);             \
        return cudaGetLastError();                                                                                 \
    }

cudaError_t launch_fused(int bps, int slots, const uint32_t *src, uint32_t *dst, const uint8_t *sites,
                         const Geometry &g, const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                         const TileShape &ts, int with_reaction, cudaStream_t stream)
{
    const uint32_t W = bps == 1 ? slots / 4 : slots;
    const size_t smem = fused_smem_bytes(ts, g.X, W, cap);
    const dim3 grid(ts.tiles_y * ts.tiles_z), block(ts.bx, ts.by);
    count_launch();
    FUSED_DISPATCH(1, 4)
    FUSED_DISPATCH(1, 8)
    FUSED_DISPATCH(1, 16)
    FUSED_DISPATCH(1, 32)
    FUSED_DISPATCH(4, 4)
    FUSED_DISPATCH(4, 8)
    FUSED_DISPATCH(4, 16)
    return cudaErrorInvalidValue;
}

}  // namespace lmb
