// lmb_fused.h -- tile plan and launcher of the fused timestep kernel.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "lmb_internal.h"

namespace lmb {

constexpr int FUSED_THREADS = 256;
constexpr size_t FUSED_MAX_SMEM = 200 * 1024;       // per block, below the 227 KB limit
constexpr size_t FUSED_PREFERRED_SMEM = 100 * 1024; // default plan: two blocks per SM
constexpr uint32_t FUSED_MAX_ROWS = 324;            // (Ty + 2) * (Tz + 2), up to 16 x 16 tiles

// A block owns Ty x Tz full x-rows; its region adds one halo row on each side
// in y and z: R = X * (Ty + 2) * (Tz + 2) sites.
struct TileShape {
    uint32_t Ty, Tz;
    uint32_t Ry, Rz;
    uint32_t tiles_y, tiles_z;
    uint32_t R;
    uint32_t MW;  // 32-bit occupancy mask words per row
    uint32_t vec;  // region rows are 16-byte aligned: load them with 16-byte accesses
    uint32_t bx, by;
};

// One lattice of a batch run: both buffers (the run starts from buf[cur0]),
// its model, run state, overflow queue and tile plan, and where its tiles
// start in the batch's block numbering.
struct FusedJob {
    uint32_t *buf[2];
    const uint8_t *sites;
    Geometry g;
    DevTables m;
    RunState *rs;
    OverflowEntry *list;
    uint32_t cap;
    TileShape ts;
    int with_reaction;
    uint32_t cur0;
    uint32_t tile_begin;
};

cudaError_t launch_fused_batch(int bytes_per_slot, int slots, const FusedJob *jobs, uint32_t njobs,
                               uint32_t total_tiles, size_t smem, uint32_t parity, cudaStream_t stream);

bool fused_make_shape(const Geometry &g, int bytes_per_slot, int slots, uint32_t Ty, uint32_t Tz, TileShape &ts);
bool fused_default_shape(const Geometry &g, int bytes_per_slot, int slots, TileShape &ts);
bool fused_batch_shape(const Geometry &g, int bytes_per_slot, int slots, TileShape &ts);
bool fused_batch_shape_ok(const Geometry &g, int bytes_per_slot, int slots, uint32_t Ty, uint32_t Tz, TileShape &ts);
size_t fused_smem_bytes(const TileShape &ts, uint32_t X, uint32_t W, uint32_t cap, uint32_t stage_bytes);
cudaError_t launch_fused(int bytes_per_slot, int slots, const uint32_t *src, uint32_t *dst, const uint8_t *sites,
                         const Geometry &g, const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                         const TileShape &ts, int with_reaction, cudaStream_t stream);

// Cluster-resident runs of small lattices (lmb_fused.cu): the whole lattice
// in the shared memory of one thread-block cluster of C CTAs (P = Z / C z
// planes each), every timestep of a run in one launch.  cluster_plan is
// false when the lattice does not fit or the device cannot place the cluster
// (it sets the kernel's attributes on the current device).  The run starts
// from buf0 and ends in buf0 or buf1 by the parity of its timestep count (of
// the failing timestep + 1 when it fails), as alternating launches would.
bool cluster_plan(const Geometry &g, int bytes_per_slot, int slots, uint32_t cap, uint32_t stage_bytes, uint32_t &C,
                  uint32_t &P);
cudaError_t launch_cluster_run(int bytes_per_slot, int slots, uint32_t *buf0, uint32_t *buf1, const uint8_t *sites,
                               const Geometry &g, const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                               cudaStream_t stream);

// Grid-resident fused tiles (lmb_fused.cu): the tiles of a fused plan held
// in shared memory by a cooperative launch of one block per tile, every
// timestep of a run in one launch; halo rows exchanged through the two
// buffers (which alternate as between fused launches), a bounded grid barrier
// per timestep (LMB_E_TIMEOUT in the run state when a wait gives up).  The
// run starts from buf0 and ends in buf0 or buf1 by the parity of its timestep
// count (of the failing timestep + 1 when it fails).  fused_grid_fits: the
// plan's tiles fit on the current device at once (it sets the kernel's
// shared-memory attribute); fused_grid_default_shape: among the shapes that
// do, the one with the most tiles, then the least halo.
bool fused_grid_fits(const Geometry &g, int bytes_per_slot, int slots, uint32_t cap, uint32_t stage_bytes,
                     const TileShape &ts);
bool fused_grid_default_shape(const Geometry &g, int bytes_per_slot, int slots, uint32_t cap, uint32_t stage_bytes,
                              TileShape &ts);
cudaError_t launch_fused_grid(int bytes_per_slot, int slots, uint32_t *buf0, uint32_t *buf1, const uint8_t *sites,
                              const Geometry &g, const DevTables &m, RunState *rs, OverflowEntry *list, uint32_t cap,
                              const TileShape &ts, int with_reaction, cudaStream_t stream);

}  // namespace lmb
