// lmb_internal.h -- structures shared by the C ABI and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

struct lmb_lattice;

// A context: one device and one stream.  It lives until its handle and every
// model, lattice, batch and CME ensemble made from it are destroyed, whatever
// the order of those calls.
struct lmb_ctx {
    int device;
    cudaStream_t stream;
    bool own_stream;
    std::atomic<int> refs;
};

static inline void ctx_retain(lmb_ctx *c) { c->refs.fetch_add(1); }

static inline void ctx_release(lmb_ctx *c)
{
    if (c->refs.fetch_sub(1) == 1) {
        cudaSetDevice(c->device);
        if (c->own_stream) cudaStreamDestroy(c->stream);
        delete c;
    }
}

namespace lmb {

// Lattice geometry; site i = x + y*X + z*X*Y.
struct Geometry {
    uint32_t X, Y, Z;
    uint32_t XY;
    uint32_t N;
};

// Device-resident model tables (FP32 per-timestep values).  The sparse
// stoichiometry (stoich_*) lists each reaction's nonzero S entries in
// ascending species order; it replaces the dense column the reference copies
// per reaction event (byte_reaction_dev.cu:182-199).
struct DevTables {
    uint32_t ns, nst, nr;
    const float *T;
    const float *qp0, *qp1, *qp2;
    const uint32_t *order, *D1, *D2;
    const float *rate;
    const uint8_t *RL;
    const uint32_t *stoich_off;  // [nr+1]
    const uint32_t *stoich_sp;   // 0-based species
    const int32_t *stoich_d;     // stoichiometric change
    uint32_t nnz;                // entries of the sparse stoichiometry
    uint32_t stage_bytes;        // shared-memory copy size of all tables, 0 if too large to stage
    const float *qpmax;          // [nst] largest qp1 entry, then [nst] largest qp2 entry, per site type
    // Reactions a site can fire, by first reactant: [rx_off[0], rx_off[1])
    // lists the zeroth-order reactions, [rx_off[s], rx_off[s+1]) those whose
    // first reactant is species s (1-based), each list ascending.
    const uint32_t *rx_off;      // [ns + 2]
    const uint32_t *rx_list;     // [nr]
};

// One queued overflow: the sort key orders entries by (phase, site, seq);
// phase 0 marks entries carried over by the relaxed handler.
struct OverflowEntry {
    unsigned long long key;
    uint32_t site;
    uint32_t particle;
};

constexpr int KEY_PHASE_SHIFT = 60;
constexpr int KEY_SITE_SHIFT = 20;

// Per-lattice run state in device memory, read by every kernel.
struct RunState {
    uint32_t seed;
    uint32_t step;        // timestep index the next kernels work on
    uint32_t end_step;    // exclusive end of the current run
    int32_t status;       // LMB_OK or the error that stopped the run
    uint32_t failed_step;
    uint32_t ovf_count;   // entries in the list, carried ones first
    uint32_t carried;     // relaxed handler: entries kept from earlier steps
    uint32_t mode;        // LMB_OVERFLOW_*
    unsigned long long overflows;
    unsigned long long reactions;
    uint32_t max_species; // validation scratch
    uint32_t max_site_type;
    uint32_t tiles_done;  // fused kernel: blocks finished in this launch
    uint32_t rx_count;    // per-phase schedule: sites the z sweep listed for the reaction step
    uint32_t rx_skip;     // timesteps left to run without the list (it overflowed recently)
    // timestep_hash(seed, step, k) for the sub-steps k = 0..3 of `step`, set
    // with every change of step (the per-phase kernels read them here).
    unsigned long long th[4];
    // Species counts taken inside the run: at timestep count_step the fused
    // kernel adds the particles of the sites it stores (and the overflow
    // resolution those it puts back) into counts[0..count_ns]; count_step is
    // ~0u when no count is asked for.
    uint32_t count_step;
    uint32_t count_ns;
    unsigned long long *counts;
    // Grid-resident schedule, zeroed before each of its launches: the
    // arrivals at the grid barrier so far, and the "an overflow was queued"
    // flags of the timesteps, by timestep index modulo 3.
    unsigned long long grid_bar;
    uint32_t grid_full[3];
};


// Plane bounds (per-phase schedule, lattices whose X is a multiple of 32):
// for each segment of 32 consecutive sites (site i in segment i >> PB_SHIFT),
// and for each of a lattice's two buffers, a count of word planes such that
// every word of those sites in planes at or above it is zero.  Sites are
// packed by every sweep and the reaction, so a segment's bound is the largest
// number of words any of its sites uses; a larger bound is always allowed.
// A sweep reads only the planes below its source segment's bound and writes
// the planes below the larger of its new bound and the destination's old one
// (clearing what the destination held above the new content), then stores the
// new bound.  The reaction and overflow reinsertion raise a bound when they
// fill a slot above it.  Both buffers' bounds are set to the full plane count
// at the start of every run, so the first sweep reads and writes every plane.
constexpr uint32_t PB_SHIFT = 5;

// Kernel launchers (lmb_kernels.cu).  Each returns a cudaError_t.
// The z sweep (dim 2) lists in rx_sites the sites whose reaction step could
// change them, when rx_sites is given (rx_cap entries of two words: the site
// and its type << 8 | particle count); launch_reaction then visits only
// those (every site when the list is absent or overflowed rx_cap).
// pb_src / pb_dst (sweeps) and pb (reaction, resolution): the plane bounds of
// the buffers read and written, or null when the lattice keeps none.
cudaError_t launch_sweep(int bytes_per_slot, int slots, int dim, const uint32_t *src, uint32_t *dst,
                         const uint8_t *sites, const Geometry &g, const DevTables &m, RunState *rs,
                         OverflowEntry *list, uint32_t cap, uint32_t *rx_sites, uint32_t rx_cap,
                         const uint32_t *pb_src, uint32_t *pb_dst, cudaStream_t stream);
cudaError_t launch_reaction(int bytes_per_slot, int slots, uint32_t *lat, const uint8_t *sites,
                            const Geometry &g, const DevTables &m, RunState *rs, OverflowEntry *list,
                            uint32_t cap, const uint32_t *rx_sites, uint32_t rx_cap, uint32_t *pb,
                            cudaStream_t stream);
// Also closes the timestep's reaction list (rx_cap: its capacity, 0 when
// there is none).
cudaError_t launch_resolve(int bytes_per_slot, int slots, uint32_t *lat, const uint8_t *sites,
                           const Geometry &g, RunState *rs, OverflowEntry *list, uint32_t cap, uint32_t rx_cap,
                           uint32_t *pb, cudaStream_t stream);
// Sets `count` plane bounds to `planes`.
cudaError_t launch_fill_bounds(uint32_t *pb, uint32_t count, uint32_t planes, cudaStream_t stream);
// count_step / count_ns / counts: RunState's in-run species count (count_step
// ~0u: none).
cudaError_t launch_begin_run(RunState *rs, uint32_t seed, uint32_t first, uint32_t n, uint32_t mode,
                             cudaStream_t stream, uint32_t count_step = ~0u, uint32_t count_ns = 0,
                             unsigned long long *counts = nullptr);
cudaError_t launch_begin_batch(RunState *const *rs_ptrs, const uint32_t *seeds, uint32_t count, uint32_t first,
                               uint32_t n, const uint32_t *firsts, const uint32_t *counts, uint32_t mode,
                               cudaStream_t stream);
cudaError_t launch_gather_states(RunState *const *rs_ptrs, uint32_t count, RunState *out, cudaStream_t stream);
// pb: the plane bounds of `lat` (only the planes below them are read), or
// null.
cudaError_t launch_counts(int bytes_per_slot, int slots, const uint32_t *lat, const Geometry &g,
                          uint32_t ns, unsigned long long *counts, cudaStream_t stream,
                          const uint32_t *pb = nullptr);
// Fails the run (LMB_E_ARG) when the maxima launch_validate left in the run
// state exceed the model's species or site types.
cudaError_t launch_check_contents(RunState *rs, uint32_t ns, uint32_t nst, cudaStream_t stream);
cudaError_t launch_validate(int bytes_per_slot, int slots, const uint32_t *lat, const uint8_t *sites,
                            const Geometry &g, RunState *rs, cudaStream_t stream);
cudaError_t launch_row_major_to_native(int bytes_per_slot, int slots, const void *rm_particles,
                                       const uint8_t *rm_sites, uint32_t *native, uint8_t *sites,
                                       const Geometry &g, RunState *rs, cudaStream_t stream);
cudaError_t launch_native_to_row_major(int bytes_per_slot, int slots, const uint32_t *native,
                                       const uint8_t *sites, void *rm_particles, uint8_t *rm_sites,
                                       const Geometry &g, cudaStream_t stream);

bool slots_supported(int bytes_per_slot, int slots);
void count_launch(uint64_t n = 1);

// Launches kernel k as a link of the timestep chain (programmatic stream
// serialization): the kernel must begin with chain_enter(), which waits for
// the kernel before it, so only the launch itself overlaps that kernel's end.
template <typename... KArgs, typename... Args>
static inline cudaError_t launch_chain(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                                       Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

// Read-only view of a lattice for code outside the C ABI file (the .lm
// writer): its context, geometry, layout and current device buffers.
struct LatticeView {
    lmb_ctx *ctx;
    Geometry g;
    uint32_t bytes_per_slot, slots;
    const uint32_t *particles;
    const uint8_t *sites;
    bool pending;  // an asynchronous run is in flight
};
int lattice_view(const lmb_lattice *lattice, LatticeView *view);

}  // namespace lmb
