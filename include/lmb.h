/*
 * lmb.h -- C ABI of the B200-native MPD-RDME solver (liblmb200.so).
 *
 * The ABI carries plain pointers, sizes and status codes only.  Every entry
 * returns an int status (LMB_OK = 0, negative = error) and never throws.
 * Host pointers are host memory unless a name says "device".  All work of a
 * lattice is ordered on the stream of the context that created it.
 *
 * Each declaration names the reference interface it stands in for (paths
 * relative to the Lattice Microbes source tree).
 */
#ifndef LMB_H
#define LMB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LMB_ABI_VERSION 1

/* Status codes.  The reference throws lm::Exception / InvalidArgException /
 * CUDAException (core/Exceptions.h, cuda/lm_cuda.h:89-92); here the same
 * failures come back as codes and the C++ layer re-raises them. */
#define LMB_OK 0
#define LMB_E_ARG (-1)                 /* InvalidArgException */
#define LMB_E_CUDA (-2)                /* CUDAException */
#define LMB_E_NOMEM (-3)               /* device allocation failed */
#define LMB_E_MODEL (-4)               /* model rejected (e.g. q > 0.5, MpdRdmeSolver.cu:415-421) */
#define LMB_E_STATE (-5)               /* call out of order (no model, wrong lattice kind) */
#define LMB_E_OVERFLOW_EXHAUSTED (-6)  /* "Too many particle overflows" (MpdRdmeSolver.cu:1122-1124) */
#define LMB_E_OVERFLOW_UNRESOLVED (-7) /* "Unable to find an available site" (MpdRdmeSolver.cu:1155-1156) */
#define LMB_E_TIMEOUT (-8)             /* a bounded device wait gave up */
#define LMB_E_UNSUPPORTED (-9)         /* size or layout outside the compiled variants */
#define LMB_E_IO (-10)                 /* IOException: a file could not be created or written */

/* Overflow handlers: parameter "rdme.mpd.overflowhandler" (MpdRdmeSolver.cu:126-146). */
#define LMB_OVERFLOW_CLASSIC 0
#define LMB_OVERFLOW_RELAXED 1

/* Timestep schedules.  FUSED runs the x, y, z sweeps and the reaction of a
 * tile of Ty x Tz full x-rows in shared memory, one launch per timestep;
 * PHASES launches one kernel per sweep, the reaction and the overflow pass
 * (the reference's schedule, MpdRdmeSolver.cu:1011-1090); CLUSTER, for small
 * lattices, holds the whole lattice in the shared memory of one thread-block
 * cluster and runs every timestep of a run in one launch; GRID runs the
 * FUSED tiles of a Ty x Tz plan (0, 0 = the plan with the most tiles, then
 * the least halo, among those that fit) all
 * resident at once, one cooperative launch per run: each block keeps its
 * region in shared memory from one timestep to the next and reloads only its
 * halo rows, which the neighbouring blocks store, after a bounded grid
 * barrier (a wait that gives up ends the run with LMB_E_TIMEOUT).  CLUSTER
 * and GRID: classic overflow handling only; lmb_lattice_set_schedule refuses
 * a lattice (or plan) that does not fit with LMB_E_UNSUPPORTED.  All give
 * the same lattice bit for bit. */
#define LMB_SCHEDULE_FUSED 0
#define LMB_SCHEDULE_PHASES 1
#define LMB_SCHEDULE_CLUSTER 2
#define LMB_SCHEDULE_GRID 3

/* Reaction types (CMESolver.h:79-112). */
#define LMB_REACTION_ZEROTH 0
#define LMB_REACTION_FIRST 1
#define LMB_REACTION_SECOND 2
#define LMB_REACTION_SECOND_SELF 3

typedef struct lmb_ctx lmb_ctx;
typedef struct lmb_model lmb_model;
typedef struct lmb_lattice lmb_lattice;

/* The reaction and diffusion model as the reference solver receives it:
 * CMESolver::buildModel (cme/CMESolver.h:200-201) and
 * RDMESolver::buildDiffusionModel (rdme/RDMESolver.h:57-67), plus the
 * "timestep" parameter and the lattice spacing. */
typedef struct {
    uint32_t number_species;
    uint32_t number_reactions;
    uint32_t number_site_types;
    const uint32_t *reaction_types; /* [R], LMB_REACTION_* */
    const double *K;                /* [R * k_cols], rate constant in column 0 */
    uint32_t k_cols;
    const int32_t *S;               /* [NS * R] stoichiometry, species-major */
    const uint32_t *D;              /* [NS * R] dependency (1 = reactant) */
    const double *DF;               /* [NST * NST * NS] diffusion, m^2/s */
    const uint32_t *RL;             /* [R * NST] reaction locations */
    double timestep;                /* tau, s */
    double lattice_spacing;         /* lambda, m */
} lmb_model_desc;

/* The FP32 per-timestep tables the kernels read (MpdRdmeSolver.cu:232-483,
 * 697-787): T[src][dst][sp], qp0[st], qp1[st][sp], qp2[st][sp][sp], per-reaction
 * order (1..4), 1-based reactants D1/D2, scaled rate, transposed S[rx][sp],
 * RL[rx][st]. */
typedef struct {
    uint32_t number_species;
    uint32_t number_reactions;
    uint32_t number_site_types;
    const float *T;
    const float *qp0;
    const float *qp1;
    const float *qp2;
    const uint32_t *order;
    const uint32_t *D1;
    const uint32_t *D2;
    const float *rate;
    const int8_t *S;
    const uint8_t *RL;
} lmb_tables;

typedef struct {
    int32_t status;         /* LMB_OK or the error that stopped the run */
    uint32_t steps_done;    /* timesteps completed */
    uint32_t failed_step;   /* timestep index that failed (if status != OK) */
    uint32_t unresolved;    /* relaxed handler: particles still queued */
    uint64_t overflows;     /* particles that left a full site */
    uint64_t reactions;     /* reaction events */
} lmb_run_stats;

/* ---- library ------------------------------------------------------------ */
int lmb_abi_version(void);
const char *lmb_status_string(int status);

/* MpdRdmeSolver::initialize seed composition (MpdRdmeSolver.cu:112-123). */
uint32_t lmb_compose_seed(uint32_t seed_top, uint32_t replicate);
/* MpdRdmeSolver::getTimestepSeed (MpdRdmeSolver.cu:987-994). */
uint64_t lmb_timestep_hash(uint32_t seed, uint32_t timestep, uint32_t substep);

/* ---- context: one device, one stream ------------------------------------
 * Replaces the per-solver cudaSetDevice + cudaStreamCreate of
 * ReplicateRunner::run / MpdRdmeSolver::initialize (MpdRdmeSolver.cu:161). */
int lmb_ctx_create(int device, lmb_ctx **out);
/* Uses an existing cudaStream_t (passed as void*) instead of creating one. */
int lmb_ctx_create_on_stream(int device, void *cuda_stream, lmb_ctx **out);
int lmb_ctx_destroy(lmb_ctx *ctx);
void *lmb_ctx_stream(lmb_ctx *ctx);
int lmb_ctx_synchronize(lmb_ctx *ctx);

/* ---- model ---------------------------------------------------------------
 * MpdRdmeSolver::buildModel + buildDiffusionModel + computePropensities +
 * copyModelsToDevice (MpdRdmeSolver.cu:232-483, 697-787) for a lattice of
 * X*Y*Z sites (the rates scale with the site count). */
int lmb_model_create(lmb_ctx *ctx, const lmb_model_desc *desc, uint32_t X, uint32_t Y, uint32_t Z,
                     lmb_model **out);
/* The host half of lmb_model_create alone: fills caller arrays with the
 * tables it would upload (sizes as in lmb_tables).  Needs no device. */
int lmb_tables_build(const lmb_model_desc *desc, uint32_t X, uint32_t Y, uint32_t Z, float *T, float *qp0,
                     float *qp1, float *qp2, uint32_t *order, uint32_t *D1, uint32_t *D2, float *rate,
                     int8_t *S, uint8_t *RL);
/* Same from ready FP32 tables (test and batch use). */
int lmb_model_create_from_tables(lmb_ctx *ctx, const lmb_tables *tables, lmb_model **out);
/* Copies the host copy of the tables out; NULL arrays are skipped. */
int lmb_model_get_tables(const lmb_model *model, float *T, float *qp0, float *qp1, float *qp2,
                         uint32_t *order, uint32_t *D1, uint32_t *D2, float *rate, int8_t *S,
                         uint8_t *RL);
/* MpdRdmeSolver::setReactionRate (MpdRdmeSolver.h:85, .cu:670-695): new
 * rate constant (LM units) for one reaction; tables are rebuilt and uploaded
 * before the next run. */
int lmb_model_set_reaction_rate(lmb_model *model, uint32_t reaction, double rate);
int lmb_model_destroy(lmb_model *model);

/* ---- lattice -------------------------------------------------------------
 * CudaByteLattice / CudaIntLattice (rdme/CudaByteLattice.cu:75-220,
 * CudaIntLattice.cu:78-189): two device particle buffers and the site types.
 * bytes_per_particle 1 = ByteLattice (4 slots per uint32 word), 4 = IntLattice.
 * Native layout: word w of site i = x + y*X + z*X*Y at particles[w*N + i]. */
int lmb_lattice_create(lmb_ctx *ctx, uint32_t X, uint32_t Y, uint32_t Z, uint32_t particles_per_site,
                       uint32_t bytes_per_particle, lmb_lattice **out);
int lmb_lattice_destroy(lmb_lattice *lattice);
/* CudaByteLattice::copyToGPU / copyFromGPU with native host buffers
 * (W*N uint32 words; N site types).  Either pointer may be NULL. */
int lmb_lattice_set_native(lmb_lattice *lattice, const uint32_t *particles, const uint8_t *sites);
int lmb_lattice_get_native(lmb_lattice *lattice, uint32_t *particles, uint8_t *sites);
/* RDMESolver::setLatticeData / setLatticeSitesData (RDMESolver.cpp:144-189):
 * row-major [x][y][z][p] particles (uint8 for byte lattices, uint32 for int
 * lattices) and [x][y][z] site types; each particle is added to the first
 * free slot; ids above number_species or site types >= number_site_types are
 * rejected.  get_row_major is ByteLattice::copyNativeToRowMajorByte
 * (ByteLattice.cpp:371-402). */
int lmb_lattice_set_row_major(lmb_lattice *lattice, const void *particles, const uint8_t *sites,
                              uint32_t number_species, uint32_t number_site_types);
int lmb_lattice_get_row_major(lmb_lattice *lattice, void *particles, uint8_t *sites);
/* Timestep schedule of this lattice: LMB_SCHEDULE_FUSED with tile Ty x Tz
 * (0, 0 = default plan), LMB_SCHEDULE_GRID with tile Ty x Tz (0, 0 = the
 * plan with the most tiles, then the least halo, whose tiles fit on the
 * device at once),
 * LMB_SCHEDULE_PHASES or LMB_SCHEDULE_CLUSTER (Ty, Tz unused).  The reference has fixed block sizes instead
 * (options.cmake:89-95). */
int lmb_lattice_set_schedule(lmb_lattice *lattice, int schedule, uint32_t Ty, uint32_t Tz);
int lmb_lattice_get_schedule(lmb_lattice *lattice, int *schedule, uint32_t *Ty, uint32_t *Tz);
/* Autotuner: times the per-phase schedule, the cluster-resident one where it
 * fits and every fused tile shape that fits for `timesteps` on a saved copy
 * of the lattice state, restores the state and keeps the fastest.  The
 * grid-resident schedule is chosen only by lmb_lattice_set_schedule: its
 * cooperative launch does not overlap other lattices' runs on other streams,
 * which fused launches do. */
int lmb_lattice_autotune(lmb_lattice *lattice, const lmb_model *model, uint32_t seed, uint32_t first_timestep,
                         uint32_t timesteps, int *schedule, uint32_t *Ty, uint32_t *Tz, float *best_ms);
/* Device pointers of the current particle buffer and of the site types. */
int lmb_lattice_device_buffers(lmb_lattice *lattice, void **particles, void **sites);
/* ByteLattice::getParticleCounts (ByteLattice.cpp:495-520), computed on the
 * device: counts[s] for s = 0..number_species (counts[0] is 0). */
int lmb_lattice_species_counts(lmb_lattice *lattice, uint32_t number_species, uint64_t *counts);

/* Species counts for callers that cannot allocate device memory (a host
 * program whose own pool allocator owns the device memory, a hook or
 * callback where cudaMalloc would synchronize or exceed a memory cap, a
 * serving loop with a fixed footprint).  No counterpart in the reference: it
 * has no device-side count at all.  `particles` is a native lattice in
 * device memory; `counts` (host, number_species + 1 entries) receives the
 * totals as lmb_lattice_species_counts gives them.  The device-side totals
 * live in one fixed 32 KiB array per device that stays allocated until the
 * process exits; sizes above LMB_NOALLOC_MAX_SPECIES species return
 * LMB_E_UNSUPPORTED.  The first call on a device looks up that array's
 * address, so make it before any stream capture.  Each call clears the array
 * on `cuda_stream` before counting and waits for the result; calls whose
 * work overlaps on the GPU share the array and race.  The looked-up address
 * is kept for the life of the process: after cudaDeviceReset on a device
 * (which ends every lmb handle on it too) this entry point must not be
 * called on that device again. */
#define LMB_NOALLOC_MAX_SPECIES 4095
int lmb_species_counts_noalloc(const uint32_t *particles, uint32_t X, uint32_t Y, uint32_t Z,
                               uint32_t particles_per_site, uint32_t bytes_per_particle, uint32_t number_species,
                               uint64_t *counts, void *cuda_stream);

/* ---- timesteps -----------------------------------------------------------
 * number_timesteps calls of MpdRdmeSolver::runTimestep (MpdRdmeSolver.cu:
 * 996-1193), timestep indices first_timestep.., with `seed` the composed
 * 32-bit solver seed.  Overflow handling runs on the device; the classic
 * handler gives the reference's result for the reinsertion order sorted by
 * (sweep, site, slot).  Blocks until done; stats may be NULL. */
int lmb_run(lmb_lattice *lattice, const lmb_model *model, uint32_t seed, uint32_t first_timestep,
            uint32_t number_timesteps, int overflow_mode, lmb_run_stats *stats);
/* Enqueues the same work and returns; lmb_run_wait blocks and reports. */
int lmb_run_async(lmb_lattice *lattice, const lmb_model *model, uint32_t seed, uint32_t first_timestep,
                  uint32_t number_timesteps, int overflow_mode);
int lmb_run_wait(lmb_lattice *lattice, lmb_run_stats *stats);
/* One solve queued as a whole on the lattice's stream: new native contents
 * (lmb_lattice_set_native; either pointer NULL keeps that part), the run
 * (lmb_run_async), and the final particles copied to out_particles (NULL:
 * not copied) -- the copyToGPU / timesteps / copyFromGPU of a trajectory
 * (MpdRdmeSolver.cu:485-668, CudaByteLattice.cu:128-140) with no host wait
 * between them.  New contents are checked on the device ahead of the
 * timesteps: a species id above the model's or a site type beyond it fails
 * the solve with LMB_E_ARG (from lmb_run_wait, no timestep run, the uploaded
 * contents left in place).  lmb_run_wait ends the solve; the host
 * buffers must stay valid until then, and pinned host buffers let the copies
 * overlap work on other streams (two lattices on two contexts pipeline their
 * solves this way).  After a failed run out_particles is not the partial
 * lattice: lmb_lattice_get_native after lmb_run_wait gives it. */
int lmb_run_native_async(lmb_lattice *lattice, const lmb_model *model, uint32_t seed, uint32_t first_timestep,
                         uint32_t number_timesteps, int overflow_mode, const uint32_t *in_particles,
                         const uint8_t *in_sites, uint32_t *out_particles);
/* lmb_run_async that also takes the lattice's species totals at the end of
 * the run (recordSpeciesCounts, MpdRdmeSolver.cu:933-942, with
 * ByteLattice::getParticleCounts, ByteLattice.cpp:495-520) inside the run's
 * own work: on the fused schedule the last timestep's kernel adds the
 * particles of the sites each block stores into per-block histograms, one
 * atomic per species, and the overflow resolution adds those it puts back;
 * on the per-phase schedule one pass after the last timestep reads only the
 * word planes below each segment's plane bound.  The totals come back with
 * the run state: lmb_run_counts_wait returns them, counts[0..number_species]
 * as lmb_lattice_species_counts gives them, with no further launch or
 * synchronization. */
int lmb_run_counts_async(lmb_lattice *lattice, const lmb_model *model, uint32_t seed, uint32_t first_timestep,
                         uint32_t number_timesteps, int overflow_mode, uint32_t number_species);
int lmb_run_counts_wait(lmb_lattice *lattice, lmb_run_stats *stats, uint64_t *counts);

/* lmb_run with a CUDA event pair around every kernel on the lattice's
 * stream; phase_ms[6] / phase_launches[6] receive the summed device time and
 * launch count of the x, y, z sweeps, the reaction, the overflow kernel and
 * the fused timestep kernel. */
int lmb_run_profiled(lmb_lattice *lattice, const lmb_model *model, uint32_t seed, uint32_t first_timestep,
                     uint32_t number_timesteps, int overflow_mode, float *phase_ms, uint32_t *phase_launches,
                     lmb_run_stats *stats);

/* ---- batches ---------------------------------------------------------------
 * Many lattices (replicates, uneven sizes) advanced together: one launch per
 * timestep covers every tile of every lattice, replayed from a captured CUDA
 * graph.  Replaces running the reference's ReplicateRunner threads
 * (core/ReplicateRunner.cpp:84-166), one MpdRdmeSolver each, on one device.
 * All lattices share the context, slot count (16 at most) and bytes per
 * slot; each has its own model (rates scale with its site count) and its own
 * seed.  The batch tiles each lattice with its largest efficient tile (the
 * batch itself fills the GPU).  Each lattice gives the same result as lmb_run
 * on it. */
typedef struct lmb_batch lmb_batch;
int lmb_batch_create(lmb_ctx *ctx, uint32_t count, lmb_lattice *const *lattices, const lmb_model *const *models,
                     lmb_batch **out);
/* seeds[count]; stats[count] may be NULL.  Returns the first error of any
 * lattice; the others still ran. */
int lmb_batch_run(lmb_batch *batch, const uint32_t *seeds, uint32_t first_timestep, uint32_t number_timesteps,
                  int overflow_mode, lmb_run_stats *stats);
int lmb_batch_run_async(lmb_batch *batch, const uint32_t *seeds, uint32_t first_timestep,
                        uint32_t number_timesteps, int overflow_mode);
int lmb_batch_wait(lmb_batch *batch, lmb_run_stats *stats);
/* Per-lattice timestep ranges: lattice j runs timesteps firsts[j] ..
 * firsts[j] + counts[j] - 1 with seeds[j]; the launches cover the longest
 * range and a lattice whose range is done sits them out.  Each lattice still
 * gives lmb_run's result for its range.  Used for continuous batching, where
 * the lattices of a batch are at different points of their runs. */
int lmb_batch_run_ranges_async(lmb_batch *batch, const uint32_t *seeds, const uint32_t *firsts,
                               const uint32_t *counts, int overflow_mode);
/* Replaces the batch's lattices (same context, slot count and bytes per
 * slot); no run may be pending. */
int lmb_batch_set_lattices(lmb_batch *batch, uint32_t count, lmb_lattice *const *lattices,
                           const lmb_model *const *models);
/* Chooses the tile shape of each lattice size in the batch by timing: for
 * each size (largest total first) every tile shape the batch kernel can use
 * runs `number_timesteps` timesteps of the whole batch from the lattices'
 * current states, and the fastest is kept (best_ms: that run's time).  The
 * lattices end where they started.  The choice holds for lattices of that
 * size from then on, after lmb_batch_set_lattices too.  No counterpart in the
 * reference (one solver per lattice, fixed launch geometry). */
int lmb_batch_autotune(lmb_batch *batch, const uint32_t *seeds, uint32_t first_timestep,
                       uint32_t number_timesteps, float *best_ms);
/* The tile plan: Ty[j] x Tz[j] x-rows per block for lattice j. */
int lmb_batch_plan(lmb_batch *batch, uint32_t *Ty, uint32_t *Tz);
int lmb_batch_destroy(lmb_batch *batch);

/* ---- serving: continuous batching of solves ------------------------------------
 * A request is one MPD-RDME solve: a model (as lmb_model_create takes it), a
 * native lattice with its site types, the composed seed and a timestep
 * count.  The server keeps every admitted solve's lattice resident on the
 * device and advances all of them together, one launch per timestep for
 * all (lmb_batch_run_ranges_async).  Each lmb_server_step admits queued
 * requests in arrival order while fewer than max_active solves are resident
 * and their device bytes fit hbm_budget_bytes, runs chunk_timesteps
 * timesteps of every resident solve (fewer for a solve near its end), and
 * retires the solves that are done.  Solves of at least 131,072 sites
 * (which fill the device alone) run their chunks on their own instead, on
 * two streams beside the small solves' batch (each stream one solve at a
 * time, in arrival order), with the per-phase schedule when they hold 0.05
 * particles per site or more.  A solve's result is lmb_run's result for it
 * alone, bit for bit.  Replaces the reference's one-solver-per-thread
 * replicate runner (core/ReplicateRunner.cpp:84-166) for many independent
 * solves on one device. */
typedef struct lmb_server lmb_server;
typedef struct {
    uint64_t id;                 /* caller's tag, returned with the result */
    const lmb_model_desc *model; /* copied by lmb_server_submit */
    uint32_t X, Y, Z;
    const uint32_t *particles;   /* native lattice, copied */
    const uint8_t *sites;        /* site types, copied */
    uint32_t seed;               /* composed 32-bit solver seed */
    uint32_t timesteps;          /* timesteps 0 .. timesteps - 1 */
} lmb_request;
typedef struct {
    uint64_t id;
    lmb_run_stats stats;         /* status LMB_E_NOMEM: larger than the budget */
    uint32_t X, Y, Z;
    uint32_t number_species;
    double t_submit, t_admit, t_done; /* seconds on the server's steady clock */
} lmb_result_info;
typedef struct {
    uint32_t active, queued, ready, peak_active;
    uint64_t bytes_in_use, peak_bytes, completed;
    uint64_t next_ready_words;   /* particle words of the next result */
} lmb_server_status_info;
int lmb_server_create(lmb_ctx *ctx, uint32_t particles_per_site, uint32_t bytes_per_particle,
                      uint64_t hbm_budget_bytes, uint32_t max_active, uint32_t chunk_timesteps,
                      lmb_server **out);
int lmb_server_destroy(lmb_server *server);
int lmb_server_submit(lmb_server *server, const lmb_request *request);
/* Admit, run one chunk, retire; blocks until the chunk is done. */
int lmb_server_step(lmb_server *server, uint32_t *active, uint32_t *queued);
/* Pops the oldest finished solve: its info, native lattice (optional) and
 * species counts [0..number_species] (optional).  LMB_E_STATE when none. */
int lmb_server_pop_result(lmb_server *server, lmb_result_info *info, uint32_t *particles,
                          uint64_t particles_words, uint64_t *species_counts, uint32_t counts_len);
int lmb_server_status(const lmb_server *server, lmb_server_status_info *status);

/* ---- CME ensembles -----------------------------------------------------------
 * Many independent replicates of a well-mixed model, each advanced by the
 * direct method of lm::cme::GillespieDSolver (cme/GillespieDSolver.cpp:
 * 107-382), one GPU thread per replicate.  Replaces running one
 * GillespieDSolver per replicate thread (core/ReplicateRunner.cpp:84-166).
 * The model arguments are those of CMESolver::buildModel (cme/CMESolver.h:
 * 200-201) with reaction types LMB_REACTION_ZEROTH..SECOND_SELF; at most 32
 * species and 64 reactions.  Counts are int32 and propensities FP32; time is
 * FP64.  Random numbers come from the counter hash keyed by (seed, replicate,
 * event), so a replicate's trajectory depends on neither the ensemble size
 * nor how the run is cut into segments. */
typedef struct lmb_cme lmb_cme;
int lmb_cme_create(lmb_ctx *ctx, uint32_t number_species, uint32_t number_reactions,
                   const uint32_t *reaction_types, const double *K, uint32_t k_cols, const int32_t *S,
                   const uint32_t *D, uint32_t replicates, lmb_cme **out);
int lmb_cme_destroy(lmb_cme *cme);
/* Initial counts: [number_species] for every replicate (per_replicate = 0) or
 * [replicates][number_species].  Takes effect at the next lmb_cme_begin. */
int lmb_cme_set_initial_counts(lmb_cme *cme, const uint32_t *counts, int per_replicate);
/* Starts a run to t_end recording the counts every write_interval seconds
 * from t = 0, as GillespieDSolver records them (the counts before the first
 * event past each write time, GillespieDSolver.cpp:202-213, 329-338).
 * lmb_cme_entries gives the number of records. */
int lmb_cme_begin(lmb_cme *cme, uint32_t seed, double t_end, double write_interval);
/* Enqueues the segment up to time `until` (clamped to t_end) on the
 * context stream and returns. */
int lmb_cme_advance_async(lmb_cme *cme, double until);
/* begin + one segment to t_end + wait. */
int lmb_cme_run(lmb_cme *cme, uint32_t seed, double t_end, double write_interval);
int lmb_cme_entries(const lmb_cme *cme, uint32_t *entries);
/* Waits and copies the records out as [replicates][entries][number_species]
 * (one SpeciesCounts data set per replicate). */
int lmb_cme_get_counts(lmb_cme *cme, uint32_t *counts);
/* Device pointer of the records, laid out [entries][number_species][replicates]. */
int lmb_cme_device_counts(lmb_cme *cme, void **counts);
/* Waits; total events applied and replicates that reached t_end. */
int lmb_cme_stats(lmb_cme *cme, uint64_t *events, uint32_t *finished);
/* Kernel form: LMB_CME_KERNEL_AUTO (default) runs models of up to 8 species
 * and 16 reactions whose stoichiometric changes lie in -8..7 with the rates
 * and reactant codes in registers; LMB_CME_KERNEL_GENERIC runs every model
 * from shared-memory tables.  Both give the same trajectories bit for bit. */
#define LMB_CME_KERNEL_AUTO 0
#define LMB_CME_KERNEL_GENERIC 1
int lmb_cme_set_kernel(lmb_cme *cme, int kernel);

/* Launch counters for the bench's kernel accounting. */
uint64_t lmb_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif
