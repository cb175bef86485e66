/*
 * mpd_oracle.h -- CPU restatement of the Lattice Microbes MPD-RDME timestep.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the parity tests, smoke() and
 * the bench's cpu_baseline leg compare the CUDA path against.  The product
 * (lattice_microbes_b200) never links, loads or calls it.
 *
 * Every rule below restates the reference's behaviour; each function cites the
 * reference file:line it follows (paths relative to the Lattice Microbes tree).
 * Parity of this restatement with the reference is pinned by tests that run
 * the reference's own device functions, compiled for the host from the
 * reference sources (oracle/ref_host_harness.cpp), on the same inputs.
 */
#ifndef LMB_MPD_ORACLE_H
#define LMB_MPD_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Reaction orders as encoded on the device (byte_reaction_dev.cu:55-58). */
#define ORC_ZERO_ORDER 1
#define ORC_FIRST_ORDER 2
#define ORC_SECOND_ORDER 3
#define ORC_SECOND_ORDER_SELF 4

/* Overflow handling modes (MpdRdmeSolver.cu:126-146). */
#define ORC_OVERFLOW_CLASSIC 0
#define ORC_OVERFLOW_RELAXED 1

/* Error codes shared with the product's C ABI. */
#define ORC_OK 0
#define ORC_E_ARG -1
#define ORC_E_OVERFLOW_EXHAUSTED -6
#define ORC_E_OVERFLOW_UNRESOLVED -7

/* Device-side model tables, already scaled to FP32 per-timestep values. */
typedef struct {
    uint32_t X, Y, Z;
    uint32_t slots;          /* particles per site (S) */
    uint32_t bytes_per_slot; /* 1 = ByteLattice, 4 = IntLattice */
    uint32_t ns, nst, nr;    /* species, site types, reactions */
    const float *T;          /* [nst][nst][ns] transition probabilities */
    const float *qp0;        /* [nst] */
    const float *qp1;        /* [nst][ns] */
    const float *qp2;        /* [nst][ns][ns] */
    const uint32_t *order;   /* [nr] 1..4 */
    const uint32_t *D1;      /* [nr] 1-based reactant ids (0 = none) */
    const uint32_t *D2;      /* [nr] */
    const float *rate;       /* [nr] rate*tau scaled */
    const int8_t *S;         /* [nr][ns] transposed stoichiometry */
    const uint8_t *RL;       /* [nr][nst] reaction locations */
    uint32_t overflow_capacity; /* 2048 in the reference build */
} orc_model;

typedef struct {
    uint64_t overflows;       /* particles that left a full site */
    uint64_t reactions;       /* reaction events */
    uint64_t unresolved;      /* relaxed mode: still queued at the end */
    uint32_t steps_done;
} orc_stats;

/* One overflow record: (site, particle), tagged with the phase that made it. */
typedef struct {
    uint32_t site;
    uint32_t particle;
    uint32_t phase;   /* 0..2 sweeps x/y/z, 3 reaction */
    uint32_t seq;     /* order within the (phase, site) group */
} orc_overflow;

uint64_t orc_timestep_hash(uint32_t seed, uint32_t timestep, uint32_t substep);
uint32_t orc_hash(uint64_t key, uint64_t timestep_hash);
float orc_hash_float(uint64_t key, uint64_t timestep_hash);
uint32_t orc_count_bits(uint32_t slots);
uint32_t orc_compose_seed(uint32_t seed_top, uint32_t replicate);

/* One x/y/z sweep (dim 0/1/2) from src to dst; overflows appended to list. */
int orc_sweep(const orc_model *m, int dim, const uint32_t *src, uint32_t *dst,
              const uint8_t *sites, uint64_t th,
              orc_overflow *list, uint32_t *list_count, uint32_t list_cap,
              uint64_t *overflow_total);

/* Precomputed-table reaction step, in place. */
int orc_reaction(const orc_model *m, uint32_t *lat, const uint8_t *sites, uint64_t th,
                 orc_overflow *list, uint32_t *list_count, uint32_t list_cap,
                 uint64_t *overflow_total, uint64_t *reactions);

/* Canonical ordering of an overflow list: (phase, site, seq). */
void orc_sort_overflows(orc_overflow *list, uint32_t n);

/* Classic host reinsertion (radius search, same site type). */
int orc_reinsert_classic(const orc_model *m, uint32_t *lat, const uint8_t *sites,
                         const orc_overflow *list, uint32_t n);

/* Relaxed reinsertion: into the first free slot of the same site; the
 * particles that do not fit stay queued (returned count in *n). */
int orc_reinsert_relaxed(const orc_model *m, uint32_t *lat,
                         orc_overflow *list, uint32_t *n);

/* Runs nsteps timesteps starting at timestep index step0.  lat is the native
 * word-planar lattice (W*N uint32 words), updated in place. */
int orc_run(const orc_model *m, uint32_t *lat, const uint8_t *sites,
            uint32_t seed, uint32_t step0, uint32_t nsteps, int overflow_mode,
            orc_stats *stats);

/* Particle counts per species id (counts[0..ns]; index 0 unused). */
void orc_counts(const orc_model *m, const uint32_t *lat, uint64_t *counts);

/* Host model building (MpdRdmeSolver.cu:697-774, :407-421, :312-321). */
int orc_build_T(uint32_t nst, uint32_t ns, const double *DF, double tau,
                double spacing, float *T_out);
int orc_compute_propensities(uint32_t ns, uint32_t nr, uint32_t nst,
                             const uint32_t *rtype, const double *K, uint32_t kcols,
                             const uint32_t *rl_rxn_major, double tau,
                             uint32_t X, uint32_t Y, uint32_t Z,
                             float *rate_out, float *qp0, float *qp1, float *qp2,
                             uint32_t *order_out, uint32_t *D1_out, uint32_t *D2_out);
void orc_transpose_S(uint32_t ns, uint32_t nr, const int32_t *S_species_major, int8_t *S_out);

#ifdef __cplusplus
}
#endif
#endif
