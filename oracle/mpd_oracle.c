/*
 * mpd_oracle.c -- CPU restatement of the Lattice Microbes MPD-RDME timestep.
 *
 * TEST INFRASTRUCTURE ONLY (the checker); see mpd_oracle.h.  Build with
 * -ffp-contract=off so that no multiply-add is fused: the reference sums and
 * products are evaluated as separate FP32 operations here.
 *
 * Parity pin: tests/test_oracle_vs_reference.py runs this restatement and the
 * reference's own device functions (compiled for the host by
 * oracle/ref_host_harness.cpp) on the same seeded lattices and asserts equal
 * lattices bit for bit.
 */
#include "mpd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Random numbers                                                            */
/* ------------------------------------------------------------------------ */

/* MpdRdmeSolver.cu:987-994 (IntMpdRdmeSolver.cu:840-847): the host mixes
 * (seed, timestep, substep) into one 64-bit value per kernel launch. */
uint64_t orc_timestep_hash(uint32_t seed, uint32_t timestep, uint32_t substep)
{
    uint64_t h = ((((uint64_t)seed << 30) + timestep) << 2) + substep;
    h = h * 3202034522624059733ULL + 4354685564936845319ULL;
    h ^= h >> 20;
    h ^= h << 41;
    h ^= h >> 5;
    h *= 7664345821815920749ULL;
    return h;
}

/* xor_random_dev.cu:46-53: the device hash of (key ^ timestep hash). */
uint32_t orc_hash(uint64_t v, uint64_t th)
{
    v ^= th;
    v = v * 3935559000370003845ULL + 2691343689449507681ULL;
    v ^= v >> 21;
    v ^= v << 37;
    v ^= v >> 4;
    v *= 2685821657736338717ULL;
    return (uint32_t)(v >> 32);
}

/* xor_random_dev.cu:44,66-70: (float)r * 2^-32 with round-to-nearest. */
float orc_hash_float(uint64_t key, uint64_t th)
{
    uint32_t r = orc_hash(key, th);
    volatile float f = (float)r; /* keep the conversion a separate rounding */
    return f * 2.32830643654e-10f;
}

/* byte_diffusion_1d_dev.cu:51-60 / word_diffusion_1d_dev.cu:51-60. */
uint32_t orc_count_bits(uint32_t slots)
{
    if (slots <= 4) return 2;
    if (slots <= 8) return 3;
    return 4;
}

/* MpdRdmeSolver.cu:112-123: seed = (seedTop << 16) | (replicate & 0xFFFF),
 * truncated to 32 bits. */
uint32_t orc_compose_seed(uint32_t seed_top, uint32_t replicate)
{
    return (uint32_t)((seed_top << 16) | (replicate & 0xFFFFu));
}

/* ------------------------------------------------------------------------ */
/* Lattice access (word-planar native layout)                                */
/* ------------------------------------------------------------------------ */

/* ByteLattice.cpp:237-262 (4 uint8 slots per uint32 word, slot 4w+b) and
 * IntLattice.h:122-127 (one uint32 slot per word).  Word w of site i lives at
 * lat[w*N + i]. */
static inline uint32_t slot_get(const orc_model *m, const uint32_t *lat, size_t N,
                                size_t i, uint32_t k)
{
    if (m->bytes_per_slot == 1) {
        uint32_t w = lat[(size_t)(k >> 2) * N + i];
        return (w >> (8u * (k & 3u))) & 0xFFu;
    }
    return lat[(size_t)k * N + i];
}

static inline void site_store(const orc_model *m, uint32_t *lat, size_t N, size_t i,
                              const uint32_t *vals /* slots entries */)
{
    if (m->bytes_per_slot == 1) {
        uint32_t W = m->slots / 4u;
        for (uint32_t w = 0; w < W; w++) {
            uint32_t word = 0;
            for (uint32_t b = 0; b < 4; b++) word |= (vals[w * 4 + b] & 0xFFu) << (8u * b);
            lat[(size_t)w * N + i] = word;
        }
    } else {
        for (uint32_t w = 0; w < m->slots; w++) lat[(size_t)w * N + i] = vals[w];
    }
}

static inline void site_load(const orc_model *m, const uint32_t *lat, size_t N, size_t i,
                             uint32_t *vals)
{
    for (uint32_t k = 0; k < m->slots; k++) vals[k] = slot_get(m, lat, N, i, k);
}

/* byte_diffusion_1d_dev.cu:70-78: out-of-range species or site types give 0. */
static inline float lookup_T(const orc_model *m, uint32_t p, uint32_t src, uint32_t dst)
{
    if ((uint32_t)(p - 1u) >= m->ns || dst >= m->nst || src >= m->nst) return 0.0f;
    return m->T[(size_t)src * m->nst * m->ns + (size_t)dst * m->ns + (p - 1u)];
}

static int push_overflow(orc_overflow *list, uint32_t *count, uint32_t cap,
                         uint32_t site, uint32_t particle, uint32_t phase, uint32_t seq)
{
    uint32_t idx = (*count)++;
    if (idx < cap) {
        list[idx].site = site;
        list[idx].particle = particle;
        list[idx].phase = phase;
        list[idx].seq = seq;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Diffusion sweep                                                           */
/* ------------------------------------------------------------------------ */

/*
 * One 1-D sweep along dim (0 = x, 1 = y, 2 = z), periodic boundaries
 * (config.h.in:61 defines MPD_BOUNDARY_PERIODIC in every build and the loaders
 * test it with #if defined, lattice_sim_1d_dev.cu:141).
 *
 * Per occupied slot k of site i, r = hash float of ((i << cb) | k)
 * (byte_diffusion_1d_dev.cu:114; word_diffusion_1d_dev.cu:106).  The choice is
 * MINUS if r < q(i -> i-1), PLUS if 0.5 <= r < q(i -> i+1) + 0.5, else STAY
 * (byte_diffusion_1d_dev.cu:115-117).  The new content of site i is its
 * stayers, then the PLUS movers of i-1, then the MINUS movers of i+1, each in
 * slot order; the first S are kept and the rest overflow
 * (byte_diffusion_1d_dev.cu:199-269).  Because q <= 0.5 is enforced at model
 * build (MpdRdmeSolver.cu:415-421), "MINUS" is exactly r < q(i -> i-1).
 * Every site's choices are a pure function of (hash, site types), so the
 * block apron recomputation in the reference (byte_diffusion_1d_dev.cu:127-192)
 * yields the same choices as computing each site once, as done here.
 */
int orc_sweep(const orc_model *m, int dim, const uint32_t *src, uint32_t *dst,
              const uint8_t *sites, uint64_t th,
              orc_overflow *list, uint32_t *list_count, uint32_t list_cap,
              uint64_t *overflow_total)
{
    const uint32_t X = m->X, Y = m->Y, Z = m->Z;
    const size_t N = (size_t)X * Y * Z;
    const uint32_t S = m->slots;
    const uint32_t cb = orc_count_bits(S);
    uint32_t newp[3 * 64];
    uint32_t own[64], mn[64], pl[64];
    if (S > 64) return ORC_E_ARG;

    for (uint32_t z = 0; z < Z; z++)
        for (uint32_t y = 0; y < Y; y++)
            for (uint32_t x = 0; x < X; x++) {
                size_t i = (size_t)z * X * Y + (size_t)y * X + x;
                size_t im, ip;
                if (dim == 0) {
                    im = i - x + (x == 0 ? X - 1 : x - 1);
                    ip = i - x + (x == X - 1 ? 0 : x + 1);
                } else if (dim == 1) {
                    size_t base = i - (size_t)y * X;
                    im = base + (size_t)(y == 0 ? Y - 1 : y - 1) * X;
                    ip = base + (size_t)(y == Y - 1 ? 0 : y + 1) * X;
                } else {
                    size_t base = i - (size_t)z * X * Y;
                    im = base + (size_t)(z == 0 ? Z - 1 : z - 1) * X * Y;
                    ip = base + (size_t)(z == Z - 1 ? 0 : z + 1) * X * Y;
                }
                const uint32_t t = sites[i], tm = sites[im], tp = sites[ip];
                site_load(m, src, N, i, own);
                site_load(m, src, N, im, mn);
                site_load(m, src, N, ip, pl);
                uint32_t n = 0;
                /* Stayers of site i. */
                for (uint32_t k = 0; k < S; k++) {
                    uint32_t p = own[k];
                    if (!p) continue;
                    float r = orc_hash_float(((uint64_t)i << cb) | k, th);
                    float qm = lookup_T(m, p, t, tm);
                    float qp = lookup_T(m, p, t, tp);
                    int plus = (r >= 0.5f && r < (qp + 0.5f));
                    int minus = (r < qm);
                    if (!plus && !minus) newp[n++] = p;
                }
                /* PLUS movers of the minus neighbour. */
                for (uint32_t k = 0; k < S; k++) {
                    uint32_t p = mn[k];
                    if (!p) continue;
                    float r = orc_hash_float(((uint64_t)im << cb) | k, th);
                    float qp = lookup_T(m, p, tm, t);
                    if (r >= 0.5f && r < (qp + 0.5f)) newp[n++] = p;
                }
                /* MINUS movers of the plus neighbour. */
                for (uint32_t k = 0; k < S; k++) {
                    uint32_t p = pl[k];
                    if (!p) continue;
                    float r = orc_hash_float(((uint64_t)ip << cb) | k, th);
                    float qm = lookup_T(m, p, tp, t);
                    if (r < qm) newp[n++] = p;
                }
                uint32_t outv[64];
                for (uint32_t k = 0; k < S; k++) outv[k] = k < n ? newp[k] : 0u;
                site_store(m, dst, N, i, outv);
                for (uint32_t k = S; k < n; k++) {
                    push_overflow(list, list_count, list_cap, (uint32_t)i, newp[k],
                                  (uint32_t)dim, k - S);
                    if (overflow_total) (*overflow_total)++;
                }
            }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Reaction                                                                  */
/* ------------------------------------------------------------------------ */

/* byte_reaction_dev.cu:62-102 (MPD_GLOBAL_R_MATRIX branch, the default build):
 * per-reaction propensity from FP32 particle counts.  The self reaction is
 * rate*n*(n-1) with no factor 1/2 in this branch. */
static float rx_propensity(const orc_model *m, uint32_t t, const uint32_t *p, uint32_t rx)
{
    if (!m->RL[(size_t)rx * m->nst + t]) return 0.0f;
    float n1 = 0.0f, n2 = 0.0f;
    for (uint32_t k = 0; k < m->slots; k++) {
        if (p[k] > 0) {
            n1 += (p[k] == m->D1[rx]) ? 1.0f : 0.0f;
            n2 += (p[k] == m->D2[rx]) ? 1.0f : 0.0f;
        }
    }
    switch (m->order[rx]) {
    case ORC_ZERO_ORDER: return m->rate[rx];
    case ORC_FIRST_ORDER: return m->rate[rx] * n1;
    case ORC_SECOND_ORDER: {
        float a = m->rate[rx] * n1;
        return a * n2;
    }
    case ORC_SECOND_ORDER_SELF: {
        float a = m->rate[rx] * n1;
        return a * (n1 - 1.0f);
    }
    default: return 0.0f;
    }
}

/*
 * MpdRdmeSolver.cu:1590-1675 (precomp_reaction_kernel, the MPD_FREAKYFAST
 * default) with byte_reaction_dev.cu:121-258:
 *  - total propensity a = qp0[t] + sum_k qp1[t][p_k] + sum_{k<j} qp2[t][p_k][p_j]
 *    accumulated in FP32 in slot order (:1617-1638);
 *  - p = (float)(1 - exp(-(double)a)) (RNG_CUDA_DOUBLE_PRECISION, :130-137);
 *  - react iff r0 <= p with r0 from key (i<<1)|0 (:141);
 *  - rp = r1 * a, r1 from key (i<<1)|1; scan reactions in index order with
 *    "if prop > 0 { if rp > 0 idx = rx; rp -= prop }" (:154-176);
 *  - drop consumed reactants in slot order, append products by ascending
 *    species id, extra products overflow (:179-258).
 */
int orc_reaction(const orc_model *m, uint32_t *lat, const uint8_t *sites, uint64_t th,
                 orc_overflow *list, uint32_t *list_count, uint32_t list_cap,
                 uint64_t *overflow_total, uint64_t *reactions)
{
    const size_t N = (size_t)m->X * m->Y * m->Z;
    const uint32_t S = m->slots, NS = m->ns;
    uint32_t p[64];
    int32_t *col = (int32_t *)malloc(sizeof(int32_t) * (NS ? NS : 1));
    if (!col) return ORC_E_ARG;

    for (size_t i = 0; i < N; i++) {
        const uint32_t t = sites[i];
        site_load(m, lat, N, i, p);
        float a = m->qp0[t];
        for (uint32_t k = 0; k < S; k++) {
            uint32_t p1 = p[k];
            if (p1 > 0) {
                a += m->qp1[(size_t)t * NS + (p1 - 1)];
                for (uint32_t j = k + 1; j < S; j++) {
                    uint32_t p2 = p[j];
                    if (p2 > 0)
                        a += m->qp2[(size_t)t * NS * NS + (size_t)(p1 - 1) * NS + (p2 - 1)];
                }
            }
        }
        if (a == 0.0f) continue;
        float prob = (float)(1.0 - exp(-(double)a));
        float r0 = orc_hash_float(((uint64_t)i << 1) | 0u, th);
        if (!(prob > 0.0f && r0 <= prob)) continue;

        float rp = orc_hash_float(((uint64_t)i << 1) | 1u, th) * a;
        uint32_t idx = 0;
        for (uint32_t rx = 0; rx < m->nr; rx++) {
            float prop = rx_propensity(m, t, p, rx);
            if (prop > 0.0f) {
                if (rp > 0.0f) idx = rx;
                rp = rp - prop;
            }
        }
        if (reactions) (*reactions)++;

        for (uint32_t s = 0; s < NS; s++) col[s] = m->S[(size_t)idx * NS + s];
        uint32_t n = 0;
        for (uint32_t k = 0; k < S; k++) {
            uint32_t q = p[k];
            if (q > 0) {
                if (col[q - 1] >= 0) p[n++] = q;
                else col[q - 1]++;
            }
        }
        uint32_t seq = 0;
        for (uint32_t s = 0; s < NS; s++) {
            /* A stoichiometry left negative (a reactant missing from the
             * site) adds nothing here; the reference's unsigned loop bound
             * would instead flood the overflow list and throw. */
            for (int32_t j = 0; j < col[s]; j++) {
                if (n < S) p[n++] = s + 1;
                else {
                    push_overflow(list, list_count, list_cap, (uint32_t)i, s + 1, 3u, seq++);
                    if (overflow_total) (*overflow_total)++;
                }
            }
        }
        while (n < S) p[n++] = 0;
        site_store(m, lat, N, i, p);
    }
    free(col);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Overflow handling                                                         */
/* ------------------------------------------------------------------------ */

static int ovf_cmp(const void *a, const void *b)
{
    const orc_overflow *x = (const orc_overflow *)a, *y = (const orc_overflow *)b;
    if (x->phase != y->phase) return x->phase < y->phase ? -1 : 1;
    if (x->site != y->site) return x->site < y->site ? -1 : 1;
    if (x->seq != y->seq) return x->seq < y->seq ? -1 : 1;
    return 0;
}

/* The reference's list order comes from atomicAdd (byte_diffusion_1d_dev.cu:
 * 260-268) and is not deterministic; kernels run in x, y, z, reaction order and
 * each site's own entries are appended in order.  Sorting by (phase, site, seq)
 * picks one order the reference can produce. */
void orc_sort_overflows(orc_overflow *list, uint32_t n)
{
    qsort(list, n, sizeof(orc_overflow), ovf_cmp);
}

/* ByteLattice.cpp:187-206 / IntLattice.cpp:172-190: slots up to the first 0. */
static uint32_t occupancy(const orc_model *m, const uint32_t *lat, size_t N, size_t i)
{
    uint32_t k = 0;
    while (k < m->slots && slot_get(m, lat, N, i, k) != 0) k++;
    return k;
}

/* ByteLattice.cpp:265-289: the particle goes into the first empty slot. */
static int add_particle(const orc_model *m, uint32_t *lat, size_t N, size_t i, uint32_t p)
{
    uint32_t vals[64];
    site_load(m, lat, N, i, vals);
    for (uint32_t k = 0; k < m->slots; k++)
        if (vals[k] == 0) {
            vals[k] = p;
            site_store(m, lat, N, i, vals);
            return 1;
        }
    return 0;
}

/*
 * MpdRdmeSolver.cu:1103-1189: for each overflowed particle, search radius
 * 0..TUNE_MPD_MAX_OVERFLOW_REPLACEMENT_DIST (4, options.cmake:87) and put it
 * into the first site that has a free slot and the same site type.  Candidate
 * sites come from Lattice::getNearbySites (Lattice.cpp:106-128): the shell
 * minDistance < r <= maxDistance (or r == 0 when both are 0), clamped to the
 * lattice (not periodic), visited x-outer, then y, then z.
 */
int orc_reinsert_classic(const orc_model *m, uint32_t *lat, const uint8_t *sites,
                         const orc_overflow *list, uint32_t n)
{
    const uint32_t X = m->X, Y = m->Y, Z = m->Z;
    const size_t N = (size_t)X * Y * Z;
    for (uint32_t e = 0; e < n; e++) {
        const uint32_t idx = list[e].site, particle = list[e].particle;
        const uint32_t xc = idx % X, yc = (idx / X) % Y, zc = idx / (X * Y);
        const uint8_t tc = sites[idx];
        int placed = 0;
        for (uint32_t radius = 0; !placed && radius <= 4; radius++) {
            uint32_t mind = radius > 0 ? radius - 1 : 0, maxd = radius;
            double min2 = (double)(mind * mind), max2 = (double)(maxd * maxd);
            uint32_t x0 = xc >= maxd ? xc - maxd : 0, x1 = (xc + maxd < X) ? xc + maxd : X - 1;
            uint32_t y0 = yc >= maxd ? yc - maxd : 0, y1 = (yc + maxd < Y) ? yc + maxd : Y - 1;
            uint32_t z0 = zc >= maxd ? zc - maxd : 0, z1 = (zc + maxd < Z) ? zc + maxd : Z - 1;
            for (uint32_t x = x0; !placed && x <= x1; x++)
                for (uint32_t y = y0; !placed && y <= y1; y++)
                    for (uint32_t z = z0; !placed && z <= z1; z++) {
                        double dx = (double)x - xc, dy = (double)y - yc, dz = (double)z - zc;
                        double r2 = dx * dx + dy * dy + dz * dz;
                        if (!(r2 <= max2 && (r2 > min2 || mind == maxd))) continue;
                        size_t j = (size_t)z * X * Y + (size_t)y * X + x;
                        if (occupancy(m, lat, N, j) < m->slots && sites[j] == tc) {
                            placed = add_particle(m, lat, N, j, particle);
                        }
                    }
        }
        if (!placed) return ORC_E_OVERFLOW_UNRESOLVED;
    }
    return ORC_OK;
}

/* MpdRdmeSolver.cu:1677-1761 (correct_overflows): each queued particle goes
 * into the first empty slot of its own site, duplicates of one site in list
 * order; what does not fit stays queued for the next timestep. */
int orc_reinsert_relaxed(const orc_model *m, uint32_t *lat, orc_overflow *list, uint32_t *n)
{
    const size_t N = (size_t)m->X * m->Y * m->Z;
    uint32_t kept = 0;
    for (uint32_t e = 0; e < *n; e++) {
        if (!add_particle(m, lat, N, list[e].site, list[e].particle)) {
            orc_overflow o = list[e];
            o.phase = 0; /* carried entries sort ahead of the next step's */
            o.seq = kept;
            list[kept++] = o;
        }
    }
    *n = kept;
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Timestep driver                                                           */
/* ------------------------------------------------------------------------ */

/* MpdRdmeSolver.cu:996-1193: x, y, z sweeps (substeps 0-2, buffer swap after
 * each), the reaction (substep 3, only when there are reactions), then
 * overflow handling. */
int orc_run(const orc_model *m, uint32_t *lat, const uint8_t *sites,
            uint32_t seed, uint32_t step0, uint32_t nsteps, int overflow_mode,
            orc_stats *stats)
{
    const size_t N = (size_t)m->X * m->Y * m->Z;
    const size_t words = (size_t)(m->bytes_per_slot == 1 ? m->slots / 4 : m->slots) * N;
    const uint32_t cap = m->overflow_capacity ? m->overflow_capacity : 2048u;
    uint32_t *tmp = (uint32_t *)malloc(words * sizeof(uint32_t));
    orc_overflow *list = (orc_overflow *)malloc(sizeof(orc_overflow) * ((size_t)cap + 1));
    uint32_t count = 0;
    int rc = ORC_OK;
    if (!tmp || !list) { free(tmp); free(list); return ORC_E_ARG; }
    if (stats) memset(stats, 0, sizeof(*stats));
    uint64_t ovf = 0, rxn = 0;

    for (uint32_t s = 0; s < nsteps; s++) {
        const uint32_t step = step0 + s;
        if (overflow_mode == ORC_OVERFLOW_CLASSIC) count = 0;
        /* Carried relaxed entries keep their slots at the head of the list. */
        uint32_t carried = count;
        orc_sweep(m, 0, lat, tmp, sites, orc_timestep_hash(seed, step, 0), list, &count, cap, &ovf);
        orc_sweep(m, 1, tmp, lat, sites, orc_timestep_hash(seed, step, 1), list, &count, cap, &ovf);
        orc_sweep(m, 2, lat, tmp, sites, orc_timestep_hash(seed, step, 2), list, &count, cap, &ovf);
        memcpy(lat, tmp, words * sizeof(uint32_t));
        if (m->nr > 0)
            orc_reaction(m, lat, sites, orc_timestep_hash(seed, step, 3), list, &count, cap, &ovf, &rxn);
        if (count > cap) { rc = ORC_E_OVERFLOW_EXHAUSTED; break; }
        if (count > 0) {
            /* The carried prefix keeps its order; new entries are sorted. */
            orc_sort_overflows(list + carried, count - carried);
            if (overflow_mode == ORC_OVERFLOW_CLASSIC) {
                rc = orc_reinsert_classic(m, lat, sites, list, count);
                count = 0;
                if (rc) break;
            } else {
                orc_reinsert_relaxed(m, lat, list, &count);
            }
        }
        if (stats) stats->steps_done = s + 1;
    }
    if (stats) {
        stats->overflows = ovf;
        stats->reactions = rxn;
        stats->unresolved = overflow_mode == ORC_OVERFLOW_RELAXED ? count : 0;
    }
    free(tmp);
    free(list);
    return rc;
}

void orc_counts(const orc_model *m, const uint32_t *lat, uint64_t *counts)
{
    const size_t N = (size_t)m->X * m->Y * m->Z;
    memset(counts, 0, sizeof(uint64_t) * (m->ns + 1));
    for (size_t i = 0; i < N; i++)
        for (uint32_t k = 0; k < m->slots; k++) {
            uint32_t p = slot_get(m, lat, N, i, k);
            if (p && p <= m->ns) counts[p]++;
        }
}

/* ------------------------------------------------------------------------ */
/* Host model building                                                       */
/* ------------------------------------------------------------------------ */

/* MpdRdmeSolver.cu:407-421: q = (float)(DF * tau / spacing^2); q > 0.5
 * rejects the model. */
int orc_build_T(uint32_t nst, uint32_t ns, const double *DF, double tau,
                double spacing, float *T_out)
{
    size_t n = (size_t)nst * nst * ns;
    for (size_t i = 0; i < n; i++) {
        float q = (float)(DF[i] * tau / pow(spacing, 2));
        if (q > 0.50f) return ORC_E_ARG;
        T_out[i] = q;
    }
    return ORC_OK;
}

/* MpdRdmeSolver.cu:265-302 (orders, D1/D2) and :697-774 (rates and the
 * qp0/qp1/qp2 tables).  Reaction types follow CMESolver.h:79-112 (0 zeroth,
 * 1 first, 2 second, 3 second-self); reactant indices come from the
 * dependency columns as CMESolver.cpp:340-430 reads them and are passed here
 * already resolved: K[r*kcols] is the rate, and for the reactant ids this
 * restatement takes D1_out/D2_out as inputs (0-based species, ~0 = none). */
int orc_compute_propensities(uint32_t ns, uint32_t nr, uint32_t nst,
                             const uint32_t *rtype, const double *K, uint32_t kcols,
                             const uint32_t *rl_rxn_major, double tau,
                             uint32_t X, uint32_t Y, uint32_t Z,
                             float *rate_out, float *qp0, float *qp1, float *qp2,
                             uint32_t *order_out, uint32_t *D1_io, uint32_t *D2_io)
{
    /* float scale = X*Y*Z (MpdRdmeSolver.cu:730), an unsigned product first. */
    const float scale = (float)(X * Y * Z);
    for (uint32_t r = 0; r < nr; r++) {
        const double k = K[(size_t)r * kcols];
        switch (rtype[r]) {
        case 0: rate_out[r] = (float)(k * tau / (double)(X * Y * Z)); order_out[r] = ORC_ZERO_ORDER; break;
        case 1: rate_out[r] = (float)(k * tau); order_out[r] = ORC_FIRST_ORDER; break;
        case 2: rate_out[r] = (float)(k * tau * X * Y * Z); order_out[r] = ORC_SECOND_ORDER; break;
        case 3: rate_out[r] = (float)(k * tau * X * Y * Z); order_out[r] = ORC_SECOND_ORDER_SELF; break;
        default: return ORC_E_ARG;
        }
    }
    for (uint32_t st = 0; st < nst; st++) {
        const size_t o1 = (size_t)st * ns, o2 = (size_t)st * ns * ns;
        qp0[st] = 0.0f;
        for (uint32_t i = 0; i < ns; i++) {
            qp1[o1 + i] = 0.0f;
            for (uint32_t j = 0; j < ns; j++) qp2[o2 + (size_t)i * ns + j] = 0.0f;
        }
        for (uint32_t r = 0; r < nr; r++) {
            if (!rl_rxn_major[(size_t)r * nst + st]) continue;
            const double k = K[(size_t)r * kcols];
            const uint32_t s1 = D1_io[r], s2 = D2_io[r];
            /* "float += double" rounds once, after a double add (:735-769). */
            switch (rtype[r]) {
            case 0: qp0[st] = (float)((double)qp0[st] + k * tau / (double)scale); break;
            case 1: qp1[o1 + s1] = (float)((double)qp1[o1 + s1] + k * tau); break;
            case 2:
                qp2[o2 + (size_t)s1 * ns + s2] = (float)(k * tau * (double)scale);
                qp2[o2 + (size_t)s2 * ns + s1] = (float)(k * tau * (double)scale);
                break;
            case 3: {
                size_t e = o2 + (size_t)s1 * ns + s1;
                qp2[e] = (float)((double)qp2[e] + k * tau * (double)scale * 2);
                break;
            }
            }
        }
    }
    /* Device D1/D2 are 1-based species ids, 0 = unused (:270-297). */
    for (uint32_t r = 0; r < nr; r++) {
        uint32_t s1 = D1_io[r], s2 = D2_io[r];
        switch (rtype[r]) {
        case 0: D1_io[r] = 0; D2_io[r] = 0; break;
        case 1: D1_io[r] = s1 + 1; D2_io[r] = 0; break;
        case 2: D1_io[r] = s1 + 1; D2_io[r] = s2 + 1; break;
        case 3: D1_io[r] = s1 + 1; D2_io[r] = 0; break;
        }
    }
    return ORC_OK;
}

/* MpdRdmeSolver.cu:312-321: SG[rx*NS + p] = S[p*NR + rx] as int8. */
void orc_transpose_S(uint32_t ns, uint32_t nr, const int32_t *S_species_major, int8_t *S_out)
{
    for (uint32_t rx = 0; rx < nr; rx++)
        for (uint32_t p = 0; p < ns; p++)
            S_out[(size_t)rx * ns + p] = (int8_t)S_species_major[(size_t)p * nr + rx];
}
