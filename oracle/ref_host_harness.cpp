/*
 * ref_host_harness.cpp -- runs the reference's own MPD-RDME device functions
 * on the CPU, as a pin for the C restatement in mpd_oracle.c.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into oracle/_ref/ from
 * the reference sources where they lie; nothing from the reference is copied
 * here.  The translation unit #includes, by path through -I:
 *   src/cuda/constant.cu                  (the __constant__ model symbols)
 *   src/rdme/dev/xor_random_dev.cu        (counter hash)
 *   src/rdme/dev/lattice_sim_1d_dev.cu    (window and apron loaders)
 *   src/rdme/dev/{byte,word}_diffusion_1d_dev.cu  (choices, propagation)
 *   src/rdme/dev/{byte,word}_reaction_dev.cu      (reaction functions)
 * and links src/rdme/{Lattice,ByteLattice,IntLattice}.cpp for the classic
 * overflow search.  shim/cuda.h turns the CUDA qualifiers into host C++.
 *
 * What is restated here (the kernel bodies live in MpdRdmeSolver.cu, which
 * needs HDF5/protobuf and cannot be compiled in this tree): the launch
 * geometry of MpdRdmeSolver.cu:1195-1261, the order in which a block's
 * threads call the device functions in mpd_{x,y,z}_kernel
 * (MpdRdmeSolver.cu:1342-1490), the precomputed-table propensity sum of
 * precomp_reaction_kernel (:1613-1638) and the classic overflow loop
 * (:1103-1189).  Blocks run one after another and the threads of a block run
 * phase by phase between the kernel's __syncthreads() calls.
 *
 * Build variants (one .so each): -DREF_BYTE or -DREF_INT, with
 * MPD_LATTICE_MAX_OCCUPANCY set in the generated config.h.
 */
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <vector>
#include <algorithm>

#include "cuda.h"
#include "config.h"

lmb_shim_dim3 threadIdx, blockIdx, blockDim, gridDim;

#if defined(REF_BYTE)
#define MPD_WORDS_PER_SITE (MPD_LATTICE_MAX_OCCUPANCY / 4)
#elif defined(REF_INT)
#define MPD_WORDS_PER_SITE (MPD_LATTICE_MAX_OCCUPANCY)
#else
#error "define REF_BYTE or REF_INT"
#endif
#define MPD_APRON_SIZE 1

/* The device paths for __CUDA_ARCH__ >= 350 (device malloc in
 * evaluateReaction, __ldg reads) are the ones the reference build runs. */
#define __CUDA_ARCH__ 1000
#include "cuda/constant.cu"
namespace refdev {
#include "rdme/dev/xor_random_dev.cu"
#include "rdme/dev/lattice_sim_1d_dev.cu"
#if defined(REF_BYTE)
#include "rdme/dev/byte_diffusion_1d_dev.cu"
#include "rdme/dev/byte_reaction_dev.cu"
#else
#include "rdme/dev/word_diffusion_1d_dev.cu"
#include "rdme/dev/word_reaction_dev.cu"
#endif
}  // namespace refdev
#undef __CUDA_ARCH__

#include "rdme/Lattice.h"
#include "rdme/ByteLattice.h"
#include "rdme/IntLattice.h"

using namespace refdev;

static const unsigned REF_LIST_CAP_C = TUNE_MPD_MAX_PARTICLE_OVERFLOWS;
#include "ref_classic.h"


/* Model tables kept alive for the duration of a run. */
static std::vector<float> g_T, g_qp0, g_qp1, g_qp2, g_rate;
static std::vector<unsigned> g_order, g_sitesR, g_D1, g_D2;
static std::vector<int8_t> g_S;
static std::vector<uint8_t> g_RL;
static unsigned g_X, g_Y, g_Z;

extern "C" int ref_words_per_site() { return (int)REF_WORDS; }
extern "C" int ref_slots_per_site() { return MPD_LATTICE_MAX_OCCUPANCY; }
extern "C" int ref_list_capacity() { return (int)REF_LIST_CAP_C; }

extern "C" uint32_t ref_device_hash(uint64_t key, uint64_t th)
{
    return getRandomHash((unsigned long long)key, (unsigned long long)th);
}

extern "C" float ref_device_hash_float(uint32_t v1, uint32_t shift, uint32_t v2, uint64_t th)
{
    return getRandomHashFloat(v1, shift, v2, (unsigned long long)th);
}

extern "C" float ref_reaction_probability(float rate)
{
    return calculateReactionProbability(rate);
}

extern "C" int ref_set_model(uint32_t X, uint32_t Y, uint32_t Z, uint32_t ns, uint32_t nst, uint32_t nr,
                             const float *T, const float *qp0, const float *qp1, const float *qp2,
                             const uint32_t *order, const uint32_t *D1, const uint32_t *D2,
                             const float *rate, const int8_t *S, const uint8_t *RL)
{
    if (nst > 256) return -1;
    g_X = X; g_Y = Y; g_Z = Z;
    g_T.assign(T, T + (size_t)nst * nst * ns);
    g_qp0.assign(qp0, qp0 + nst);
    g_qp1.assign(qp1, qp1 + (size_t)nst * ns);
    g_qp2.assign(qp2, qp2 + (size_t)nst * ns * ns);
    g_order.assign(order, order + nr);
    g_sitesR.assign(nr, 0u);
    g_D1.assign(D1, D1 + nr);
    g_D2.assign(D2, D2 + nr);
    g_rate.assign(rate, rate + nr);
    g_S.assign(S, S + (size_t)nr * ns);
    g_RL.assign(RL, RL + (size_t)nr * nst);
    if (g_order.empty()) { g_order.push_back(0); g_sitesR.push_back(0); g_D1.push_back(0); g_D2.push_back(0); g_rate.push_back(0); }
    if (g_S.empty()) g_S.push_back(0);
    if (g_RL.empty()) g_RL.push_back(0);
    /* The values MpdRdmeSolver::buildDiffusionModel copies to the symbols. */
    numberSpeciesC = ns;
    numberSiteTypesC = nst;
    numberReactionsC = nr;
    latticeXSizeC = X;
    latticeYSizeC = Y;
    latticeZSizeC = Z;
    global_latticeZSizeC = Z;
    latticeXYSizeC = X * Y;
    latticeXYZSizeC = X * Y * Z;
    global_latticeXYZSizeC = X * Y * Z;
    TC = g_T.data();
    return 0;
}

/* MpdRdmeSolver.cu:1195-1214 (3-D grid launch). */
static unsigned x_block_size(unsigned X)
{
    unsigned bx = std::min((unsigned)TUNE_MPD_X_BLOCK_MAX_X_SIZE, X);
    if ((X / bx) * bx != X) {
        for (unsigned tryx = 32; tryx < TUNE_MPD_X_BLOCK_MAX_X_SIZE; tryx += 32)
            if (X % tryx == 0) bx = tryx;
    }
    return bx;
}

static void set_thread(unsigned tx, unsigned ty, unsigned tz)
{
    threadIdx.x = tx; threadIdx.y = ty; threadIdx.z = tz;
}

static void sweep_x(const unsigned *in, const uint8_t *sites, unsigned *out, uint64_t th, unsigned *list)
{
    const unsigned bxs = x_block_size(g_X);
    static unsigned window[MPD_X_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    static unsigned choices[MPD_X_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    static uint8_t sitesWindow[MPD_X_WINDOW_SIZE];
    blockDim.x = bxs; blockDim.y = 1; blockDim.z = 1;
    for (unsigned bz = 0; bz < g_Z; bz++)
        for (unsigned by = 0; by < g_Y; by++)
            for (unsigned bx = 0; bx < g_X / bxs; bx++) {
                blockIdx.x = bx; blockIdx.y = by; blockIdx.z = bz;
                for (unsigned t = 0; t < bxs; t++) {
                    set_thread(t, 0, 0);
                    unsigned lx = bx * bxs + t, li = bz * latticeXYSizeC + by * latticeXSizeC + lx;
                    copyXWindowFromLattice(bx, in, window, li, lx, t + MPD_APRON_SIZE);
                    copyXWindowFromSites(bx, sites, sitesWindow, li, lx, t + MPD_APRON_SIZE);
                }
                for (unsigned t = 0; t < bxs; t++) {
                    set_thread(t, 0, 0);
                    unsigned lx = bx * bxs + t, li = bz * latticeXYSizeC + by * latticeXSizeC + lx;
                    makeXDiffusionChoices(window, sitesWindow, choices, li, lx, t + MPD_APRON_SIZE, bxs, th);
                }
                for (unsigned t = 0; t < bxs; t++) {
                    set_thread(t, 0, 0);
                    unsigned lx = bx * bxs + t, li = bz * latticeXYSizeC + by * latticeXSizeC + lx;
                    unsigned wi = t + MPD_APRON_SIZE;
                    performPropagation(out, window, choices, li, wi - 1, wi, wi + 1, MPD_X_WINDOW_SIZE, list);
                }
            }
}

static void sweep_y(const unsigned *in, const uint8_t *sites, unsigned *out, uint64_t th, unsigned *list)
{
    const unsigned BX = TUNE_MPD_Y_BLOCK_X_SIZE, BY = TUNE_MPD_Y_BLOCK_Y_SIZE;
    static unsigned window[MPD_Y_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    static unsigned choices[MPD_Y_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    static uint8_t sitesWindow[MPD_Y_WINDOW_SIZE];
    blockDim.x = BX; blockDim.y = BY; blockDim.z = 1;
    for (unsigned bz = 0; bz < g_Z; bz++)
        for (unsigned by = 0; by < g_Y / BY; by++)
            for (unsigned bx = 0; bx < g_X / BX; bx++) {
                blockIdx.x = bx; blockIdx.y = by; blockIdx.z = bz;
                for (int phase = 0; phase < 3; phase++)
                    for (unsigned ty = 0; ty < BY; ty++)
                        for (unsigned tx = 0; tx < BX; tx++) {
                            set_thread(tx, ty, 0);
                            unsigned ly = by * BY + ty;
                            unsigned li = bz * latticeXYSizeC + ly * latticeXSizeC + bx * BX + tx;
                            unsigned wy = ty + MPD_APRON_SIZE, wi = wy * BX + tx;
                            if (phase == 0) {
                                copyYWindowFromLattice(in, window, li, ly, wi, wy);
                                copyYWindowFromSites(sites, sitesWindow, li, ly, wi, wy);
                            } else if (phase == 1) {
                                makeYDiffusionChoices(window, sitesWindow, choices, li, ly, wi, wy, th);
                            } else {
                                performPropagation(out, window, choices, li, wi - BX, wi, wi + BX, MPD_Y_WINDOW_SIZE, list);
                            }
                        }
            }
}

static void sweep_z(const unsigned *in, const uint8_t *sites, unsigned *out, uint64_t th, unsigned *list)
{
    const unsigned BX = TUNE_MPD_Z_BLOCK_X_SIZE, BZ = TUNE_MPD_Z_BLOCK_Z_SIZE;
    static unsigned window[MPD_Z_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    static unsigned choices[MPD_Z_WINDOW_SIZE * MPD_WORDS_PER_SITE];
    static uint8_t sitesWindow[MPD_Z_WINDOW_SIZE];
    blockDim.x = BX; blockDim.y = 1; blockDim.z = BZ;
    for (unsigned bz = 0; bz < g_Z / BZ; bz++)
        for (unsigned by = 0; by < g_Y; by++)
            for (unsigned bx = 0; bx < g_X / BX; bx++) {
                blockIdx.x = bx; blockIdx.y = by; blockIdx.z = bz;
                for (int phase = 0; phase < 3; phase++)
                    for (unsigned tz = 0; tz < BZ; tz++)
                        for (unsigned tx = 0; tx < BX; tx++) {
                            set_thread(tx, 0, tz);
                            unsigned lz = bz * BZ + tz;
                            unsigned li = lz * latticeXYSizeC + by * latticeXSizeC + bx * BX + tx;
                            unsigned wz = tz + MPD_APRON_SIZE, wi = wz * BX + tx;
                            if (phase == 0) {
                                copyZWindowFromLattice(in, window, li, lz, wi, wz);
                                copyZWindowFromSites(sites, sitesWindow, li, lz, wi, wz);
                            } else if (phase == 1) {
                                makeZDiffusionChoices(window, sitesWindow, choices, li, lz, wi, wz, th);
                            } else {
                                performPropagation(out, window, choices, li, wi - BX, wi, wi + BX, MPD_Z_WINDOW_SIZE, list);
                            }
                        }
            }
}

/* One thread of precomp_reaction_kernel: the table sum (MpdRdmeSolver.cu:
 * 1613-1638) followed by the reference's reaction functions. */
static void reaction_site(unsigned *lat, const uint8_t *sites, unsigned li, uint64_t th, unsigned *list,
                          uint64_t *reactions)
{
    unsigned particles[MPD_WORDS_PER_SITE];
    for (unsigned w = 0; w < MPD_WORDS_PER_SITE; w++) particles[w] = lat[li + w * latticeXYZSizeC];
    uint8_t siteType = sites[li];
    const unsigned NS = numberSpeciesC;
#if defined(REF_BYTE)
    typedef uint8_t slot_t;
    const slot_t *p = (const slot_t *)particles;
#else
    typedef unsigned slot_t;
    const slot_t *p = particles;
#endif
    float total = g_qp0[siteType];
    for (unsigned i = 0; i < MPD_LATTICE_MAX_OCCUPANCY; i++) {
        slot_t p1 = p[i];
        if (p1 > 0) {
            total += g_qp1[siteType * NS + (p1 - 1)];
            for (unsigned j = i + 1; j < MPD_LATTICE_MAX_OCCUPANCY; j++) {
                slot_t p2 = p[j];
                if (p2 > 0) total += g_qp2[siteType * NS * NS + (p1 - 1) * NS + (p2 - 1)];
            }
        }
    }
    if (total == 0.0f) return;
    float prob = calculateReactionProbability(total);
    if (!checkForReaction(li, prob, th)) return;
#if defined(REF_BYTE)
    unsigned idx = determineReactionIndex(siteType, (uint8_t *)particles, li, total, th, g_RL.data(), g_order.data(),
                                          g_sitesR.data(), g_D1.data(), g_D2.data(), g_rate.data());
    evaluateReaction(li, siteType, (uint8_t *)particles, idx, list, g_S.data());
#else
    unsigned idx = determineReactionIndex(siteType, particles, li, total, th, g_RL.data(), g_order.data(),
                                          g_sitesR.data(), g_D1.data(), g_D2.data(), g_rate.data());
    evaluateReaction(li, siteType, particles, idx, list, g_S.data());
#endif
    (*reactions)++;
    for (unsigned w = 0; w < MPD_WORDS_PER_SITE; w++) lat[li + w * latticeXYZSizeC] = particles[w];
}

static void reaction(unsigned *lat, const uint8_t *sites, uint64_t th, unsigned *list, uint64_t *reactions)
{
    const unsigned BX = TUNE_MPD_REACTION_BLOCK_X_SIZE, BY = TUNE_MPD_REACTION_BLOCK_Y_SIZE;
    for (unsigned bz = 0; bz < g_Z; bz++)
        for (unsigned by = 0; by < g_Y / BY; by++)
            for (unsigned bx = 0; bx < g_X / BX; bx++)
                for (unsigned ty = 0; ty < BY; ty++)
                    for (unsigned tx = 0; tx < BX; tx++) {
                        unsigned li = bz * latticeXYSizeC + (by * BY + ty) * latticeXSizeC + bx * BX + tx;
                        reaction_site(lat, sites, li, th, list, reactions);
                    }
}

/*
 * Runs nsteps timesteps.  th[4*s + k] is the timestep hash of step s,
 * substep k (computed by the caller with the getTimestepSeed mixing).
 * Returns 0, -6 (overflow list exhausted) or -7 (unplaceable particle).
 */
extern "C" int ref_run(uint32_t *lat, const uint8_t *sites, const uint64_t *th, uint32_t nsteps,
                       uint64_t *overflows_out, uint64_t *reactions_out)
{
    const size_t N = (size_t)g_X * g_Y * g_Z;
    std::vector<unsigned> tmp(N * REF_WORDS);
    std::vector<unsigned> list(1 + 2 * REF_LIST_CAP_C, 0u);
    uint64_t ovf = 0, rx = 0;
    for (uint32_t s = 0; s < nsteps; s++) {
        list[0] = 0;
        std::vector<Entry> entries;
        unsigned mark = 0;
        sweep_x(lat, sites, tmp.data(), th[4 * s + 0], list.data());
        collect(list.data(), mark, list[0], 0, entries); mark = list[0];
        sweep_y(tmp.data(), sites, lat, th[4 * s + 1], list.data());
        collect(list.data(), mark, list[0], 1, entries); mark = list[0];
        sweep_z(lat, sites, tmp.data(), th[4 * s + 2], list.data());
        collect(list.data(), mark, list[0], 2, entries); mark = list[0];
        memcpy(lat, tmp.data(), N * REF_WORDS * sizeof(unsigned));
        if (numberReactionsC > 0) {
            reaction(lat, sites, th[4 * s + 3], list.data(), &rx);
            collect(list.data(), mark, list[0], 3, entries); mark = list[0];
        }
        ovf += list[0];
        int rc = 0;
        if (list[0] > REF_LIST_CAP_C) rc = -6;
        else if (list[0] > 0) rc = classic_reinsert(lat, sites, entries, g_X, g_Y, g_Z);
        if (rc) {
            if (overflows_out) *overflows_out = ovf;
            if (reactions_out) *reactions_out = rx;
            return rc;
        }
    }
    if (overflows_out) *overflows_out = ovf;
    if (reactions_out) *reactions_out = rx;
    return 0;
}

/* Row-major [x][y][z][p] -> native conversion through the reference class
 * (RDMESolver.cpp:144-167 adds each particle with addParticle). */
extern "C" int ref_rowmajor_to_native(uint32_t X, uint32_t Y, uint32_t Z, const void *rowmajor, uint32_t *native_out)
{
    const unsigned S = MPD_LATTICE_MAX_OCCUPANCY;
    RefLattice lattice(X, Y, Z, S);
#if defined(REF_BYTE)
    const uint8_t *rm = (const uint8_t *)rowmajor;
#else
    const uint32_t *rm = (const uint32_t *)rowmajor;
#endif
    size_t index = 0;
    for (unsigned i = 0; i < X; i++)
        for (unsigned j = 0; j < Y; j++)
            for (unsigned k = 0; k < Z; k++)
                for (unsigned l = 0; l < S; l++, index++)
                    if (rm[index] != 0) lattice.addParticle(i, j, k, rm[index]);
    memcpy(native_out, lattice.particles(), (size_t)X * Y * Z * REF_WORDS * sizeof(uint32_t));
    return 0;
}

extern "C" int ref_particle_counts(uint32_t X, uint32_t Y, uint32_t Z, const uint32_t *native, uint32_t max_species,
                                   uint64_t *counts)
{
    RefLattice lattice(X, Y, Z, MPD_LATTICE_MAX_OCCUPANCY);
    memcpy(lattice.particles(), native, (size_t)X * Y * Z * REF_WORDS * sizeof(uint32_t));
    std::map<particle_t, uint> c = lattice.getParticleCounts();
    for (uint32_t s = 0; s <= max_species; s++) counts[s] = c.count(s) ? c[s] : 0;
    return 0;
}
