/*
 * ref_classic.h -- pieces shared by the host and GPU reference checkers
 * (TEST INFRASTRUCTURE ONLY): the reference lattice classes opened for the
 * checker, the canonical ordering of the overflow list, and the classic host
 * reinsertion loop of MpdRdmeSolver.cu:1103-1189 restated over the reference's
 * own Lattice / ByteLattice / IntLattice code.
 *
 * Expects MPD_WORDS_PER_SITE, MPD_LATTICE_MAX_OCCUPANCY, REF_LIST_CAP_C and
 * REF_BYTE / REF_INT to be defined by the including file.
 */
#ifndef LMB_REF_CLASSIC_H
#define LMB_REF_CLASSIC_H

#include <algorithm>
#include <cstring>
#include <vector>

#include "rdme/Lattice.h"
#include "rdme/ByteLattice.h"
#include "rdme/IntLattice.h"

static const unsigned REF_WORDS = MPD_WORDS_PER_SITE;

/* The native buffers are protected members; the reference's CUDA lattices
 * reach them by derivation, and so does this checker. */
template <class Base>
struct OpenLattice : public Base {
    OpenLattice(lattice_size_t x, lattice_size_t y, lattice_size_t z, unsigned s) : Base(x, y, z, 1.0, s) {}
    uint32_t *particles() { return this->getParticlesMemory(); }
    uint8_t *site_types() { return this->getSitesMemory(); }
};
#if defined(REF_BYTE)
typedef OpenLattice<lm::rdme::ByteLattice> RefLattice;
#else
typedef OpenLattice<lm::rdme::IntLattice> RefLattice;
#endif

struct Entry {
    uint32_t site, particle, phase, seq;
};

/* Collects list entries [from, to) as (phase, site, seq) records; the entries
 * of one site come from one thread, in order. */
static void collect(const unsigned *list, unsigned from, unsigned to, unsigned phase, std::vector<Entry> &out)
{
    std::vector<Entry> seg;
    for (unsigned e = from; e < to && e < REF_LIST_CAP_C; e++)
        seg.push_back(Entry{list[2 * e + 1], list[2 * e + 2], phase, 0});
    std::stable_sort(seg.begin(), seg.end(), [](const Entry &a, const Entry &b) { return a.site < b.site; });
    for (size_t k = 0; k < seg.size(); k++) {
        seg[k].seq = (k > 0 && seg[k - 1].site == seg[k].site) ? seg[k - 1].seq + 1 : 0;
        out.push_back(seg[k]);
    }
}

/* MpdRdmeSolver.cu:1113-1150 with the reference lattice class. */
static int classic_reinsert(unsigned *lat, const uint8_t *sites, const std::vector<Entry> &entries, unsigned g_X,
                            unsigned g_Y, unsigned g_Z)
{
    const size_t N = (size_t)g_X * g_Y * g_Z;
    RefLattice lattice(g_X, g_Y, g_Z, MPD_LATTICE_MAX_OCCUPANCY);
    memcpy(lattice.particles(), lat, N * REF_WORDS * sizeof(uint32_t));
    memcpy(lattice.site_types(), sites, N);
    for (const Entry &e : entries) {
        lattice_size_t x = e.site % g_X, y = (e.site / g_X) % g_Y, z = e.site / (g_X * g_Y);
        bool placed = false;
        for (unsigned radius = 0; !placed && radius <= TUNE_MPD_MAX_OVERFLOW_REPLACEMENT_DIST; radius++) {
            std::vector<lattice_coord_t> near = lattice.getNearbySites(x, y, z, radius > 0 ? radius - 1 : 0, radius);
            for (const lattice_coord_t &s : near) {
                if (lattice.getOccupancy(s.x, s.y, s.z) < lattice.getMaxOccupancy() &&
                    lattice.getSiteType(s.x, s.y, s.z) == lattice.getSiteType(x, y, z)) {
                    lattice.addParticle(s.x, s.y, s.z, e.particle);
                    placed = true;
                    break;
                }
            }
        }
        if (!placed) {
            /* The reference throws here with the host lattice partly updated;
             * the checker keeps that partial state for comparison. */
            memcpy(lat, lattice.particles(), N * REF_WORDS * sizeof(uint32_t));
            return -7;
        }
    }
    memcpy(lat, lattice.particles(), N * REF_WORDS * sizeof(uint32_t));
    return 0;
}

#endif
