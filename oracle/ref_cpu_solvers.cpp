/*
 * ref_cpu_solvers.cpp -- runs the reference's own CPU solvers,
 * lm::rdme::NextSubvolumeSolver and lm::cme::GillespieDSolver, behind a
 * plain C entry point per solver.
 *
 * TEST INFRASTRUCTURE ONLY: the statistical comparator for MPD-RDME and CME
 * ensembles and the timed CPU baseline.  Built by oracle/Makefile into
 * oracle/_ref/ from the reference sources where they lie (nothing is copied):
 *   src/rdme/NextSubvolumeSolver.cpp, src/rdme/RDMESolver.cpp,
 *   src/cme/CMESolver.cpp, src/cme/GillespieDSolver.cpp,
 *   src/rng/RandomGenerator.cpp, src/rng/XORShift.cpp,
 *   src/rdme/Lattice.cpp, src/rdme/ByteLattice.cpp, src/core/Print.cpp,
 *   src/me/MESolver.cpp
 * with config.h from oracle/gen_ref_config.py (no OPT_CUDA: the solvers draw
 * from XORShift, as they do when no GPU is assigned, CMESolver.cpp:95-125)
 * and the stand-in headers of oracle/shim_lm/ in place of the generated
 * protobuf messages and of the HDF5 output queue.
 *
 * Each call builds a solver, initialises it with the parameters the reference
 * reads from a .lm file (seed, maxTime, writeInterval; lattice frames off),
 * gives it the model through the same calls the reference's runSolver makes
 * (CMESolver::buildModel, NextSubvolumeSolver::buildDiffusionModel), runs
 * generateTrajectory() and returns the species counts it recorded.
 */
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "SpeciesCounts.pb.h"
#include "core/DataOutputQueue.h"
#include "core/Exceptions.h"
#include "cme/GillespieDSolver.h"
#include "rdme/ByteLattice.h"
#include "rdme/NextSubvolumeSolver.h"

/* ---- the capturing output queue (one per thread) ----------------------- */

namespace lm {
namespace main {

DataOutputQueue *DataOutputQueue::getInstance()
{
    static thread_local DataOutputQueue queue;
    return &queue;
}

void DataOutputQueue::pushDataSet(uint type, uint, ::google::protobuf::Message *message, void *, size_t,
                                  void (*)(void *, void *, size_t))
{
    if (type == SPECIES_COUNTS) {
        lm::io::SpeciesCounts *sc = dynamic_cast<lm::io::SpeciesCounts *>(message);
        if (sc == NULL) return;
        numberSpecies = (uint)sc->number_species();
        for (int e = 0; e < sc->time_size(); e++) times.push_back(sc->time(e));
        for (int k = 0; k < sc->species_count_size(); k++) counts.push_back((uint32_t)sc->species_count(k));
    } else if (type == BYTE_LATTICE) {
        latticeFrames++;
    }
}

}  // namespace main
}  // namespace lm

namespace {

using lm::main::DataOutputQueue;
using lm::main::ResourceAllocator;

void reset_queue()
{
    lm::Print::verbosityLevel(lm::Print::WARNING);
    DataOutputQueue *q = DataOutputQueue::getInstance();
    q->times.clear();
    q->counts.clear();
    q->numberSpecies = 0;
    q->latticeFrames = 0;
    lm::io::record_walls().clear();
}

int copy_out(uint32_t ns, uint32_t max_entries, double *times, uint32_t *counts, uint32_t *entries)
{
    DataOutputQueue *q = DataOutputQueue::getInstance();
    size_t n = q->times.size();
    if (q->numberSpecies != ns && n > 0) return -2;
    if (entries) *entries = (uint32_t)n;
    size_t m = n < max_entries ? n : max_entries;
    if (times) memcpy(times, q->times.data(), m * sizeof(double));
    if (counts) memcpy(counts, q->counts.data(), m * ns * sizeof(uint32_t));
    return n > max_entries ? -3 : 0;
}

std::map<std::string, std::string> make_params(uint32_t seed, double max_time, double write_interval)
{
    std::map<std::string, std::string> p;
    char buf[64];
    snprintf(buf, sizeof buf, "%u", seed);
    p["seed"] = buf;
    snprintf(buf, sizeof buf, "%.17g", max_time);
    p["maxTime"] = buf;
    snprintf(buf, sizeof buf, "%.17g", write_interval);
    p["writeInterval"] = buf;
    p["latticeWriteInterval"] = "0";
    return p;
}

void set_error(char *err, size_t errlen, const char *what)
{
    if (err && errlen) {
        strncpy(err, what, errlen - 1);
        err[errlen - 1] = 0;
    }
}

/* Exposes the protected lattice so the final state can be read back. */
class NSM : public lm::rdme::NextSubvolumeSolver {
public:
    lm::rdme::Lattice *getLattice() { return lattice; }
};

}  // namespace

extern "C" {

/*
 * One NextSubvolumeSolver trajectory.  Model arguments are those of
 * CMESolver::buildModel (cme/CMESolver.h:200-201, one rate column) and
 * NextSubvolumeSolver::buildDiffusionModel (rdme/NextSubvolumeSolver.h:61):
 * row-major particle lattice [x][y][z][p] (uint8) and site types [x][y][z].
 * `init_counts` must equal the lattice's species totals (the solver checks,
 * NextSubvolumeSolver.cpp:330-338).  Species counts recorded every
 * `write_interval` seconds (entry 0 at t = 0) are copied into
 * times[max_entries] / counts[max_entries][ns]; `final_lattice` (optional)
 * receives the row-major lattice at the end.  Returns 0, or -1 with the
 * solver's exception text in `err`.
 */
int ref_nsm_run(uint32_t ns, uint32_t nr, const uint32_t *init_counts, const uint32_t *rtype, const double *K,
                const int32_t *S, const uint32_t *D, uint32_t nst, const double *DF, const uint32_t *RL, uint32_t X,
                uint32_t Y, uint32_t Z, uint32_t pps, double spacing, const uint8_t *lattice_rm,
                const uint8_t *sites_rm, uint32_t seed, uint32_t replicate, double max_time, double write_interval,
                uint32_t max_entries, double *times, uint32_t *counts, uint32_t *entries, uint8_t *final_lattice,
                char *err, size_t errlen)
{
    try {
        reset_queue();
        std::map<std::string, std::string> params = make_params(seed, max_time, write_interval);
        ResourceAllocator::ComputeResources resources;
        resources.processNumber = 0;
        NSM solver;
        solver.initialize(replicate, &params, &resources);
        std::vector<uint> types(rtype, rtype + nr);
        std::vector<int> Sv(S, S + (size_t)ns * nr);
        std::vector<uint> Dv(D, D + (size_t)ns * nr);
        std::vector<uint> init(init_counts, init_counts + ns);
        solver.buildModel(ns, nr, init.data(), types.data(), K, Sv.data(), Dv.data(), 1);
        std::vector<uint> RLv(RL, RL + (size_t)nr * nst);
        solver.buildDiffusionModel(nst, DF, RLv.data(), X, Y, Z, pps, 1, spacing, lattice_rm, sites_rm, true);
        solver.generateTrajectory();
        if (final_lattice) {
            lm::rdme::Lattice *lat = solver.getLattice();
            size_t idx = 0;
            for (uint32_t x = 0; x < X; x++)
                for (uint32_t y = 0; y < Y; y++)
                    for (uint32_t z = 0; z < Z; z++)
                        for (uint32_t p = 0; p < pps; p++, idx++)
                            final_lattice[idx] =
                                p < lat->getOccupancy(x, y, z) ? (uint8_t)lat->getParticle(x, y, z, p) : 0;
        }
        int rc = copy_out(ns, max_entries, times, counts, entries);
        if (rc) set_error(err, errlen, "species count buffer too small or inconsistent");
        return rc;
    } catch (lm::Exception &e) {
        set_error(err, errlen, e.what());
        return -1;
    } catch (std::exception &e) {
        set_error(err, errlen, e.what());
        return -1;
    }
}

/*
 * One GillespieDSolver trajectory of a well-mixed model (CMESolver::buildModel
 * arguments with k_cols rate columns).  Recording as for ref_nsm_run.
 */
int ref_gillespie_run(uint32_t ns, uint32_t nr, const uint32_t *init_counts, const uint32_t *rtype, const double *K,
                      uint32_t k_cols, const int32_t *S, const uint32_t *D, uint32_t seed, uint32_t replicate,
                      double max_time, double write_interval, uint32_t max_entries, double *times, uint32_t *counts,
                      uint32_t *entries, char *err, size_t errlen)
{
    try {
        reset_queue();
        std::map<std::string, std::string> params = make_params(seed, max_time, write_interval);
        ResourceAllocator::ComputeResources resources;
        resources.processNumber = 0;
        lm::cme::GillespieDSolver solver;
        solver.initialize(replicate, &params, &resources);
        std::vector<uint> types(rtype, rtype + nr);
        std::vector<int> Sv(S, S + (size_t)ns * nr);
        std::vector<uint> Dv(D, D + (size_t)ns * nr);
        std::vector<uint> init(init_counts, init_counts + ns);
        solver.buildModel(ns, nr, init.data(), types.data(), K, Sv.data(), Dv.data(), k_cols);
        solver.generateTrajectory();
        int rc = copy_out(ns, max_entries, times, counts, entries);
        if (rc) set_error(err, errlen, "species count buffer too small or inconsistent");
        return rc;
    } catch (lm::Exception &e) {
        set_error(err, errlen, e.what());
        return -1;
    } catch (std::exception &e) {
        set_error(err, errlen, e.what());
        return -1;
    }
}

/*
 * Wall-clock stamps (steady clock, seconds) of the species-count records of
 * the last trajectory run on this thread, one per record in record order:
 * entry 0 is the record at t = 0, taken after the solver's set-up, and entry
 * k the record at k write intervals.  Returns how many there were; copies at
 * most max_entries.
 */
uint32_t ref_record_walls(double *walls, uint32_t max_entries)
{
    const std::vector<double> &w = lm::io::record_walls();
    const size_t m = w.size() < max_entries ? w.size() : max_entries;
    if (walls && m) memcpy(walls, w.data(), m * sizeof(double));
    return (uint32_t)w.size();
}

}  // extern "C"
