/*
 * lmb_solver.hpp -- C++ solver classes over the C ABI of lmb.h, with the
 * interface of the reference's lm::rdme::MpdRdmeSolver / IntMpdRdmeSolver
 * (rdme/MpdRdmeSolver.h:66-156, rdme/IntMpdRdmeSolver.h) and the parts of
 * lm::cme::CMESolver / lm::rdme::RDMESolver they inherit
 * (cme/CMESolver.h:200-204, rdme/RDMESolver.h:57-67).  Header only; link
 * with liblmb200.so.
 *
 * Same calls, same argument meaning, same order of use as the reference:
 *   initialize(replicate, &parameters)       seed, overflow handler
 *   buildModel(...)                          reaction model
 *   buildDiffusionModel(...)                 diffusion model + row-major lattice
 *   setReactionRate(rx, rate)                change a rate (e.g. from a hook)
 *   generateTrajectory()                     the timestep loop with the
 *                                            writeInterval / latticeWriteInterval /
 *                                            hookInterval cadence in timesteps
 * Errors the reference throws as lm::Exception are thrown as lmb::Exception
 * with the reference's message.  What the reference pushes to its HDF5
 * output queue (species counts, lattice frames, site frames) goes to virtual
 * output functions a subclass overrides; hookSimulation / onBeginTrajectory /
 * onEndTrajectory / onWriteLattice are virtual as in the reference and see
 * the lattice as a host copy (HostLattice) in the native layout.
 */
#ifndef LMB_SOLVER_HPP
#define LMB_SOLVER_HPP

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <ctime>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "lmb.h"
#include "lmb_lmfile.h"

namespace lmb {

/* lm::Exception (core/Exceptions.h) for a status code of the C ABI. */
class Exception : public std::runtime_error {
public:
    Exception(int status, const std::string &where)
        : std::runtime_error(where + ": " + lmb_status_string(status)), status_(status) {}
    int status() const { return status_; }

private:
    int status_;
};

inline void check(int status, const char *where)
{
    if (status != LMB_OK) throw Exception(status, where);
}

/* Host copy of a lattice in the native layout (word w of site
 * i = x + y*X + z*X*Y at particles[w*N + i]; ByteLattice: 4 slots per word),
 * with the reference lattice's accessors (rdme/Lattice.h:131-259). */
class HostLattice {
public:
    uint32_t X = 0, Y = 0, Z = 0, slots = 0, bytes_per_particle = 1;
    std::vector<uint32_t> particles;
    std::vector<uint8_t> sites;

    uint32_t numberSites() const { return X * Y * Z; }
    uint32_t words() const { return bytes_per_particle == 1 ? slots / 4 : slots; }
    uint32_t index(uint32_t x, uint32_t y, uint32_t z) const { return x + y * X + z * X * Y; }
    uint8_t getSiteType(uint32_t x, uint32_t y, uint32_t z) const { return sites[index(x, y, z)]; }
    void setSiteType(uint32_t x, uint32_t y, uint32_t z, uint8_t t) { sites[index(x, y, z)] = t; }
    uint32_t getParticle(uint32_t x, uint32_t y, uint32_t z, uint32_t slot) const
    {
        const size_t N = numberSites(), i = index(x, y, z);
        if (bytes_per_particle == 1) return (particles[(slot / 4) * N + i] >> (8 * (slot % 4))) & 0xFFu;
        return particles[slot * N + i];
    }
    uint32_t getOccupancy(uint32_t x, uint32_t y, uint32_t z) const
    {
        uint32_t n = 0;
        while (n < slots && getParticle(x, y, z, n) != 0) n++;
        return n;
    }
    /* ByteLattice::addParticle: first free slot; false if the site is full. */
    bool addParticle(uint32_t x, uint32_t y, uint32_t z, uint32_t particle)
    {
        const uint32_t n = getOccupancy(x, y, z);
        if (n >= slots) return false;
        setSlot(x, y, z, n, particle);
        return true;
    }
    /* Lattice::removeParticles: empties the site. */
    void removeParticles(uint32_t x, uint32_t y, uint32_t z)
    {
        for (uint32_t s = 0; s < slots; s++) setSlot(x, y, z, s, 0);
    }

private:
    void setSlot(uint32_t x, uint32_t y, uint32_t z, uint32_t slot, uint32_t v)
    {
        const size_t N = numberSites(), i = index(x, y, z);
        if (bytes_per_particle == 1) {
            uint32_t &w = particles[(slot / 4) * N + i];
            const uint32_t sh = 8 * (slot % 4);
            w = (w & ~(0xFFu << sh)) | ((v & 0xFFu) << sh);
        } else {
            particles[slot * N + i] = v;
        }
    }
};

/* lm::rdme::MpdRdmeSolver (bytes_per_particle 1) and, with
 * bytesPerParticle() == 4, IntMpdRdmeSolver. */
class MpdRdmeSolver {
public:
    explicit MpdRdmeSolver(int device = 0) { check(lmb_ctx_create(device, &ctx_), "lmb_ctx_create"); }
    virtual ~MpdRdmeSolver()
    {
        if (lattice_) lmb_lattice_destroy(lattice_);
        if (model_) lmb_model_destroy(model_);
        if (ctx_) lmb_ctx_destroy(ctx_);
    }
    MpdRdmeSolver(const MpdRdmeSolver &) = delete;
    MpdRdmeSolver &operator=(const MpdRdmeSolver &) = delete;

    virtual bool needsReactionModel() { return true; }
    virtual bool needsDiffusionModel() { return true; }
    virtual uint32_t bytesPerParticle() const { return 1; }

    /* MpdRdmeSolver::initialize (MpdRdmeSolver.cu:107-162): seed =
     * (seedTop << 16) | (replicate & 0xFFFF), seedTop from parameter "seed"
     * (the clock's nanoseconds when 0); "rdme.mpd.overflowhandler" classic
     * (default) or relaxed. */
    virtual void initialize(unsigned int replicate, std::map<std::string, std::string> *parameters)
    {
        replicate_ = replicate;
        parameters_ = parameters;
        uint32_t seedTop = (uint32_t)atoi(param("seed").c_str());
        if (seedTop == 0) {
            struct timespec ts;
            clock_gettime(CLOCK_REALTIME, &ts);
            seedTop = (uint32_t)ts.tv_nsec;
        }
        seed_ = lmb_compose_seed(seedTop, replicate);
        const std::string s = param("rdme.mpd.overflowhandler");
        overflow_ = s == "relaxed" ? LMB_OVERFLOW_RELAXED : LMB_OVERFLOW_CLASSIC;
    }

    /* CMESolver::buildModel (cme/CMESolver.h:200-201): reaction types
     * 0..3, K[R * kCols] (column 0 used), S and D species-major [NS * R]. */
    virtual void buildModel(uint32_t numberSpecies, uint32_t numberReactions, const uint32_t *initialSpeciesCounts,
                            const uint32_t *reactionTypes, const double *K, const int32_t *S, const uint32_t *D,
                            uint32_t kCols = 1)
    {
        ns_ = numberSpecies;
        nr_ = numberReactions;
        initial_.assign(initialSpeciesCounts, initialSpeciesCounts + numberSpecies);
        rtype_.assign(reactionTypes, reactionTypes + numberReactions);
        K_.assign(K, K + (size_t)numberReactions * kCols);
        kcols_ = kCols;
        S_.assign(S, S + (size_t)numberSpecies * numberReactions);
        D_.assign(D, D + (size_t)numberSpecies * numberReactions);
    }

    /* RDMESolver::buildDiffusionModel (RDMESolver.cpp:110-142): DF
     * [NST * NST * NS] m^2/s, RL [R * NST], lattice [x][y][z][p] and site
     * types [x][y][z] row-major; "timestep" comes from the parameters. */
    virtual void buildDiffusionModel(uint32_t numberSiteTypes, const double *DF, const uint32_t *RL, uint32_t X,
                                     uint32_t Y, uint32_t Z, uint32_t particlesPerSite, uint32_t bytesPerParticle,
                                     double latticeSpacing, const void *latticeData, const uint8_t *latticeSitesData,
                                     bool rowMajorData = true)
    {
        if (!rowMajorData) throw std::invalid_argument("columns major lattice data is not currently supported");
        if (bytesPerParticle != this->bytesPerParticle())
            throw std::invalid_argument("bytes_per_particle does not match the solver's lattice type");
        nst_ = numberSiteTypes;
        DF_.assign(DF, DF + (size_t)numberSiteTypes * numberSiteTypes * ns_);
        RL_.assign(RL, RL + (size_t)nr_ * numberSiteTypes);
        spacing_ = latticeSpacing;
        tau_ = atof(param("timestep").c_str());
        if (lattice_) lmb_lattice_destroy(lattice_);
        lattice_ = nullptr;
        if (model_) lmb_model_destroy(model_);
        model_ = nullptr;
        lmb_model_desc d = desc();
        check(lmb_model_create(ctx_, &d, X, Y, Z, &model_), "buildDiffusionModel");
        check(lmb_lattice_create(ctx_, X, Y, Z, particlesPerSite, bytesPerParticle, &lattice_), "buildDiffusionModel");
        check(lmb_lattice_set_row_major(lattice_, latticeData, latticeSitesData, ns_, nst_), "setLatticeData");
        host_.X = X;
        host_.Y = Y;
        host_.Z = Z;
        host_.slots = particlesPerSite;
        host_.bytes_per_particle = bytesPerParticle;
    }

    /* Writes the trajectory into a `.lm` file, as the reference's
     * DataOutputQueue writes it into the simulation file
     * (core/LocalDataOutputWorker.cpp): this replicate's species counts,
     * lattice frames (from the device, through the file's writer thread),
     * site frames and, for the byte lattice, the max counts.  With
     * writeInputs the parameters, both models and the initial lattice go in
     * too when the trajectory starts.  The caller closes the file. */
    void setOutputFile(lmb_lmfile *file, bool writeInputs = true)
    {
        out_ = file;
        outInputs_ = writeInputs;
    }

    /* MpdRdmeSolver::setReactionRate (MpdRdmeSolver.h:85): the new rate is
     * used from the next timestep on. */
    virtual void setReactionRate(unsigned int rxid, float rate)
    {
        check(lmb_model_set_reaction_rate(model_, rxid, rate), "setReactionRate");
    }

    /* MpdRdmeSolver::generateTrajectory (MpdRdmeSolver.cu:485-668): runs
     * timesteps while timestep * tau < maxTime; after a timestep that reaches
     * the next hook, lattice-write or species-write step (intervals in
     * timesteps), calls the hook, writes the lattice, records the counts,
     * in that order.  Counts and lattice are also written at t = 0. */
    virtual void generateTrajectory()
    {
        const uint32_t countsInterval = (uint32_t)atof(param("writeInterval").c_str());
        const uint32_t latticeInterval = (uint32_t)atof(param("latticeWriteInterval").c_str());
        const double maxTime = atof(param("maxTime").c_str());
        bool hookEnabled = false;
        uint32_t hookInterval = 0, nextHook = 0;
        if (param("hookInterval") != "") {
            hookInterval = (uint32_t)atof(param("hookInterval").c_str());
            hookEnabled = true;
            nextHook = hookInterval;
        }
        uint32_t nextCounts = countsInterval, nextLattice = latticeInterval;
        stop_ = false;
        download();
        onBeginTrajectory(host_);
        upload(true);
        if (out_ && outInputs_) writeInputs();
        double time = 0.0;
        maxParticleCounts_.assign(ns_ + 1, 0);
        maxSiteCounts_.assign(nst_, 0);
        recordSpeciesCounts(time);
        writeLatticeRecord(time);
        updateMaxSiteCounts();  // initMaxCounts (MpdRdmeSolver.cu:548, 824-850)
        hookCheck(time);
        // The reference loops while timestep * tau < maxTime: that many
        // timesteps in all.
        uint64_t total = tau_ > 0.0 ? (uint64_t)std::floor(maxTime / tau_) : 0;
        if (tau_ > 0.0) {
            while ((double)total * tau_ < maxTime) total++;
            while (total > 0 && (double)(total - 1) * tau_ >= maxTime) total--;
        }
        uint32_t step = 0;
        while (step < total && !stop_) {
            // Run to the next step that has an event (an interval of 0 has
            // one after every timestep), or to the end.
            uint64_t ev = total;
            ev = std::min<uint64_t>(ev, nextCounts > step ? nextCounts : step + 1);
            ev = std::min<uint64_t>(ev, nextLattice > step ? nextLattice : step + 1);
            if (hookEnabled) ev = std::min<uint64_t>(ev, nextHook > step ? nextHook : step + 1);
            // A step whose records need the species totals, with no hook that
            // could change the lattice first, takes them in the run's own work.
            const bool records = ev >= nextCounts || ev >= nextLattice;
            const bool hooks = hookEnabled && ev >= nextHook;
            run(step, (uint32_t)(ev - step), records && !hooks);
            step = (uint32_t)ev;
            time = step * tau_;
            if (step >= nextLattice || step >= nextCounts || (hookEnabled && step >= nextHook)) {
                if (hookEnabled && step >= nextHook) {
                    download();
                    hookCheck(time);
                    nextHook += hookInterval;
                }
                if (step >= nextLattice) {
                    download();
                    if (onWriteLattice(time, host_)) upload(true);
                    writeLatticeRecord(time);
                    nextLattice += latticeInterval;
                }
                if (step >= nextCounts) {
                    recordSpeciesCounts(time);
                    nextCounts += countsInterval;
                }
            }
        }
        download();
        onEndTrajectory(host_);
        if (tracksMaxCounts()) {
            if (out_)
                check(lmb_lmfile_write_max_counts(out_, replicate_, maxParticleCounts_.data(),
                                                  (uint32_t)maxParticleCounts_.size(), maxSiteCounts_.data(),
                                                  (uint32_t)maxSiteCounts_.size()),
                      "writeMaxCounts");
            writeMaxCounts(maxParticleCounts_, maxSiteCounts_);
        }
    }

    uint32_t seed() const { return seed_; }
    lmb_lattice *lattice() { return lattice_; }
    lmb_model *model() { return model_; }
    const lmb_run_stats &lastRunStats() const { return stats_; }

protected:
    /* Hooks (MpdRdmeSolver.cu:789-822).  hookSimulation returns 0 (lattice
     * unchanged), 1 (lattice changed: copied to the device), 2 (sites changed
     * too: copied and written), 3 (stop after writing the sites). */
    virtual int hookSimulation(double /*time*/, HostLattice &/*lattice*/) { return 0; }
    virtual int onBeginTrajectory(HostLattice &/*lattice*/) { return 0; }
    virtual int onEndTrajectory(HostLattice &/*lattice*/) { return 0; }
    virtual int onWriteLattice(double /*time*/, HostLattice &/*lattice*/) { return 0; }

    /* Outputs (the reference's DataOutputQueue data sets). */
    virtual void writeSpeciesCounts(double /*time*/, const std::vector<uint64_t> &/*counts*/) {}
    virtual void writeLattice(double /*time*/, const HostLattice &/*lattice*/) {}
    virtual void writeLatticeSites(double /*time*/, const HostLattice &/*lattice*/) {}
    /* MpdRdmeSolver::writeMaxCounts (MpdRdmeSolver.cu:921-932), at the end of
     * the trajectory: per species id (index 0 unused) the largest count seen
     * at the start and at each lattice write; per site type (type 0 not
     * counted) the largest number of sites seen at the start and at each
     * site write. */
    virtual void writeMaxCounts(const std::vector<uint32_t> & /*maxParticleCounts*/,
                                const std::vector<uint32_t> & /*maxSiteCounts*/)
    {
    }
    /* IntMpdRdmeSolver::generateTrajectory keeps no maxima (its initMaxCounts
     * call is disabled, IntMpdRdmeSolver.cu:617) and writes none. */
    virtual bool tracksMaxCounts() const { return true; }

    std::string param(const char *key) const
    {
        if (!parameters_) return std::string();
        auto it = parameters_->find(key);
        return it == parameters_->end() ? std::string() : it->second;
    }

private:
    lmb_model_desc desc() const
    {
        lmb_model_desc d;
        d.number_species = ns_;
        d.number_reactions = nr_;
        d.number_site_types = nst_;
        d.reaction_types = rtype_.data();
        d.K = K_.data();
        d.k_cols = kcols_;
        d.S = S_.data();
        d.D = D_.data();
        d.DF = DF_.data();
        d.RL = RL_.data();
        d.timestep = tau_;
        d.lattice_spacing = spacing_;
        return d;
    }

    void run(uint32_t first, uint32_t n, bool withCounts = false)
    {
        int rc;
        if (withCounts) {
            runCounts_.assign(ns_ + 1, 0);
            rc = lmb_run_counts_async(lattice_, model_, seed_, first, n, overflow_, ns_);
            if (rc == LMB_OK) rc = lmb_run_counts_wait(lattice_, &stats_, runCounts_.data());
        } else {
            rc = lmb_run(lattice_, model_, seed_, first, n, overflow_, &stats_);
        }
        runCountsValid_ = withCounts && rc == LMB_OK;
        if (rc != LMB_OK) throw Exception(rc, "runTimestep");
    }

    /* The lattice's species totals: those the last run took, unless the
     * lattice was changed since. */
    std::vector<uint64_t> speciesCounts()
    {
        if (runCountsValid_) return runCounts_;
        std::vector<uint64_t> c(ns_ + 1);
        check(lmb_lattice_species_counts(lattice_, ns_, c.data()), "recordSpeciesCounts");
        return c;
    }

    void download()
    {
        host_.particles.resize((size_t)host_.words() * host_.numberSites());
        host_.sites.resize(host_.numberSites());
        check(lmb_lattice_get_native(lattice_, host_.particles.data(), host_.sites.data()), "copyFromGPU");
    }

    void upload(bool withSites)
    {
        check(lmb_lattice_set_native(lattice_, host_.particles.data(), withSites ? host_.sites.data() : nullptr),
              "copyToGPU");
        runCountsValid_ = false;
    }

    void recordSpeciesCounts(double time)
    {
        std::vector<uint64_t> c = speciesCounts();
        c.erase(c.begin());  // species ids are 1-based
        if (out_) {
            std::vector<int32_t> row(c.begin(), c.end());
            check(lmb_lmfile_append_species_counts(out_, replicate_, 1, ns_, &time, row.data()), "writeSpeciesCounts");
        }
        writeSpeciesCounts(time, c);
    }

    /* writeLatticeData (MpdRdmeSolver.cu:854-883): the particle maxima, then
     * the frame. */
    void writeLatticeRecord(double time)
    {
        const std::vector<uint64_t> c = speciesCounts();
        for (uint32_t s = 1; s <= ns_; s++)
            if (c[s] > maxParticleCounts_[s]) maxParticleCounts_[s] = (uint32_t)c[s];
        if (out_) check(lmb_lmfile_append_lattice_device(out_, replicate_, time, lattice_), "writeLatticeData");
        writeLattice(time, host_);
    }

    /* The site-type maxima (MpdRdmeSolver.cu:896-912), from the host copy. */
    void updateMaxSiteCounts()
    {
        std::vector<uint32_t> c(nst_, 0);
        for (uint8_t t : host_.sites)
            if (t > 0 && t < nst_) c[t]++;
        for (uint32_t t = 0; t < nst_; t++)
            if (c[t] > maxSiteCounts_[t]) maxSiteCounts_[t] = c[t];
    }

    /* The host site types, [z][y][x], as a [x][y][z] site frame. */
    void writeSitesToFile(double time)
    {
        if (!out_) return;
        const uint32_t X = host_.X, Y = host_.Y, Z = host_.Z;
        std::vector<uint8_t> rm((size_t)X * Y * Z);
        for (uint32_t z = 0; z < Z; z++)
            for (uint32_t y = 0; y < Y; y++)
                for (uint32_t x = 0; x < X; x++)
                    rm[((size_t)x * Y + y) * Z + z] = host_.sites[x + (size_t)X * (y + (size_t)Y * z)];
        check(lmb_lmfile_append_sites(out_, replicate_, time, X, Y, Z, rm.data()), "writeLatticeSites");
    }

    /* Parameters, models and the initial lattice (SimulationFile::
     * setParameter / setReactionModel / setDiffusionModel /
     * setDiffusionModelLattice). */
    void writeInputs()
    {
        if (parameters_)
            for (auto &kv : *parameters_)
                check(lmb_lmfile_set_parameter(out_, kv.first.c_str(), kv.second.c_str()), "setParameter");
        std::vector<double> k((size_t)nr_ * 10, std::nan(""));
        for (uint32_t r = 0; r < nr_; r++)
            for (uint32_t c = 0; c < kcols_ && c < 10; c++) k[(size_t)r * 10 + c] = K_[(size_t)r * kcols_ + c];
        check(lmb_lmfile_set_reaction_model(out_, ns_, nr_, initial_.data(), rtype_.data(), k.data(), nullptr,
                                            S_.data(), D_.data()),
              "setReactionModel");
        check(lmb_lmfile_set_diffusion_model(out_, ns_, nr_, nst_, spacing_, host_.X, host_.Y, host_.Z, host_.slots,
                                             host_.bytes_per_particle, DF_.data(), RL_.data()),
              "setDiffusionModel");
        std::vector<uint8_t> p((size_t)host_.numberSites() * host_.slots * host_.bytes_per_particle);
        std::vector<uint8_t> s(host_.numberSites());
        check(lmb_lattice_get_row_major(lattice_, p.data(), s.data()), "setDiffusionModelLattice");
        check(lmb_lmfile_set_diffusion_model_lattice(out_, p.data(), s.data()), "setDiffusionModelLattice");
    }

    void hookCheck(double time)
    {
        switch (hookSimulation(time, host_)) {
        case 0: break;
        case 1: upload(false); break;
        case 2:
            upload(true);
            updateMaxSiteCounts();
            writeSitesToFile(time);
            writeLatticeSites(time, host_);
            break;
        case 3:
            updateMaxSiteCounts();
            writeSitesToFile(time);
            writeLatticeSites(time, host_);
            stop_ = true;
            break;
        default: throw std::runtime_error("Unknown hook return value");
        }
    }

    lmb_ctx *ctx_ = nullptr;
    lmb_model *model_ = nullptr;
    lmb_lattice *lattice_ = nullptr;
    std::map<std::string, std::string> *parameters_ = nullptr;
    unsigned int replicate_ = 0;
    uint32_t seed_ = 0;
    int overflow_ = LMB_OVERFLOW_CLASSIC;
    uint32_t ns_ = 0, nr_ = 0, nst_ = 0, kcols_ = 1;
    std::vector<uint32_t> initial_, rtype_, D_, RL_;
    std::vector<int32_t> S_;
    std::vector<double> K_, DF_;
    double spacing_ = 0.0, tau_ = 0.0;
    HostLattice host_;
    lmb_run_stats stats_{};
    std::vector<uint64_t> runCounts_;  // species totals the last run took
    bool runCountsValid_ = false;      // and the lattice is unchanged since
    bool stop_ = false;
    std::vector<uint32_t> maxParticleCounts_, maxSiteCounts_;
    lmb_lmfile *out_ = nullptr;
    bool outInputs_ = false;
};

/* lm::rdme::IntMpdRdmeSolver: the same solver on an IntLattice. */
class IntMpdRdmeSolver : public MpdRdmeSolver {
public:
    explicit IntMpdRdmeSolver(int device = 0) : MpdRdmeSolver(device) {}
    uint32_t bytesPerParticle() const override { return 4; }

protected:
    bool tracksMaxCounts() const override { return false; }
};

}  // namespace lmb

#endif
