/*
 * solver_driver.cpp -- runs lmb::MpdRdmeSolver / IntMpdRdmeSolver
 * (include/lmb_solver.hpp) the way the reference's runSolver drives a solver
 * (core/runSimulation.cpp:130-280): initialize with a parameter map,
 * buildModel, buildDiffusionModel with row-major lattice data,
 * generateTrajectory.  Test program for tests/test_gpu_cpp_solver.py.
 *
 *   solver_driver <dir>
 *
 * <dir>/params.txt    key=value lines: the solver parameters plus X, Y, Z,
 *                     slots, bytes, ns, nr, nst, spacing, replicate, hook
 * <dir>/{rtype.u32,K.f64,S.i32,D.u32,init.u32,DF.f64,RL.u32,lattice.bin,sites.u8}
 * Writes <dir>/counts.txt (time and counts per record), frames.u32 (native
 * lattice at each lattice write), sites_frames.u8 (site types at each site
 * write), final.u32 (native lattice at the end) and events.txt.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "lmb_solver.hpp"

template <typename T>
static std::vector<T> load(const std::string &path)
{
    std::ifstream f(path, std::ios::binary);
    std::vector<char> raw((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    std::vector<T> v(raw.size() / sizeof(T));
    if (!v.empty()) memcpy(v.data(), raw.data(), v.size() * sizeof(T));
    return v;
}

template <typename T>
static void append(const std::string &path, const T *p, size_t n)
{
    std::ofstream f(path, std::ios::binary | std::ios::app);
    f.write(reinterpret_cast<const char *>(p), n * sizeof(T));
}

template <typename Base>
class Driver : public Base {
public:
    std::string dir;
    std::string hook;
    std::ofstream counts, events;

    Driver(const std::string &d, const std::string &h) : dir(d), hook(h)
    {
        counts.open(dir + "/counts.txt");
        events.open(dir + "/events.txt");
    }

protected:
    /* The hook the test mirrors: "clear_left:<species>" removes every
     * particle of that species from the sites with x < X/2 (keeping slot
     * order, as Lattice::removeParticle does) and returns 1;
     * "stop_after:<n>" returns 3 at the n-th hook call. */
    int hook_calls = 0;
    int hookSimulation(double time, lmb::HostLattice &lat) override
    {
        hook_calls++;
        events << "hook " << time << "\n";
        if (hook.rfind("clear_left:", 0) == 0) {
            const uint32_t sp = (uint32_t)atoi(hook.c_str() + 11);
            for (uint32_t z = 0; z < lat.Z; z++)
                for (uint32_t y = 0; y < lat.Y; y++)
                    for (uint32_t x = 0; x < lat.X / 2; x++) {
                        std::vector<uint32_t> keep;
                        for (uint32_t s = 0; s < lat.getOccupancy(x, y, z); s++) {
                            const uint32_t p = lat.getParticle(x, y, z, s);
                            if (p != sp) keep.push_back(p);
                        }
                        lat.removeParticles(x, y, z);
                        for (uint32_t p : keep) lat.addParticle(x, y, z, p);
                    }
            return 1;
        }
        if (hook.rfind("stop_after:", 0) == 0 && hook_calls >= atoi(hook.c_str() + 11)) return 3;
        return 0;
    }
    void writeSpeciesCounts(double time, const std::vector<uint64_t> &c) override
    {
        char buf[64];
        snprintf(buf, sizeof buf, "%.17g", time);
        counts << buf;
        for (uint64_t v : c) counts << " " << v;
        counts << "\n";
    }
    void writeLattice(double time, const lmb::HostLattice &lat) override
    {
        events << "lattice " << time << "\n";
        append(dir + "/frames.u32", lat.particles.data(), lat.particles.size());
    }
    void writeLatticeSites(double time, const lmb::HostLattice &lat) override
    {
        events << "sites " << time << "\n";
        append(dir + "/sites_frames.u8", lat.sites.data(), lat.sites.size());
    }
    int onEndTrajectory(lmb::HostLattice &lat) override
    {
        append(dir + "/final.u32", lat.particles.data(), lat.particles.size());
        return 0;
    }
    void writeMaxCounts(const std::vector<uint32_t> &mp, const std::vector<uint32_t> &ms) override
    {
        std::ofstream f(dir + "/max.txt");
        for (uint32_t v : mp) f << v << " ";
        f << "\n";
        for (uint32_t v : ms) f << v << " ";
        f << "\n";
    }
};

template <typename Base>
static int run(const std::string &dir, std::map<std::string, std::string> &p)
{
    auto u = [&](const char *k) { return (uint32_t)atol(p[k].c_str()); };
    Driver<Base> s(dir, p["hook"]);
    s.initialize(u("replicate"), &p);
    auto rtype = load<uint32_t>(dir + "/rtype.u32");
    auto K = load<double>(dir + "/K.f64");
    auto S = load<int32_t>(dir + "/S.i32");
    auto D = load<uint32_t>(dir + "/D.u32");
    auto init = load<uint32_t>(dir + "/init.u32");
    auto DF = load<double>(dir + "/DF.f64");
    auto RL = load<uint32_t>(dir + "/RL.u32");
    auto lattice = load<uint8_t>(dir + "/lattice.bin");
    auto sites = load<uint8_t>(dir + "/sites.u8");
    s.buildModel(u("ns"), u("nr"), init.data(), rtype.data(), K.data(), S.data(), D.data(), 1);
    s.buildDiffusionModel(u("nst"), DF.data(), RL.data(), u("X"), u("Y"), u("Z"), u("slots"), u("bytes"),
                          atof(p["spacing"].c_str()), lattice.data(), sites.data(), true);
    lmb_lmfile *out = nullptr;
    if (!p["lmfile"].empty()) {
        if (lmb_lmfile_create(p["lmfile"].c_str(), &out) != LMB_OK) return 4;
        s.setOutputFile(out, true);
    }
    try {
        s.generateTrajectory();
    } catch (lmb::Exception &e) {
        std::ofstream(dir + "/error.txt") << e.status() << " " << e.what() << "\n";
        if (out) lmb_lmfile_close(out);
        return 3;
    }
    if (out && lmb_lmfile_close(out) != LMB_OK) return 5;
    std::cout << "seed " << s.seed() << "\n";
    return 0;
}

int main(int argc, char **argv)
{
    if (argc != 2) {
        std::cerr << "usage: solver_driver <dir>\n";
        return 2;
    }
    const std::string dir = argv[1];
    std::map<std::string, std::string> p;
    std::ifstream f(dir + "/params.txt");
    std::string line;
    while (std::getline(f, line)) {
        const size_t eq = line.find('=');
        if (eq != std::string::npos) p[line.substr(0, eq)] = line.substr(eq + 1);
    }
    if (p["bytes"] == "4") return run<lmb::IntMpdRdmeSolver>(dir, p);
    return run<lmb::MpdRdmeSolver>(dir, p);
}
