"""The pyLM-style solver classes (lattice_microbes_b200.rdme) driven as pyLM
and jLM drive lm::rdme::MpdRdmeSolver: parameter map, buildModel,
buildDiffusionModel with row-major lattice data, generateTrajectory with a
hookSimulation override.  Every record and the final lattice must equal the
same trajectory replayed range by range through the C ABI."""
import numpy as np
import pytest

from lattice_microbes_b200 import configs
from tests import ref_cpu_lib
from tests.test_gpu_cpp_solver import _row_major_int, check_lmfile, clear_left, expected_maxima, replay

pytestmark = pytest.mark.gpu


def _solver(kind, spec, hook, params, replicate=3):
    from lattice_microbes_b200.rdme import IntMpdRdmeSolver, MpdRdmeSolver
    base = MpdRdmeSolver if kind == "byte" else IntMpdRdmeSolver

    class Solver(base):
        calls = 0

        def hookSimulation(self, time, lattice):
            Solver.calls += 1
            if hook.startswith("clear_left:"):
                lattice.particles[:] = clear_left(spec, lattice.particles, int(hook.split(":")[1]))
                return 1
            if hook.startswith("stop_after:") and Solver.calls >= int(hook.split(":")[1]):
                return 3
            return 0

    s = Solver(0)
    s.initialize(replicate, params)
    init = configs.species_counts(spec.lattice, spec.nsites, spec.slots, spec.bytes_per_slot, spec.ns)[1:]
    s.buildModel(spec.ns, spec.nr, init, spec.rtype, spec.K, np.asarray(spec.S).reshape(-1),
                 np.asarray(spec.D).reshape(-1))
    lat_rm, sites_rm = ref_cpu_lib.row_major(spec) if kind == "byte" else _row_major_int(spec)
    s.buildDiffusionModel(spec.nst, np.asarray(spec.DF).reshape(-1), np.asarray(spec.RL).reshape(-1), spec.X,
                          spec.Y, spec.Z, spec.slots, spec.bytes_per_slot, spec.spacing, lat_rm, sites_rm)
    return s, Solver


@pytest.mark.parametrize("kind", ["byte", "int"])
def test_python_solver_matches_replay(gpu, kind, tmp_path):
    if kind == "byte":
        spec = configs.config0(seed=5, edge=16, nA=600, nB=600)
        spec.K = spec.K * np.array([300.0, 30.0])
    else:
        spec = configs.random_problem(8, X=16, Y=8, Z=8, slots=16, bytes_per_slot=4, density=1.5, nst=2)
    steps, ce, le, he = 301, 50, 100, 70
    params = {"seed": "9", "timestep": repr(spec.tau), "maxTime": repr((steps - 0.5) * spec.tau),
              "writeInterval": str(ce), "latticeWriteInterval": str(le), "hookInterval": str(he)}
    s, cls = _solver(kind, spec, "clear_left:1", params)
    from lattice_microbes_b200.lmfile import LMFileWriter
    lm = str(tmp_path / "py.lm")
    w = LMFileWriter(lm)
    s.setOutputFile(w)
    s.generateTrajectory()
    w.close()
    ref_c, ref_f, ref_final = replay(spec, s.seed, steps, ce, le, he, "clear_left:1")
    assert s.seed == (9 << 16) | 3
    assert len(s.speciesCounts) == len(ref_c) == 1 + steps // ce
    for (ta, a), (tb, b) in zip(s.speciesCounts, ref_c):
        assert ta == tb and np.array_equal(a, b)
    assert len(s.latticeFrames) == len(ref_f)
    for (_, a, _), b in zip(s.latticeFrames, ref_f):
        assert np.array_equal(a, b)
    assert np.array_equal(s.lattice.particles, ref_final)
    assert cls.calls == 1 + steps // he
    if kind == "byte":
        mp, ms = expected_maxima(spec, ref_f)
        assert np.array_equal(s.maxParticleCounts, mp) and np.array_equal(s.maxSiteCounts, ms)
    else:
        assert s.maxParticleCounts is None  # the Int solver writes no maxima
    maxima = None if kind != "byte" else (s.maxParticleCounts, s.maxSiteCounts)
    check_lmfile(lm, spec, 3, [(t, c.astype(np.int64)) for t, c in s.speciesCounts], [b for _, b, _ in s.latticeFrames],
                 [t for t, _, _ in s.latticeFrames], maxima, params)
    s.close()


def test_python_solver_hook_3_stops(gpu):
    spec = configs.config0(seed=6, edge=16, nA=300, nB=300)
    steps, ce, le, he = 200, 20, 1000, 30
    params = {"seed": "9", "timestep": repr(spec.tau), "maxTime": repr((steps - 0.5) * spec.tau),
              "writeInterval": str(ce), "latticeWriteInterval": str(le), "hookInterval": str(he)}
    s, _ = _solver("byte", spec, "stop_after:3", params)
    s.generateTrajectory()
    ref_c, _, ref_final = replay(spec, s.seed, steps, ce, le, he, "stop_after:3")
    assert np.array_equal(s.lattice.particles, ref_final)
    assert len(s.speciesCounts) == len(ref_c)
    assert all(np.array_equal(a[1], b[1]) for a, b in zip(s.speciesCounts, ref_c))
    assert s.speciesCounts[-1][0] == 60 * spec.tau
    s.close()


@pytest.mark.parametrize("kind", ["byte", "int"])
def test_run_solver_from_an_lm_file(gpu, kind, tmp_path):
    """lm.runSolver on a `.lm` file: a first replicate written with its
    inputs, then runSolver reads the parameters, models and lattice back
    from the file and appends replicate 4; its records equal a solver set up
    directly for replicate 4, and replicate 3 is carried over unchanged."""
    from lattice_microbes_b200.lmfile import LMFile, LMFileWriter
    from lattice_microbes_b200.rdme import IntMpdRdmeSolver, MpdRdmeSolver, runSolver
    if kind == "byte":
        spec = configs.config0(seed=11, edge=16, nA=500, nB=500)
        spec.K = spec.K * np.array([300.0, 30.0])
    else:
        spec = configs.random_problem(8, X=16, Y=8, Z=8, slots=16, bytes_per_slot=4, density=1.5, nst=2)
    steps, ce, le = 120, 20, 40
    params = {"seed": "9", "timestep": repr(spec.tau), "maxTime": repr((steps - 0.5) * spec.tau),
              "writeInterval": str(ce), "latticeWriteInterval": str(le)}
    lm = str(tmp_path / "run.lm")
    first, _ = _solver(kind, spec, "none", params, replicate=3)
    w = LMFileWriter(lm)
    first.setOutputFile(w)
    first.generateTrajectory()
    w.close()
    first.close()
    cls = MpdRdmeSolver if kind == "byte" else IntMpdRdmeSolver
    runSolver(lm, 4, cls(0), checkpointInterval=1e-9)  # a checkpoint at every record
    direct, _ = _solver(kind, spec, "none", params, replicate=4)
    direct.generateTrajectory()
    with LMFile(lm) as f:
        assert f.replicates() == [3, 4]
        t, c = f.species_counts(4)
        assert np.array_equal(t, [a for a, _ in direct.speciesCounts])
        assert np.array_equal(c, np.array([b for _, b in direct.speciesCounts]))
        assert np.array_equal(f.lattice_times(4), [a for a, _, _ in direct.latticeFrames])
        from tests.test_gpu_cpp_solver import row_major_frame
        for i, (_, fr, _) in enumerate(direct.latticeFrames):
            assert np.array_equal(f.lattice(4, i), row_major_frame(spec, fr))
        t3, c3 = f.species_counts(3)
        assert len(t3) == 1 + steps // ce and not np.array_equal(c3, c)  # replicate 3 kept, another seed
    import os
    with LMFile(lm + ".chk") as k:  # the last checkpoint: every species-count record
        assert k.replicates() == [3, 4]
        tk, ck = k.species_counts(4)
        assert np.array_equal(tk, t) and np.array_equal(ck, c)
    os.unlink(lm + ".chk")
    direct.close()


def test_python_solver_site_frames_in_the_lm_file(gpu, tmp_path):
    """A hook that changes a site type and returns 2 (sites copied to the
    device and written): the file's site frame is the changed [x][y][z]
    site-type lattice, and the site maxima count the change."""
    from lattice_microbes_b200.lmfile import LMFile, LMFileWriter
    from lattice_microbes_b200.rdme import MpdRdmeSolver
    spec = configs.random_problem(8, X=16, Y=8, Z=8, slots=8, bytes_per_slot=1, density=0.5, nst=3)

    class Solver(MpdRdmeSolver):
        def hookSimulation(self, time, lattice):
            if time > 0.0:
                return 0
            old = lattice.getSiteType(3, 2, 1)
            lattice.setSiteType(3, 2, 1, 2 if old != 2 else 1)
            return 2

    params = {"seed": "5", "timestep": repr(spec.tau), "maxTime": repr(39.5 * spec.tau), "writeInterval": "10",
              "latticeWriteInterval": "20", "hookInterval": "20"}
    s = Solver(0)
    s.initialize(1, params)
    init = configs.species_counts(spec.lattice, spec.nsites, spec.slots, spec.bytes_per_slot, spec.ns)[1:]
    s.buildModel(spec.ns, spec.nr, init, spec.rtype, spec.K, np.asarray(spec.S).reshape(-1),
                 np.asarray(spec.D).reshape(-1))
    lat_rm, sites_rm = ref_cpu_lib.row_major(spec)
    s.buildDiffusionModel(spec.nst, np.asarray(spec.DF).reshape(-1), np.asarray(spec.RL).reshape(-1), spec.X,
                          spec.Y, spec.Z, spec.slots, spec.bytes_per_slot, spec.spacing, lat_rm, sites_rm)
    p = str(tmp_path / "sites.lm")
    w = LMFileWriter(p)
    s.setOutputFile(w)
    s.generateTrajectory()
    w.close()
    want = spec.sites.reshape(spec.Z, spec.Y, spec.X).transpose(2, 1, 0).copy()
    want[3, 2, 1] = 2 if want[3, 2, 1] != 2 else 1
    with LMFile(p) as f:
        assert np.array_equal(f.site_times(1), [0.0])
        assert np.array_equal(f.sites(1, 0), want)
        ms = f.max_counts(1)[1]
    t = want.ravel()
    expect = np.maximum(np.bincount(spec.sites[(spec.sites > 0) & (spec.sites < spec.nst)], minlength=spec.nst),
                        np.bincount(t[(t > 0) & (t < spec.nst)], minlength=spec.nst))
    assert np.array_equal(ms, expect) and np.array_equal(s.maxSiteCounts, expect)
    s.close()


def test_jlm_sim_run_sequence(gpu, tmp_path):
    """jLM's Sim, call for call: the lattice made as RDME.py:145-150 makes it
    (lm.getCompiledLatticeMaxOccupancy, lm.ByteLattice), the file written with
    LmWriteMixin.finalize's lm calls (LmInteract.py:55-84), then Sim.run
    (RDME.py:447-455): lm.MpdRdmeSolver(), lm.simulationFile(name) with
    setParameter("seed", ...) and close, lm.runSolver(name, replicate, solver,
    cudaDevices, checkpointInterval).  The replicate read back from the file
    equals the same solver set up directly with those inputs."""
    import lattice_microbes_b200.lm  # noqa: F401  (makes `import lm` this package's)
    import lm
    from lattice_microbes_b200.lmfile import LMFile
    from lattice_microbes_b200.rdme import MpdRdmeSolver
    from tests.test_lm_module import write_jlm_file
    spec = configs.config0(seed=11, edge=16, nA=500, nB=500)
    spec.K = spec.K * np.array([300.0, 30.0])
    steps, ce, le = 120, 20, 40
    params = {"writeInterval": str(ce), "latticeWriteInterval": str(le),
              "maxTime": "{:.10e}".format((steps - 0.5) * spec.tau), "timestep": "{:.10e}".format(spec.tau),
              "hookInterval": ""}
    path = str(tmp_path / "sim.lm")
    pps = lm.getCompiledLatticeMaxOccupancy()
    lattice, init = write_jlm_file(lm, path, spec, pps, params)
    solver = lm.MpdRdmeSolver()
    f = lm.simulationFile(path)
    f.setParameter("seed", str(77))
    f.close()
    lm.runSolver(path, 1, solver, [0], int(0))
    direct = MpdRdmeSolver(0)
    direct.initialize(1, dict(params, seed="77"))
    direct.buildModel(spec.ns, spec.nr, init, spec.rtype, spec.K, np.asarray(spec.S).reshape(-1),
                      np.asarray(spec.D).reshape(-1))
    p, s = lattice.rowMajor()
    direct.buildDiffusionModel(spec.nst, np.asarray(spec.DF).reshape(-1), np.asarray(spec.RL).reshape(-1), spec.X,
                               spec.Y, spec.Z, pps, 1, spec.spacing, p.reshape(-1), s.reshape(-1))
    direct.generateTrajectory()
    with LMFile(path) as g:
        assert g.replicates() == [1]
        assert g.getParameter("seed") == "77"
        t, c = g.species_counts(1)
        assert len(t) == 1 + steps // ce
        assert np.array_equal(t, [a for a, _ in direct.speciesCounts])
        assert np.array_equal(c, np.array([b for _, b in direct.speciesCounts]))
        assert c[-1, 2] > 0  # C formed
        assert np.array_equal(g.lattice_times(1), [a for a, _, _ in direct.latticeFrames])
        for i, (_, fr, _) in enumerate(direct.latticeFrames):
            X, Y, Z = spec.X, spec.Y, spec.Z
            v = fr.view(np.uint8).reshape(pps // 4, Z, Y, X, 4)
            expect = np.moveaxis(v, 0, 3).reshape(Z, Y, X, pps).transpose(2, 1, 0, 3)
            assert np.array_equal(g.lattice(1, i), expect)
    direct.close()
    solver.close()
