"""The C++ solver layer (include/lmb_solver.hpp) driven like the reference's
runSolver drives lm::rdme::MpdRdmeSolver: parameter map, buildModel,
buildDiffusionModel with row-major lattice data, generateTrajectory with the
writeInterval / latticeWriteInterval / hookInterval cadence.

tests/cpp/solver_driver runs it; the same trajectory is replayed here through
the Python face of the C ABI, timestep range by timestep range with the same
hook edits, and every record (species counts, lattice frames, the final
lattice) must agree bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

from lattice_microbes_b200 import configs
from tests import ref_cpu_lib

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "tests", "cpp", "_build", "solver_driver")


@pytest.fixture(scope="module")
def driver(gpu):
    if not os.path.exists(DRIVER):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "cpp")], check=True)
    return DRIVER


def write_inputs(d, spec, params):
    spec_rm, sites_rm = ref_cpu_lib.row_major(spec) if spec.bytes_per_slot == 1 else _row_major_int(spec)
    init = configs.species_counts(spec.lattice, spec.nsites, spec.slots, spec.bytes_per_slot, spec.ns)[1:]
    arrays = {
        "rtype.u32": np.asarray(spec.rtype, np.uint32), "K.f64": np.asarray(spec.K, np.float64),
        "S.i32": np.asarray(spec.S, np.int32), "D.u32": np.asarray(spec.D, np.uint32),
        "init.u32": init.astype(np.uint32), "DF.f64": np.asarray(spec.DF, np.float64),
        "RL.u32": np.asarray(spec.RL, np.uint32), "lattice.bin": spec_rm, "sites.u8": sites_rm,
    }
    for name, a in arrays.items():
        np.ascontiguousarray(a).tofile(os.path.join(d, name))
    p = dict(params)
    p.update(X=spec.X, Y=spec.Y, Z=spec.Z, slots=spec.slots, bytes=spec.bytes_per_slot, ns=spec.ns, nr=spec.nr,
             nst=spec.nst, spacing=repr(spec.spacing), timestep=repr(spec.tau))
    with open(os.path.join(d, "params.txt"), "w") as f:
        for k, v in p.items():
            f.write("%s=%s\n" % (k, v))


def _row_major_int(spec):
    X, Y, Z = spec.X, spec.Y, spec.Z
    slots = configs.native_to_slots(spec.lattice, X, Y, Z, spec.slots, spec.bytes_per_slot)
    lat = slots.reshape(Z, Y, X, spec.slots).transpose(2, 1, 0, 3)
    sites = spec.sites.reshape(Z, Y, X).transpose(2, 1, 0)
    return (np.ascontiguousarray(lat, dtype=np.uint32).reshape(-1),
            np.ascontiguousarray(sites, dtype=np.uint8).reshape(-1))


def clear_left(spec, native, species):
    """The driver's hook edit on a native lattice: drop `species` from the
    sites with x < X/2, keeping the other particles' slot order."""
    X, Y, Z, S = spec.X, spec.Y, spec.Z, spec.slots
    slots = configs.native_to_slots(native, X, Y, Z, S, spec.bytes_per_slot).reshape(Z, Y, X, S)
    left = slots[:, :, : X // 2, :]
    keep = left != species
    out = np.zeros_like(left)
    order = np.argsort(~keep, axis=-1, kind="stable")
    out[...] = np.take_along_axis(np.where(keep, left, 0), order, axis=-1)
    slots[:, :, : X // 2, :] = out
    flat = slots.reshape(-1, S)
    lat = configs.empty_lattice(X, Y, Z, S, spec.bytes_per_slot)
    N = spec.nsites
    for k in range(S):
        v = flat[:, k].astype(np.uint32)
        if spec.bytes_per_slot == 1:
            lat[(k // 4) * N:(k // 4 + 1) * N] |= v << np.uint32(8 * (k % 4))
        else:
            lat[k * N:(k + 1) * N] = v
    return lat


def replay(spec, seed, steps, count_every, lattice_every, hook_every, hook):
    """The trajectory generateTrajectory produces, through the Python face."""
    from lattice_microbes_b200.solver import Context, Lattice, Model
    ctx = Context(0)
    m = Model.from_spec(ctx, spec)
    lat = Lattice(ctx, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
    lat.set_native(spec.lattice, spec.sites)
    counts, frames = [], []
    counts.append((0.0, lat.species_counts(spec.ns)[1:]))
    frames.append(lat.get_native()[0])
    step, hook_calls, stopped = 0, 0, False
    # t = 0: the initial hook check
    hook_calls += 1
    if hook.startswith("stop_after:") and hook_calls >= int(hook.split(":")[1]):
        stopped = True
    if hook.startswith("clear_left:"):
        lat.set_native(clear_left(spec, lat.get_native()[0], int(hook.split(":")[1])), None)
    nc, nl, nh = count_every, lattice_every, hook_every
    while step < steps and not stopped:
        ev = min(steps, nc if nc > step else step + 1, nl if nl > step else step + 1,
                 nh if nh > step else step + 1)
        lat.run(m, seed, step, ev - step)
        step = ev
        t = step * spec.tau
        if step >= nh:
            hook_calls += 1
            if hook.startswith("clear_left:"):
                lat.set_native(clear_left(spec, lat.get_native()[0], int(hook.split(":")[1])), None)
            if hook.startswith("stop_after:") and hook_calls >= int(hook.split(":")[1]):
                stopped = True
            nh += hook_every
        if step >= nl:
            frames.append(lat.get_native()[0])
            nl += lattice_every
        if step >= nc:
            counts.append((t, lat.species_counts(spec.ns)[1:]))
            nc += count_every
    final = lat.get_native()[0]
    lat.close()
    m.close()
    ctx.close()
    return counts, frames, final


def run_driver(driver, tmp_path, spec, steps, count_every, lattice_every, hook_every, hook, seed_top=9,
               replicate=3, lmfile=""):
    d = str(tmp_path)
    params = {"seed": seed_top, "replicate": replicate, "maxTime": repr((steps - 0.5) * spec.tau),
              "writeInterval": count_every, "latticeWriteInterval": lattice_every, "hookInterval": hook_every,
              "hook": hook, "lmfile": lmfile}
    write_inputs(d, spec, params)
    r = subprocess.run([driver, d], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    counts = []
    for line in open(os.path.join(d, "counts.txt")):
        v = line.split()
        counts.append((float(v[0]), np.array([int(x) for x in v[1:]])))
    W = spec.words * spec.nsites
    frames = np.fromfile(os.path.join(d, "frames.u32"), dtype=np.uint32).reshape(-1, W)
    final = np.fromfile(os.path.join(d, "final.u32"), dtype=np.uint32)
    events = open(os.path.join(d, "events.txt")).read().split("\n")
    maxima = None
    if os.path.exists(os.path.join(d, "max.txt")):
        lines = open(os.path.join(d, "max.txt")).read().strip().split("\n")
        maxima = [np.array([int(v) for v in ln.split()]) for ln in lines]
    return counts, frames, final, events, (seed_top << 16) | (replicate & 0xFFFF), maxima


def row_major_frame(spec, native):
    """A native frame as the .lm file holds it: [x][y][z][p]."""
    slots = configs.native_to_slots(native, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
    dt = np.uint8 if spec.bytes_per_slot == 1 else np.uint32
    return np.ascontiguousarray(slots.reshape(spec.Z, spec.Y, spec.X, spec.slots).transpose(2, 1, 0, 3), dtype=dt)


def check_lmfile(path, spec, replicate, counts, frames, lattice_times, maxima, parameters):
    """The .lm file a solver wrote holds the records its callbacks saw."""
    from lattice_microbes_b200.lmfile import LMFile
    with LMFile(path) as f:
        assert f.version == 4 and f.replicates() == [replicate]
        for k, v in parameters.items():
            assert f.parameters()[k] == str(v)
        m = f.reaction_model()
        assert (m["numberSpecies"], m["numberReactions"]) == (spec.ns, spec.nr)
        assert m["stoichiometricMatrix"] == [int(v) for v in np.asarray(spec.S).ravel()]
        d = f.diffusion_model()
        assert (d["latticeXSize"], d["latticeYSize"], d["latticeZSize"]) == (spec.X, spec.Y, spec.Z)
        assert d["particlesPerSite"] == spec.slots and d["bytes_per_particle"] == spec.bytes_per_slot
        assert np.array_equal(d["DiffusionMatrix"].ravel(), np.asarray(spec.DF).ravel())
        assert np.array_equal(d["Lattice"], row_major_frame(spec, spec.lattice))
        assert np.array_equal(d["LatticeSites"], spec.sites.reshape(spec.Z, spec.Y, spec.X).transpose(2, 1, 0))
        t, c = f.species_counts(replicate)
        assert np.array_equal(t, [a for a, _ in counts])
        assert np.array_equal(c, np.array([b for _, b in counts]))
        assert np.array_equal(f.lattice_times(replicate), lattice_times)
        assert len(f.h5["Simulations/%07d/Lattice" % replicate].keys()) == len(frames)
        for i, fr in enumerate(frames):
            assert np.array_equal(f.lattice(replicate, i), row_major_frame(spec, fr))
        got = f.max_counts(replicate)
        if maxima is None:
            assert got is None
        else:
            assert np.array_equal(got[0], maxima[0]) and np.array_equal(got[1], maxima[1])


def expected_maxima(spec, frames):
    """Particle maxima over the lattice frames (the start is the first), site
    maxima from the site types (the hooks here do not change them)."""
    mp = np.zeros(spec.ns + 1, dtype=np.int64)
    for f in frames:
        c = configs.species_counts(f, spec.nsites, spec.slots, spec.bytes_per_slot, spec.ns).astype(np.int64)
        c[0] = 0
        mp = np.maximum(mp, c)
    t = spec.sites
    ms = np.bincount(t[(t > 0) & (t < spec.nst)], minlength=spec.nst)[:spec.nst]
    return mp, ms


@pytest.mark.parametrize("kind", ["byte", "int"])
def test_generate_trajectory_matches_replay(driver, tmp_path, kind):
    if kind == "byte":
        spec = configs.config0(seed=5, edge=16, nA=600, nB=600)
        spec.K = spec.K * np.array([300.0, 30.0])  # more reactions in a short run
    else:
        spec = configs.random_problem(8, X=16, Y=8, Z=8, slots=16, bytes_per_slot=4, density=1.5, nst=2)
    steps, ce, le, he = 301, 50, 100, 70
    lm = str(tmp_path / "out.lm")
    got_c, got_f, got_final, events, seed, maxima = run_driver(driver, tmp_path, spec, steps, ce, le, he,
                                                               "clear_left:1", lmfile=lm)
    ref_c, ref_f, ref_final = replay(spec, seed, steps, ce, le, he, "clear_left:1")
    assert [t for t, _ in got_c] == pytest.approx([t for t, _ in ref_c], rel=0, abs=0)
    assert len(got_c) == len(ref_c) == 1 + steps // ce
    for (_, a), (_, b) in zip(got_c, ref_c):
        assert np.array_equal(a, b)
    assert len(got_f) == len(ref_f)
    for a, b in zip(got_f, ref_f):
        assert np.array_equal(a, b)
    assert np.array_equal(got_final, ref_final)
    if kind == "byte":
        mp, ms = expected_maxima(spec, ref_f)
        assert np.array_equal(maxima[0], mp) and np.array_equal(maxima[1], ms)
    else:
        assert maxima is None  # the Int solver writes no maxima
    assert sum(1 for e in events if e.startswith("hook")) == 1 + steps // he
    # The same records in the .lm file the solver wrote.
    check_lmfile(lm, spec, 3, got_c, got_f, [i * le * spec.tau for i in range(len(got_f))], maxima,
                 {"writeInterval": ce, "latticeWriteInterval": le})
    # The hook really changed the trajectory: species 1 is gone from the left half at each hook.
    assert got_c[-1][1][0] < got_c[0][1][0]


def test_hook_return_3_stops(driver, tmp_path):
    spec = configs.config0(seed=6, edge=16, nA=300, nB=300)
    steps, ce, le, he = 200, 20, 1000, 30
    lm = str(tmp_path / "stop.lm")
    got_c, _, got_final, events, seed, _ = run_driver(driver, tmp_path, spec, steps, ce, le, he, "stop_after:3",
                                                      lmfile=lm)
    ref_c, _, ref_final = replay(spec, seed, steps, ce, le, he, "stop_after:3")
    assert np.array_equal(got_final, ref_final)
    assert len(got_c) == len(ref_c) and all(np.array_equal(a[1], b[1]) for a, b in zip(got_c, ref_c))
    assert sum(1 for e in events if e.startswith("sites")) == 1
    assert got_c[-1][0] == pytest.approx(60 * spec.tau, abs=0)
    from lattice_microbes_b200.lmfile import LMFile
    with LMFile(lm) as f:  # the hook's return 3 wrote one site frame
        assert np.array_equal(f.site_times(3), [60 * spec.tau])
        assert np.array_equal(f.sites(3, 0), spec.sites.reshape(spec.Z, spec.Y, spec.X).transpose(2, 1, 0))
