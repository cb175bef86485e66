"""Host logic of the pyLM-style solver classes (lattice_microbes_b200.rdme):
the trajectory cadence against a step-by-step restatement of
MpdRdmeSolver::generateTrajectory's loop (MpdRdmeSolver.cu:485-668), the
timestep count, and the reference lattice accessors on a host lattice."""
import numpy as np
import pytest

from lattice_microbes_b200 import configs
from lattice_microbes_b200.rdme import HostLattice, timesteps_for, trajectory_events


def reference_loop(total, ce, le, he):
    """One timestep at a time, as the reference loop checks after each."""
    out, nc, nl, nh = [], ce, le, he
    for step in range(1, total + 1):
        if step >= nl or step >= nc or (he is not None and step >= nh):
            hook = he is not None and step >= nh
            lat, cnt = step >= nl, step >= nc
            if hook:
                nh += he
            if lat:
                nl += le
            if cnt:
                nc += ce
            out.append((step, hook, lat, cnt))
    return out


@pytest.mark.parametrize("total,ce,le,he", [(301, 50, 100, 70), (200, 20, 1000, 30), (17, 0, 5, None),
                                            (40, 7, 0, 3), (1, 1, 1, 1), (0, 3, 3, 3), (1000, 999, 1001, None),
                                            (64, 8, 16, 0)])
def test_trajectory_events_match_reference_loop(total, ce, le, he):
    assert list(trajectory_events(total, ce, le, he)) == reference_loop(total, ce, le, he)


@pytest.mark.parametrize("max_time,tau", [(1.0, 5e-5), (0.5, 25e-6), (301.5 * 5e-5, 5e-5), (1e-3, 3e-4), (0.0, 1e-3)])
def test_timesteps_for_matches_reference_loop(max_time, tau):
    n, time = 0, 0.0
    while time < max_time:
        n += 1
        time = n * tau
    assert timesteps_for(max_time, tau) == n


@pytest.mark.parametrize("slots,bps", [(8, 1), (16, 4)])
def test_host_lattice_accessors(slots, bps):
    spec = configs.random_problem(3, X=8, Y=6, Z=4, slots=slots, bytes_per_slot=bps, density=0.3 * slots)
    h = HostLattice(spec.X, spec.Y, spec.Z, slots, bps, 1e-8)
    h.particles[:] = spec.lattice
    h.sites[:] = spec.sites
    table = configs.native_to_slots(spec.lattice, spec.X, spec.Y, spec.Z, slots, bps)
    x, y, z = 5, 2, 3
    i = x + y * spec.X + z * spec.X * spec.Y
    assert [h.getParticle(x, y, z, k) for k in range(slots)] == [int(v) for v in table[i]]
    assert h.getOccupancy(x, y, z) == int(np.count_nonzero(table[i]))
    assert h.getSiteType(x, y, z) == int(spec.sites[i])
    view = h.getParticleLatticeView()
    per = 4 if bps == 1 else 1
    assert view.shape == (h.words, spec.Z, spec.Y, spec.X, per)
    assert [int(view[k // per, z, y, x, k % per]) for k in range(slots)] == [int(v) for v in table[i]]
    assert h.getSiteLatticeView()[z, y, x] == spec.sites[i]
    counts = h.getParticleCounts()
    ref = configs.species_counts(spec.lattice, spec.nsites, slots, bps, spec.ns)
    assert counts == {s: int(ref[s]) for s in range(1, spec.ns + 1) if ref[s]}
    h.removeParticles(x, y, z)
    assert h.getOccupancy(x, y, z) == 0
    h.addParticle(x, y, z, 2)
    h.addParticle(x, y, z, 1)
    assert [h.getParticle(x, y, z, 0), h.getParticle(x, y, z, 1)] == [2, 1]
    for _ in range(slots - 2):
        h.addParticle(x, y, z, 3)
    with pytest.raises(ValueError):
        h.addParticle(x, y, z, 3)
    with pytest.raises(IndexError):
        h.getSiteType(spec.X, 0, 0)


def test_lattice_constructors_and_row_major_export():
    """lm.ByteLattice / lm.IntLattice built in a script, filled with
    addParticle, exported in the row-major order buildDiffusionModel takes."""
    from lattice_microbes_b200 import configs
    from lattice_microbes_b200.rdme import ByteLattice, IntLattice, getCompiledLatticeMaxOccupancy
    assert getCompiledLatticeMaxOccupancy() == 16
    for cls, bps in ((ByteLattice, 1), (IntLattice, 4)):
        lat = cls(6, 5, 4, 16e-9, 8)
        assert (lat.getXSize(), lat.getMaxOccupancy(), lat.getSpacing()) == (6, 8, 16e-9)
        rng = np.random.default_rng(bps)
        want = np.zeros((6, 5, 4, 8), dtype=np.uint8 if bps == 1 else np.uint32)
        for _ in range(60):
            x, y, z = (int(v) for v in rng.integers(0, (6, 5, 4)))
            n = lat.getOccupancy(x, y, z)
            if n < 8:
                sp = int(rng.integers(1, 200))
                lat.addParticle(x, y, z, sp)
                want[x, y, z, n] = sp
        lat.setSiteType(1, 2, 3, 2)
        p, s = lat.rowMajor()
        assert p.dtype == want.dtype and np.array_equal(p, want)
        assert s.shape == (6, 5, 4) and s[1, 2, 3] == 2 and s.sum() == 2
        # the native words agree with the oracle-side reader
        slots = configs.native_to_slots(lat.particles, 6, 5, 4, 8, bps)
        assert np.array_equal(slots.reshape(4, 5, 6, 8).transpose(2, 1, 0, 3), want)


def test_checkpoint_timer_checkpoints_at_the_next_record():
    """The CheckpointSignaler stand-in: a checkpoint at the first record once
    the interval has passed, none before, none without an interval."""
    from lattice_microbes_b200.rdme import MpdRdmeSolver

    class Out:
        n = 0

        def checkpoint(self):
            Out.n += 1

    s = MpdRdmeSolver.__new__(MpdRdmeSolver)
    s.output, s.checkpointInterval, s._last_checkpoint = Out(), 0.0, 0.0
    s._maybe_checkpoint()
    assert Out.n == 0
    import time
    s.checkpointInterval, s._last_checkpoint = 3600.0, time.monotonic()
    s._maybe_checkpoint()
    assert Out.n == 0
    s._last_checkpoint -= 3601.0
    s._maybe_checkpoint()
    s._maybe_checkpoint()
    assert Out.n == 1
