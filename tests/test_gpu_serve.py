"""Continuous batching: batch runs with per-lattice timestep ranges and the
solve server (lmb_server).

Every solve must end exactly where a run of it alone ends (lmb_run on the
same lattice, model, seed and timesteps): bit for bit, with the same
reaction and overflow counts, whatever else is resident beside it, however
its run is cut into chunks, and whenever it was admitted.
"""
import numpy as np
import pytest

from lattice_microbes_b200 import configs
from tests.cases import oracle_tables
from tests.oracle_lib import oracle_run

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(gpu):
    from lattice_microbes_b200.solver import Context
    c = Context(0)
    yield c
    c.close()


def solo(ctx, spec, seed, first, n, lattice=None):
    from lattice_microbes_b200.solver import Lattice, Model
    m = Model.from_spec(ctx, spec)
    lat = Lattice(ctx, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
    lat.set_native(spec.lattice if lattice is None else lattice, spec.sites)
    rc, st = lat.run(m, seed, first, n, check=False)
    out, _ = lat.get_native()
    counts = lat.species_counts(spec.ns)
    lat.close()
    m.close()
    return rc, st, out, counts


def small_requests(count, seed=0):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(count):
        r = configs.ServeRequest(index=k, arrival=0.0, edge=int(rng.choice([16, 24, 32])),
                                 ns=int(rng.integers(2, 9)), density=float(rng.uniform(0.5, 2.0)),
                                 timesteps=int(rng.integers(40, 400)), seed=int(rng.integers(1, 2 ** 31)))
        spec = configs.serve_problem(r)
        spec = _byte16(spec)
        reqs.append((r, spec, 1000 + 17 * k))
    return reqs


def _byte16(spec):
    """Same particles in a 16-slot byte lattice (the server's layout)."""
    N = spec.nsites
    slots = configs.native_to_slots(spec.lattice, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
    lat = configs.empty_lattice(spec.X, spec.Y, spec.Z, 16, 1)
    for k in range(spec.slots):
        v = slots[:, k].astype(np.uint32)
        lat[(k // 4) * N:(k // 4 + 1) * N] |= v << np.uint32(8 * (k % 4))
    spec.lattice, spec.slots = lat, 16
    return spec


def test_batch_ranges_match_single_runs(ctx):
    from lattice_microbes_b200.solver import Batch, Lattice, Model
    specs = [configs.config0(seed=40 + k, edge=e, nA=int(0.3 * e ** 3), nB=int(0.3 * e ** 3))
             for k, e in enumerate([16, 24, 32, 16])]
    seeds = [31, 32, 33, 34]
    firsts = [0, 5, 100, 7]
    counts = [70, 3, 41, 66]
    pairs = []
    for s in specs:
        m = Model.from_spec(ctx, s)
        lat = Lattice(ctx, s.X, s.Y, s.Z, 8, 1)
        lat.set_native(s.lattice, s.sites)
        pairs.append((lat, m))
    b = Batch(ctx, [p[0] for p in pairs], [p[1] for p in pairs])
    b.run_ranges_async(seeds, firsts, counts)
    rc, st = b.wait()
    assert rc == 0
    for (lat, m), s, sd, f, n, x in zip(pairs, specs, seeds, firsts, counts, st):
        assert x.steps_done == n
        out, _ = lat.get_native()
        rc1, st1, ref, _ = solo(ctx, s, sd, f, n)
        assert rc1 == 0
        assert np.array_equal(out, ref)
        assert (x.reactions, x.overflows) == (st1.reactions, st1.overflows)
    # A second run on another member set, continuing two of the lattices.
    b.set_lattices([pairs[2][0], pairs[0][0]], [pairs[2][1], pairs[0][1]])
    b.run_ranges_async([33, 31], [141, 70], [30, 90])
    rc, st = b.wait()
    assert rc == 0
    for (lat, m), s, sd, n in ((pairs[2], specs[2], 33, 171), (pairs[0], specs[0], 31, 160)):
        out, _ = lat.get_native()
        _, _, ref, _ = solo(ctx, s, sd, 100 if sd == 33 else 0, n - (100 if sd == 33 else 0))
        # lattice 2 started at timestep 100: replay from its initial state
        assert np.array_equal(out, ref)
    b.close()
    for lat, m in pairs:
        lat.close()
        m.close()


def drain(server, limit=10000):
    results = {}
    for _ in range(limit):
        a, q = server.step()
        while True:
            r = server.pop_result()
            if r is None:
                break
            results[r[0].id] = r
        if a == 0 and q == 0:
            break
    return results


def test_server_results_equal_solo_runs(ctx):
    from lattice_microbes_b200.solver import Server
    reqs = small_requests(12)
    # Two large solves (>= 128 Ki sites) run their chunks on their own: one
    # dense (per-phase kernels), one sparse (fused kernel).
    for k, dens in ((12, 1.0), (13, 0.02)):
        r = configs.ServeRequest(index=k, arrival=0.0, edge=56, ns=5, density=dens, timesteps=150, seed=99 + k)
        reqs.append((r, _byte16(configs.serve_problem(r)), 4000 + k))
    srv = Server(ctx, slots=16, bytes_per_slot=1, max_active=5, chunk_timesteps=64)
    for r, spec, seed in reqs[:7] + reqs[12:13]:
        srv.submit(r.index, spec, seed, r.timesteps)
    srv.step()
    srv.step()  # the rest arrive while the first ones are on the device
    for r, spec, seed in reqs[7:12] + reqs[13:]:
        srv.submit(r.index, spec, seed, r.timesteps)
    results = drain(srv)
    st = srv.status()
    assert st.peak_active == 5 and st.active == 0 and st.bytes_in_use == 0
    srv.close()
    assert sorted(results) == list(range(14))
    for r, spec, seed in reqs:
        info, lat, counts = results[r.index]
        assert info.stats.status == 0 and info.stats.steps_done == r.timesteps
        rc, st1, ref, ref_counts = solo(ctx, spec, seed, 0, r.timesteps)
        assert rc == 0
        assert np.array_equal(lat, ref), r
        assert np.array_equal(counts, ref_counts)
        assert (info.stats.reactions, info.stats.overflows) == (st1.reactions, st1.overflows)
        assert info.t_submit <= info.t_admit <= info.t_done


def test_server_budget_limits_residency(ctx):
    from lattice_microbes_b200.solver import Server
    rng = np.random.default_rng(3)
    reqs = []
    for k in range(6):  # all 32^3: the budget holds two of them
        r = configs.ServeRequest(index=k, arrival=0.0, edge=32, ns=int(rng.integers(2, 6)), density=1.0,
                                 timesteps=int(rng.integers(50, 300)), seed=int(rng.integers(1, 2 ** 31)))
        reqs.append((r, _byte16(configs.serve_problem(r)), 300 + k))
    one = 2 * 16 * 32 ** 3 + 32 ** 3 + 2048 * 16  # two 16-byte-per-site buffers, site types, overflow queue
    budget = int(2.5 * one)
    srv = Server(ctx, slots=16, bytes_per_slot=1, hbm_budget_bytes=budget, max_active=64, chunk_timesteps=128)
    for r, spec, seed in reqs:
        srv.submit(r.index, spec, seed, r.timesteps)
    big = configs.serve_problem(configs.ServeRequest(99, 0.0, 128, 3, 0.5, 10, 7))
    big = _byte16(big)
    srv.submit(99, big, 5, 10)  # larger than the whole budget: rejected, the rest continue
    results = drain(srv)
    st = srv.status()
    srv.close()
    assert st.peak_bytes <= budget
    assert 1 <= st.peak_active <= 2
    assert results[99][0].stats.status == -3  # LMB_E_NOMEM
    for r, spec, seed in reqs:
        info, lat, _ = results[r.index]
        assert info.stats.status == 0
        _, _, ref, _ = solo(ctx, spec, seed, 0, r.timesteps)
        assert np.array_equal(lat, ref)


def test_server_isolates_a_failing_solve(ctx):
    """A solve that ends in the reference's overflow error stops at the same
    timestep as the oracle says; its neighbours in the batch are untouched."""
    from lattice_microbes_b200.solver import Server
    bad = None
    for seed in range(1, 8):
        spec = configs.random_problem(seed, X=32, Y=8, Z=8, slots=16, bytes_per_slot=1, density=13.0, nst=2)
        ref, rc_ref, st_ref = oracle_run(oracle_tables(spec), spec.lattice, spec.sites, 500 + seed, 0, 12)
        if rc_ref != 0:
            bad = (spec, 500 + seed, rc_ref, ref)
            break
    assert bad is not None
    reqs = small_requests(4, seed=9)
    srv = Server(ctx, slots=16, bytes_per_slot=1, max_active=8, chunk_timesteps=8)
    for r, spec, seed in reqs[:2]:
        srv.submit(r.index, spec, seed, r.timesteps)
    srv.submit(77, bad[0], bad[1], 12)
    for r, spec, seed in reqs[2:]:
        srv.submit(r.index, spec, seed, r.timesteps)
    results = drain(srv)
    srv.close()
    info, lat, _ = results[77]
    assert info.stats.status == bad[2]
    assert np.array_equal(lat, bad[3])
    for r, spec, seed in reqs:
        info, lat, _ = results[r.index]
        assert info.stats.status == 0
        _, _, ref, _ = solo(ctx, spec, seed, 0, r.timesteps)
        assert np.array_equal(lat, ref)
