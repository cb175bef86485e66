"""Batched lattices: one launch per timestep for many lattices of uneven
size must leave every lattice exactly where a run of that lattice alone
leaves it (and where the oracle does)."""
import numpy as np
import pytest

from lattice_microbes_b200 import configs
from tests.cases import oracle_tables
from tests.oracle_lib import oracle_run

pytestmark = pytest.mark.gpu


def _make(ctx, spec):
    from lattice_microbes_b200.solver import Lattice, Model
    m = Model.from_spec(ctx, spec)
    lat = Lattice(ctx, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
    lat.set_native(spec.lattice, spec.sites)
    return lat, m


@pytest.mark.parametrize("steps", [7, 70])
def test_batch_of_uneven_lattices_vs_single_runs_and_oracle(gpu, steps):
    from lattice_microbes_b200.solver import Batch, Context
    ctx = Context(0)
    edges = [16, 24, 32, 48, 16, 24]
    specs = [configs.config0(seed=100 + k, edge=e, nA=int(0.4 * e ** 3), nB=int(0.4 * e ** 3))
             for k, e in enumerate(edges)]
    seeds = [1000 + 7 * k for k in range(len(specs))]
    pairs = [_make(ctx, s) for s in specs]
    batch = Batch(ctx, [p[0] for p in pairs], [p[1] for p in pairs])
    # Two runs in a row: the second starts from a different buffer parity.
    rc, st = batch.run(seeds, 0, steps)
    assert rc == 0
    rc, st2 = batch.run(seeds, steps, steps + 3)
    assert rc == 0
    for (lat, m), spec, seed, s1, s2 in zip(pairs, specs, seeds, st, st2):
        out, _ = lat.get_native()
        ref, rc_ref, st_ref = oracle_run(oracle_tables(spec), spec.lattice, spec.sites, seed, 0, 2 * steps + 3)
        assert rc_ref == 0
        assert s1.overflows + s2.overflows == st_ref.overflows
        assert s1.reactions + s2.reactions == st_ref.reactions
        assert np.array_equal(out, ref), spec.name
    batch.close()
    for lat, m in pairs:
        lat.close()
        m.close()
    ctx.close()


def test_batch_failure_is_per_lattice(gpu):
    """An over-full lattice fails with the overflow error; its neighbours in
    the batch still finish."""
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import Batch, Context
    ctx = Context(0)
    good = configs.config0(seed=5, edge=16)
    bad = configs.random_problem(1, X=32, Y=8, Z=8, slots=8, bytes_per_slot=1, density=5.0, nst=2)
    pg, pb = _make(ctx, good), _make(ctx, bad)
    batch = Batch(ctx, [pg[0], pb[0]], [pg[1], pb[1]])
    rc, st = batch.run([3, 4], 0, 12, check=False)
    ref_bad, rc_bad, _ = oracle_run(oracle_tables(bad), bad.lattice, bad.sites, 4, 0, 12)
    assert rc_bad != 0 and rc == rc_bad
    assert st[0].status == 0 and st[1].status == rc_bad
    ref_good, _, _ = oracle_run(oracle_tables(good), good.lattice, good.sites, 3, 0, 12)
    assert np.array_equal(pg[0].get_native()[0], ref_good)
    assert np.array_equal(pb[0].get_native()[0], ref_bad)
    batch.close()
    ctx.close()


def test_batch_autotune_keeps_state_and_results(gpu):
    """lmb_batch_autotune times tile shapes per lattice size from the saved
    states and leaves every lattice where it was; the batch then runs with the
    chosen plan and still gives every lattice the oracle's result."""
    from lattice_microbes_b200.solver import Batch, Context
    ctx = Context(0)
    edges = [16, 24, 32, 48, 64, 16, 32]
    specs = [configs.config0(seed=200 + k, edge=e, nA=int(0.2 * e ** 3), nB=int(0.2 * e ** 3))
             for k, e in enumerate(edges)]
    seeds = [77 + k for k in range(len(specs))]
    pairs = [_make(ctx, s) for s in specs]
    batch = Batch(ctx, [p[0] for p in pairs], [p[1] for p in pairs])
    before = [lat.get_native()[0] for lat, _ in pairs]
    ms = batch.autotune(seeds, 0, 8)
    assert 0 < ms < 1e6
    for (lat, _), b in zip(pairs, before):
        assert np.array_equal(lat.get_native()[0], b)
    plan = batch.plan()
    assert len(plan) == len(edges)
    for e, (ty, tz) in zip(edges, plan):
        assert ty >= 1 and tz >= 1 and e % ty == 0 and e % tz == 0
    # Lattices of one size share a plan.
    assert plan[0] == plan[5] and plan[2] == plan[6]
    rc, st = batch.run(seeds, 0, 20)
    assert rc == 0
    for (lat, m), spec, seed in zip(pairs, specs, seeds):
        ref, rc_ref, _ = oracle_run(oracle_tables(spec), spec.lattice, spec.sites, seed, 0, 20)
        assert rc_ref == 0
        assert np.array_equal(lat.get_native()[0], ref), spec.name
    batch.close()
    for lat, m in pairs:
        lat.close()
        m.close()
    ctx.close()
