"""Edge cases of the CUDA path against the oracle: empty lattices (with and
without zeroth-order reactions, which fill them), runs of zero timesteps, a
single-site lattice, byte lattices whose species ids reach 250, and the
sizes and slot layouts the library rejects before allocating anything."""
import numpy as np
import pytest

from lattice_microbes_b200 import configs
from tests.cases import oracle_tables
from tests.oracle_lib import oracle_run
from tests.test_gpu_parity import SCHEDULES, _gpu_run

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(gpu):
    from lattice_microbes_b200.solver import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("schedule", SCHEDULES)
@pytest.mark.parametrize("zeroth", [False, True])
@pytest.mark.parametrize("slots,bps", [(8, 1), (16, 4)])
def test_empty_lattice_vs_oracle(ctx, zeroth, slots, bps, schedule):
    """No particles at all: without zeroth-order reactions the lattice stays
    empty; with them particles appear exactly where the oracle puts them."""
    spec = configs.random_problem(31, X=32, Y=8, Z=8, slots=slots, bytes_per_slot=bps, density=0.0, zeroth=zeroth)
    assert not spec.lattice.any()
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 3, 0, 12)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 3, 0, 12, schedule=schedule)
    assert rc == rc_ref == 0
    assert st[0].reactions == st_ref.reactions
    assert np.array_equal(out, ref)
    assert out.any() == zeroth


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_zero_timesteps_leave_the_lattice(ctx, schedule):
    spec = configs.random_problem(32, X=32, Y=8, Z=8, density=1.0)
    t = oracle_tables(spec)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 3, 5, 0, schedule=schedule)
    assert rc == 0
    assert (st[0].overflows, st[0].reactions) == (0, 0)
    assert np.array_equal(out, spec.lattice)


@pytest.mark.parametrize("schedule", SCHEDULES)
@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 1, 5), (3, 1, 1)])
def test_tiny_lattices_vs_oracle(ctx, shape, schedule):
    """Every neighbour of a site is the site itself or its only partner."""
    X, Y, Z = shape
    spec = configs.random_problem(33, X=X, Y=Y, Z=Z, density=3.0, nst=1)
    t = oracle_tables(spec)
    ref, rc_ref, _ = oracle_run(t, spec.lattice, spec.sites, 4, 0, 9)
    out, rc, _ = _gpu_run(ctx, t, spec.lattice, spec.sites, 4, 0, 9, schedule=schedule)
    assert rc == rc_ref
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_byte_lattice_with_250_species_vs_oracle(ctx, schedule):
    """Species ids up to 250 in byte slots (the byte lattice's range)."""
    spec = configs.random_problem(34, X=32, Y=16, Z=8, slots=8, bytes_per_slot=1, ns=250, nr=40, density=2.0)
    assert int(configs.native_to_slots(spec.lattice, spec.X, spec.Y, spec.Z, 8, 1).max()) > 200
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 6, 0, 10)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 6, 0, 10, schedule=schedule)
    assert rc == rc_ref == 0
    assert st[0].reactions == st_ref.reactions
    assert np.array_equal(out, ref)


def test_rejected_sizes_and_layouts(ctx):
    """Site indices are 32-bit and the slot layouts are the reference's:
    anything else is refused before any device allocation."""
    import ctypes as C
    from lattice_microbes_b200 import _lib as L
    h = L.vp()
    lib = L.lib()
    assert lib.lmb_lattice_create(ctx.handle, 2048, 2048, 1025, 8, 1, C.byref(h)) == L.LMB_E_UNSUPPORTED
    assert lib.lmb_lattice_create(ctx.handle, 0, 8, 8, 8, 1, C.byref(h)) == L.LMB_E_ARG
    assert lib.lmb_lattice_create(ctx.handle, 8, 8, 8, 12, 1, C.byref(h)) == L.LMB_E_UNSUPPORTED
    assert lib.lmb_lattice_create(ctx.handle, 8, 8, 8, 32, 4, C.byref(h)) == L.LMB_E_UNSUPPORTED
    assert lib.lmb_lattice_create(ctx.handle, 8, 8, 8, 8, 2, C.byref(h)) == L.LMB_E_UNSUPPORTED
