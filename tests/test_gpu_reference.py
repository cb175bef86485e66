"""The reference's own kernels, compiled for sm_100a from its sources, on the
GPU: they must agree bit for bit with the oracle and with the product's
kernels on lattices the reference accepts (X % 32, Y % 8, Z % 8).  This pins
the device-side arithmetic (CUDA double exp, nvcc's default contraction)."""
import numpy as np
import pytest

from lattice_microbes_b200 import configs
from tests.cases import oracle_tables
from tests.oracle_lib import oracle_run, reference_gpu, reference_gpu_run

pytestmark = pytest.mark.gpu


def _need(kind, slots, nofma=False):
    if reference_gpu(kind, slots, nofma) is None:
        pytest.skip("GPU reference checker not built (make -C oracle ref-gpu)")


def _ours(spec_or_tables, lattice, sites, seed, step0, n, from_spec=False):
    from lattice_microbes_b200.solver import Context, Lattice, Model
    ctx = Context(0)
    t = spec_or_tables
    m = Model.from_spec(ctx, t) if from_spec else Model.from_tables(ctx, t)
    lat = Lattice(ctx, t.X, t.Y, t.Z, t.slots, t.bytes_per_slot)
    lat.set_native(lattice, sites)
    rc, st = lat.run(m, seed, step0, n, check=False)
    out, _ = lat.get_native()
    lat.close()
    m.close()
    ctx.close()
    return out, rc, st


@pytest.mark.parametrize("nofma", [False, True])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_reference_kernels_byte8(gpu, seed, nofma):
    _need("byte", 8, nofma)
    spec = configs.random_problem(seed, X=32, Y=16, Z=16, slots=8, bytes_per_slot=1, density=0.7)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 808 + seed, 2, 15)
    r = reference_gpu_run(t, spec.lattice, spec.sites, 808 + seed, 2, 15, nofma)
    assert r is not None
    g, rc_g, ovf_g = r
    assert rc_g == rc_ref == 0
    assert ovf_g == st_ref.overflows
    assert np.array_equal(g, ref)
    ours, rc, st = _ours(t, spec.lattice, spec.sites, 808 + seed, 2, 15)
    assert rc == 0
    assert np.array_equal(ours, g)


@pytest.mark.parametrize("seed", [3, 4])
def test_reference_kernels_int16(gpu, seed):
    _need("int", 16)
    spec = configs.random_problem(seed, X=32, Y=16, Z=8, slots=16, bytes_per_slot=4, density=2.0, ns=9)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 9 + seed, 0, 10)
    g, rc_g, ovf_g = reference_gpu_run(t, spec.lattice, spec.sites, 9 + seed, 0, 10)
    assert rc_g == rc_ref == 0
    assert np.array_equal(g, ref)
    ours, rc, st = _ours(t, spec.lattice, spec.sites, 9 + seed, 0, 10)
    assert np.array_equal(ours, g)


def test_reference_kernels_config0_long(gpu):
    """Config-0 chemistry, 2000 timesteps: reference kernels vs ours."""
    _need("byte", 8)
    spec = configs.config0(seed=11)
    t = oracle_tables(spec)
    g, rc_g, _ = reference_gpu_run(t, spec.lattice, spec.sites, 4242, 0, 2000)
    assert rc_g == 0
    ours, rc, st = _ours(spec, spec.lattice, spec.sites, 4242, 0, 2000, from_spec=True)
    assert rc == 0
    assert st.reactions > 0
    assert np.array_equal(ours, g)


def test_reference_kernels_config1_short(gpu):
    _need("byte", 8)
    spec = configs.config1(seed=5)
    t = oracle_tables(spec)
    g, rc_g, _ = reference_gpu_run(t, spec.lattice, spec.sites, 77, 0, 200)
    assert rc_g == 0
    ours, rc, st = _ours(spec, spec.lattice, spec.sites, 77, 0, 200, from_spec=True)
    assert rc == 0
    assert np.array_equal(ours, g)


@pytest.mark.parametrize("schedule", ["phases", "fused"])
def test_reference_kernels_config2_full_size(gpu, schedule):
    """The crowded cell at full size (128x128x256 IntLattice-16, 8 site types,
    200 species, 500 reactions, 1M particles), 30 timesteps: the reference
    kernels and ours give the same lattice, with no overflow on either side
    (an overflow's reinsertion order is not deterministic in the reference)."""
    _need("int", 16)
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import Context, Lattice, Model
    spec = configs.config2(seed=3)
    t = oracle_tables(spec)
    g, rc_g, ovf_g = reference_gpu_run(t, spec.lattice, spec.sites, 5150, 0, 30)
    assert rc_g == 0 and ovf_g == 0
    assert not np.array_equal(g, spec.lattice)
    ctx = Context(0)
    m = Model.from_spec(ctx, spec)
    lat = Lattice(ctx, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
    lat.set_native(spec.lattice, spec.sites)
    if schedule == "phases":
        lat.set_schedule(L.LMB_SCHEDULE_PHASES)
    else:
        lat.set_schedule(L.LMB_SCHEDULE_FUSED, 1, 1)  # the one tile of 128-site Int-16 rows that fits
    rc, st = lat.run(m, 5150, 0, 30, check=False)
    out, _ = lat.get_native()
    lat.close()
    m.close()
    ctx.close()
    assert rc == 0
    assert st.overflows == 0
    assert st.reactions > 0
    assert np.array_equal(out, g)
