"""The oracle restatement against the reference (CPU only).

1. Known answers of the device hash and reaction probability, recorded from
   the reference's own device functions (tests/golden/hash_kat.npz).
2. Golden lattices produced by the reference's device functions
   (tests/golden/*.npz) replayed through the C restatement, bit for bit.
3. Where the reference checkers are built (oracle/_ref), fresh seeded problems
   run through both, bit for bit, including heavy overflow traffic and the
   error paths (overflow list exhausted, unplaceable particle).
"""
import numpy as np
import pytest

from lattice_microbes_b200 import configs
from tests.cases import oracle_tables
from tests.golden_lib import case_names, load_case, load_kat
from tests.oracle_lib import oracle, oracle_counts, oracle_run, reference, reference_run


def test_hash_known_answers():
    kat = load_kat()
    lib = oracle()
    for k, t, h in zip(kat["keys"], kat["ths"], kat["hash"]):
        assert lib.orc_hash(int(k), int(t)) == int(h)
    for a, b, t, f in zip(kat["v1"], kat["v2"], kat["ths"], kat["hash_float"]):
        key = (int(a) << 3) | int(b)
        assert np.float32(lib.orc_hash_float(key, int(t))) == f


def test_reaction_probability_known_answers():
    kat = load_kat()
    r = kat["rates"].astype(np.float32)
    p = (1.0 - np.exp(-r.astype(np.float64))).astype(np.float32)
    assert np.array_equal(p, kat["prob"])


def test_timestep_hash_properties():
    lib = oracle()
    seen = {lib.orc_timestep_hash(s, t, k) for s in (1, 2) for t in range(50) for k in range(4)}
    assert len(seen) == 400
    assert lib.orc_compose_seed(0x12345, 7) == ((0x12345 << 16) | 7) & 0xFFFFFFFF


@pytest.mark.parametrize("name", case_names())
def test_golden_replay(name):
    t, g = load_case(name)
    out, rc, stats = oracle_run(t, g["lattice_in"], g["sites"], int(g["seed"]), int(g["step0"]),
                                int(g["nsteps"]))
    assert rc == 0
    assert stats.overflows == int(g["overflows"])
    assert stats.reactions == int(g["reactions"])
    assert np.array_equal(out, g["lattice_out"])


def _have_reference(kind, slots):
    return reference(kind, slots) is not None


VARIANTS = [(8, 1), (16, 1), (16, 4), (8, 4)]


@pytest.mark.parametrize("slots,bps", VARIANTS)
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_vs_reference(seed, slots, bps):
    kind = "byte" if bps == 1 else "int"
    if not _have_reference(kind, slots):
        pytest.skip("reference checker not built")
    spec = configs.random_problem(seed, X=32, Y=16, Z=16, slots=slots, bytes_per_slot=bps,
                                  density=0.4 if slots == 8 else 0.9)
    t = oracle_tables(spec)
    a, rc, st = oracle_run(t, spec.lattice, spec.sites, 1234 + seed, 3, 8)
    b, rc2, ovf, rx = reference_run(t, spec.lattice, spec.sites, 1234 + seed, 3, 8)
    assert rc == rc2 == 0
    assert (st.overflows, st.reactions) == (ovf, rx)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("slots,bps,dens", [(8, 1, 5.0), (16, 4, 12.0), (8, 4, 6.0)])
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_overflow_storm_vs_reference(seed, slots, bps, dens):
    kind = "byte" if bps == 1 else "int"
    if not _have_reference(kind, slots):
        pytest.skip("reference checker not built")
    spec = configs.random_problem(seed, X=32, Y=8, Z=8, slots=slots, bytes_per_slot=bps, density=dens, nst=2)
    t = oracle_tables(spec)
    a, rc, st = oracle_run(t, spec.lattice, spec.sites, 99 + seed, 5, 8)
    b, rc2, ovf, rx = reference_run(t, spec.lattice, spec.sites, 99 + seed, 5, 8)
    assert rc == rc2
    assert (st.overflows, st.reactions) == (ovf, rx)
    assert np.array_equal(a, b)


def test_config0_vs_reference():
    if not _have_reference("byte", 8):
        pytest.skip("reference checker not built")
    spec = configs.config0(seed=3)
    t = oracle_tables(spec)
    a, rc, st = oracle_run(t, spec.lattice, spec.sites, 77, 0, 60)
    b, rc2, ovf, rx = reference_run(t, spec.lattice, spec.sites, 77, 0, 60)
    assert rc == rc2 == 0
    assert np.array_equal(a, b)


def test_counts_vs_reference():
    if not _have_reference("int", 16):
        pytest.skip("reference checker not built")
    import ctypes as C
    spec = configs.random_problem(5, X=32, Y=8, Z=8, slots=16, bytes_per_slot=4, density=3.0)
    t = oracle_tables(spec)
    ours = oracle_counts(t, spec.lattice)
    ref = np.zeros(spec.ns + 1, dtype=np.uint64)
    lat = np.ascontiguousarray(spec.lattice)
    reference("int", 16).ref_particle_counts(spec.X, spec.Y, spec.Z, lat.ctypes.data_as(C.POINTER(C.c_uint32)),
                                             spec.ns, ref.ctypes.data_as(C.POINTER(C.c_uint64)))
    assert np.array_equal(ours[1:], ref[1:])


def test_pure_diffusion_conserves_species():
    spec = configs.random_problem(9, X=32, Y=8, Z=8, slots=8, bytes_per_slot=1, density=0.8, nr=0)
    t = oracle_tables(spec)
    before = oracle_counts(t, spec.lattice)
    out, rc, st = oracle_run(t, spec.lattice, spec.sites, 5, 0, 30)
    assert rc == 0
    assert np.array_equal(before, oracle_counts(t, out))
