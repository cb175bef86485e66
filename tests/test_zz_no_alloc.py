"""The species count that allocates no device memory, against the regular one.

lmb_species_counts_noalloc serves callers that cannot allocate device memory
when they count (their own pool allocator owns the device, or they count from
a hook or a memory-capped serving loop).  It keeps its device totals in a
fixed array instead of a buffer from cudaMalloc.  This file is collected last
so that a failure here comes after every other test has run; it also passes
alone in a fresh process, where its first call sets up the array.
"""
import ctypes as C

import numpy as np
import pytest

from lattice_microbes_b200 import configs

pytestmark = pytest.mark.gpu


def _noalloc_counts(lat, ns):
    from lattice_microbes_b200 import _lib as L
    dev_particles, _ = lat.device_buffers()
    out = np.zeros(ns + 1, dtype=np.uint64)
    rc = L.lib().lmb_species_counts_noalloc(C.c_void_p(dev_particles), lat.X, lat.Y, lat.Z, lat.slots,
                                            lat.bytes_per_slot, ns, out.ctypes.data_as(L.u64p),
                                            C.c_void_p(lat.ctx.stream))
    return rc, out


@pytest.mark.parametrize("slots,bps", [(8, 1), (16, 4)])
def test_noalloc_counts_match_regular_counts_twice(gpu, slots, bps):
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import Context, Lattice, Model
    spec = configs.random_problem(31, X=32, Y=16, Z=16, slots=slots, bytes_per_slot=bps, density=0.8, ns=7)
    ctx = Context(0)
    model = Model.from_spec(ctx, spec)
    lat = Lattice(ctx, spec.X, spec.Y, spec.Z, slots, bps)
    lat.set_native(spec.lattice, spec.sites)
    # First call: counts of the initial lattice.
    rc, got = _noalloc_counts(lat, spec.ns)
    assert rc == L.LMB_OK
    assert np.array_equal(got, lat.species_counts(spec.ns))
    # Second call after the lattice changed: the shared array must not carry
    # the first call's totals.
    lat.run(model, 99, 0, 25)
    rc, got2 = _noalloc_counts(lat, spec.ns)
    assert rc == L.LMB_OK
    assert np.array_equal(got2, lat.species_counts(spec.ns))
    assert got2.sum() > 0
    lat.close()
    model.close()
    ctx.close()


def test_noalloc_rejects_too_many_species(gpu):
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import Context, Lattice
    ctx = Context(0)
    lat = Lattice(ctx, 16, 8, 8, 8, 1)
    dev_particles, _ = lat.device_buffers()
    out = np.zeros(L.LMB_NOALLOC_MAX_SPECIES + 2, dtype=np.uint64)
    rc = L.lib().lmb_species_counts_noalloc(C.c_void_p(dev_particles), 16, 8, 8, 8, 1,
                                            L.LMB_NOALLOC_MAX_SPECIES + 1, out.ctypes.data_as(L.u64p),
                                            C.c_void_p(ctx.stream))
    assert rc == L.LMB_E_UNSUPPORTED
    lat.close()
    ctx.close()
