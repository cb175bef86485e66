"""CUDA path (through the C ABI) against the oracle and the golden fixtures.

Integer lattice state must match bit for bit.  The classic overflow handler
is compared for the canonical reinsertion order (sorted by sweep, site,
slot); the oracle uses the same order and is itself pinned to the
reference's device functions.
"""
import numpy as np
import pytest

from lattice_microbes_b200 import configs
from tests.cases import oracle_tables
from tests.golden_lib import case_names, load_case
from tests.oracle_lib import oracle_counts, oracle_run

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(gpu):
    from lattice_microbes_b200.solver import Context
    c = Context(0)
    yield c
    c.close()


SCHEDULES = ["fused", "phases"]


def _gpu_run(ctx, tables_or_spec, lattice, sites, seed, step0, nsteps, mode=0, from_spec=False, chunks=None,
             schedule="fused", tile=(0, 0)):
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import Lattice, Model
    t = tables_or_spec
    model = Model.from_spec(ctx, t) if from_spec else Model.from_tables(ctx, t)
    lat = Lattice(ctx, t.X, t.Y, t.Z, t.slots, t.bytes_per_slot)
    if schedule == "phases":
        lat.set_schedule(L.LMB_SCHEDULE_PHASES)
    elif schedule == "cluster":
        lat.set_schedule(L.LMB_SCHEDULE_CLUSTER)
    elif schedule == "grid":
        lat.set_schedule(L.LMB_SCHEDULE_GRID, *tile)
    else:
        lat.set_schedule(L.LMB_SCHEDULE_FUSED, *tile)
    lat.set_native(lattice, sites)
    if chunks is None:
        chunks = [nsteps]
    step, stats, rc = step0, [], 0
    for n in chunks:
        rc, st = lat.run(model, seed, step, n, mode, check=False)
        stats.append(st)
        step += n
        if rc:
            break
    out, _ = lat.get_native()
    lat.close()
    model.close()
    return out, rc, stats


@pytest.mark.parametrize("schedule", SCHEDULES)
@pytest.mark.parametrize("name", case_names())
def test_golden_fixture(ctx, name, schedule):
    t, g = load_case(name)
    out, rc, st = _gpu_run(ctx, t, g["lattice_in"], g["sites"], int(g["seed"]), int(g["step0"]), int(g["nsteps"]),
                           schedule=schedule)
    assert rc == 0
    assert st[0].overflows == int(g["overflows"])
    assert st[0].reactions == int(g["reactions"])
    assert np.array_equal(out, g["lattice_out"])


VARIANTS = [(4, 1), (8, 1), (16, 1), (32, 1), (4, 4), (8, 4), (16, 4)]


@pytest.mark.parametrize("schedule", SCHEDULES)
@pytest.mark.parametrize("slots,bps", VARIANTS)
@pytest.mark.parametrize("seed", [0, 1])
def test_random_problem_vs_oracle(ctx, seed, slots, bps, schedule):
    if schedule == "fused" and slots > 16:
        pytest.skip("the fused schedule covers up to 16 slots; 32-slot lattices use the per-phase kernels")
    dens = {4: 0.3, 8: 0.5, 16: 1.2, 32: 2.0}[slots]
    spec = configs.random_problem(seed, X=32, Y=16, Z=16, slots=slots, bytes_per_slot=bps, density=dens)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 4321 + seed, 11, 12)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 4321 + seed, 11, 12, schedule=schedule)
    assert rc == rc_ref == 0
    assert (st[0].overflows, st[0].reactions) == (st_ref.overflows, st_ref.reactions)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("schedule", SCHEDULES)
@pytest.mark.parametrize("shape", [(16, 24, 8), (24, 16, 40), (7, 5, 3), (48, 8, 16), (1, 8, 8), (200, 2, 1)])
def test_odd_shapes_vs_oracle(ctx, shape, schedule):
    X, Y, Z = shape
    spec = configs.random_problem(5, X=X, Y=Y, Z=Z, density=0.6)
    t = oracle_tables(spec)
    ref, rc_ref, _ = oracle_run(t, spec.lattice, spec.sites, 99, 0, 10)
    out, rc, _ = _gpu_run(ctx, t, spec.lattice, spec.sites, 99, 0, 10, schedule=schedule)
    assert rc == rc_ref
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("slots,bps", [(8, 1), (16, 1), (16, 4), (4, 4)])
@pytest.mark.parametrize("shape", [(96, 3, 5), (300, 4, 12), (40, 12, 9), (33, 1, 2), (64, 2, 17)])
def test_sweep_tiles_vs_oracle(ctx, shape, slots, bps):
    """Per-phase sweeps on shapes that exercise every tile form: x rows longer
    than one block, y and z axes shorter than a tile, tiles cut off by the
    end of the axis, blocks wider than the lattice, dense sites."""
    X, Y, Z = shape
    spec = configs.random_problem(11, X=X, Y=Y, Z=Z, slots=slots, bytes_per_slot=bps, density=0.4 * slots, nst=3)
    t = oracle_tables(spec)
    ref, rc_ref, _ = oracle_run(t, spec.lattice, spec.sites, 7, 3, 6)
    out, rc, _ = _gpu_run(ctx, t, spec.lattice, spec.sites, 7, 3, 6, schedule="phases")
    assert rc == rc_ref
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("slots,bps", VARIANTS)
@pytest.mark.parametrize("shape,per_slot", [((32, 20, 7), 0.3), ((64, 16, 33), 0.05), ((256, 3, 18), 0.12),
                                             ((96, 1, 1), 0.2), ((32, 17, 16), 0.25)])
def test_particle_sweep_vs_oracle(ctx, shape, per_slot, slots, bps):
    """Per-phase runs on lattices whose x rows are whole segments of 32 sites
    and fit one block, which sweep by particle with plane bounds (IntLattices
    and ByteLattices of up to 16 slots; ByteLattice-32 keeps the sweep by
    site): y and z tiles cut off by the end of the axis, axes of one site,
    sparse sites whose bounds stay low and full sites that overflow (up to
    2,962 overflows in six timesteps)."""
    X, Y, Z = shape
    spec = configs.random_problem(61, X=X, Y=Y, Z=Z, slots=slots, bytes_per_slot=bps, density=per_slot * slots,
                                  nst=3)
    t = oracle_tables(spec)
    ref, rc_ref, _ = oracle_run(t, spec.lattice, spec.sites, 17, 2, 6)
    out, rc, _ = _gpu_run(ctx, t, spec.lattice, spec.sites, 17, 2, 6, schedule="phases")
    assert rc == rc_ref
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("slots,bps", [(8, 1), (16, 4)])
@pytest.mark.parametrize("shape,per_slot", [((64, 32, 32), 0.03), ((64, 32, 32), 0.15), ((64, 64, 32), 0.3)])
def test_reaction_site_list_vs_oracle(ctx, shape, per_slot, slots, bps):
    """Per-phase schedule: the z sweep lists the sites whose reaction step
    could change them.  Sparse lattices react over the list; the dense one
    lists more sites than the list holds (N / 8 + 4096) and reacts over every
    site.  Zeroth-order reactions list empty sites too."""
    X, Y, Z = shape
    spec = configs.random_problem(21, X=X, Y=Y, Z=Z, slots=slots, bytes_per_slot=bps, density=per_slot * slots,
                                  nst=3, qmax=0.3)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 5, 0, 3)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 5, 0, 3, schedule="phases")
    assert rc == rc_ref
    if rc == 0:
        assert st[0].reactions == st_ref.reactions
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("slots,bps,zeroth", [(8, 1, False), (16, 1, True), (16, 4, True)])
def test_reaction_list_skip_window_vs_oracle(ctx, slots, bps, zeroth):
    """A dense lattice whose reaction list overflows: the next 31 timesteps
    react over every site without building the list, then the list is
    tried again; 40 timesteps cross that window, in graph replays and in
    single launches."""
    spec = configs.random_problem(22, X=64, Y=32, Z=32, slots=slots, bytes_per_slot=bps, density=0.2 * slots,
                                  nst=3, qmax=0.3, zeroth=zeroth)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 8, 0, 40)
    assert rc_ref == 0
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 8, 0, 40, schedule="phases", chunks=[33, 7])
    assert rc == rc_ref
    if rc == 0:
        assert sum(x.reactions for x in st) == st_ref.reactions
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("schedule", SCHEDULES)
@pytest.mark.parametrize("slots,bps,dens", [(8, 1, 5.0), (16, 4, 12.0), (8, 4, 6.0)])
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_overflow_storm_vs_oracle(ctx, seed, slots, bps, dens, schedule):
    """Heavy overflow traffic; seeds 1-3 end in the reference's two errors
    (list exhausted / no free site), which must stop at the same step with
    the same partial lattice."""
    spec = configs.random_problem(seed, X=32, Y=8, Z=8, slots=slots, bytes_per_slot=bps, density=dens, nst=2)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 99 + seed, 5, 8)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 99 + seed, 5, 8, schedule=schedule)
    assert rc == rc_ref
    if rc == 0:
        assert st[0].overflows == st_ref.overflows
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_relaxed_handler_vs_oracle(ctx, schedule):
    spec = configs.random_problem(2, X=32, Y=8, Z=8, slots=8, bytes_per_slot=1, density=3.0, nst=2)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 7, 0, 6, mode=1)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 7, 0, 6, mode=1, schedule=schedule)
    assert rc == rc_ref
    assert st[-1].unresolved == st_ref.unresolved
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("X", [32, 24])
@pytest.mark.parametrize("tile", [(1, 1), (2, 4), (4, 2), (8, 8), (16, 8)])
def test_fused_tile_shapes_vs_oracle(ctx, tile, X):
    spec = configs.random_problem(12, X=X, Y=16, Z=32, density=0.8, nst=3)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 1717, 3, 9)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 1717, 3, 9, tile=tile)
    assert rc == rc_ref == 0
    assert st[0].overflows == st_ref.overflows
    assert np.array_equal(out, ref)


def test_autotune_keeps_state_and_result(ctx):
    from lattice_microbes_b200.solver import Lattice, Model
    spec = configs.config0(seed=7)
    t = oracle_tables(spec)
    m = Model.from_spec(ctx, spec)
    lat = Lattice(ctx, spec.X, spec.Y, spec.Z, 8, 1)
    lat.set_native(spec.lattice, spec.sites)
    sched, ty, tz, ms = lat.autotune(m, 5, 0, 20)
    assert ms > 0
    assert lat.schedule()[0] == sched
    p, _ = lat.get_native()
    assert np.array_equal(p, spec.lattice)  # state restored
    lat.run(m, 5, 0, 30)
    out, _ = lat.get_native()
    ref, _, _ = oracle_run(t, spec.lattice, spec.sites, 5, 0, 30)
    assert np.array_equal(out, ref)
    lat.close()
    m.close()


@pytest.mark.parametrize("slots,bps,schedule", [(16, 4, "phases"), (8, 1, "fused"), (8, 1, "phases")])
def test_run_native_async_pipelined(ctx, slots, bps, schedule):
    """lmb_run_native_async on two lattices of two contexts, their solves
    pipelined (the next solve of one queued while the other runs), each from
    new contents and with its own seed: every result equals
    lmb_lattice_set_native + lmb_run + lmb_lattice_get_native of the same
    solve, and the first one the oracle's."""
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import Context, Lattice, Model
    spec = configs.random_problem(71, X=64, Y=16, Z=24, slots=slots, bytes_per_slot=bps, density=0.05 * slots,
                                  nst=3)  # ~20 K overflows resolved over the 70 timesteps, none exhausted
    t = oracle_tables(spec)
    sched = L.LMB_SCHEDULE_PHASES if schedule == "phases" else L.LMB_SCHEDULE_FUSED
    ctx2 = Context(0)
    models = [Model.from_tables(ctx, t), Model.from_tables(ctx2, t)]
    lats = [Lattice(ctx, t.X, t.Y, t.Z, t.slots, t.bytes_per_slot),
            Lattice(ctx2, t.X, t.Y, t.Z, t.slots, t.bytes_per_slot)]
    for lat in lats:
        lat.set_schedule(sched)
    rng = np.random.default_rng(5)
    inputs = []
    for k in range(5):
        lat_k = spec.lattice.copy()
        if k:  # other contents: the same particles, shuffled over the sites
            N = spec.nsites
            perm = rng.permutation(N)
            lat_k = lat_k.reshape(-1, N)[:, perm].reshape(-1).copy()
        inputs.append(np.ascontiguousarray(lat_k, dtype=np.uint32))
    sites = np.ascontiguousarray(spec.sites, dtype=np.uint8)
    outs = [np.zeros_like(x) for x in inputs]
    T = 70  # two captured graphs of 32 timesteps and six single launches
    for k in range(5):
        lat = lats[k % 2]
        if k >= 2:
            lat.wait()
        lat.run_native_async(models[k % 2], 100 + k, 3, T, inputs[k].ctypes.data, sites.ctypes.data,
                             outs[k].ctypes.data)
    for lat in lats:
        lat.wait()
    ref, rc_ref, _ = oracle_run(t, inputs[0], sites, 100, 3, T)
    assert rc_ref == 0
    assert np.array_equal(outs[0], ref)
    solo = Lattice(ctx, t.X, t.Y, t.Z, t.slots, t.bytes_per_slot)
    solo.set_schedule(sched)
    for k in range(1, 5):
        solo.set_native(inputs[k], sites)
        solo.run(models[0], 100 + k, 3, T)
        got, _ = solo.get_native()
        assert np.array_equal(outs[k], got), k
    for obj in [solo] + lats + models:
        obj.close()
    ctx2.close()


@pytest.mark.parametrize("shape,slots,bps,per_slot,nsteps", [
    ((32, 32, 32), 8, 1, 0.01, 40),    # the plain bimolecular size: 16 CTAs of two planes
    ((16, 16, 16), 4, 1, 0.2, 40),     # one plane per CTA: both z neighbours remote
    ((24, 20, 48), 16, 1, 0.05, 30),   # odd plane sizes, three planes per CTA
    ((32, 16, 32), 4, 4, 0.15, 30),    # IntLattice
    ((32, 8, 16), 8, 1, 0.5, 20),      # dense: overflows resolved in global memory most timesteps
    ((32, 8, 12), 8, 1, 0.9, 10),      # denser still: four CTAs, the run may fail as the oracle's does
])
def test_cluster_schedule_vs_oracle(ctx, shape, slots, bps, per_slot, nsteps):
    """The cluster-resident schedule (the whole lattice in one thread-block
    cluster, every timestep of the run in one launch) against the oracle: the
    same status, statistics and lattice, including timesteps whose overflows
    go through global memory and runs that stop at a failed resolution."""
    X, Y, Z = shape
    spec = configs.random_problem(81, X=X, Y=Y, Z=Z, slots=slots, bytes_per_slot=bps, density=per_slot * slots,
                                  nst=3)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 31, 5, nsteps)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 31, 5, nsteps, schedule="cluster",
                           chunks=[nsteps // 2, nsteps - nsteps // 2])
    assert rc == rc_ref
    if rc == 0:
        assert sum(x.overflows for x in st) == st_ref.overflows
        assert sum(x.reactions for x in st) == st_ref.reactions
    assert np.array_equal(out, ref)


def test_cluster_schedule_bimolecular_vs_oracle(ctx):
    """The plain 32^3 bimolecular model on the cluster-resident schedule,
    300 timesteps in three runs, against the oracle."""
    spec = configs.config0(seed=3)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 77, 0, 300)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 77, 0, 300, schedule="cluster", chunks=[100, 100, 100])
    assert rc == rc_ref == 0
    assert sum(x.reactions for x in st) == st_ref.reactions > 0
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("shape,slots,bps,per_slot,nsteps,tile", [
    ((32, 32, 32), 8, 1, 0.01, 40, (0, 0)),    # the default plan: the most tiles that fit at once
    ((16, 16, 16), 4, 1, 0.2, 40, (1, 1)),     # 256 tiles of one row
    ((24, 20, 48), 16, 1, 0.05, 30, (4, 2)),   # rows not 16-byte aligned
    ((32, 16, 32), 4, 4, 0.15, 30, (2, 4)),    # IntLattice
    ((32, 8, 16), 8, 1, 0.5, 20, (2, 2)),      # dense: overflows resolved in global memory most timesteps
    ((32, 8, 12), 8, 1, 0.9, 10, (4, 2)),      # denser still: the run may fail as the oracle's does
    ((64, 64, 128), 8, 1, 0.01, 12, (4, 8)),   # 256 tiles, two per SM
])
def test_grid_schedule_vs_oracle(ctx, shape, slots, bps, per_slot, nsteps, tile):
    """The grid-resident schedule (every tile of a fused plan held in shared
    memory by one cooperative launch, halo rows exchanged through global
    memory, every timestep of the run in one launch) against the oracle: the
    same status, statistics and lattice, including overflow resolutions and
    runs that stop at a failed resolution."""
    X, Y, Z = shape
    spec = configs.random_problem(83, X=X, Y=Y, Z=Z, slots=slots, bytes_per_slot=bps, density=per_slot * slots,
                                  nst=3)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 37, 5, nsteps)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 37, 5, nsteps, schedule="grid", tile=tile,
                           chunks=[nsteps // 2, nsteps - nsteps // 2])
    assert rc == rc_ref
    if rc == 0:
        assert sum(x.overflows for x in st) == st_ref.overflows
        assert sum(x.reactions for x in st) == st_ref.reactions
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("tile", [(4, 8), (8, 4), (2, 16)])
def test_grid_schedule_rodcell_vs_oracle(ctx, tile):
    """The 64x64x128 rod cell (membrane, cytoplasm and nucleoid site types,
    membrane-only reactions) on the grid-resident schedule, 24 timesteps in
    two runs, against the oracle."""
    spec = configs.config1(seed=2)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 31, 0, 24)
    out, rc, st = _gpu_run(ctx, spec, spec.lattice, spec.sites, 31, 0, 24, from_spec=True, schedule="grid",
                           tile=tile, chunks=[11, 13])
    assert rc == rc_ref == 0
    assert sum(x.reactions for x in st) == st_ref.reactions
    assert np.array_equal(out, ref)


def test_grid_schedule_refuses_what_does_not_fit(ctx):
    """A lattice none of whose tile plans fit on the device at once is
    refused with LMB_E_UNSUPPORTED, and the lattice keeps its schedule."""
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import Lattice
    lat = Lattice(ctx, 256, 256, 64, 16, 4)
    before = lat.schedule()
    with pytest.raises(L.LmbError) as err:
        lat.set_schedule(L.LMB_SCHEDULE_GRID)
    assert err.value.status == L.LMB_E_UNSUPPORTED
    with pytest.raises(L.LmbError) as err:
        lat.set_schedule(L.LMB_SCHEDULE_GRID, 1, 1)
    assert err.value.status == L.LMB_E_UNSUPPORTED
    assert lat.schedule() == before
    lat.close()


@pytest.mark.parametrize("schedule", ["phases", "fused", "cluster", "grid"])
def test_run_native_async_refuses_bad_contents(ctx, schedule):
    """New contents given to lmb_run_native_async are checked on the device
    ahead of the timesteps: a species id above the model's fails the solve
    with LMB_E_ARG before its first timestep and leaves the uploaded lattice
    as it is, as lmb_lattice_set_native + lmb_run does; the next solve with
    good contents runs as usual."""
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import Lattice, Model
    spec = configs.random_problem(91, X=32, Y=16, Z=16, slots=8, bytes_per_slot=1, density=0.1, nst=3)
    t = oracle_tables(spec)
    sched = {"phases": L.LMB_SCHEDULE_PHASES, "fused": L.LMB_SCHEDULE_FUSED, "cluster": L.LMB_SCHEDULE_CLUSTER,
             "grid": L.LMB_SCHEDULE_GRID}
    model = Model.from_tables(ctx, t)
    lat = Lattice(ctx, t.X, t.Y, t.Z, t.slots, t.bytes_per_slot)
    lat.set_schedule(sched[schedule])
    good = np.ascontiguousarray(spec.lattice, dtype=np.uint32)
    sites = np.ascontiguousarray(spec.sites, dtype=np.uint8)
    bad = good.copy()
    bad[7] = (bad[7] & ~np.uint32(0xFF)) | np.uint32(spec.ns + 5)  # slot 0 of site 7: no such species
    out = np.zeros_like(good)
    lat.run_native_async(model, 9, 0, 70, bad.ctypes.data, sites.ctypes.data, out.ctypes.data)
    rc, st = lat.wait(check=False)
    assert rc == L.LMB_E_ARG and st.steps_done == 0
    now, _ = lat.get_native()
    assert np.array_equal(now, bad)
    lat.run_native_async(model, 9, 0, 70, good.ctypes.data, sites.ctypes.data, out.ctypes.data)
    rc, _ = lat.wait(check=False)
    assert rc == 0
    ref, rc_ref, _ = oracle_run(t, good, sites, 9, 0, 70)
    assert rc_ref == 0
    assert np.array_equal(out, ref)
    lat.close()
    model.close()


def test_chunked_run_equals_single_run(ctx):
    spec = configs.random_problem(8, X=32, Y=16, Z=8, density=0.7)
    t = oracle_tables(spec)
    a, rc1, _ = _gpu_run(ctx, t, spec.lattice, spec.sites, 3, 0, 20)
    b, rc2, _ = _gpu_run(ctx, t, spec.lattice, spec.sites, 3, 0, 20, chunks=[1, 7, 5, 7])
    assert rc1 == rc2 == 0
    assert np.array_equal(a, b)


def test_model_from_spec_equals_oracle(ctx):
    spec = configs.config0(seed=4)
    t = oracle_tables(spec)
    ref, _, _ = oracle_run(t, spec.lattice, spec.sites, 55, 0, 100)
    out, rc, _ = _gpu_run(ctx, spec, spec.lattice, spec.sites, 55, 0, 100, from_spec=True)
    assert rc == 0
    assert np.array_equal(out, ref)


def test_config1_short_vs_oracle(ctx):
    spec = configs.config1(seed=2)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 31, 0, 6)
    out, rc, st = _gpu_run(ctx, spec, spec.lattice, spec.sites, 31, 0, 6, from_spec=True)
    assert rc == rc_ref == 0
    assert np.array_equal(out, ref)


def test_set_reaction_rate(ctx):
    from lattice_microbes_b200.solver import Model
    spec = configs.config0(seed=5)
    m = Model.from_spec(ctx, spec)
    spec.K = spec.K.copy()
    spec.K[1] *= 50.0
    m.set_reaction_rate(1, float(spec.K[1]))
    ref = oracle_tables(spec)
    got = m.tables()
    assert np.array_equal(got["rate"], ref.rate)
    assert np.array_equal(got["qp1"], ref.qp1)
    m.close()


def test_species_counts_and_layouts(ctx):
    from lattice_microbes_b200.solver import Lattice
    spec = configs.random_problem(6, X=24, Y=16, Z=8, slots=16, bytes_per_slot=4, density=2.0, ns=9)
    t = oracle_tables(spec)
    lat = Lattice(ctx, spec.X, spec.Y, spec.Z, 16, 4)
    lat.set_native(spec.lattice, spec.sites)
    counts = lat.species_counts(spec.ns)
    assert np.array_equal(counts, oracle_counts(t, spec.lattice))
    rm, rs = lat.get_row_major()
    slots = configs.native_to_slots(spec.lattice, spec.X, spec.Y, spec.Z, 16, 4)
    expect = slots.reshape(spec.Z, spec.Y, spec.X, 16).transpose(2, 1, 0, 3)
    assert np.array_equal(rm, expect)
    assert np.array_equal(rs, spec.sites.reshape(spec.Z, spec.Y, spec.X).transpose(2, 1, 0))
    # Row-major with holes packs each site (RDMESolver.cpp:144-167).
    holes = rm.copy()
    holes[..., 0] = 0
    lat.set_row_major(holes, rs, spec.ns, spec.nst)
    back, _ = lat.get_row_major()
    for site in [(0, 0, 0), (5, 3, 2), (23, 15, 7)]:
        v = holes[site]
        nz = v[v != 0]
        assert np.array_equal(back[site][: len(nz)], nz)
        assert not back[site][len(nz):].any()
    lat.close()


def test_pure_diffusion_conserves_counts_large(ctx):
    """Size-independent property at a larger lattice: no reactions, counts
    are conserved exactly over many steps."""
    from lattice_microbes_b200.solver import Lattice, Model
    spec = configs.config1(seed=3, X=64, Y=64, Z=128)
    spec.rtype = spec.rtype[:0]
    spec.K = spec.K[:0]
    spec.S = spec.S[:, :0]
    spec.D = spec.D[:, :0]
    spec.RL = spec.RL[:0]
    m = Model.from_spec(ctx, spec)
    lat = Lattice(ctx, spec.X, spec.Y, spec.Z, 8, 1)
    lat.set_native(spec.lattice, spec.sites)
    before = lat.species_counts(spec.ns)
    rc, st = lat.run(m, 9, 0, 300)
    assert rc == 0
    assert np.array_equal(before, lat.species_counts(spec.ns))
    lat.close()
    m.close()


def test_invalid_species_rejected(ctx):
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import Lattice, Model
    spec = configs.config0(seed=1, edge=16)
    m = Model.from_spec(ctx, spec)
    lat = Lattice(ctx, 16, 16, 16, 8, 1)
    bad = spec.lattice.copy()
    bad[0] = 9  # species 9 > 3
    lat.set_native(bad, spec.sites)
    rc, _ = lat.run(m, 1, 0, 1, check=False)
    assert rc == L.LMB_E_ARG
    lat.close()
    m.close()


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_graph_replay_long_run_vs_oracle(ctx, schedule):
    """Runs long enough to replay captured timestep graphs (and a remainder
    launched directly), in two calls that start at different buffer parities."""
    spec = configs.config0(seed=3, nA=40000, nB=40000)  # dense: thousands of overflows
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 31337, 0, 141)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 31337, 0, 141, chunks=[73, 68], schedule=schedule)
    assert rc == rc_ref == 0
    assert sum(s.overflows for s in st) == st_ref.overflows
    assert sum(s.reactions for s in st) == st_ref.reactions
    assert np.array_equal(out, ref)


def _busy_problem(seed, promiscuous, ns=60, nr=150):
    """Many species and reactions on a small Int-16 lattice, with fast
    reactions so that sites react every few timesteps: exercises the
    candidate-reaction scan (and, when `promiscuous`, sites with more
    candidate reactions than a short list holds: one species is the first
    reactant of 80 reactions) and the propensity bound of the reaction step."""
    spec = configs.config2(seed=seed, X=32, Y=16, Z=16, ns=ns, nr=nr, nparticles=12000, nst=4,
                           obstacle_fraction=0.1)
    spec.tau = 2e-4  # larger rates per timestep
    if promiscuous:
        R = spec.nr
        for j in range(80):
            spec.S[:, j] = 0
            spec.D[:, j] = 0
            spec.rtype[j] = configs.FIRST
            spec.K[j] = 50.0
            spec.S[0, j] = -1
            spec.D[0, j] = 1
            spec.S[1 + j % (spec.ns - 1), j] += 1
        assert R == spec.nr
    # D limited so that q stays <= 0.5 at the longer timestep.
    spec.DF = np.minimum(spec.DF, 0.45 * spec.spacing ** 2 / spec.tau)
    return spec


@pytest.mark.parametrize("schedule", SCHEDULES)
@pytest.mark.parametrize("promiscuous", [False, True])
def test_many_reactions_vs_oracle(ctx, schedule, promiscuous):
    spec = _busy_problem(21, promiscuous)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 4242, 0, 12)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 4242, 0, 12, schedule=schedule)
    assert rc == rc_ref == 0
    assert st_ref.reactions > 50  # the reaction step really fires
    assert st[0].reactions == st_ref.reactions
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_reactions_past_the_candidate_bitmap_vs_oracle(ctx, schedule):
    """4200 reactions, more than the per-phase reaction step's candidate
    bitmap covers (4096): its candidates go through the 64-entry list, and
    the full scan of every reaction when a site has more."""
    spec = _busy_problem(21, True, ns=120, nr=4200)
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 4242, 0, 12)
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 4242, 0, 12, schedule=schedule)
    assert rc == rc_ref == 0
    assert st_ref.reactions > 50
    assert st[0].reactions == st_ref.reactions
    assert np.array_equal(out, ref)


def _with_holes(spec, seed=3):
    """The same particles with holes: in a third of the occupied sites the
    first particle moves to the last slot (an empty slot now precedes
    occupied ones).  The reference processes every nonzero slot, holes or
    not (byte_diffusion_1d_dev.cu:100-118), and keys each draw by its slot."""
    rng = np.random.default_rng(seed)
    X, Y, Z, S, b = spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot
    slots = configs.native_to_slots(spec.lattice, X, Y, Z, S, b).copy()
    occ = (slots != 0).sum(axis=1)
    pick = np.nonzero((occ >= 1) & (occ < S) & (rng.random(len(occ)) < 0.33))[0]
    slots[pick, S - 1] = slots[pick, 0]
    slots[pick, 0] = 0
    N = spec.nsites
    lat = configs.empty_lattice(X, Y, Z, S, b)
    for k in range(S):
        v = slots[:, k].astype(np.uint32)
        if b == 1:
            lat[(k // 4) * N:(k // 4 + 1) * N] |= v << np.uint32(8 * (k % 4))
        else:
            lat[k * N:(k + 1) * N] = v
    spec.lattice = lat
    return spec


@pytest.mark.parametrize("schedule", SCHEDULES)
@pytest.mark.parametrize("slots,bps", [(8, 1), (16, 1), (16, 4)])
def test_lattice_with_holes_vs_oracle(ctx, schedule, slots, bps):
    spec = _with_holes(configs.random_problem(31, X=32, Y=8, Z=8, slots=slots, bytes_per_slot=bps, density=1.2,
                                              nst=2))
    t = oracle_tables(spec)
    ref, rc_ref, st_ref = oracle_run(t, spec.lattice, spec.sites, 777, 0, 9)
    # In pieces: the holes flag must survive a one-timestep run.
    out, rc, st = _gpu_run(ctx, t, spec.lattice, spec.sites, 777, 0, 9, schedule=schedule, chunks=[1, 1, 7])
    assert rc == rc_ref == 0
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("slots,bps", [(8, 1), (16, 1), (16, 4), (8, 4)])
def test_plane_bounds_across_runs_and_edits(ctx, slots, bps):
    """Per-phase schedule on lattices whose rows are multiples of 32 sites
    (the sweeps keep per-segment plane bounds): a sparse lattice run in
    chunks, edited between chunks so that some segments fill every slot (far
    above the bounds the previous run ended with), then run again; a second
    lattice starts empty and fills through zeroth-order reactions.  Every
    chunk equals the oracle."""
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import Lattice, Model
    spec = configs.random_problem(41, X=64, Y=8, Z=16, slots=slots, bytes_per_slot=bps, density=0.05, nst=2)
    t = oracle_tables(spec)
    model = Model.from_tables(ctx, t)
    lat = Lattice(ctx, t.X, t.Y, t.Z, t.slots, t.bytes_per_slot)
    lat.set_schedule(L.LMB_SCHEDULE_PHASES)
    lat.set_native(spec.lattice, spec.sites)
    ref = spec.lattice.copy()
    rng = np.random.default_rng(7)
    step = 0
    N = spec.nsites
    words = spec.words
    for chunk in (3, 9, 4, 40):
        rc, _ = lat.run(model, 99, step, chunk, check=False)
        assert rc == 0
        ref, rc_ref, _ = oracle_run(t, ref, spec.sites, 99, step, chunk)
        assert rc_ref == 0
        out, _ = lat.get_native()
        assert np.array_equal(out, ref), "chunk at step %d" % step
        step += chunk
        # Fill every slot of a few sites (one full site per edited segment
        # is enough to lift the segment's bound to every plane).
        edited = ref.copy()
        for i in rng.choice(N, size=6, replace=False):
            if bps == 1:
                for w in range(words):
                    edited[w * N + i] = 0x01010101
            else:
                for w in range(words):
                    edited[w * N + i] = 1 + (w % spec.ns)
        lat.set_native(edited, None)
        ref = edited
    lat.close()
    model.close()

    empty = configs.empty_lattice(t.X, t.Y, t.Z, slots, bps)
    out, rc, _ = _gpu_run(ctx, t, empty, spec.sites, 5, 0, 30, schedule="phases")
    ref, rc_ref, _ = oracle_run(t, empty, spec.sites, 5, 0, 30)
    assert rc == rc_ref == 0
    assert out.any()
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("schedule", SCHEDULES + ["cluster", "grid"])
@pytest.mark.parametrize("case", ["sparse", "storm", "relaxed", "zero_steps"])
def test_run_counts_equal_separate_counts(ctx, schedule, case):
    """lmb_run_counts_async takes the species totals inside the run (the fused
    kernel's last launch and its overflow resolution, or one bounded pass
    after a per-phase run): they equal lmb_lattice_species_counts of the final
    lattice and the oracle's, overflow storms and the relaxed handler's
    unresolved particles (left out of the lattice) included."""
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import Lattice, Model
    if case == "sparse":
        spec = configs.random_problem(51, X=64, Y=16, Z=16, slots=8, bytes_per_slot=1, density=0.3, nst=3)
    else:
        spec = configs.random_problem(52, X=32, Y=8, Z=8, slots=8, bytes_per_slot=1, density=5.0, nst=2)
    mode = L.LMB_OVERFLOW_RELAXED if case == "relaxed" else L.LMB_OVERFLOW_CLASSIC
    n = 0 if case == "zero_steps" else 9
    t = oracle_tables(spec)
    model = Model.from_tables(ctx, t)
    lat = Lattice(ctx, t.X, t.Y, t.Z, t.slots, t.bytes_per_slot)
    if schedule == "phases":
        lat.set_schedule(L.LMB_SCHEDULE_PHASES)
    elif schedule == "cluster":
        lat.set_schedule(L.LMB_SCHEDULE_CLUSTER)
    elif schedule == "grid":
        lat.set_schedule(L.LMB_SCHEDULE_GRID)
    else:
        lat.set_schedule(L.LMB_SCHEDULE_FUSED)
    lat.set_native(spec.lattice, spec.sites)
    if schedule in ("cluster", "grid") and mode == L.LMB_OVERFLOW_RELAXED:
        # The shared-memory-resident schedules resolve overflows the classic way only.
        with pytest.raises(L.LmbError) as err:
            lat.run_counts(model, 17, 0, n, spec.ns, mode, check=False)
        assert err.value.status == L.LMB_E_UNSUPPORTED
        lat.close()
        model.close()
        return
    rc, st, counts = lat.run_counts(model, 17, 0, n, spec.ns, mode, check=False)
    ref, rc_ref, _ = oracle_run(t, spec.lattice, spec.sites, 17, 0, n, mode)
    assert rc == rc_ref
    if rc == 0:
        out, _ = lat.get_native()
        assert np.array_equal(out, ref)
        assert np.array_equal(counts, lat.species_counts(spec.ns))
        assert np.array_equal(counts, oracle_counts(t, ref))
    lat.close()
    model.close()
