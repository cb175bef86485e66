"""MPD-RDME ensembles on the GPU against the reference's exact RDME solver.

Independent-seed MPD ensembles of the bimolecular model A + B <-> C
(configs.config0: D = 1e-12 m^2/s, kf = 1.07e6 /M/s, kr = 0.351 /s,
tau = 50 us) are compared with NextSubvolumeSolver ensembles made by the
reference's own code from the same initial lattices
(tests/golden/ensembles/nsm_bimolecular_<edge>.npz), on the C count:
  * at the last record (t = 0.5 s, 10,000 timesteps): two-sample KS
    p > 0.01 and the mean difference within 2 standard errors;
  * at all ten 0.05 s records: the same checks at a family-wise level of 5 %
    (Bonferroni over the ten records: KS p > 0.001, means within
    z(1 - 0.0025) = 2.81 standard errors).  The batch
runs every replicate in one launch per timestep; each replicate is also the
plain solver's result (tests/test_gpu_batch.py).
"""
import os

import numpy as np
import pytest
from scipy import stats

from lattice_microbes_b200 import configs

pytestmark = pytest.mark.gpu

ENS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ensembles")
CHUNK = 1000  # timesteps between records: 0.05 s


def nsm(edge):
    z = np.load(os.path.join(ENS, "nsm_bimolecular_%d.npz" % edge))
    return z["times"], z["counts"]


def compare(a, b, p_min, z, what):
    """Two-sample KS, means within z standard errors, and equal variances
    (Brown-Forsythe: Levene's test about the medians), each at p_min."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    ks = stats.ks_2samp(a, b)
    assert ks.pvalue > p_min, (what, ks)
    se = np.sqrt(a.var() / a.size + b.var() / b.size)
    assert abs(a.mean() - b.mean()) <= z * se, (what, a.mean(), b.mean(), se)
    if a.var() > 0 or b.var() > 0:
        bf = stats.levene(a, b, center="median")
        assert bf.pvalue > p_min, (what, "variance", a.var(), b.var(), bf)


def mpd_ensemble(edge, reps, seed_top=2024):
    from lattice_microbes_b200.solver import Batch, Context, Lattice, Model, compose_seed
    ctx = Context(0)
    lats, models = [], []
    for k in range(reps):
        spec = configs.config0(seed=k + 1, edge=edge)
        m = Model.from_spec(ctx, spec)
        lat = Lattice(ctx, edge, edge, edge, 8, 1)
        lat.set_native(spec.lattice, spec.sites)
        lats.append(lat)
        models.append(m)
    batch = Batch(ctx, lats, models)
    seeds = [compose_seed(seed_top, k + 1) for k in range(reps)]
    rec = np.zeros((reps, 11, 3), dtype=np.int64)
    rec[:, 0, :] = [lat.species_counts(3)[1:] for lat in lats]
    for e in range(1, 11):
        rc, st = batch.run(seeds, (e - 1) * CHUNK, CHUNK)
        assert rc == 0 and all(s.status == 0 for s in st)
        rec[:, e, :] = [lat.species_counts(3)[1:] for lat in lats]
    batch.close()
    for lat, m in zip(lats, models):
        lat.close()
        m.close()
    ctx.close()
    return rec


@pytest.mark.parametrize("edge,reps", [(16, 512), (32, 384)])
def test_mpd_ensemble_matches_reference_nsm(gpu, edge, reps):
    times, ref = nsm(edge)
    out = mpd_ensemble(edge, reps)
    assert np.array_equal(out[:, 0, :], ref[:reps, 0, :].astype(np.int64))  # same initial lattices
    n0 = out[:, 0, 0]
    assert np.all(out[:, :, 0] + out[:, :, 2] == n0[:, None])  # A + C conserved
    compare(out[:, 10, 2], ref[:, 10, 2], 0.01, 2.0, (edge, "t_end"))
    z = stats.norm.ppf(1 - 0.025 / 10)
    for e in range(1, 11):
        compare(out[:, e, 2], ref[:, e, 2], 0.01 / 10, z, (edge, e))


def test_rodcell_ensemble_matches_reference_nsm(gpu):
    """The rod-cell model (membrane-only binding, three site types, per-type
    diffusion): 256 MPD replicates in one batch against 256 reference
    NextSubvolumeSolver replicates from the same initial lattices
    (tests/golden/ensembles/nsm_rodcell.npz), every species at every 5 ms
    record to t = 50 ms: KS, means and variances at a family-wise 5 % level
    (Bonferroni over the records and species that vary)."""
    from lattice_microbes_b200.solver import Batch, Context, Lattice, Model, compose_seed
    z = np.load(os.path.join(ENS, "nsm_rodcell.npz"))
    times, ref = z["times"], z["counts"].astype(np.int64)
    reps, entries, ns = ref.shape
    every = int(round((times[1] - times[0]) / 25e-6))
    ctx = Context(0)
    lats, models = [], []
    for k in range(reps):
        spec = configs.config1(seed=k + 1)
        m = Model.from_spec(ctx, spec)
        lat = Lattice(ctx, spec.X, spec.Y, spec.Z, 8, 1)
        lat.set_native(spec.lattice, spec.sites)
        lats.append(lat)
        models.append(m)
    batch = Batch(ctx, lats, models)
    seeds = [compose_seed(99, k + 1) for k in range(reps)]
    out = np.zeros((reps, entries, ns), dtype=np.int64)
    out[:, 0, :] = [lat.species_counts(ns)[1:] for lat in lats]
    for e in range(1, entries):
        rc, st = batch.run(seeds, (e - 1) * every, every)
        assert rc == 0 and all(s.status == 0 for s in st)
        out[:, e, :] = [lat.species_counts(ns)[1:] for lat in lats]
    batch.close()
    for lat, m in zip(lats, models):
        lat.close()
        m.close()
    ctx.close()
    assert np.array_equal(out[:, 0, :], ref[:, 0, :])  # same initial lattices
    # D (ATP, ADP, membrane, with E) and E (free and bound) are conserved.
    assert np.all(out[:, :, [0, 1, 3, 4]].sum(axis=2) == out[:, :1, [0, 1, 3, 4]].sum(axis=2))
    assert np.all(out[:, :, [2, 3]].sum(axis=2) == out[:, :1, [2, 3]].sum(axis=2))
    pairs = [(e, s) for e in range(1, entries) for s in range(ns) if ref[:, e, s].var() > 0]
    assert len(pairs) >= entries
    m = len(pairs)
    zc = stats.norm.ppf(1 - 0.025 / m)
    for e, s in pairs:
        compare(out[:, e, s], ref[:, e, s], 0.01 / m, zc, ("rod cell", e, s))
