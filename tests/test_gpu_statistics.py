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


def rod_ensemble(reps, entries, ns, tau_div, seed_top):
    """`reps` rod-cell replicates in one batch at timestep tau / tau_div,
    species counts every 5 ms: [reps, entries, ns]."""
    from lattice_microbes_b200.solver import Batch, Context, Lattice, Model, compose_seed
    ctx = Context(0)
    lats, models = [], []
    for k in range(reps):
        spec = configs.config1(seed=k + 1)
        spec.tau = spec.tau / tau_div
        m = Model.from_spec(ctx, spec)
        lat = Lattice(ctx, spec.X, spec.Y, spec.Z, 8, 1)
        lat.set_native(spec.lattice, spec.sites)
        lats.append(lat)
        models.append(m)
    batch = Batch(ctx, lats, models)
    every = 200 * tau_div  # 5 ms
    seeds = [compose_seed(seed_top, k + 1) for k in range(reps)]
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
    return out


def test_rodcell_ensemble_vs_reference_nsm(gpu):
    """The rod-cell model (membrane-only binding, three site types, per-type
    diffusion) against 256 reference NextSubvolumeSolver replicates from the
    same initial lattices (tests/golden/ensembles/nsm_rodcell.npz), species
    counts every 5 ms to t = 50 ms.

    MPD splits each timestep into x, y and z hops and then at most one
    reaction per site, so it carries an O(tau) bias against the exact NSM.
    At this model's tau = 25 us (cytoplasm hop probability 0.244 per sweep)
    the bias becomes resolvable with 256 replicates after about 15 ms: at
    50 ms D_ATP is 2.9 % low and membrane D 2.8 % high.  The reference's own
    MPD kernels give the same distributions (the kernels here replay them bit
    for bit).  So the ensemble is checked for what MPD promises:
      * D and E are conserved exactly;
      * at the first record (5 ms), every varying species passes KS, means
        within z standard errors and Brown-Forsythe variances at a
        family-wise 5 % level (Bonferroni);
      * the bias shrinks with the timestep: at tau / 4 the squared
        standardized mean differences of the species that vary, summed over
        the records from 25 ms on, are below 0.6 of those at tau (a first-
        order bias would give 0.06 plus noise);
      * at tau / 4 the variances pass Brown-Forsythe at the family-wise
        level, and every mean of at least 100 particles lies within 6 % (or
        4 standard errors) of NSM's: a bound on what remains of the bias
        (measured at most 4 %, on DE at 20 ms), which a wrong rate or
        transition probability would exceed."""
    z = np.load(os.path.join(ENS, "nsm_rodcell.npz"))
    times, ref = z["times"], z["counts"].astype(np.int64)
    reps, entries, ns = ref.shape
    out = rod_ensemble(reps, entries, ns, 1, 99)
    fine = rod_ensemble(reps, entries, ns, 4, 103)
    for o in (out, fine):
        assert np.array_equal(o[:, 0, :], ref[:, 0, :])  # same initial lattices
        assert np.all(o[:, :, [0, 1, 3, 4]].sum(axis=2) == o[:, :1, [0, 1, 3, 4]].sum(axis=2))
        assert np.all(o[:, :, [2, 3]].sum(axis=2) == o[:, :1, [2, 3]].sum(axis=2))
    early = [(1, s) for s in range(ns) if ref[:, 1, s].var() > 0]
    zc = stats.norm.ppf(1 - 0.025 / len(early))
    for e, s in early:
        compare(out[:, e, s], ref[:, e, s], 0.01 / len(early), zc, ("rod cell", e, s))

    def zsq(o, e, s):
        a, b = o[:, e, s].astype(np.float64), ref[:, e, s].astype(np.float64)
        se = np.sqrt(a.var() / a.size + b.var() / b.size)
        return ((a.mean() - b.mean()) / se) ** 2

    late = [(e, s) for e in range(5, entries) for s in range(ns) if ref[:, e, s].mean() >= 100]
    coarse = sum(zsq(out, e, s) for e, s in late)
    refined = sum(zsq(fine, e, s) for e, s in late)
    assert refined < 0.6 * coarse, (refined, coarse)
    varying = [(e, s) for e in range(1, entries) for s in range(ns) if ref[:, e, s].var() > 0]
    p_min = 0.01 / len(varying)
    for e, s in varying:
        a, b = fine[:, e, s].astype(np.float64), ref[:, e, s].astype(np.float64)
        bf = stats.levene(a, b, center="median")
        assert bf.pvalue > p_min, (e, s, "variance", a.var(), b.var(), bf)
    for e, s in varying:
        a, b = fine[:, e, s].astype(np.float64), ref[:, e, s].astype(np.float64)
        if b.mean() >= 100:
            se = np.sqrt(a.var() / a.size + b.var() / b.size)
            assert abs(a.mean() - b.mean()) <= max(0.06 * b.mean(), 4 * se), (e, s, a.mean(), b.mean())
