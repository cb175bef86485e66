"""CME ensembles on the GPU (lmb_cme) against the reference GillespieDSolver.

The GPU ensemble uses FP32 propensities and its own counter-hash random
numbers, so it is compared with the reference statistically, against 8192
reference replicates (tests/golden/ensembles/gillespie_two_state.npz):
  * the model's output, the protein count at the last record (t = 3600 s):
    two-sample KS p > 0.01 and the difference of the means within 2
    standard errors;
  * every species at every record: the same two checks at a family-wise
    level of 5 % over all m comparisons (Bonferroni: KS p > 0.01 / m, means
    within z(1 - 0.025 / m) standard errors), since 2 sigma on each of m
    comparisons fails by chance about m / 20 times.
Determinism checks are exact: the same replicate gives the same trajectory
whatever the ensemble size and however the run is cut into segments.
"""
import os

import numpy as np
import pytest
from scipy import stats

from lattice_microbes_b200 import configs

pytestmark = pytest.mark.gpu

ENS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ensembles")


def golden():
    z = np.load(os.path.join(ENS, "gillespie_two_state.npz"))
    return z["times"], z["counts"]


def compare(a, b, p_min, z, what):
    """Two-sample KS, means within z standard errors, and equal variances
    (Brown-Forsythe: Levene's test about the medians), each at p_min."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    ks = stats.ks_2samp(a, b)
    assert ks.pvalue > p_min, (what, ks)
    se = np.sqrt(a.var() / a.size + b.var() / b.size)
    assert abs(a.mean() - b.mean()) <= z * se + 1e-12, (what, a.mean(), b.mean(), se)
    if a.var() > 0 or b.var() > 0:
        bf = stats.levene(a, b, center="median")
        assert bf.pvalue > p_min, (what, "variance", a.var(), b.var(), bf)


def run_ensemble(ctx, reps, seed=5, segments=1, spec=None):
    from lattice_microbes_b200.solver import CMEEnsemble
    m = spec or configs.two_state_gene()
    e = CMEEnsemble(ctx, m, reps)
    if segments == 1:
        e.run(seed, m.max_time, m.write_interval)
    else:
        e.begin(seed, m.max_time, m.write_interval)
        for k in range(1, segments + 1):
            e.advance_async(m.max_time * k / segments)
    out = e.counts()
    ev, fin = e.stats()
    e.close()
    return out, ev, fin


@pytest.fixture(scope="module")
def ctx(gpu):
    from lattice_microbes_b200.solver import Context
    c = Context(0)
    yield c
    c.close()


def test_two_state_ensemble_matches_reference_gillespie(ctx):
    times, ref = golden()
    out, ev, fin = run_ensemble(ctx, 65536)
    assert fin == 65536
    assert out.shape == (65536, len(times), 4)
    assert np.all(out[:, :, 0] + out[:, :, 1] == 1)  # one gene copy, always
    assert np.array_equal(out[:, 0, :], np.tile([1, 0, 0, 0], (65536, 1)))
    compare(out[:, -1, 3], ref[:, -1, 3], 0.01, 2.0, "protein at t_end")
    # The reference's own regression bar for expression models
    # (testing/regression/testsuites/CMEBase/testCME.py:117-178): mean and
    # variance of the output within 10 %.
    a, b = out[:, -1, 3].astype(np.float64), ref[:, -1, 3].astype(np.float64)
    assert abs(a.mean() / b.mean() - 1) < 0.10 and abs(a.var() / b.var() - 1) < 0.10, (a.mean(), b.mean(),
                                                                                        a.var(), b.var())
    pairs = [(e, s) for e in range(1, len(times)) for s in range(1, 4)]
    m = len(pairs)
    z = stats.norm.ppf(1 - 0.025 / m)
    for e, s in pairs:
        compare(out[:, e, s], ref[:, e, s], 0.01 / m, z, (e, s))
    # ~17 events per second per replicate at steady state.
    assert 10 * 3600 * 65536 < ev < 25 * 3600 * 65536


def test_segments_and_ensemble_size_do_not_change_trajectories(ctx):
    one, ev1, _ = run_ensemble(ctx, 4096, seed=11)
    cut, ev7, _ = run_ensemble(ctx, 4096, seed=11, segments=7)
    assert np.array_equal(one, cut)
    assert ev1 == ev7
    small, _, _ = run_ensemble(ctx, 100, seed=11)
    assert np.array_equal(small, one[:100])


def test_second_order_and_zeroth_order_reactions(ctx):
    """Dimerisation 2A <-> B with a source of A: k_self, k_back, k_in.  The
    reference GillespieD run from its sources is the comparator."""
    from tests import ref_cpu_lib
    if not ref_cpu_lib.available():
        pytest.skip("reference CPU solvers not built")
    S = np.array([[-2, 2, 1, -1], [1, -1, 0, 0]], dtype=np.int32)
    D = np.array([[1, 0, 0, 1], [0, 1, 0, 0]], dtype=np.uint32)
    rtype = np.array([3, 1, 0, 1], dtype=np.uint32)
    K = np.array([0.02, 0.5, 5.0, 0.1])
    spec = configs.CMESpec("dimer", 2, rtype, K, S, D, np.array([10, 0], np.uint32), 50.0, 10.0)
    out, _, fin = run_ensemble(ctx, 8192, seed=3, spec=spec)
    assert fin == 8192
    ref = np.stack([ref_cpu_lib.gillespie_run(2, rtype, K, S, D, spec.init, 9, k + 1, 50.0, 10.0)[1]
                    for k in range(2000)])
    compare(out[:, -1, 1], ref[:, -1, 1], 0.01, 2.0, "dimer at t_end")
    pairs = [(e, s) for e in range(1, ref.shape[1]) for s in range(2)]
    z = stats.norm.ppf(1 - 0.025 / len(pairs))
    for e, s in pairs:
        compare(out[:, e, s], ref[:, e, s], 0.01 / len(pairs), z, (e, s))


def _ensemble_with_kernel(ctx, spec, reps, seed, kernel, segments=1):
    from lattice_microbes_b200 import _lib as L
    from lattice_microbes_b200.solver import CMEEnsemble
    ens = CMEEnsemble(ctx, spec, reps)
    ens.set_kernel(kernel)
    ens.begin(seed, spec.max_time, spec.write_interval)
    for k in range(1, segments + 1):
        ens.advance_async(spec.max_time * k / segments)
    out = ens.counts()
    ev, fin = ens.stats()
    ens.close()
    return out, ev, fin


@pytest.mark.parametrize("model", ["two_state_gene", "dimer", "wide"])
def test_compact_kernel_equals_generic(ctx, model):
    """The register-resident kernel for small models against the generic one:
    the same trajectories, event counts and records, also when the run is cut
    into segments.  'wide' has a stoichiometric change of 9, outside the
    compact form, so both settings run the generic kernel."""
    from lattice_microbes_b200 import _lib as L
    if model == "two_state_gene":
        spec = configs.two_state_gene(max_time=600.0, write_interval=120.0)
    else:
        d = 9 if model == "wide" else 2
        S = np.array([[-d, d, 1, -1], [1, -1, 0, 0]], dtype=np.int32)
        D = np.array([[1, 0, 0, 1], [0, 1, 0, 0]], dtype=np.uint32)
        spec = configs.CMESpec(model, 2, np.array([3, 1, 0, 1], np.uint32), np.array([0.02, 0.5, 5.0, 0.1]), S, D,
                               np.array([20, 0], np.uint32), 50.0, 10.0)
    gen, ev_g, fin_g = _ensemble_with_kernel(ctx, spec, 3000, 21, L.LMB_CME_KERNEL_GENERIC)
    auto, ev_a, fin_a = _ensemble_with_kernel(ctx, spec, 3000, 21, L.LMB_CME_KERNEL_AUTO, segments=3)
    assert fin_g == fin_a == 3000
    assert ev_g == ev_a and ev_g > 3000
    assert np.array_equal(gen, auto)
