"""The reference's CPU solvers built from its sources (NextSubvolumeSolver,
GillespieDSolver) and the statistical fixtures made from them.

These pin the comparators the GPU ensemble tests use: the fixtures replay
bit for bit from the reference code, the reference NSM conserves what the
model conserves, and the reference GillespieD ensemble matches the analytic
moments of the two-state gene model (the kind of check the reference's own
CME regression suite makes, testing/regression/testsuites/CMEBase/testCME.py).
"""
import os

import numpy as np
import pytest

from lattice_microbes_b200 import configs
from tests import ref_cpu_lib

ENS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ensembles")

needs_ref = pytest.mark.skipif(not ref_cpu_lib.available(), reason="reference CPU solvers not built")


def load(name):
    z = np.load(os.path.join(ENS, name + ".npz"))
    return {k: z[k] for k in z.files}


def test_fixtures_have_the_expected_shape():
    for edge in (16, 32):
        g = load("nsm_bimolecular_%d" % edge)
        assert g["counts"].shape == (512, 11, 3)
        assert np.allclose(g["times"], np.arange(11) * 0.05)
    g = load("gillespie_two_state")
    assert g["counts"].shape == (8192, 7, 4)
    assert np.allclose(g["times"], np.arange(7) * 600.0)


@needs_ref
@pytest.mark.parametrize("edge", [16, 32])
def test_nsm_fixture_replays_from_the_reference(edge):
    g = load("nsm_bimolecular_%d" % edge)
    for k in (0, 7):
        spec = configs.config0(seed=k + 1, edge=edge)
        t, c = ref_cpu_lib.nsm_run(spec, int(g["seed"]), k + 1, float(g["t_end"]), 0.05)
        assert np.array_equal(c, g["counts"][k])


@needs_ref
def test_nsm_conserves_and_keeps_the_lattice_consistent():
    spec = configs.config0(seed=3, edge=16)
    t, c, fin = ref_cpu_lib.nsm_run(spec, 99, 1, 0.2, 0.02, final_lattice=True)
    n0 = configs.species_counts(spec.lattice, spec.nsites, 8, 1, 3)[1:]
    assert np.all(c[:, 0] + c[:, 2] == n0[0])
    assert np.all(c[:, 1] + c[:, 2] == n0[1])
    # The final lattice holds exactly the final counts.
    counts = np.bincount(fin, minlength=4)[1:]
    assert np.array_equal(counts, c[-1])


@needs_ref
def test_gillespie_fixture_replays_from_the_reference():
    g = load("gillespie_two_state")
    m = configs.two_state_gene()
    for k in (0, 4000):
        t, c = ref_cpu_lib.gillespie_run(m.ns, m.rtype, m.K, m.S, m.D, m.init, int(g["seed"]), k + 1, m.max_time,
                                         m.write_interval)
        assert np.array_equal(c, g["counts"][k])


def test_gillespie_fixture_matches_the_analytic_moments():
    """Steady state of the two-state model: P(active) = k_on / (k_on + k_off),
    E[mRNA] = P(active) v0 / d0, E[protein] = E[mRNA] v1 / d1 (t = 3600 s is
    36 protein lifetimes, so the last record is stationary)."""
    g = load("gillespie_two_state")
    m = configs.two_state_gene()
    kon, koff, v0, v1, d0, d1 = m.K
    last = g["counts"][:, -1, :].astype(np.float64)
    n = last.shape[0]
    p_on = kon / (kon + koff)
    assert np.all(last[:, 0] + last[:, 1] == 1)
    se = np.sqrt(p_on * (1 - p_on) / n)
    assert abs(last[:, 1].mean() - p_on) < 4 * se
    mrna = p_on * v0 / d0
    assert abs(last[:, 2].mean() - mrna) < 4 * last[:, 2].std() / np.sqrt(n)
    prot = mrna * v1 / d1
    assert abs(last[:, 3].mean() - prot) < 4 * last[:, 3].std() / np.sqrt(n)


def test_nsm_fixture_conservation():
    for edge in (16, 32):
        g = load("nsm_bimolecular_%d" % edge)
        c = g["counts"].astype(np.int64)
        assert np.all(c[:, :, 0] == c[:, :1, 0] - c[:, :, 2])
        assert np.all(c[:, :, 1] == c[:, :1, 1] - c[:, :, 2])
