"""Host-side workload generators and schedule bookkeeping (CPU)."""
import numpy as np

from vlxb import basis
from vlxb.serve import perturbed_densities
from vlxb.tune import compiled_variants


def test_perturbed_densities_are_symmetric_and_log_spaced():
    D0 = np.eye(6)
    Ds = perturbed_densities(D0, 5, np.random.default_rng(0), hi=1e-2, lo=1e-6)
    assert len(Ds) == 5 and Ds[0] is D0
    norms = [np.linalg.norm(D - D0) for D in Ds[1:]]
    assert np.allclose(norms, np.logspace(-2, -6, 4), rtol=1e-12)
    for D in Ds:
        assert np.array_equal(D, D.T)


def test_batch_and_serve_workloads():
    wls = basis.config_batch(6, (3, 5), 30.0, seed=1)
    assert len(wls) == 6
    for w in wls:
        n = len(w.mol.coords)
        assert 3 <= n <= 5
        side = (30.0 * n) ** (1 / 3)
        assert np.all(w.mol.coords >= -1e-9) and np.all(w.mol.coords <= side + 1e-9)
        assert w.D.shape == (w.mol.naos, w.mol.naos)
    counts = basis.serve_atom_counts(200, 5, 120, seed=3)
    assert counts.min() >= 5 and counts.max() <= 120
    assert np.median(counts) < 0.5 * (5 + 120)  # log-uniform: median well below the midpoint


def test_compiled_variants():
    assert compiled_variants("J", "ssss") == [0, 1, 2, 3]
    assert 0 not in compiled_variants("J", "dddd")  # its thread kernel spills and is never timed
    kv = compiled_variants("K", "pddd")
    assert set(kv) <= set(range(13)) and {1, 3, 7, 11} <= set(kv) and 0 not in kv
    assert 5 in compiled_variants("K", "dpdd") and 6 in compiled_variants("K", "dddp")
