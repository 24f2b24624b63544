"""The oracle restatement against the reference's own emitted expressions,
compiled for the host (oracle/_ref, built by oracle/make_ref.py), on a small
s/p/d system: every J and K class, full rows, plus the bounded-sample mode
and the shell-quartet counts used by the benchmark's CPU leg.
"""
import numpy as np
import pytest

import helpers
from oracle import ref
from vlxb import basis, lists

pytestmark = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built (needs the reference tree)")


@pytest.fixture(scope="module")
def system():
    wl = basis.config_custom(2, 3.0, {0: 1, 1: 1, 2: 1}, 2, 0.3, 2.5, 3, 1e-12, 23)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, ref.schwarz_fn)
    return wl, rl


def test_reference_schwarz_matches_oracle(system):
    wl, rl = system
    pd = rl.pd
    for la in range(3):
        for lb in range(la, 3):
            a = lists.all_shell_pairs(pd, la, lb, ref.schwarz_fn)
            b = lists.all_shell_pairs(pd, la, lb, helpers.oracle_schwarz_fn)
            assert np.allclose(a.q, b.q, rtol=1e-12, atol=0)


def test_reference_J_and_K_match_oracle(system):
    wl, rl = system
    for cls in lists.j_classes():
        got, npass, neval = ref.coulomb(rl, cls)
        exp = helpers.oracle_J(rl, cls)
        assert npass == neval
        assert np.abs(got - exp).max() <= 1e-12 * max(np.abs(exp).max(), 1e-300), cls
    for cls in lists.k_classes():
        got, npass, neval = ref.exchange(rl, cls)
        exp = helpers.oracle_K(rl, cls)
        assert np.abs(got - exp).max() <= 1e-12 * max(np.abs(exp).max(), 1e-300), cls


def test_bounded_sampling_counts(system):
    wl, rl = system
    _, npass, neval = ref.coulomb(rl, "ppdd", rows=np.arange(5), max_eval=3)
    assert neval <= 15 and npass >= neval
    _, npass, neval = ref.exchange(rl, "sdpd", rows=np.arange(4), max_eval=7)
    assert neval <= 28 and npass >= neval


def test_shell_quartet_counts_positive(system):
    wl, rl = system
    assert ref.count_j(rl, "ssss") > 0
    assert ref.count_k(rl, "dddd") > 0
