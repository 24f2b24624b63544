"""Classes with f shells (this library's own entry points; the reference's
writer emits s, p and d only), through the C ABI, against the FP64 oracle.

The oracle's f-shell integrals are pinned to the reference's own symbolic
engine run with three Cartesian indices on f centres
(tests/golden/eri_f_components.npz, test_oracle_golden.py); its J / K loops
are the ones pinned on the s/p/d classes.  Here: a two-atom s/p/d/f system,
every J and K list (the 100 Coulomb and 160 exchange classes of s..f) against
the oracle at the FP64 bar, AO J / K and the energy, range-separated
exchange, the f-pair Schwarz values, and bit-for-bit repeatability.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import helpers
from vlxb import basis, fock, lists
from vlxb._lib import lib

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def close(got, exp):
    scale = float(np.abs(exp).max()) if exp.size else 0.0
    return float(np.abs(got - exp).max()) <= RTOL * scale + 1e-14 if exp.size else True


@pytest.fixture(scope="module")
def spdf():
    lib().init(0)
    wl = basis.config_custom(2, 3.0, {0: 1, 1: 1, 2: 1, 3: 1}, 2, 0.3, 2.5, 4, 1e-12, 7)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    return wl, rl


def test_fpair_schwarz_matches_oracle(spdf):
    wl, rl = spdf
    pd = rl.pd
    g = fock.gpu_schwarz_fn()
    for la, lb in ((0, 3), (1, 3), (2, 3), (3, 3)):
        sp_g = lists.all_shell_pairs(pd, la, lb, g)
        sp_o = lists.all_shell_pairs(pd, la, lb, helpers.oracle_schwarz_fn)
        assert np.allclose(sp_g.q, sp_o.q, rtol=1e-11, atol=1e-300), (la, lb)


def test_spdf_every_class_vs_oracle(spdf):
    wl, rl = spdf
    assert "ff" in rl.jlists and "fd" in rl.kpartners
    dl = fock.to_device(rl)
    runs = []
    for _ in range(2):
        matJ, matK = fock.build_jk(dl)
        torch.cuda.synchronize()
        runs.append(({k: v.cpu().numpy() for k, v in matJ.items()}, {k: v.cpu().numpy() for k, v in matK.items()}))
    gJ, gK = runs[0]
    for t in (0, 1):
        for k in runs[0][t]:
            assert np.array_equal(runs[0][t][k], runs[1][t][k]), (t, k)
    oJ, oK = helpers.oracle_jk_all(rl)
    bad = [("J", k) for k in oJ if not close(gJ[k], oJ[k])] + [("K", k) for k in oK if not close(gK[k], oK[k])]
    assert not bad, bad
    J, K = lists.contract_J(rl, gJ), lists.contract_K(rl, gK)
    Jo, Ko = lists.contract_J(rl, oJ), lists.contract_K(rl, oK)
    assert np.abs(J - Jo).max() <= 1e-10 * np.abs(Jo).max()
    assert np.abs(K - Ko).max() <= 1e-10 * np.abs(Ko).max()
    assert abs(lists.energy(wl.D, J, K) - lists.energy(wl.D, Jo, Ko)) < 1e-10


def test_spdf_device_built_lists(spdf):
    """The device list builder with f shells (pair data and Schwarz values of
    f pairs on the GPU): the same J / K as the host-built lists."""
    from vlxb import devlists

    wl, rl = spdf
    dl_h = fock.to_device(rl)
    dl_d = devlists.build_device_lists(wl.mol, wl.D, wl.threshold)
    Jh, Kh = fock.build_jk(dl_h)
    Jd, Kd = fock.build_jk(dl_d)
    torch.cuda.synchronize()
    host_d = devlists.to_host(dl_d, wl.mol)
    a = lists.contract_J(rl, {k: v.cpu().numpy() for k, v in Jh.items()})
    b = lists.contract_J(host_d, {k: v.cpu().numpy() for k, v in Jd.items()})
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()
    a = lists.contract_K(rl, {k: v.cpu().numpy() for k, v in Kh.items()})
    b = lists.contract_K(host_d, {k: v.cpu().numpy() for k, v in Kd.items()})
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()


def test_spdf_range_separated_exchange(spdf):
    wl, rl = spdf
    dl = fock.to_device(rl)
    _, matK = fock.build_jk(dl, omega=0.4, do_j=False)
    torch.cuda.synchronize()
    _, oK = helpers.oracle_jk_all(rl, omega=0.4)
    for k in oK:
        assert close(matK[k].cpu().numpy(), oK[k]), k
