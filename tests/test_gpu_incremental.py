"""Incremental builds on a density difference (the large sparse workload's
mode) on a smaller cluster of the same recipe: 4s3p2d atoms at 25 bohr^3 per
atom, lists built on the device with Schwarz and density-weighted screening.

  * J and K are linear in D: without screening, J(D0) + J(dD) equals
    J(D0 + dD) to rounding (a size-independent property);
  * with the workload's screening at 1e-11 on dD (|dD|_F = 1e-3), the
    incremental result J(D0) + J(dD) stays within 1e-8 of the full rebuild
    J(D0 + dD) at the same threshold, for J, K and E = Tr[D(J - K/2)];
  * in mixed precision (FP32 below a Schwarz bound of 1e-6 inside the FP32
    error budget, FP64 accumulation) the incremental result stays within the
    mixed-precision bar of 1e-7 of the FP64 one.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from vlxb import basis, devlists, fock, lists
from vlxb._lib import lib

pytestmark = pytest.mark.gpu
ATOMS = 10


def _build_ao(mol, D, thr, cut=0.0):
    L = lib()
    dl = devlists.build_device_lists(mol, D, thr)
    try:
        L.set_fp32_cut(cut)
        mJ, mK = fock.build_jk(dl)
        torch.cuda.synchronize()
    finally:
        L.set_fp32_cut(0.0)
    host = devlists.to_host(dl, mol)
    J = lists.contract_J(host, {k: v.cpu().numpy() for k, v in mJ.items()})
    K = lists.contract_K(host, {k: v.cpu().numpy() for k, v in mK.items()})
    return J, K


@pytest.fixture(scope="module")
def cluster():
    lib().init(0)
    wl = basis.molecule_at_density(ATOMS, 25.0, 2, threshold=1e-11)
    rng = np.random.default_rng(9)
    P = rng.standard_normal(wl.D.shape)
    P = 0.5 * (P + P.T)
    dD = P * (1e-3 / np.linalg.norm(P))
    return wl, dD


def test_linearity_without_screening(cluster):
    wl, dD = cluster
    J0, K0 = _build_ao(wl.mol, wl.D, 0.0)
    Jd, Kd = _build_ao(wl.mol, dD, 0.0)
    J1, K1 = _build_ao(wl.mol, wl.D + dD, 0.0)
    assert np.abs(J0 + Jd - J1).max() <= 1e-12 * np.abs(J1).max()
    assert np.abs(K0 + Kd - K1).max() <= 1e-12 * np.abs(K1).max()


def test_incremental_matches_full_rebuild(cluster):
    wl, dD = cluster
    thr = 1e-11
    D1 = wl.D + dD
    J0, K0 = _build_ao(wl.mol, wl.D, thr)
    Jd, Kd = _build_ao(wl.mol, dD, thr)
    J1, K1 = _build_ao(wl.mol, D1, thr)
    Ji, Ki = J0 + Jd, K0 + Kd
    assert np.abs(Ji - J1).max() <= 1e-8
    assert np.abs(Ki - K1).max() <= 1e-8
    assert abs(lists.energy(D1, Ji, Ki) - lists.energy(D1, J1, K1)) <= 1e-8
    # mixed precision on the increment: within the mixed-precision bar
    Jm, Km = _build_ao(wl.mol, dD, thr, cut=1e-6)
    assert np.abs(Jm - Jd).max() <= 1e-7
    assert np.abs(Km - Kd).max() <= 1e-7
