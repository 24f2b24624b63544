"""GPU parity of the Coulomb and exchange nuclear gradients against the oracle.

The oracle's gradients are pinned by finite differences of its J and K
energies (test_gradient_oracle.py); here every
vlxb_computeCoulombGradient<ABCD> and vlxb_computeExchangeGradient<ABCD> entry
point, called through the C ABI, is compared with the oracle's derivatives of
the same class, and the per-atom gradients with the oracle's.

Tolerances (FP64): per class and per atom, max |GPU - oracle| <= 1e-10 *
max |oracle| + 1e-14, the bar of the FP64 J build.  Mixed precision (FP32
below a screening bound of 1e-6): max |dG| <= 1e-6 on gradients of order 1.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import helpers
from vlxb import basis, fock, gradient, lists
from vlxb._lib import lib

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def g_params(cls):
    """Parameter names of vlxb_computeCoulombGradient<cls>, in ABI order."""
    return lib().g_params[cls]


def close(got, exp):
    scale = float(np.abs(exp).max()) if exp.size else 0.0
    return float(np.abs(got - exp).max()) <= RTOL * scale + 1e-14 if exp.size else True


@pytest.fixture(scope="module")
def system():
    lib().init(0)
    wl = basis.config_custom(3, 4.0, {0: 2, 1: 1, 2: 1}, 2, 0.2, 2.5, 3, 1e-12, 29)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    g, grads = helpers.oracle_coulomb_gradient(rl, wl.mol.natoms)
    return wl, rl, g, grads


@pytest.fixture(scope="module")
def kref(system):
    wl, rl, _, _ = system
    return helpers.oracle_exchange_gradient(rl, wl.mol.natoms)


def test_every_gradient_class_vs_oracle(system):
    wl, rl, _, _ = system
    dl = fock.to_device(rl)
    s = torch.cuda.current_stream().cuda_stream
    bad = []
    for cls in lists.j_classes():
        n = len(rl.jlists[cls[:2]].first)
        G = torch.zeros((6, n + 3), dtype=torch.float64, device="cuda")  # stride > count
        lib().coulomb_grad(cls, gradient.grad_args(dl, cls, G, 0, n + 3, s))
        got = G.cpu().numpy()
        exp = helpers.oracle_grad_class(rl, cls)
        if not close(got[:, :n], exp) or np.any(got[:, n:] != 0.0):
            bad.append((cls, float(np.abs(got[:, :n] - exp).max())))
    assert not bad, bad


def test_atom_gradient_vs_oracle_and_invariance(system):
    wl, rl, g_or, _ = system
    dl = fock.to_device(rl)
    cg = gradient.CoulombGradient(dl, wl.mol)
    g1 = cg.compute().cpu().numpy()
    g2 = cg.compute().cpu().numpy()
    assert np.array_equal(g1, g2)  # fixed summation order: bit-reproducible
    assert close(g1, g_or), float(np.abs(g1 - g_or).max())
    assert np.abs(g1.sum(axis=0)).max() <= 1e-9 * max(1.0, np.abs(g1).max())


def test_device_lists_gradient(system):
    """The convenience call (lists built on the GPU) gives the host-list result."""
    wl, _, g_or, _ = system
    g = gradient.coulomb_gradient(wl.mol, wl.D, wl.threshold).cpu().numpy()
    assert np.abs(g - g_or).max() <= 1e-10 * max(1.0, np.abs(g_or).max())


def test_mixed_precision_gradient(system):
    wl, rl, g_or, _ = system
    dl = fock.to_device(rl)
    L = lib()
    try:
        L.set_fp32_cut(1e-6)
        g32 = gradient.CoulombGradient(dl, wl.mol).compute().cpu().numpy()
    finally:
        L.set_fp32_cut(0.0)
    assert np.abs(g32 - g_or).max() <= 1e-6


def test_gradient_argument_checks(system):
    wl, rl, _, _ = system
    dl = fock.to_device(rl)
    s = torch.cuda.current_stream().cuda_stream
    n = len(rl.jlists["pd"].first)
    G = torch.zeros((6, n), dtype=torch.float64, device="cuda")
    args = gradient.grad_args(dl, "pdpd", G, 0, n - 1, s)  # stride below the entry count
    vals = [args[p] for p in g_params("pdpd")]
    rc = getattr(lib().cdll, "vlxb_computeCoulombGradientPDPD")(*vals)
    assert rc == 1  # VLXB_EINVAL
    torch.cuda.synchronize()
    assert float(G.abs().max()) == 0.0


def test_every_exchange_gradient_class_vs_oracle(system):
    """Each class's block values (at the block's lowest list position, nothing
    elsewhere) against the oracle's per-entry values summed per block."""
    wl, rl, _, _ = system
    dl = fock.to_device(rl)
    s = torch.cuda.current_stream().cuda_stream
    bad = []
    for cls in lists.k_classes():
        ac = cls[0] + cls[2]
        n = len(rl.kpairs[ac].pair_i)
        G = torch.zeros((6, n + 5), dtype=torch.float64, device="cuda")
        lib().exchange_grad(cls, gradient.kgrad_args(dl, cls, G, 0, n + 5, s))
        got = G.cpu().numpy()
        exp = helpers.kgrad_blocks(rl, ac, helpers.oracle_kgrad_class(rl, cls))
        if not close(got[:, :n], exp) or np.any(got[:, n:] != 0.0) or np.any(got[:, :n][exp == 0.0] != 0.0):
            bad.append((cls, float(np.abs(got[:, :n] - exp).max())))
    assert not bad, bad


def test_exchange_atom_gradient_vs_oracle(system, kref):
    wl, rl, _, _ = system
    g_or, _ = kref
    dl = fock.to_device(rl)
    eg = gradient.ExchangeGradient(dl, wl.mol)
    g1 = eg.compute().cpu().numpy()
    g2 = eg.compute().cpu().numpy()
    assert np.array_equal(g1, g2)
    assert close(g1, g_or), float(np.abs(g1 - g_or).max())
    assert np.abs(g1.sum(axis=0)).max() <= 1e-9 * max(1.0, np.abs(g1).max())


def test_range_separated_exchange_gradient(system):
    wl, rl, _, _ = system
    g_or, _ = helpers.oracle_exchange_gradient(rl, wl.mol.natoms, omega=0.4)
    g = gradient.ExchangeGradient(fock.to_device(rl), wl.mol).compute(omega=0.4).cpu().numpy()
    assert close(g, g_or), float(np.abs(g - g_or).max())


def test_device_lists_exchange_gradient(system, kref):
    wl, _, _, _ = system
    g_or, _ = kref
    g = gradient.exchange_gradient(wl.mol, wl.D, wl.threshold).cpu().numpy()
    assert np.abs(g - g_or).max() <= 1e-10 * max(1.0, np.abs(g_or).max())


def test_exchange_gradient_argument_checks_and_edges(system):
    """Stride below the (i, k) count: VLXB_EINVAL, nothing written.  A
    threshold that screens every quartet: exact zeros.  An empty (i, k) list:
    success, nothing written."""
    wl, rl, _, _ = system
    dl = fock.to_device(rl)
    s = torch.cuda.current_stream().cuda_stream
    L = lib()
    n = len(rl.kpairs["pp"].pair_i)  # class (pd|pd): (i, k) list of type pp
    G = torch.zeros((6, n), dtype=torch.float64, device="cuda")
    args = gradient.kgrad_args(dl, "pdpd", G, 0, n - 1, s)
    rc = getattr(L.cdll, "vlxb_computeExchangeGradientPDPD")(*[args[p] for p in L.kg_params["pdpd"]])
    assert rc == 1  # VLXB_EINVAL
    dl.threshold = 1e30
    nj = len(rl.jlists["pd"].first)
    GJ = torch.zeros((6, nj), dtype=torch.float64, device="cuda")
    L.exchange_grad("pdpd", gradient.kgrad_args(dl, "pdpd", G, 0, n, s))
    L.coulomb_grad("pdpd", gradient.grad_args(dl, "pdpd", GJ, 0, nj, s))
    torch.cuda.synchronize()
    assert float(G.abs().max()) == 0.0 and float(GJ.abs().max()) == 0.0
    dl.threshold = wl.threshold
    args = gradient.kgrad_args(dl, "pdpd", G, 0, n, s)
    args["pair_inds_count_for_K_pp"] = 0
    L.exchange_grad("pdpd", args)
    torch.cuda.synchronize()
    assert float(G.abs().max()) == 0.0


def test_gradient_fold_of_zero_entries():
    """A system whose lists are all empty after screening folds to zeros."""
    lib().init(0)
    wl = basis.config_custom(2, 3.0, {0: 1, 1: 1}, 1, 0.3, 2.5, 1, 1e-12, 5)
    rl = lists.build_lists(wl.mol, wl.D, 1e30, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    gj = gradient.CoulombGradient(dl, wl.mol).compute().cpu().numpy()
    gk = gradient.ExchangeGradient(dl, wl.mol).compute().cpu().numpy()
    assert gj.shape == (2, 3) and gk.shape == (2, 3)
    assert not gj.any() and not gk.any()
