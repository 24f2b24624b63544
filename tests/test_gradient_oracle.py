"""Nuclear gradients of E_J = 1/2 Tr[D J] and E_K = 1/2 Tr[D K]: the oracle's
derivative integrals, pinned by central finite differences of the oracle's
own J and K energies (themselves pinned by the reference-generated golden
vectors), and the host-side folding rules.

System: three atoms at a bent geometry with one s, p and d shell each (one
primitive), threshold 0, so that every pair is in every list and the energy
is a smooth function of the coordinates.
"""
import numpy as np

import helpers
from vlxb import basis, lists
from vlxb.basis import Molecule

H = 1e-4          # central-difference step (bohr): truncation ~ H^2, rounding ~ 1e-16 / H
FD_TOL = 2e-8     # absolute, on gradients of order 0.1


def _system():
    rng = np.random.default_rng(5)
    coords = np.array([[0.0, 0.0, 0.0], [1.9, 0.3, -0.2], [0.4, 1.7, 0.6]])
    mol = basis.build_molecule(coords, {0: 1, 1: 1, 2: 1}, degree=1, alpha0=0.45, ratio=2.0, rng=rng)
    D = basis.make_density(mol, 6, rng)
    return mol, D


def _lists(mol, D):
    return lists.build_lists(mol, D, 0.0, helpers.oracle_schwarz_fn)


def _moved(mol, atom, x, h):
    c = mol.coords.copy()
    c[atom, x] += h
    return Molecule(coords=c, shells=mol.shells, naos=mol.naos)


def test_energy_matches_ao_trace():
    mol, D = _system()
    rl = _lists(mol, D)
    matJ = {k: np.zeros(len(v.first)) for k, v in rl.jlists.items()}
    for cls in lists.j_classes():
        matJ[cls[:2]] += helpers.oracle_J(rl, cls)
    J = lists.contract_J(rl, matJ)
    assert abs(0.5 * np.sum(D * J) - helpers.oracle_coulomb_energy(rl)) <= 1e-12 * abs(np.sum(D * J))


def test_oracle_gradient_matches_finite_differences():
    mol, D = _system()
    g, _ = helpers.oracle_coulomb_gradient(_lists(mol, D), mol.natoms)
    assert np.abs(g).max() > 1e-3
    for atom in (1, 2):
        for x in range(3):
            ep = helpers.oracle_coulomb_energy(_lists(_moved(mol, atom, x, H), D))
            em = helpers.oracle_coulomb_energy(_lists(_moved(mol, atom, x, -H), D))
            fd = (ep - em) / (2 * H)
            assert abs(fd - g[atom, x]) <= FD_TOL, (atom, x, fd, g[atom, x])


def test_oracle_gradient_translation_invariant():
    mol, D = _system()
    g, _ = helpers.oracle_coulomb_gradient(_lists(mol, D), mol.natoms)
    assert np.abs(g.sum(axis=0)).max() <= 1e-11 * max(1.0, np.abs(g).max())


def test_derivative_sides_sum_to_product_derivative():
    """d/dA + d/dB of a bra entry equals minus the ket-side derivative of the
    same class summed over C and D, checked here through the swap symmetry:
    on an s-only system, every class is (ss|ss) and the bra-centre
    derivatives of the entry pair (o, kl) equal minus those of (kl, o)
    computed with the roles exchanged."""
    rng = np.random.default_rng(2)
    coords = np.array([[0.0, 0.0, 0.0], [1.3, -0.4, 0.5]])
    mol = basis.build_molecule(coords, {0: 2}, degree=1, alpha0=0.5, ratio=3.0, rng=rng)
    D = basis.make_density(mol, 1, rng)
    rl = _lists(mol, D)
    _, grads = helpers.oracle_coulomb_gradient(rl, mol.natoms)
    G = grads["ss"]
    w = helpers.bra_weights(rl, "ss")
    # sum over all bra entries of w D (dA + dB) is the total translation of
    # the bra side, which must cancel the ket side: total sum zero
    tot = (w * (G[:3] + G[3:])).sum(axis=1)
    assert np.abs(tot).max() <= 1e-12 * max(1.0, np.abs(G).max())


def test_oracle_exchange_gradient_matches_finite_differences():
    """dE_K/dR for E_K = 1/2 Tr[D K] against central differences of the
    oracle's K energy (threshold 0)."""
    mol, D = _system()
    g, _ = helpers.oracle_exchange_gradient(_lists(mol, D), mol.natoms)
    assert np.abs(g).max() > 1e-3
    assert np.abs(g.sum(axis=0)).max() <= 1e-11 * max(1.0, np.abs(g).max())
    for atom, x in ((1, 0), (2, 1), (2, 2)):
        ep = helpers.oracle_exchange_energy(_lists(_moved(mol, atom, x, H), D))
        em = helpers.oracle_exchange_energy(_lists(_moved(mol, atom, x, -H), D))
        fd = (ep - em) / (2 * H)
        assert abs(fd - g[atom, x]) <= FD_TOL, (atom, x, fd, g[atom, x])


def test_oracle_range_separated_exchange_gradient():
    """The same with the erf-attenuated operator (omega = 0.4)."""
    mol, D = _system()
    om = 0.4
    g, _ = helpers.oracle_exchange_gradient(_lists(mol, D), mol.natoms, omega=om)
    ep = helpers.oracle_exchange_energy(_lists(_moved(mol, 1, 1, H), D), omega=om)
    em = helpers.oracle_exchange_energy(_lists(_moved(mol, 1, 1, -H), D), omega=om)
    assert abs((ep - em) / (2 * H) - g[1, 1]) <= FD_TOL
