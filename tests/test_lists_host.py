"""Host-side list building, AO contraction and energy (CPU, oracle-backed)."""
import numpy as np

import helpers
from vlxb import basis, lists
from vlxb.basis import NCART


def tiny_molecule(seed=3, recipe=None):
    rng = np.random.default_rng(seed)
    coords = basis.place_atoms(2, 2.5, rng)
    mol = basis.build_molecule(coords, recipe or {0: 1, 1: 1, 2: 1}, degree=2, alpha0=0.4, ratio=2.2, rng=rng)
    D = basis.make_density(mol, 3, np.random.default_rng(seed + 1))
    return mol, D


def test_basis_normalisation_and_density():
    mol, D = tiny_molecule()
    S = basis.overlap_matrix(mol)
    assert np.allclose(S, S.T, atol=1e-14)
    # x^l components are unit-normalised
    for sh in mol.shells:
        assert abs(S[sh.ao0, sh.ao0] - 1.0) < 1e-12
    # D S D = D for an S-orthonormal occupied space
    assert np.allclose(D @ S @ D, D, atol=1e-10)


def test_list_formats():
    mol, D = tiny_molecule()
    rl = lists.build_lists(mol, D, 1e-12, helpers.oracle_schwarz_fn)
    for key, jl in rl.jlists.items():
        t = np.abs(jl.Q * jl.D)
        assert np.all(t[:-1] >= t[1:]), key  # sorted for the reference's break
        if key[0] == key[1]:
            assert np.all(jl.first <= jl.second)
    for key, kp in rl.kpartners.items():
        la = lists.LV[key[0]]
        assert len(kp.counts) == rl.pd.count[la] * NCART[la]
        for i in range(len(kp.counts)):
            q = kp.Q[kp.displs[i]:kp.displs[i] + kp.counts[i]]
            assert np.all(q[:-1] >= q[1:])


def test_ao_contraction_matches_ao_tensor():
    """J and K assembled from the prim-pair lists equal J/K from the full AO
    ERI tensor contracted with D (both from the oracle)."""
    mol, D = tiny_molecule(recipe={0: 1, 1: 1})
    rl = lists.build_lists(mol, D, 0.0, helpers.oracle_schwarz_fn)
    matJ, matK = helpers.oracle_jk_all(rl)
    J = lists.contract_J(rl, matJ)
    K = lists.contract_K(rl, matK)
    G = helpers.ao_eri_tensor(mol)
    J_ref = np.einsum("ijkl,kl->ij", G, D)
    K_ref = np.einsum("ikjl,kl->ij", G, D)
    assert np.abs(J - J_ref).max() < 1e-11
    assert np.abs(K - K_ref).max() < 1e-11
    E = lists.energy(D, J, K)
    assert abs(E - np.sum(D * (J_ref - 0.5 * K_ref))) < 1e-10
