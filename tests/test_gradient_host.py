"""Host logic of the gradient fold, on CPU tensors: the CSR (entry, side) ->
atom layout of vlxb.gradient.GradientMap, evaluated with numpy, equals the
direct per-entry fold used by the oracle helpers."""
import numpy as np
import torch

import helpers
from vlxb import basis, fock, gradient, lists


def _fold_csr(gmap, G, w):
    src = gmap.src.numpy().view(np.uint32)
    rowptr = gmap.rowptr.numpy()
    out = np.zeros((gmap.natoms, 3))
    for t in range(gmap.natoms):
        for e in src[rowptr[t]:rowptr[t + 1]]:
            p, side = int(e & 0x7FFFFFFF), int(e >> 31)
            out[t] += (w[p] if w is not None else 1.0) * G[3 * side:3 * side + 3, p]
    return out


def test_gradient_maps_fold_like_the_oracle_helpers():
    wl = basis.config_custom(3, 4.0, {0: 1, 1: 1, 2: 1}, 2, 0.3, 2.5, 3, 1e-12, 17)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, helpers.oracle_schwarz_fn)
    dl = fock.to_device(rl, device="cpu")
    atoms = gradient.prim_atoms(wl.mol, "cpu")
    rng = np.random.default_rng(0)
    # J: flat [6][total] values, weights w_o D_o
    jm = gradient.GradientMap(dl.j, ("first", "second"), atoms, wl.mol.natoms, "cpu")
    G = rng.standard_normal((6, jm.total))
    w = gradient.coulomb_weights(dl, jm).numpy()
    exp = np.zeros((wl.mol.natoms, 3))
    for k in jm.keys:
        jl = rl.jlists[k]
        la, lb = lists.LV[k[0]], lists.LV[k[1]]
        o = jm.offsets[k]
        Gk = G[:, o:o + len(jl.first)]
        wk = helpers.bra_weights(rl, k)
        assert np.array_equal(w[o:o + len(jl.first)], wk)
        np.add.at(exp, rl.pd.atom[la][jl.first // lists.NCART[la]], (wk * Gk[:3]).T)
        np.add.at(exp, rl.pd.atom[lb][jl.second // lists.NCART[lb]], (wk * Gk[3:]).T)
    assert np.allclose(_fold_csr(jm, G, w), exp, rtol=1e-13, atol=1e-13)
    # K: values come weighted, the fold adds them unweighted
    km = gradient.GradientMap(dl.kpair, ("i", "k"), atoms, wl.mol.natoms, "cpu")
    GK = rng.standard_normal((6, km.total))
    expk = np.zeros((wl.mol.natoms, 3))
    for k in km.keys:
        kp = rl.kpairs[k]
        la, lc = lists.LV[k[0]], lists.LV[k[1]]
        o = km.offsets[k]
        Gk = GK[:, o:o + len(kp.pair_i)]
        np.add.at(expk, rl.pd.atom[la][kp.pair_i // lists.NCART[la]], Gk[:3].T)
        np.add.at(expk, rl.pd.atom[lc][kp.pair_k // lists.NCART[lc]], Gk[3:].T)
    assert np.allclose(_fold_csr(km, GK, None), expk, rtol=1e-13, atol=1e-13)
    # every (entry, side) appears exactly once
    assert jm.rowptr[-1].item() == 2 * jm.total and km.rowptr[-1].item() == 2 * km.total


def test_kgrad_blocks_places_block_sums_at_lowest_position():
    wl = basis.config_custom(2, 3.0, {1: 1, 2: 1}, 2, 0.3, 2.5, 2, 1e-12, 3)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, helpers.oracle_schwarz_fn)
    key = "pd"
    kp = rl.kpairs[key]
    G = np.arange(6 * len(kp.pair_i), dtype=float).reshape(6, -1) + 1.0
    B = helpers.kgrad_blocks(rl, key, G)
    assert np.allclose(B.sum(axis=1), G.sum(axis=1))
    blk = (kp.pair_i // 3).astype(np.int64) * (1 << 32) + kp.pair_k // 6
    for b in np.unique(blk):
        pos = np.nonzero(blk == b)[0]
        assert np.allclose(B[:, pos[0]], G[:, pos].sum(axis=1))
        assert np.all(B[:, pos[1:]] == 0.0)
