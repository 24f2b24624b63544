"""AO map (the layout vlxb_pairsToAO reads): its numpy evaluation equals the
host contraction lists.contract_J / contract_K on every list of an s/p/d system."""
import numpy as np

import helpers
from test_lists_host import tiny_molecule
from vlxb import aomap, lists


def _flat(values: dict, keys):
    return np.concatenate([values[k] for k in keys]) if keys else np.zeros(0)


def test_map_equals_host_contraction():
    mol, D = tiny_molecule(seed=5)
    rl = lists.build_lists(mol, D, 1e-12, helpers.oracle_schwarz_fn)
    rng = np.random.default_rng(0)
    vJ = {k: rng.standard_normal(len(v.first)) for k, v in rl.jlists.items()}
    vK = {k: rng.standard_normal(len(v.pair_i)) for k, v in rl.kpairs.items()}
    for kind, vals, ref, tg in (("J", vJ, lists.contract_J, aomap._targets_J),
                                ("K", vK, lists.contract_K, aomap._targets_K)):
        keys = sorted(vals)
        sizes = [len(vals[k]) for k in keys]
        off = np.concatenate([[0], np.cumsum(sizes)])
        rowptr, row_ao, src = aomap.build_map(rl.naos, [(off[i], *tg(rl, k)) for i, k in enumerate(keys)])
        assert rowptr[-1] == sum(sizes) and np.all(np.diff(rowptr) > 0)
        assert np.all(np.diff(row_ao) > 0)  # one row per AO pair, ascending
        a, b = np.divmod(row_ao, rl.naos)
        assert np.all(a <= b)
        M = aomap.contract_host(rl.naos, _flat(vals, keys), rowptr, row_ao, src)
        R = ref(rl, vals)
        assert np.allclose(M, R, rtol=0, atol=1e-13 * max(1.0, np.abs(R).max())), kind
        assert np.array_equal(M, M.T)


def test_empty_map():
    rowptr, row_ao, src = aomap.build_map(7, [])
    assert rowptr.tolist() == [0] and len(row_ao) == 0 and len(src) == 0


def test_torch_map_equals_numpy_map():
    """AOMap.from_device (torch ops; run here on CPU tensors) builds exactly
    the numpy map of AOMap(rl)."""
    import torch
    from vlxb import fock

    mol, D = tiny_molecule(seed=9)
    rl = lists.build_lists(mol, D, 1e-12, helpers.oracle_schwarz_fn)
    ref = aomap.AOMap(rl, device="cpu")
    dl = fock.to_device(rl, "cpu")
    got = aomap.AOMap.from_device(dl)
    for a, b in ((ref.J, got.J), (ref.K, got.K)):
        assert a.keys == b.keys and a.sizes == b.sizes
        assert torch.equal(a.rowptr, b.rowptr)
        assert torch.equal(a.row_ao, b.row_ao)
        assert torch.equal(a.src, b.src)
