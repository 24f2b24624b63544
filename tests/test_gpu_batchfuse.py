"""Fused batches (vlxb_coulombBatch / vlxb_exchangeBatch through
vlxb.batchfuse): one class call for many molecules gives every molecule the
J and K of its own class calls, the same quartet count, also from a captured
graph and after a density update."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from vlxb import basis, fock, lists
from vlxb._lib import lib
from vlxb.batchfuse import FusedBatch, FusedBatchGroups

pytestmark = pytest.mark.gpu


def _mols(n, seed=0):
    return [basis.molecule_at_density(3 + (t * 2) % 5, 30.0, seed + t) for t in range(n)]


def _direct(wl, rl=None):
    """The molecule's own class calls (on its fused-batch lists when given)."""
    rl = rl or lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    mJ, mK = fock.alloc_outputs(dl)
    L = lib()
    L.reset_counters()
    fock.build_jk(dl, matJ=mJ, matK=mK)
    torch.cuda.synchronize()
    q = sum(L.quartet_counters())
    return {k: v.cpu().numpy() for k, v in mJ.items()}, {k: v.cpu().numpy() for k, v in mK.items()}, q


def _same(a, b):
    for k in b:
        assert np.abs(a[k] - b[k]).max(initial=0.0) <= 1e-13 * max(1.0, np.abs(b[k]).max(initial=0.0)), k


def test_fused_batch_equals_per_molecule_calls():
    L = lib()
    L.init(0)
    wls = _mols(5)
    fb = FusedBatch([w.mol for w in wls], [w.D for w in wls], 1e-12)
    L.reset_counters()
    fb.run()
    torch.cuda.synchronize()
    qf = sum(L.quartet_counters())
    qd = 0
    for t, wl in enumerate(wls):
        dJ, dK, q = _direct(wl)
        qd += q
        gJ, gK = fb.results(t)
        _same(gJ, dJ)
        _same(gK, dK)
    assert qf == qd
    # captured graph, then a new density of one molecule (larger max |D|)
    fb.capture()
    D2 = 1.3 * wls[2].D
    fb.set_density(2, D2)
    fb.run()
    gJ, gK = fb.results(2)
    dJ, dK, _ = _direct(wls[2], fb.rls[2])  # same lists, new density values and bounds
    _same(gJ, dJ)
    _same(gK, dK)
    gJ0, gK0 = fb.results(0)
    dJ0, dK0, _ = _direct(wls[0])
    _same(gJ0, dJ0)
    _same(gK0, dK0)


def test_grouped_fused_batch_equals_per_molecule_calls():
    """A batch split into fused unions of at most two molecules: every
    molecule's J and K equal its own class calls, the quartet count equals
    theirs, also from one captured graph over all groups and after a density
    update."""
    L = lib()
    L.init(0)
    wls = _mols(5, seed=3)
    fg = FusedBatchGroups([w.mol for w in wls], [w.D for w in wls], 1e-12, group=2)
    assert len(fg.parts) == 3 and fg.nmol == 5
    fg.capture()
    L.reset_counters()
    fg.run()
    torch.cuda.synchronize()
    qf = sum(L.quartet_counters())
    assert qf == fg.quartets_per_iteration
    qd = 0
    for t, wl in enumerate(wls):
        dJ, dK, q = _direct(wl)
        qd += q
        gJ, gK = fg.results(t)
        _same(gJ, dJ)
        _same(gK, dK)
    assert qf == qd
    D3 = 0.8 * wls[3].D
    fg.set_density(3, D3)
    fg.run()
    gJ, gK = fg.results(3)
    p, k = fg.where[3]
    dJ, dK, _ = _direct(wls[3], fg.parts[p].rls[k])
    _same(gJ, dJ)
    _same(gK, dK)
