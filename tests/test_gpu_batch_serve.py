"""Batched (one CUDA graph per iteration) and served builds.

* the graph-replayed batch gives bitwise the J/K of direct per-molecule builds,
  also after a density update;
* a served request gives the same J/K and energies alone and in a mix of
  concurrent requests;
* incremental (dD) serving agrees with full rebuilds within the screening
  threshold's reach.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from vlxb import basis, fock, lists
from vlxb._lib import lib
from vlxb.batch import BatchedBuilder
from vlxb.serve import Request, Server, perturbed_densities

pytestmark = pytest.mark.gpu


def small_mols(n, seed=0):
    out = []
    for t in range(n):
        wl = basis.config_custom(2 + t % 3, 3.0 + t % 3, {0: 2, 1: 1, 2: 1}, 2, 0.3, 2.5, 3, 1e-12, seed + t)
        out.append(wl)
    return out


def direct(wl, D=None):
    rl = lists.build_lists(wl.mol, wl.D if D is None else D, wl.threshold, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    mJ, mK = fock.build_jk(dl)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in mJ.items()}, {k: v.cpu().numpy() for k, v in mK.items()}


def test_batched_graph_equals_direct_builds():
    lib().init(0)
    wls = small_mols(5)
    bb = BatchedBuilder([w.mol for w in wls], [w.D for w in wls], 1e-12, streams=3)
    bb.capture()
    bb.run()
    bb.run()  # a second replay must give the same complete build
    for t, wl in enumerate(wls):
        gJ, gK = bb.results(t)
        dJ, dK = direct(wl)
        for k in dJ:
            assert np.array_equal(gJ[k], dJ[k]), (t, k)
        for k in dK:
            assert np.array_equal(gK[k], dK[k]), (t, k)
    # new density for member 1, smaller than before: same graph, new result
    D2 = 0.9 * wls[1].D
    bb.set_density(1, D2)
    bb.run()
    gJ, gK = bb.results(1)
    dJ, dK = direct(wls[1], D2)
    for k in dJ:
        assert np.allclose(gJ[k], dJ[k], rtol=0, atol=1e-12 * max(1.0, np.abs(dJ[k]).max()))
    assert bb.quartets_per_iteration > 0


def _requests(seed, n=4, iters=3):
    rng = np.random.default_rng(seed)
    out = []
    for t, wl in enumerate(small_mols(n, seed=10 + seed)):
        Ds = perturbed_densities(wl.D, iters, np.random.default_rng(100 + t))
        out.append(Request(t, wl.mol, Ds, wl.threshold, arrival=float(rng.exponential(0.002)) * t))
    return out


def test_served_results_same_alone_and_in_mix():
    lib().init(0)
    mix = _requests(0)
    Server(budget_bytes=1e9, max_active=4).run(mix)
    for r in mix:
        alone = _requests(0)[r.rid]
        alone.arrival = 0.0
        st = Server(budget_bytes=1e9, max_active=1).run([alone])
        assert st["requests"] == 1
        assert np.array_equal(alone.J, r.J) and np.array_equal(alone.K, r.K)
        assert alone.energies == r.energies


def test_incremental_serving_matches_full_rebuilds():
    lib().init(0)
    full = _requests(1, n=2, iters=4)
    inc = _requests(1, n=2, iters=4)
    Server(max_active=2).run(full)
    stats = Server(max_active=2, incremental=True).run(inc)
    assert stats["builds"] == 8
    for a, b in zip(full, inc):
        assert np.abs(a.J - b.J).max() < 1e-9
        assert np.abs(a.K - b.K).max() < 1e-9
        assert abs(a.energies[-1] - b.energies[-1]) < 1e-8
