"""Reference-format lists built on the GPU (vlxb.devlists, with the library's
vlxb_shellPairData / vlxb_gatherPairDensity / vlxb_blockMaxAbs) against the
host builder lists.build_lists, and the J/K they give."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from vlxb import aomap, basis, devlists, fock, lists
from vlxb._lib import lib

pytestmark = pytest.mark.gpu


def _system(seed=4, atoms=4):
    return basis.config_custom(atoms, 4.5, {0: 2, 1: 1, 2: 1}, 3, 0.2, 2.5, 4, 1e-12, seed)


def _close(a, b, rtol=1e-13):
    return np.allclose(a, b, rtol=rtol, atol=rtol * max(1e-300, float(np.abs(b).max(initial=0.0))))


def test_device_lists_match_host_builder():
    lib().init(0)
    wl = _system()
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    dl = devlists.build_device_lists(wl.mol, wl.D, wl.threshold)
    assert set(dl.j) == set(rl.jlists) and set(dl.kpart) == set(rl.kpartners) and set(dl.kpair) == set(rl.kpairs)
    for k in dl.maxD:
        assert dl.maxD[k] == rl.maxD[k], k
    for k, jl in rl.jlists.items():
        d = {n: t.cpu().numpy() for n, t in dl.j[k].items()}
        # same prim-cart pairs; values equal to rounding; sorted by descending |Q D|
        hk = np.lexsort((jl.second, jl.first))
        dk = np.lexsort((d["second"], d["first"]))
        assert np.array_equal(d["first"][dk].astype(np.uint32), jl.first[hk]), k
        assert np.array_equal(d["second"][dk].astype(np.uint32), jl.second[hk]), k
        assert _close(d["pdata"][dk], jl.pdata[hk]) and _close(d["Q"][dk], jl.Q[hk]), k
        assert np.array_equal(d["D"][dk], jl.D[hk]), k  # a gather: exact
        t = np.abs(d["Q"] * d["D"])
        assert np.all(t[:-1] >= t[1:]), k
    for k, kp in rl.kpartners.items():
        d = {n: t.cpu().numpy() for n, t in dl.kpart[k].items()}
        assert np.array_equal(d["counts"].astype(np.uint32), kp.counts), k
        assert np.array_equal(d["displs"].astype(np.uint32), kp.displs), k
        assert _close(d["Q"], kp.Q) and _close(d["pdata"], kp.pdata), k
        # partners of each first index: same set, descending Q
        for i in range(len(kp.counts)):
            a, n = kp.displs[i], kp.counts[i]
            assert np.array_equal(np.sort(d["Dinds"][a:a + n].astype(np.uint32)), np.sort(kp.Dinds[a:a + n])), k
            q = d["Q"][a:a + n]
            assert np.all(q[:-1] >= q[1:]), k
    for k, kq in rl.kpairs.items():
        assert np.array_equal(dl.kpair[k]["i"].cpu().numpy().astype(np.uint32), kq.pair_i), k
        assert np.array_equal(dl.kpair[k]["k"].cpu().numpy().astype(np.uint32), kq.pair_k), k


def test_device_lists_give_host_lists_jk_and_density_refresh():
    lib().init(0)
    wl = _system(seed=6)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    hdl = fock.to_device(rl)
    ddl = devlists.build_device_lists(wl.mol, wl.D, wl.threshold)

    def ao_jk(dl):
        am = aomap.AOMap.from_device(dl)
        fj, mJ, fk, mK = am.alloc_outputs()
        fock.build_jk(dl, matJ=mJ, matK=mK)
        return am.to_ao("J", fj).cpu().numpy(), am.to_ao("K", fk).cpu().numpy()

    Jh, Kh = ao_jk(hdl)
    Jd, Kd = ao_jk(ddl)
    assert np.abs(Jd - Jh).max() <= 1e-12 * np.abs(Jh).max()
    assert np.abs(Kd - Kh).max() <= 1e-12 * np.abs(Kh).max()
    # a new density through the per-SCF device refresh equals fresh host lists
    rng = np.random.default_rng(3)
    P = rng.standard_normal(wl.D.shape)
    D2 = wl.D + 1e-3 * (P + P.T)
    devlists.set_density(ddl, torch.from_numpy(D2).cuda())
    rl2 = lists.build_lists(wl.mol, D2, wl.threshold, fock.gpu_schwarz_fn())
    for k in ddl.maxD:
        assert ddl.maxD[k] == rl2.maxD[k]
    J2, K2 = ao_jk(fock.to_device(rl2))
    Jd2, Kd2 = ao_jk(ddl)
    assert np.abs(Jd2 - J2).max() <= 1e-12 * np.abs(J2).max()
    assert np.abs(Kd2 - K2).max() <= 1e-12 * np.abs(K2).max()


def test_block_max_and_gather_reject_bad_arguments():
    L = lib()
    L.init(0)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(Exception):
        L.block_max_abs(0, 3, 0, 1, 0, 1, out.data_ptr(), 0)
    with pytest.raises(Exception):
        L.gather_pair_density(0, 3, 0, 0, 0, 1, 1, 0, 1, 1, 5, out.data_ptr(), 0)
