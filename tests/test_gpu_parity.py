"""GPU parity: every J and K entry point, called through the C ABI, against
the reference-generated golden fixture and against the CPU oracle.

Tolerance (FP64 mode): max |GPU - expected| <= 1e-10 * max |expected| + 1e-14
per class and list, the bar of 1e-10 stated for the FP64 build.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import helpers
import tiny_fixture as tf
from vlxb import basis, fock, lists
from vlxb._lib import lib
from vlxb.fock import DeviceLists

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def close(got, exp):
    scale = float(np.abs(exp).max()) if exp.size else 0.0
    return float(np.abs(got - exp).max()) <= RTOL * scale + 1e-14 if exp.size else True


def fixture_lists(z, thr):
    dev = torch.device("cuda")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    U = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).to(dev)
    info, aoinds, count = tf.prim_tables(z)
    dl = DeviceLists(device=dev, naos=int(z["naos"][0]), threshold=thr, count=count)
    dl.D_AO = T(z["D_AO"])
    for l in range(3):
        dl.info[l] = T(info[l])
        dl.aoinds[l] = U(aoinds[l])
    for ab in ("ss", "sp", "sd", "pp", "pd", "dd"):
        dl.j[ab] = {"first": U(z[f"J_{ab}_first"]), "second": U(z[f"J_{ab}_second"]),
                    "pdata": T(z[f"J_{ab}_pdata"]), "Q": T(z[f"J_{ab}_Q"]), "D": T(z[f"J_{ab}_D"])}
    for a in "spd":
        for b in "spd":
            dl.kpart[a + b] = {"displs": U(z[f"K_{a}{b}_displs"]), "counts": U(z[f"K_{a}{b}_counts"]),
                               "Dinds": U(z[f"K_{a}{b}_Dinds"]), "Q": T(z[f"K_{a}{b}_Q"]),
                               "pdata": T(z[f"K_{a}{b}_pdata"])}
    for i, a in enumerate("spd"):
        for c in "spd"[i:]:
            dl.kpair[a + c] = {"i": U(z[f"K_{a}{c}_pair_i"]), "k": U(z[f"K_{a}{c}_pair_k"])}
    for cls in tf.k_classes():
        dl.maxD[cls[1] + cls[3]] = float(z[f"K_{cls}_maxD"][0])
    return dl


@pytest.fixture(scope="module")
def golden():
    lib().init(0)
    return tf.load()


@pytest.mark.parametrize("tag", ["t12", "t3"])
def test_golden_all_coulomb_classes(golden, tag):
    z = golden
    dl = fixture_lists(z, tf.THRESHOLDS[tag])
    s = torch.cuda.current_stream().cuda_stream
    bad = []
    for cls in tf.j_classes():
        out = torch.zeros(dl.j[cls[:2]]["first"].numel(), dtype=torch.float64, device="cuda")
        lib().coulomb(cls, fock.coulomb_args(dl, cls, out, s))
        got = out.cpu().numpy()
        if not close(got, z[f"J_{cls}_{tag}"]):
            bad.append((cls, float(np.abs(got - z[f"J_{cls}_{tag}"]).max())))
    assert not bad, bad


@pytest.mark.parametrize("variant", tf.K_VARIANTS, ids=[v[0] for v in tf.K_VARIANTS])
def test_golden_all_exchange_classes(golden, variant):
    z = golden
    tag, thr, omega, nrow = variant
    dl = fixture_lists(z, thr)
    s = torch.cuda.current_stream().cuda_stream
    bad = []
    for cls in tf.k_classes():
        ac = cls[0] + cls[2]
        out = torch.zeros(dl.kpair[ac]["i"].numel(), dtype=torch.float64, device="cuda")
        lib().exchange(cls, fock.exchange_args(dl, cls, out, s, omega))
        got = out.cpu().numpy()
        exp = z[f"K_{cls}_{tag}"]
        if nrow is not None:
            got = got[:len(exp)]
        if not close(got, exp):
            bad.append((cls, float(np.abs(got - exp).max())))
    assert not bad, bad


def small_system(recipe, natoms, side, degree=2, alpha0=0.3, ratio=2.5, nocc=4, thr=1e-12, seed=11):
    wl = basis.config_custom(natoms, side, recipe, degree, alpha0, ratio, nocc, thr, seed)
    rl = lists.build_lists(wl.mol, wl.D, thr, fock.gpu_schwarz_fn())
    return wl, rl


def test_gpu_schwarz_matches_oracle():
    lib().init(0)
    wl = basis.config_custom(2, 3.0, {0: 1, 1: 1, 2: 1}, 2, 0.4, 2.3, 3, 1e-12, 5)
    pd = lists.prim_data(wl.mol)
    g = fock.gpu_schwarz_fn()
    for la in range(3):
        for lb in range(la, 3):
            sp_g = lists.all_shell_pairs(pd, la, lb, g)
            sp_o = lists.all_shell_pairs(pd, la, lb, helpers.oracle_schwarz_fn)
            assert np.allclose(sp_g.q, sp_o.q, rtol=1e-12, atol=1e-300)


def test_spd_molecule_full_vs_oracle():
    """Two atoms with s, p and d shells: every J/K class vs the oracle, AO J/K
    and the energy Tr[D(J - K/2)]."""
    lib().init(0)
    wl, rl = small_system({0: 1, 1: 1, 2: 1}, 2, 3.0)
    dl = fock.to_device(rl)
    matJ, matK = fock.build_jk(dl)
    torch.cuda.synchronize()
    oJ, oK = helpers.oracle_jk_all(rl)
    for k in oJ:
        assert close(matJ[k].cpu().numpy(), oJ[k]), k
    for k in oK:
        assert close(matK[k].cpu().numpy(), oK[k]), k
    J = lists.contract_J(rl, {k: v.cpu().numpy() for k, v in matJ.items()})
    K = lists.contract_K(rl, {k: v.cpu().numpy() for k, v in matK.items()})
    Jo, Ko = lists.contract_J(rl, oJ), lists.contract_K(rl, oK)
    assert np.abs(J - Jo).max() <= 1e-10 * np.abs(Jo).max()
    assert np.abs(K - Ko).max() <= 1e-10 * np.abs(Ko).max()
    assert abs(lists.energy(wl.D, J, K) - lists.energy(wl.D, Jo, Ko)) < 1e-10


def test_range_separated_exchange_vs_oracle():
    lib().init(0)
    wl, rl = small_system({0: 1, 1: 1, 2: 1}, 2, 3.0, seed=13)
    dl = fock.to_device(rl)
    _, matK = fock.build_jk(dl, omega=0.33, do_j=False)
    torch.cuda.synchronize()
    _, oK = helpers.oracle_jk_all(rl, omega=0.33)
    for k in oK:
        assert close(matK[k].cpu().numpy(), oK[k]), k


def test_small_sp_workload_full_vs_oracle():
    """The 5-atom 3s+2p workload (45 Cartesian AOs) in full: every entry of
    every J and K list, the AO J and K and the energy against the FP64 oracle,
    at an absolute bar of 1e-10 (the FP64 bar) besides the relative one."""
    lib().init(0)
    wl = basis.config_small(0)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    matJ, matK = fock.build_jk(dl)
    torch.cuda.synchronize()
    oJ, oK = helpers.oracle_jk_all(rl)
    gJ = {k: v.cpu().numpy() for k, v in matJ.items()}
    gK = {k: v.cpu().numpy() for k, v in matK.items()}
    for k in oJ:
        assert close(gJ[k], oJ[k]), k
        assert float(np.abs(gJ[k] - oJ[k]).max()) <= 1e-10, k
    for k in oK:
        assert close(gK[k], oK[k]), k
        assert float(np.abs(gK[k] - oK[k]).max()) <= 1e-10, k
    J, K = lists.contract_J(rl, gJ), lists.contract_K(rl, gK)
    Jo, Ko = lists.contract_J(rl, oJ), lists.contract_K(rl, oK)
    assert np.abs(J - Jo).max() <= 1e-10
    assert np.abs(K - Ko).max() <= 1e-10
    assert abs(lists.energy(wl.D, J, K) - lists.energy(wl.D, Jo, Ko)) <= 1e-10


def test_bitwise_reproducible():
    lib().init(0)
    wl, rl = small_system({0: 2, 1: 1, 2: 1}, 3, 4.0, seed=17)
    dl = fock.to_device(rl)
    runs = []
    for _ in range(2):
        matJ, matK = fock.build_jk(dl)
        torch.cuda.synchronize()
        runs.append(({k: v.cpu().numpy() for k, v in matJ.items()}, {k: v.cpu().numpy() for k, v in matK.items()}))
    for k in runs[0][0]:
        assert np.array_equal(runs[0][0][k], runs[1][0][k]), k
    for k in runs[0][1]:
        assert np.array_equal(runs[0][1][k], runs[1][1][k]), k


def test_quartet_counters_count_screened_work():
    lib().init(0)
    wl, rl = small_system({0: 1, 1: 1}, 3, 4.0, seed=19)
    dl = fock.to_device(rl)
    L = lib()
    L.reset_counters()
    fock.build_jk(dl)
    c1 = L.quartet_counters(reset=True)
    fock.build_jk(dl)
    c2 = L.quartet_counters(reset=True)
    assert c1 == c2 and c1[0] > 0 and c1[1] > 0


def test_edge_cases_empty_and_invalid():
    lib().init(0)
    z = tf.load()
    dl = fixture_lists(z, 1e-12)
    s = torch.cuda.current_stream().cuda_stream
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    A = fock.coulomb_args(dl, "ssss", out, s)
    A["ss_prim_pair_count_local"] = 0  # empty bra list: nothing to do
    lib().coulomb("ssss", A)
    A = fock.coulomb_args(dl, "ssss", out, s)
    A["ss_prim_pair_count"] = 0  # empty ket list: J unchanged
    lib().coulomb("ssss", A)
    torch.cuda.synchronize()
    assert float(out.abs().max()) == 0.0
    # null pointer with a non-zero count is rejected before any launch
    A = fock.coulomb_args(dl, "ssss", out, s)
    A["ss_mat_D"] = None
    rc = getattr(lib().cdll, "vlxb_computeCoulombFockSSSS")(*[A[n] for n in lib().j_params["ssss"]])
    assert rc == 1
    # a threshold above every bound screens everything out
    out2 = torch.zeros(dl.j["ss"]["first"].numel(), dtype=torch.float64, device="cuda")
    A = fock.coulomb_args(dl, "ssss", out2, s)
    A["eri_threshold"] = 1e30
    lib().coulomb("ssss", A)
    torch.cuda.synchronize()
    assert float(out2.abs().max()) == 0.0


def test_tma_staged_coulomb_matches_thread_kernel():
    """J variant 3 (the ket stream staged into shared memory by TMA bulk
    copies) against variant 0 on ket lists of several tiles, in FP64 and with
    an FP32 pass (whose ket ranges start at odd positions, so the copies start
    one ket early): same J to rounding, the same quartet counts, and no
    bounded wait ran out."""
    L = lib()
    L.init(0)
    wl = basis.config_custom(4, 5.0, {0: 2, 1: 2, 2: 1}, 3, 0.1, 2.5, 4, 1e-12, 37)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    assert max(len(v.first) for v in rl.jlists.values()) > 4 * 128
    dl = fock.to_device(rl)
    saved = {c: L.get_schedule("J", c) for c in lists.j_classes()}
    budget = L.get_fp32_budget()
    L.kernel_errors(reset=True)
    try:
        L.set_fp32_budget(0.0)
        for cut in (0.0, 1e-6):
            res = {}
            for v in (0, 3):
                for c in lists.j_classes():
                    L.set_schedule("J", c, v)
                L.set_fp32_cut(cut)
                L.reset_counters()
                mJ, _ = fock.build_jk(dl, do_k=False)
                torch.cuda.synchronize()
                res[v] = ({k: t.cpu().numpy() for k, t in mJ.items()}, L.quartet_counters(reset=True)[0])
            for k in res[0][0]:
                assert close(res[3][0][k], res[0][0][k]), (cut, k)
            assert res[3][1] == res[0][1]
    finally:
        L.set_fp32_cut(0.0)
        L.set_fp32_budget(budget)
        for c, v in saved.items():
            L.set_schedule("J", c, v)
    assert L.kernel_errors() == 0


def _k_variants(cls):
    """Exchange variants compiled for a class (column ones only when their
    shared memory fits; the library falls back to the thread kernel)."""
    import sys as _s
    import os as _o
    _s.path.insert(0, _o.path.join(_o.path.dirname(_o.path.dirname(_o.path.abspath(__file__))),
                                   "vlx-twoe-ints_b200", "csrc"))
    from gen_column import k_variants

    l = [{"s": 0, "p": 1, "d": 2}[x] for x in cls]
    return k_variants(*l)


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
def test_golden_every_coulomb_variant(golden, variant):
    """Every Coulomb kernel (thread per quartet, warp column, McMurchie-Davidson,
    thread per quartet with TMA-staged kets) on every class."""
    z = golden
    L = lib()
    saved = {c: L.get_schedule("J", c) for c in tf.j_classes()}
    try:
        for c in tf.j_classes():
            L.set_schedule("J", c, variant)
        for tag in ("t12", "t3"):
            dl = fixture_lists(z, tf.THRESHOLDS[tag])
            s = torch.cuda.current_stream().cuda_stream
            bad = []
            for cls in tf.j_classes():
                out = torch.zeros(dl.j[cls[:2]]["first"].numel(), dtype=torch.float64, device="cuda")
                L.coulomb(cls, fock.coulomb_args(dl, cls, out, s))
                if not close(out.cpu().numpy(), z[f"J_{cls}_{tag}"]):
                    bad.append(cls)
            assert not bad, (variant, tag, bad)
    finally:
        for c, v in saved.items():
            L.set_schedule("J", c, v)


@pytest.mark.parametrize("variant", list(range(13)))
def test_golden_every_exchange_variant(golden, variant):
    """All exchange kernels (thread per quartet; column with bra or ket lanes;
    the same with contracted partners; packed column plans, also on the
    pair's second centre, with and without contracted partners) on every
    class where the variant is compiled."""
    z = golden
    L = lib()
    saved = {c: L.get_schedule("K", c) for c in tf.k_classes()}
    try:
        for c in tf.k_classes():
            L.set_schedule("K", c, variant if variant in _k_variants(c) else 0)
        for tag, thr, omega, nrow in tf.K_VARIANTS:
            dl = fixture_lists(z, thr)
            s = torch.cuda.current_stream().cuda_stream
            bad = []
            for cls in tf.k_classes():
                ac = cls[0] + cls[2]
                out = torch.zeros(dl.kpair[ac]["i"].numel(), dtype=torch.float64, device="cuda")
                L.exchange(cls, fock.exchange_args(dl, cls, out, s, omega))
                got = out.cpu().numpy()
                exp = z[f"K_{cls}_{tag}"]
                if nrow is not None:
                    got = got[:len(exp)]
                if not close(got, exp):
                    bad.append(cls)
            assert not bad, (variant, tag, bad)
    finally:
        for c, v in saved.items():
            L.set_schedule("K", c, v)


def test_mixed_precision_errors_within_tolerance():
    """FP32 below a Schwarz bound of 1e-6, FP64 above and for all accumulation:
    AO J and K within 1e-7 and E within 1e-6 Eh of the FP64 oracle."""
    lib().init(0)
    wl, rl = small_system({0: 2, 1: 1, 2: 1}, 3, 4.0, seed=29)
    dl = fock.to_device(rl)
    L = lib()
    try:
        L.set_fp32_cut(1e-6)
        matJ, matK = fock.build_jk(dl)
        torch.cuda.synchronize()
    finally:
        L.set_fp32_cut(0.0)
    oJ, oK = helpers.oracle_jk_all(rl)
    J = lists.contract_J(rl, {k: v.cpu().numpy() for k, v in matJ.items()})
    K = lists.contract_K(rl, {k: v.cpu().numpy() for k, v in matK.items()})
    Jo, Ko = lists.contract_J(rl, oJ), lists.contract_K(rl, oK)
    assert np.abs(J - Jo).max() <= 1e-7
    assert np.abs(K - Ko).max() <= 1e-7
    assert abs(lists.energy(wl.D, J, K) - lists.energy(wl.D, Jo, Ko)) <= 1e-6
    # a cutoff above every bound runs everything in FP32: still close, not exact
    try:
        L.set_fp32_cut(1e30)
        mJ, mK = fock.build_jk(dl)
        torch.cuda.synchronize()
    finally:
        L.set_fp32_cut(0.0)
    J2 = lists.contract_J(rl, {k: v.cpu().numpy() for k, v in mJ.items()})
    assert np.abs(J2 - Jo).max() <= 1e-4 * np.abs(Jo).max()


def test_fp32_budget_bounds_the_fp32_work():
    """The FP32 error budget on top of the cutoff: with every quartet below the
    cutoff, a vanishing budget leaves no quartet with a non-zero bound in FP32
    (the FP64 build, bit for bit), an unlimited one runs the whole tail in
    FP32 (different from FP64, still close), and every kernel variant of the
    classes honours it."""
    L = lib()
    L.init(0)
    wl, rl = small_system({0: 2, 1: 1, 2: 1}, 3, 4.0, seed=29)
    dl = fock.to_device(rl)
    L.set_fp32_cut(0.0)
    rJ, rK = fock.build_jk(dl)
    torch.cuda.synchronize()
    ref = ({k: v.cpu().numpy() for k, v in rJ.items()}, {k: v.cpu().numpy() for k, v in rK.items()})
    saved = L.get_fp32_budget()
    out = {}
    try:
        L.set_fp32_cut(1e30)
        for b in (1e-300, 0.0):  # 0 = no budget: the cutoff alone decides
            L.set_fp32_budget(b)
            mJ, mK = fock.build_jk(dl)
            torch.cuda.synchronize()
            out[b] = ({k: v.cpu().numpy() for k, v in mJ.items()}, {k: v.cpu().numpy() for k, v in mK.items()})
    finally:
        L.set_fp32_cut(0.0)
        L.set_fp32_budget(saved)
    for t in (0, 1):
        for k in ref[t]:
            assert np.array_equal(out[1e-300][t][k], ref[t][k]), (t, k)
    diff = max(float(np.abs(out[0.0][t][k] - ref[t][k]).max()) for t in (0, 1) for k in ref[t])
    scale = max(float(np.abs(ref[t][k]).max()) for t in (0, 1) for k in ref[t])
    assert 0.0 < diff <= 1e-4 * scale


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 9, 10, 11, 12])
def test_contracted_exchange_variants_vs_oracle(variant):
    """Degree-3 contracted s/p/d shells (partner groups of up to 3 primitives
    with one S per record): every exchange class through one kernel variant
    against the FP64 oracle, also with range separation, and the quartet
    counter equal to the record-by-record variant's."""
    L = lib()
    L.init(0)
    wl = basis.config_custom(3, 4.0, {0: 2, 1: 1, 2: 1}, 3, 0.2, 2.5, 3, 1e-12, 17)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    saved = {c: L.get_schedule("K", c) for c in lists.k_classes()}
    try:
        for omega in (0.0, 0.4):
            counts = {}
            for v in (1, variant) if variant != 1 else (1,):
                for c in lists.k_classes():
                    L.set_schedule("K", c, v if v in _k_variants(c) else 0)
                L.reset_counters()
                _, mK = fock.build_jk(dl, omega=omega, do_j=False)
                torch.cuda.synchronize()
                counts[v] = L.quartet_counters()[1]
            K = lists.contract_K(rl, {k: t.cpu().numpy() for k, t in mK.items()})
            _, oK = helpers.oracle_jk_all(rl, omega=omega)
            Ko = lists.contract_K(rl, oK)
            assert np.abs(K - Ko).max() <= 1e-10 * max(1.0, np.abs(Ko).max()), (variant, omega)
            assert counts[variant] == counts[1], counts
    finally:
        for c, v in saved.items():
            L.set_schedule("K", c, v)


def test_md_coulomb_vs_oracle_and_counts():
    """The McMurchie-Davidson Coulomb kernel (variant 2) on every class of a
    degree-3 s/p/d system: AO J within 1e-10 of the FP64 oracle, quartet
    counts equal to the thread kernel's, and its FP32 pass within the mixed
    tolerance of its FP64 result."""
    L = lib()
    L.init(0)
    wl = basis.config_custom(3, 4.0, {0: 2, 1: 1, 2: 1}, 3, 0.2, 2.5, 3, 1e-12, 23)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    saved = {c: L.get_schedule("J", c) for c in lists.j_classes()}
    try:
        res = {}
        for v in (0, 2):
            for c in lists.j_classes():
                L.set_schedule("J", c, v)
            L.reset_counters()
            mJ, _ = fock.build_jk(dl, do_k=False)
            torch.cuda.synchronize()
            res[v] = (lists.contract_J(rl, {k: t.cpu().numpy() for k, t in mJ.items()}), L.quartet_counters()[0])
        oJ, _ = helpers.oracle_jk_all(rl)
        Jo = lists.contract_J(rl, oJ)
        assert np.abs(res[2][0] - Jo).max() <= 1e-10 * max(1.0, np.abs(Jo).max())
        assert res[2][1] == res[0][1]
        L.set_fp32_cut(1e-6)
        mJ, _ = fock.build_jk(dl, do_k=False)
        torch.cuda.synchronize()
        L.set_fp32_cut(0.0)
        J32 = lists.contract_J(rl, {k: t.cpu().numpy() for k, t in mJ.items()})
        assert np.abs(J32 - res[2][0]).max() <= 1e-7
    finally:
        L.set_fp32_cut(0.0)
        for c, v in saved.items():
            L.set_schedule("J", c, v)
