"""Pins the CPU oracle against golden vectors generated from the reference.

eri_components.npz: the reference generator's emitted per-component ERI
expressions (eriwriter.py:35-160) evaluated for all 81 s/p/d classes, with and
without range separation.  jk_tiny.npz: mat_J / mat_K of every J (36) and K (54)
class of a two-atom s/p/d system, computed with the emitted kernels' loop
semantics (gen_coulomb.py:205-297, gen_exchange.py:139-342).
eri_grad_components.npz: the generator's derivative expressions
(gradient='a'..'d', eriwriter.py:72-86) for every s/p/d class.
eri_f_components.npz: twelve classes with f centres from the same engine.
"""
import numpy as np
import pytest

from oracle import oracle
import tiny_fixture as tf

LV = {"s": 0, "p": 1, "d": 2, "f": 3}


def test_boys_against_mpmath():
    for T in [0.0, 1e-10, 0.025, 0.7, 3.3, 11.9, 24.0, 35.99, 36.0, 50.0, 160.0]:
        F = oracle.boys(16, T)
        G = oracle.boys_mpmath(16, T)
        for m in range(17):
            assert abs(F[m] - float(G[m])) <= 1e-15 * float(G[m]), (T, m)


def test_components_all_classes():
    z = np.load(f"{tf.HERE}/golden/eri_components.npz")
    worst = 0.0
    for a in "spd":
        for b in "spd":
            for c in "spd":
                for d in "spd":
                    cls = a + b + c + d
                    for tag in ("w0", "w4"):
                        ex = z[f"{cls}_{tag}_exps"]
                        R = z[f"{cls}_{tag}_centers"]
                        w = float(z[f"{cls}_{tag}_omega"][0])
                        v = oracle.eri_shell_quartet(LV[a], LV[b], LV[c], LV[d], ex[0], R[0], ex[1], R[1],
                                                     ex[2], R[2], ex[3], R[3], w)
                        g = z[f"{cls}_{tag}_vals"]
                        err = np.abs(v - g).max() / np.abs(g).max()
                        worst = max(worst, err)
    assert worst < 1e-12, worst


def test_gradient_components_all_classes():
    """The oracle's derivative integrals (Obara-Saika derivative relation)
    against the reference generator's own derivative expressions
    (write_eri_code(..., gradient='a'..'d'), eri_grad_components.npz): every
    s/p/d class, one centre each (rotating over a..d), omega 0 and 0.4."""
    z = np.load(f"{tf.HERE}/golden/eri_grad_components.npz")
    worst = 0.0
    seen = set()
    for a in "spd":
        for b in "spd":
            for c in "spd":
                for d in "spd":
                    cls = a + b + c + d
                    ex = z[f"{cls}_exps"]
                    R = z[f"{cls}_centers"]
                    w = float(z[f"{cls}_omega"][0])
                    centre = int(z[f"{cls}_centre"][0])
                    seen.add((centre, w))
                    v = oracle.eri_shell_quartet_grad(LV[a], LV[b], LV[c], LV[d], centre, ex[0], R[0], ex[1], R[1],
                                                      ex[2], R[2], ex[3], R[3], w)
                    g = z[f"{cls}_vals"]
                    err = np.abs(v - g).max() / np.abs(g).max()
                    worst = max(worst, err)
    assert len(seen) == 8  # every centre with both omegas
    assert worst < 1e-12, worst


def test_f_shell_components():
    """Classes with f centres: the oracle against the reference's symbolic
    engine run with three Cartesian indices on those centres
    (eri_f_components.npz; one and two f centres, omega 0 and 0.4)."""
    z = np.load(f"{tf.HERE}/golden/eri_f_components.npz")
    classes = sorted({k.split("_")[0] for k in z.files})
    assert len(classes) == 12
    worst = 0.0
    for cls in classes:
        ex, R, w = z[f"{cls}_exps"], z[f"{cls}_centers"], float(z[f"{cls}_omega"][0])
        v = oracle.eri_shell_quartet(*(LV[x] for x in cls), ex[0], R[0], ex[1], R[1], ex[2], R[2], ex[3], R[3], w)
        g = z[f"{cls}_vals"]
        worst = max(worst, np.abs(v - g).max() / np.abs(g).max())
    assert worst < 1e-12, worst


def test_closed_form_ssss_and_symmetry():
    A, B, C, D = (np.array(x) for x in ([0.1, 0.2, 0.3], [1.0, -0.5, 0.2], [-0.7, 0.4, 1.1], [0.3, 0.9, -1.2]))
    a, b, c, d = 0.8, 1.3, 0.5, 2.1
    v = oracle.eri_shell_quartet(0, 0, 0, 0, a, A, b, B, c, C, d, D)[0, 0, 0, 0]
    p, q = a + b, c + d
    P, Q = (a * A + b * B) / p, (c * C + d * D) / q
    T = p * q / (p + q) * np.sum((P - Q) ** 2)
    F0 = oracle.boys(0, T)[0]
    # Lambda * F0 with Lambda = 2 sqrt(rho/pi) (gen_coulomb.py:255)
    assert abs(v - 2.0 * np.sqrt(p * q / (p + q) / np.pi) * F0) < 1e-15
    I = oracle.eri_shell_quartet(1, 2, 2, 1, a, A, b, B, c, C, d, D)
    I2 = oracle.eri_shell_quartet(2, 1, 1, 2, c, C, d, D, a, A, b, B)
    assert np.abs(I - I2.transpose(2, 3, 0, 1)).max() < 1e-14
    I3 = oracle.eri_shell_quartet(2, 1, 2, 1, b, B, a, A, c, C, d, D)
    assert np.abs(I - I3.transpose(1, 0, 2, 3)).max() < 1e-14


@pytest.mark.parametrize("cls", tf.j_classes())
def test_oracle_J_tiny(cls):
    z = tf.load()
    info, _, count = tf.prim_tables(z)
    args = tf.j_args(z, cls)
    la, lb, lc, ld = (LV[x] for x in cls)
    for tag, thr in tf.THRESHOLDS.items():
        J = oracle.coulomb_fock(la, lb, lc, ld, info, count, args["cd_D"], args["ab_Q"], args["cd_Q"],
                                args["ab_first"], args["ab_second"], args["ab_pdata"], args["cd_first"],
                                args["cd_second"], args["cd_pdata"], thr)
        g = z[f"J_{cls}_{tag}"]
        scale = max(np.abs(g).max(), 1e-30)
        assert np.abs(J - g).max() <= 1e-12 * scale + 1e-16, (cls, tag)


@pytest.mark.parametrize("cls", tf.k_classes())
def test_oracle_K_tiny(cls):
    z = tf.load()
    info, aoinds, count = tf.prim_tables(z)
    args = tf.k_args(z, cls)
    la, lb, lc, ld = (LV[x] for x in cls)
    for tag, thr, omega, nrow in tf.K_VARIANTS:
        rows = None if nrow is None else np.arange(min(nrow, len(args["pair_i"])))
        K = oracle.exchange_fock(la, lb, lc, ld, args["pair_i"], args["pair_k"], info, aoinds, count,
                                 args["maxD"], args["D_AO"], args["Q_ab"], args["Q_cd"], args["Dinds_ab"],
                                 args["Dinds_cd"], args["displs_ab"], args["displs_cd"], args["counts_ab"],
                                 args["counts_cd"], args["pdata_ab"], args["pdata_cd"], omega, thr, rows=rows)
        g = z[f"K_{cls}_{tag}"]
        if rows is not None:
            K = K[rows]
        scale = max(np.abs(g).max(), 1e-30)
        assert np.abs(K - g).max() <= 1e-12 * scale + 1e-16, (cls, tag)
