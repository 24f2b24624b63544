"""Shared test helpers: oracle-backed Schwarz values and oracle J/K over
reference-format lists (the oracle is the checker; see oracle/__init__.py)."""
from __future__ import annotations

import numpy as np

from oracle import oracle
from vlxb.lists import ANG, LV, ReferenceLists


def oracle_schwarz_fn(la, lb, pd, P, Q):
    out = np.zeros(len(P))
    ia, ib = pd.info[la], pd.info[lb]
    for t, (p, q) in enumerate(zip(P, Q)):
        A, B = ia[2:5, p], ib[2:5, q]
        I = oracle.eri_shell_quartet(la, lb, la, lb, ia[0, p], A, ib[0, q], B, ia[0, p], A, ib[0, q], B)
        n = I.shape[0] * I.shape[1]
        out[t] = np.sqrt(np.abs(np.diag(I.reshape(n, n))).max())
    return out


def oracle_J(rl: ReferenceLists, cls: str, rows=None):
    a, b, c, d = cls
    jab, jcd = rl.jlists[a + b], rl.jlists[c + d]
    return oracle.coulomb_fock(LV[a], LV[b], LV[c], LV[d], rl.pd.info, rl.pd.count, jcd.D, jab.Q, jcd.Q,
                               jab.first, jab.second, jab.pdata, jcd.first, jcd.second, jcd.pdata,
                               rl.threshold, rows=rows)


def oracle_K(rl: ReferenceLists, cls: str, omega=0.0, rows=None):
    a, b, c, d = cls
    kq = rl.kpairs[a + c]
    p1, p2 = rl.kpartners[a + b], rl.kpartners[c + d]
    return oracle.exchange_fock(LV[a], LV[b], LV[c], LV[d], kq.pair_i, kq.pair_k, rl.pd.info, rl.pd.aoinds,
                                rl.pd.count, rl.maxD[b + d], rl.D_AO, p1.Q, p2.Q, p1.Dinds, p2.Dinds, p1.displs,
                                p2.displs, p1.counts, p2.counts, p1.pdata, p2.pdata, omega, rl.threshold,
                                rows=rows)


def oracle_jk_all(rl: ReferenceLists, omega=0.0):
    from vlxb.lists import j_classes_all as j_classes, k_classes_all as k_classes

    matJ = {k: np.zeros(len(v.first)) for k, v in rl.jlists.items()}
    matK = {k: np.zeros(len(v.pair_i)) for k, v in rl.kpairs.items()}
    for cls in j_classes():
        if cls[:2] in rl.jlists and cls[2:] in rl.jlists:
            matJ[cls[:2]] += oracle_J(rl, cls)
    for cls in k_classes():
        if cls[0] + cls[2] in rl.kpairs and cls[:2] in rl.kpartners and cls[2:] in rl.kpartners:
            matK[cls[0] + cls[2]] += oracle_K(rl, cls, omega)
    return matJ, matK


def bra_weights(rl: ReferenceLists, key: str) -> np.ndarray:
    """w_o D_o of the entries of J list `key` (w_o = 1 on the diagonal of a
    same-type list, else 2), so that 1/2 Tr[D J] = 1/2 sum_o w_o D_o mat_J[o]."""
    jl = rl.jlists[key]
    same = key[0] == key[1]
    return np.where(same & (jl.first == jl.second), 1.0, 2.0) * jl.D


def oracle_coulomb_energy(rl: ReferenceLists) -> float:
    """E_J = 1/2 Tr[D J] from the oracle J of every class."""
    from vlxb.lists import j_classes

    E = 0.0
    for cls in j_classes():
        if cls[:2] in rl.jlists and cls[2:] in rl.jlists:
            E += 0.5 * float(np.dot(bra_weights(rl, cls[:2]), oracle_J(rl, cls)))
    return E


def oracle_grad_class(rl: ReferenceLists, cls: str, grad=None):
    a, b, c, d = cls
    jab, jcd = rl.jlists[a + b], rl.jlists[c + d]
    return oracle.coulomb_grad(LV[a], LV[b], LV[c], LV[d], rl.pd.info, rl.pd.count, jcd.D, jab.Q, jcd.Q,
                               jab.first, jab.second, jab.pdata, jcd.first, jcd.second, jcd.pdata,
                               rl.threshold, grad=grad)


def oracle_coulomb_gradient(rl: ReferenceLists, natoms: int):
    """dE_J/dR (natoms x 3) from the oracle's bra-centre derivatives of every
    class, and the per-list derivative arrays (6, n) it was folded from."""
    from vlxb.lists import NCART, j_classes

    grads = {k: np.zeros((6, len(v.first))) for k, v in rl.jlists.items()}
    for cls in j_classes():
        if cls[:2] in rl.jlists and cls[2:] in rl.jlists:
            oracle_grad_class(rl, cls, grad=grads[cls[:2]])
    g = np.zeros((natoms, 3))
    for k, G in grads.items():
        jl = rl.jlists[k]
        la, lb = LV[k[0]], LV[k[1]]
        w = bra_weights(rl, k)
        np.add.at(g, rl.pd.atom[la][jl.first // NCART[la]], (w * G[:3]).T)
        np.add.at(g, rl.pd.atom[lb][jl.second // NCART[lb]], (w * G[3:]).T)
    return g, grads


def k_weights(rl: ReferenceLists, key: str) -> np.ndarray:
    """w_ik D_ik of the entries of K (i, k) list `key`, so that
    1/2 Tr[D K] = 1/2 sum_ik w_ik D_ik mat_K[ik]."""
    from vlxb.lists import NCART

    kp = rl.kpairs[key]
    la, lc = LV[key[0]], LV[key[1]]
    ai = rl.pd.aoinds[la][kp.pair_i % NCART[la], kp.pair_i // NCART[la]]
    ck = rl.pd.aoinds[lc][kp.pair_k % NCART[lc], kp.pair_k // NCART[lc]]
    w = np.where((la == lc) & (kp.pair_i == kp.pair_k), 1.0, 2.0)
    return w * rl.D_AO[ai, ck]


def oracle_exchange_energy(rl: ReferenceLists, omega=0.0) -> float:
    """E_K = 1/2 Tr[D K] from the oracle K of every class."""
    from vlxb.lists import k_classes

    E = 0.0
    for cls in k_classes():
        ac = cls[0] + cls[2]
        if ac in rl.kpairs and cls[:2] in rl.kpartners and cls[2:] in rl.kpartners:
            E += 0.5 * float(np.dot(k_weights(rl, ac), oracle_K(rl, cls, omega)))
    return E


def oracle_kgrad_class(rl: ReferenceLists, cls: str, omega=0.0, grad=None):
    a, b, c, d = cls
    kq = rl.kpairs[a + c]
    p1, p2 = rl.kpartners[a + b], rl.kpartners[c + d]
    return oracle.exchange_grad(LV[a], LV[b], LV[c], LV[d], kq.pair_i, kq.pair_k, rl.pd.info, rl.pd.aoinds,
                                rl.pd.count, rl.maxD[b + d], rl.D_AO, p1.Q, p2.Q, p1.Dinds, p2.Dinds, p1.displs,
                                p2.displs, p1.counts, p2.counts, p1.pdata, p2.pdata, omega, rl.threshold, grad=grad)


def oracle_exchange_gradient(rl: ReferenceLists, natoms: int, omega=0.0):
    """dE_K/dR (natoms x 3) for E_K = 1/2 Tr[D K], and the per-list (6, n_ik)
    arrays of per-entry values it was folded from."""
    from vlxb.lists import NCART, k_classes

    grads = {k: np.zeros((6, len(v.pair_i))) for k, v in rl.kpairs.items()}
    for cls in k_classes():
        ac = cls[0] + cls[2]
        if ac in rl.kpairs and cls[:2] in rl.kpartners and cls[2:] in rl.kpartners:
            oracle_kgrad_class(rl, cls, omega, grad=grads[ac])
    g = np.zeros((natoms, 3))
    for k, G in grads.items():
        kp = rl.kpairs[k]
        la, lc = LV[k[0]], LV[k[1]]
        np.add.at(g, rl.pd.atom[la][kp.pair_i // NCART[la]], G[:3].T)
        np.add.at(g, rl.pd.atom[lc][kp.pair_k // NCART[lc]], G[3:].T)
    return g, grads


def kgrad_blocks(rl: ReferenceLists, key: str, G: np.ndarray) -> np.ndarray:
    """Per-entry K-gradient values summed onto each primitive shell block's
    lowest list position (the layout of vlxb_computeExchangeGradient)."""
    from vlxb.lists import NCART

    kp = rl.kpairs[key]
    la, lc = LV[key[0]], LV[key[1]]
    blk = (kp.pair_i // NCART[la]).astype(np.int64) * (1 << 32) + kp.pair_k // NCART[lc]
    out = np.zeros_like(G)
    first = {}
    for p, bk in enumerate(blk):
        q = first.setdefault(int(bk), p)
        out[:, q] += G[:, p]
    return out


def ao_eri_tensor(mol):
    """Full contracted Cartesian AO ERI tensor from the oracle (tiny systems only)."""
    from vlxb.basis import NCART

    n = mol.naos
    G = np.zeros((n, n, n, n))
    sh = mol.shells
    for A in sh:
        for B in sh:
            for C in sh:
                for D in sh:
                    blk = np.zeros((NCART[A.l], NCART[B.l], NCART[C.l], NCART[D.l]))
                    for ea, ca in zip(A.exps, A.coefs):
                        for eb, cb in zip(B.exps, B.coefs):
                            for ec, cc in zip(C.exps, C.coefs):
                                for ed, cd in zip(D.exps, D.coefs):
                                    RA, RB = mol.coords[A.atom], mol.coords[B.atom]
                                    RC, RD = mol.coords[C.atom], mol.coords[D.atom]
                                    p, q = ea + eb, ec + ed
                                    Sab = ca * cb * (np.pi / p) ** 1.5 * np.exp(-ea * eb / p * np.sum((RA - RB) ** 2))
                                    Scd = cc * cd * (np.pi / q) ** 1.5 * np.exp(-ec * ed / q * np.sum((RC - RD) ** 2))
                                    blk += Sab * Scd * oracle.eri_shell_quartet(A.l, B.l, C.l, D.l, ea, RA, eb, RB,
                                                                                ec, RC, ed, RD)
                    G[A.ao0:A.ao0 + NCART[A.l], B.ao0:B.ao0 + NCART[B.l], C.ao0:C.ao0 + NCART[C.l],
                      D.ao0:D.ao0 + NCART[D.l]] = blk
    return G
