"""Reference-format input lists for the J/K entry points.

Builds, from a Molecule and an AO density, exactly the arrays that the
reference's emitted kernels take (gen_coulomb.py:74-93, gen_exchange.py:75-115):

  prim_info[l]   (5, count)     row 0 exponent, row 1 coefficient, rows 2..4 centre
  prim_aoinds[l] (ncart, count) Cartesian AO index of (primitive, component)
  J lists per type pair a <= b: first/second prim-cart indices (i <= j when
     a == b), pair_data S_ij_00, Schwarz Q_ij, density D_ij = D_AO[ao(i), ao(j)];
     sorted by descending |Q D| as the emitted kernels' break requires
     (gen_coulomb.py:209-212)
  K partner lists per ordered type pair (a, b): CSR over prim-cart i of type a
     (displs, counts) of partners j (D_inds) sorted by descending Q_ij, with
     Q and pair_data (gen_exchange.py:161-251)
  K (i, k) lists per a <= c (i <= k when a == c)

S_ij_00 = c_i c_j (pi/p)^(3/2) exp(-a_i a_j/p |A-B|^2) (the per-pair factor of
gen_coulomb.py:255,270).  Q is the shell-pair Schwarz bound: |S_ij_00| times
sqrt of the largest diagonal bare integral over the pair's components, shared
by all components of the pair.  Pairs that cannot pass the threshold against
the largest bound of the system are dropped.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .basis import NCART, Molecule

ANG = "spdf"   # letters by angular momentum (s, p, d and f)
SPD = "spd"    # the classes the reference emits
LV = {"s": 0, "p": 1, "d": 2, "f": 3}
LMAX = 3


@dataclass
class PrimData:
    info: dict
    aoinds: dict
    count: dict
    atom: dict


def prim_data(mol: Molecule) -> PrimData:
    rows = {l: [] for l in range(LMAX + 1)}
    for sh in mol.shells:
        R = mol.coords[sh.atom]
        for e, c in zip(sh.exps, sh.coefs):
            rows[sh.l].append((e, c, R[0], R[1], R[2], sh.ao0, sh.atom))
    info, aoinds, count, atom = {}, {}, {}, {}
    for l in range(LMAX + 1):
        r = rows[l]
        n = len(r)
        inf = np.zeros((5, max(n, 0)))
        aoi = np.zeros((NCART[l], n), dtype=np.uint32)
        at = np.zeros(n, dtype=np.int64)
        for p, (e, c, x, y, z, ao0, a) in enumerate(r):
            inf[:, p] = (e, c, x, y, z)
            aoi[:, p] = ao0 + np.arange(NCART[l])
            at[p] = a
        info[l], aoinds[l], count[l], atom[l] = inf, aoi, n, at
    return PrimData(info, aoinds, count, atom)


def pair_prefactor(pd: PrimData, la: int, lb: int, P: np.ndarray, Q: np.ndarray) -> np.ndarray:
    ia, ib = pd.info[la], pd.info[lb]
    a, b = ia[0, P], ib[0, Q]
    p = a + b
    R2 = np.sum((ia[2:5, P] - ib[2:5, Q]) ** 2, axis=0)
    return ia[1, P] * ib[1, Q] * (math.pi / p) ** 1.5 * np.exp(-a * b / p * R2)


@dataclass
class ShellPairs:
    la: int
    lb: int
    P: np.ndarray
    Q: np.ndarray
    S: np.ndarray
    q: np.ndarray  # Schwarz bound per shell pair


def all_shell_pairs(pd: PrimData, la: int, lb: int, schwarz_fn) -> ShellPairs:
    """All primitive shell pairs (P, Q) with P <= Q when la == lb."""
    na, nb = pd.count[la], pd.count[lb]
    if la == lb:
        P, Q = np.triu_indices(na)
    else:
        P, Q = np.meshgrid(np.arange(na), np.arange(nb), indexing="ij")
        P, Q = P.ravel(), Q.ravel()
    S = pair_prefactor(pd, la, lb, P, Q)
    bare = schwarz_fn(la, lb, pd, P, Q)  # max over components of sqrt|bare diagonal|
    return ShellPairs(la, lb, P, Q, S, np.abs(S) * bare)


@dataclass
class JList:
    first: np.ndarray
    second: np.ndarray
    pdata: np.ndarray
    Q: np.ndarray
    D: np.ndarray


@dataclass
class KPartners:
    displs: np.ndarray
    counts: np.ndarray
    Dinds: np.ndarray
    Q: np.ndarray
    pdata: np.ndarray


@dataclass
class KPairs:
    pair_i: np.ndarray
    pair_k: np.ndarray


@dataclass
class ReferenceLists:
    pd: PrimData
    naos: int
    D_AO: np.ndarray
    threshold: float
    shell_pairs: dict = field(default_factory=dict)  # (la, lb) la <= lb -> ShellPairs
    jlists: dict = field(default_factory=dict)       # "ab" -> JList
    kpartners: dict = field(default_factory=dict)    # "ab" (ordered) -> KPartners
    kpairs: dict = field(default_factory=dict)       # "ac" -> KPairs
    maxD: dict = field(default_factory=dict)         # "bd" -> max |D_AO| over the block


def _expand(sp: ShellPairs, keep: np.ndarray, upper: bool):
    """Shell pairs -> prim-cart pairs (i, j); for same-type pairs with P == Q
    only components ca <= cb (i <= j)."""
    na, nb = NCART[sp.la], NCART[sp.lb]
    P, Q, S, q = sp.P[keep], sp.Q[keep], sp.S[keep], sp.q[keep]
    ca, cb = np.meshgrid(np.arange(na), np.arange(nb), indexing="ij")
    ca, cb = ca.ravel(), cb.ravel()
    i = (P[:, None] * na + ca[None, :]).ravel()
    j = (Q[:, None] * nb + cb[None, :]).ravel()
    Sx = np.repeat(S, na * nb)
    qx = np.repeat(q, na * nb)
    if upper:
        m = i <= j
        i, j, Sx, qx = i[m], j[m], Sx[m], qx[m]
    return i, j, Sx, qx


def build_lists(mol: Molecule, D_AO: np.ndarray, threshold: float, schwarz_fn) -> ReferenceLists:
    pd = prim_data(mol)
    rl = ReferenceLists(pd=pd, naos=mol.naos, D_AO=np.ascontiguousarray(D_AO), threshold=threshold)
    ls = [l for l in range(LMAX + 1) if pd.count[l] > 0]
    for la in ls:
        for lb in ls:
            if la <= lb:
                rl.shell_pairs[(la, lb)] = all_shell_pairs(pd, la, lb, schwarz_fn)
    qmax = max(float(sp.q.max()) for sp in rl.shell_pairs.values() if len(sp.q))
    dmax = float(np.abs(D_AO).max())
    for b in ANG:
        for d in ANG:
            lb, ld = LV[b], LV[d]
            if lb in ls and ld in ls:
                blk = D_AO[np.ix_(pd.aoinds[lb].ravel(), pd.aoinds[ld].ravel())]
                rl.maxD[b + d] = float(np.abs(blk).max())
    aoi = {l: pd.aoinds[l] for l in ls}

    def ao_of(l, idx):
        n = NCART[l]
        return aoi[l][idx % n, idx // n]

    # ---------------- J lists
    for (la, lb), sp in rl.shell_pairs.items():
        keep = sp.q * qmax * dmax > threshold
        i, j, S, q = _expand(sp, keep, upper=(la == lb))
        D = D_AO[ao_of(la, i), ao_of(lb, j)]
        order = np.argsort(-np.abs(q * D), kind="stable")
        key = ANG[la] + ANG[lb]
        rl.jlists[key] = JList(i[order].astype(np.uint32), j[order].astype(np.uint32), S[order].copy(),
                               q[order].copy(), D[order].copy())

    # ---------------- K partner lists (all ordered type pairs)
    for la in ls:
        for lb in ls:
            if la <= lb:
                sp = rl.shell_pairs[(la, lb)]
                P, Q, S, q = sp.P, sp.Q, sp.S, sp.q
                if la == lb:  # add the mirrored pairs P > Q
                    off = P != Q
                    P, Q = np.concatenate([P, Q[off]]), np.concatenate([Q, P[off]])
                    S, q = np.concatenate([S, S[off]]), np.concatenate([q, q[off]])
            else:
                sp = rl.shell_pairs[(lb, la)]
                P, Q, S, q = sp.Q, sp.P, sp.S, sp.q
            keep = q * qmax * dmax > threshold
            tmp = ShellPairs(la, lb, P[keep], Q[keep], S[keep], q[keep])
            i, j, Sx, qx = _expand(tmp, np.ones(len(tmp.P), dtype=bool), upper=False)
            order = np.lexsort((-qx, i))
            i, j, Sx, qx = i[order], j[order], Sx[order], qx[order]
            n_first = pd.count[la] * NCART[la]
            counts = np.bincount(i, minlength=n_first).astype(np.uint32)
            displs = np.zeros(n_first, dtype=np.uint32)
            if n_first > 1:
                displs[1:] = np.cumsum(counts[:-1], dtype=np.uint64).astype(np.uint32)
            rl.kpartners[ANG[la] + ANG[lb]] = KPartners(displs, counts, j.astype(np.uint32), qx.copy(), Sx.copy())

    # ---------------- K (i, k) lists: keep (i, k) if some partner product can pass
    qpart = {}
    for la in ls:
        best = np.zeros(pd.count[la] * NCART[la])
        for lb in ls:
            kp = rl.kpartners[ANG[la] + ANG[lb]]
            has = kp.counts > 0
            best[has] = np.maximum(best[has], kp.Q[kp.displs[has]])
        qpart[la] = best
    for la in ls:
        for lc in ls:
            if la > lc:
                continue
            qi, qk = qpart[la], qpart[lc]
            ii, kk = np.nonzero(qi[:, None] * qk[None, :] * dmax > threshold)
            if la == lc:
                m = ii <= kk
                ii, kk = ii[m], kk[m]
            rl.kpairs[ANG[la] + ANG[lc]] = KPairs(ii.astype(np.uint32), kk.astype(np.uint32))
    return rl


# ------------------------------------------------------------------ AO maps

def contract_J(rl: ReferenceLists, matJ: dict) -> np.ndarray:
    """Prim-cart pair J (one array per "ab" list) -> symmetric AO J."""
    n = rl.naos
    M = np.zeros((n, n))
    for key, v in matJ.items():
        jl = rl.jlists[key]
        la, lb = LV[key[0]], LV[key[1]]
        ai = rl.pd.aoinds[la][jl.first % NCART[la], jl.first // NCART[la]]
        bj = rl.pd.aoinds[lb][jl.second % NCART[lb], jl.second // NCART[lb]]
        w = np.where((la == lb) & (jl.first == jl.second), 0.5, 1.0)
        np.add.at(M, (ai, bj), w * v)
    return M + M.T


def contract_K(rl: ReferenceLists, matK: dict) -> np.ndarray:
    """Prim-cart pair K (one array per "ac" list) -> symmetric AO K."""
    n = rl.naos
    M = np.zeros((n, n))
    for key, v in matK.items():
        kp = rl.kpairs[key]
        la, lc = LV[key[0]], LV[key[1]]
        ai = rl.pd.aoinds[la][kp.pair_i % NCART[la], kp.pair_i // NCART[la]]
        ck = rl.pd.aoinds[lc][kp.pair_k % NCART[lc], kp.pair_k // NCART[lc]]
        w = np.where((la == lc) & (kp.pair_i == kp.pair_k), 0.5, 1.0)
        np.add.at(M, (ai, ck), w * v)
    return M + M.T


def energy(D: np.ndarray, J: np.ndarray, K: np.ndarray) -> float:
    """E = Tr[D (J - K/2)]."""
    return float(np.sum(D * (J - 0.5 * K)))


def j_classes(ang: str = SPD):
    """Coulomb classes (ab|cd), a <= b and c <= d in angular momentum; the
    reference's 36 s/p/d classes by default."""
    pairs = [a + b for i, a in enumerate(ang) for b in ang[i:]]
    return [ab + cd for ab in pairs for cd in pairs]


def k_classes(ang: str = SPD):
    """Exchange classes (ab|cd), a <= c; the reference's 54 by default."""
    return [a + b + c + d for i, a in enumerate(ang) for c in ang[i:] for b in ang for d in ang]


def j_classes_all():
    """The 100 Coulomb classes of s, p, d and f shells."""
    return j_classes(ANG)


def k_classes_all():
    """The 160 exchange classes of s, p, d and f shells."""
    return k_classes(ANG)
