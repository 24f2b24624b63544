"""Generate golden vectors from the reference generator itself.

The reference (VeloxChem/vlx-twoe-ints) is a Python code generator: for each
(ab|cd) class, ``eriwriter.write_eri_code`` (eriwriter.py:35-160) returns the C
expression that the emitted kernels evaluate per Cartesian component quartet.
These expressions are valid Python once their free names are bound, so this
script binds them exactly as the emitted kernel prologues do
(gen_coulomb.py:165-268, gen_exchange.py:161-315) and evaluates them, with
Boys values taken from mpmath (the reference's own Boys function is external to
it).  Its outputs are committed; the tests only read the .npz files.

    python tests/golden/make_golden.py --ref <reference tree>

(or with VLX_REFERENCE_DIR=<reference tree> in the environment)

Writes:
  eri_components.npz  every one of the 81 s/p/d classes, bare component
                      integrals Lambda * poly(F_m) at seeded geometries, for
                      omega = 0 and omega = 0.4 (gen_exchange.py:278-298).
  jk_tiny.npz         a two-atom s/p/d system: the ABI arrays of every J class
                      (36) and K class (54) and mat_J / mat_K computed with the
                      emitted kernels' loop semantics (break on sorted lists).
  eri_grad_components.npz  every s/p/d class, the generator's derivative
                      expressions (write_eri_code(..., gradient='a'..'d'),
                      eriwriter.py:72-86, eri.py:85-175) for one centre per
                      class (rotating a..d; omega 0 / 0.4), all components and
                      directions.
  eri_f_components.npz  twelve classes with f centres (one or two), all
                      components, from the reference's symbolic engine with
                      three Cartesian indices on the f centres (eri.py).
"""
from __future__ import annotations

import argparse
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NCART = {"s": 1, "p": 3, "d": 6, "f": 10}
LVAL = {"s": 0, "p": 1, "d": 2, "f": 3}
D_CART = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]  # gen_coulomb.py:143-148
# f components in the same convention (sorted index triples: xxx, xxy, xxz, xyy,
# xyz, xzz, yyy, yyz, yzz, zzz)
F_CART = [(i, j, k) for i in range(3) for j in range(i, 3) for k in range(j, 3)]


def boys_mp(M, T):
    import mpmath as mp

    with mp.workdps(34):
        t = mp.mpf(T)
        out = []
        for m in range(M + 1):
            if t == 0:
                out.append(1.0 / (2 * m + 1))
            else:
                a = mp.mpf(m) + mp.mpf(1) / 2
                out.append(float(mp.gammainc(a, 0, t) / (2 * t ** a)))
        return out


class Classes:
    def __init__(self, ref):
        sys.path.insert(0, ref)
        from eriwriter import write_eri_code  # noqa: E402  (reference module)

        self._w = write_eri_code
        self._cache = {}

    def code(self, cls):
        if cls not in self._cache:
            src = self._w_f(cls) if "f" in cls else self._w(cls, indent=0)
            self._cache[cls] = compile("(" + src + ")", f"<eri {cls}>", "eval")
        return self._cache[cls]

    def _w_f(self, cls):
        """write_eri_code for a class with f centres.  The writer maps only the
        letters p and d to index lists (eriwriter.py:44-62) while its ERI
        class takes any number of Cartesian indices per centre (eri.py:59
        labels up to I), so the ERI constructor it calls is wrapped to give
        the f centres three indices (x0, x1, x2); everything else is the
        reference's own pipeline."""
        import eriwriter

        orig = eriwriter.ERI
        fpos = [n for n, x in enumerate(cls) if x == "f"]

        class ERIWithF(orig):
            def __init__(self, la, lb, lc, ld, *rest):
                lists = [list(la), list(lb), list(lc), list(ld)]
                for n in fpos:
                    lists[n] = [f"{'abcd'[n]}{k}" for k in range(3)]
                super().__init__(*lists, *rest)

        eriwriter.ERI = ERIWithF
        try:
            return self._w(cls.replace("f", "s"), indent=0)
        finally:
            eriwriter.ERI = orig

    def code_grad(self, cls, centre):
        """Compiled derivative expression of write_eri_code(cls, gradient=centre)
        (eriwriter.py:72-86) and the order of its Boys array (F<m>_t)."""
        key = (cls, centre)
        if key not in self._cache:
            import re

            src = self._w(cls, indent=0, gradient=centre)
            m = int(re.search(r"F(\d+)_t", src).group(1))
            self._cache[key] = (compile("(" + src + ")", f"<eri {cls} d{centre}>", "eval"), m)
        return self._cache[key]


def comp_indices(x, comp):
    """Component index variables of gen_coulomb.py:187-192 for one centre."""
    if x == "p":
        return [comp % 3]
    if x == "d":
        return list(D_CART[comp % 6])
    if x == "f":
        return list(F_CART[comp % 10])
    return []


_F_CACHE = {}


def eval_component(classes, cls, ai, ri, aj, rj, ak, rk, al, rl, comps, omega, F_cache=None):
    """Lambda * expression for one component quartet (gen_coulomb.py:244-274,
    gen_exchange.py:267-321).  comps = prim-cart indices (i, j, k, l)."""
    a, b, c, d = cls
    S1 = ai + aj
    inv_S1 = 1.0 / S1
    S2 = ak + al
    inv_S2 = 1.0 / S2
    inv_S4 = 1.0 / (S1 + S2)
    PQ = [(ak * rk[x] + al * rl[x]) * inv_S2 - (ai * ri[x] + aj * rj[x]) * inv_S1 for x in range(3)]
    r2 = PQ[0] ** 2 + PQ[1] ** 2 + PQ[2] ** 2
    rho = S1 * S2 * inv_S4
    d2 = 1.0
    if omega != 0.0:
        d2 = omega * omega / (rho + omega * omega)
    lam = math.sqrt(4.0 * rho * d2 / math.pi)
    L = sum(LVAL[x] for x in cls)
    key = (ai, aj, ak, al, tuple(ri), tuple(rj), tuple(rk), tuple(rl), omega)
    if F_cache is None:
        F_cache = _F_CACHE
    if key in F_cache:
        F = F_cache[key]
    else:
        F = boys_mp(L, rho * d2 * r2)
        if omega != 0.0:
            F = [F[m] * d2 ** m for m in range(L + 1)]
        F_cache[key] = F
    ns = {"PQ": PQ, "S1": S1, "S2": S2, "inv_S1": inv_S1, "inv_S2": inv_S2, "inv_S4": inv_S4,
          "delta": [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]], f"F{L}_t": F}
    ia, jb, kc, ld = comps
    ca = comp_indices(a, ia)
    cb = comp_indices(b, jb)
    cc = comp_indices(c, kc)
    cd = comp_indices(d, ld)
    for n, v in enumerate(ca):
        ns[f"a{n}"] = v
        ns[f"PA_{n}"] = (aj * inv_S1) * (rj[v] - ri[v])
    for n, v in enumerate(cb):
        ns[f"b{n}"] = v
        ns[f"PB_{n}"] = (-ai * inv_S1) * (rj[v] - ri[v])
    for n, v in enumerate(cc):
        ns[f"c{n}"] = v
        ns[f"QC_{n}"] = (al * inv_S2) * (rl[v] - rk[v])
    for n, v in enumerate(cd):
        ns[f"d{n}"] = v
        ns[f"QD_{n}"] = (-ak * inv_S2) * (rl[v] - rk[v])
    return lam * eval(classes.code(cls), {}, ns)


def eval_grad_component(classes, cls, centre, g, ai, ri, aj, rj, ak, rk, al, rl, comps, omega):
    """Lambda * the reference's derivative expression d/dX_g of one component
    quartet, X the centre `centre` ('a'..'d').  Binds the names of
    eval_component plus a_i..a_l (the four exponents), g / grad_cart_ind (the
    Cartesian direction) and PA_x, PB_x, QC_x, QD_x (the g components of
    P - A, P - B, Q - C, Q - D), as the generator's replacements at
    eriwriter.py:152-156 name them."""
    code, M = classes.code_grad(cls, centre)
    S1 = ai + aj
    inv_S1 = 1.0 / S1
    S2 = ak + al
    inv_S2 = 1.0 / S2
    inv_S4 = 1.0 / (S1 + S2)
    PQ = [(ak * rk[x] + al * rl[x]) * inv_S2 - (ai * ri[x] + aj * rj[x]) * inv_S1 for x in range(3)]
    r2 = PQ[0] ** 2 + PQ[1] ** 2 + PQ[2] ** 2
    rho = S1 * S2 * inv_S4
    d2 = 1.0
    if omega != 0.0:
        d2 = omega * omega / (rho + omega * omega)
    lam = math.sqrt(4.0 * rho * d2 / math.pi)
    F = boys_mp(M, rho * d2 * r2)
    if omega != 0.0:
        F = [F[m] * d2 ** m for m in range(M + 1)]
    ns = {"PQ": PQ, "S1": S1, "S2": S2, "inv_S1": inv_S1, "inv_S2": inv_S2, "inv_S4": inv_S4,
          "delta": [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]], f"F{M}_t": F,
          "a_i": ai, "a_j": aj, "a_k": ak, "a_l": al, "g": g, "grad_cart_ind": g,
          "PA_x": (aj * inv_S1) * (rj[g] - ri[g]), "PB_x": (-ai * inv_S1) * (rj[g] - ri[g]),
          "QC_x": (al * inv_S2) * (rl[g] - rk[g]), "QD_x": (-ak * inv_S2) * (rl[g] - rk[g])}
    a, b, c, d = cls
    ia, jb, kc, ld = comps
    for n, v in enumerate(comp_indices(a, ia)):
        ns[f"a{n}"] = v
        ns[f"PA_{n}"] = (aj * inv_S1) * (rj[v] - ri[v])
    for n, v in enumerate(comp_indices(b, jb)):
        ns[f"b{n}"] = v
        ns[f"PB_{n}"] = (-ai * inv_S1) * (rj[v] - ri[v])
    for n, v in enumerate(comp_indices(c, kc)):
        ns[f"c{n}"] = v
        ns[f"QC_{n}"] = (al * inv_S2) * (rl[v] - rk[v])
    for n, v in enumerate(comp_indices(d, ld)):
        ns[f"d{n}"] = v
        ns[f"QD_{n}"] = (-ak * inv_S2) * (rl[v] - rk[v])
    return lam * eval(code, {}, ns)


def make_grad_components(classes, rng):
    """Every s/p/d class once, the differentiated centre rotating over
    a, b, c, d and omega over 0 / 0.4 with the class index; all components,
    all three directions."""
    out = {}
    t = 0
    for a in "spd":
        for b in "spd":
            for c in "spd":
                for d in "spd":
                    cls = a + b + c + d
                    centre = "abcd"[t % 4]
                    omega = 0.4 if (t // 4) % 2 else 0.0
                    t += 1
                    ex = rng.uniform(0.3, 2.5, size=4)
                    R = rng.uniform(-1.2, 1.2, size=(4, 3))
                    vals = np.zeros((3, NCART[a], NCART[b], NCART[c], NCART[d]))
                    for g in range(3):
                        for ia in range(NCART[a]):
                            for ib in range(NCART[b]):
                                for ic in range(NCART[c]):
                                    for id_ in range(NCART[d]):
                                        vals[g, ia, ib, ic, id_] = eval_grad_component(
                                            classes, cls, centre, g, ex[0], R[0], ex[1], R[1], ex[2], R[2],
                                            ex[3], R[3], (ia, ib, ic, id_), omega)
                    out[f"{cls}_centre"] = np.array(["abcd".index(centre)])
                    out[f"{cls}_exps"] = ex
                    out[f"{cls}_centers"] = R
                    out[f"{cls}_omega"] = np.array([omega])
                    out[f"{cls}_vals"] = vals
    return out


F_CLASSES = ["fsss", "sfss", "ssfs", "sssf", "fpps", "psfp", "fdss", "sdsf", "ffss", "fsfs", "fpfp", "dfsd"]


def make_f_components(classes, rng):
    """Classes with f centres, from the reference's symbolic engine (see
    Classes._w_f): all components, omega 0 and 0.4 alternating."""
    out = {}
    for t, cls in enumerate(F_CLASSES):
        a, b, c, d = cls
        omega = 0.4 if t % 2 else 0.0
        ex = rng.uniform(0.3, 2.5, size=4)
        R = rng.uniform(-1.2, 1.2, size=(4, 3))
        vals = np.zeros((NCART[a], NCART[b], NCART[c], NCART[d]))
        Fc = {}
        for ia in range(NCART[a]):
            for ib in range(NCART[b]):
                for ic in range(NCART[c]):
                    for id_ in range(NCART[d]):
                        vals[ia, ib, ic, id_] = eval_component(classes, cls, ex[0], R[0], ex[1], R[1], ex[2], R[2],
                                                               ex[3], R[3], (ia, ib, ic, id_), omega, Fc)
        out[f"{cls}_exps"] = ex
        out[f"{cls}_centers"] = R
        out[f"{cls}_omega"] = np.array([omega])
        out[f"{cls}_vals"] = vals
    return out


# ------------------------------------------------------------ component set

def make_components(classes, rng):
    out = {}
    for a in "spd":
        for b in "spd":
            for c in "spd":
                for d in "spd":
                    cls = a + b + c + d
                    for tag, omega in (("w0", 0.0), ("w4", 0.4)):
                        ex = rng.uniform(0.3, 2.5, size=4)
                        R = rng.uniform(-1.2, 1.2, size=(4, 3))
                        vals = np.zeros((NCART[a], NCART[b], NCART[c], NCART[d]))
                        Fc = {}
                        for ia in range(NCART[a]):
                            for ib in range(NCART[b]):
                                for ic in range(NCART[c]):
                                    for id_ in range(NCART[d]):
                                        vals[ia, ib, ic, id_] = eval_component(
                                            classes, cls, ex[0], R[0], ex[1], R[1], ex[2], R[2],
                                            ex[3], R[3], (ia, ib, ic, id_), omega, Fc)
                        out[f"{cls}_{tag}_exps"] = ex
                        out[f"{cls}_{tag}_centers"] = R
                        out[f"{cls}_{tag}_omega"] = np.array([omega])
                        out[f"{cls}_{tag}_vals"] = vals
    return out


# ------------------------------------------------------------ tiny system

def tiny_system():
    """Two atoms; per atom: one s shell of 2 primitives, one p and one d shell
    of 1 primitive each.  Cartesian AOs: 2 x (1 + 3 + 6) = 20."""
    atoms = np.array([[0.0, 0.0, 0.0], [0.9, -0.4, 1.1]])
    shells = [  # (atom, l, exponents, coefficients)
        (0, 0, [3.1, 0.8], [0.4, 0.7]),
        (0, 1, [1.1], [1.0]),
        (0, 2, [0.9], [1.0]),
        (1, 0, [2.2, 0.5], [0.5, 0.6]),
        (1, 1, [0.7], [1.0]),
        (1, 2, [0.6], [1.0]),
    ]
    return atoms, shells


def dfact(n):
    return 1.0 if n <= 0 else n * dfact(n - 2)


CART = {0: [(0, 0, 0)], 1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
        2: [(2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)]}


def prim_norm(alpha, lxyz):
    lx, ly, lz = lxyz
    l = lx + ly + lz
    return math.sqrt((2 * alpha / math.pi) ** 1.5 * (4 * alpha) ** l /
                     (dfact(2 * lx - 1) * dfact(2 * ly - 1) * dfact(2 * lz - 1)))


def build_tiny(classes, rng):
    atoms, shells = tiny_system()
    prims = {0: [], 1: [], 2: []}  # per l: list of (alpha, center, coef, ao_base)
    ao = 0
    for (at, l, exps, coefs) in shells:
        for e, c in zip(exps, coefs):
            prims[l].append((e, atoms[at], c, ao))
        ao += len(CART[l])
    naos = ao
    prim_info, prim_aoinds, count = {}, {}, {}
    for l in range(3):
        n = len(prims[l])
        info = np.zeros((5, n))
        aoi = np.zeros((len(CART[l]), n), dtype=np.uint32)
        for p, (e, R, c, base) in enumerate(prims[l]):
            info[0, p] = e
            info[1, p] = c
            info[2:5, p] = R
            for comp in range(len(CART[l])):
                aoi[comp, p] = base + comp
        prim_info[l], prim_aoinds[l], count[l] = info, aoi, n

    # random symmetric AO density
    C = rng.standard_normal((naos, 4))
    D = C @ C.T / 4.0

    def pc(l, i):
        p = i // len(CART[l])
        comp = i % len(CART[l])
        e, R, c, base = prims[l][p]
        return e, R, c, comp, base + comp

    def S00(la, i, lb, j):
        # per-component overlap prefactor incl. coefficients and norms
        ea, Ra, ca, ka, _ = pc(la, i)
        eb, Rb, cb, kb, _ = pc(lb, j)
        p = ea + eb
        kab = math.exp(-ea * eb / p * float(np.sum((Ra - Rb) ** 2)))
        return (ca * cb * prim_norm(ea, CART[la][ka]) * prim_norm(eb, CART[lb][kb])
                * (math.pi / p) ** 1.5 * kab)

    def eri(cls, i, j, k, l, omega=0.0):
        la, lb, lc, ld = (LVAL[x] for x in cls)
        ea, Ra, _, ka, _ = pc(la, i)
        eb, Rb, _, kb, _ = pc(lb, j)
        ec, Rc, _, kc, _ = pc(lc, k)
        ed, Rd, _, kd, _ = pc(ld, l)
        return eval_component(classes, cls, ea, Ra, eb, Rb, ec, Rc, ed, Rd, (ka, kb, kc, kd), omega)

    def nprc(l):
        return count[l] * len(CART[l])

    Qcache = {}

    def Qij(a, b, i, j):
        key = (a, b, i, j)
        if key not in Qcache:
            v = eri(a + b + a + b, i, j, i, j) * S00(LVAL[a], i, LVAL[b], j) ** 2
            Qcache[key] = math.sqrt(abs(v))
        return Qcache[key]

    out = {"naos": np.array([naos]), "D_AO": D}
    for l in range(3):
        out[f"prim_info_{l}"] = prim_info[l]
        out[f"prim_aoinds_{l}"] = prim_aoinds[l]

    # J pair lists (gen_coulomb.py:80-90): a <= b by angular momentum;
    # same-type pairs keep i <= j, and the ket list is sorted by descending |Q D|.
    pairs = {}
    for a in "spd":
        for b in "spd":
            if LVAL[a] > LVAL[b]:
                continue
            la, lb = LVAL[a], LVAL[b]
            lst = []
            for i in range(nprc(la)):
                for j in range(nprc(lb)):
                    if a == b and j < i:
                        continue
                    q = Qij(a, b, i, j)
                    dval = D[pc(la, i)[4], pc(lb, j)[4]]
                    lst.append((i, j, S00(la, i, lb, j), q, dval))
            lst.sort(key=lambda t: -abs(t[3] * t[4]))
            arr = np.array(lst)
            pairs[a + b] = arr
            out[f"J_{a}{b}_first"] = arr[:, 0].astype(np.uint32)
            out[f"J_{a}{b}_second"] = arr[:, 1].astype(np.uint32)
            out[f"J_{a}{b}_pdata"] = arr[:, 2]
            out[f"J_{a}{b}_Q"] = arr[:, 3]
            out[f"J_{a}{b}_D"] = arr[:, 4]

    thresholds = {"t12": 1e-12, "t3": 2e-3}
    out["thresholds"] = np.array([1e-12, 2e-3])
    # J: reference loop semantics (gen_coulomb.py:205-297) with sequential break
    for ab, bra in pairs.items():
        for cd, ket in pairs.items():
            cls = ab + cd
            for tname, thr in thresholds.items():
                J = np.zeros(len(bra))
                for ij in range(len(bra)):
                    i, j = int(bra[ij, 0]), int(bra[ij, 1])
                    acc = 0.0
                    for kl in range(len(ket)):
                        if abs(bra[ij, 3] * ket[kl, 3] * ket[kl, 4]) <= thr:
                            break
                        k, l = int(ket[kl, 0]), int(ket[kl, 1])
                        v = bra[ij, 2] * ket[kl, 2] * eri(cls, i, j, k, l)
                        w = 2.0 if cd[0] != cd[1] else (2.0 if k != l else 1.0)
                        acc += v * ket[kl, 4] * w
                    J[ij] = acc
                out[f"J_{cls}_{tname}"] = J

    # K partner lists (gen_exchange.py:161-251): for every prim-cart i of type a,
    # all partners j of type b, sorted by descending Q_ij.
    for a in "spd":
        for b in "spd":
            la, lb = LVAL[a], LVAL[b]
            displs, counts, Dinds, Qs, pd = [], [], [], [], []
            for i in range(nprc(la)):
                part = sorted(((Qij(a, b, i, j), j) for j in range(nprc(lb))), key=lambda t: -t[0])
                displs.append(len(Dinds))
                counts.append(len(part))
                for q, j in part:
                    Dinds.append(j)
                    Qs.append(q)
                    pd.append(S00(la, i, lb, j))
            out[f"K_{a}{b}_displs"] = np.array(displs, dtype=np.uint32)
            out[f"K_{a}{b}_counts"] = np.array(counts, dtype=np.uint32)
            out[f"K_{a}{b}_Dinds"] = np.array(Dinds, dtype=np.uint32)
            out[f"K_{a}{b}_Q"] = np.array(Qs)
            out[f"K_{a}{b}_pdata"] = np.array(pd)

    # K classes: ac over the upper triangle, bd over all 9 (gen_eri_exchange.py:39-56)
    for ia_, a in enumerate("spd"):
        for c in "spd"[ia_:]:
            la, lc = LVAL[a], LVAL[c]
            ik = [(i, k) for i in range(nprc(la)) for k in range(nprc(lc)) if not (a == c and k < i)]
            out[f"K_{a}{c}_pair_i"] = np.array([t[0] for t in ik], dtype=np.uint32)
            out[f"K_{a}{c}_pair_k"] = np.array([t[1] for t in ik], dtype=np.uint32)
            for b in "spd":
                for d in "spd":
                    cls = a + b + c + d
                    lb, ld = LVAL[b], LVAL[d]
                    maxD = max(abs(D[pc(lb, j)[4], pc(ld, l)[4]])
                               for j in range(nprc(lb)) for l in range(nprc(ld)))
                    out[f"K_{cls}_maxD"] = np.array([maxD])
                    for tname, thr, omega, nrow in (("t12", 1e-12, 0.0, None), ("t3", 2e-3, 0.0, None),
                                                    ("w3", 1e-12, 0.3, 6)):
                        rows = range(len(ik)) if nrow is None else range(min(nrow, len(ik)))
                        K = np.zeros(len(rows))
                        for r, n in enumerate(rows):
                            i, k = ik[n]
                            acc = 0.0
                            di, ci_ = out[f"K_{a}{b}_displs"][i], out[f"K_{a}{b}_counts"][i]
                            dk, ck = out[f"K_{c}{d}_displs"][k], out[f"K_{c}{d}_counts"][k]
                            for jj in range(ci_):
                                qij = out[f"K_{a}{b}_Q"][di + jj]
                                j = int(out[f"K_{a}{b}_Dinds"][di + jj])
                                for ll in range(ck):
                                    qkl = out[f"K_{c}{d}_Q"][dk + ll]
                                    if abs(qij * qkl * maxD) <= thr:
                                        break
                                    l = int(out[f"K_{c}{d}_Dinds"][dk + ll])
                                    v = (out[f"K_{a}{b}_pdata"][di + jj] * out[f"K_{c}{d}_pdata"][dk + ll]
                                         * eri(cls, i, j, k, l, omega))
                                    acc += v * D[pc(lb, j)[4], pc(ld, l)[4]]
                            K[r] = acc
                        out[f"K_{cls}_{tname}"] = K
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("VLX_REFERENCE_DIR"),
                    help="the vlx-twoe-ints source tree (default: $VLX_REFERENCE_DIR)")
    ap.add_argument("--only", choices=["components", "tiny", "grad", "f"], default=None)
    args = ap.parse_args()
    if not args.ref or not os.path.isdir(args.ref):
        ap.error("the reference tree is needed: --ref <dir> or VLX_REFERENCE_DIR")
    classes = Classes(args.ref)
    if args.only in (None, "components"):
        comp = make_components(classes, np.random.default_rng(1234))
        np.savez_compressed(os.path.join(HERE, "eri_components.npz"), **comp)
        print("eri_components.npz:", len(comp), "arrays")
    if args.only in (None, "grad"):
        grad = make_grad_components(classes, np.random.default_rng(2468))
        np.savez_compressed(os.path.join(HERE, "eri_grad_components.npz"), **grad)
        print("eri_grad_components.npz:", len(grad), "arrays")
    if args.only in (None, "f"):
        fc = make_f_components(classes, np.random.default_rng(1357))
        np.savez_compressed(os.path.join(HERE, "eri_f_components.npz"), **fc)
        print("eri_f_components.npz:", len(fc), "arrays")
    if args.only in (None, "tiny"):
        tiny = build_tiny(classes, np.random.default_rng(4321))
        np.savez_compressed(os.path.join(HERE, "jk_tiny.npz"), **tiny)
        print("jk_tiny.npz:", len(tiny), "arrays")


if __name__ == "__main__":
    main()
