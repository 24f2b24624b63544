"""Generator of the per-class shell-quartet device code (our own design).

For one (ab|cd) class with angular momenta (la, lb, lc, ld) <= 2 it emits
straight-line CUDA that evaluates, for ONE primitive shell quartet and ALL its
Cartesian components at once:

  VRR   [e0|f0]^(m) by Obara-Saika: VRR on c (building f) on top of VRR on a
        (building e), |e| in [la, la+lb], |f| in [lc, lc+ld].  The coefficient
        conventions are those of the reference's symbolic engine
        (eri.py:237-355: PQ = Q - P, W - P = S2/S4 PQ, W - Q = -S1/S4 PQ).
  HRR   (e0|cd) from (e0|f0) with CD = C - D, then (ab|cd) from (e0|cd) with
        AB = A - B (eri.py:177-235).

The reference instead expands one Cartesian COMPONENT quartet into a flat
polynomial per thread (eriwriter.py:35-160), re-deriving every shared
intermediate for each of up to 1296 components.  Here every intermediate is
computed once per primitive shell quartet.

Emitted functions (all __device__ __forceinline__, templated on the class):
  eri_full   : all (ab|cd) into out[((a*nb+b)*nc+c)*nd+d]
  j_contract : X_e += sum_f (e0|f0) * Dpp_f  (Coulomb: ket density already
               carried through the transposed ket HRR, so only the VRR runs
               per quartet)
  hrr_ket_adjoint<lc,ld>: Dpp_f = sum_cd H(cd <- f) Dm_cd   (per ket pair)
  hrr_bra_vector<la,lb> : J_ab  = sum_e H(ab <- e) X_e      (per bra pair)

Usage:  python gen_quartets.py OUTDIR      (writes q_<class>.cuh, hrr_pairs.cuh and
        quartet_flops.json)
"""
from __future__ import annotations

import json
import os
import sys

LNAME = "spd"


def comps(l):
    """Cartesian components of shell l in the reference's order
    (gen_coulomb.py:143-148): p x,y,z; d xx,xy,xz,yy,yz,zz."""
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


def ncart(l):
    return (l + 1) * (l + 2) // 2


def sub1(v, i):
    w = list(v)
    w[i] -= 1
    return tuple(w)


def add1(v, i):
    w = list(v)
    w[i] += 1
    return tuple(w)


def first_nz(v):
    for i in range(3):
        if v[i] > 0:
            return i
    return -1


def erange(l0, l1):
    out = []
    for l in range(l0, l1 + 1):
        out += comps(l)
    return out


class Flops:
    def __init__(self):
        self.mul = 0
        self.add = 0
        self.fma = 0

    def total(self):
        return self.mul + self.add + 2 * self.fma


# --------------------------------------------------------------------- VRR

class VRR:
    """Dependency-closed VRR node set for given targets, in DFS post-order."""

    def __init__(self, targets):
        self.order = []
        self.index = {}
        for t in targets:
            self._need(*t)

    def _need(self, e, f, m):
        if min(e) < 0 or min(f) < 0:
            return
        k = (e, f, m)
        if k in self.index:
            return
        for d in self.deps(e, f, m):
            self._need(*d)
        self.index[k] = len(self.order)
        self.order.append(k)

    @staticmethod
    def deps(e, f, m):
        out = []
        if sum(f) > 0:
            i = first_nz(f)
            f1 = sub1(f, i)
            out += [(e, f1, m), (e, f1, m + 1)]
            if f1[i] > 0:
                f2 = sub1(f1, i)
                out += [(e, f2, m), (e, f2, m + 1)]
            if e[i] > 0:
                out.append((sub1(e, i), f1, m + 1))
        elif sum(e) > 0:
            i = first_nz(e)
            e1 = sub1(e, i)
            out += [(e1, f, m), (e1, f, m + 1)]
            if e1[i] > 0:
                e2 = sub1(e1, i)
                out += [(e2, f, m), (e2, f, m + 1)]
        return out

    def expr(self, node, name, fl: Flops):
        """C expression for one node; name(node) gives operand names."""
        e, f, m = node
        X = "xyz"
        if sum(f) > 0:
            i = first_nz(f)
            f1 = sub1(f, i)
            terms = f"q.QC{X[i]} * {name((e, f1, m))}"
            fl.mul += 1
            terms = f"fma(q.WQ{X[i]}, {name((e, f1, m + 1))}, {terms})"
            fl.fma += 1
            if f1[i] > 0:
                f2 = sub1(f1, i)
                inner = f"fma(-q.re, {name((e, f2, m + 1))}, {name((e, f2, m))})"
                terms = f"fma(c2e_{f1[i]}, {inner}, {terms})"
                fl.fma += 2
            if e[i] > 0:
                terms = f"fma(c2ze_{e[i]}, {name((sub1(e, i), f1, m + 1))}, {terms})"
                fl.fma += 1
            return terms
        if sum(e) > 0:
            i = first_nz(e)
            e1 = sub1(e, i)
            terms = f"q.PA{X[i]} * {name((e1, f, m))}"
            fl.mul += 1
            terms = f"fma(q.WP{X[i]}, {name((e1, f, m + 1))}, {terms})"
            fl.fma += 1
            if e1[i] > 0:
                e2 = sub1(e1, i)
                inner = f"fma(-q.rz, {name((e2, f, m + 1))}, {name((e2, f, m))})"
                terms = f"fma(c2z_{e1[i]}, {inner}, {terms})"
                fl.fma += 2
            return terms
        return f"F[{m}]"


# --------------------------------------------------------------------- HRR

class HRR:
    """Node set of (x, y) with y built from x: (x, y) = (x+1_i, y-1_i) + R_i (x, y-1_i)."""

    def __init__(self, lx, ly):
        self.lx, self.ly = lx, ly
        self.order = []
        self.index = {}
        for x in comps(lx):
            for y in comps(ly):
                self._need(x, y)

    def _need(self, x, y):
        k = (x, y)
        if k in self.index:
            return
        if sum(y) > 0:
            i = first_nz(y)
            self._need(add1(x, i), sub1(y, i))
            self._need(x, sub1(y, i))
        self.index[k] = len(self.order)
        self.order.append(k)

    def bases(self):
        return [n for n in self.order if sum(n[1]) == 0]


def q_prologue(la, lb, lc, ld, T="double"):
    lit = "f" if T == "float" else ""
    lines = []
    for k in range(1, la + lb + 1):
        lines.append(f"    const {T} c2z_{k} = {k}.0{lit} * q.inv2z; (void)c2z_{k};")
    for k in range(1, lc + ld + 1):
        lines.append(f"    const {T} c2e_{k} = {k}.0{lit} * q.inv2e; (void)c2e_{k};")
    for k in range(1, la + lb + 1):
        lines.append(f"    const {T} c2ze_{k} = {k}.0{lit} * q.inv2ze; (void)c2ze_{k};")
    return lines


def gen_vrr_block(la, lb, lc, ld, fl, sink, T="double"):
    """Straight-line VRR; sink(node, varname) -> extra lines after a target."""
    E = erange(la, la + lb)
    Fs = erange(lc, lc + ld)
    targets = [(e, f, 0) for e in E for f in Fs]
    v = VRR(targets)
    names = {}

    def name(n):
        return names[n]

    lines = []
    tset = set(targets)
    for idx, node in enumerate(v.order):
        nm = f"v{idx}"
        names[node] = nm
        lines.append(f"    const {T} {nm} = {v.expr(node, name, fl)};")
        if node in tset:
            lines += sink(node, nm)
    return lines, E, Fs


def gen_eri_full(la, lb, lc, ld, T="double"):
    fl = Flops()
    E = erange(la, la + lb)
    Fs = erange(lc, lc + ld)
    eidx = {e: i for i, e in enumerate(E)}
    fidx = {f: i for i, f in enumerate(Fs)}
    lines = [f"template <> __device__ __forceinline__ void eri_full<{la}, {lb}, {lc}, {ld}, {T}>"
             f"(const QVT<{T}>& q, const {T}* F, {T}* out)", "{"]
    lines += q_prologue(la, lb, lc, ld, T)
    tnames = {}

    def sink(node, nm):
        tnames[(node[0], node[1])] = nm
        return []

    vl, _, _ = gen_vrr_block(la, lb, lc, ld, fl, sink, T)
    lines += vl
    # ket HRR per e
    hk = HRR(lc, ld)
    ket_names = {}
    for e in E:
        for node in hk.order:
            x, y = node
            if sum(y) == 0:
                ket_names[(e, x, y)] = tnames[(e, x)]
                continue
            i = first_nz(y)
            a1 = ket_names[(e, add1(x, i), sub1(y, i))]
            a2 = ket_names[(e, x, sub1(y, i))]
            nm = f"k{eidx[e]}_{hk.index[node]}"
            lines.append(f"    const {T} {nm} = fma(q.CD{'xyz'[i]}, {a2}, {a1});")
            fl.fma += 1
            ket_names[(e, x, y)] = nm
    # bra HRR per (c, d)
    hb = HRR(la, lb)
    Cc, Dd = comps(lc), comps(ld)
    Aa, Bb = comps(la), comps(lb)
    nb, nc, nd = len(Bb), len(Cc), len(Dd)
    for ic, c in enumerate(Cc):
        for id_, d in enumerate(Dd):
            bra_names = {}
            for node in hb.order:
                x, y = node
                if sum(y) == 0:
                    bra_names[node] = ket_names[(x, c, d)]
                    continue
                i = first_nz(y)
                a1 = bra_names[(add1(x, i), sub1(y, i))]
                a2 = bra_names[(x, sub1(y, i))]
                nm = f"b{ic}_{id_}_{hb.index[node]}"
                lines.append(f"    const {T} {nm} = fma(q.AB{'xyz'[i]}, {a2}, {a1});")
                fl.fma += 1
                bra_names[node] = nm
            for ia, a in enumerate(Aa):
                for ib, b in enumerate(Bb):
                    o = ((ia * nb + ib) * nc + ic) * nd + id_
                    lines.append(f"    out[{o}] = {bra_names[(a, b)]};")
    lines.append("}")
    return lines, fl


def gen_j_contract(la, lb, lc, ld, T="double"):
    fl = Flops()
    E = erange(la, la + lb)
    Fs = erange(lc, lc + ld)
    eidx = {e: i for i, e in enumerate(E)}
    fidx = {f: i for i, f in enumerate(Fs)}
    lines = [f"template <> __device__ __forceinline__ void j_contract<{la}, {lb}, {lc}, {ld}, {T}>"
             f"(const QVT<{T}>& q, const {T}* F, const {T}* Dpp, {T}* X)", "{"]
    lines += q_prologue(la, lb, lc, ld, T)

    def sink(node, nm):
        fl.fma += 1
        return [f"    X[{eidx[node[0]]}] = fma({nm}, Dpp[{fidx[node[1]]}], X[{eidx[node[0]]}]);"]

    vl, _, _ = gen_vrr_block(la, lb, lc, ld, fl, sink, T)
    lines += vl
    lines.append("}")
    return lines, fl


def gen_hrr_ket_adjoint(lc, ld, T="double"):
    """Dpp_f (f over erange(lc, lc+ld)) = sum_{c,d} H(cd <- f) Dm[c*nd+d]."""
    hk = HRR(lc, ld)
    Fs = erange(lc, lc + ld)
    fidx = {f: i for i, f in enumerate(Fs)}
    Cc, Dd = comps(lc), comps(ld)
    nd = len(Dd)
    lines = [f"template <> __device__ __forceinline__ void hrr_ket_adjoint<{lc}, {ld}, {T}>"
             f"({T} CDx, {T} CDy, {T} CDz, const {T}* Dm, {T}* Dpp)", "{",
             f"    const {T} CDv[3] = {{CDx, CDy, CDz}}; (void)CDv;"]
    # adjoint accumulators per node
    adj = {n: f"a{hk.index[n]}" for n in hk.order}
    for n in hk.order:
        lines.append(f"    {T} {adj[n]} = 0;")
    for ic, c in enumerate(Cc):
        for id_, d in enumerate(Dd):
            lines.append(f"    {adj[(c, d)]} += Dm[{ic * nd + id_}];")
    for n in reversed(hk.order):
        x, y = n
        if sum(y) == 0:
            continue
        i = first_nz(y)
        p1 = (add1(x, i), sub1(y, i))
        p2 = (x, sub1(y, i))
        lines.append(f"    {adj[p1]} += {adj[n]};")
        lines.append(f"    {adj[p2]} = fma(CDv[{i}], {adj[n]}, {adj[p2]});")
    for f in Fs:
        lines.append(f"    Dpp[{fidx[f]}] = {adj[(f, (0, 0, 0))]};")
    lines.append("}")
    return lines


def gen_hrr_bra_vector(la, lb, T="double"):
    """J[a*nb+b] = sum_e H(ab <- e) X_e, e over erange(la, la+lb)."""
    hb = HRR(la, lb)
    E = erange(la, la + lb)
    eidx = {e: i for i, e in enumerate(E)}
    Aa, Bb = comps(la), comps(lb)
    nb = len(Bb)
    lines = [f"template <> __device__ __forceinline__ void hrr_bra_vector<{la}, {lb}, {T}>"
             f"({T} ABx, {T} ABy, {T} ABz, const {T}* X, {T}* J)", "{",
             f"    const {T} ABv[3] = {{ABx, ABy, ABz}}; (void)ABv;"]
    names = {}
    for n in hb.order:
        x, y = n
        if sum(y) == 0:
            names[n] = f"X[{eidx[x]}]"
            continue
        i = first_nz(y)
        nm = f"h{hb.index[n]}"
        lines.append(f"    const {T} {nm} = fma(ABv[{i}], {names[(x, sub1(y, i))]}, "
                     f"{names[(add1(x, i), sub1(y, i))]});")
        names[n] = nm
    for ia, a in enumerate(Aa):
        for ib, b in enumerate(Bb):
            lines.append(f"    J[{ia * nb + ib}] = {names[(a, b)]};")
    lines.append("}")
    return lines


def write_if_changed(path, text):
    if os.path.exists(path):
        with open(path) as fh:
            if fh.read() == text:
                return
    with open(path, "w") as fh:
        fh.write(text)


def all_classes():
    return [(a, b, c, d) for a in range(3) for b in range(3) for c in range(3) for d in range(3)]


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    flops = {}
    for (la, lb, lc, ld) in all_classes():
        name = LNAME[la] + LNAME[lb] + LNAME[lc] + LNAME[ld]
        l1, f1 = gen_eri_full(la, lb, lc, ld)
        l2, f2 = gen_j_contract(la, lb, lc, ld)
        l3, _ = gen_eri_full(la, lb, lc, ld, "float")
        l4, _ = gen_j_contract(la, lb, lc, ld, "float")
        write_if_changed(os.path.join(outdir, f"q_{name}.cuh"),
                         "\n".join(["// Generated by gen_quartets.py -- do not edit.", "#pragma once",
                                    "namespace vlxb {", ""] + l1 + [""] + l2 + [""] + l3 + [""] + l4
                                   + ["", "}  // namespace vlxb", ""]))
        flops[name] = {"vrr_hrr_full": f1.total(), "j_contract": f2.total(),
                       "n_vrr": len(VRR([(e, f, 0) for e in erange(la, la + lb)
                                         for f in erange(lc, lc + ld)]).order)}
    pairs = []
    for lc in range(3):
        for ld in range(3):
            for T in ("double", "float"):
                pairs += gen_hrr_ket_adjoint(lc, ld, T) + [""]
                pairs += gen_hrr_bra_vector(lc, ld, T) + [""]
    write_if_changed(os.path.join(outdir, "hrr_pairs.cuh"),
                     "\n".join(["// Generated by gen_quartets.py -- do not edit.", "#pragma once",
                                "namespace vlxb {", ""] + pairs + ["}  // namespace vlxb", ""]))
    write_if_changed(os.path.join(outdir, "quartet_flops.json"), json.dumps(flops, indent=1, sort_keys=True))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(__file__), "generated"))
