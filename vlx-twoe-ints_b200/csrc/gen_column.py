"""Warp-cooperative ("column") Obara-Saika VRR for the heavy classes (our design).

One primitive shell quartet is spread over a group of lanes.  Each lane owns
one Cartesian component x of the "lane side" (bra e in orientation 0, ket f
in orientation 1) and holds the whole column [x|y]^(m) of that component in
its registers; the "step side" y is built by identical straight-line steps on
every lane:

  ori 0 (lanes = e):  [e|f+1_i]^m = QC_i [e|f]^m + WQ_i [e|f]^{m+1}
                        + f_i/(2 eta) ([e|f-1_i]^m - rho/eta [e|f-1_i]^{m+1})
                        + e_i/(2(zeta+eta)) [e-1_i|f]^{m+1}
  ori 1 (lanes = f):  the same with the roles of (PA, WP, zeta) and
                        (QC, WQ, eta) exchanged (VRR on a with f coupling).

(coefficients as in the reference's eri.py:237-355).  The coupling term comes
from the lane that owns x - 1_i, through one __shfl_sync per step.  A lane's
own base column [x|0]^m is built by the other side's recursion along a path
from 0 to x.  When the lane side needs more than 32 components (d+d pairs:
35), the two lowest levels get no lane: the lanes of level 2 derive the
level-1 values they couple to from a short uniform tower [0|y]^m that every
lane computes.

ColumnPlan holds every table the CUDA emitter and the Python emulator share,
so the emulator (tests) validates exactly the schedule that is compiled.
"""
from __future__ import annotations

import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from gen_quartets import HRR, add1, comps, erange, first_nz, sub1  # noqa: E402

XYZ = "xyz"


def level_comps(l0, l1):
    out = []
    for l in range(l0, l1 + 1):
        out += comps(l)
    return out


# Plan kinds ("ori"): bit 0 is the orientation (0: lanes = bra e, 1: lanes =
# ket f); 2 and 3 are the packed plans of orientations 0 and 1 (lanes only
# for the target levels, which must start at level 2: the level-1 coupling
# partners come from the uniform tower, so a d+p lane side needs 16 lanes
# instead of 20 and a warp holds two quartets); 4 and 5 are packed plans
# whose lane-side pair is built on its second centre (B for the bra, D for
# the ket: e in [lb, la + lb]), for the pairs whose second shell is the
# higher one (p+d, s+d).  The kernels turn PA into PB = PA + AB and AB into
# BA before the VRR (QC, CD likewise) and read the lane-side HRR result
# transposed.
PLAN_KINDS = range(6)


def lane_pair(la, lb, lc, ld, ori):
    """(first, second) shell of the lane-side pair and of the step-side pair."""
    x, y = ((la, lb), (lc, ld)) if ori % 2 == 0 else ((lc, ld), (la, lb))
    if ori >= 4:
        x = (x[1], x[0])
    return x, y


class ColumnPlan:
    def __init__(self, la, lb, lc, ld, ori):
        self.cls = (la, lb, lc, ld)
        self.ori = ori
        self.orient = ori % 2
        self.packed = ori >= 2
        self.swapped = ori >= 4
        (xa, xb), (ya, yb) = lane_pair(la, lb, lc, ld, ori)
        lx0, lx1, ly0, ly1 = xa, xa + xb, ya, ya + yb
        self.lx0, self.lx1, self.ly0, self.ly1 = lx0, lx1, ly0, ly1
        self.L = la + lb + lc + ld
        self.lmin = max(0, lx0 - ly1)
        if self.packed:
            lam = lx0
        else:
            lam = self.lmin
            while len(level_comps(lam, lx1)) > 32:
                lam += 1
        self.lam = lam
        self.lanes = level_comps(lam, lx1)          # lane side components, lane index = position
        self.NL = len(self.lanes)
        self.P = max(1, 32 // self.NL) if self.NL <= 16 else 1
        self.xtargets = level_comps(lx0, lx1)        # lane side targets
        self.ytargets = level_comps(ly0, ly1)        # step side targets
        self.derive = lam > self.lmin                 # level-lam lanes derive their coupling source
        self.applies = self._applies()
        if not self.applies:
            return
        assert lam - self.lmin <= 2, "derivation deeper than one level is not supported"
        self._step_closure()
        self._chain()
        self._tower()

    def _applies(self):
        """Whether this plan kind is built for the class: the plain kinds
        always; a packed kind when its lanes start at level 2 below a
        derivation (lam - 1 = 1, the tower's one-step partners), it holds more
        quartets per warp than the plain plan of its orientation, and (for
        4, 5) the lane-side pair's second shell is the higher one."""
        if not self.packed:
            return True
        if self.lam != 2 or not self.derive or self.NL > 16:
            return False
        la, lb, lc, ld = self.cls
        xa, xb = (la, lb) if self.orient == 0 else (lc, ld)
        if self.swapped and not xa < xb:
            return False
        plain = ColumnPlan(la, lb, lc, ld, self.orient)
        return self.P > plain.P

    # ---------------------------------------------------------- step nodes
    def _step_deps(self, y, m):
        i = first_nz(y)
        y1 = sub1(y, i)
        d = [(y1, m), (y1, m + 1)]
        if y1[i] > 0:
            y2 = sub1(y1, i)
            d += [(y2, m), (y2, m + 1)]
        return d

    def _step_closure(self):
        order, seen = [], set()

        def need(y, m):
            if (y, m) in seen:
                return
            if sum(y) > 0:
                for d in self._step_deps(y, m):
                    need(*d)
            seen.add((y, m))
            order.append((y, m))

        for y in self.ytargets:
            need(y, 0)
        self.step_nodes = [n for n in order if sum(n[0]) > 0]
        self.base_m = max(m for (y, m) in order if sum(y) == 0)
        self.Mb = self.base_m
        # a node (x, y) is needed only if |x| - |y| >= lx0 - ly1 (the coupling
        # term lowers both levels by one); level-lam lanes derive their
        # coupling source on the steps where their own node is needed.
        dmin = self.lx0 - self.ly1
        self.need_derived = {n: self.derive and sum(n[0]) <= self.lam - dmin for n in self.step_nodes}

    # ---------------------------------------------------------- base chain
    def _chain(self):
        # path from 0 to x: add z's, then y's, then x's (reverse of the
        # first-nonzero decrement), so repeated directions are consecutive.
        self.chain = []
        for x in self.lanes:
            steps = []
            cur = [0, 0, 0]
            for d in (2, 1, 0):
                for _ in range(x[d]):
                    steps.append((d, cur[d]))  # (direction, count of d before the step)
                    cur[d] += 1
            self.chain.append(steps)
        self.chain_len = self.lx1
        # m range of chain step s (1-based): base needs m <= Mb at level |x|
        self.chain_m = {s: self.Mb + (self.lx1 - s) for s in range(0, self.lx1 + 1)}

    # ---------------------------------------------------------- tower
    def _tower(self):
        self.tower_nodes = []
        if not self.derive:
            return
        need = set()
        for (y, m), nd in self.need_derived.items():
            if not nd:
                continue
            i = first_nz(y)
            g = sub1(y, i)
            need.add((g, m + 1))
            need.add((g, m + 2))
            for j in range(3):
                if g[j] > 0:
                    need.add((sub1(g, j), m + 2))
        order, seen = [], set()

        def close(g, m):
            if (g, m) in seen:
                return
            if sum(g) > 0:
                for d in self._step_deps(g, m):
                    close(*d)
            seen.add((g, m))
            order.append((g, m))

        for g, m in sorted(need, key=lambda t: (sum(t[0]), t)):
            close(g, m)
        self.tower_nodes = order
        self.tower_maxm = max(m for (g, m) in order)

    # ---------------------------------------------------------- lane tables
    def lane_index(self, x):
        return self.lanes.index(x) if x in self.lanes else -1

    def lane_static(self, k):
        x = self.lanes[k]
        src, jdir = [], []
        for i in range(3):
            if x[i] > 0:
                x1 = sub1(x, i)
                s = self.lane_index(x1)
                src.append(s if s >= 0 else k)
                jdir.append(first_nz(x1) if (sum(x) == self.lam and self.derive and sum(x1) == 1) else -1)
            else:
                src.append(k)
                jdir.append(-1)
        cd = [-1] * 4
        ck = [0] * 4
        for s, (d, c) in enumerate(self.chain[k]):
            cd[s] = d
            ck[s] = c
        tidx = self.xtargets.index(x) if x in self.xtargets else -1
        return dict(x=x, level=sum(x), src=src, jdir=jdir, cdir=cd, ck=ck, tidx=tidx)

    def name(self):
        return "".join("spd"[l] for l in self.cls) + f"_o{self.ori}"


# ======================================================================
# Python emulator (test infrastructure for the schedule)
# ======================================================================

def emulate(plan: ColumnPlan, q: dict, F: list):
    """Run the column schedule for one quartet over plan.NL emulated lanes.
    q: quartet scalars (PAx.., WPx.., QCx.., WQx.., inv2z, inv2e, inv2ze, rz, re).
    Returns {(x, y): [x|y]^0} for x in lane targets, y in step targets."""
    if plan.orient == 0:
        PX, WX, i2X, rX = [q["PA" + c] for c in XYZ], [q["WP" + c] for c in XYZ], q["inv2z"], q["rz"]
        PY, WY, i2Y, rY = [q["QC" + c] for c in XYZ], [q["WQ" + c] for c in XYZ], q["inv2e"], q["re"]
    else:
        PX, WX, i2X, rX = [q["QC" + c] for c in XYZ], [q["WQ" + c] for c in XYZ], q["inv2e"], q["re"]
        PY, WY, i2Y, rY = [q["PA" + c] for c in XYZ], [q["WP" + c] for c in XYZ], q["inv2z"], q["rz"]
    cpl = q["inv2ze"]
    NL = plan.NL
    lanes = [plan.lane_static(k) for k in range(NL)]
    # chain
    cols = []
    for k in range(NL):
        st = lanes[k]
        b = [F[m] for m in range(plan.chain_m[0] + 1)]
        p = [0.0] * len(b)
        for s in range(1, plan.chain_len + 1):
            d = st["cdir"][s - 1]
            M = plan.chain_m[s]
            if d >= 0:
                kk = st["ck"][s - 1] * i2X
                n = [PX[d] * b[m] + WX[d] * b[m + 1] + kk * (p[m] - rX * p[m + 1]) for m in range(M + 1)]
                p, b = b, n + [0.0] * (len(b) - len(n))
        col = {((0, 0, 0), m): b[m] for m in range(plan.Mb + 1)}
        cols.append(col)
    # tower (uniform)
    T = {((0, 0, 0), m): F[m] for m in range(plan.L + 1)}
    for (g, m) in plan.tower_nodes:
        if sum(g) == 0:
            continue
        i = first_nz(g)
        g1 = sub1(g, i)
        v = PY[i] * T[(g1, m)] + WY[i] * T[(g1, m + 1)]
        if g1[i] > 0:
            g2 = sub1(g1, i)
            v += g1[i] * i2Y * (T[(g2, m)] - rY * T[(g2, m + 1)])
        T[(g, m)] = v
    # steps
    for (y, m) in plan.step_nodes:
        i = first_nz(y)
        y1 = sub1(y, i)
        shuf = [cols[lanes[k]["src"][i]].get((y1, m + 1), 0.0) for k in range(NL)]
        newv = []
        for k in range(NL):
            st = lanes[k]
            c = cols[k]
            v = PY[i] * c[(y1, m)] + WY[i] * c[(y1, m + 1)]
            if y1[i] > 0:
                y2 = sub1(y1, i)
                v += y1[i] * i2Y * (c[(y2, m)] - rY * c[(y2, m + 1)])
            cp = shuf[k]
            if plan.need_derived[(y, m)] and st["level"] == plan.lam and st["jdir"][i] >= 0:
                j = st["jdir"][i]
                g = y1
                cp = PX[j] * T[(g, m + 1)] + WX[j] * T[(g, m + 2)]
                if g[j] > 0:
                    cp += g[j] * cpl * T[(sub1(g, j), m + 2)]
            v += st["x"][i] * cpl * cp
            newv.append(v)
        for k in range(NL):
            cols[k][(y, m)] = newv[k]
    out = {}
    for k in range(NL):
        x = lanes[k]["x"]
        if x in plan.xtargets:
            for y in plan.ytargets:
                out[(x, y)] = cols[k][(y, 0)]
    return out


# ======================================================================
# CUDA emitter
# ======================================================================

K_JCHUNK = 256            # jk_kernels.cuh
K_SMEM_LIMIT = 48 * 1024  # static shared memory of one kernel


def k_smem_bytes(plan: ColumnPlan, warps: int = 4) -> int:
    """Static shared memory of the exchange column kernels: the lane-side HRR
    rows U and the block's reduction buffer share one array (red is written
    only after the block's last quartet), plus the chunk tables."""
    if not plan.applies:
        return 1 << 30
    na, nb, nc, nd = ((l + 1) * (l + 2) // 2 for l in plan.cls)
    n2 = nc * nd if plan.orient == 0 else na * nb
    nacc = na if plan.orient == 0 else nc
    U = warps * plan.P * len(plan.xtargets) * (n2 | 1) * 8
    red = warps * plan.P * n2 * nacc * 8
    return max(U, red) + 4 * (K_JCHUNK + 1) * 4


def k_fits(plan: ColumnPlan) -> bool:
    return plan.applies and k_smem_bytes(plan) <= K_SMEM_LIMIT


def k_variants(la, lb, lc, ld, spilling=False):
    """Exchange kernel variants (schedule values) built for a class: 0 thread
    per quartet (unless its code spills), 1 / 2 column with bra / ket lanes,
    3 / 4 the contracted-partner column kernels, 5 / 6 packed column plans
    (kinds 2 / 3), 7 / 8 packed plans on the second centre (kinds 4 / 5),
    9..12 the contracted-partner kernels of kinds 2..5."""
    out = [] if spilling else [0]
    for ori in (0, 1):
        if k_fits(ColumnPlan(la, lb, lc, ld, ori)):
            out += [1 + ori, 3 + ori]
    for ori in (2, 3, 4, 5):
        if k_fits(ColumnPlan(la, lb, lc, ld, ori)):
            out += [ori + 3, ori + 7]
    return sorted(out)


def _yname(y):
    return f"{y[0]}{y[1]}{y[2]}"


def emit_cuda(plan: ColumnPlan, T: str = "double", with_tables: bool = True, acc: bool = False):
    """Device function col_vrr<LA,LB,LC,LD,ORI>(q, F, ln, out): out[t] = [x|y_t]^0 for
    the lane's component x and the step-side targets y_t (plan.ytargets order).
    Also the lane table col_tab<...> (plan.NL rows of 20 int8).  With acc, the
    function is col_vrr_acc(q, F, ln, out, w) and adds w * [x|y_t]^0 to out[t]
    (primitive quartets summed before the HRR)."""
    la, lb, lc, ld = plan.cls
    ori = plan.ori
    TT = T
    lit = "f" if T == "float" else ""
    T = f"{la}, {lb}, {lc}, {ld}, {ori}"
    if not plan.applies:
        if not with_tables:
            return ""
        return "\n".join([f"template <> struct ColTab<{T}> {{",
                          "    static constexpr int NL = 1, P = 1, NXT = 1, NYT = 1, LAM = 0;",
                          "    static constexpr bool K_FITS = false;  // plan kind not built for this class",
                          "};", ""])
    if plan.orient == 0:
        PX, WX, i2X, rX = ["q.PAx", "q.PAy", "q.PAz"], ["q.WPx", "q.WPy", "q.WPz"], "q.inv2z", "q.rz"
        PY, WY, i2Y, rY = ["q.QCx", "q.QCy", "q.QCz"], ["q.WQx", "q.WQy", "q.WQz"], "q.inv2e", "q.re"
    else:
        PX, WX, i2X, rX = ["q.QCx", "q.QCy", "q.QCz"], ["q.WQx", "q.WQy", "q.WQz"], "q.inv2e", "q.re"
        PY, WY, i2Y, rY = ["q.PAx", "q.PAy", "q.PAz"], ["q.WPx", "q.WPy", "q.WPz"], "q.inv2z", "q.rz"
    L = []
    rows = []
    for k in range(plan.NL if with_tables else 0):
        st = plan.lane_static(k)
        row = list(st["x"]) + st["src"] + st["jdir"] + st["cdir"] + st["ck"] + [st["level"], st["tidx"], 0]
        rows.append("{" + ", ".join(str(v) for v in row) + "}")
    if with_tables:
        L.append(f"template <> struct ColTab<{T}> {{")
        L.append(f"    static constexpr int NL = {plan.NL}, P = {plan.P}, NXT = {len(plan.xtargets)}, "
                 f"NYT = {len(plan.ytargets)}, LAM = {plan.lam};")
        L.append(f"    static constexpr bool K_FITS = {'true' if k_fits(plan) else 'false'};"
                 f"  // exchange kernel shared memory: {k_smem_bytes(plan)} bytes")
        L.append("};")
        L.append(f"__device__ const int8_t col_tab_{plan.name()}[{plan.NL}][20] = {{" + ", ".join(rows) + "};")
        L.append(f"template <> __device__ __forceinline__ const int8_t* col_tab_ptr<{T}>() "
                 f"{{ return &col_tab_{plan.name()}[0][0]; }}")
        L.append("")
    if acc:
        L.append(f"template <> __device__ __forceinline__ void col_vrr_acc<{T}, {TT}>(const QVT<{TT}>& q, "
                 f"const {TT}* F, const ColLane& ln, {TT}* out, {TT} w)")
    else:
        L.append(f"template <> __device__ __forceinline__ void col_vrr<{T}, {TT}>(const QVT<{TT}>& q, const {TT}* F, "
                 f"const ColLane& ln, {TT}* out)")
    L.append("{")
    L.append(f"    const {TT} cpl = q.inv2ze;")
    L.append(f"    const {TT} cp0 = ({TT})ln.xi[0] * cpl, cp1 = ({TT})ln.xi[1] * cpl, cp2 = ({TT})ln.xi[2] * cpl;")
    L.append("    (void)cp0; (void)cp1; (void)cp2;")
    # chain
    M0 = plan.chain_m[0]
    for m in range(M0 + 2):
        L.append(f"    {TT} b{m} = {'F[' + str(m) + ']' if m <= M0 else '0'}, p{m} = 0;")
    for s in range(1, plan.chain_len + 1):
        M = plan.chain_m[s]
        L.append("    {")
        L.append(f"        const int d = ln.cdir[{s - 1}];")
        L.append("        const bool act = d >= 0;")
        L.append(f"        const {TT} Pd = d == 0 ? {PX[0]} : (d == 1 ? {PX[1]} : {PX[2]});")
        L.append(f"        const {TT} Wd = d == 0 ? {WX[0]} : (d == 1 ? {WX[1]} : {WX[2]});")
        L.append(f"        const {TT} kd = ({TT})ln.ck[{s - 1}] * {i2X};")
        for m in range(M + 1):
            L.append(f"        const {TT} n{m} = fma(kd, fma(-{rX}, p{m + 1}, p{m}), fma(Pd, b{m}, Wd * b{m + 1}));")
        for m in range(M + 1):
            L.append(f"        p{m} = act ? b{m} : p{m}; b{m} = act ? n{m} : b{m};")
        L.append("    }")
    cname = {}
    for m in range(plan.Mb + 1):
        cname[((0, 0, 0), m)] = f"b{m}"
    # tower
    tname = {((0, 0, 0), m): f"F[{m}]" for m in range(plan.L + 1)}
    for (g, m) in plan.tower_nodes:
        if sum(g) == 0:
            continue
        i = first_nz(g)
        g1 = sub1(g, i)
        e = f"fma({WY[i]}, {tname[(g1, m + 1)]}, {PY[i]} * {tname[(g1, m)]})"
        if g1[i] > 0:
            g2 = sub1(g1, i)
            e = f"fma({g1[i]}.0{lit} * {i2Y}, fma(-{rY}, {tname[(g2, m + 1)]}, {tname[(g2, m)]}), {e})"
        nm = f"t{_yname(g)}_{m}"
        L.append(f"    const {TT} {nm} = {e};")
        tname[(g, m)] = nm
    if plan.derive:
        L.append("    // level-lam lanes: coupling partners of level lam-1 derived from the tower")
        for i in range(3):
            L.append(f"    const int jd{i} = ln.jdir[{i}];")
            L.append(f"    const {TT} jP{i} = jd{i} == 0 ? {PX[0]} : (jd{i} == 1 ? {PX[1]} : {PX[2]});")
            L.append(f"    const {TT} jW{i} = jd{i} == 0 ? {WX[0]} : (jd{i} == 1 ? {WX[1]} : {WX[2]});")
    # steps
    for (y, m) in plan.step_nodes:
        i = first_nz(y)
        y1 = sub1(y, i)
        nm = f"c{_yname(y)}_{m}"
        # every lane at level lam (a packed plan over one level): the
        # coupling source is always derived, no lane owns level lam - 1
        one_level = plan.lx1 == plan.lam
        if one_level:
            cp = f"0.0{lit}"
        else:
            L.append(f"    const {TT} sh_{nm} = __shfl_sync(0xffffffffu, {cname[(y1, m + 1)]}, ln.src[{i}]);")
            cp = f"sh_{nm}"
        if plan.need_derived[(y, m)]:
            g = y1
            gj = f"(jd{i} == 0 ? {g[0]}.0{lit} : (jd{i} == 1 ? {g[1]}.0{lit} : {g[2]}.0{lit}))"
            tl = []
            for j in range(3):
                tl.append(tname[(sub1(g, j), m + 2)] if g[j] > 0 else f"0.0{lit}")
            tsel = f"(jd{i} == 0 ? {tl[0]} : (jd{i} == 1 ? {tl[1]} : {tl[2]}))"
            der = (f"fma({gj} * cpl, {tsel}, fma(jP{i}, {tname[(g, m + 1)]}, jW{i} * {tname[(g, m + 2)]}))")
            if one_level:
                L.append(f"    const {TT} cv_{nm} = {der};")
            else:
                L.append(f"    const {TT} cv_{nm} = ln.lamlane ? {der} : sh_{nm};")
            cp = f"cv_{nm}"
        e = f"fma({WY[i]}, {cname[(y1, m + 1)]}, {PY[i]} * {cname[(y1, m)]})"
        if y1[i] > 0:
            y2 = sub1(y1, i)
            e = f"fma({y1[i]}.0{lit} * {i2Y}, fma(-{rY}, {cname[(y2, m + 1)]}, {cname[(y2, m)]}), {e})"
        e = f"fma(cp{i}, {cp}, {e})"
        L.append(f"    const {TT} {nm} = {e};")
        cname[(y, m)] = nm
    for t, y in enumerate(plan.ytargets):
        if acc:
            L.append(f"    out[{t}] = fma(w, {cname[(y, 0)]}, out[{t}]);")
        else:
            L.append(f"    out[{t}] = {cname[(y, 0)]};")
    L.append("}")
    return "\n".join(L)


def column_classes():
    """Classes generated with column kernels (both orientations)."""
    out = []
    for la in range(3):
        for lb in range(3):
            for lc in range(3):
                for ld in range(3):
                    out.append((la, lb, lc, ld))
    return out


def default_schedule():
    """Kernel variant per class before autotuning.  J: 0 thread-per-quartet,
    1 column.  K: 0 thread-per-quartet, 1 column with bra lanes, 2 column with
    ket lanes.  Column kernels for the classes whose thread kernels spill
    (total angular momentum >= 6 for J, >= 5 for K); for K the orientation that
    keeps more lanes busy and fits in shared memory."""
    j, k = {}, {}
    for cls in column_classes():
        L = sum(cls)
        j[cls] = 1 if L >= 6 else 0
        best = None
        for ori in (0, 1):
            p = ColumnPlan(*cls, ori)
            if not k_fits(p):
                continue
            util = p.P * p.NL / 32.0
            key = (-util, len(p.step_nodes) + len(p.tower_nodes))
            if best is None or key < best[0]:
                best = (key, ori)
        k[cls] = (1 + best[1]) if (L >= 5 and best is not None) else 0
    return j, k


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    j, k = default_schedule()
    lines = ["// Generated by gen_column.py -- do not edit.",
             "// default kernel variant per class, index la*27 + lb*9 + lc*3 + ld"]
    lines.append("static const int kDefaultScheduleJ[81] = {" + ", ".join(str(j[c]) for c in column_classes()) + "};")
    lines.append("static const int kDefaultScheduleK[81] = {" + ", ".join(str(k[c]) for c in column_classes()) + "};")
    text = "\n".join(lines) + "\n"
    path = os.path.join(outdir, "schedule_default.inc")
    if not (os.path.exists(path) and open(path).read() == text):
        with open(path, "w") as fh:
            fh.write(text)
    for cls in column_classes():
        name = "".join("spd"[l] for l in cls)
        parts = ["// Generated by gen_column.py -- do not edit.", "#pragma once", "namespace vlxb {", ""]
        for ori in PLAN_KINDS:
            plan = ColumnPlan(*cls, ori)
            parts.append(emit_cuda(plan, "double", True))
            parts.append("")
            if not plan.applies:
                continue
            parts.append(emit_cuda(plan, "float", False))
            parts.append("")
            parts.append(emit_cuda(plan, "double", False, acc=True))
            parts.append("")
            parts.append(emit_cuda(plan, "float", False, acc=True))
            parts.append("")
        parts.append("}  // namespace vlxb")
        text = "\n".join(parts) + "\n"
        path = os.path.join(outdir, f"col_{name}.cuh")
        if not (os.path.exists(path) and open(path).read() == text):
            with open(path, "w") as fh:
                fh.write(text)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)), "generated"))
