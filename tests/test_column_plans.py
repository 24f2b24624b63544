"""The warp-column VRR schedules (csrc/gen_column.py) against a direct
Obara-Saika recursion, on the CPU.

The generator's Python emulator runs exactly the schedule the CUDA emitter
compiles (lane tables, base chains, step nodes, the uniform tower and the
derived coupling partners of packed plans).  For every exchange class and
every plan kind built for it, the emulated [x|y]^0 of all lane-side and
step-side targets must equal the memoised recursion
  [x|y+1_i]^m = PY_i [x|y]^m + WY_i [x|y]^(m+1)
                + y_i/(2 eta) ([x|y-1_i]^m - rho/eta [x|y-1_i]^(m+1))
                + x_i/(2(zeta+eta)) [x-1_i|y]^(m+1)
(and the same along x for [x|0]^m), with random quartet scalars.
"""
import functools
import os
import sys
import zlib

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "vlx-twoe-ints_b200",
                                "csrc"))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "vlx-twoe-ints_b200"))

import gen_column as gc  # noqa: E402
from vlxb import lists  # noqa: E402

XYZ = "xyz"


def direct(q, F, orient):
    if orient == 0:
        PX, WX, i2X, rX = [q["PA" + c] for c in XYZ], [q["WP" + c] for c in XYZ], q["inv2z"], q["rz"]
        PY, WY, i2Y, rY = [q["QC" + c] for c in XYZ], [q["WQ" + c] for c in XYZ], q["inv2e"], q["re"]
    else:
        PX, WX, i2X, rX = [q["QC" + c] for c in XYZ], [q["WQ" + c] for c in XYZ], q["inv2e"], q["re"]
        PY, WY, i2Y, rY = [q["PA" + c] for c in XYZ], [q["WP" + c] for c in XYZ], q["inv2z"], q["rz"]
    cpl = q["inv2ze"]

    @functools.lru_cache(maxsize=None)
    def v(x, y, m):
        if min(x) < 0 or min(y) < 0:
            return 0.0
        if sum(y) > 0:
            i = next(k for k in range(3) if y[k] > 0)
            y1 = tuple(y[k] - (k == i) for k in range(3))
            y2 = tuple(y1[k] - (k == i) for k in range(3))
            x1 = tuple(x[k] - (k == i) for k in range(3))
            return (PY[i] * v(x, y1, m) + WY[i] * v(x, y1, m + 1)
                    + y1[i] * i2Y * (v(x, y2, m) - rY * v(x, y2, m + 1)) + x[i] * cpl * v(x1, y1, m + 1))
        if sum(x) > 0:
            i = next(k for k in range(3) if x[k] > 0)
            x1 = tuple(x[k] - (k == i) for k in range(3))
            x2 = tuple(x1[k] - (k == i) for k in range(3))
            return PX[i] * v(x1, y, m) + WX[i] * v(x1, y, m + 1) + x1[i] * i2X * (v(x2, y, m) - rX * v(x2, y, m + 1))
        return F[m]

    return v


def _cases():
    out = []
    for cls in lists.k_classes():
        l = tuple({"s": 0, "p": 1, "d": 2}[x] for x in cls)
        for ori in gc.PLAN_KINDS:
            if gc.ColumnPlan(*l, ori).applies:
                out.append((cls, ori))
    return out


@pytest.mark.parametrize("cls,ori", _cases(), ids=[f"{c}-{o}" for c, o in _cases()])
def test_plan_matches_direct_recursion(cls, ori):
    l = tuple({"s": 0, "p": 1, "d": 2}[x] for x in cls)
    plan = gc.ColumnPlan(*l, ori)
    rng = np.random.default_rng(zlib.crc32(f"{cls}{ori}".encode()))
    keys = [p + c for p in ("PA", "WP", "QC", "WQ") for c in XYZ]
    q = {k: float(rng.uniform(-1.0, 1.0)) for k in keys}
    q.update(inv2z=float(rng.uniform(0.2, 1.0)), inv2e=float(rng.uniform(0.2, 1.0)),
             inv2ze=float(rng.uniform(0.1, 0.5)), rz=float(rng.uniform(0.2, 0.8)), re=float(rng.uniform(0.2, 0.8)))
    F = [float(rng.uniform(0.1, 1.0)) / (m + 1) for m in range(plan.L + 1)]
    got = gc.emulate(plan, q, F)
    ref = direct(q, F, plan.orient)
    assert len(got) == len(plan.xtargets) * len(plan.ytargets)
    for (x, y), val in got.items():
        exp = ref(tuple(x), tuple(y), 0)
        assert abs(val - exp) <= 1e-11 * max(1.0, abs(exp)), (cls, ori, x, y, val, exp)


def test_packed_plans_hold_more_quartets_per_warp():
    """PDDD on the d centre and DPDD: 16 lanes (two quartets per warp) where
    the plain plan needs 20 lanes (one quartet); kinds that do not apply are
    reported as such and never compiled."""
    p = gc.ColumnPlan(1, 2, 2, 2, 4)
    assert p.applies and p.NL == 16 and p.P == 2 and p.lx0 == 2 and p.lx1 == 3
    assert gc.ColumnPlan(1, 2, 2, 2, 0).P == 1
    assert gc.ColumnPlan(2, 1, 2, 2, 2).applies and gc.ColumnPlan(2, 1, 2, 2, 2).P == 2
    assert not gc.ColumnPlan(2, 1, 2, 2, 4).applies  # second shell lower: not built
    assert not gc.ColumnPlan(2, 2, 2, 2, 2).applies  # 31 lanes either way
    assert 7 in gc.k_variants(1, 2, 2, 2) and 5 in gc.k_variants(2, 1, 2, 2)


def test_generated_tables_match_variant_list(tmp_path):
    """The ColTab flags the CUDA side dispatches on (K_FITS per class and plan
    kind, written by the generator) agree with the variant list the tuner and
    the tests use, and every built plan fits a warp and the static shared
    memory."""
    import re

    gc.main(str(tmp_path))
    for cls in lists.k_classes():
        l = tuple({"s": 0, "p": 1, "d": 2}[x] for x in cls)
        text = (tmp_path / f"col_{cls}.cuh").read_text()
        fits = {}
        for m in re.finditer(r"struct ColTab<(\d), (\d), (\d), (\d), (\d)> \{\s*static constexpr int NL = (\d+), "
                             r"P = (\d+).*?K_FITS = (true|false)", text, re.S):
            ori, nl, p = int(m.group(5)), int(m.group(6)), int(m.group(7))
            fits[ori] = m.group(8) == "true"
            if fits[ori]:
                assert nl * p <= 32
                assert gc.k_smem_bytes(gc.ColumnPlan(*l, ori)) <= gc.K_SMEM_LIMIT
        assert sorted(fits) == list(gc.PLAN_KINDS), cls
        kv = set(gc.k_variants(*l))
        for ori in (0, 1):
            assert fits[ori] == ({1 + ori, 3 + ori} <= kv), (cls, ori)
        for ori in (2, 3, 4, 5):
            assert fits[ori] == ({ori + 3, ori + 7} <= kv), (cls, ori)


def _hrr(col, R, l1, l2):
    """(x y| for x of level l1, y of level l2 from e = x + y values on the
    first centre: (x, y + 1_i) = (x + 1_i, y) + R_i (x, y), R = first - second."""

    @functools.lru_cache(maxsize=None)
    def h(x, y):
        if sum(y) == 0:
            return col[x]
        i = next(k for k in range(3) if y[k] > 0)
        y1 = tuple(y[k] - (k == i) for k in range(3))
        x1 = tuple(x[k] + (k == i) for k in range(3))
        return h(x1, y1) + R[i] * h(x, y1)

    return {(x, y): h(tuple(x), tuple(y)) for x in gc.level_comps(l1, l1) for y in gc.level_comps(l2, l2)}


@pytest.mark.parametrize("cls,ori", [("pddd", 4), ("pdpd", 4), ("pdpd", 5), ("sddd", 4)])
def test_second_centre_plan_gives_the_same_integrals(cls, ori):
    """A second-centre plan (the lane-side pair built on B, or D) with PA
    turned into PB = PA + AB and the HRR run from B to A with R = BA, read
    transposed, gives the plain plan's (a b| (or |c d)) for every step-side
    target: the transformation the column kernels apply before and after the
    packed VRR."""
    l = tuple({"s": 0, "p": 1, "d": 2}[x] for x in cls)
    orient = ori % 2
    plain, swapped = gc.ColumnPlan(*l, orient), gc.ColumnPlan(*l, ori)
    assert swapped.applies
    rng = np.random.default_rng(zlib.crc32(f"swap{cls}{ori}".encode()))
    keys = [p + c for p in ("PA", "WP", "QC", "WQ") for c in XYZ]
    q = {k: float(rng.uniform(-1.0, 1.0)) for k in keys}
    q.update(inv2z=float(rng.uniform(0.2, 1.0)), inv2e=float(rng.uniform(0.2, 1.0)),
             inv2ze=float(rng.uniform(0.1, 0.5)), rz=float(rng.uniform(0.2, 0.8)), re=float(rng.uniform(0.2, 0.8)))
    R = [float(v) for v in rng.uniform(-1.0, 1.0, 3)]  # AB (orientation 0) or CD (orientation 1)
    F = [float(rng.uniform(0.1, 1.0)) / (m + 1) for m in range(plain.L + 1)]
    P = "PA" if orient == 0 else "QC"
    q2 = dict(q)
    for t, c in enumerate(XYZ):
        q2[P + c] = q[P + c] + R[t]
    a = gc.emulate(plain, q, F)
    b = gc.emulate(swapped, q2, F)
    l1, l2 = (l[0], l[1]) if orient == 0 else (l[2], l[3])
    for y in plain.ytargets:
        ab = _hrr({x: a[(x, y)] for x in plain.xtargets}, R, l1, l2)
        ba = _hrr({x: b[(x, y)] for x in swapped.xtargets}, [-r for r in R], l2, l1)
        for (x1, x2), v in ab.items():
            w = ba[(x2, x1)]
            assert abs(v - w) <= 1e-11 * max(1.0, abs(v)), (cls, ori, x1, x2, y, v, w)
