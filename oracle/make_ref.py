"""Recipe for oracle/_ref/libvlxref.so: the reference's own emitted ERI
expressions, compiled for the host.

TEST / BASELINE INFRASTRUCTURE ONLY (see oracle/__init__.py).

    python oracle/make_ref.py --ref <reference tree> [-j N]

(or VLX_REFERENCE_DIR=<reference tree> python oracle/make_ref.py)

For every Coulomb class (36, gen_coulomb.py:47-56) and exchange class (54,
new_exchange_code/gen_eri_exchange.py:39-56) it asks the reference's
eriwriter.write_eri_code (eriwriter.py:35-160) for the class's expression and
writes a C++ unit, oracle/_ref/src/<kind>_<class>.cpp, whose loops restate the
emitted kernel around it (see ref_harness.h).  Units also provide the Schwarz
diagonal of each pair type from the (ab|ab) expressions.  All units are
compiled with g++ -O3 -fopenmp (-march=x86-64-v3, so the library built here
runs on the GPU hosts) and linked with ref_count.cpp into
oracle/_ref/libvlxref.so.  Outputs go only to oracle/_ref/ (git-ignored); the
reference tree is read, never written.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SRC = os.path.join(OUT, "src")
OBJ = os.path.join(OUT, "obj")
LIB = os.path.join(OUT, "libvlxref.so")
ANG = "spd"
LV = {"s": 0, "p": 1, "d": 2}
CXX = ["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-std=c++17", "-w"]


def j_classes():
    pairs = [a + b for i, a in enumerate(ANG) for b in ANG[i:]]
    return [ab + cd for ab in pairs for cd in pairs]


def k_classes():
    return [a + b + c + d for i, a in enumerate(ANG) for c in ANG[i:] for b in ANG for d in ANG]


def setup_comp(cls, names):
    """Lines declaring a0.., b0.., c0.., d0.. from prim-cart indices names=(i, j, k, l)."""
    out = []
    for x, m, n in zip(cls, "abcd", names):
        lv = LV[x]
        if lv == 0:
            continue
        out.append(f"uint32_t {m}v[2]; comp_vars({lv}, {n}, {m}v);")
        out.append(f"const uint32_t {m}0 = {m}v[0]; (void){m}0;")
        if lv == 2:
            out.append(f"const uint32_t {m}1 = {m}v[1]; (void){m}1;")
    return out


def geom_lines(cls):
    """PA/PB/QC/QD of gen_coulomb.py:194-201, 261-268."""
    a, b, c, d = cls
    out = []
    if a in "pd":
        out.append("const double PA_0 = (a_j * inv_S1) * (r_j[a0] - r_i[a0]);")
    if a == "d":
        out.append("const double PA_1 = (a_j * inv_S1) * (r_j[a1] - r_i[a1]);")
    if b in "pd":
        out.append("const double PB_0 = (-a_i * inv_S1) * (r_j[b0] - r_i[b0]);")
    if b == "d":
        out.append("const double PB_1 = (-a_i * inv_S1) * (r_j[b1] - r_i[b1]);")
    if c in "pd":
        out.append("const double QC_0 = (a_l * inv_S2) * (r_l[c0] - r_k[c0]);")
    if c == "d":
        out.append("const double QC_1 = (a_l * inv_S2) * (r_l[c1] - r_k[c1]);")
    if d in "pd":
        out.append("const double QD_0 = (-a_k * inv_S2) * (r_l[d0] - r_k[d0]);")
    if d == "d":
        out.append("const double QD_1 = (-a_k * inv_S2) * (r_l[d1] - r_k[d1]);")
    return out


def j_unit(cls, expr):
    a, b, c, d = cls
    la, lb, lc, ld = (LV[x] for x in cls)
    L = la + lb + lc + ld
    w = "2.0" if c != d else "(static_cast<double>(k != l) + 1.0)"
    body = "\n".join([
        '#include "../../ref_harness.h"',
        "using namespace vlxref;",
        f'extern "C" void vlxref_coulomb_{cls}(double* mat_J, const double* const* info, const uint32_t* count,',
        "    const double* cd_mat_D, const double* ab_mat_Q, const double* cd_mat_Q,",
        "    const uint32_t* ab_first, const uint32_t* ab_second, const double* ab_pdata, uint32_t n_ab,",
        "    const uint32_t* cd_first, const uint32_t* cd_second, const double* cd_pdata, uint32_t n_cd,",
        "    double eri_threshold, const uint32_t* rows, uint32_t nrows, uint64_t max_eval,",
        "    uint64_t* cq_pass, uint64_t* cq_eval)",
        "{",
        "    const double* tab = boys_table();",
        "    const int64_t nwork = rows ? (int64_t)nrows : (int64_t)n_ab;",
        "    uint64_t tot_pass = 0, tot_eval = 0;",
        "#pragma omp parallel for schedule(dynamic, 1) reduction(+ : tot_pass, tot_eval)",
        "    for (int64_t w = 0; w < nwork; w++) {",
        "        const uint32_t ij = rows ? rows[w] : (uint32_t)w;",
        "        // passing prefix of the sorted ket list (the emitted kernel's break point)",
        "        uint32_t lo = 0, hi = n_cd;",
        "        while (lo < hi) { uint32_t mid = (lo + hi) / 2;",
        "            if (fabs(ab_mat_Q[ij] * cd_mat_Q[mid] * cd_mat_D[mid]) <= eri_threshold) hi = mid; else lo = mid + 1; }",
        "        const uint32_t n_eval = (uint64_t)lo < max_eval ? lo : (uint32_t)max_eval;",
        "        tot_pass += lo; tot_eval += n_eval;",
        "        const uint32_t i = ab_first[ij], j = ab_second[ij];",
        f"        const Prim pi = prim(info[{la}], count[{la}], {la}, i), pj = prim(info[{lb}], count[{lb}], {lb}, j);",
        "        const double a_i = pi.a, a_j = pj.a; const double* r_i = pi.r; const double* r_j = pj.r;",
        "        const double S1 = a_i + a_j, inv_S1 = 1.0 / S1; (void)inv_S1;",
        "        const double S_ij_00 = ab_pdata[ij];",
        "        double J_ij = 0.0;",
        "        for (uint32_t kl = 0; kl < n_eval; kl++) {",
        "            if (fabs(ab_mat_Q[ij] * cd_mat_Q[kl] * cd_mat_D[kl]) <= eri_threshold) break;",
        "            const uint32_t k = cd_first[kl], l = cd_second[kl];",
        f"            const Prim pk = prim(info[{lc}], count[{lc}], {lc}, k), pl = prim(info[{ld}], count[{ld}], {ld}, l);",
        "            const double a_k = pk.a, a_l = pl.a; const double* r_k = pk.r; const double* r_l = pl.r;",
        "            const double S_kl_00 = cd_pdata[kl];",
    ] + ["            " + x for x in setup_comp(cls, ("i", "j", "k", "l"))] + [
        "            const double S2 = a_k + a_l, inv_S2 = 1.0 / S2, inv_S4 = 1.0 / (S1 + S2); (void)inv_S2;",
        "            const double PQ[3] = {(a_k * r_k[0] + a_l * r_l[0]) * inv_S2 - (a_i * r_i[0] + a_j * r_j[0]) * inv_S1,",
        "                                  (a_k * r_k[1] + a_l * r_l[1]) * inv_S2 - (a_i * r_i[1] + a_j * r_j[1]) * inv_S1,",
        "                                  (a_k * r_k[2] + a_l * r_l[2]) * inv_S2 - (a_i * r_i[2] + a_j * r_j[2]) * inv_S1};",
        "            const double r2_PQ = PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2];",
        "            const double Lambda = sqrt(4.0 * S1 * S2 * MATH_CONST_INV_PI * inv_S4);",
        f"            double F{L}_t[{L + 1}];",
        f"            boys(F{L}_t, S1 * S2 * inv_S4 * r2_PQ, {L}, tab);",
    ] + ["            " + x for x in geom_lines(cls)] + [
        "            const double eri_ijkl = Lambda * S_ij_00 * S_kl_00 * (",
        expr,
        "            );",
        f"            J_ij += eri_ijkl * cd_mat_D[kl] * {w};",
        "        }",
        "        mat_J[ij] += J_ij;",
        "    }",
        "    if (cq_pass) *cq_pass = tot_pass;",
        "    if (cq_eval) *cq_eval = tot_eval;",
        "}",
    ])
    return body


def k_unit(cls, expr):
    a, b, c, d = cls
    la, lb, lc, ld = (LV[x] for x in cls)
    L = la + lb + lc + ld
    nb, nd = (lb + 1) * (lb + 2) // 2, (ld + 1) * (ld + 2) // 2
    body = "\n".join([
        '#include "../../ref_harness.h"',
        "using namespace vlxref;",
        f'extern "C" void vlxref_exchange_{cls}(double* mat_K, const uint32_t* pair_i, const uint32_t* pair_k,',
        "    uint32_t n_ik, const double* const* info, const uint32_t* const* aoinds, const uint32_t* count,",
        "    double bd_max_D, const double* mat_D_full_AO, uint32_t naos,",
        "    const double* Q_ab, const double* Q_cd, const uint32_t* Dinds_ab, const uint32_t* Dinds_cd,",
        "    const uint32_t* displs_ab, const uint32_t* displs_cd, const uint32_t* counts_ab,",
        "    const uint32_t* counts_cd, const double* pdata_ab, const double* pdata_cd,",
        "    double omega, double eri_threshold, const uint32_t* rows, uint32_t nrows, uint64_t max_eval,",
        "    uint64_t* cq_pass, uint64_t* cq_eval)",
        "{",
        "    const double* tab = boys_table();",
        "    const int64_t nwork = rows ? (int64_t)nrows : (int64_t)n_ik;",
        "    uint64_t tot_pass = 0, tot_eval = 0;",
        "#pragma omp parallel for schedule(dynamic, 1) reduction(+ : tot_pass, tot_eval)",
        "    for (int64_t w = 0; w < nwork; w++) {",
        "        const uint32_t ik = rows ? rows[w] : (uint32_t)w;",
        "        const uint32_t i = pair_i[ik], k = pair_k[ik];",
        "        const uint32_t count_i = counts_ab[i], count_k = counts_cd[k];",
        "        const uint32_t displ_i = displs_ab[i], displ_k = displs_cd[k];",
        "        uint64_t row_pass = 0;",
        "        for (uint32_t j = 0; j < count_i; j++) {",
        "            uint32_t lo = 0, hi = count_k;",
        "            while (lo < hi) { uint32_t mid = (lo + hi) / 2;",
        "                if (fabs(Q_ab[displ_i + j] * Q_cd[displ_k + mid] * bd_max_D) <= eri_threshold) hi = mid; else lo = mid + 1; }",
        "            row_pass += lo;",
        "        }",
        "        uint64_t budget = row_pass < max_eval ? row_pass : max_eval;",
        "        tot_pass += row_pass; tot_eval += budget;",
        f"        const Prim pi = prim(info[{la}], count[{la}], {la}, i), pk = prim(info[{lc}], count[{lc}], {lc}, k);",
        "        const double a_i = pi.a, a_k = pk.a; const double* r_i = pi.r; const double* r_k = pk.r;",
        "        double K_ik = 0.0;",
        "        for (uint32_t j = 0; j < count_i && budget > 0; j++) {",
        "            const double Q_ij = Q_ab[displ_i + j];",
        "            const uint32_t j_prim = Dinds_ab[displ_i + j];",
        f"            const uint32_t j_cgto = aoinds[{lb}][(j_prim / {nb}) + count[{lb}] * (j_prim % {nb})];",
        f"            const Prim pj = prim(info[{lb}], count[{lb}], {lb}, j_prim);",
        "            const double a_j = pj.a; const double* r_j = pj.r;",
        "            const double S1 = a_i + a_j, inv_S1 = 1.0 / S1; (void)inv_S1;",
        "            const double S_ij_00 = pdata_ab[displ_i + j];",
        "            for (uint32_t l = 0; l < count_k && budget > 0; l++) {",
        "                if (fabs(Q_ij * Q_cd[displ_k + l] * bd_max_D) <= eri_threshold) break;",
        "                budget--;",
        "                const uint32_t l_prim = Dinds_cd[displ_k + l];",
        f"                const uint32_t l_cgto = aoinds[{ld}][(l_prim / {nd}) + count[{ld}] * (l_prim % {nd})];",
        f"                const Prim pl = prim(info[{ld}], count[{ld}], {ld}, l_prim);",
        "                const double a_l = pl.a; const double* r_l = pl.r;",
        "                const double S_kl_00 = pdata_cd[displ_k + l];",
    ] + ["                " + x for x in setup_comp(cls, ("i", "j_prim", "k", "l_prim"))] + [
        "                const double S2 = a_k + a_l, inv_S2 = 1.0 / S2, inv_S4 = 1.0 / (S1 + S2); (void)inv_S2;",
        "                const double PQ[3] = {(a_k * r_k[0] + a_l * r_l[0]) * inv_S2 - (a_i * r_i[0] + a_j * r_j[0]) * inv_S1,",
        "                                      (a_k * r_k[1] + a_l * r_l[1]) * inv_S2 - (a_i * r_i[1] + a_j * r_j[1]) * inv_S1,",
        "                                      (a_k * r_k[2] + a_l * r_l[2]) * inv_S2 - (a_i * r_i[2] + a_j * r_j[2]) * inv_S1};",
        "                const double r2_PQ = PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2];",
        "                const double rho = S1 * S2 * inv_S4;",
        "                double d2 = 1.0;",
        "                if (omega != 0.0) d2 = omega * omega / (rho + omega * omega);",
        "                const double Lambda = sqrt(4.0 * rho * d2 * MATH_CONST_INV_PI);",
        f"                double F{L}_t[{L + 1}];",
        f"                boys(F{L}_t, rho * d2 * r2_PQ, {L}, tab);",
        "                if (omega != 0.0) {",
        "                    double dm = d2;",
        f"                    for (int m = 1; m <= {L}; m++) {{ F{L}_t[m] *= dm; dm *= d2; }}",
        "                }",
    ] + ["                " + x for x in geom_lines(cls)] + [
        "                const double eri_ijkl = Lambda * S_ij_00 * S_kl_00 * (",
        expr,
        "                );",
        "                K_ik += eri_ijkl * mat_D_full_AO[j_cgto * naos + l_cgto];",
        "            }",
        "        }",
        "        mat_K[ik] += K_ik;",
        "    }",
        "    if (cq_pass) *cq_pass = tot_pass;",
        "    if (cq_eval) *cq_eval = tot_eval;",
        "}",
    ])
    return body


def schwarz_unit(ab, expr):
    """sqrt of the largest bare diagonal (ij|ij) over the pair's components,
    from the (ab|ab) expression, per primitive shell pair (P, Q)."""
    a, b = ab
    la, lb = LV[a], LV[b]
    L = 2 * (la + lb)
    cls = ab + ab
    na, nb = (la + 1) * (la + 2) // 2, (lb + 1) * (lb + 2) // 2
    return "\n".join([
        '#include "../../ref_harness.h"',
        "using namespace vlxref;",
        f'extern "C" void vlxref_schwarz_{ab}(const double* const* info, const uint32_t* count, const uint32_t* P,',
        "    const uint32_t* Q, uint32_t n, double* out)",
        "{",
        "    const double* tab = boys_table();",
        "#pragma omp parallel for schedule(dynamic, 16)",
        "    for (int64_t t = 0; t < (int64_t)n; t++) {",
        "        double best = 0.0;",
        f"        for (uint32_t ca = 0; ca < {na}; ca++)",
        f"        for (uint32_t cb = 0; cb < {nb}; cb++) {{",
        f"            const uint32_t i = P[t] * {na} + ca, j = Q[t] * {nb} + cb, k = i, l = j;",
        f"            const Prim pi = prim(info[{la}], count[{la}], {la}, i), pj = prim(info[{lb}], count[{lb}], {lb}, j);",
        "            const double a_i = pi.a, a_j = pj.a, a_k = pi.a, a_l = pj.a;",
        "            const double* r_i = pi.r; const double* r_j = pj.r; const double* r_k = pi.r; const double* r_l = pj.r;",
        "            const double S1 = a_i + a_j, inv_S1 = 1.0 / S1; (void)inv_S1;",
    ] + ["            " + x for x in setup_comp(cls, ("i", "j", "k", "l"))] + [
        "            const double S2 = a_k + a_l, inv_S2 = 1.0 / S2, inv_S4 = 1.0 / (S1 + S2); (void)inv_S2;",
        "            const double PQ[3] = {0.0, 0.0, 0.0};",
        "            const double Lambda = sqrt(4.0 * S1 * S2 * MATH_CONST_INV_PI * inv_S4);",
        f"            double F{L}_t[{L + 1}];",
        f"            boys(F{L}_t, 0.0, {L}, tab);",
    ] + ["            " + x for x in geom_lines(cls)] + [
        "            const double v = Lambda * (",
        expr,
        "            );",
        "            best = fmax(best, fabs(v));",
        "        }",
        "        out[t] = sqrt(best);",
        "    }",
        "}",
    ])


def write_if_changed(path, text):
    if os.path.exists(path) and open(path).read() == text:
        return
    with open(path, "w") as fh:
        fh.write(text)


def compile_one(src):
    obj = os.path.join(OBJ, os.path.basename(src)[:-4] + ".o")
    deps = [src, os.path.join(HERE, "ref_harness.h")]
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    subprocess.run(CXX + ["-c", src, "-o", obj], check=True)
    return obj


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("VLX_REFERENCE_DIR"),
                    help="the vlx-twoe-ints source tree (default: $VLX_REFERENCE_DIR)")
    ap.add_argument("-j", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    if not args.ref or not os.path.isdir(args.ref):
        print(f"reference tree {args.ref} not found; oracle/_ref left as is")
        return 0
    os.makedirs(SRC, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    sys.path.insert(0, args.ref)
    from eriwriter import write_eri_code  # the reference's own expression writer

    cache = {}

    def expr(cls):
        if cls not in cache:
            cache[cls] = write_eri_code(cls, indent=16)
        return cache[cls]

    srcs = []
    for cls in j_classes():
        p = os.path.join(SRC, f"j_{cls}.cpp")
        write_if_changed(p, j_unit(cls, expr(cls)))
        srcs.append(p)
    for cls in k_classes():
        p = os.path.join(SRC, f"k_{cls}.cpp")
        write_if_changed(p, k_unit(cls, expr(cls)))
        srcs.append(p)
    for ab in ("ss", "sp", "sd", "pp", "pd", "dd"):
        p = os.path.join(SRC, f"q_{ab}.cpp")
        write_if_changed(p, schwarz_unit(ab, expr(ab + ab)))
        srcs.append(p)
    srcs.append(os.path.join(HERE, "ref_count.cpp"))
    # largest expressions first
    srcs.sort(key=lambda s: -os.path.getsize(s))
    with cf.ThreadPoolExecutor(max_workers=args.j) as ex:
        objs = list(ex.map(compile_one, srcs))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        subprocess.run(["g++", "-shared", "-fopenmp", "-o", LIB] + objs, check=True)
    print(f"built {LIB}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
