"""Writes the C-ABI boundary of the engine.

Outputs:
  include/vlxb.h                  public C header (committed)
  csrc/generated/abi.cu           the extern "C" entry points
  csrc/generated/cls_<abcd>_j.cu  one translation unit per Coulomb class
  csrc/generated/cls_<abcd>_k.cu  one translation unit per exchange class

Entry-point names and argument lists mirror the kernels the reference
generator emits, so a caller that binds those kernels binds these instead:
  computeCoulombFock<ABCD>   gen_coulomb.py:74-93, classes gen_coulomb.py:47-56
  computeExchangeFock<ABCD>  gen_exchange.py:75-115 (identical in
                             new_exchange_code/exchangefockwriter.py:55-104),
                             classes new_exchange_code/gen_eri_exchange.py:39-56
plus vlxb_computeCoulombGradient<ABCD> (bra-centre derivatives of J, the
generator's unused gradient='a'/'b' terms, eri.py:85-129) with the J arguments
and vlxb_computeExchangeGradient<ABCD> (energy-weighted centre derivatives of K,
gradient='a'/'c', eri.py:85-152, McMurchie-Davidson form) with the K arguments.
Each entry point takes one extra trailing argument, the CUDA stream (void*,
NULL = default stream), and returns a status code instead of void.
"""
from __future__ import annotations

import os
import sys

ANG = "spd"     # the classes the reference emits (the drop-in set)
ANG_F = "spdf"  # with the f classes, this library's own entry points
LV = {"s": 0, "p": 1, "d": 2, "f": 3}


def j_classes(ang=ANG):
    pairs = [a + b for i, a in enumerate(ang) for b in ang[i:]]
    return [ab + cd for ab in pairs for cd in pairs]


def k_classes(ang=ANG):
    out = []
    for i, a in enumerate(ang):
        for c in ang[i:]:
            for b in ang:
                for d in ang:
                    out.append(a + b + c + d)
    return out


def jf_classes():
    """Coulomb classes with at least one f shell (64)."""
    return [c for c in j_classes(ANG_F) if "f" in c]


def kf_classes():
    """Exchange classes with at least one f shell (106)."""
    return [c for c in k_classes(ANG_F) if "f" in c]


def j_params(cls):
    a, b, c, d = cls
    p = ["double* mat_J"]
    for x in ANG_F:
        if x in cls:
            p += [f"const double* {x}_prim_info", f"uint32_t {x}_prim_count"]
    p += [f"const double* {c}{d}_mat_D", f"const double* {a}{b}_mat_Q_local", f"const double* {c}{d}_mat_Q",
          f"const uint32_t* {a}{b}_first_inds_local", f"const uint32_t* {a}{b}_second_inds_local",
          f"const double* {a}{b}_pair_data_local", f"uint32_t {a}{b}_prim_pair_count_local",
          f"const uint32_t* {c}{d}_first_inds", f"const uint32_t* {c}{d}_second_inds",
          f"const double* {c}{d}_pair_data", f"uint32_t {c}{d}_prim_pair_count",
          "const double* boys_func_table", "const double* boys_func_ft", "double eri_threshold",
          "void* stream"]
    return p


def g_params(cls):
    """Coulomb gradient: the J arguments with mat_J replaced by the derivative
    output and its component stride."""
    return ["double* grad_J", "uint64_t grad_stride"] + j_params(cls)[1:]


def k_params(cls):
    a, b, c, d = cls
    same = (c + d) == (a + b)
    p = ["double* mat_K", f"const uint32_t* pair_inds_i_for_K_{a}{c}", f"const uint32_t* pair_inds_k_for_K_{a}{c}",
         f"uint32_t pair_inds_count_for_K_{a}{c}"]
    for x in ANG_F:
        if x in cls:
            p += [f"const double* {x}_prim_info", f"const uint32_t* {x}_prim_aoinds", f"uint32_t {x}_prim_count"]
    p += [f"double {b}{d}_max_D", "const double* mat_D_full_AO", "uint32_t naos"]
    for typ, nm in (("const double*", "Q_K"), ("const uint32_t*", "D_inds_K"), ("const uint32_t*", "pair_displs_K"),
                    ("const uint32_t*", "pair_counts_K"), ("const double*", "pair_data_K")):
        p.append(f"{typ} {nm}_{a}{b}")
        if not same:
            p.append(f"{typ} {nm}_{c}{d}")
    p += ["const double* boys_func_table", "const double* boys_func_ft", "double omega", "double eri_threshold",
          "void* stream"]
    return p


def kg_params(cls):
    """Exchange gradient: the K arguments with mat_K replaced by the derivative
    output and its component stride."""
    return ["double* grad_K", "uint64_t grad_stride"] + k_params(cls)[1:]


def pname(p):
    return p.split()[-1]


def header():
    L = ["/*",
         " * vlxb.h -- C ABI of the B200 (sm_100a) two-electron J/K engine.",
         " *",
         " * Drop-in for the CUDA/HIP kernels that VeloxChem's vlx-twoe-ints generator",
         " * emits.  Every computeCoulombFock<ABCD> / computeExchangeFock<ABCD> kernel of",
         " * the reference has one entry point here, vlxb_computeCoulombFock<ABCD> /",
         " * vlxb_computeExchangeFock<ABCD>, with the same arguments in the same order and",
         " * the same meaning, plus a trailing CUDA stream (void*, NULL = default stream).",
         " *",
         " * Conventions (as for the reference kernels):",
         " *  - every pointer is caller-owned DEVICE memory; mat_J / mat_K are accumulated",
         " *    with += (zero them first for a fresh build);",
         " *  - prim-cart index i of type x is primitive shell i / ncart(x), Cartesian",
         " *    component i % ncart(x) (p: x,y,z; d: xx,xy,xz,yy,yz,zz);",
         " *  - prim_info is [5][prim_count] (row 0 exponent, rows 2..4 centre);",
         " *    prim_aoinds is [ncart][prim_count] (AO index of each component);",
         " *  - screening keeps a term iff |Q_ij Q_kl D_kl| > eri_threshold (J) or",
         " *    |Q_ij Q_kl max_D| > eri_threshold (K).  This is the set the reference's",
         " *    per-thread `break` selects when its ket/partner lists are sorted by",
         " *    descending bound; here no ordering of the input lists is required.",
         " *  - boys_func_table / boys_func_ft are accepted for signature compatibility",
         " *    and ignored: the engine carries its own FP64 Boys table.",
         " *  - work is enqueued on `stream`; calls do not synchronise the host.",
         " *    Scratch comes from the device's default memory pool (cudaMallocAsync).",
         " *  - return value: VLXB_OK or an error code (never traps).",
         " */",
         "#ifndef VLXB_H", "#define VLXB_H", "", "#include <stdint.h>", "",
         "#ifdef __cplusplus", 'extern "C" {', "#endif", "",
         "#define VLXB_OK 0", "#define VLXB_EINVAL 1", "#define VLXB_ECUDA 2", "#define VLXB_ENOMEM 3",
         "#define VLXB_ETOOBIG 4", "",
         "/* Select `device`, configure its memory pool and upload the Boys table.",
         "   Call once per device before any stream capture.  No reference",
         "   counterpart (the reference's caller owns its Boys table). */",
         "int vlxb_init(int device);", "",
         "/* Human-readable text for a status code.  No reference counterpart. */",
         "const char* vlxb_status_string(int status);", "",
         "/* ABI version (major * 10000 + minor * 100 + patch).  No reference counterpart. */",
         "int vlxb_version(void);", "",
         "/* Schwarz helper for callers that build the lists: for n primitive shell",
         "   pairs (P[t] of type la, Q[t] of type lb, la <= lb <= 3) writes",
         "   out[t] = max over components of sqrt|(ab|ab)| / |S_ab|, S_ab the pair",
         "   prefactor.  The reference's caller computes its Q_ij outside the",
         "   generator (inputs ab_mat_Q_local, Q_K_ab of gen_coulomb.py:81,",
         "   gen_exchange.py:92), so this has no counterpart in the reference. */",
         "int vlxb_schwarzBareMax(int la, int lb, const double* info_a, uint32_t cnt_a, const double* info_b,",
         "                        uint32_t cnt_b, const uint32_t* P, const uint32_t* Q, uint32_t n, double* out,",
         "                        void* stream);", "",
         "/* Screened-in primitive shell quartets processed by the J ([0]) and K ([1])",
         "   kernels on the current device since the last reset.  Reads into host_out",
         "   (2 values; synchronises `stream`) when host_out is not NULL, then zeroes",
         "   the counters when reset != 0.  No reference counterpart. */",
         "int vlxb_quartetCounters(unsigned long long* host_out, int reset, void* stream);", "",
         "/* Device error word of the kernels (flags OR-ed in on the device): bit 0 =",
         "   a bulk copy into shared memory (J schedule variant 3) did not land within",
         "   its bounded wait; the kernel then stopped without finishing its work.",
         "   Reads it into *host_out (if non-NULL, synchronising `stream`) and zeroes it",
         "   if `reset`.  No reference counterpart. */",
         "int vlxb_kernelErrors(unsigned long long* host_out, int reset, void* stream);", "",
         "/* Number of this library's own kernel launches since the last reset",
         "   (host-side count; reset != 0 zeroes it after reading).  No reference",
         "   counterpart. */",
         "int vlxb_launchCount(unsigned long long* out, int reset);", "",
         "/* FP64 FMA throughput probe: `blocks` x 256 threads, each running 8",
         "   independent fma chains of `iters` steps (2*8*iters flops per thread);",
         "   out needs blocks*256 doubles.  Used by the benchmark to measure the",
         "   DFMA peak.  No reference counterpart. */",
         "int vlxb_fp64Probe(double* out, int iters, int blocks, void* stream);", "",
         "/* Kernel variant used for one class (kind 0 = Coulomb: 0 one thread per",
         "   shell quartet, 1 warp-cooperative column kernel, 2 McMurchie-Davidson",
         "   kernel (Hermite ket densities, one quartet per warp), 3 one thread per",
         "   quartet with the sorted ket stream staged into shared memory by TMA bulk",
         "   copies, double-buffered; kind 1 = exchange: 0",
         "   one thread per quartet, 1 column kernel with bra lanes, 2 column kernel",
         "   with ket lanes, 3 / 4 the column kernels with bra / ket lanes that sum",
         "   the primitive partners of one contracted shell before the HRR, 5 / 6",
         "   packed column kernels with bra / ket lanes (lanes for the target",
         "   levels only, from d up, so that a warp holds two or five quartets;",
         "   the lower levels the VRR couples to are derived in each lane), 7 / 8",
         "   the packed kernels with the lane-side pair built on its second",
         "   centre (p+d and s+d pairs), 9..12 the contracted-partner kernels of",
         "   the packed plans 5..8).  A column variant that is not built for",
         "   the class, or whose kernel does not fit it, falls back to 0.",
         "   Every variant gives the same J/K to rounding; the",
         "   choice only changes speed.  Set by the autotuner.  No reference",
         "   counterpart. */",
         "int vlxb_setSchedule(int kind, int la, int lb, int lc, int ld, int variant);",
         "int vlxb_getSchedule(int kind, int la, int lb, int lc, int ld);", "",
         "/* Mixed precision: shell quartets whose screening bound (|Q_ij| max|Q_kl D_kl|",
         "   for J, |Q_ij Q_kl max_D| for K) is below `cutoff` are evaluated in FP32",
         "   (Boys argument and Boys values in FP64, rounded once), everything else",
         "   and all accumulation in FP64.  0 (the default) = plain FP64, the drop-in",
         "   behaviour.  Process-wide.  No reference counterpart. */",
         "int vlxb_setFp32Cutoff(double cutoff);",
         "double vlxb_getFp32Cutoff(void);", "",
         "/* FP32 error budget (with a cutoff > 0; default 0.2; 0 = no budget, the",
         "   cutoff alone decides).  A quartet below the cutoff runs in FP32 only inside the tail",
         "   of its list whose summed error proxy stays within `budget`: per J bra",
         "   record, |Q_ij| A_ij * sum over the FP32 kets of max|Q_kl D_kl| A_kl; per",
         "   K output block and partner j, |Q_ij| A_ij max_D * sum over the FP32 l",
         "   of |Q_kl| A_kl, against budget / (the block's number of j).  A is the",
         "   growth the horizontal recurrence gives rounding errors across a pair,",
         "   (1 + sqrt(2 zeta) |R|)^l (R = AB or CD, l the momentum it moves).  The",
         "   FP32 error of an output element then scales with the budget, not with",
         "   the number of quartets below the cutoff.  Process-wide.  No reference",
         "   counterpart. */",
         "int vlxb_setFp32Budget(double budget);",
         "double vlxb_getFp32Budget(void);", "",
         "/* Primitive-pair -> AO contraction (the step after the class entry points,",
         "   whose mat_J / mat_K hold one value per list entry, gen_coulomb.py:296,",
         "   gen_exchange.py:341; the reference's caller does it on the host).",
         "   Overwrites mat_AO (naos x naos, row-major) with the symmetric AO matrix",
         "   M[a][b] = M[b][a] = sum of the row of (a, b), a <= b: rows r < n_rows",
         "   with row_ao[r] = a * naos + b and entries rowptr[r] .. rowptr[r+1]-1 of",
         "   src, each the position (bits 0..30) in pair_values of one value and a",
         "   weight flag (bit 31: weight 2, else 1).  Summation order is the stored",
         "   order, so results are bit-reproducible.  No reference counterpart. */",
         "int vlxb_pairsToAO(const double* pair_values, const int64_t* rowptr, const int32_t* row_ao,",
         "                   const uint32_t* src, int64_t n_rows, double* mat_AO, int32_t naos, void* stream);", "",
         "/* SCF energy terms of AO matrices on the device, summed in a fixed order:",
         "   out3[0] = Tr[D J] - Tr[D K] / 2, out3[1] = Tr[D J], out3[2] = Tr[D K]",
         "   (device pointer; J_AO or K_AO may be NULL = zero).  No reference",
         "   counterpart. */",
         "int vlxb_fockEnergy(const double* D_AO, const double* J_AO, const double* K_AO, int32_t naos,",
         "                    double* out3, void* stream);", "",
         "/* Caller-side list inputs on the device (the reference's caller computes",
         "   them outside the generator: pair data, Q, cd_mat_D and bd_max_D of",
         "   gen_coulomb.py:80-90 and gen_exchange.py:78-110).  No reference",
         "   counterpart.",
         "   vlxb_shellPairData: for n primitive shell pairs (P[t] of type la, Q[t]",
         "   of type lb, la <= lb <= 3) S_out[t] = c_P c_Q (pi/p)^(3/2)",
         "   exp(-ab/p |A-B|^2) and q_out[t] = |S_out[t]| * max over components",
         "   sqrt|(ab|ab)| / |S_ab| (the Schwarz value of every component pair).",
         "   vlxb_gatherPairDensity: out[t] = D_AO[ao_a(first[t])][ao_b(second[t])]",
         "   with ao_x(i) = aoinds_x[(i % ncart_x) * cnt_x + i / ncart_x].",
         "   vlxb_blockMaxAbs: *out (device) = max |D_AO[r][c]|, r in rows[0..nrows),",
         "   c in cols[0..ncols). */",
         "int vlxb_shellPairData(int la, int lb, const double* info_a, uint32_t cnt_a, const double* info_b,",
         "                       uint32_t cnt_b, const uint32_t* P, const uint32_t* Q, uint32_t n, double* S_out,",
         "                       double* q_out, void* stream);",
         "int vlxb_gatherPairDensity(const double* D_AO, uint32_t naos, const uint32_t* first, const uint32_t* second,",
         "                           const uint32_t* aoinds_a, int ncart_a, uint32_t cnt_a, const uint32_t* aoinds_b,",
         "                           int ncart_b, uint32_t cnt_b, int64_t n, double* out, void* stream);",
         "int vlxb_blockMaxAbs(const double* D_AO, uint32_t naos, const uint32_t* rows, int64_t nrows,",
         "                     const uint32_t* cols, int64_t ncols, double* out, void* stream);", "",
         "/* Batched class calls: one call of class (la lb|lc ld) covers many",
         "   independent molecules whose lists are concatenated (the union of their",
         "   primitives per type, no pair across two molecules).  No reference",
         "   counterpart (the reference ABI carries no molecule boundaries).",
         "   Coulomb: a bra pairs only with kets of its own molecule (prim_mol[la],",
         "   prim_mol[lc]); the lists are the reference's J lists of the union, the",
         "   result per molecule is the class call of that molecule alone.",
         "   Exchange: the reference's K lists of the union; the density is read as",
         "   D[row][col] with row = prim_aoinds (AO index in the union), col =",
         "   prim_aocols (column in a stack of per-molecule density blocks of row",
         "   stride D_stride), and each output block is screened with its own",
         "   molecule's bound maxD_mol[prim_mol[la][i]].  Unused fields: 0 / NULL. */",
         "typedef struct {",
         "    double* mat;                      /* mat_J or mat_K (accumulated with +=) */",
         "    const double* prim_info[3];       /* union prim_info of s, p, d */",
         "    const uint32_t* prim_aoinds[3];   /* AO index per component (union numbering) */",
         "    const uint32_t* prim_aocols[3];   /* exchange: density column per component */",
         "    uint32_t prim_count[3];",
         "    const int32_t* prim_mol[3];       /* molecule of every primitive */",
         "    int32_t n_mol;",
         "    /* Coulomb (gen_coulomb.py:80-90 arguments of the union) */",
         "    const double *ab_Q, *cd_Q, *cd_D, *ab_pdata, *cd_pdata;",
         "    const uint32_t *ab_first, *ab_second, *cd_first, *cd_second;",
         "    uint32_t n_ab, n_cd;",
         "    /* Exchange (gen_exchange.py:78-110 arguments of the union) */",
         "    const uint32_t *pair_i, *pair_k;",
         "    uint32_t n_ik;",
         "    const double* D;",
         "    uint32_t D_stride;                /* row stride of D */",
         "    uint32_t naos;                    /* AOs of the union (bound on prim_aoinds) */",
         "    const double* maxD_mol;           /* [n_mol] max |D| of each molecule's bd block */",
         "    const double *Q_ab, *Q_cd, *pdata_ab, *pdata_cd;",
         "    const uint32_t *Dinds_ab, *Dinds_cd, *displs_ab, *displs_cd, *counts_ab, *counts_cd;",
         "    double omega;",
         "    double thr;",
         "} VlxbBatchCall;",
         "int vlxb_coulombBatch(int la, int lb, int lc, int ld, const VlxbBatchCall* call, void* stream);",
         "int vlxb_exchangeBatch(int la, int lb, int lc, int ld, const VlxbBatchCall* call, void* stream);", "",
         "/* Allocation-free variant of vlxb_computeCoulombFockSSSS (same arguments,",
         "   same result) for callers that cannot allocate device memory, e.g. hosts",
         "   whose device memory is owned by their own allocator, or plugins that are",
         "   not allowed to allocate.  No counterpart in the reference: the reference's",
         "   emitted kernels need no scratch, this engine's entry points do.  Scratch",
         "   comes from a fixed device array of VLXB_NOALLOC_SCRATCH_BYTES (64 MiB) that",
         "   every GPU loading the library holds until exit; calls needing more",
         "   return VLXB_ETOOBIG before queuing any work.  The first call on a device",
         "   resolves the array and uploads the Boys tables (synchronously): make it",
         "   before any stream capture.  Calls share the array, so calls that overlap",
         "   on the GPU race; serialise them.  Its quartets are not added to the",
         "   counters of vlxb_quartetCounters (those live in allocated memory). */",
         "#define VLXB_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)",
         "int vlxb_computeCoulombFockSSSS_noalloc(" + ", ".join(j_params("ssss")) + ");", ""]
    L.append("/* ---- Coulomb: replace computeCoulombFock<ABCD> of gen_coulomb.py:74-93 ---- */")
    for cls in j_classes():
        L.append(f"/* replaces computeCoulombFock{cls.upper()} (gen_coulomb.py:74-93; class list gen_coulomb.py:47-56) */")
        L.append(f"int vlxb_computeCoulombFock{cls.upper()}(" + ", ".join(j_params(cls)) + ");")
    L.append("")
    L += ["/* ---- Coulomb nuclear gradient ----",
          "   vlxb_computeCoulombGradient<ABCD>: same arguments as",
          "   vlxb_computeCoulombFock<ABCD> with mat_J replaced by grad_J, a",
          "   [6][grad_stride] array (grad_stride >= ab_prim_pair_count_local):",
          "   grad_J[k * grad_stride + o] += d mat_J[o] / d X_k for every bra list entry",
          "   o, X = (A_x, A_y, A_z, B_x, B_y, B_z) the centres of the entry's first and",
          "   second primitive, the ket pairs and cd_mat_D held fixed.  Derivative of",
          "   a Cartesian Gaussian: d/dA_x phi_a = 2 alpha phi_{a+1x} - a_x phi_{a-1x}",
          "   (the reference generator's gradient='a'/'b' terms, eri.py:85-129, which",
          "   no reference generator emits).  Same screening (|Q_ij Q_kl D_kl| >",
          "   eri_threshold), same mixed-precision cutoff as the J entry points.  For",
          "   E_J = 1/2 Tr[D J] every J class's bra derivative weighted by",
          "   w_o D_o (w_o = 1 for a diagonal entry of a same-type list, else 2) sums to",
          "   dE_J/dR, the ket side being the same sum by symmetry.  No reference",
          "   counterpart. */"]
    for cls in j_classes():
        L.append(f"int vlxb_computeCoulombGradient{cls.upper()}(" + ", ".join(g_params(cls)) + ");")
    L += ["",
          "/* Per-atom reduction of pair derivatives (after the gradient entry points):",
          "   grad_atoms[3 * t + x] = sum over CSR entries e in rowptr[t] .. rowptr[t+1]-1",
          "   of weight[p] * pair_grad[(3 * side + x) * grad_stride + p], with",
          "   p = src[e] & 0x7fffffff (< grad_stride) and side = src[e] >> 31 (0:",
          "   first centre, 1: second); weight NULL = 1 (the exchange gradient comes",
          "   weighted).  Overwrites grad_atoms (3 * n_atoms doubles).  Entries are",
          "   summed in a fixed order: results are bit-reproducible.  grad_stride 0",
          "   means an empty CSR (no pair derivatives): grad_atoms is zeroed and",
          "   nothing else is read; otherwise pair_grad and src must be non-NULL.",
          "   No reference counterpart. */",
          "int vlxb_pairGradientToAtoms(const double* pair_grad, uint64_t grad_stride, const double* weight,",
          "                             const int64_t* rowptr, const uint32_t* src, int32_t n_atoms,",
          "                             double* grad_atoms, void* stream);",
          ""]
    L += ["/* ---- Exchange nuclear gradient ----",
          "   vlxb_computeExchangeGradient<ABCD>: same arguments as",
          "   vlxb_computeExchangeFock<ABCD> with mat_K replaced by grad_K, a",
          "   [6][grad_stride] array (grad_stride >= pair_inds_count_for_K_ac).  For",
          "   every primitive shell block (i / ncart_a, k / ncart_c) of the (i, k) list",
          "   it adds, at the block's lowest list position p,",
          "     grad_K[x * grad_stride + p] += sum over the block's entries (i, k) of",
          "       w_ik D_ik sum_jl D_jl d(ij|kl)/dX_x,",
          "   X = (A_x, A_y, A_z, C_x, C_y, C_z) the centres of i and k, D the AO",
          "   density (D_ik = mat_D_full_AO[ao(i)][ao(k)]), w_ik = 1 for i == k of a",
          "   same-type list, else 2; the block's other positions receive nothing,",
          "   so grad_K is meaningful per primitive shell block only (unlike the",
          "   Coulomb gradient's per-entry values): fold it onto atoms with",
          "   vlxb_pairGradientToAtoms (weight NULL), never read it per entry.",
          "   Summed over the 54 classes and credited to the atoms of i (x < 3) and",
          "   k (x >= 3) this is dE_K/dR for E_K = 1/2 Tr[D K] (the j and l centres",
          "   are covered by the symmetry of the sum).  Same screening and omega as",
          "   the K entry points; FP64 whatever the mixed-precision cutoff.  The",
          "   derivative terms are the generator's gradient='a'/'c' terms",
          "   (eri.py:85-152), which no reference generator emits.  No reference",
          "   counterpart. */"]
    for cls in k_classes():
        L.append(f"int vlxb_computeExchangeGradient{cls.upper()}(" + ", ".join(kg_params(cls)) + ");")
    L.append("")
    L.append("/* ---- Exchange: replace computeExchangeFock<ABCD> of gen_exchange.py:75-115 ---- */")
    for cls in k_classes():
        L.append(f"/* replaces computeExchangeFock{cls.upper()} (gen_exchange.py:75-115; "
                 "class list new_exchange_code/gen_eri_exchange.py:39-56) */")
        L.append(f"int vlxb_computeExchangeFock{cls.upper()}(" + ", ".join(k_params(cls)) + ");")
    L += ["", "/* ---- f shells: this library's own entry points ----",
          "   The reference's writer emits s, p and d classes only (eriwriter.py:44-62),",
          "   although its ERI engine takes any number of Cartesian indices (eri.py:59).",
          "   These entry points extend the scheme to f with the same argument",
          "   conventions, f components ordered like d (x^3 first, then by decreasing",
          "   y power: xxx xxy xxz xyy xyz xzz yyy yyz yzz zzz).  One generic kernel per",
          "   kind evaluates them component quartet by component quartet (runtime",
          "   angular momenta, McMurchie-Davidson form); FP64 whatever the",
          "   mixed-precision cutoff; not counted by vlxb_quartetCounters; no",
          "   gradient or batched entry points.  No reference counterpart. */"]
    for cls in jf_classes():
        L.append(f"int vlxb_computeCoulombFock{cls.upper()}(" + ", ".join(j_params(cls)) + ");")
    for cls in kf_classes():
        L.append(f"int vlxb_computeExchangeFock{cls.upper()}(" + ", ".join(k_params(cls)) + ");")
    L += ["", "#ifdef __cplusplus", "}", "#endif", "", "#endif /* VLXB_H */", ""]
    return "\n".join(L)


def abi_cu():
    L = ["// Generated by gen_abi.py -- do not edit.",
         '#include "../classes.cuh"',
         '#include "../../../include/vlxb.h"', "",
         "namespace vlxb {"]
    for cls in j_classes():
        la, lb, lc, ld = (LV[x] for x in cls)
        L.append(f"int coulomb_{cls}(const CoulombArgs&, cudaStream_t);")
    for cls in j_classes():
        L.append(f"int coulomb_grad_{cls}(const CoulombArgs&, int64_t, cudaStream_t);")
    for cls in k_classes():
        L.append(f"int exchange_{cls}(const ExchangeArgs&, cudaStream_t);")
        L.append(f"int exchange_grad_{cls}(const ExchangeArgs&, int64_t, cudaStream_t);")
    L.append("int run_coulomb_f(int la, int lb, int lc, int ld, const CoulombArgs&, cudaStream_t);")
    L.append("int run_exchange_f(int la, int lb, int lc, int ld, const ExchangeArgs&, cudaStream_t);")
    L += ["}  // namespace vlxb", "", 'extern "C" {', ""]
    for cls in jf_classes():
        a, b, c, d = cls
        la, lb, lc, ld = (LV[x] for x in cls)
        L.append(f"int vlxb_computeCoulombFock{cls.upper()}(" + ", ".join(j_params(cls)) + ")")
        L.append("{")
        L.append("    (void)boys_func_table; (void)boys_func_ft;")
        L.append("    vlxb::CoulombArgs A{};")
        L.append("    A.mat_J = mat_J;")
        for x in ANG_F:
            if x in cls:
                L.append(f"    A.info[{LV[x]}] = {x}_prim_info; A.count[{LV[x]}] = {x}_prim_count;")
        L += [f"    A.cd_D = {c}{d}_mat_D; A.ab_Q = {a}{b}_mat_Q_local; A.cd_Q = {c}{d}_mat_Q;",
              f"    A.ab_first = {a}{b}_first_inds_local; A.ab_second = {a}{b}_second_inds_local;",
              f"    A.ab_pdata = {a}{b}_pair_data_local; A.n_ab = {a}{b}_prim_pair_count_local;",
              f"    A.cd_first = {c}{d}_first_inds; A.cd_second = {c}{d}_second_inds;",
              f"    A.cd_pdata = {c}{d}_pair_data; A.n_cd = {c}{d}_prim_pair_count;",
              "    A.thr = eri_threshold;",
              f"    return vlxb::run_coulomb_f({la}, {lb}, {lc}, {ld}, A, (cudaStream_t)stream);", "}", ""]
    for cls in kf_classes():
        a, b, c, d = cls
        la, lb, lc, ld = (LV[x] for x in cls)
        same = (c + d) == (a + b)
        L.append(f"int vlxb_computeExchangeFock{cls.upper()}(" + ", ".join(k_params(cls)) + ")")
        L.append("{")
        L.append("    (void)boys_func_table; (void)boys_func_ft;")
        L.append("    vlxb::ExchangeArgs A{};")
        L.append(f"    A.mat_K = mat_K; A.pair_i = pair_inds_i_for_K_{a}{c}; A.pair_k = pair_inds_k_for_K_{a}{c};")
        L.append(f"    A.n_ik = pair_inds_count_for_K_{a}{c};")
        for x in ANG_F:
            if x in cls:
                L.append(f"    A.info[{LV[x]}] = {x}_prim_info; A.aoinds[{LV[x]}] = {x}_prim_aoinds; "
                         f"A.count[{LV[x]}] = {x}_prim_count;")
        L.append(f"    A.maxD = {b}{d}_max_D; A.D = mat_D_full_AO; A.naos = naos;")
        cd = f"{a}{b}" if same else f"{c}{d}"
        L.append(f"    A.Q_ab = Q_K_{a}{b}; A.Q_cd = Q_K_{cd};")
        L.append(f"    A.Dinds_ab = D_inds_K_{a}{b}; A.Dinds_cd = D_inds_K_{cd};")
        L.append(f"    A.displs_ab = pair_displs_K_{a}{b}; A.displs_cd = pair_displs_K_{cd};")
        L.append(f"    A.counts_ab = pair_counts_K_{a}{b}; A.counts_cd = pair_counts_K_{cd};")
        L.append(f"    A.pdata_ab = pair_data_K_{a}{b}; A.pdata_cd = pair_data_K_{cd};")
        L.append("    A.omega = omega; A.thr = eri_threshold;")
        L.append(f"    return vlxb::run_exchange_f({la}, {lb}, {lc}, {ld}, A, (cudaStream_t)stream);")
        L += ["}", ""]
    for cls in j_classes():
        a, b, c, d = cls
        ps = j_params(cls)
        L.append(f"int vlxb_computeCoulombFock{cls.upper()}(" + ", ".join(ps) + ")")
        L.append("{")
        L.append("    (void)boys_func_table; (void)boys_func_ft;")
        L.append("    vlxb::CoulombArgs A{};")
        L.append("    A.mat_J = mat_J;")
        for x in ANG:
            if x in cls:
                L.append(f"    A.info[{LV[x]}] = {x}_prim_info; A.count[{LV[x]}] = {x}_prim_count;")
        L += [f"    A.cd_D = {c}{d}_mat_D; A.ab_Q = {a}{b}_mat_Q_local; A.cd_Q = {c}{d}_mat_Q;",
              f"    A.ab_first = {a}{b}_first_inds_local; A.ab_second = {a}{b}_second_inds_local;",
              f"    A.ab_pdata = {a}{b}_pair_data_local; A.n_ab = {a}{b}_prim_pair_count_local;",
              f"    A.cd_first = {c}{d}_first_inds; A.cd_second = {c}{d}_second_inds;",
              f"    A.cd_pdata = {c}{d}_pair_data; A.n_cd = {c}{d}_prim_pair_count;",
              "    A.thr = eri_threshold;",
              f"    return vlxb::coulomb_{cls}(A, (cudaStream_t)stream);", "}", ""]
    for cls in j_classes():
        a, b, c, d = cls
        L.append(f"int vlxb_computeCoulombGradient{cls.upper()}(" + ", ".join(g_params(cls)) + ")")
        L.append("{")
        L.append("    (void)boys_func_table; (void)boys_func_ft;")
        L.append("    if (grad_stride > (uint64_t)INT64_MAX) return VLXB_EINVAL;")
        L.append("    vlxb::CoulombArgs A{};")
        L.append("    A.mat_J = grad_J;")
        for x in ANG:
            if x in cls:
                L.append(f"    A.info[{LV[x]}] = {x}_prim_info; A.count[{LV[x]}] = {x}_prim_count;")
        L += [f"    A.cd_D = {c}{d}_mat_D; A.ab_Q = {a}{b}_mat_Q_local; A.cd_Q = {c}{d}_mat_Q;",
              f"    A.ab_first = {a}{b}_first_inds_local; A.ab_second = {a}{b}_second_inds_local;",
              f"    A.ab_pdata = {a}{b}_pair_data_local; A.n_ab = {a}{b}_prim_pair_count_local;",
              f"    A.cd_first = {c}{d}_first_inds; A.cd_second = {c}{d}_second_inds;",
              f"    A.cd_pdata = {c}{d}_pair_data; A.n_cd = {c}{d}_prim_pair_count;",
              "    A.thr = eri_threshold;",
              f"    return vlxb::coulomb_grad_{cls}(A, (int64_t)grad_stride, (cudaStream_t)stream);", "}", ""]
    for cls in k_classes():
        a, b, c, d = cls
        same = (c + d) == (a + b)
        ps = k_params(cls)
        L.append(f"int vlxb_computeExchangeFock{cls.upper()}(" + ", ".join(ps) + ")")
        L.append("{")
        L.append("    (void)boys_func_table; (void)boys_func_ft;")
        L.append("    vlxb::ExchangeArgs A{};")
        L.append(f"    A.mat_K = mat_K; A.pair_i = pair_inds_i_for_K_{a}{c}; A.pair_k = pair_inds_k_for_K_{a}{c};")
        L.append(f"    A.n_ik = pair_inds_count_for_K_{a}{c};")
        for x in ANG:
            if x in cls:
                L.append(f"    A.info[{LV[x]}] = {x}_prim_info; A.aoinds[{LV[x]}] = {x}_prim_aoinds; "
                         f"A.count[{LV[x]}] = {x}_prim_count;")
        L.append(f"    A.maxD = {b}{d}_max_D; A.D = mat_D_full_AO; A.naos = naos;")
        cd = f"{a}{b}" if same else f"{c}{d}"
        L.append(f"    A.Q_ab = Q_K_{a}{b}; A.Q_cd = Q_K_{cd};")
        L.append(f"    A.Dinds_ab = D_inds_K_{a}{b}; A.Dinds_cd = D_inds_K_{cd};")
        L.append(f"    A.displs_ab = pair_displs_K_{a}{b}; A.displs_cd = pair_displs_K_{cd};")
        L.append(f"    A.counts_ab = pair_counts_K_{a}{b}; A.counts_cd = pair_counts_K_{cd};")
        L.append(f"    A.pdata_ab = pair_data_K_{a}{b}; A.pdata_cd = pair_data_K_{cd};")
        L.append("    A.omega = omega; A.thr = eri_threshold;")
        L.append(f"    return vlxb::exchange_{cls}(A, (cudaStream_t)stream);")
        L += ["}", ""]
    for cls in k_classes():
        a, b, c, d = cls
        same = (c + d) == (a + b)
        L.append(f"int vlxb_computeExchangeGradient{cls.upper()}(" + ", ".join(kg_params(cls)) + ")")
        L.append("{")
        L.append("    (void)boys_func_table; (void)boys_func_ft;")
        L.append("    if (grad_stride > (uint64_t)INT64_MAX) return VLXB_EINVAL;")
        L.append("    vlxb::ExchangeArgs A{};")
        L.append(f"    A.mat_K = grad_K; A.pair_i = pair_inds_i_for_K_{a}{c}; A.pair_k = pair_inds_k_for_K_{a}{c};")
        L.append(f"    A.n_ik = pair_inds_count_for_K_{a}{c};")
        for x in ANG:
            if x in cls:
                L.append(f"    A.info[{LV[x]}] = {x}_prim_info; A.aoinds[{LV[x]}] = {x}_prim_aoinds; "
                         f"A.count[{LV[x]}] = {x}_prim_count;")
        L.append(f"    A.maxD = {b}{d}_max_D; A.D = mat_D_full_AO; A.naos = naos;")
        cd = f"{a}{b}" if same else f"{c}{d}"
        L.append(f"    A.Q_ab = Q_K_{a}{b}; A.Q_cd = Q_K_{cd};")
        L.append(f"    A.Dinds_ab = D_inds_K_{a}{b}; A.Dinds_cd = D_inds_K_{cd};")
        L.append(f"    A.displs_ab = pair_displs_K_{a}{b}; A.displs_cd = pair_displs_K_{cd};")
        L.append(f"    A.counts_ab = pair_counts_K_{a}{b}; A.counts_cd = pair_counts_K_{cd};")
        L.append(f"    A.pdata_ab = pair_data_K_{a}{b}; A.pdata_cd = pair_data_K_{cd};")
        L.append("    A.omega = omega; A.thr = eri_threshold;")
        L.append(f"    return vlxb::exchange_grad_{cls}(A, (int64_t)grad_stride, (cudaStream_t)stream);")
        L += ["}", ""]
    # batched calls: runtime class -> the class units
    L += ["int vlxb_coulombBatch(int la, int lb, int lc, int ld, const VlxbBatchCall* c, void* stream)", "{",
          "    if (la < 0 || la > 2 || lb < 0 || lb > 2 || lc < 0 || lc > 2 || ld < 0 || ld > 2) return VLXB_EINVAL;",
          "    if (!c || c->n_mol <= 0 || !c->prim_mol[la] || !c->prim_mol[lc]) return VLXB_EINVAL;",
          "    vlxb::CoulombArgs A{};",
          "    A.mat_J = c->mat;",
          "    for (int l = 0; l < 3; l++) { A.info[l] = c->prim_info[l]; A.count[l] = c->prim_count[l]; }",
          "    A.cd_D = c->cd_D; A.ab_Q = c->ab_Q; A.cd_Q = c->cd_Q;",
          "    A.ab_first = c->ab_first; A.ab_second = c->ab_second; A.ab_pdata = c->ab_pdata; A.n_ab = c->n_ab;",
          "    A.cd_first = c->cd_first; A.cd_second = c->cd_second; A.cd_pdata = c->cd_pdata; A.n_cd = c->n_cd;",
          "    A.thr = c->thr;",
          "    A.prim_mol_a = c->prim_mol[la]; A.prim_mol_c = c->prim_mol[lc]; A.n_mol = c->n_mol;",
          "    switch (la * 27 + lb * 9 + lc * 3 + ld) {"]
    for cls in j_classes():
        la, lb, lc, ld = (LV[x] for x in cls)
        L.append(f"        case {la * 27 + lb * 9 + lc * 3 + ld}: return vlxb::coulomb_{cls}(A, (cudaStream_t)stream);")
    L += ["        default: return VLXB_EINVAL;", "    }", "}", ""]
    L += ["int vlxb_exchangeBatch(int la, int lb, int lc, int ld, const VlxbBatchCall* c, void* stream)", "{",
          "    if (la < 0 || la > 2 || lb < 0 || lb > 2 || lc < 0 || lc > 2 || ld < 0 || ld > 2) return VLXB_EINVAL;",
          "    if (!c || c->n_mol <= 0 || !c->prim_mol[la] || !c->maxD_mol) return VLXB_EINVAL;",
          "    vlxb::ExchangeArgs A{};",
          "    A.mat_K = c->mat; A.pair_i = c->pair_i; A.pair_k = c->pair_k; A.n_ik = c->n_ik;",
          "    for (int l = 0; l < 3; l++) {",
          "        A.info[l] = c->prim_info[l]; A.aoinds[l] = c->prim_aoinds[l]; A.count[l] = c->prim_count[l];",
          "        A.aoinds_col[l] = c->prim_aocols[l];",
          "    }",
          "    A.maxD = 0.0; A.D = c->D; A.naos = c->naos; A.D_stride = c->D_stride; A.key_naos = c->naos;",
          "    A.Q_ab = c->Q_ab; A.Q_cd = c->Q_cd; A.Dinds_ab = c->Dinds_ab; A.Dinds_cd = c->Dinds_cd;",
          "    A.displs_ab = c->displs_ab; A.displs_cd = c->displs_cd; A.counts_ab = c->counts_ab;",
          "    A.counts_cd = c->counts_cd; A.pdata_ab = c->pdata_ab; A.pdata_cd = c->pdata_cd;",
          "    A.omega = c->omega; A.thr = c->thr;",
          "    A.prim_mol_a = c->prim_mol[la]; A.maxD_mol = c->maxD_mol;",
          "    switch (la * 27 + lb * 9 + lc * 3 + ld) {"]
    for cls in k_classes():
        la, lb, lc, ld = (LV[x] for x in cls)
        L.append(f"        case {la * 27 + lb * 9 + lc * 3 + ld}: return vlxb::exchange_{cls}(A, (cudaStream_t)stream);")
    L += ["        default: return VLXB_EINVAL;", "    }", "}", ""]
    L += ["}  // extern \"C\"", ""]
    return "\n".join(L)


def class_tu(cls, kind):
    la, lb, lc, ld = (LV[x] for x in cls)
    L = ["// Generated by gen_abi.py -- do not edit.",
         '#include "../common.cuh"',
         f'#include "q_{cls}.cuh"',
         '#include "hrr_pairs.cuh"',
         '#include "../col_kernels.cuh"',
         f'#include "col_{cls}.cuh"',
         '#include "../classes.cuh"', "",
         "namespace vlxb {"]
    if kind == "j":
        L.append(f"int coulomb_{cls}(const CoulombArgs& a, cudaStream_t s) "
                 f"{{ return run_coulomb<{la}, {lb}, {lc}, {ld}>(a, s); }}")
        L.append(f"int coulomb_grad_{cls}(const CoulombArgs& a, int64_t gs, cudaStream_t s) "
                 f"{{ return run_coulomb_grad<{la}, {lb}, {lc}, {ld}>(a, gs, s); }}")
    else:
        L.append(f"int exchange_{cls}(const ExchangeArgs& a, cudaStream_t s) "
                 f"{{ return run_exchange<{la}, {lb}, {lc}, {ld}>(a, s); }}")
        L.append(f"int exchange_grad_{cls}(const ExchangeArgs& a, int64_t gs, cudaStream_t s) "
                 f"{{ return run_exchange_grad<{la}, {lb}, {lc}, {ld}>(a, gs, s); }}")
    L += ["}  // namespace vlxb", ""]
    return "\n".join(L)


def write_if_changed(path, text):
    if os.path.exists(path):
        with open(path) as fh:
            if fh.read() == text:
                return
    with open(path, "w") as fh:
        fh.write(text)


def main(pkg_root, repo_root):
    gen = os.path.join(pkg_root, "csrc", "generated")
    os.makedirs(gen, exist_ok=True)
    write_if_changed(os.path.join(repo_root, "include", "vlxb.h"), header())
    write_if_changed(os.path.join(gen, "abi.cu"), abi_cu())
    for cls in j_classes():
        write_if_changed(os.path.join(gen, f"cls_{cls}_j.cu"), class_tu(cls, "j"))
    for cls in k_classes():
        write_if_changed(os.path.join(gen, f"cls_{cls}_k.cu"), class_tu(cls, "k"))


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    pkg = os.path.dirname(here)
    main(pkg, os.path.dirname(pkg))
