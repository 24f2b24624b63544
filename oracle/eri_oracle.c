/*
 * eri_oracle.c -- CPU restatement of the vlx-twoe-ints J/K path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls
 * this file; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg do, and only as the checker.
 *
 * What it restates (reference paths are relative to the vlx-twoe-ints tree):
 *   - Obara-Saika VRR on c then on a, and HGP HRR on d and b, in the
 *     reference's coefficient and sign conventions: eri.py:177-355
 *     (PQ = Q - P, W - P = S2/S4 PQ, W - Q = -S1/S4 PQ, AB written as PB - PA,
 *     CD written as QD - QC).  The HRR is applied through its binomial closed
 *     form, which is algebraically identical to repeated use of eri.py:177-235.
 *     The known quirk at eri.py:326-329 (delta_{c,c[-1]} inside VRR on a) is
 *     unreachable in the reference and is restated here in its correct
 *     delta_{a,c} form, inside VRR on c.
 *   - The per-component prefactor Lambda * S_ij_00 * S_kl_00 with
 *     Lambda = sqrt(4 S1 S2 / (pi S4)): gen_coulomb.py:244-270.
 *   - Range separation: d2 = w^2/(rho + w^2), Lambda *= sqrt(d2),
 *     T *= d2, F_m *= d2^m: gen_exchange.py:278-298.
 *   - J digestion with the k<->l doubling weights: gen_coulomb.py:205-297.
 *   - Bra-centre derivatives of J and the energy-weighted centre derivatives
 *     of K (nuclear gradient) by the Obara-Saika derivative relation, the
 *     generator's gradient='a' / 'b' / 'c' terms (eri.py:85-152), on the same
 *     integrals, digestion and screening.
 *   - K digestion over partner lists with the max-D screen and the AO-density
 *     gather: gen_exchange.py:139-342.
 * Screening follows the set semantics that the reference's per-thread
 * `break` produces when its lists are sorted by descending bound
 * (gen_coulomb.py:209-212, gen_exchange.py:229-232): a term is kept iff
 * |bound| > threshold.
 *
 * Boys function: long-double Taylor series, F_m(T) = e^{-T} sum_k (2T)^k /
 * prod_{i=0..k}(2m+2i+1), with downward recursion; closed asymptotic form
 * with exact upward recursion for large T.  The reference's Boys function is
 * external to it (VeloxChem's BoysFuncGPU.hpp, not vendored), so this one is
 * pinned against mpmath in the tests instead.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_MAXL 4          /* max angular momentum of one e or f index     */
#define OR_MAXM 16         /* max Boys order                               */

static const long double OR_PI_L = 3.141592653589793238462643383279502884L;

/* ------------------------------------------------------------------ Boys */

void oracle_boys(int M, double T, double* F)
{
    long double t = (long double)T;
    long double Fl[OR_MAXM + 2];
    if (t < 1e-40L) {
        for (int m = 0; m <= M; m++) F[m] = 1.0 / (2.0 * m + 1.0);
        return;
    }
    long double ex = expl(-t);
    if (t > 150.0L) {
        Fl[0] = 0.5L * sqrtl(OR_PI_L / t);
        for (int m = 0; m < M; m++)
            Fl[m + 1] = ((2.0L * m + 1.0L) * Fl[m] - ex) / (2.0L * t);
    } else {
        /* series for F_M */
        long double term = 1.0L / (2.0L * M + 1.0L);
        long double sum = term;
        for (int k = 1; k < 2000; k++) {
            term *= 2.0L * t / (2.0L * M + 2.0L * k + 1.0L);
            sum += term;
            if (k > t && term < 1e-24L * sum) break;
        }
        Fl[M] = ex * sum;
        for (int m = M - 1; m >= 0; m--)
            Fl[m] = (2.0L * t * Fl[m + 1] + ex) / (2.0L * m + 1.0L);
    }
    for (int m = 0; m <= M; m++) F[m] = (double)Fl[m];
}

/* ------------------------------------------------- one primitive quartet */

typedef struct {
    double PA[3], WP[3], QC[3], WQ[3], AB[3], CD[3];
    double inv2z, inv2e, inv2ze, rho_z, rho_e;
    double base[OR_MAXM + 1];
    double* memo;      /* nci * nci * (OR_MAXM+1) values */
    uint32_t* stamp;   /* same shape */
    uint32_t cur;
    int nb, nci;       /* Cartesian triplet slots: components 0..nb-1, nci = nb^3 */
} OrCtx;

static inline int ci(const OrCtx* c, const int v[3]) { return (v[0] * c->nb + v[1]) * c->nb + v[2]; }

static double vrr(OrCtx* c, const int e[3], const int f[3], int m)
{
    if (e[0] < 0 || e[1] < 0 || e[2] < 0 || f[0] < 0 || f[1] < 0 || f[2] < 0)
        return 0.0;
    size_t key = ((size_t)ci(c, e) * c->nci + (size_t)ci(c, f)) * (OR_MAXM + 1) + (size_t)m;
    if (c->stamp[key] == c->cur) return c->memo[key];
    double v;
    if (f[0] + f[1] + f[2] > 0) {
        /* VRR on c (eri.py:237-295):
           [e|f]^m = QC_i [e|f-1i]^m + WQ_i [e|f-1i]^{m+1}
                   + (f_i-1)/(2 eta) ([e|f-2i]^m - rho/eta [e|f-2i]^{m+1})
                   + e_i/(2(zeta+eta)) [e-1i|f-1i]^{m+1}                     */
        int i = (f[0] > 0) ? 0 : ((f[1] > 0) ? 1 : 2);
        int f1[3] = {f[0], f[1], f[2]}; f1[i] -= 1;
        int f2[3] = {f1[0], f1[1], f1[2]}; f2[i] -= 1;
        int e1[3] = {e[0], e[1], e[2]}; e1[i] -= 1;
        v = c->QC[i] * vrr(c, e, f1, m) + c->WQ[i] * vrr(c, e, f1, m + 1);
        if (f1[i] > 0)
            v += f1[i] * c->inv2e * (vrr(c, e, f2, m) - c->rho_e * vrr(c, e, f2, m + 1));
        if (e[i] > 0)
            v += e[i] * c->inv2ze * vrr(c, e1, f1, m + 1);
    } else if (e[0] + e[1] + e[2] > 0) {
        /* VRR on a (eri.py:297-355), c empty:
           [e|0]^m = PA_i [e-1i]^m + WP_i [e-1i]^{m+1}
                   + (e_i-1)/(2 zeta) ([e-2i]^m - rho/zeta [e-2i]^{m+1})      */
        int i = (e[0] > 0) ? 0 : ((e[1] > 0) ? 1 : 2);
        int e1[3] = {e[0], e[1], e[2]}; e1[i] -= 1;
        int e2[3] = {e1[0], e1[1], e1[2]}; e2[i] -= 1;
        v = c->PA[i] * vrr(c, e1, f, m) + c->WP[i] * vrr(c, e1, f, m + 1);
        if (e1[i] > 0)
            v += e1[i] * c->inv2z * (vrr(c, e2, f, m) - c->rho_z * vrr(c, e2, f, m + 1));
    } else {
        v = c->base[m];
    }
    c->stamp[key] = c->cur;
    c->memo[key] = v;
    return v;
}

static const int binom_tab[5][5] = {
    {1, 0, 0, 0, 0}, {1, 1, 0, 0, 0}, {1, 2, 1, 0, 0}, {1, 3, 3, 1, 0}, {1, 4, 6, 4, 1}};

/* (ab|cd) / (S_ab S_cd) for one Cartesian component quartet, via the HRR
   closed form (a b| = sum_t prod_x C(b_x,t_x) AB_x^{b_x-t_x} (a+t 0|.      */
static double quartet_component(OrCtx* c, const int a[3], const int b[3],
                                const int cc[3], const int d[3])
{
    double acc = 0.0;
    for (int tx = 0; tx <= b[0]; tx++)
    for (int ty = 0; ty <= b[1]; ty++)
    for (int tz = 0; tz <= b[2]; tz++) {
        double cb = binom_tab[b[0]][tx] * binom_tab[b[1]][ty] * binom_tab[b[2]][tz]
                  * pow(c->AB[0], b[0] - tx) * pow(c->AB[1], b[1] - ty) * pow(c->AB[2], b[2] - tz);
        int e[3] = {a[0] + tx, a[1] + ty, a[2] + tz};
        for (int ux = 0; ux <= d[0]; ux++)
        for (int uy = 0; uy <= d[1]; uy++)
        for (int uz = 0; uz <= d[2]; uz++) {
            double cd = binom_tab[d[0]][ux] * binom_tab[d[1]][uy] * binom_tab[d[2]][uz]
                      * pow(c->CD[0], d[0] - ux) * pow(c->CD[1], d[1] - uy) * pow(c->CD[2], d[2] - uz);
            int f[3] = {cc[0] + ux, cc[1] + uy, cc[2] + uz};
            acc += cb * cd * vrr(c, e, f, 0);
        }
    }
    return acc;
}

/* Set up the quartet scalars of eri.py / gen_coulomb.py:244-268. */
static void setup_quartet(OrCtx* c, int L, double ai, const double* Ai, double aj, const double* Bj,
                          double ak, const double* Ck, double al, const double* Dl, double omega)
{
    double S1 = ai + aj, S2 = ak + al, S4 = S1 + S2;
    double P[3], Q[3], PQ[3];
    for (int x = 0; x < 3; x++) {
        P[x] = (ai * Ai[x] + aj * Bj[x]) / S1;
        Q[x] = (ak * Ck[x] + al * Dl[x]) / S2;
        PQ[x] = Q[x] - P[x];
        c->PA[x] = P[x] - Ai[x];
        c->QC[x] = Q[x] - Ck[x];
        c->WP[x] = S2 / S4 * PQ[x];
        c->WQ[x] = -S1 / S4 * PQ[x];
        c->AB[x] = Ai[x] - Bj[x];
        c->CD[x] = Ck[x] - Dl[x];
    }
    c->inv2z = 0.5 / S1;
    c->inv2e = 0.5 / S2;
    c->inv2ze = 0.5 / S4;
    c->rho_z = S2 / S4;
    c->rho_e = S1 / S4;
    double rho = S1 * S2 / S4;
    double r2 = PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2];
    double d2 = 1.0;
    if (omega != 0.0) d2 = omega * omega / (rho + omega * omega);
    double F[OR_MAXM + 1];
    oracle_boys(L, rho * d2 * r2, F);
    double lam = sqrt(4.0 * rho * d2 / (double)OR_PI_L);
    double dm = 1.0;
    for (int m = 0; m <= L; m++) { c->base[m] = lam * F[m] * dm; dm *= d2; }
    c->cur++;
    if (c->cur == 0) { memset(c->stamp, 0, sizeof(uint32_t) * (size_t)c->nci * c->nci * (OR_MAXM + 1)); c->cur = 1; }
}

/* nb = 1 + the largest Cartesian exponent an e or f index reaches: OR_MAXL + 1
   for (ab|cd) over s, p, d; one more for the derivative integrals. */
static OrCtx* ctx_new_nb(int nb)
{
    OrCtx* c = (OrCtx*)calloc(1, sizeof(OrCtx));
    c->nb = nb;
    c->nci = nb * nb * nb;
    size_t n = (size_t)c->nci * c->nci * (OR_MAXM + 1);
    c->memo = (double*)malloc(sizeof(double) * n);
    c->stamp = (uint32_t*)calloc(n, sizeof(uint32_t));
    c->cur = 0;
    return c;
}

static OrCtx* ctx_new(void) { return ctx_new_nb(OR_MAXL + 1); }

/* Context large enough for a class: Cartesian exponents of e = a + b and
   f = c + d reach la + lb and lc + ld (up to 6 with f shells). */
static OrCtx* ctx_for(int la, int lb, int lc, int ld)
{
    int emax = (la + lb > lc + ld) ? la + lb : lc + ld;
    return ctx_new_nb(emax + 1 > OR_MAXL + 1 ? emax + 1 : OR_MAXL + 1);
}

static void ctx_free(OrCtx* c) { free(c->memo); free(c->stamp); free(c); }

/* Cartesian component tables, in the reference's order (gen_coulomb.py:143-148):
   p: x, y, z; d: xx, xy, xz, yy, yz, zz. */
static const int cart_s[1][3] = {{0, 0, 0}};
static const int cart_p[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
static const int cart_d[6][3] = {{2, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 2, 0}, {0, 1, 1}, {0, 0, 2}};
/* f in the same convention (x^3 first, then by decreasing y power): the
   component tables the reference's emitted kernels would use for a third
   index (sorted index triples xxx, xxy, ..., zzz). */
static const int cart_f[10][3] = {{3, 0, 0}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0}, {1, 1, 1},
                                  {1, 0, 2}, {0, 3, 0}, {0, 2, 1}, {0, 1, 2}, {0, 0, 3}};
static const int ncart_of[4] = {1, 3, 6, 10};

static const int* cart_comp(int l, int k)
{
    if (l == 0) return cart_s[0];
    if (l == 1) return cart_p[k];
    if (l == 2) return cart_d[k];
    return cart_f[k];
}

/* ------------------------------------------------------- public helpers */

/* Bare integrals (ab|cd)/(S_ab S_cd) for every Cartesian component quartet of
   one primitive shell quartet; out[((ca*nb+cb)*nc+cc)*nd+cd].  Shells up to
   f (l <= 3). */
void oracle_eri_shell_quartet(int la, int lb, int lc, int ld,
                              double ai, const double* A, double aj, const double* B,
                              double ak, const double* C, double al, const double* D,
                              double omega, double* out)
{
    int emax = (la + lb > lc + ld) ? la + lb : lc + ld;
    OrCtx* c = ctx_new_nb(emax + 1 > OR_MAXL + 1 ? emax + 1 : OR_MAXL + 1);
    int L = la + lb + lc + ld;
    setup_quartet(c, L, ai, A, aj, B, ak, C, al, D, omega);
    int na = ncart_of[la], nb = ncart_of[lb], nc = ncart_of[lc], nd = ncart_of[ld];
    for (int ia = 0; ia < na; ia++)
    for (int ib = 0; ib < nb; ib++)
    for (int ic = 0; ic < nc; ic++)
    for (int id = 0; id < nd; id++)
        out[((ia * nb + ib) * nc + ic) * nd + id] =
            quartet_component(c, cart_comp(la, ia), cart_comp(lb, ib), cart_comp(lc, ic), cart_comp(ld, id));
    ctx_free(c);
}

/* Derivatives of the bare integrals of one primitive shell quartet with
   respect to one centre (center 0..3 = A, B, C, D), by the Obara-Saika
   derivative relation (eri.py:85-175, the generator's gradient='a'..'d'):
   d/dX_g (.. x ..) = 2 zeta_x (.. x+1_g ..) - x_g (.. x-1_g ..).
   out[(g * na * nb + ...)] = out[g][ca][cb][cc][cd], g = 0..2. */
void oracle_eri_shell_quartet_grad(int la, int lb, int lc, int ld, int center,
                                   double ai, const double* A, double aj, const double* B,
                                   double ak, const double* C, double al, const double* D,
                                   double omega, double* out)
{
    OrCtx* c = ctx_new_nb(OR_MAXL + 2);
    int L = la + lb + lc + ld + 1;
    setup_quartet(c, L, ai, A, aj, B, ak, C, al, D, omega);
    int na = ncart_of[la], nb = ncart_of[lb], nc = ncart_of[lc], nd = ncart_of[ld];
    const double zeta[4] = {ai, aj, ak, al};
    size_t ncomp = (size_t)na * nb * nc * nd;
    for (int g = 0; g < 3; g++)
    for (int ia = 0; ia < na; ia++)
    for (int ib = 0; ib < nb; ib++)
    for (int ic = 0; ic < nc; ic++)
    for (int id = 0; id < nd; id++) {
        int v[4][3];
        const int* src[4] = {cart_comp(la, ia), cart_comp(lb, ib), cart_comp(lc, ic), cart_comp(ld, id)};
        for (int t = 0; t < 4; t++)
            for (int x = 0; x < 3; x++) v[t][x] = src[t][x];
        int n = v[center][g];
        v[center][g] += 1;
        double val = 2.0 * zeta[center] * quartet_component(c, v[0], v[1], v[2], v[3]);
        if (n > 0) {
            v[center][g] -= 2;
            val -= n * quartet_component(c, v[0], v[1], v[2], v[3]);
        }
        out[(size_t)g * ncomp + ((ia * nb + ib) * nc + ic) * nd + id] = val;
    }
    ctx_free(c);
}

/* prim_info layout of gen_coulomb.py:170-180: row 0 exponent, rows 2..4 xyz,
   row stride = prim_count; prim-cart index i -> primitive i / ncart,
   component i % ncart. */
static inline void prim_of(const double* info, uint32_t count, int l, uint32_t i,
                           double* alpha, double r[3], int* comp)
{
    int nc = ncart_of[l];
    uint32_t p = i / (uint32_t)nc;
    *comp = (int)(i % (uint32_t)nc);
    *alpha = info[p];
    r[0] = info[p + count * 2];
    r[1] = info[p + count * 3];
    r[2] = info[p + count * 4];
}

/* J of one (ab|cd) class in prim-cart pair space (gen_coulomb.py:74-297).
   prim_info[l] / prim_count[l] for l = 0..3 (s, p, d, f; entries for unused
   l ignored).
   rows: optional subset of bra indices (NULL = all); results go to mat_J[ij]
   with +=, as the emitted kernel does. */
void oracle_coulomb_fock(int la, int lb, int lc, int ld, double* mat_J,
                         const double* const* prim_info, const uint32_t* prim_count,
                         const double* cd_mat_D, const double* ab_mat_Q, const double* cd_mat_Q,
                         const uint32_t* ab_first, const uint32_t* ab_second,
                         const double* ab_pair_data, uint32_t n_ab,
                         const uint32_t* cd_first, const uint32_t* cd_second,
                         const double* cd_pair_data, uint32_t n_cd,
                         double thr, const uint32_t* rows, uint32_t nrows)
{
    uint32_t nwork = rows ? nrows : n_ab;
    int L = la + lb + lc + ld;
    #pragma omp parallel
    {
        OrCtx* c = ctx_for(la, lb, lc, ld);
        #pragma omp for schedule(dynamic, 4)
        for (int64_t w = 0; w < (int64_t)nwork; w++) {
            uint32_t ij = rows ? rows[w] : (uint32_t)w;
            double ai, aj, ri[3], rj[3];
            int ca, cb;
            prim_of(prim_info[la], prim_count[la], la, ab_first[ij], &ai, ri, &ca);
            prim_of(prim_info[lb], prim_count[lb], lb, ab_second[ij], &aj, rj, &cb);
            double J = 0.0;
            for (uint32_t kl = 0; kl < n_cd; kl++) {
                if (fabs(ab_mat_Q[ij] * cd_mat_Q[kl] * cd_mat_D[kl]) <= thr) continue;
                double ak, al, rk[3], rl[3];
                int cc, cd;
                uint32_t k = cd_first[kl], l = cd_second[kl];
                prim_of(prim_info[lc], prim_count[lc], lc, k, &ak, rk, &cc);
                prim_of(prim_info[ld], prim_count[ld], ld, l, &al, rl, &cd);
                setup_quartet(c, L, ai, ri, aj, rj, ak, rk, al, rl, 0.0);
                double eri = ab_pair_data[ij] * cd_pair_data[kl] *
                    quartet_component(c, cart_comp(la, ca), cart_comp(lb, cb),
                                      cart_comp(lc, cc), cart_comp(ld, cd));
                double w8 = (lc != ld) ? 2.0 : ((k != l) ? 2.0 : 1.0);
                J += eri * cd_mat_D[kl] * w8;
            }
            mat_J[ij] += J;
        }
        ctx_free(c);
    }
}

/* Bra-centre derivatives of J for one (ab|cd) class: the derivative of
   oracle_coulomb_fock's mat_J[ij] with respect to the centres A (first) and
   B (second) of bra entry ij, kets and cd_mat_D fixed, by the Obara-Saika
   derivative relation of a Cartesian Gaussian (Obara & Saika 1986, Eq. 5; the
   generator's gradient='a' / 'b' terms, eri.py:85-129):
     d/dA_x (a b|c d) = 2 alpha (a+1x b|c d) - a_x (a-1x b|c d),
     d/dB_x (a b|c d) = 2 beta  (a b+1x|c d) - b_x (a b-1x|c d).
   grad_J[k * gstride + ij] +=, k = 0..2 for A_x..A_z, 3..5 for B_x..B_z.
   Same screening and ket weights as oracle_coulomb_fock. */
void oracle_coulomb_grad(int la, int lb, int lc, int ld, double* grad_J, uint64_t gstride,
                         const double* const* prim_info, const uint32_t* prim_count,
                         const double* cd_mat_D, const double* ab_mat_Q, const double* cd_mat_Q,
                         const uint32_t* ab_first, const uint32_t* ab_second,
                         const double* ab_pair_data, uint32_t n_ab,
                         const uint32_t* cd_first, const uint32_t* cd_second,
                         const double* cd_pair_data, uint32_t n_cd,
                         double thr, const uint32_t* rows, uint32_t nrows)
{
    uint32_t nwork = rows ? nrows : n_ab;
    int L = la + lb + lc + ld + 1;
    #pragma omp parallel
    {
        OrCtx* c = ctx_new_nb(OR_MAXL + 2);
        #pragma omp for schedule(dynamic, 4)
        for (int64_t w = 0; w < (int64_t)nwork; w++) {
            uint32_t ij = rows ? rows[w] : (uint32_t)w;
            double ai, aj, ri[3], rj[3];
            int ca, cb;
            prim_of(prim_info[la], prim_count[la], la, ab_first[ij], &ai, ri, &ca);
            prim_of(prim_info[lb], prim_count[lb], lb, ab_second[ij], &aj, rj, &cb);
            const int* a = cart_comp(la, ca);
            const int* b = cart_comp(lb, cb);
            double g[6] = {0, 0, 0, 0, 0, 0};
            for (uint32_t kl = 0; kl < n_cd; kl++) {
                if (fabs(ab_mat_Q[ij] * cd_mat_Q[kl] * cd_mat_D[kl]) <= thr) continue;
                double ak, al, rk[3], rl[3];
                int cc, cd;
                uint32_t k = cd_first[kl], l = cd_second[kl];
                prim_of(prim_info[lc], prim_count[lc], lc, k, &ak, rk, &cc);
                prim_of(prim_info[ld], prim_count[ld], ld, l, &al, rl, &cd);
                setup_quartet(c, L, ai, ri, aj, rj, ak, rk, al, rl, 0.0);
                const int* kc = cart_comp(lc, cc);
                const int* kd = cart_comp(ld, cd);
                double w8 = (lc != ld) ? 2.0 : ((k != l) ? 2.0 : 1.0);
                double f = ab_pair_data[ij] * cd_pair_data[kl] * cd_mat_D[kl] * w8;
                for (int x = 0; x < 3; x++) {
                    int ap[3] = {a[0], a[1], a[2]}, am[3] = {a[0], a[1], a[2]};
                    int bp[3] = {b[0], b[1], b[2]}, bm[3] = {b[0], b[1], b[2]};
                    ap[x] += 1; am[x] -= 1; bp[x] += 1; bm[x] -= 1;
                    double dA = 2.0 * ai * quartet_component(c, ap, b, kc, kd);
                    if (a[x] > 0) dA -= a[x] * quartet_component(c, am, b, kc, kd);
                    double dB = 2.0 * aj * quartet_component(c, a, bp, kc, kd);
                    if (b[x] > 0) dB -= b[x] * quartet_component(c, a, bm, kc, kd);
                    g[x] += f * dA;
                    g[3 + x] += f * dB;
                }
            }
            for (int t = 0; t < 6; t++) grad_J[(uint64_t)t * gstride + ij] += g[t];
        }
        ctx_free(c);
    }
}

/* K of one (ab|cd) class in prim-cart pair space (gen_exchange.py:75-342).
   ab_* / cd_* are the partner lists of i (type a -> partners of type b) and of
   k (type c -> partners of type d); pass the ab arrays twice when cd == ab.
   rows: optional subset of ik indices. */
void oracle_exchange_fock(int la, int lb, int lc, int ld, double* mat_K,
                          const uint32_t* pair_i, const uint32_t* pair_k, uint32_t n_ik,
                          const double* const* prim_info, const uint32_t* const* prim_aoinds,
                          const uint32_t* prim_count,
                          double bd_max_D, const double* D_AO, uint32_t naos,
                          const double* Q_ab, const double* Q_cd,
                          const uint32_t* Dinds_ab, const uint32_t* Dinds_cd,
                          const uint32_t* displs_ab, const uint32_t* displs_cd,
                          const uint32_t* counts_ab, const uint32_t* counts_cd,
                          const double* pdata_ab, const double* pdata_cd,
                          double omega, double thr, const uint32_t* rows, uint32_t nrows)
{
    uint32_t nwork = rows ? nrows : n_ik;
    int L = la + lb + lc + ld;
    int ncb = ncart_of[lb], ncd = ncart_of[ld];
    #pragma omp parallel
    {
        OrCtx* c = ctx_for(la, lb, lc, ld);
        #pragma omp for schedule(dynamic, 1)
        for (int64_t w = 0; w < (int64_t)nwork; w++) {
            uint32_t ik = rows ? rows[w] : (uint32_t)w;
            uint32_t i = pair_i[ik], k = pair_k[ik];
            double ai, ak, ri[3], rk[3];
            int ca, cc;
            prim_of(prim_info[la], prim_count[la], la, i, &ai, ri, &ca);
            prim_of(prim_info[lc], prim_count[lc], lc, k, &ak, rk, &cc);
            double K = 0.0;
            for (uint32_t j = 0; j < counts_ab[i]; j++) {
                uint32_t pj = displs_ab[i] + j;
                double Qij = Q_ab[pj];
                uint32_t jp = Dinds_ab[pj];
                double aj, rj[3];
                int cb;
                prim_of(prim_info[lb], prim_count[lb], lb, jp, &aj, rj, &cb);
                uint32_t jao = prim_aoinds[lb][jp / (uint32_t)ncb + prim_count[lb] * (jp % (uint32_t)ncb)];
                for (uint32_t l = 0; l < counts_cd[k]; l++) {
                    uint32_t pl = displs_cd[k] + l;
                    if (fabs(Qij * Q_cd[pl] * bd_max_D) <= thr) continue;
                    uint32_t lp = Dinds_cd[pl];
                    double al, rl[3];
                    int cd;
                    prim_of(prim_info[ld], prim_count[ld], ld, lp, &al, rl, &cd);
                    uint32_t lao = prim_aoinds[ld][lp / (uint32_t)ncd + prim_count[ld] * (lp % (uint32_t)ncd)];
                    setup_quartet(c, L, ai, ri, aj, rj, ak, rk, al, rl, omega);
                    double eri = pdata_ab[pj] * pdata_cd[pl] *
                        quartet_component(c, cart_comp(la, ca), cart_comp(lb, cb),
                                          cart_comp(lc, cc), cart_comp(ld, cd));
                    K += eri * D_AO[(size_t)jao * naos + lao];
                }
            }
            mat_K[ik] += K;
        }
        ctx_free(c);
    }
}

/* Energy-weighted centre derivatives of K for one (ab|cd) class, per (i, k)
   list entry (the exchange gradient):
     grad[x * gstride + ik]     += w_ik D_ik sum_jl D_jl d(ij|kl)/dA_x,
     grad[(3+x) * gstride + ik] += w_ik D_ik sum_jl D_jl d(ij|kl)/dC_x,
   A, C the centres of i and k, w_ik = 1 for i == k of a same-type list, else
   2, D_ik and D_jl read from the AO density as in oracle_exchange_fock, by the
   Obara-Saika derivative relation (eri.py:85-152, the generator's gradient='a'
   / 'c' terms).  Same partner loops and screening as oracle_exchange_fock. */
void oracle_exchange_grad(int la, int lb, int lc, int ld, double* grad, uint64_t gstride,
                          const uint32_t* pair_i, const uint32_t* pair_k, uint32_t n_ik,
                          const double* const* prim_info, const uint32_t* const* prim_aoinds,
                          const uint32_t* prim_count,
                          double bd_max_D, const double* D_AO, uint32_t naos,
                          const double* Q_ab, const double* Q_cd,
                          const uint32_t* Dinds_ab, const uint32_t* Dinds_cd,
                          const uint32_t* displs_ab, const uint32_t* displs_cd,
                          const uint32_t* counts_ab, const uint32_t* counts_cd,
                          const double* pdata_ab, const double* pdata_cd,
                          double omega, double thr, const uint32_t* rows, uint32_t nrows)
{
    uint32_t nwork = rows ? nrows : n_ik;
    int L = la + lb + lc + ld + 1;
    int nca = ncart_of[la], ncb = ncart_of[lb], ncc = ncart_of[lc], ncd = ncart_of[ld];
    #pragma omp parallel
    {
        OrCtx* c = ctx_new_nb(OR_MAXL + 2);
        #pragma omp for schedule(dynamic, 1)
        for (int64_t w = 0; w < (int64_t)nwork; w++) {
            uint32_t ik = rows ? rows[w] : (uint32_t)w;
            uint32_t i = pair_i[ik], k = pair_k[ik];
            double ai, ak, ri[3], rk[3];
            int ca, cc;
            prim_of(prim_info[la], prim_count[la], la, i, &ai, ri, &ca);
            prim_of(prim_info[lc], prim_count[lc], lc, k, &ak, rk, &cc);
            uint32_t iao = prim_aoinds[la][i / (uint32_t)nca + prim_count[la] * (i % (uint32_t)nca)];
            uint32_t kao = prim_aoinds[lc][k / (uint32_t)ncc + prim_count[lc] * (k % (uint32_t)ncc)];
            double wik = ((la == lc) && (i == k) ? 1.0 : 2.0) * D_AO[(size_t)iao * naos + kao];
            const int* a = cart_comp(la, ca);
            const int* kc = cart_comp(lc, cc);
            double g[6] = {0, 0, 0, 0, 0, 0};
            for (uint32_t j = 0; j < counts_ab[i]; j++) {
                uint32_t pj = displs_ab[i] + j;
                double Qij = Q_ab[pj];
                uint32_t jp = Dinds_ab[pj];
                double aj, rj[3];
                int cb;
                prim_of(prim_info[lb], prim_count[lb], lb, jp, &aj, rj, &cb);
                uint32_t jao = prim_aoinds[lb][jp / (uint32_t)ncb + prim_count[lb] * (jp % (uint32_t)ncb)];
                const int* b = cart_comp(lb, cb);
                for (uint32_t l = 0; l < counts_cd[k]; l++) {
                    uint32_t pl = displs_cd[k] + l;
                    if (fabs(Qij * Q_cd[pl] * bd_max_D) <= thr) continue;
                    uint32_t lp = Dinds_cd[pl];
                    double al, rl[3];
                    int cd;
                    prim_of(prim_info[ld], prim_count[ld], ld, lp, &al, rl, &cd);
                    uint32_t lao = prim_aoinds[ld][lp / (uint32_t)ncd + prim_count[ld] * (lp % (uint32_t)ncd)];
                    const int* d = cart_comp(ld, cd);
                    setup_quartet(c, L, ai, ri, aj, rj, ak, rk, al, rl, omega);
                    double f = pdata_ab[pj] * pdata_cd[pl] * D_AO[(size_t)jao * naos + lao];
                    for (int x = 0; x < 3; x++) {
                        int ap[3] = {a[0], a[1], a[2]}, am[3] = {a[0], a[1], a[2]};
                        int cp[3] = {kc[0], kc[1], kc[2]}, cm[3] = {kc[0], kc[1], kc[2]};
                        ap[x] += 1; am[x] -= 1; cp[x] += 1; cm[x] -= 1;
                        double dA = 2.0 * ai * quartet_component(c, ap, b, kc, d);
                        if (a[x] > 0) dA -= a[x] * quartet_component(c, am, b, kc, d);
                        double dC = 2.0 * ak * quartet_component(c, a, b, cp, d);
                        if (kc[x] > 0) dC -= kc[x] * quartet_component(c, a, b, cm, d);
                        g[x] += f * dA;
                        g[3 + x] += f * dC;
                    }
                }
            }
            for (int t = 0; t < 6; t++) grad[(uint64_t)t * gstride + ik] += wik * g[t];
        }
        ctx_free(c);
    }
}

int oracle_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
