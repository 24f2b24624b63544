// Host harness around the reference generator's emitted ERI expressions.
//
// TEST / BASELINE INFRASTRUCTURE ONLY (see oracle/__init__.py): used by the
// parity tests and by bench.py's CPU-baseline / reference arm.  make_ref.py
// generates one source per class that includes this header, pastes the
// expression returned by the reference's eriwriter.write_eri_code and
// instantiates the loops below, which restate the emitted kernels:
//   J: gen_coulomb.py:165-297 (per bra prim-cart pair ij: scan the ket list,
//      break on |Q_ij Q_kl D_kl| <= thr, weight 2 or (k != l) + 1)
//   K: gen_exchange.py:161-342 (per (i, k): loop partners j of i and l of k,
//      break on |Q_ij Q_kl max_D| <= thr, gather D_AO[j_cgto, l_cgto])
// One OpenMP thread plays the role of one GPU thread row; rows are
// independent, so the result does not depend on the thread count.
//
// The reference's Boys function is external to it (VeloxChem), so this
// harness carries its own: F_L by a 7-term Taylor expansion around a grid of
// step 0.05 (table built once from the convergent series in long double) and
// downward recursion, asymptotic form with upward recursion for T >= 36.
#pragma once
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace vlxref {

constexpr int NGRID = 721, NCOL = 18, NT = 8;
constexpr double MATH_CONST_INV_PI = 0.318309886183790671537767526745028724;

inline const double* boys_table()
{
    static double tab[NGRID * NCOL];
    static bool done = false;
#pragma omp critical(vlxref_boys)
    {
        if (!done) {
            const int M = NCOL - 1;
            for (int k = 0; k < NGRID; k++) {
                long double T = 0.05L * k, term = 1.0L / (2 * M + 1), sum = term;
                for (int i = 1; i < 4000; i++) {
                    term *= 2.0L * T / (2.0L * M + 2.0L * i + 1.0L);
                    sum += term;
                    if (i > T && term < 1e-25L * sum) break;
                }
                long double ex = expl(-T), F[NCOL];
                F[M] = ex * sum;
                for (int m = M - 1; m >= 0; m--) F[m] = (2.0L * T * F[m + 1] + ex) / (2.0L * m + 1.0L);
                for (int m = 0; m < NCOL; m++) tab[k * NCOL + m] = (double)F[m];
            }
            done = true;
        }
    }
    return tab;
}

inline void boys(double* F, double T, int L, const double* tab)
{
    if (T < 36.0) {
        int k = (int)lrint(T * 20.0);
        double md = 0.05 * k - T;
        const double* row = tab + k * NCOL + L;
        double acc = row[NT - 1];
        for (int j = NT - 1; j >= 1; j--) acc = acc * md / j + row[j - 1];
        F[L] = acc;
        double ex = exp(-T);
        for (int m = L - 1; m >= 0; m--) F[m] = (2.0 * T * F[m + 1] + ex) / (2.0 * m + 1.0);
    } else {
        F[0] = 0.5 * sqrt(M_PI / T);
        double ex = exp(-T);
        for (int m = 0; m < L; m++) F[m + 1] = ((2.0 * m + 1.0) * F[m] - ex) / (2.0 * T);
    }
}

static const uint32_t d_cart_inds[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
static const double delta[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

struct Prim {
    double a, r[3];
};
inline Prim prim(const double* info, uint32_t count, int l, uint32_t i)
{
    uint32_t p = i / (uint32_t)ncart(l);
    Prim x;
    x.a = info[p];
    x.r[0] = info[p + count * 2];
    x.r[1] = info[p + count * 3];
    x.r[2] = info[p + count * 4];
    return x;
}

// Cartesian component index variables of gen_coulomb.py:187-192.
inline void comp_vars(int l, uint32_t i, uint32_t* v)
{
    if (l == 1) v[0] = i % 3;
    if (l == 2) { v[0] = d_cart_inds[i % 6][0]; v[1] = d_cart_inds[i % 6][1]; }
}

}  // namespace vlxref
