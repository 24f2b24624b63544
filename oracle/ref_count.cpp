// Screened-in primitive SHELL quartet counts of one J or K class, from the
// reference-format lists.  TEST / BASELINE INFRASTRUCTURE ONLY: gives the
// reference arm of bench.py the unit of its quartets/s figure.
//
// Definitions (the same predicates the GPU kernels count with):
//   a record is one primitive shell pair together with one distinct Schwarz
//   value q among its components;
//   J: a (bra record, ket shell pair) counts if q * tmax > thr, where
//      tmax = max over the ket pair's components of |Q_kl D_kl|;
//   K: for an output block (i shell, k shell), a (partner record of i,
//      partner record of k) counts if |q1 q2 max_D| > thr.
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <functional>
#include <tuple>
#include <vector>

namespace {

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// number of leading entries of a descending array v with pred(v[n]) true
template <typename F>
inline int64_t prefix(const double* v, int64_t n, F pred)
{
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) / 2;
        if (pred(v[mid])) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// distinct (key, q) pairs -> per key, the list of distinct q
struct KeyQ {
    uint64_t key;
    double q;
};

void unique_sorted(std::vector<KeyQ>& v)
{
    std::sort(v.begin(), v.end(), [](const KeyQ& a, const KeyQ& b) {
        return a.key < b.key || (a.key == b.key && a.q < b.q);
    });
    v.erase(std::unique(v.begin(), v.end(), [](const KeyQ& a, const KeyQ& b) { return a.key == b.key && a.q == b.q; }),
            v.end());
}

}  // namespace

extern "C" uint64_t vlxref_count_j(int la, int lb, int lc, int ld, const double* ab_Q, const uint32_t* ab_first,
                                   const uint32_t* ab_second, uint32_t n_ab, const double* cd_Q, const double* cd_D,
                                   const uint32_t* cd_first, const uint32_t* cd_second, uint32_t n_cd, double thr)
{
    const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
    std::vector<KeyQ> bra(n_ab);
    for (uint32_t e = 0; e < n_ab; e++)
        bra[e] = {((uint64_t)(ab_first[e] / na) << 32) | (ab_second[e] / nb), ab_Q[e]};
    unique_sorted(bra);
    std::vector<std::pair<uint64_t, double>> ket(n_cd);
    for (uint32_t e = 0; e < n_cd; e++)
        ket[e] = {((uint64_t)(cd_first[e] / nc) << 32) | (cd_second[e] / nd), fabs(cd_Q[e] * cd_D[e])};
    std::sort(ket.begin(), ket.end());
    std::vector<double> tmax;
    for (size_t e = 0; e < ket.size();) {
        size_t f = e;
        double t = 0.0;
        while (f < ket.size() && ket[f].first == ket[e].first) t = fmax(t, ket[f++].second);
        tmax.push_back(t);
        e = f;
    }
    std::sort(tmax.begin(), tmax.end(), std::greater<double>());
    uint64_t total = 0;
#pragma omp parallel for reduction(+ : total)
    for (int64_t r = 0; r < (int64_t)bra.size(); r++) {
        const double q = bra[r].q;
        total += (uint64_t)prefix(tmax.data(), (int64_t)tmax.size(), [&](double t) { return q * t > thr; });
    }
    return total;
}

// Records of a CSR partner list grouped by first primitive shell: seg offsets
// into a flat q array, q descending inside each segment.
static void partner_records(int lx, int ly, uint32_t nprim_x, const double* Q, const uint32_t* Dinds,
                            const uint32_t* displs, const uint32_t* counts, std::vector<int64_t>& seg,
                            std::vector<double>& qs)
{
    const int nx = ncart(lx), ny = ncart(ly);
    std::vector<std::tuple<uint32_t, uint32_t, double>> v;
    for (uint32_t i = 0; i < nprim_x * (uint32_t)nx; i++)
        for (uint32_t t = 0; t < counts[i]; t++) {
            const uint32_t e = displs[i] + t;
            v.emplace_back(i / nx, Dinds[e] / ny, Q[e]);
        }
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    seg.assign(nprim_x + 1, 0);
    for (auto& x : v) seg[std::get<0>(x) + 1]++;
    for (uint32_t s = 0; s < nprim_x; s++) seg[s + 1] += seg[s];
    qs.resize(v.size());
    for (size_t k = 0; k < v.size(); k++) qs[k] = std::get<2>(v[k]);
    for (uint32_t s = 0; s < nprim_x; s++)
        std::sort(qs.begin() + seg[s], qs.begin() + seg[s + 1], std::greater<double>());
}

extern "C" uint64_t vlxref_count_k(int la, int lb, int lc, int ld, uint32_t nprim_a, uint32_t nprim_c,
                                   const uint32_t* pair_i, const uint32_t* pair_k, uint32_t n_ik,
                                   const double* Q_ab, const uint32_t* Dinds_ab, const uint32_t* displs_ab,
                                   const uint32_t* counts_ab, const double* Q_cd, const uint32_t* Dinds_cd,
                                   const uint32_t* displs_cd, const uint32_t* counts_cd, double maxD, double thr)
{
    const int na = ncart(la), nc = ncart(lc);
    std::vector<int64_t> sa, sc;
    std::vector<double> qa, qc;
    partner_records(la, lb, nprim_a, Q_ab, Dinds_ab, displs_ab, counts_ab, sa, qa);
    partner_records(lc, ld, nprim_c, Q_cd, Dinds_cd, displs_cd, counts_cd, sc, qc);
    std::vector<uint64_t> blocks(n_ik);
    for (uint32_t e = 0; e < n_ik; e++) blocks[e] = ((uint64_t)(pair_i[e] / na) << 32) | (pair_k[e] / nc);
    std::sort(blocks.begin(), blocks.end());
    blocks.erase(std::unique(blocks.begin(), blocks.end()), blocks.end());
    uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
    for (int64_t b = 0; b < (int64_t)blocks.size(); b++) {
        const uint32_t I = (uint32_t)(blocks[b] >> 32), K = (uint32_t)(blocks[b] & 0xffffffffu);
        const double* q2 = qc.data() + sc[K];
        const int64_t n2 = sc[K + 1] - sc[K];
        for (int64_t r = sa[I]; r < sa[I + 1]; r++) {
            const double q1 = qa[r];
            total += (uint64_t)prefix(q2, n2, [&](double q) { return fabs(q1 * q * maxD) > thr; });
        }
    }
    return total;
}
