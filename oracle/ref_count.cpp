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
#include <map>
#include <utility>
#include <vector>

namespace {

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// number of leading entries of a descending array v with pred(v[n]) true
template <typename F>
inline int64_t prefix(const std::vector<double>& v, F pred)
{
    int64_t lo = 0, hi = (int64_t)v.size();
    while (lo < hi) {
        int64_t mid = (lo + hi) / 2;
        if (pred(v[mid])) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

}  // namespace

extern "C" uint64_t vlxref_count_j(int la, int lb, int lc, int ld, const double* ab_Q, const uint32_t* ab_first,
                                   const uint32_t* ab_second, uint32_t n_ab, const double* cd_Q, const double* cd_D,
                                   const uint32_t* cd_first, const uint32_t* cd_second, uint32_t n_cd, double thr)
{
    const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
    std::map<std::pair<uint32_t, uint32_t>, std::vector<double>> bra;
    for (uint32_t e = 0; e < n_ab; e++) {
        auto& v = bra[{ab_first[e] / na, ab_second[e] / nb}];
        if (std::find(v.begin(), v.end(), ab_Q[e]) == v.end()) v.push_back(ab_Q[e]);
    }
    std::map<std::pair<uint32_t, uint32_t>, double> ket;
    for (uint32_t e = 0; e < n_cd; e++) {
        const double t = fabs(cd_Q[e] * cd_D[e]);
        auto key = std::make_pair(cd_first[e] / nc, cd_second[e] / nd);
        auto it = ket.find(key);
        if (it == ket.end()) ket[key] = t;
        else it->second = fmax(it->second, t);
    }
    std::vector<double> tmax;
    for (auto& kv : ket) tmax.push_back(kv.second);
    std::sort(tmax.begin(), tmax.end(), std::greater<double>());
    uint64_t total = 0;
    for (auto& kv : bra)
        for (double q : kv.second) total += (uint64_t)prefix(tmax, [&](double t) { return q * t > thr; });
    return total;
}

static std::vector<std::vector<double>> partner_records(int lx, int ly, uint32_t nprim_x, const double* Q,
                                                        const uint32_t* Dinds, const uint32_t* displs,
                                                        const uint32_t* counts)
{
    const int nx = ncart(lx), ny = ncart(ly);
    std::vector<std::map<uint32_t, std::vector<double>>> by(nprim_x);
    for (uint32_t i = 0; i < nprim_x * (uint32_t)nx; i++)
        for (uint32_t t = 0; t < counts[i]; t++) {
            const uint32_t e = displs[i] + t;
            auto& v = by[i / nx][Dinds[e] / ny];
            if (std::find(v.begin(), v.end(), Q[e]) == v.end()) v.push_back(Q[e]);
        }
    std::vector<std::vector<double>> out(nprim_x);
    for (uint32_t s = 0; s < nprim_x; s++) {
        for (auto& kv : by[s])
            for (double q : kv.second) out[s].push_back(q);
        std::sort(out[s].begin(), out[s].end(), std::greater<double>());
    }
    return out;
}

extern "C" uint64_t vlxref_count_k(int la, int lb, int lc, int ld, uint32_t nprim_a, uint32_t nprim_c,
                                   const uint32_t* pair_i, const uint32_t* pair_k, uint32_t n_ik,
                                   const double* Q_ab, const uint32_t* Dinds_ab, const uint32_t* displs_ab,
                                   const uint32_t* counts_ab, const double* Q_cd, const uint32_t* Dinds_cd,
                                   const uint32_t* displs_cd, const uint32_t* counts_cd, double maxD, double thr)
{
    const int na = ncart(la), nc = ncart(lc);
    auto rab = partner_records(la, lb, nprim_a, Q_ab, Dinds_ab, displs_ab, counts_ab);
    auto rcd = partner_records(lc, ld, nprim_c, Q_cd, Dinds_cd, displs_cd, counts_cd);
    std::vector<std::pair<uint32_t, uint32_t>> blocks;
    blocks.reserve(n_ik);
    for (uint32_t e = 0; e < n_ik; e++) blocks.push_back({pair_i[e] / na, pair_k[e] / nc});
    std::sort(blocks.begin(), blocks.end());
    blocks.erase(std::unique(blocks.begin(), blocks.end()), blocks.end());
    uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
    for (int64_t b = 0; b < (int64_t)blocks.size(); b++) {
        const auto& q1s = rab[blocks[b].first];
        const auto& q2s = rcd[blocks[b].second];
        for (double q1 : q1s) total += (uint64_t)prefix(q2s, [&](double q2) { return fabs(q1 * q2 * maxD) > thr; });
    }
    return total;
}
