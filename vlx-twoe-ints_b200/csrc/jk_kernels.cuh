// J and K integral kernels over primitive-shell-pair records (sm_100a).
//
// Work unit: one primitive SHELL quartet, all Cartesian components at once
// (the reference's unit is one Cartesian COMPONENT quartet per thread,
// gen_coulomb.py:115,205-207 and gen_exchange.py:139,189-226).
//
// Coulomb (gen_coulomb.py:205-297): one CTA per bra record; its threads
// stride over the screened prefix of the ket list (sorted by descending
// max |Q_kl D_kl|), each accumulating X_e = sum_f (e0|f0) D''_f in registers,
// where D'' is the ket density carried through the transposed ket HRR.  The
// CTA then reduces X in a fixed order (warp butterfly, then warps in index
// order), applies the bra HRR and writes mat_J[ij] += S_ij J_ij for the
// components it owns.  No atomics: results are bit-reproducible.
//
// Exchange (gen_exchange.py:139-342): one CTA per (i_shell, k_shell) output
// block; its threads stride over the flattened list of (j, l) partner pairs
// that pass |Q_ij Q_kl max_D| > thr, each accumulating K_ac partials, then
// reduce in a fixed order and write mat_K[ik] += K_ik.
//
// Mixed precision (fp32_cut > 0): quartets whose screening bound
// (|Q_ij| max|Q_kl D_kl| for J, |Q_ij Q_kl max_D| for K) is below fp32_cut run
// the same generated code in FP32 (Boys argument formed in FP64); each
// quartet's result is added to FP64 accumulators.  The sorted lists make the
// FP64 quartets a prefix and the FP32 ones the segment after it.
#pragma once
#include <type_traits>

#include "common.cuh"

namespace vlxb {

constexpr int J_THREADS = 128;
constexpr int K_THREADS = 128;
constexpr int K_JCHUNK = 256;
// Screening slack: tests on per-shell max/min bounds are widened by this
// relative margin; quartets inside the margin take the exact per-component
// test, so the screened set equals the reference's exactly.
constexpr double SCREEN_SLACK = 1e-12;

struct JBraRecs {
    const int32_t* rec_sp;     // [n_rec] shell pair of the record
    const double* rec_q;       // [n_rec] Schwarz value shared by the record's components
    const uint64_t* rec_mask;  // [n_rec] components owned by the record
    const int* n_rec;          // device-side record count
    const double* geo;         // [GEO_N][sp_stride] shell-pair geometry
    const int32_t* entry;      // [NAB][sp_stride] bra list position or -1
    int64_t sp_stride;
    const double* pdata;       // caller's ab_pair_data (S_ij_00 per bra list position)
    const int32_t* mol;        // [n_rec] molecule of the record (batched calls), or null
};

struct JKetPairs {
    const double* geo;   // [GEO_N][stride], sorted by descending tmax
    const double* tmax;  // [stride] max over components of |Q_kl D_kl|
    const double* tmin;  // [stride] min over present components
    const double* Dpp;   // [NF][stride]  transposed-HRR ket density (all components)
    const double* Dm;    // [NCD][stride] w_kl * D_kl * S_kl (0 if absent)
    const double* Qc;    // [NCD][stride] Q_kl per component (0 if absent)
    const double* Dc;    // [NCD][stride] D_kl per component
    int64_t stride;
    const int* n;
    const int* seg;      // [molecules + 1] ket range of each molecule (batched calls), or null
    const double* Dh;    // [stride][nherm(LC+LD)] Hermite ket density (McMurchie-Davidson kernel), or null
    const double* tpre;  // [stride] inclusive prefix sum of tmax * HRR growth (FP32 error budget), or null
};

struct BoysTabs {
    const double* f64;
    const float* f32;
};

// Ket density of one quartet as T: the stored D'' when every component passes
// the screen, else the exact per-component screen (same product order as the
// reference: fabs(Q_ij * Q_kl * D_kl) <= thr -> skip) through the transposed
// ket HRR.
template <int LC, int LD, typename T>
__device__ __forceinline__ void ket_density(const JKetPairs& ket, int kt, double qb, double thr, const PairGeo& k,
                                            T* Dpp)
{
    constexpr int NCD = ncart(LC) * ncart(LD), NF = nrange(LC, LD);
    if (qb * __ldg(ket.tmin + kt) > thr * (1.0 + SCREEN_SLACK)) {
#pragma unroll
        for (int f = 0; f < NF; f++) Dpp[f] = (T)__ldg(ket.Dpp + f * ket.stride + kt);
    } else {
        T Dm[NCD];
#pragma unroll
        for (int c = 0; c < NCD; c++) {
            const double qk = __ldg(ket.Qc + c * ket.stride + kt);
            const double dk = __ldg(ket.Dc + c * ket.stride + kt);
            Dm[c] = (fabs(qb * qk * dk) > thr) ? (T)__ldg(ket.Dm + c * ket.stride + kt) : (T)0;
        }
        hrr_ket_adjoint<LC, LD, T>((T)k.Rx, (T)k.Ry, (T)k.Rz, Dm, Dpp);
    }
}

template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void j_quartet(const PairGeo& b, double qb, const JKetPairs& ket, int kt, double thr,
                                          const BoysTabs& tabs, double* X)
{
    constexpr int L = LA + LB + LC + LD;
    constexpr int NE = nrange(LA, LB), NF = nrange(LC, LD);
    const PairGeo k = load_geo(ket.geo, ket.stride, kt);
    QVT<T> q;
    T F[L + 1];
    make_quartet_t<L>(b, k, 0.0, tabs.f64, tabs.f32, q, F);
    T Dpp[NF];
    ket_density<LC, LD, T>(ket, kt, qb, thr, k, Dpp);
    if constexpr (std::is_same<T, double>::value) {
        j_contract<LA, LB, LC, LD, double>(q, F, Dpp, X);
    } else {
        T Xq[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) Xq[e] = (T)0;
        j_contract<LA, LB, LC, LD, T>(q, F, Dpp, Xq);
#pragma unroll
        for (int e = 0; e < NE; e++) X[e] += (double)Xq[e];
    }
}

// HRR growth factor of a pair (the factor hrr_amp of the list preparation,
// from the pair's geometry record): (1 + sqrt(2 zeta) |R|)^lh.
__device__ __forceinline__ double pair_amp(const PairGeo& g, int lh)
{
    if (lh == 0) return 1.0;
    const double f = 1.0 + sqrt(2.0 * g.z * (g.Rx * g.Rx + g.Ry * g.Ry + g.Rz * g.Rz));
    double a = f;
    for (int k = 1; k < lh; k++) a *= f;
    return a;
}

// Prefix lengths of the descending ket bound list for one bra: ncut (slack
// included: candidates), nexact (screened-in quartets, for the counters),
// n64 (evaluated in FP64; all of ncut when fp32_cut <= 0).
// Kets k0 <= t < k1 (one molecule's, sorted by descending bound): ncut / nexact
// / n64 = end (absolute index) of the kets inside the screening slack band /
// passing the exact screen / in FP64.  A ket runs in FP32 when its bound is
// below fp32_cut and, with a budget > 0, when it lies in the tail [n64, ncut)
// whose summed error proxy qa * sum(tmax * HRR growth) stays <= budget
// (qa = the bra's Q times its own HRR growth).
__device__ __forceinline__ void ket_prefixes(const JKetPairs& ket, int k0, int k1, double qb, double thr,
                                             double fp32_cut, double qa, double budget, int& ncut, int& nexact,
                                             int& n64)
{
    int lo = k0, hi = k1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (qb * __ldg(ket.tmax + mid) * (1.0 + SCREEN_SLACK) > thr) lo = mid + 1;
        else hi = mid;
    }
    ncut = lo;
    int lo2 = k0, hi2 = lo;
    while (lo2 < hi2) {
        const int mid = (lo2 + hi2) >> 1;
        if (qb * __ldg(ket.tmax + mid) > thr) lo2 = mid + 1;
        else hi2 = mid;
    }
    nexact = lo2;
    if (fp32_cut <= 0.0) {
        n64 = ncut;
    } else {
        int lo3 = k0, hi3 = ncut;
        while (lo3 < hi3) {
            const int mid = (lo3 + hi3) >> 1;
            if (qb * __ldg(ket.tmax + mid) >= fp32_cut) lo3 = mid + 1;
            else hi3 = mid;
        }
        n64 = lo3;
        if (budget > 0.0 && ket.tpre && n64 < ncut) {
            const double pend = __ldg(ket.tpre + ncut - 1);
            int lo4 = n64, hi4 = ncut;
            while (lo4 < hi4) {
                const int mid = (lo4 + hi4) >> 1;
                const double tail = pend - (mid > 0 ? __ldg(ket.tpre + mid - 1) : 0.0);
                if (qa * tail <= budget) hi4 = mid;
                else lo4 = mid + 1;
            }
            n64 = lo4;
        }
    }
}

// PM (precision pass): 0 = the FP64 quartets (every quartet when fp32_cut is
// 0), 1 = the FP32 quartets.  The two passes are separate launches so that
// the FP32 kernel gets its own, smaller register allocation and higher
// occupancy; both add into mat_J, quartets are counted in pass 0.
template <int LA, int LB, int LC, int LD, int PM>
__global__ void __launch_bounds__(J_THREADS)
coulomb_kernel(JBraRecs bra, JKetPairs ket, double* __restrict__ mat_J, double thr, BoysTabs tabs,
               unsigned long long* __restrict__ qcount, double fp32_cut, double fp32_budget)
{
    constexpr int NE = nrange(LA, LB);
    constexpr int NAB = ncart(LA) * ncart(LB);
    constexpr int NW = J_THREADS / 32;
    __shared__ double red[NW][NE];
    __shared__ int s_ncut, s_n64;
    const int nbra = *bra.n_rec;
    const int nket = *ket.n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    for (int r = blockIdx.x; r < nbra; r += gridDim.x) {
        const int sp = __ldg(bra.rec_sp + r);
        const PairGeo b = load_geo(bra.geo, bra.sp_stride, sp);
        const double qb = __ldg(bra.rec_q + r);
        int k0 = 0, k1 = nket;
        if (bra.mol) {
            const int m = __ldg(bra.mol + r);
            k0 = __ldg(ket.seg + m);
            k1 = __ldg(ket.seg + m + 1);
        }
        if (threadIdx.x == 0) {
            int ncut, nexact, n64;
            ket_prefixes(ket, k0, k1, qb, thr, fp32_cut, fabs(qb) * pair_amp(b, LB), fp32_budget, ncut, nexact, n64);
            s_ncut = ncut;
            s_n64 = n64;
            if (qcount && PM == 0) atomicAdd(qcount, (unsigned long long)(nexact - k0));
        }
        __syncthreads();
        const int ncut = s_ncut, n64 = s_n64;
        if (PM == 1 && n64 >= ncut) {
            __syncthreads();
            continue;  // no FP32 quartets for this bra
        }

        double X[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) X[e] = 0.0;
        if (PM == 0) {
            for (int kt = k0 + threadIdx.x; kt < n64; kt += J_THREADS)
                j_quartet<LA, LB, LC, LD, double>(b, qb, ket, kt, thr, tabs, X);
        } else {
            for (int kt = n64 + threadIdx.x; kt < ncut; kt += J_THREADS)
                j_quartet<LA, LB, LC, LD, float>(b, qb, ket, kt, thr, tabs, X);
        }

#pragma unroll
        for (int e = 0; e < NE; e++) {
            const double v = warp_sum(X[e]);
            if (lane == 0) red[warp][e] = v;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double Xs[NE];
#pragma unroll
            for (int e = 0; e < NE; e++) {
                double s = red[0][e];
#pragma unroll
                for (int w = 1; w < NW; w++) s += red[w][e];
                Xs[e] = s;
            }
            double J[NAB];
            hrr_bra_vector<LA, LB, double>(b.Rx, b.Ry, b.Rz, Xs, J);
            const uint64_t mask = __ldg(bra.rec_mask + r);
#pragma unroll
            for (int c = 0; c < NAB; c++) {
                if ((mask >> c) & 1ull) {
                    const int32_t o = __ldg(bra.entry + c * bra.sp_stride + sp);
                    mat_J[o] += __ldg(bra.pdata + o) * J[c];
                }
            }
        }
        __syncthreads();
    }
}

struct KOutBlocks {
    const int32_t* ish;  // [stride] primitive shell of i (type a)
    const int32_t* ksh;  // [stride] primitive shell of k (type c)
    const int32_t* idx;  // [NAC][stride] ik list position or -1
    int64_t stride;
    const int* n;
    const double* maxD;  // [stride] max |D| bound per block (batched calls), or null: the call's scalar
};

struct KPartnerRecs {
    const int32_t* rec_sp;     // [n_rec] shell pair, sorted by q descending inside each segment
    const double* rec_q;       // [n_rec] Schwarz value of the record
    const uint64_t* rec_mask;  // [n_rec] components owned by the record
    const int* seg;            // [nprim_first + 1] record offsets by first primitive shell
    const double* geo;         // [GEO_N][sp_stride]
    const double* S;           // [NXY][sp_stride] S_ij_00 (0 where absent)
    const int32_t* partner;    // [sp_stride] partner primitive shell (j or l)
    int64_t sp_stride;
    const double* su;          // [n_rec] S shared by all components of the record, or NaN
    const double* qa;          // [n_rec] |q| times the record's HRR growth (FP32 error budget), or null
    const double* qpre;        // [n_rec] inclusive prefix sum of qa, or null
};

struct KDensity {
    const uint32_t* b_aoinds;
    uint32_t b_count;
    const uint32_t* d_aoinds;
    uint32_t d_count;
    const double* D;
    uint32_t naos;
};

// Partner-pair enumeration of one chunk of j records of an output block:
// nl[t] / n64[t] = passing / FP64 prefix lengths of the l list for j record
// jb + t, then exclusive scans c64 (FP64 pairs) and c32 (FP32 pairs).
struct KChunk {
    int* nl;
    int* n64;
    int* c64;
    int* c32;
};

// FP32 error budget (budget > 0, aqa / cqpre non-null): the l tail of j runs
// in FP32 only as far as |q_j| A_j max_D * sum(|q_l| A_l) stays within
// budget / njtot (njtot = the block's j count, A the HRR growth of a pair).
__device__ __forceinline__ void k_chunk_scan(const double* __restrict__ aq, const double* __restrict__ cq, int jb,
                                             int nj, int c0, int c1, double maxD, double thr, double fp32_cut,
                                             KChunk s, const double* __restrict__ aqa = nullptr,
                                             const double* __restrict__ cqpre = nullptr, int njtot = 1,
                                             double budget = 0.0)
{
    for (int t = threadIdx.x; t < nj; t += blockDim.x) {
        const double qij = __ldg(aq + jb + t);
        int lo = c0, hi = c1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (fabs(qij * __ldg(cq + mid) * maxD) > thr) lo = mid + 1;
            else hi = mid;
        }
        const int nl = lo - c0;
        int n64 = nl;
        if (fp32_cut > 0.0) {
            int lo2 = c0, hi2 = lo;
            while (lo2 < hi2) {
                const int mid = (lo2 + hi2) >> 1;
                if (fabs(qij * __ldg(cq + mid) * maxD) >= fp32_cut) lo2 = mid + 1;
                else hi2 = mid;
            }
            n64 = lo2 - c0;
            if (budget > 0.0 && aqa && cqpre && n64 < nl) {
                const double qa = __ldg(aqa + jb + t) * fabs(maxD);
                const double bj = budget / (double)(njtot > 0 ? njtot : 1);
                const double pend = __ldg(cqpre + c0 + nl - 1);
                int lo4 = c0 + n64, hi4 = c0 + nl;
                while (lo4 < hi4) {
                    const int mid = (lo4 + hi4) >> 1;
                    const double tail = pend - (mid > 0 ? __ldg(cqpre + mid - 1) : 0.0);
                    if (qa * tail <= bj) hi4 = mid;
                    else lo4 = mid + 1;
                }
                n64 = lo4 - c0;
            }
        }
        s.nl[t] = nl;
        s.n64[t] = n64;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        s.c64[0] = 0;
        s.c32[0] = 0;
        for (int t = 0; t < nj; t++) {
            s.c64[t + 1] = s.c64[t] + s.n64[t];
            s.c32[t + 1] = s.c32[t] + (s.nl[t] - s.n64[t]);
        }
    }
    __syncthreads();
}

__device__ __forceinline__ void k_chunk_scan(const KPartnerRecs& ab, const KPartnerRecs& cd, int jb, int nj, int c0,
                                             int c1, double maxD, double thr, double fp32_cut, KChunk s,
                                             int njtot = 1, double budget = 0.0)
{
    k_chunk_scan(ab.rec_q, cd.rec_q, jb, nj, c0, c1, maxD, thr, fp32_cut, s, ab.qa, cd.qpre, njtot, budget);
}

// index t of the last entry with c[t] <= w (c ascending, c[0] = 0 <= w)
__device__ __forceinline__ int k_find(const int* c, int n, int w)
{
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (c[mid] <= w) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void k_quartet(const KPartnerRecs& ab, const KPartnerRecs& cd, int jr, int lr,
                                          const KDensity& dm, double omega, const BoysTabs& tabs, double* Kacc)
{
    constexpr int L = LA + LB + LC + LD;
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    const int spj = __ldg(ab.rec_sp + jr), spl = __ldg(cd.rec_sp + lr);
    const PairGeo bg = load_geo(ab.geo, ab.sp_stride, spj);
    const PairGeo kg = load_geo(cd.geo, cd.sp_stride, spl);
    QVT<T> q;
    T F[L + 1];
    make_quartet_t<L>(bg, kg, omega, tabs.f64, tabs.f32, q, F);
    T I[NA * NB * NC * ND];
    eri_full<LA, LB, LC, LD, T>(q, F, I);
    const int jsh = __ldg(ab.partner + spj), lsh = __ldg(cd.partner + spl);
    T Dv[NB * ND];
#pragma unroll
    for (int cb = 0; cb < NB; cb++) {
        const uint32_t jao = __ldg(dm.b_aoinds + jsh + (int64_t)dm.b_count * cb);
#pragma unroll
        for (int cdd = 0; cdd < ND; cdd++) {
            const uint32_t lao = __ldg(dm.d_aoinds + lsh + (int64_t)dm.d_count * cdd);
            Dv[cb * ND + cdd] = (T)__ldg(dm.D + (int64_t)jao * dm.naos + lao);
        }
    }
    const double suj = __ldg(ab.su + jr), sul = __ldg(cd.su + lr);
    if (!isnan(suj) && !isnan(sul)) {
        // every component of both records shares one S: K[a][c] += Sij Skl sum_bd (ab|cd) D[b][d]
        const T fs = (T)(suj * sul);
#pragma unroll
        for (int ca = 0; ca < NA; ca++)
#pragma unroll
            for (int cc = 0; cc < NC; cc++) {
                T acc = (T)0;
#pragma unroll
                for (int cb = 0; cb < NB; cb++)
#pragma unroll
                    for (int cdd = 0; cdd < ND; cdd++)
                        acc = fma(I[((ca * NB + cb) * NC + cc) * ND + cdd], Dv[cb * ND + cdd], acc);
                Kacc[ca * NC + cc] += (double)(acc * fs);
            }
        return;
    }
    T Sij[NA * NB], Skl[NC * ND];
    const uint64_t mj = __ldg(ab.rec_mask + jr), ml = __ldg(cd.rec_mask + lr);
#pragma unroll
    for (int x = 0; x < NA * NB; x++)
        Sij[x] = ((mj >> x) & 1ull) ? (T)__ldg(ab.S + x * ab.sp_stride + spj) : (T)0;
#pragma unroll
    for (int x = 0; x < NC * ND; x++)
        Skl[x] = ((ml >> x) & 1ull) ? (T)__ldg(cd.S + x * cd.sp_stride + spl) : (T)0;
#pragma unroll
    for (int ca = 0; ca < NA; ca++)
#pragma unroll
        for (int cc = 0; cc < NC; cc++) {
            T acc = (T)0;
#pragma unroll
            for (int cb = 0; cb < NB; cb++) {
                T s = (T)0;
#pragma unroll
                for (int cdd = 0; cdd < ND; cdd++)
                    s = fma(I[((ca * NB + cb) * NC + cc) * ND + cdd] * Skl[cc * ND + cdd], Dv[cb * ND + cdd], s);
                acc = fma(s, Sij[ca * NB + cb], acc);
            }
            Kacc[ca * NC + cc] += (double)acc;
        }
}

// PM as for coulomb_kernel.
template <int LA, int LB, int LC, int LD, int PM>
__global__ void __launch_bounds__(K_THREADS)
exchange_kernel(KOutBlocks out, KPartnerRecs ab, KPartnerRecs cd, KDensity dm, double maxD, double omega, double thr,
                double* __restrict__ mat_K, BoysTabs tabs, unsigned long long* __restrict__ qcount, double fp32_cut,
                double fp32_budget)
{
    constexpr int NA = ncart(LA), NC = ncart(LC);
    constexpr int NAC = NA * NC;
    constexpr int NW = K_THREADS / 32;
    __shared__ int s_nl[K_JCHUNK], s_n64[K_JCHUNK], s_c64[K_JCHUNK + 1], s_c32[K_JCHUNK + 1];
    __shared__ double red[NW][NAC];
    const KChunk ch{s_nl, s_n64, s_c64, s_c32};
    const int nout = *out.n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    for (int o = blockIdx.x; o < nout; o += gridDim.x) {
        const int ish = __ldg(out.ish + o), ksh = __ldg(out.ksh + o);
        const double mD = out.maxD ? __ldg(out.maxD + o) : maxD;
        const int a0 = __ldg(ab.seg + ish), a1 = __ldg(ab.seg + ish + 1);
        const int c0 = __ldg(cd.seg + ksh), c1 = __ldg(cd.seg + ksh + 1);
        double Kacc[NAC];
#pragma unroll
        for (int x = 0; x < NAC; x++) Kacc[x] = 0.0;

        for (int jb = a0; jb < a1; jb += K_JCHUNK) {
            const int nj = min(K_JCHUNK, a1 - jb);
            k_chunk_scan(ab, cd, jb, nj, c0, c1, mD, thr, fp32_cut, ch, a1 - a0, fp32_budget);
            const int t64 = s_c64[nj], t32 = s_c32[nj];
            if (qcount && PM == 0 && threadIdx.x == 0) atomicAdd(qcount, (unsigned long long)(t64 + t32));
            if (PM == 0) {
                for (int w = threadIdx.x; w < t64; w += K_THREADS) {
                    const int jj = k_find(s_c64, nj, w);
                    k_quartet<LA, LB, LC, LD, double>(ab, cd, jb + jj, c0 + (w - s_c64[jj]), dm, omega, tabs, Kacc);
                }
            } else {
                for (int w = threadIdx.x; w < t32; w += K_THREADS) {
                    const int jj = k_find(s_c32, nj, w);
                    k_quartet<LA, LB, LC, LD, float>(ab, cd, jb + jj, c0 + s_n64[jj] + (w - s_c32[jj]), dm, omega,
                                                     tabs, Kacc);
                }
            }
            __syncthreads();
        }

#pragma unroll
        for (int x = 0; x < NAC; x++) {
            const double v = warp_sum(Kacc[x]);
            if (lane == 0) red[warp][x] = v;
        }
        __syncthreads();
        if (threadIdx.x < NAC) {
            double s = red[0][threadIdx.x];
#pragma unroll
            for (int w = 1; w < NW; w++) s += red[w][threadIdx.x];
            const int32_t p = __ldg(out.idx + threadIdx.x * out.stride + o);
            if (p >= 0) mat_K[p] += s;
        }
        __syncthreads();
    }
}

}  // namespace vlxb
