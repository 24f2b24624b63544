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
#pragma once
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
};

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(J_THREADS)
coulomb_kernel(JBraRecs bra, JKetPairs ket, double* __restrict__ mat_J, double thr,
               const double* __restrict__ boys_tab, unsigned long long* __restrict__ qcount)
{
    constexpr int L = LA + LB + LC + LD;
    constexpr int NE = nrange(LA, LB), NF = nrange(LC, LD);
    constexpr int NAB = ncart(LA) * ncart(LB), NCD = ncart(LC) * ncart(LD);
    constexpr int NW = J_THREADS / 32;
    __shared__ double red[NW][NE];
    __shared__ int s_ncut;
    const int nbra = *bra.n_rec;
    const int nket = *ket.n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    for (int r = blockIdx.x; r < nbra; r += gridDim.x) {
        const int sp = __ldg(bra.rec_sp + r);
        const PairGeo b = load_geo(bra.geo, bra.sp_stride, sp);
        const double qb = __ldg(bra.rec_q + r);
        if (threadIdx.x == 0) {
            // kets with qb * tmax * (1 + slack) > thr form a prefix (tmax descending)
            int lo = 0, hi = nket;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (qb * __ldg(ket.tmax + mid) * (1.0 + SCREEN_SLACK) > thr) lo = mid + 1;
                else hi = mid;
            }
            s_ncut = lo;
            // screened-in shell quartets of this record (exact bound, no slack)
            int lo2 = 0, hi2 = lo;
            while (lo2 < hi2) {
                const int mid = (lo2 + hi2) >> 1;
                if (qb * __ldg(ket.tmax + mid) > thr) lo2 = mid + 1;
                else hi2 = mid;
            }
            if (qcount) atomicAdd(qcount, (unsigned long long)lo2);
        }
        __syncthreads();
        const int ncut = s_ncut;

        double X[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) X[e] = 0.0;

        for (int kt = threadIdx.x; kt < ncut; kt += J_THREADS) {
            const PairGeo k = load_geo(ket.geo, ket.stride, kt);
            QV q;
            double F[L + 1];
            make_quartet<L>(b, k, 0.0, boys_tab, q, F);
            double Dpp[NF];
            if (qb * __ldg(ket.tmin + kt) > thr * (1.0 + SCREEN_SLACK)) {
#pragma unroll
                for (int f = 0; f < NF; f++) Dpp[f] = __ldg(ket.Dpp + f * ket.stride + kt);
            } else {
                // exact per-component screen, same product order as the
                // reference: fabs(Q_ij * Q_kl * D_kl) <= thr -> skip
                double Dm[NCD];
#pragma unroll
                for (int c = 0; c < NCD; c++) {
                    const double qk = __ldg(ket.Qc + c * ket.stride + kt);
                    const double dk = __ldg(ket.Dc + c * ket.stride + kt);
                    Dm[c] = (fabs(qb * qk * dk) > thr) ? __ldg(ket.Dm + c * ket.stride + kt) : 0.0;
                }
                hrr_ket_adjoint<LC, LD>(k.Rx, k.Ry, k.Rz, Dm, Dpp);
            }
            j_contract<LA, LB, LC, LD>(q, F, Dpp, X);
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
            hrr_bra_vector<LA, LB>(b.Rx, b.Ry, b.Rz, Xs, J);
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
};

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(K_THREADS)
exchange_kernel(KOutBlocks out, KPartnerRecs ab, KPartnerRecs cd,
                const uint32_t* __restrict__ b_aoinds, uint32_t b_count,
                const uint32_t* __restrict__ d_aoinds, uint32_t d_count,
                const double* __restrict__ Dao, uint32_t naos, double maxD, double omega, double thr,
                double* __restrict__ mat_K, const double* __restrict__ boys_tab,
                unsigned long long* __restrict__ qcount)
{
    constexpr int L = LA + LB + LC + LD;
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr int NAC = NA * NC;
    constexpr int NW = K_THREADS / 32;
    __shared__ int s_cnt[K_JCHUNK + 1];
    __shared__ double red[NW][NAC];
    const int nout = *out.n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    for (int o = blockIdx.x; o < nout; o += gridDim.x) {
        const int ish = __ldg(out.ish + o), ksh = __ldg(out.ksh + o);
        const int a0 = __ldg(ab.seg + ish), a1 = __ldg(ab.seg + ish + 1);
        const int c0 = __ldg(cd.seg + ksh), c1 = __ldg(cd.seg + ksh + 1);
        double Kacc[NAC];
#pragma unroll
        for (int x = 0; x < NAC; x++) Kacc[x] = 0.0;

        for (int jb = a0; jb < a1; jb += K_JCHUNK) {
            const int nj = min(K_JCHUNK, a1 - jb);
            for (int t = threadIdx.x; t < nj; t += K_THREADS) {
                const double qij = __ldg(ab.rec_q + jb + t);
                int lo = c0, hi = c1;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (fabs(qij * __ldg(cd.rec_q + mid) * maxD) > thr) lo = mid + 1;
                    else hi = mid;
                }
                s_cnt[t + 1] = lo - c0;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                s_cnt[0] = 0;
                for (int t = 1; t <= nj; t++) s_cnt[t] += s_cnt[t - 1];
            }
            __syncthreads();
            const int total = s_cnt[nj];
            if (qcount && threadIdx.x == 0) atomicAdd(qcount, (unsigned long long)total);
            int jj = 0;
            for (int w = threadIdx.x; w < total; w += K_THREADS) {
                while (s_cnt[jj + 1] <= w) jj++;
                const int jr = jb + jj;
                const int lr = c0 + (w - s_cnt[jj]);
                const int spj = __ldg(ab.rec_sp + jr), spl = __ldg(cd.rec_sp + lr);
                const PairGeo bg = load_geo(ab.geo, ab.sp_stride, spj);
                const PairGeo kg = load_geo(cd.geo, cd.sp_stride, spl);
                QV q;
                double F[L + 1];
                make_quartet<L>(bg, kg, omega, boys_tab, q, F);
                double I[NA * NB * NC * ND];
                eri_full<LA, LB, LC, LD>(q, F, I);
                const int jsh = __ldg(ab.partner + spj), lsh = __ldg(cd.partner + spl);
                double Dv[NB * ND];
#pragma unroll
                for (int cb = 0; cb < NB; cb++) {
                    const uint32_t jao = __ldg(b_aoinds + jsh + (int64_t)b_count * cb);
#pragma unroll
                    for (int cdd = 0; cdd < ND; cdd++) {
                        const uint32_t lao = __ldg(d_aoinds + lsh + (int64_t)d_count * cdd);
                        Dv[cb * ND + cdd] = __ldg(Dao + (int64_t)jao * naos + lao);
                    }
                }
                double Sij[NA * NB], Skl[NC * ND];
                const uint64_t mj = __ldg(ab.rec_mask + jr), ml = __ldg(cd.rec_mask + lr);
#pragma unroll
                for (int x = 0; x < NA * NB; x++)
                    Sij[x] = ((mj >> x) & 1ull) ? __ldg(ab.S + x * ab.sp_stride + spj) : 0.0;
#pragma unroll
                for (int x = 0; x < NC * ND; x++)
                    Skl[x] = ((ml >> x) & 1ull) ? __ldg(cd.S + x * cd.sp_stride + spl) : 0.0;
#pragma unroll
                for (int ca = 0; ca < NA; ca++)
#pragma unroll
                    for (int cb = 0; cb < NB; cb++)
#pragma unroll
                        for (int cc = 0; cc < NC; cc++) {
                            double acc = 0.0;
#pragma unroll
                            for (int cdd = 0; cdd < ND; cdd++)
                                acc = fma(I[((ca * NB + cb) * NC + cc) * ND + cdd] * Skl[cc * ND + cdd],
                                          Dv[cb * ND + cdd], acc);
                            Kacc[ca * NC + cc] = fma(acc, Sij[ca * NB + cb], Kacc[ca * NC + cc]);
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
