// Per-class host drivers: regroup the caller's lists on the device, then
// launch the class's integral kernel, all on the caller's stream.
#pragma once
#include <atomic>

#include "col_kernels.cuh"
#include "engine.cuh"
#include "jk_kernels.cuh"
#include "jtma_kernels.cuh"
#include "md_kernels.cuh"
#include "jgrad_kernels.cuh"
#include "kgrad_kernels.cuh"

namespace vlxb {

struct CoulombArgs {
    double* mat_J;
    const double* info[4];  // prim_info by angular momentum (s, p, d, f)
    uint32_t count[4];      // prim_count by angular momentum
    const double* cd_D;
    const double* ab_Q;
    const double* cd_Q;
    const uint32_t* ab_first;
    const uint32_t* ab_second;
    const double* ab_pdata;
    uint32_t n_ab;
    const uint32_t* cd_first;
    const uint32_t* cd_second;
    const double* cd_pdata;
    uint32_t n_cd;
    double thr;
    // batched calls over several molecules (null / 0 for a class call): the
    // molecule of every primitive of types a and c; a bra pairs only with
    // kets of its own molecule
    const int32_t* prim_mol_a;
    const int32_t* prim_mol_c;
    int n_mol;
};

struct ExchangeArgs {
    double* mat_K;
    const uint32_t* pair_i;
    const uint32_t* pair_k;
    uint32_t n_ik;
    const double* info[4];
    const uint32_t* aoinds[4];
    uint32_t count[4];
    double maxD;
    const double* D;
    uint32_t naos;
    const double *Q_ab, *Q_cd;
    const uint32_t *Dinds_ab, *Dinds_cd;
    const uint32_t *displs_ab, *displs_cd;
    const uint32_t *counts_ab, *counts_cd;
    const double *pdata_ab, *pdata_cd;
    double omega;
    double thr;
    // batched calls over several molecules (all null / 0 for a class call):
    const uint32_t* aoinds_col[4];  // density column index per prim component (default: aoinds)
    uint32_t D_stride;              // row stride of D (default: naos)
    uint32_t key_naos;              // bound on the AO indices in aoinds (default: naos)
    const int32_t* prim_mol_a;      // molecule of every type-a primitive
    const double* maxD_mol;         // [molecules] max |D| bound of each molecule
};

// The staged Coulomb kernel's shared memory exceeds the 48 KB default for
// kets with d functions: raise the limit once per device for each of its
// two instantiations.
template <int LA, int LB, int LC, int LD>
int jtma_prepare_launch()
{
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    VLXB_CHECK_CUDA(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return VLXB_OK;
    const int smem = (int)JTmaShape<LC, LD>::SMEM;
    VLXB_CHECK_CUDA(cudaFuncSetAttribute(coulomb_tma_kernel<LA, LB, LC, LD, 0>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    VLXB_CHECK_CUDA(cudaFuncSetAttribute(coulomb_tma_kernel<LA, LB, LC, LD, 1>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    done.fetch_or(bit, std::memory_order_acq_rel);
    return VLXB_OK;
}

// Coulomb class call on a given arena (pool, static or measuring) with given
// Boys tables and quartet counter (may be null).  G = 1: the bra-centre
// derivatives of J instead (coulomb_grad_kernel), written to
// a.mat_J[k * gstride + o], k = 0..5.
template <int LA, int LB, int LC, int LD, int G = 0>
int run_coulomb_impl(const CoulombArgs& a, cudaStream_t st, Arena& ar, const BoysTabs& tab,
                     unsigned long long* qc, double cut, int64_t gstride = 0)
{
    if (a.n_ab == 0 || a.n_cd == 0) return VLXB_OK;
    if (!a.mat_J || !a.cd_D || !a.ab_Q || !a.cd_Q || !a.ab_first || !a.ab_second || !a.ab_pdata || !a.cd_first ||
        !a.cd_second || !a.cd_pdata)
        return VLXB_EINVAL;
    const int L4[4] = {LA, LB, LC, LD};
    for (int t = 0; t < 4; t++)
        if (!a.info[L4[t]] || a.count[L4[t]] == 0) return VLXB_EINVAL;
    if (!(a.thr >= 0.0)) return VLXB_EINVAL;
    if (G && gstride < (int64_t)a.n_ab) return VLXB_EINVAL;
    if (!tab.f64 || !tab.f32) return VLXB_ECUDA;
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    PairGroups gb, gk;
    int rc = group_flat(ar, NA, NB, (int)a.count[LA], (int)a.count[LB], a.ab_first, a.ab_second, a.n_ab,
                        a.info[LA], a.count[LA], a.info[LB], a.count[LB], gb);
    if (rc) return rc;
    rc = make_records(ar, NA * NB, gb, a.ab_Q, a.n_ab);
    if (rc) return rc;
    rc = group_flat(ar, NC, ND, (int)a.count[LC], (int)a.count[LD], a.cd_first, a.cd_second, a.n_cd, a.info[LC],
                    a.count[LC], a.info[LD], a.count[LD], gk);
    if (rc) return rc;
    const bool batched = a.prim_mol_a && a.prim_mol_c && a.n_mol > 0;
    JKetData kd;
    const int jvar = G ? 2 : schedule_get(0, LA, LB, LC, LD);
    rc = jket_prepare<LC, LD>(ar, gk, a.cd_first, a.cd_second, a.cd_D, a.cd_Q, a.cd_pdata, kd,
                              batched ? a.prim_mol_c : nullptr, batched ? a.n_mol : 0, jvar == 2);
    if (rc) return rc;
    const double budget = (cut > 0.0 && !G) ? fp32_budget_get() : 0.0;
    if (budget > 0.0) {
        rc = budget_prefix_kets(ar, kd, LD);
        if (rc) return rc;
    }
    int32_t* bmol = nullptr;
    if (batched) {
        rc = bra_record_mol(ar, gb, a.prim_mol_a, &bmol);
        if (rc) return rc;
    }
    if (ar.failed()) return VLXB_ENOMEM;
    if (ar.measuring()) return VLXB_OK;
    JBraRecs bra{gb.rec_sp, gb.rec_q, gb.rec_mask, gb.n_rec, gb.geo, gb.entry, gb.sp_stride, a.ab_pdata, bmol};
    JKetPairs ket{kd.geo, kd.tmax, kd.tmin, kd.Dpp, kd.Dm, kd.Qc, kd.Dc, kd.stride, kd.n, batched ? kd.seg : nullptr,
                  kd.Dh, kd.tpre};
    int grid = launch_grid_limit();
    if ((int64_t)grid > (int64_t)a.n_ab) grid = (int)a.n_ab;
    unsigned long long* kerr = kernel_errors_device();
    if (jvar == 3 && !kerr) return VLXB_ECUDA;
    for (int pm = 0; pm < (cut > 0.0 ? 2 : 1); pm++) {
        if constexpr (G == 1) {
            constexpr int GT = JGradShape<LA, LB, LC, LD>::THREADS;
            if (pm == 0)
                coulomb_grad_kernel<LA, LB, LC, LD, 0><<<grid, GT, 0, st>>>(bra, ket, a.mat_J, gstride, a.thr, tab,
                                                                            cut);
            else
                coulomb_grad_kernel<LA, LB, LC, LD, 1><<<grid, GT, 0, st>>>(bra, ket, a.mat_J, gstride, a.thr, tab,
                                                                            cut);
        } else if (jvar == 2) {
            if (pm == 0)
                coulomb_md_kernel<LA, LB, LC, LD, 0><<<grid, MD_THREADS, 0, st>>>(bra, ket, a.mat_J, a.thr, tab, qc,
                                                                                  cut, budget);
            else
                coulomb_md_kernel<LA, LB, LC, LD, 1><<<grid, MD_THREADS, 0, st>>>(bra, ket, a.mat_J, a.thr, tab, qc,
                                                                                  cut, budget);
        } else if (jvar == 3) {
            using JS = JTmaShape<LC, LD>;
            int rc2 = jtma_prepare_launch<LA, LB, LC, LD>();
            if (rc2) return rc2;
            if (pm == 0)
                coulomb_tma_kernel<LA, LB, LC, LD, 0><<<grid, JT_TILE, JS::SMEM, st>>>(bra, ket, a.mat_J, a.thr, tab,
                                                                                      qc, cut, budget, kerr);
            else
                coulomb_tma_kernel<LA, LB, LC, LD, 1><<<grid, JT_TILE, JS::SMEM, st>>>(bra, ket, a.mat_J, a.thr, tab,
                                                                                      qc, cut, budget, kerr);
        } else if (jvar == 1) {
            if (pm == 0)
                coulomb_col_kernel<LA, LB, LC, LD, 0><<<grid, J_THREADS, 0, st>>>(bra, ket, a.mat_J, a.thr, tab, qc,
                                                                                  cut, budget);
            else
                coulomb_col_kernel<LA, LB, LC, LD, 1><<<grid, J_THREADS, 0, st>>>(bra, ket, a.mat_J, a.thr, tab, qc,
                                                                                  cut, budget);
        } else {
            if (pm == 0)
                coulomb_kernel<LA, LB, LC, LD, 0><<<grid, J_THREADS, 0, st>>>(bra, ket, a.mat_J, a.thr, tab, qc, cut,
                                                                               budget);
            else
                coulomb_kernel<LA, LB, LC, LD, 1><<<grid, J_THREADS, 0, st>>>(bra, ket, a.mat_J, a.thr, tab, qc, cut,
                                                                               budget);
        }
        note_launches();
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

template <int LA, int LB, int LC, int LD>
int run_coulomb(const CoulombArgs& a, cudaStream_t st)
{
    if (a.n_ab == 0 || a.n_cd == 0) return VLXB_OK;
    int rc = ensure_pool_configured();
    if (rc) return rc;
    const BoysTabs tab{boys_table_device(), boys_table32_device()};
    if (!tab.f64 || !tab.f32) return VLXB_ECUDA;
    Arena ar(st);
    return run_coulomb_impl<LA, LB, LC, LD>(a, st, ar, tab, quartet_counters_device(), fp32_cut_get());
}

// Bra-centre derivatives of one Coulomb class: grad[k * gstride + o] +=
// d mat_J[o] / d (A_x, A_y, A_z, B_x, B_y, B_z)[k], ket held fixed.
template <int LA, int LB, int LC, int LD>
int run_coulomb_grad(const CoulombArgs& a, int64_t gstride, cudaStream_t st)
{
    if (a.n_ab == 0 || a.n_cd == 0) return VLXB_OK;
    int rc = ensure_pool_configured();
    if (rc) return rc;
    const BoysTabs tab{boys_table_device(), boys_table32_device()};
    if (!tab.f64 || !tab.f32) return VLXB_ECUDA;
    Arena ar(st);
    return run_coulomb_impl<LA, LB, LC, LD, 1>(a, st, ar, tab, nullptr, fp32_cut_get(), gstride);
}

// One contracted-partner column exchange launch of plan kind ORI when that
// plan is built for the class; false otherwise.
template <int LA, int LB, int LC, int LD, int ORI>
bool launch_exchange_colc(int pm, int grid, cudaStream_t st, const KOutBlocks& out, const KPartnerRecs& rab,
                          const KPartnerRecs& rcd, const KGroups& kgab, const KGroups& kgcd, const KDensity& dm,
                          const ExchangeArgs& a, const BoysTabs& tab, unsigned long long* qk, double cut, double budget)
{
    if constexpr (ColTab<LA, LB, LC, LD, ORI>::K_FITS) {
        if (pm == 0)
            exchange_colc_kernel<LA, LB, LC, LD, ORI, 0><<<grid, K_THREADS, 0, st>>>(
                out, rab, rcd, kgab, kgcd, dm, a.maxD, a.omega, a.thr, a.mat_K, tab, qk, cut, budget);
        else
            exchange_colc_kernel<LA, LB, LC, LD, ORI, 1><<<grid, K_THREADS, 0, st>>>(
                out, rab, rcd, kgab, kgcd, dm, a.maxD, a.omega, a.thr, a.mat_K, tab, qk, cut, budget);
        return true;
    } else {
        return false;
    }
}

// One column exchange launch of plan kind ORI when that plan is built for the
// class (its ColTab fits); false otherwise.
template <int LA, int LB, int LC, int LD, int ORI>
bool launch_exchange_col(int pm, int grid, cudaStream_t st, const KOutBlocks& out, const KPartnerRecs& rab,
                         const KPartnerRecs& rcd, const KDensity& dm, const ExchangeArgs& a, const BoysTabs& tab,
                         unsigned long long* qk, double cut, double budget)
{
    if constexpr (ColTab<LA, LB, LC, LD, ORI>::K_FITS) {
        if (pm == 0)
            exchange_col_kernel<LA, LB, LC, LD, ORI, 0><<<grid, K_THREADS, 0, st>>>(
                out, rab, rcd, dm, a.maxD, a.omega, a.thr, a.mat_K, tab, qk, cut, budget);
        else
            exchange_col_kernel<LA, LB, LC, LD, ORI, 1><<<grid, K_THREADS, 0, st>>>(
                out, rab, rcd, dm, a.maxD, a.omega, a.thr, a.mat_K, tab, qk, cut, budget);
        return true;
    } else {
        return false;
    }
}

template <int LA, int LB, int LC, int LD>
int run_exchange(const ExchangeArgs& a, cudaStream_t st)
{
    if (a.n_ik == 0) return VLXB_OK;
    if (!a.mat_K || !a.pair_i || !a.pair_k || !a.D || !a.Q_ab || !a.Q_cd || !a.Dinds_ab || !a.Dinds_cd ||
        !a.displs_ab || !a.displs_cd || !a.counts_ab || !a.counts_cd || !a.pdata_ab || !a.pdata_cd || a.naos == 0)
        return VLXB_EINVAL;
    const int L4[4] = {LA, LB, LC, LD};
    for (int t = 0; t < 4; t++)
        if (!a.info[L4[t]] || !a.aoinds[L4[t]] || a.count[L4[t]] == 0) return VLXB_EINVAL;
    if (!(a.thr >= 0.0) || !(a.omega >= 0.0)) return VLXB_EINVAL;
    int rc = ensure_pool_configured();
    if (rc) return rc;
    const BoysTabs tab{boys_table_device(), boys_table32_device()};
    if (!tab.f64 || !tab.f32) return VLXB_ECUDA;
    const double cut = fp32_cut_get();
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    Arena ar(st);
    KOutData ko;
    rc = kout_prepare(ar, NA, NC, (int)a.count[LA], (int)a.count[LC], a.pair_i, a.pair_k, a.n_ik, ko);
    if (rc) return rc;
    const int npa = (int)a.count[LA], npb = (int)a.count[LB], npc = (int)a.count[LC], npd = (int)a.count[LD];
    PairGroups gab;
    rc = group_csr(ar, NA, NB, npa, npb, a.displs_ab, a.counts_ab, a.Dinds_ab, (int64_t)npa * npb, a.info[LA],
                   a.count[LA], a.info[LB], a.count[LB], gab);
    if (rc) return rc;
    rc = make_records(ar, NA * NB, gab, a.Q_ab, (int64_t)npa * npb * NA * NB);
    if (rc) return rc;
    rc = segment_records(ar, NA * NB, npa, npb, gab, a.pdata_ab);
    if (rc) return rc;
    PairGroups gcd;
    const bool same = (LA == LC && LB == LD && a.Q_ab == a.Q_cd && a.Dinds_ab == a.Dinds_cd &&
                       a.displs_ab == a.displs_cd && a.counts_ab == a.counts_cd && a.pdata_ab == a.pdata_cd);
    if (same) {
        gcd = gab;
    } else {
        rc = group_csr(ar, NC, ND, npc, npd, a.displs_cd, a.counts_cd, a.Dinds_cd, (int64_t)npc * npd, a.info[LC],
                       a.count[LC], a.info[LD], a.count[LD], gcd);
        if (rc) return rc;
        rc = make_records(ar, NC * ND, gcd, a.Q_cd, (int64_t)npc * npd * NC * ND);
        if (rc) return rc;
        rc = segment_records(ar, NC * ND, npc, npd, gcd, a.pdata_cd);
        if (rc) return rc;
    }
    const int var = schedule_get(1, LA, LB, LC, LD);
    const double budget = cut > 0.0 ? fp32_budget_get() : 0.0;
    KGroups kgab{}, kgcd{};
    const uint32_t key_naos = a.key_naos ? a.key_naos : a.naos;
    if (var == 3 || var == 4 || var >= 9) {
        // contracted variants: group partner records by contracted partner shell
        rc = contract_groups(ar, npa, gab, a.aoinds[LB], key_naos);
        if (rc) return rc;
        if (same) {
            gcd = gab;
        } else {
            rc = contract_groups(ar, npc, gcd, a.aoinds[LD], key_naos);
            if (rc) return rc;
        }
    }
    if (budget > 0.0) {
        // after contract_groups: groups get their amplified sums too
        rc = budget_prefix_records(ar, gab, npa, LB);
        if (rc) return rc;
        if (same) {
            gcd = gab;
        } else {
            rc = budget_prefix_records(ar, gcd, npc, LD);
            if (rc) return rc;
        }
    }
    if (var == 3 || var == 4 || var >= 9) {
        kgab = KGroups{gab.gseg, gab.gq, gab.gbeg, gab.gcnt, gab.msp, gab.mq, gab.msu, gab.mmask, gab.gqa, gab.gqpre};
        kgcd = KGroups{gcd.gseg, gcd.gq, gcd.gbeg, gcd.gcnt, gcd.msp, gcd.mq, gcd.msu, gcd.mmask, gcd.gqa, gcd.gqpre};
    }
    double* blk_maxD = nullptr;
    if (a.prim_mol_a && a.maxD_mol) {
        rc = kout_block_maxd(ar, ko, a.prim_mol_a, a.maxD_mol, &blk_maxD);
        if (rc) return rc;
    }
    KOutBlocks out{ko.ish, ko.ksh, ko.idx, ko.stride, ko.n, blk_maxD};
    KPartnerRecs rab{gab.rec_sp, gab.rec_q, gab.rec_mask, gab.seg, gab.geo, gab.S, gab.sp_j, gab.sp_stride, gab.su,
                     gab.rec_qa, gab.rec_qpre};
    KPartnerRecs rcd{gcd.rec_sp, gcd.rec_q, gcd.rec_mask, gcd.seg, gcd.geo, gcd.S, gcd.sp_j, gcd.sp_stride, gcd.su,
                     gcd.rec_qa, gcd.rec_qpre};
    int grid = launch_grid_limit();
    if ((int64_t)grid > (int64_t)a.n_ik) grid = (int)a.n_ik;
    unsigned long long* qc = quartet_counters_device();
    unsigned long long* qk = qc ? qc + 1 : nullptr;
    const KDensity dm{a.aoinds[LB], a.count[LB], a.aoinds_col[LD] ? a.aoinds_col[LD] : a.aoinds[LD], a.count[LD],
                      a.D, a.D_stride ? a.D_stride : a.naos};
    for (int pm = 0; pm < (cut > 0.0 ? 2 : 1); pm++) {
        bool launched = false;
        // column kernels: variants 1, 2 = plan kinds 0, 1; variants 5..8 = packed kinds 2..5;
        // contracted-partner column kernels: variants 3, 4 = kinds 0, 1; 9..12 = kinds 2..5
        switch (var) {
            case 3: launched = launch_exchange_colc<LA, LB, LC, LD, 0>(pm, grid, st, out, rab, rcd, kgab, kgcd, dm, a, tab, qk, cut, budget); break;
            case 4: launched = launch_exchange_colc<LA, LB, LC, LD, 1>(pm, grid, st, out, rab, rcd, kgab, kgcd, dm, a, tab, qk, cut, budget); break;
            case 9: launched = launch_exchange_colc<LA, LB, LC, LD, 2>(pm, grid, st, out, rab, rcd, kgab, kgcd, dm, a, tab, qk, cut, budget); break;
            case 10: launched = launch_exchange_colc<LA, LB, LC, LD, 3>(pm, grid, st, out, rab, rcd, kgab, kgcd, dm, a, tab, qk, cut, budget); break;
            case 11: launched = launch_exchange_colc<LA, LB, LC, LD, 4>(pm, grid, st, out, rab, rcd, kgab, kgcd, dm, a, tab, qk, cut, budget); break;
            case 12: launched = launch_exchange_colc<LA, LB, LC, LD, 5>(pm, grid, st, out, rab, rcd, kgab, kgcd, dm, a, tab, qk, cut, budget); break;
            default: break;
        }
        switch (var) {
            case 1: launched = launch_exchange_col<LA, LB, LC, LD, 0>(pm, grid, st, out, rab, rcd, dm, a, tab, qk, cut, budget); break;
            case 2: launched = launch_exchange_col<LA, LB, LC, LD, 1>(pm, grid, st, out, rab, rcd, dm, a, tab, qk, cut, budget); break;
            case 5: launched = launch_exchange_col<LA, LB, LC, LD, 2>(pm, grid, st, out, rab, rcd, dm, a, tab, qk, cut, budget); break;
            case 6: launched = launch_exchange_col<LA, LB, LC, LD, 3>(pm, grid, st, out, rab, rcd, dm, a, tab, qk, cut, budget); break;
            case 7: launched = launch_exchange_col<LA, LB, LC, LD, 4>(pm, grid, st, out, rab, rcd, dm, a, tab, qk, cut, budget); break;
            case 8: launched = launch_exchange_col<LA, LB, LC, LD, 5>(pm, grid, st, out, rab, rcd, dm, a, tab, qk, cut, budget); break;
            default: break;
        }
        if (!launched) {
            if (pm == 0)
                exchange_kernel<LA, LB, LC, LD, 0><<<grid, K_THREADS, 0, st>>>(out, rab, rcd, dm, a.maxD, a.omega,
                                                                               a.thr, a.mat_K, tab, qk, cut, budget);
            else
                exchange_kernel<LA, LB, LC, LD, 1><<<grid, K_THREADS, 0, st>>>(out, rab, rcd, dm, a.maxD, a.omega,
                                                                               a.thr, a.mat_K, tab, qk, cut, budget);
        }
        note_launches();
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

// Energy-weighted centre derivatives of one exchange class (see
// exchange_grad_kernel): grad[x * gstride + p] += ..., p the lowest (i, k)
// list position of each primitive shell block.  FP64, single-molecule calls.
template <int LA, int LB, int LC, int LD>
int run_exchange_grad(const ExchangeArgs& a, int64_t gstride, cudaStream_t st)
{
    if (a.n_ik == 0) return VLXB_OK;
    if (!a.mat_K || !a.pair_i || !a.pair_k || !a.D || !a.Q_ab || !a.Q_cd || !a.Dinds_ab || !a.Dinds_cd ||
        !a.displs_ab || !a.displs_cd || !a.counts_ab || !a.counts_cd || !a.pdata_ab || !a.pdata_cd || a.naos == 0)
        return VLXB_EINVAL;
    const int L4[4] = {LA, LB, LC, LD};
    for (int t = 0; t < 4; t++)
        if (!a.info[L4[t]] || !a.aoinds[L4[t]] || a.count[L4[t]] == 0) return VLXB_EINVAL;
    if (!(a.thr >= 0.0) || !(a.omega >= 0.0)) return VLXB_EINVAL;
    if (gstride < (int64_t)a.n_ik) return VLXB_EINVAL;
    int rc = ensure_pool_configured();
    if (rc) return rc;
    const BoysTabs tab{boys_table_device(), boys_table32_device()};
    if (!tab.f64) return VLXB_ECUDA;
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    Arena ar(st);
    KOutData ko;
    rc = kout_prepare(ar, NA, NC, (int)a.count[LA], (int)a.count[LC], a.pair_i, a.pair_k, a.n_ik, ko);
    if (rc) return rc;
    const int npa = (int)a.count[LA], npb = (int)a.count[LB], npc = (int)a.count[LC], npd = (int)a.count[LD];
    PairGroups gab;
    rc = group_csr(ar, NA, NB, npa, npb, a.displs_ab, a.counts_ab, a.Dinds_ab, (int64_t)npa * npb, a.info[LA],
                   a.count[LA], a.info[LB], a.count[LB], gab);
    if (rc) return rc;
    rc = make_records(ar, NA * NB, gab, a.Q_ab, (int64_t)npa * npb * NA * NB);
    if (rc) return rc;
    rc = segment_records(ar, NA * NB, npa, npb, gab, a.pdata_ab);
    if (rc) return rc;
    PairGroups gcd;
    const bool same = (LA == LC && LB == LD && a.Q_ab == a.Q_cd && a.Dinds_ab == a.Dinds_cd &&
                       a.displs_ab == a.displs_cd && a.counts_ab == a.counts_cd && a.pdata_ab == a.pdata_cd);
    if (same) {
        gcd = gab;
    } else {
        rc = group_csr(ar, NC, ND, npc, npd, a.displs_cd, a.counts_cd, a.Dinds_cd, (int64_t)npc * npd, a.info[LC],
                       a.count[LC], a.info[LD], a.count[LD], gcd);
        if (rc) return rc;
        rc = make_records(ar, NC * ND, gcd, a.Q_cd, (int64_t)npc * npd * NC * ND);
        if (rc) return rc;
        rc = segment_records(ar, NC * ND, npc, npd, gcd, a.pdata_cd);
        if (rc) return rc;
    }
    if (ar.failed()) return VLXB_ENOMEM;
    KOutBlocks out{ko.ish, ko.ksh, ko.idx, ko.stride, ko.n, nullptr};
    KPartnerRecs rab{gab.rec_sp, gab.rec_q, gab.rec_mask, gab.seg, gab.geo, gab.S, gab.sp_j, gab.sp_stride, gab.su,
                     nullptr, nullptr};
    KPartnerRecs rcd{gcd.rec_sp, gcd.rec_q, gcd.rec_mask, gcd.seg, gcd.geo, gcd.S, gcd.sp_j, gcd.sp_stride, gcd.su,
                     nullptr, nullptr};
    const KDensity dm{a.aoinds[LB], a.count[LB], a.aoinds[LD], a.count[LD], a.D, a.naos};
    const KGradBlockD bd{a.aoinds[LA], a.count[LA], a.aoinds[LC], a.count[LC], LA == LC ? 1 : 0};
    int grid = launch_grid_limit();
    if ((int64_t)grid > (int64_t)a.n_ik) grid = (int)a.n_ik;
    exchange_grad_kernel<LA, LB, LC, LD><<<grid, KGradShape<LA, LB, LC, LD>::THREADS, 0, st>>>(
        out, rab, rcd, dm, bd, a.maxD, a.omega, a.thr, a.mat_K, gstride, tab);
    note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

}  // namespace vlxb
