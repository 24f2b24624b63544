// Coulomb kernel with the sorted ket stream staged into shared memory by the
// TMA engine (J schedule variant 3).
//
// Same work, screening, counters and precision passes as coulomb_kernel
// (jk_kernels.cuh): CTA per bra record, one ket per thread.  The kets of the
// record's screened prefix are consumed in tiles of JT_TILE (one per
// thread).  Per tile, one elected thread issues plain 1-D bulk copies
// (cp.async.bulk, no multicast) of the tile's rows of the sorted ket SoA --
// the 11 geometry rows, tmin and the transposed-HRR ket density D'' -- into
// one of two shared-memory stages, with an mbarrier counting the bytes; the
// CTA computes on the other stage meanwhile (double buffering), so the ket
// stream's latency is off the threads' critical path and every thread reads
// its ket from shared memory instead of through L1.
//
// Rows of the sorted ket arrays start on 16-byte boundaries (even row stride,
// jket_prepare); a tile starting at an odd ket is copied from the even ket
// before it, and its length rounded up to an even count (both stay inside
// the allocation), so every copy meets the bulk-copy alignment rules.
//
// A copy that has not landed after TMA_WAIT_LIMIT polls sets
// VLXB_KERR_TMA_TIMEOUT in the device error word; the CTA then waits (again
// bounded) for its copies in flight and stops.
#pragma once
#include <type_traits>

#include "jk_kernels.cuh"
#include "tma.cuh"

namespace vlxb {

constexpr int JT_TILE = 128;         // kets per tile, one per thread
constexpr int JT_ROW = JT_TILE + 2;  // a staged row: the tile plus the even-alignment slack
constexpr int JT_STAGES = 2;
constexpr int JT_GEO = 11;           // geometry rows the integrals read (G_Z .. G_RZ)

template <int LC, int LD>
struct JTmaShape {
    static constexpr int NF = nrange(LC, LD);
    static constexpr int NFLD = JT_GEO + 1 + NF;  // geometry, tmin, D''
    static constexpr size_t STAGE_DOUBLES = (size_t)NFLD * JT_ROW;
    static constexpr size_t SMEM = JT_STAGES * STAGE_DOUBLES * sizeof(double);
};

// Copies of kets [lo, hi) (hi - lo <= JT_TILE) into the stage buffer `buf`.
template <int LC, int LD>
__device__ __forceinline__ void jt_issue(const JKetPairs& ket, int lo, int hi, double* buf, uint64_t* bar)
{
    using S = JTmaShape<LC, LD>;
    const int al = lo & ~1;
    const int cnt = (hi - al + 1) & ~1;
    const uint32_t bytes = (uint32_t)cnt * 8u;
    mbar_arrive_expect_tx(bar, bytes * (uint32_t)S::NFLD);
    for (int f = 0; f < JT_GEO; f++) tma_load_1d(buf + f * JT_ROW, ket.geo + f * ket.stride + al, bytes, bar);
    tma_load_1d(buf + JT_GEO * JT_ROW, ket.tmin + al, bytes, bar);
    for (int f = 0; f < S::NF; f++)
        tma_load_1d(buf + (JT_GEO + 1 + f) * JT_ROW, ket.Dpp + f * ket.stride + al, bytes, bar);
}

// The exact per-component screen of a ket in the slack band (ket_density's
// second branch), from the ket arrays in global memory.
template <int LC, int LD, typename T>
__device__ __forceinline__ void ket_density_exact(const JKetPairs& ket, int kt, double qb, double thr,
                                                  const PairGeo& k, T* Dpp)
{
    constexpr int NCD = ncart(LC) * ncart(LD);
    T Dm[NCD];
#pragma unroll
    for (int c = 0; c < NCD; c++) {
        const double qk = __ldg(ket.Qc + c * ket.stride + kt);
        const double dk = __ldg(ket.Dc + c * ket.stride + kt);
        Dm[c] = (fabs(qb * qk * dk) > thr) ? (T)__ldg(ket.Dm + c * ket.stride + kt) : (T)0;
    }
    hrr_ket_adjoint<LC, LD, T>((T)k.Rx, (T)k.Ry, (T)k.Rz, Dm, Dpp);
}

// One quartet of a staged ket: geometry, tmin and D'' from the stage buffer
// (s points at the ket's column of the stage, rows JT_ROW apart).
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void j_quartet_staged(const PairGeo& b, double qb, const JKetPairs& ket, int kt,
                                                 const double* s, double thr, const BoysTabs& tabs, double* X)
{
    constexpr int L = LA + LB + LC + LD;
    constexpr int NE = nrange(LA, LB), NF = nrange(LC, LD);
    PairGeo k;
    k.z = s[G_Z * JT_ROW];
    k.i2z = s[G_I2Z * JT_ROW];
    k.Px = s[G_PX * JT_ROW];
    k.Py = s[G_PY * JT_ROW];
    k.Pz = s[G_PZ * JT_ROW];
    k.Ax = s[G_AX * JT_ROW];
    k.Ay = s[G_AY * JT_ROW];
    k.Az = s[G_AZ * JT_ROW];
    k.Rx = s[G_RX * JT_ROW];
    k.Ry = s[G_RY * JT_ROW];
    k.Rz = s[G_RZ * JT_ROW];
    const double tmin = s[JT_GEO * JT_ROW];
    QVT<T> q;
    T F[L + 1];
    make_quartet_t<L>(b, k, 0.0, tabs.f64, tabs.f32, q, F);
    T Dpp[NF];
    if (qb * tmin > thr * (1.0 + SCREEN_SLACK)) {
#pragma unroll
        for (int f = 0; f < NF; f++) Dpp[f] = (T)s[(JT_GEO + 1 + f) * JT_ROW];
    } else {
        ket_density_exact<LC, LD, T>(ket, kt, qb, thr, k, Dpp);
    }
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

template <int LA, int LB, int LC, int LD, int PM>
__global__ void __launch_bounds__(JT_TILE)
coulomb_tma_kernel(JBraRecs bra, JKetPairs ket, double* __restrict__ mat_J, double thr, BoysTabs tabs,
                   unsigned long long* __restrict__ qcount, double fp32_cut, double fp32_budget,
                   unsigned long long* __restrict__ errs)
{
    using T = typename std::conditional<PM == 0, double, float>::type;
    using S = JTmaShape<LC, LD>;
    constexpr int NE = nrange(LA, LB);
    constexpr int NAB = ncart(LA) * ncart(LB);
    constexpr int NW = JT_TILE / 32;
    extern __shared__ __align__(128) double jt_smem[];
    __shared__ __align__(8) uint64_t bars[JT_STAGES];
    __shared__ double red[NW][NE];
    __shared__ int s_ncut, s_n64;

    if (threadIdx.x == 0) {
        for (int s = 0; s < JT_STAGES; s++) mbar_init(&bars[s], 1);
        mbar_init_fence();
    }
    __syncthreads();
    uint32_t phase = 0;  // bit s: parity of stage s's next completion
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
        const int kb = PM == 0 ? k0 : s_n64, ke = PM == 0 ? s_n64 : s_ncut;
        if (kb >= ke) {
            __syncthreads();
            continue;  // nothing for this bra in this pass
        }
        const int ntile = (ke - kb + JT_TILE - 1) / JT_TILE;
        if (threadIdx.x == 0) {
            for (int s = 0; s < JT_STAGES && s < ntile; s++) {
                fence_proxy_async_smem();
                jt_issue<LC, LD>(ket, kb + s * JT_TILE, min(ke, kb + (s + 1) * JT_TILE),
                                 jt_smem + s * S::STAGE_DOUBLES, &bars[s]);
            }
        }
        double X[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) X[e] = 0.0;
        for (int t = 0; t < ntile; t++) {
            const int s = t & (JT_STAGES - 1);
            const bool ok = tma_wait(&bars[s], (phase >> s) & 1u);
            if (__syncthreads_or(!ok)) {
                // a copy did not land: flag it, wait (bounded) for this CTA's
                // copies still in flight (tiles t and t + 1), stop
                if (threadIdx.x == 0) {
                    atomicOr(errs, VLXB_KERR_TMA_TIMEOUT);
                    tma_wait(&bars[s], (phase >> s) & 1u);
                    if (t + 1 < ntile) tma_wait(&bars[s ^ 1], (phase >> (s ^ 1)) & 1u);
                }
                return;
            }
            phase ^= 1u << s;
            const int lo = kb + t * JT_TILE;
            const int kt = lo + threadIdx.x;
            if (kt < ke)
                j_quartet_staged<LA, LB, LC, LD, T>(b, qb, ket, kt,
                                                    jt_smem + s * S::STAGE_DOUBLES + (kt - (lo & ~1)), thr, tabs,
                                                    X);
            __syncthreads();  // every thread is done with stage s
            if (threadIdx.x == 0 && t + JT_STAGES < ntile) {
                fence_proxy_async_smem();
                jt_issue<LC, LD>(ket, kb + (t + JT_STAGES) * JT_TILE, min(ke, kb + (t + JT_STAGES + 1) * JT_TILE),
                                 jt_smem + s * S::STAGE_DOUBLES, &bars[s]);
            }
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

}  // namespace vlxb
