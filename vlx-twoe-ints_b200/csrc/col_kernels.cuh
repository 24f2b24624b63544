// Warp-cooperative ("column") J and K kernels for the heavy classes (sm_100a).
//
// A group of ColTab::NL lanes evaluates one primitive shell quartet: lane x
// holds the column [x|y]^(m) of its lane-side Cartesian component x in
// registers, and the step-side components y are built by identical steps on
// all lanes with one warp shuffle per step for the coupling term (see
// gen_column.py).  A warp holds ColTab::P such groups.
//
// Plan kinds ORI (gen_column.py): bit 0 the orientation (0: lanes = bra e,
// 1: lanes = ket f); 2, 3 packed plans (lanes for the target levels only,
// which start at d; two or five quartets per warp); 4, 5 packed plans whose
// lane-side pair is built on its second centre: PA -> PB = PA + AB and
// AB -> BA before the VRR (QC, CD likewise), the lane-side HRR gives (b a|
// and its result is read transposed.
// Exchange (orientation 0, lanes = bra e; orientation 1, lanes = ket f), per quartet:
//   VRR (column) -> lane-side HRR per lane into shared memory (ori 0: ket
//   HRR (e|cd); ori 1: bra HRR (ab|f)) -> __syncwarp -> each lane takes fixed
//   units of the other side (ori 0: cd pairs; ori 1: ab pairs), applies the
//   remaining HRR and digests into K partials held in registers for the whole
//   output block.  The block's partials are then reduced in a fixed order.
// Coulomb (ori 0): lanes accumulate X_e = sum_f (e0|f0) D''_f for their own e
//   across the bra's kets; the CTA reduces X in a fixed order and applies the
//   bra HRR once.  No atomics anywhere: results are bit-reproducible.
// Mixed precision as in jk_kernels.cuh: quartets below fp32_cut run the same
// column code in FP32 with FP64 accumulation.
#pragma once
#include "common.cuh"
#include "jk_kernels.cuh"

namespace vlxb {

template <int LA, int LB, int LC, int LD, int ORI>
struct ColTab;
template <int LA, int LB, int LC, int LD, int ORI>
__device__ __forceinline__ const int8_t* col_tab_ptr();

struct ColLane {
    int src[3];     // absolute lane owning x - 1_i (self when x_i == 0)
    double xi[3];   // components of x (coupling multipliers)
    int cdir[4];    // base-chain directions (-1: inactive step)
    double ck[4];   // base-chain coefficients
    int jdir[3];    // level-lam lanes: direction j with x - 1_i = 1_j (-1 otherwise)
    bool lamlane;   // lane of the lowest lane level when that level derives its partners
    int tidx;       // index of x among the lane-side targets, -1 if x is a helper
};

template <int LA, int LB, int LC, int LD, int ORI, typename T>
__device__ __forceinline__ void col_vrr(const QVT<T>& q, const T* F, const ColLane& ln, T* out);

template <int LA, int LB, int LC, int LD, int ORI>
__device__ __forceinline__ ColLane make_lane(int lig, int gbase)
{
    const int8_t* r = col_tab_ptr<LA, LB, LC, LD, ORI>() + lig * 20;
    ColLane ln;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        ln.xi[i] = (double)r[i];
        ln.src[i] = gbase + r[3 + i];
        ln.jdir[i] = r[6 + i];
    }
#pragma unroll
    for (int s = 0; s < 4; s++) {
        ln.cdir[s] = r[9 + s];
        ln.ck[s] = (double)r[13 + s];
    }
    ln.lamlane = (r[17] == ColTab<LA, LB, LC, LD, ORI>::LAM) && (r[6] >= 0 || r[7] >= 0 || r[8] >= 0);
    ln.tidx = r[18];
    return ln;
}

// ---------------------------------------------------------------- exchange
template <int LA, int LB, int LC, int LD, int ORI>
struct KColShape {
    using CT = ColTab<LA, LB, LC, LD, ORI>;
    static constexpr int O = ORI & 1;      // orientation
    static constexpr bool SW = ORI >= 4;   // lane-side pair built on its second centre
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NL = CT::NL, P = CT::P, NXT = CT::NXT, NYT = CT::NYT;
    // phase-2 units: orientation 0 -> cd pairs (accumulate K[a][c(u)]), 1 -> ab pairs (K[a(u)][c])
    static constexpr int N2 = O == 0 ? NC * ND : NA * NB;
    // row length of the shared lane-side HRR results: odd, so that lanes
    // storing one column of U hit distinct banks
    static constexpr int N2P = N2 | 1;
    static constexpr int NACC = O == 0 ? NA : NC;
    static constexpr int NPASS = (N2 + NL - 1) / NL;
    // U (lane-side HRR rows, per quartet) and red (the block's partials, after
    // its last quartet) share one shared-memory array
    static constexpr int U_DOUBLES = (K_THREADS / 32) * P * NXT * N2P;
    static constexpr int RED_DOUBLES = (K_THREADS / 32) * P * N2 * NACC;
    static constexpr int POOL_DOUBLES = U_DOUBLES > RED_DOUBLES ? U_DOUBLES : RED_DOUBLES;
    // position of (a, b) / (c, d) in the lane-side HRR result: (b a| / (d c| when swapped
    __device__ static constexpr int iab(int a, int b) { return SW && O == 0 ? b * NA + a : a * NB + b; }
    __device__ static constexpr int icd(int c, int d) { return SW && O == 1 ? d * NC + c : c * ND + d; }
};

// Second-centre plans: the lane-side pair's VRR starts from B (D) and its
// HRR runs from B to A (D to C).
template <int ORI, typename T>
__device__ __forceinline__ void swap_lane_centre(QVT<T>& q)
{
    if constexpr (ORI >= 4) {
        if constexpr ((ORI & 1) == 0) {
            q.PAx += q.ABx; q.PAy += q.ABy; q.PAz += q.ABz;
            q.ABx = -q.ABx; q.ABy = -q.ABy; q.ABz = -q.ABz;
        } else {
            q.QCx += q.CDx; q.QCy += q.CDy; q.QCz += q.CDz;
            q.CDx = -q.CDx; q.CDy = -q.CDy; q.CDz = -q.CDz;
        }
    }
}

template <int LA, int LB, int LC, int LD, int ORI, typename T>
__device__ __forceinline__ void kcol_quartet(bool act, int jr, int lr, const KPartnerRecs& ab,
                                             const KPartnerRecs& cd, const KDensity& dm, double omega,
                                             const BoysTabs& tabs, const ColLane& ln, bool lane_ok, int lig,
                                             double (*U)[KColShape<LA, LB, LC, LD, ORI>::N2P],
                                             double (*Kacc)[KColShape<LA, LB, LC, LD, ORI>::NACC])
{
    using S = KColShape<LA, LB, LC, LD, ORI>;
    constexpr int L = LA + LB + LC + LD;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND;
    constexpr int NL = S::NL, NXT = S::NXT, NYT = S::NYT, N2 = S::N2, NPASS = S::NPASS;
    const int spj = __ldg(ab.rec_sp + jr), spl = __ldg(cd.rec_sp + lr);
    const PairGeo bg = load_geo(ab.geo, ab.sp_stride, spj);
    const PairGeo kg = load_geo(cd.geo, cd.sp_stride, spl);
    QVT<T> q;
    T F[L + 1];
    make_quartet_t<L>(bg, kg, omega, tabs.f64, tabs.f32, q, F);
    swap_lane_centre<ORI>(q);
    T col[NYT];
    col_vrr<LA, LB, LC, LD, ORI, T>(q, F, ln, col);
    // phase 2a: this lane's HRR over the step side, into shared memory
    if (lane_ok && ln.tidx >= 0) {
        T h[N2];
        if (S::O == 0) hrr_bra_vector<LC, LD, T>(q.CDx, q.CDy, q.CDz, col, h);
        else hrr_bra_vector<LA, LB, T>(q.ABx, q.ABy, q.ABz, col, h);
#pragma unroll
        for (int u = 0; u < N2; u++) U[ln.tidx][u] = (double)h[u];
    }
    __syncwarp();
    // phase 2b: fixed units of the other side per lane
    if (act) {
        const int jsh = __ldg(ab.partner + spj), lsh = __ldg(cd.partner + spl);
        const uint64_t mj = __ldg(ab.rec_mask + jr), ml = __ldg(cd.rec_mask + lr);
        const double suj = __ldg(ab.su + jr), sul = __ldg(cd.su + lr);
        const bool uni = !isnan(suj) && !isnan(sul);
#pragma unroll
        for (int p = 0; p < NPASS; p++) {
            const int u = lig + NL * p;
            if (u < N2) {
                T v[NXT];
#pragma unroll
                for (int x = 0; x < NXT; x++) v[x] = (T)U[x][u];
                if (S::O == 0) {
                    // unit = (c, d): bra HRR, then K[a][c] += sum_b (ab|cd) Sij[ab] Skl[cd] D[b][d]
                    const int dd = u % ND;
                    T I[NA * NB];
                    if constexpr (S::SW) hrr_bra_vector<LB, LA, T>(q.ABx, q.ABy, q.ABz, v, I);
                    else hrr_bra_vector<LA, LB, T>(q.ABx, q.ABy, q.ABz, v, I);
                    const double skl =
                        uni ? sul : (((ml >> u) & 1ull) ? __ldg(cd.S + u * cd.sp_stride + spl) : 0.0);
                    const uint32_t lao = __ldg(dm.d_aoinds + lsh + (int64_t)dm.d_count * dd);
                    T wv[NB];
#pragma unroll
                    for (int b = 0; b < NB; b++) {
                        const uint32_t jao = __ldg(dm.b_aoinds + jsh + (int64_t)dm.b_count * b);
                        wv[b] = (T)((uni ? skl * suj : skl) * __ldg(dm.D + (int64_t)jao * dm.naos + lao));
                    }
                    if (uni) {
#pragma unroll
                        for (int a = 0; a < NA; a++) {
                            T s = (T)0;
#pragma unroll
                            for (int b = 0; b < NB; b++) s = fma(I[S::iab(a, b)], wv[b], s);
                            Kacc[p][a] += (double)s;
                        }
                    } else {
#pragma unroll
                        for (int a = 0; a < NA; a++) {
                            T s = (T)0;
#pragma unroll
                            for (int b = 0; b < NB; b++) {
                                const T sij = ((mj >> (a * NB + b)) & 1ull)
                                                  ? (T)__ldg(ab.S + (a * NB + b) * ab.sp_stride + spj) : (T)0;
                                s = fma(I[S::iab(a, b)] * sij, wv[b], s);
                            }
                            Kacc[p][a] += (double)s;
                        }
                    }
                } else {
                    // unit = (a, b): ket HRR, then K[a][c] += Sij[ab] sum_d (ab|cd) Skl[cd] D[b][d]
                    const int bb = u % NB;
                    T I[NC * ND];
                    if constexpr (S::SW) hrr_bra_vector<LD, LC, T>(q.CDx, q.CDy, q.CDz, v, I);
                    else hrr_bra_vector<LC, LD, T>(q.CDx, q.CDy, q.CDz, v, I);
                    const double sij =
                        uni ? suj : (((mj >> u) & 1ull) ? __ldg(ab.S + u * ab.sp_stride + spj) : 0.0);
                    const uint32_t jao = __ldg(dm.b_aoinds + jsh + (int64_t)dm.b_count * bb);
                    T wv[ND];
#pragma unroll
                    for (int d = 0; d < ND; d++) {
                        const uint32_t lao = __ldg(dm.d_aoinds + lsh + (int64_t)dm.d_count * d);
                        wv[d] = (T)((uni ? sij * sul : sij) * __ldg(dm.D + (int64_t)jao * dm.naos + lao));
                    }
                    if (uni) {
#pragma unroll
                        for (int c = 0; c < NC; c++) {
                            T s = (T)0;
#pragma unroll
                            for (int d = 0; d < ND; d++) s = fma(I[S::icd(c, d)], wv[d], s);
                            Kacc[p][c] += (double)s;
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < NC; c++) {
                            T s = (T)0;
#pragma unroll
                            for (int d = 0; d < ND; d++) {
                                const T skl = ((ml >> (c * ND + d)) & 1ull)
                                                  ? (T)__ldg(cd.S + (c * ND + d) * cd.sp_stride + spl) : (T)0;
                                s = fma(I[S::icd(c, d)] * skl, wv[d], s);
                            }
                            Kacc[p][c] += (double)s;
                        }
                    }
                }
            }
        }
    }
    __syncwarp();
}

template <int LA, int LB, int LC, int LD, int ORI, int PM>
__global__ void __launch_bounds__(K_THREADS)
exchange_col_kernel(KOutBlocks out, KPartnerRecs ab, KPartnerRecs cd, KDensity dm, double maxD, double omega,
                    double thr, double* __restrict__ mat_K, BoysTabs tabs, unsigned long long* __restrict__ qcount,
                    double fp32_cut, double fp32_budget)
{
    using S = KColShape<LA, LB, LC, LD, ORI>;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND;
    constexpr int NAC = NA * NC;
    constexpr int NW = K_THREADS / 32;
    constexpr int NL = S::NL, P = S::P, NXT = S::NXT;
    constexpr int N2 = S::N2, NACC = S::NACC, NPASS = S::NPASS;
    __shared__ double pool[S::POOL_DOUBLES];
    double(*U)[P][NXT][S::N2P] = reinterpret_cast<double(*)[P][NXT][S::N2P]>(pool);
    double(*red)[P][N2][NACC] = reinterpret_cast<double(*)[P][N2][NACC]>(pool);
    __shared__ int s_nl[K_JCHUNK], s_n64[K_JCHUNK], s_c64[K_JCHUNK + 1], s_c32[K_JCHUNK + 1];
    const KChunk ch{s_nl, s_n64, s_c64, s_c32};

    const int nout = *out.n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / NL, lig = lane % NL;
    const bool lane_ok = grp < P;
    const int gsel = lane_ok ? grp : 0;
    const ColLane ln = make_lane<LA, LB, LC, LD, ORI>(lane_ok ? lig : 0, lane_ok ? grp * NL : lane);

    for (int o = blockIdx.x; o < nout; o += gridDim.x) {
        const int ish = __ldg(out.ish + o), ksh = __ldg(out.ksh + o);
        const double mD = out.maxD ? __ldg(out.maxD + o) : maxD;
        const int a0 = __ldg(ab.seg + ish), a1 = __ldg(ab.seg + ish + 1);
        const int c0 = __ldg(cd.seg + ksh), c1 = __ldg(cd.seg + ksh + 1);
        double Kacc[NPASS][NACC];
#pragma unroll
        for (int p = 0; p < NPASS; p++)
#pragma unroll
            for (int x = 0; x < NACC; x++) Kacc[p][x] = 0.0;

        for (int jb = a0; jb < a1; jb += K_JCHUNK) {
            const int nj = min(K_JCHUNK, a1 - jb);
            k_chunk_scan(ab, cd, jb, nj, c0, c1, mD, thr, fp32_cut, ch, a1 - a0, fp32_budget);
            const int t64 = s_c64[nj], t32 = s_c32[nj];
            if (qcount && PM == 0 && threadIdx.x == 0) atomicAdd(qcount, (unsigned long long)(t64 + t32));
            const int n64 = PM == 0 ? (t64 + NW * P - 1) / (NW * P) : 0;
            for (int it = 0; it < n64; it++) {
                const int w = it * (NW * P) + warp * P + grp;
                const bool act = lane_ok && w < t64;
                const int wq = act ? w : 0;
                const int jj = k_find(s_c64, nj, wq);
                const int jr = jb + jj;
                const int lr = c0 + (wq - s_c64[jj]);
                kcol_quartet<LA, LB, LC, LD, ORI, double>(act, jr, act ? lr : c0, ab, cd, dm, omega, tabs, ln,
                                                          lane_ok, lig, U[warp][gsel], Kacc);
            }
            const int n32 = PM == 1 ? (t32 + NW * P - 1) / (NW * P) : 0;
            for (int it = 0; it < n32; it++) {
                const int w = it * (NW * P) + warp * P + grp;
                const bool act = lane_ok && w < t32;
                const int wq = act ? w : 0;
                const int jj = k_find(s_c32, nj, wq);
                const int jr = jb + jj;
                const int lr = c0 + s_n64[jj] + (wq - s_c32[jj]);
                kcol_quartet<LA, LB, LC, LD, ORI, float>(act, jr, act ? lr : c0, ab, cd, dm, omega, tabs, ln,
                                                         lane_ok, lig, U[warp][gsel], Kacc);
            }
            __syncthreads();
        }

        // fixed-order reduction of the block's partials
        if (lane_ok) {
#pragma unroll
            for (int p = 0; p < NPASS; p++)
                if (lig + NL * p < N2)
#pragma unroll
                    for (int x = 0; x < NACC; x++) red[warp][grp][lig + NL * p][x] = Kacc[p][x];
        }
        __syncthreads();
        if (threadIdx.x < NAC) {
            const int a = threadIdx.x / NC, c = threadIdx.x % NC;
            double s = 0.0;
            for (int w = 0; w < NW; w++)
                for (int g = 0; g < P; g++) {
                    if (S::O == 0) {
                        for (int d = 0; d < ND; d++) s += red[w][g][c * ND + d][a];
                    } else {
                        for (int b = 0; b < NB; b++) s += red[w][g][a * NB + b][c];
                    }
                }
            const int32_t pos = __ldg(out.idx + threadIdx.x * out.stride + o);
            if (pos >= 0) mat_K[pos] += s;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- contracted exchange
// The partner records of one first primitive shell whose partners belong to
// one contracted shell (same centre, same AO indices) form a group.  For a
// pair of groups (J of i, L of k) every member pair that passes the
// reference's screen |q_j q_l max_D| > thr (gen_exchange.py:229-232) is run
// through the VRR and its columns are summed with the weight S_ij S_kl; the
// two HRRs and the density digestion then run once per group pair instead of
// once per primitive quartet (Head-Gordon-Pople: the HRR coefficients AB, CD
// do not depend on the exponents).  A record whose components do not share
// one S is a group of its own and is digested with its per-component S.
template <int LA, int LB, int LC, int LD, int ORI, typename T>
__device__ __forceinline__ void col_vrr_acc(const QVT<T>& q, const T* F, const ColLane& ln, T* out, T w);

struct KGroups {
    const int* seg;          // [n_first + 1] group offsets by first primitive shell
    const double* q;         // max member q, descending inside a segment
    const int32_t* beg;      // first member
    const int32_t* cnt;      // member count
    const int32_t* msp;      // member shell pair
    const double* mq;        // member q
    const double* msu;       // member uniform S, or NaN (member alone in its group)
    const uint64_t* mmask;   // member component mask
    const double* qa;        // sum over members of |q| times HRR growth (FP32 error budget), or null
    const double* qpre;      // inclusive prefix sum of qa, or null
};

template <int LA, int LB, int LC, int LD, int ORI, typename T>
__device__ __forceinline__ int kcolc_group(bool act, int jg, int lg, const KPartnerRecs& ab, const KPartnerRecs& cd,
                                           const KGroups& gab, const KGroups& gcd, const KDensity& dm, double maxD,
                                           double thr, double omega, const BoysTabs& tabs, const ColLane& ln,
                                           bool lane_ok, int lig,
                                           double (*U)[KColShape<LA, LB, LC, LD, ORI>::N2P],
                                           double (*Kacc)[KColShape<LA, LB, LC, LD, ORI>::NACC])
{
    using S = KColShape<LA, LB, LC, LD, ORI>;
    constexpr int L = LA + LB + LC + LD;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND;
    constexpr int NL = S::NL, NXT = S::NXT, NYT = S::NYT, N2 = S::N2, NPASS = S::NPASS;
    const int jb = act ? __ldg(gab.beg + jg) : 0, nj = act ? __ldg(gab.cnt + jg) : 0;
    const int lb = act ? __ldg(gcd.beg + lg) : 0, nl = act ? __ldg(gcd.cnt + lg) : 0;
    const int npair = nj * nl;
    // every lane of the warp runs the VRR of each step (the coupling shuffles
    // need all of them): loop to the largest member-pair count of the warp
    int nmax = npair;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
    // a uniform side has its S folded into the sum; a non-uniform side is a
    // single member whose per-component S is applied in the digestion
    const bool uj = !act || !isnan(__ldg(gab.msu + jb)), ul = !act || !isnan(__ldg(gcd.msu + lb));
    T acc[NYT];
#pragma unroll
    for (int y = 0; y < NYT; y++) acc[y] = (T)0;
    int npass = 0;
    for (int t = 0; t < nmax; t++) {
        const bool valid = t < npair;
        const int mj = jb + (valid ? t / nl : 0), ml = lb + (valid ? t % nl : 0);
        const double qj = __ldg(gab.mq + mj), ql = __ldg(gcd.mq + ml);
        const bool pass = valid && fabs(qj * ql * maxD) > thr;
        npass += pass ? 1 : 0;
        double w = 0.0;
        if (pass) w = (uj ? __ldg(gab.msu + mj) : 1.0) * (ul ? __ldg(gcd.msu + ml) : 1.0);
        const int spj = __ldg(gab.msp + mj), spl = __ldg(gcd.msp + ml);
        const PairGeo bg = load_geo(ab.geo, ab.sp_stride, spj);
        const PairGeo kg = load_geo(cd.geo, cd.sp_stride, spl);
        QVT<T> q;
        T F[L + 1];
        make_quartet_t<L>(bg, kg, omega, tabs.f64, tabs.f32, q, F);
        swap_lane_centre<ORI>(q);
        col_vrr_acc<LA, LB, LC, LD, ORI, T>(q, F, ln, acc, (T)w);
    }
    // HRRs and digestion once for the group pair; AB and CD from the first members
    const int spj = __ldg(gab.msp + jb), spl = __ldg(gcd.msp + lb);
    const T ABx = (T)__ldg(ab.geo + G_RX * ab.sp_stride + spj), ABy = (T)__ldg(ab.geo + G_RY * ab.sp_stride + spj),
            ABz = (T)__ldg(ab.geo + G_RZ * ab.sp_stride + spj);
    const T CDx = (T)__ldg(cd.geo + G_RX * cd.sp_stride + spl), CDy = (T)__ldg(cd.geo + G_RY * cd.sp_stride + spl),
            CDz = (T)__ldg(cd.geo + G_RZ * cd.sp_stride + spl);
    if (lane_ok && ln.tidx >= 0) {
        T h[N2];
        if (S::O == 0) hrr_bra_vector<LC, LD, T>(CDx, CDy, CDz, acc, h);
        else hrr_bra_vector<LA, LB, T>(ABx, ABy, ABz, acc, h);
#pragma unroll
        for (int u = 0; u < N2; u++) U[ln.tidx][u] = (double)h[u];
    }
    __syncwarp();
    if (act && npass > 0) {
        const int jsh = __ldg(ab.partner + spj), lsh = __ldg(cd.partner + spl);
        const uint64_t mjm = __ldg(gab.mmask + jb), mlm = __ldg(gcd.mmask + lb);
#pragma unroll
        for (int p = 0; p < NPASS; p++) {
            const int u = lig + NL * p;
            if (u < N2) {
                T v[NXT];
#pragma unroll
                for (int x = 0; x < NXT; x++) v[x] = (T)U[x][u];
                if (S::O == 0) {
                    // unit = (c, d): bra HRR, then K[a][c] += sum_b (ab|cd) [Sij Skl] D[b][d]
                    const int dd = u % ND;
                    T I[NA * NB];
                    if constexpr (S::SW) hrr_bra_vector<LB, LA, T>(-ABx, -ABy, -ABz, v, I);
                    else hrr_bra_vector<LA, LB, T>(ABx, ABy, ABz, v, I);
                    const double skl = ul ? 1.0 : (((mlm >> u) & 1ull) ? __ldg(cd.S + u * cd.sp_stride + spl) : 0.0);
                    const uint32_t lao = __ldg(dm.d_aoinds + lsh + (int64_t)dm.d_count * dd);
                    T wv[NB];
#pragma unroll
                    for (int bq = 0; bq < NB; bq++) {
                        const uint32_t jao = __ldg(dm.b_aoinds + jsh + (int64_t)dm.b_count * bq);
                        wv[bq] = (T)(skl * __ldg(dm.D + (int64_t)jao * dm.naos + lao));
                    }
#pragma unroll
                    for (int a = 0; a < NA; a++) {
                        T sacc = (T)0;
#pragma unroll
                        for (int bq = 0; bq < NB; bq++) {
                            const T sij = uj ? (T)1 : (((mjm >> (a * NB + bq)) & 1ull)
                                                            ? (T)__ldg(ab.S + (a * NB + bq) * ab.sp_stride + spj)
                                                            : (T)0);
                            sacc = fma(I[S::iab(a, bq)] * sij, wv[bq], sacc);
                        }
                        Kacc[p][a] += (double)sacc;
                    }
                } else {
                    // unit = (a, b): ket HRR, then K[a][c] += [Sij] sum_d (ab|cd) [Skl] D[b][d]
                    const int bb = u % NB;
                    T I[NC * ND];
                    if constexpr (S::SW) hrr_bra_vector<LD, LC, T>(-CDx, -CDy, -CDz, v, I);
                    else hrr_bra_vector<LC, LD, T>(CDx, CDy, CDz, v, I);
                    const double sij = uj ? 1.0 : (((mjm >> u) & 1ull) ? __ldg(ab.S + u * ab.sp_stride + spj) : 0.0);
                    const uint32_t jao = __ldg(dm.b_aoinds + jsh + (int64_t)dm.b_count * bb);
                    T wv[ND];
#pragma unroll
                    for (int d = 0; d < ND; d++) {
                        const uint32_t lao = __ldg(dm.d_aoinds + lsh + (int64_t)dm.d_count * d);
                        wv[d] = (T)(sij * __ldg(dm.D + (int64_t)jao * dm.naos + lao));
                    }
#pragma unroll
                    for (int c = 0; c < NC; c++) {
                        T sacc = (T)0;
#pragma unroll
                        for (int d = 0; d < ND; d++) {
                            const T skl = ul ? (T)1 : (((mlm >> (c * ND + d)) & 1ull)
                                                           ? (T)__ldg(cd.S + (c * ND + d) * cd.sp_stride + spl)
                                                           : (T)0);
                            sacc = fma(I[S::icd(c, d)] * skl, wv[d], sacc);
                        }
                        Kacc[p][c] += (double)sacc;
                    }
                }
            }
        }
    }
    __syncwarp();
    return npass;
}

// Contracted-partner exchange kernel: exchange_col_kernel's output blocks and
// flattened partner enumeration, over partner groups instead of records (the
// screen on group maxima selects a superset; kcolc_group applies the exact
// per-member screen).  PM as for coulomb_kernel, split on the group maxima.
// Registers are capped for 3 CTAs per SM (168) for the plain plans: the
// heaviest classes spill a little; a 2-CTA cap (no spills, fewer warps)
// measured no faster.  The packed plans (two or five quartets per warp, the
// tower in registers) get the 2-CTA cap.
template <int LA, int LB, int LC, int LD, int ORI, int PM>
__global__ void __launch_bounds__(K_THREADS, ORI >= 2 ? 2 : 3)
exchange_colc_kernel(KOutBlocks out, KPartnerRecs ab, KPartnerRecs cd, KGroups gab, KGroups gcd, KDensity dm,
                     double maxD, double omega, double thr, double* __restrict__ mat_K, BoysTabs tabs,
                     unsigned long long* __restrict__ qcount, double fp32_cut, double fp32_budget)
{
    using S = KColShape<LA, LB, LC, LD, ORI>;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND;
    constexpr int NAC = NA * NC;
    constexpr int NW = K_THREADS / 32;
    constexpr int NL = S::NL, P = S::P, NXT = S::NXT;
    constexpr int N2 = S::N2, NACC = S::NACC, NPASS = S::NPASS;
    __shared__ double pool[S::POOL_DOUBLES];
    double(*U)[P][NXT][S::N2P] = reinterpret_cast<double(*)[P][NXT][S::N2P]>(pool);
    double(*red)[P][N2][NACC] = reinterpret_cast<double(*)[P][N2][NACC]>(pool);
    __shared__ int s_nl[K_JCHUNK], s_n64[K_JCHUNK], s_c64[K_JCHUNK + 1], s_c32[K_JCHUNK + 1];
    const KChunk ch{s_nl, s_n64, s_c64, s_c32};

    const int nout = *out.n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / NL, lig = lane % NL;
    const bool lane_ok = grp < P;
    const int gsel = lane_ok ? grp : 0;
    const ColLane ln = make_lane<LA, LB, LC, LD, ORI>(lane_ok ? lig : 0, lane_ok ? grp * NL : lane);
    unsigned long long nq = 0;

    for (int o = blockIdx.x; o < nout; o += gridDim.x) {
        const int ish = __ldg(out.ish + o), ksh = __ldg(out.ksh + o);
        const double mD = out.maxD ? __ldg(out.maxD + o) : maxD;
        const int a0 = __ldg(gab.seg + ish), a1 = __ldg(gab.seg + ish + 1);
        const int c0 = __ldg(gcd.seg + ksh), c1 = __ldg(gcd.seg + ksh + 1);
        double Kacc[NPASS][NACC];
#pragma unroll
        for (int p = 0; p < NPASS; p++)
#pragma unroll
            for (int x = 0; x < NACC; x++) Kacc[p][x] = 0.0;

        for (int jb = a0; jb < a1; jb += K_JCHUNK) {
            const int nj = min(K_JCHUNK, a1 - jb);
            k_chunk_scan(gab.q, gcd.q, jb, nj, c0, c1, mD, thr, fp32_cut, ch, gab.qa, gcd.qpre, a1 - a0,
                         fp32_budget);
            const int t64 = s_c64[nj], t32 = s_c32[nj];
            const int n64 = PM == 0 ? (t64 + NW * P - 1) / (NW * P) : 0;
            for (int it = 0; it < n64; it++) {
                const int w = it * (NW * P) + warp * P + grp;
                const bool act = lane_ok && w < t64;
                const int wq = act ? w : 0;
                const int jj = k_find(s_c64, nj, wq);
                const int np = kcolc_group<LA, LB, LC, LD, ORI, double>(
                    act, jb + jj, c0 + (wq - s_c64[jj]), ab, cd, gab, gcd, dm, mD, thr, omega, tabs, ln, lane_ok,
                    lig, U[warp][gsel], Kacc);
                if (act && lig == 0) nq += (unsigned long long)np;
            }
            const int n32 = PM == 1 ? (t32 + NW * P - 1) / (NW * P) : 0;
            for (int it = 0; it < n32; it++) {
                const int w = it * (NW * P) + warp * P + grp;
                const bool act = lane_ok && w < t32;
                const int wq = act ? w : 0;
                const int jj = k_find(s_c32, nj, wq);
                const int np = kcolc_group<LA, LB, LC, LD, ORI, float>(
                    act, jb + jj, c0 + s_n64[jj] + (wq - s_c32[jj]), ab, cd, gab, gcd, dm, mD, thr, omega, tabs,
                    ln, lane_ok, lig, U[warp][gsel], Kacc);
                if (act && lig == 0) nq += (unsigned long long)np;
            }
            __syncthreads();
        }

        // fixed-order reduction of the block's partials
        if (lane_ok) {
#pragma unroll
            for (int p = 0; p < NPASS; p++)
                if (lig + NL * p < N2)
#pragma unroll
                    for (int x = 0; x < NACC; x++) red[warp][grp][lig + NL * p][x] = Kacc[p][x];
        }
        __syncthreads();
        if (threadIdx.x < NAC) {
            const int a = threadIdx.x / NC, c = threadIdx.x % NC;
            double sum = 0.0;
            for (int w = 0; w < NW; w++)
                for (int g = 0; g < P; g++) {
                    if (S::O == 0) {
                        for (int d = 0; d < ND; d++) sum += red[w][g][c * ND + d][a];
                    } else {
                        for (int b = 0; b < NB; b++) sum += red[w][g][a * NB + b][c];
                    }
                }
            const int32_t pos = __ldg(out.idx + threadIdx.x * out.stride + o);
            if (pos >= 0) mat_K[pos] += sum;
        }
        __syncthreads();
    }
    if (qcount && nq) atomicAdd(qcount, nq);
}

// ---------------------------------------------------------------- coulomb
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void jcol_quartet(bool act, const PairGeo& b, double qb, const JKetPairs& ket, int kt,
                                             double thr, const BoysTabs& tabs, const ColLane& ln, bool lane_ok,
                                             double& X)
{
    constexpr int L = LA + LB + LC + LD;
    constexpr int NF = nrange(LC, LD);
    const PairGeo k = load_geo(ket.geo, ket.stride, kt);
    QVT<T> q;
    T F[L + 1];
    make_quartet_t<L>(b, k, 0.0, tabs.f64, tabs.f32, q, F);
    T col[NF];
    col_vrr<LA, LB, LC, LD, 0, T>(q, F, ln, col);
    if (act && lane_ok && ln.tidx >= 0) {
        T Dpp[NF];
        ket_density<LC, LD, T>(ket, kt, qb, thr, k, Dpp);
        T s = (T)0;
#pragma unroll
        for (int f = 0; f < NF; f++) s = fma(col[f], Dpp[f], s);
        X += (double)s;
    }
}

template <int LA, int LB, int LC, int LD, int PM>
__global__ void __launch_bounds__(J_THREADS)
coulomb_col_kernel(JBraRecs bra, JKetPairs ket, double* __restrict__ mat_J, double thr, BoysTabs tabs,
                   unsigned long long* __restrict__ qcount, double fp32_cut, double fp32_budget)
{
    using CT = ColTab<LA, LB, LC, LD, 0>;
    constexpr int NE = nrange(LA, LB), NF = nrange(LC, LD);
    constexpr int NAB = ncart(LA) * ncart(LB);
    constexpr int NW = J_THREADS / 32;
    constexpr int NL = CT::NL, P = CT::P;
    static_assert(CT::NXT == NE && CT::NYT == NF, "column layout");
    __shared__ double red[NW][P][NE];
    __shared__ int s_ncut, s_n64;
    const int nbra = *bra.n_rec;
    const int nket = *ket.n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / NL, lig = lane % NL;
    const bool lane_ok = grp < P;
    const ColLane ln = make_lane<LA, LB, LC, LD, 0>(lane_ok ? lig : 0, lane_ok ? grp * NL : lane);

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
        double X = 0.0;
        const int it64 = PM == 0 ? (n64 - k0 + NW * P - 1) / (NW * P) : 0;
        for (int it = 0; it < it64; it++) {
            const int kt0 = k0 + it * (NW * P) + warp * P + grp;
            const bool act = lane_ok && kt0 < n64;
            jcol_quartet<LA, LB, LC, LD, double>(act, b, qb, ket, act ? kt0 : 0, thr, tabs, ln, lane_ok, X);
        }
        const int n32 = ncut - n64;
        const int it32 = PM == 1 ? (n32 + NW * P - 1) / (NW * P) : 0;
        for (int it = 0; it < it32; it++) {
            const int kt0 = n64 + it * (NW * P) + warp * P + grp;
            const bool act = lane_ok && kt0 < ncut;
            jcol_quartet<LA, LB, LC, LD, float>(act, b, qb, ket, act ? kt0 : 0, thr, tabs, ln, lane_ok, X);
        }
        if (lane_ok && ln.tidx >= 0) red[warp][grp][ln.tidx] = X;
        __syncthreads();
        if (threadIdx.x == 0) {
            double Xs[NE];
#pragma unroll
            for (int e = 0; e < NE; e++) {
                double s = 0.0;
                for (int w = 0; w < NW; w++)
                    for (int g = 0; g < P; g++) s += red[w][g][e];
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
