// Exchange nuclear gradient kernel (McMurchie-Davidson form).
//
// E_K = 1/2 Tr[D K] = 1/2 sum_{ijkl} D_ik D_jl (ij|kl) over all primitive
// Cartesian indices.  The sum is unchanged by (i <-> j, k <-> l) and by
// (ij) <-> (kl), so the derivatives on the centres of j and l equal those on
// i and k, and over the caller's (i, k) list (gen_exchange.py:139-342: i of
// type a, k of type c, i <= k for a == c)
//   dE_K/dR = sum_{(i,k) in list} w_ik D_ik sum_{jl} D_jl (d/dA + d/dC)(ij|kl),
// w_ik = 1 for i == k of a same-type list, else 2, d/dA acting on i's centre
// (credited to i's atom), d/dC on k's (credited to k's atom).  A Cartesian
// Gaussian differentiates as d/dA_x phi_a = 2 alpha phi_{a+1x} - a_x phi_{a-1x}
// (Obara-Saika 1986, Eq. 5; the reference generator's gradient='a' / 'c'
// terms, eri.py:85-152).
//
// In Hermite form (md.cuh) (ab|cd) = sum_{e,f} E^{ab}_e Et^{cd}_f R_{e+f},
// Et = (-1)^{|f|} E, and d/dA turns E^{ab} into
// E'^{ab,x} = 2 alpha E^{a+1x,b} - a_x E^{a-1x,b} (d/dC the same on Et^{cd}).
// With Gam_abcd = Dw_ac D_bd S_ab S_cd (Dw_ac = w_ik D_ik) one quartet gives
//   A side, per b:  Y_{cf}  = sum_d D_bd S_cd Et^{cd}_f
//                   T_{af}  = S_ab sum_c Dw_ac Y_{cf}
//                   gA_x   += sum_{a,e} E'^{ab,x}_e sum_f R_{e+f} T_{af}
//   C side, per d:  Y2_{ae} = sum_b D_bd S_ab E^{ab}_e
//                   T2_{ce} = S_cd sum_a Dw_ac Y2_{ae}
//                   gC_x   += sum_{c,f} Et'^{cd,x}_f sum_e R_{e+f} T2_{ce}
// with R up to level L + 1.  The factorisation keeps every step a small
// dense loop, so one generic kernel serves all 54 classes (runtime loops over
// shared-memory tables; no straight-line derivative-class code, whose d-rich
// instances do not compile in reasonable time).
//
// Layout follows the exchange kernels: one CTA per (i, k) primitive shell
// block, its partner-pair quartets spread over groups of SG lanes (SG = 1 ..
// 32 by class size: one quartet per lane for the smallest classes, one per
// warp for the largest), the group's lanes over the items of each step, six
// accumulators per lane, fixed-order reduction, no atomics on the output.
// Screening is the K kernels' (|Q_ij Q_kl max_D| > thr), FP64.
// Output: the block's six values are added at the block's lowest (i, k) list
// position p, grad[x * gstride + p] (x = 0..2: i's centre, 3..5: k's); the
// block's other positions receive nothing (all of them share the two atoms).
#pragma once
#include "jk_kernels.cuh"
#include "md.cuh"

namespace vlxb {

// D_ik per (i, k) block: rows / columns of the (i, k) components in the AO
// density (single-molecule calls).
struct KGradBlockD {
    const uint32_t* a_aoinds;
    uint32_t a_count;
    const uint32_t* c_aoinds;
    uint32_t c_count;
    int same_type;  // a == c: the diagonal entries i == k have weight 1
};

template <int LA, int LB, int LC, int LD>
struct KGradShape {
    static constexpr int L = LA + LB + LC + LD;
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NHB = nherm(LA + LB), NHBP = nherm(LA + LB + 1);
    static constexpr int NHK = nherm(LC + LD), NHKP = nherm(LC + LD + 1);
    static constexpr int NHL = nherm(L + 1);
    static constexpr int EB = (LA + 2) * (LB + 1) * (LA + LB + 2);  // herm_e1<LA + 1, LB> per direction
    static constexpr int EK = (LC + 2) * (LD + 1) * (LC + LD + 2);  // herm_e1<LC + 1, LD>
    static constexpr int NY = (NC * NHK > NA * NHB) ? NC * NHK : NA * NHB;
    static constexpr int NT = (NA * NHK > NC * NHB) ? NA * NHK : NC * NHB;
    // lanes per quartet: a power of two near a quarter of the widest step
    // (the Y / T items and the Hermite indices of the R contractions), so that
    // small classes run many quartets per warp (down to one per lane) and
    // large ones a warp each
    static constexpr int cmax(int x, int y) { return x > y ? x : y; }
    static constexpr int WIDE = cmax(cmax(cmax(NC * NHK, NA * NHK), cmax(NA * NHB, NC * NHB)), cmax(NHBP, NHKP));
    static constexpr int SG = WIDE <= 4 ? 1 : WIDE <= 8 ? 2 : WIDE <= 16 ? 4 : WIDE <= 32 ? 8 : WIDE <= 64 ? 16 : 32;
    static constexpr int NG = 32 / SG;  // quartet groups per warp
    // doubles per group: R (two level buffers), R^{(n)}_{000}, E tables, D_bd, S_ab, S_cd, Y, T
    static constexpr int PER_GROUP = 2 * NHL + (L + 2) + 3 * EB + 3 * EK + NB * ND + NA * NB + NC * ND + NY + NT;
    static constexpr int FIXED_BYTES = NHKP * NHBP * 2 + NHL * 8 + NA * NC * 8 + 4 * (K_JCHUNK + 1) * 4 + 512;
    static constexpr int NW = (4 * NG * PER_GROUP * 8 + FIXED_BYTES <= 46 * 1024)   ? 4
                              : (2 * NG * PER_GROUP * 8 + FIXED_BYTES <= 46 * 1024) ? 2
                                                                                    : 1;
    static constexpr int THREADS = NW * 32;
};

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(KGradShape<LA, LB, LC, LD>::THREADS)
exchange_grad_kernel(KOutBlocks out, KPartnerRecs ab, KPartnerRecs cd, KDensity dm, KGradBlockD bd, double maxD,
                     double omega, double thr, double* __restrict__ grad, int64_t gstride, BoysTabs tabs)
{
    using S = KGradShape<LA, LB, LC, LD>;
    constexpr int L1 = S::L + 1;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND;
    constexpr int NHB = S::NHB, NHBP = S::NHBP, NHK = S::NHK, NHKP = S::NHKP, NHL = S::NHL;
    constexpr int NW = S::NW, NT_ = S::THREADS, SG = S::SG, NG = S::NG;
    constexpr int LSB = LA + LB + 2, LSK = LC + LD + 2;  // t extents of the E tables
    __shared__ int s_nl[K_JCHUNK], s_n64[K_JCHUNK], s_c64[K_JCHUNK + 1], s_c32[K_JCHUNK + 1];
    __shared__ int16_t sIdx[NHKP][NHBP];  // index of R_{e+f}, -1 above level L + 1
    __shared__ uint32_t sTuv[NHL];
    __shared__ uint32_t sRec[NHL];  // R recurrence per entry (as coulomb_md_kernel)
    __shared__ uint32_t sCart[4][10];  // exponents of component c of shell l: x | y << 4 | z << 8
    __shared__ double sDw[NA * NC];
    __shared__ double red[NW][6];
    __shared__ int s_pmin;
    __shared__ double sw[NW * NG][S::PER_GROUP];
    const KChunk ch{s_nl, s_n64, s_c64, s_c32};

    for (int i = threadIdx.x; i < 40; i += NT_) {
        const int l = i / 10, c = i % 10;
        sCart[l][c] = c < ncart(l) ? (uint32_t)cart_x(l, c) | ((uint32_t)cart_y(l, c) << 4) |
                                         ((uint32_t)cart_z(l, c) << 8)
                                   : 0u;
    }
    for (int i = threadIdx.x; i < NHL; i += NT_) {
        int n = 0;
        while (nherm(n) <= i) n++;
        const int r = i - (n > 0 ? nherm(n - 1) : 0);
        int s = 0;
        while ((s + 1) * (s + 2) / 2 <= r) s++;
        const int v = r - s * (s + 1) / 2, u = s - v, t = n - s;
        sTuv[i] = (uint32_t)t | ((uint32_t)u << 8) | ((uint32_t)v << 16);
        uint32_t rec = 1023u << 10;
        if (t > 0)
            rec = herm_idx(t - 1, u, v) | ((t > 1 ? herm_idx(t - 2, u, v) : 1023u) << 10) | ((uint32_t)(t - 1) << 20);
        else if (u > 0)
            rec = herm_idx(0, u - 1, v) | ((u > 1 ? herm_idx(0, u - 2, v) : 1023u) << 10) |
                  ((uint32_t)(u - 1) << 20) | (1u << 28);
        else if (v > 0)
            rec = herm_idx(0, 0, v - 1) | ((v > 1 ? herm_idx(0, 0, v - 2) : 1023u) << 10) |
                  ((uint32_t)(v - 1) << 20) | (2u << 28);
        sRec[i] = rec;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NHKP * NHBP; i += NT_) {
        const int f = i / NHBP, e = i % NHBP;
        const uint32_t a = sTuv[e], b = sTuv[f];
        const int t = (a & 255) + (b & 255), u = ((a >> 8) & 255) + ((b >> 8) & 255), v = (a >> 16) + (b >> 16);
        sIdx[f][e] = (int16_t)(t + u + v <= L1 ? herm_idx(t, u, v) : -1);
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / SG, sub = lane % SG;  // quartet group in the warp, lane in the group
    double* W = sw[warp * NG + grp];
    double* R0 = W;
    double* R1 = R0 + NHL;
    double* Rb = R1 + NHL;        // [L1 + 1] R^{(n)}_{000}
    double* Eb = Rb + (L1 + 1);   // [3][EB]
    double* Ek = Eb + 3 * S::EB;  // [3][EK]
    double* Dbd = Ek + 3 * S::EK;
    double* Sab = Dbd + NB * ND;
    double* Scd = Sab + NA * NB;
    double* Y = Scd + NC * ND;
    double* T = Y + S::NY;
    const int nout = *out.n;

    for (int o = blockIdx.x; o < nout; o += gridDim.x) {
        const int ish = __ldg(out.ish + o), ksh = __ldg(out.ksh + o);
        if (threadIdx.x == 0) s_pmin = INT32_MAX;
        __syncthreads();
        if (threadIdx.x < NA * NC) {
            const int ca = threadIdx.x / NC, cc = threadIdx.x % NC;
            const int32_t p = __ldg(out.idx + threadIdx.x * out.stride + o);
            double w = 0.0;
            if (p >= 0) {
                const uint32_t iao = __ldg(bd.a_aoinds + ish + (int64_t)bd.a_count * ca);
                const uint32_t kao = __ldg(bd.c_aoinds + ksh + (int64_t)bd.c_count * cc);
                const bool diag = bd.same_type && ish == ksh && ca == cc;
                w = (diag ? 1.0 : 2.0) * __ldg(dm.D + (int64_t)iao * dm.naos + kao);
                atomicMin(&s_pmin, (int)p);
            }
            sDw[threadIdx.x] = w;
        }
        __syncthreads();
        const int a0 = __ldg(ab.seg + ish), a1 = __ldg(ab.seg + ish + 1);
        const int c0 = __ldg(cd.seg + ksh), c1 = __ldg(cd.seg + ksh + 1);
        double g[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int jb = a0; jb < a1; jb += K_JCHUNK) {
            const int nj = min(K_JCHUNK, a1 - jb);
            k_chunk_scan(ab, cd, jb, nj, c0, c1, maxD, thr, 0.0, ch);
            const int nq = s_c64[nj];
            // every group of a warp walks the same number of slots, so the
            // warp-wide __syncwarp() calls below stay uniform; a group without a
            // quartet in its slot skips the work
            for (int base = warp * NG; base < nq; base += NW * NG) {
                const int w = base + grp;
                const bool valid = w < nq;
                const int jj = valid ? k_find(s_c64, nj, w) : 0;
                const int jr = jb + jj, lr = valid ? c0 + (w - s_c64[jj]) : c0;
                const int spj = valid ? __ldg(ab.rec_sp + jr) : 0, spl = valid ? __ldg(cd.rec_sp + lr) : 0;
                PairGeo bg{}, kg{};
                double al2 = 0.0, ga2 = 0.0;
                if (valid) {
                    bg = load_geo(ab.geo, ab.sp_stride, spj);
                    kg = load_geo(cd.geo, cd.sp_stride, spl);
                    al2 = 2.0 * __ldg(ab.geo + G_ALPHA * ab.sp_stride + spj);
                    ga2 = 2.0 * __ldg(cd.geo + G_ALPHA * cd.sp_stride + spl);
                    // per-quartet factors: D_bd, S_ab, S_cd, 1-D Hermite tables
                    const int jsh = __ldg(ab.partner + spj), lsh = __ldg(cd.partner + spl);
                    for (int t = sub; t < NB * ND; t += SG) {
                        const int cb = t / ND, cdd = t % ND;
                        const uint32_t jao = __ldg(dm.b_aoinds + jsh + (int64_t)dm.b_count * cb);
                        const uint32_t lao = __ldg(dm.d_aoinds + lsh + (int64_t)dm.d_count * cdd);
                        Dbd[t] = __ldg(dm.D + (int64_t)jao * dm.naos + lao);
                    }
                    const double suj = __ldg(ab.su + jr), sul = __ldg(cd.su + lr);
                    const uint64_t mj = __ldg(ab.rec_mask + jr), ml = __ldg(cd.rec_mask + lr);
                    for (int t = sub; t < NA * NB; t += SG)
                        Sab[t] = !isnan(suj) ? suj : (((mj >> t) & 1ull) ? __ldg(ab.S + t * ab.sp_stride + spj) : 0.0);
                    for (int t = sub; t < NC * ND; t += SG)
                        Scd[t] = !isnan(sul) ? sul : (((ml >> t) & 1ull) ? __ldg(cd.S + t * cd.sp_stride + spl) : 0.0);
                    for (int x = sub; x < 6; x += SG) {
                        if (x < 3) {
                            const double pa = x == 0 ? bg.Ax : (x == 1 ? bg.Ay : bg.Az);
                            const double abv = x == 0 ? bg.Rx : (x == 1 ? bg.Ry : bg.Rz);
                            herm_e1_flat<LA + 1, LB>(pa, pa + abv, bg.i2z, Eb + x * S::EB);
                        } else {
                            const double qc = x == 3 ? kg.Ax : (x == 4 ? kg.Ay : kg.Az);
                            const double cdv = x == 3 ? kg.Rx : (x == 4 ? kg.Ry : kg.Rz);
                            herm_e1_flat<LC + 1, LD>(qc, qc + cdv, kg.i2z, Ek + (x - 3) * S::EK);
                        }
                    }
                }
                // R^{(n)}_{000} = 2 sqrt(rho'/pi) (-2 rho')^n F_n(rho' |PQ|^2), rho' = rho d2
                // (d2 = 1, or w^2 / (rho + w^2) for the attenuated operator), then levels
                const double PQx = bg.Px - kg.Px, PQy = bg.Py - kg.Py, PQz = bg.Pz - kg.Pz;
                if (valid && sub == 0) {
                    const double inv = 1.0 / (bg.z + kg.z);
                    const double rho = bg.z * kg.z * inv;
                    const double d2 = omega != 0.0 ? omega * omega / (rho + omega * omega) : 1.0;
                    const double rp = rho * d2;
                    double F[L1 + 1];
                    boys_f64<L1>(rp * fma(PQx, PQx, fma(PQy, PQy, PQz * PQz)), tabs.f64, F);
                    double s = 2.0 * sqrt(rp * INV_PI_D);
#pragma unroll
                    for (int n = 0; n <= L1; n++) {
                        Rb[n] = F[n] * s;
                        s *= -2.0 * rp;
                    }
                    R0[0] = Rb[L1];
                }
                __syncwarp();
#pragma unroll 1
                for (int n = L1 - 1; n >= 0; n--) {
                    double* src = ((L1 - 1 - n) & 1) ? R1 : R0;
                    double* dst = ((L1 - 1 - n) & 1) ? R0 : R1;
                    const int cnt = nherm(L1 - n);
                    if (valid) {
                        for (int i = sub; i < cnt; i += SG) {
                            const uint32_t rec = sRec[i];
                            const uint32_t dir = rec >> 28, s2 = (rec >> 10) & 1023u;
                            const double pq = dir == 0 ? PQx : (dir == 1 ? PQy : PQz);
                            double val = pq * src[rec & 1023u];
                            if (s2 != 1023u) val = fma((double)((rec >> 20) & 255u), src[s2], val);
                            dst[i] = i == 0 ? Rb[n] : val;
                        }
                    }
                    __syncwarp();
                }
                const double* R = (L1 & 1) ? R1 : R0;

                // ---- A side: derivatives on i's centre
#pragma unroll 1
                for (int b = 0; b < NB; b++) {
                    const uint32_t bp_ = sCart[LB][b];
                    const int bx = bp_ & 15u, by = (bp_ >> 4) & 15u, bz = bp_ >> 8;
                    if (valid) {
                        for (int it = sub; it < NC * NHK; it += SG) {
                            const int c = it / NHK, f = it % NHK;
                            const uint32_t tf = sTuv[f];
                            const int t = tf & 255, u = (tf >> 8) & 255, v = tf >> 16;
                            const uint32_t cp_ = sCart[LC][c];
                            const int cx = cp_ & 15u, cy = (cp_ >> 4) & 15u, cz = cp_ >> 8;
                            double y = 0.0;
                            for (int d = 0; d < ND; d++) {
                                const uint32_t dp_ = sCart[LD][d];
                                const int dx = dp_ & 15u, dy = (dp_ >> 4) & 15u, dz = dp_ >> 8;
                                const double e = Ek[0 * S::EK + (cx * (LD + 1) + dx) * LSK + t] *
                                                 Ek[1 * S::EK + (cy * (LD + 1) + dy) * LSK + u] *
                                                 Ek[2 * S::EK + (cz * (LD + 1) + dz) * LSK + v];
                                y = fma(Dbd[b * ND + d] * Scd[c * ND + d], e, y);
                            }
                            Y[it] = ((t + u + v) & 1) ? -y : y;
                        }
                    }
                    __syncwarp();
                    if (valid) {
                        for (int it = sub; it < NA * NHK; it += SG) {
                            const int a = it / NHK, f = it % NHK;
                            double s = 0.0;
                            for (int c = 0; c < NC; c++) s = fma(sDw[a * NC + c], Y[c * NHK + f], s);
                            T[it] = Sab[a * NB + b] * s;
                        }
                    }
                    __syncwarp();
                    if (valid) {
                        // lanes over bra Hermite indices e; each R_{e+f} serves all a
                        for (int e = sub; e < NHBP; e += SG) {
                            const uint32_t te = sTuv[e];
                            const int t = te & 255, u = (te >> 8) & 255, v = te >> 16;
                            double dE[NA][3];
                            bool any = false;
#pragma unroll
                            for (int a = 0; a < NA; a++) {
                                const uint32_t ap_ = sCart[LA][a];
                                const int ax = ap_ & 15u, ay = (ap_ >> 4) & 15u, az = ap_ >> 8;
                                // 1-D factors E^{i,j}_t at i = a_x, a_x + 1, a_x - 1 (0 when i < 0)
                                const double x0 = Eb[0 * S::EB + (ax * (LB + 1) + bx) * LSB + t];
                                const double y0 = Eb[1 * S::EB + (ay * (LB + 1) + by) * LSB + u];
                                const double z0 = Eb[2 * S::EB + (az * (LB + 1) + bz) * LSB + v];
                                const double xp = Eb[0 * S::EB + ((ax + 1) * (LB + 1) + bx) * LSB + t];
                                const double yp = Eb[1 * S::EB + ((ay + 1) * (LB + 1) + by) * LSB + u];
                                const double zp = Eb[2 * S::EB + ((az + 1) * (LB + 1) + bz) * LSB + v];
                                const double xm = ax > 0 ? Eb[0 * S::EB + ((ax - 1) * (LB + 1) + bx) * LSB + t] : 0.0;
                                const double ym = ay > 0 ? Eb[1 * S::EB + ((ay - 1) * (LB + 1) + by) * LSB + u] : 0.0;
                                const double zm = az > 0 ? Eb[2 * S::EB + ((az - 1) * (LB + 1) + bz) * LSB + v] : 0.0;
                                dE[a][0] = (al2 * xp - ax * xm) * y0 * z0;
                                dE[a][1] = x0 * (al2 * yp - ay * ym) * z0;
                                dE[a][2] = x0 * y0 * (al2 * zp - az * zm);
                                any = any || dE[a][0] != 0.0 || dE[a][1] != 0.0 || dE[a][2] != 0.0;
                            }
                            if (!any) continue;
                            double acc[NA];
#pragma unroll
                            for (int a = 0; a < NA; a++) acc[a] = 0.0;
                            for (int f = 0; f < NHK; f++) {
                                const double r = R[sIdx[f][e]];
#pragma unroll
                                for (int a = 0; a < NA; a++) acc[a] = fma(r, T[a * NHK + f], acc[a]);
                            }
#pragma unroll
                            for (int a = 0; a < NA; a++) {
                                g[0] = fma(dE[a][0], acc[a], g[0]);
                                g[1] = fma(dE[a][1], acc[a], g[1]);
                                g[2] = fma(dE[a][2], acc[a], g[2]);
                            }
                        }
                    }
                    __syncwarp();
                }

                // ---- C side: derivatives on k's centre
#pragma unroll 1
                for (int d = 0; d < ND; d++) {
                    const uint32_t dp_ = sCart[LD][d];
                    const int dx = dp_ & 15u, dy = (dp_ >> 4) & 15u, dz = dp_ >> 8;
                    if (valid) {
                        for (int it = sub; it < NA * NHB; it += SG) {
                            const int a = it / NHB, e = it % NHB;
                            const uint32_t te = sTuv[e];
                            const int t = te & 255, u = (te >> 8) & 255, v = te >> 16;
                            const uint32_t ap_ = sCart[LA][a];
                            const int ax = ap_ & 15u, ay = (ap_ >> 4) & 15u, az = ap_ >> 8;
                            double y = 0.0;
                            for (int b = 0; b < NB; b++) {
                                const uint32_t bp_ = sCart[LB][b];
                                const int bx = bp_ & 15u, by = (bp_ >> 4) & 15u, bz = bp_ >> 8;
                                const double e1 = Eb[0 * S::EB + (ax * (LB + 1) + bx) * LSB + t] *
                                                  Eb[1 * S::EB + (ay * (LB + 1) + by) * LSB + u] *
                                                  Eb[2 * S::EB + (az * (LB + 1) + bz) * LSB + v];
                                y = fma(Dbd[b * ND + d] * Sab[a * NB + b], e1, y);
                            }
                            Y[it] = y;
                        }
                    }
                    __syncwarp();
                    if (valid) {
                        for (int it = sub; it < NC * NHB; it += SG) {
                            const int c = it / NHB, e = it % NHB;
                            double s = 0.0;
                            for (int a = 0; a < NA; a++) s = fma(sDw[a * NC + c], Y[a * NHB + e], s);
                            T[it] = Scd[c * ND + d] * s;
                        }
                    }
                    __syncwarp();
                    if (valid) {
                        // lanes over ket Hermite indices f; each R_{e+f} serves all c
                        for (int f = sub; f < NHKP; f += SG) {
                            const uint32_t tf = sTuv[f];
                            const int t = tf & 255, u = (tf >> 8) & 255, v = tf >> 16;
                            const double sg = ((t + u + v) & 1) ? -1.0 : 1.0;
                            double dE[NC][3];
                            bool any = false;
#pragma unroll
                            for (int c = 0; c < NC; c++) {
                                const uint32_t cp_ = sCart[LC][c];
                                const int cx = cp_ & 15u, cy = (cp_ >> 4) & 15u, cz = cp_ >> 8;
                                const double x0 = Ek[0 * S::EK + (cx * (LD + 1) + dx) * LSK + t];
                                const double y0 = Ek[1 * S::EK + (cy * (LD + 1) + dy) * LSK + u];
                                const double z0 = Ek[2 * S::EK + (cz * (LD + 1) + dz) * LSK + v];
                                const double xp = Ek[0 * S::EK + ((cx + 1) * (LD + 1) + dx) * LSK + t];
                                const double yp = Ek[1 * S::EK + ((cy + 1) * (LD + 1) + dy) * LSK + u];
                                const double zp = Ek[2 * S::EK + ((cz + 1) * (LD + 1) + dz) * LSK + v];
                                const double xm = cx > 0 ? Ek[0 * S::EK + ((cx - 1) * (LD + 1) + dx) * LSK + t] : 0.0;
                                const double ym = cy > 0 ? Ek[1 * S::EK + ((cy - 1) * (LD + 1) + dy) * LSK + u] : 0.0;
                                const double zm = cz > 0 ? Ek[2 * S::EK + ((cz - 1) * (LD + 1) + dz) * LSK + v] : 0.0;
                                dE[c][0] = sg * (ga2 * xp - cx * xm) * y0 * z0;
                                dE[c][1] = sg * x0 * (ga2 * yp - cy * ym) * z0;
                                dE[c][2] = sg * x0 * y0 * (ga2 * zp - cz * zm);
                                any = any || dE[c][0] != 0.0 || dE[c][1] != 0.0 || dE[c][2] != 0.0;
                            }
                            if (!any) continue;
                            double acc[NC];
#pragma unroll
                            for (int c = 0; c < NC; c++) acc[c] = 0.0;
                            for (int e = 0; e < NHB; e++) {
                                const double r = R[sIdx[f][e]];
#pragma unroll
                                for (int c = 0; c < NC; c++) acc[c] = fma(r, T[c * NHB + e], acc[c]);
                            }
#pragma unroll
                            for (int c = 0; c < NC; c++) {
                                g[3] = fma(dE[c][0], acc[c], g[3]);
                                g[4] = fma(dE[c][1], acc[c], g[4]);
                                g[5] = fma(dE[c][2], acc[c], g[5]);
                            }
                        }
                    }
                    __syncwarp();
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int x = 0; x < 6; x++) {
            const double v = warp_sum(g[x]);
            if (lane == 0) red[warp][x] = v;
        }
        __syncthreads();
        if (threadIdx.x < 6 && s_pmin != INT32_MAX) {
            double s = red[0][threadIdx.x];
#pragma unroll
            for (int w = 1; w < NW; w++) s += red[w][threadIdx.x];
            grad[threadIdx.x * gstride + s_pmin] += s;
        }
        __syncthreads();
    }
}

}  // namespace vlxb
