// Coulomb nuclear-gradient kernel: bra-centre derivatives of J in
// McMurchie-Davidson form, with several quartets per warp.
//
// Same mathematics as coulomb_md_kernel (md_kernels.cuh) one derivative up: the
// bra Hermite range grows by one level (R up to L + 1, X_e up to
// LA + LB + 1) and the epilogue sums E^{a+-1,b} and E^{a,b+-1} against X:
//   dJ_ab/dA_x = S_ab sum_e (2 alpha E^{a+1x,b}_e - a_x E^{a-1x,b}_e) X_e,
// the same with beta = p - alpha on B (Obara-Saika 1986, Eq. 5; eri.py:85-129
// of the reference generator).  Output: grad[k * gstride + o], k = 0..2 the
// A components, 3..5 the B components, accumulated with +=.
//
// Layout: one CTA per bra record (as the J kernels); its kets are spread over
// groups of SG lanes (SG = 2 .. 32 by the width of the bra Hermite range), so
// that a warp works on 32 / SG quartets at once instead of one: the light
// classes, whose Hermite ranges are a few entries wide, no longer leave most
// lanes idle.  Per quartet the group forms the Hermite Coulomb integrals
// R_{tuv} level by level in its shared-memory slice (a recurrence table built
// once per CTA), then each lane adds X_e += sum_f R_{e+f} Dh_f for its bra
// Hermite indices e.  Ket densities Dh come from the list preparation, or are
// rebuilt with the exact per-component screen for kets in the screening slack
// band.  After the record's kets, X is reduced over the groups in a fixed
// order (no atomics).  Screening, quartet set and FP32 pass are those of the J
// kernels.
#pragma once
#include <type_traits>

#include "jk_kernels.cuh"
#include "md.cuh"

namespace vlxb {

template <int LA, int LB, int LC, int LD>
struct JGradShape {
    static constexpr int L = LA + LB + LC + LD + 1;
    static constexpr int NHB = nherm(LA + LB + 1), NHK = nherm(LC + LD), NHL = nherm(L);
    static constexpr int NC = ncart(LC), ND = ncart(LD), NCD = NC * ND;
    static constexpr int NEK = (LC + 1) * (LD + 1) * (LC + LD + 1);
    static constexpr int NW = 4;
    static constexpr int THREADS = NW * 32;
    // shared memory of one quartet group (R levels, R^{(n)}_{000}, Dh, the
    // slack-band ket tables, X) and of the CTA (index tables, bra E tables)
    static constexpr int GROUP_BYTES = 8 * (2 * NHL + (L + 1) + NHK + 3 * NEK + NCD + NHB);
    static constexpr int FIXED_BYTES =
        2 * NHK * NHB + 8 * NHL + 8 * 3 * (LA + 2) * (LB + 2) * (LA + LB + 3) + 64;
    // lanes per quartet: about half the bra Hermite range (a power of two in
    // [2, 32]), doubled until the CTA's groups fit in 44 KB of shared memory
    static constexpr int pick_sg()
    {
        int sg = NHB <= 4 ? 2 : NHB <= 8 ? 4 : NHB <= 16 ? 8 : NHB <= 32 ? 16 : 32;
        while (sg < 32 && NW * (32 / sg) * GROUP_BYTES + FIXED_BYTES > 44 * 1024) sg *= 2;
        return sg;
    }
    static constexpr int SG = pick_sg();
    static constexpr int NG = 32 / SG;
    static constexpr int NEP = (NHB + SG - 1) / SG;  // bra Hermite indices per lane
};

template <int LA, int LB, int LC, int LD, int PM>
__global__ void __launch_bounds__(JGradShape<LA, LB, LC, LD>::THREADS)
coulomb_grad_kernel(JBraRecs bra, JKetPairs ket, double* __restrict__ grad, int64_t gstride, double thr,
                    BoysTabs tabs, double fp32_cut)
{
    using T = typename std::conditional<PM == 0, double, float>::type;
    using S = JGradShape<LA, LB, LC, LD>;
    constexpr int L = S::L, NHB = S::NHB, NHK = S::NHK, NHL = S::NHL;
    constexpr int NA = ncart(LA), NB = ncart(LB), NAB = NA * NB;
    constexpr int NC = S::NC, ND = S::ND, NCD = S::NCD, NEK = S::NEK;
    constexpr int SG = S::SG, NG = S::NG, NW = S::NW, NT_ = S::THREADS, NEP = S::NEP;
    constexpr int NGT = NW * NG;  // quartet groups per CTA
    constexpr int NEB = (LA + 2) * (LB + 2) * (LA + LB + 3);
    __shared__ T sR[NGT][2][NHL];
    __shared__ T sBase[NGT][L + 1];
    __shared__ T sDh[NGT][NHK];
    __shared__ double sEk[NGT][3][NEK];  // ket 1-D Hermite coefficients (slack-band kets)
    __shared__ double sDm[NGT][NCD];     // screened ket density (slack-band kets)
    __shared__ int16_t sIdx[NHK][NHB];   // index of R_{e+f}
    __shared__ uint32_t sTuv[NHL];
    __shared__ uint32_t sRec[NHL];       // R recurrence per entry (as coulomb_md_kernel)
    __shared__ double sX[NGT][NHB];
    __shared__ double sEb[3][NEB];       // bra 1-D Hermite coefficients up to (LA + 1, LB + 1)
    __shared__ int s_ncut, s_n64;

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
    for (int i = threadIdx.x; i < NHK * NHB; i += NT_) {
        const int f = i / NHB, e = i % NHB;
        const uint32_t a = sTuv[e], b = sTuv[f];
        sIdx[f][e] = (int16_t)herm_idx((a & 255) + (b & 255), ((a >> 8) & 255) + ((b >> 8) & 255),
                                       (a >> 16) + (b >> 16));
    }
    __syncthreads();

    const int nbra = *bra.n_rec;
    const int nket = *ket.n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = lane / SG, sub = lane % SG, gid = warp * NG + grp;
    T* R0 = sR[gid][0];
    T* R1 = sR[gid][1];

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
            ket_prefixes(ket, k0, k1, qb, thr, fp32_cut, 0.0, 0.0, ncut, nexact, n64);
            s_ncut = ncut;
            s_n64 = n64;
        }
        __syncthreads();
        const int ncut = s_ncut, n64 = s_n64;
        const int kb = PM == 0 ? k0 : n64, ke = PM == 0 ? n64 : ncut;
        if (PM == 1 && kb >= ke) {
            __syncthreads();
            continue;  // no FP32 quartets for this bra
        }

        double X[NEP];
#pragma unroll
        for (int p = 0; p < NEP; p++) X[p] = 0.0;
        // every group of a warp walks the same number of slots, so the
        // warp-wide __syncwarp() calls stay uniform; a group without a ket in
        // its slot skips the work
        for (int base = kb + warp * NG; base < ke; base += NW * NG) {
            const int kt = base + grp;
            const bool valid = kt < ke;
            PairGeo k{};
            bool slack = false;
            if (valid) {
                k = load_geo(ket.geo, ket.stride, kt);
                slack = !(qb * __ldg(ket.tmin + kt) > thr * (1.0 + SCREEN_SLACK));
                if (slack) {
                    for (int x = sub; x < 3; x += SG) {
                        const double qc = x == 0 ? k.Ax : (x == 1 ? k.Ay : k.Az);
                        const double cd = x == 0 ? k.Rx : (x == 1 ? k.Ry : k.Rz);
                        herm_e1_flat<LC, LD>(qc, qc + cd, k.i2z, sEk[gid][x]);
                    }
                    for (int c = sub; c < NCD; c += SG) {
                        const double qk = __ldg(ket.Qc + c * ket.stride + kt);
                        const double dk = __ldg(ket.Dc + c * ket.stride + kt);
                        sDm[gid][c] = (fabs(qb * qk * dk) > thr) ? __ldg(ket.Dm + c * ket.stride + kt) : 0.0;
                    }
                }
            }
            __syncwarp();
            if (valid) {
                if (!slack) {
                    for (int f = sub; f < NHK; f += SG) sDh[gid][f] = (T)__ldg(ket.Dh + (int64_t)kt * NHK + f);
                } else {
                    for (int f = sub; f < NHK; f += SG) {
                        const uint32_t a = sTuv[f];
                        const int t = a & 255, u = (a >> 8) & 255, v = a >> 16;
                        double h = 0.0;
#pragma unroll
                        for (int c = 0; c < NC; c++)
#pragma unroll
                            for (int d = 0; d < ND; d++) {
                                const int cx = cart_x(LC, c), cy = cart_y(LC, c), cz = cart_z(LC, c);
                                const int dx = cart_x(LD, d), dy = cart_y(LD, d), dz = cart_z(LD, d);
                                if (t <= cx + dx && u <= cy + dy && v <= cz + dz)
                                    h = fma(sDm[gid][c * ND + d] *
                                                sEk[gid][0][(cx * (LD + 1) + dx) * (LC + LD + 1) + t] *
                                                sEk[gid][1][(cy * (LD + 1) + dy) * (LC + LD + 1) + u],
                                            sEk[gid][2][(cz * (LD + 1) + dz) * (LC + LD + 1) + v], h);
                            }
                        sDh[gid][f] = (T)(((t + u + v) & 1) ? -h : h);
                    }
                }
            }
            // R^{(n)}_{000} = Lambda (-2 rho)^n F_n(T), then the levels n = L-1 .. 0
            const double inv = 1.0 / (b.z + k.z);
            const double rho = b.z * k.z * inv;
            const double PQx = b.Px - k.Px, PQy = b.Py - k.Py, PQz = b.Pz - k.Pz;
            if (valid && sub == 0) {
                const double T2 = rho * fma(PQx, PQx, fma(PQy, PQy, PQz * PQz));
                if constexpr (PM == 0) {
                    double F[L + 1];
                    boys_f64<L>(T2, tabs.f64, F);
                    double s = 2.0 * sqrt(rho * INV_PI_D);
#pragma unroll
                    for (int n = 0; n <= L; n++) {
                        sBase[gid][n] = F[n] * s;
                        s *= -2.0 * rho;
                    }
                } else {
                    float F[L + 1];
                    boys_f32<L>(T2, tabs.f64, F);
                    float s = (float)(2.0 * sqrt(rho * INV_PI_D));
                    const float m2r = (float)(-2.0 * rho);
#pragma unroll
                    for (int n = 0; n <= L; n++) {
                        sBase[gid][n] = F[n] * s;
                        s *= m2r;
                    }
                }
                R0[0] = sBase[gid][L];
            }
            __syncwarp();
            const T X_ = (T)PQx, Y_ = (T)PQy, Z_ = (T)PQz;
#pragma unroll 1
            for (int n = L - 1; n >= 0; n--) {
                T* src = ((L - 1 - n) & 1) ? R1 : R0;
                T* dst = ((L - 1 - n) & 1) ? R0 : R1;
                const int cnt = nherm(L - n);
                if (valid) {
                    for (int i = sub; i < cnt; i += SG) {
                        const uint32_t rec = sRec[i];
                        const uint32_t dir = rec >> 28, s2 = (rec >> 10) & 1023u;
                        const T pq = dir == 0 ? X_ : (dir == 1 ? Y_ : Z_);
                        T val = pq * src[rec & 1023u];
                        if (s2 != 1023u) val = fma((T)((rec >> 20) & 255u), src[s2], val);
                        dst[i] = i == 0 ? sBase[gid][n] : val;
                    }
                }
                __syncwarp();
            }
            const T* R = (L & 1) ? R1 : R0;  // level 0: written by pass L-1 (R1 when L is odd)
            if (valid) {
#pragma unroll
                for (int p = 0; p < NEP; p++) {
                    const int e = sub + SG * p;
                    if (e < NHB) {
                        T s = (T)0;
#pragma unroll 7
                        for (int f = 0; f < NHK; f++) s = fma(sDh[gid][f], R[sIdx[f][e]], s);
                        X[p] += (double)s;
                    }
                }
            }
            __syncwarp();
        }
        // fixed-order reduction of X over the groups, then the derivative epilogue
#pragma unroll
        for (int p = 0; p < NEP; p++) {
            const int e = sub + SG * p;
            if (e < NHB) sX[gid][e] = X[p];
        }
        __syncthreads();
        for (int e = threadIdx.x; e < NHB; e += NT_) {
            double s = sX[0][e];
            for (int w = 1; w < NGT; w++) s += sX[w][e];
            sX[0][e] = s;
        }
        if (threadIdx.x < 3) {
            const double pa = threadIdx.x == 0 ? b.Ax : (threadIdx.x == 1 ? b.Ay : b.Az);
            const double ab = threadIdx.x == 0 ? b.Rx : (threadIdx.x == 1 ? b.Ry : b.Rz);
            herm_e1_flat<LA + 1, LB + 1>(pa, pa + ab, b.i2z, sEb[threadIdx.x]);
        }
        __syncthreads();
        const uint64_t mask = __ldg(bra.rec_mask + r);
        if (threadIdx.x < NAB && ((mask >> threadIdx.x) & 1ull)) {
            const int c = threadIdx.x;
            const int ai = c / NB, bi = c % NB;
            const int ax = cart_x(LA, ai), ay = cart_y(LA, ai), az = cart_z(LA, ai);
            const int bx = cart_x(LB, bi), by = cart_y(LB, bi), bz = cart_z(LB, bi);
            constexpr int LS = LA + LB + 3, NJ = LB + 2;
            // sum_e E^{(ix,iy,iz),(jx,jy,jz)}_e X_e over the product's Hermite box
            auto hsum = [&](int ix, int iy, int iz, int jx, int jy, int jz) {
                double acc = 0.0;
                for (int t = 0; t <= ix + jx; t++)
                    for (int u = 0; u <= iy + jy; u++) {
                        const double etu = sEb[0][(ix * NJ + jx) * LS + t] * sEb[1][(iy * NJ + jy) * LS + u];
                        for (int v = 0; v <= iz + jz; v++)
                            acc = fma(etu * sEb[2][(iz * NJ + jz) * LS + v], sX[0][herm_idx(t, u, v)], acc);
                    }
                return acc;
            };
            const int32_t o = __ldg(bra.entry + c * bra.sp_stride + sp);
            const double Sv = __ldg(bra.pdata + o);
            const double al2 = 2.0 * __ldg(bra.geo + G_ALPHA * bra.sp_stride + sp);
            const double be2 = 2.0 * b.z - al2;
            const int av[3] = {ax, ay, az}, bv[3] = {bx, by, bz};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const int ex = d == 0, ey = d == 1, ez = d == 2;
                double gA = al2 * hsum(ax + ex, ay + ey, az + ez, bx, by, bz);
                if (av[d] > 0) gA -= av[d] * hsum(ax - ex, ay - ey, az - ez, bx, by, bz);
                double gB = be2 * hsum(ax, ay, az, bx + ex, by + ey, bz + ez);
                if (bv[d] > 0) gB -= bv[d] * hsum(ax, ay, az, bx - ex, by - ey, bz - ez);
                grad[d * gstride + o] += Sv * gA;
                grad[(3 + d) * gstride + o] += Sv * gB;
            }
        }
        __syncthreads();
    }
}

}  // namespace vlxb
