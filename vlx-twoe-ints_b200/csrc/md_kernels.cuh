// Coulomb kernel in McMurchie-Davidson form (the "J engine", md.cuh).
//
// CTA per bra record (as coulomb_kernel); its warps take the record's kets
// one quartet per warp.  Per quartet the warp forms the Hermite Coulomb
// integrals R_{tuv}, t+u+v <= L, level by level in shared memory (lanes share
// the entries of a level; each entry's recurrence comes from a table built
// once per CTA), then each lane owns bra Hermite indices e and adds
// X_e += sum_f R_{e+f} Dh_f with the ket pair's signed Hermite density Dh
// (formed once per ket pair in the list preparation; recomputed with the
// exact per-component screen for kets in the screening slack band).  After
// the record's kets: fixed-order reduction of X over the warps and
// J_ab = S_ab sum_e E^{ab}_e X_e per present component pair.  Same screening,
// same counters, same FP32/FP64 passes as coulomb_kernel; no atomics on J.
//
// The nuclear-gradient form of the same mathematics (bra Hermite range one
// level higher, derivative epilogue) is coulomb_grad_kernel in
// jgrad_kernels.cuh.
#pragma once
#include <type_traits>

#include "jk_kernels.cuh"
#include "md.cuh"

namespace vlxb {

constexpr int MD_THREADS = 128;

template <int LA, int LB, int LC, int LD, int PM>
__global__ void __launch_bounds__(MD_THREADS)
coulomb_md_kernel(JBraRecs bra, JKetPairs ket, double* __restrict__ mat_J, double thr, BoysTabs tabs,
                  unsigned long long* __restrict__ qcount, double fp32_cut, double fp32_budget)
{
    using T = typename std::conditional<PM == 0, double, float>::type;
    constexpr int L = LA + LB + LC + LD;
    constexpr int NHB = nherm(LA + LB), NHK = nherm(LC + LD), NHL = nherm(L);
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr int NAB = NA * NB, NCD = NC * ND;
    constexpr int NW = MD_THREADS / 32;
    constexpr int NEP = (NHB + 31) / 32;  // bra Hermite indices per lane
    constexpr int NEK = (LC + 1) * (LD + 1) * (LC + LD + 1), NEB = (LA + 1) * (LB + 1) * (LA + LB + 1);
    __shared__ T sR[NW][2][NHL];
    __shared__ T sDh[NW][NHK];
    __shared__ int16_t sIdx[NHK][NHB];  // index of R_{e+f}
    __shared__ uint32_t sTuv[NHL];      // t | u << 8 | v << 16 of Hermite index i
    // recurrence of entry i (the same at every level): R_i = PQ_dir * R_s1 + c * R_s2,
    // packed s1 | s2 << 10 | c << 20 | dir << 28 (s2 = 1023: no second term)
    __shared__ uint32_t sRec[NHL];
    __shared__ double sX[NW][NHB];
    __shared__ double sEk[NW][3][NEK];  // ket 1-D Hermite coefficients (slack-band kets)
    __shared__ double sDm[NW][NCD];     // screened ket density (slack-band kets)
    __shared__ double sEb[3][NEB];      // bra 1-D Hermite coefficients
    __shared__ T sBase[NW][L + 1];      // R^{(n)}_{000} of the warp's quartet
    __shared__ int s_ncut, s_n64;

    for (int i = threadIdx.x; i < NHL; i += MD_THREADS) {
        int n = 0;
        while (nherm(n) <= i) n++;
        const int r = i - (n > 0 ? nherm(n - 1) : 0);  // position inside level n
        int s = 0;                                      // s = u + v
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
    for (int i = threadIdx.x; i < NHK * NHB; i += MD_THREADS) {
        const int f = i / NHB, e = i % NHB;
        const uint32_t a = sTuv[e], b = sTuv[f];
        sIdx[f][e] = (int16_t)herm_idx((a & 255) + (b & 255), ((a >> 8) & 255) + ((b >> 8) & 255),
                                       (a >> 16) + (b >> 16));
    }
    __syncthreads();

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
        const int kb = PM == 0 ? k0 : n64, ke = PM == 0 ? n64 : ncut;
        if (PM == 1 && kb >= ke) {
            __syncthreads();
            continue;  // no FP32 quartets for this bra
        }

        double X[NEP];
#pragma unroll
        for (int p = 0; p < NEP; p++) X[p] = 0.0;
        for (int kt = kb + warp; kt < ke; kt += NW) {
            const PairGeo k = load_geo(ket.geo, ket.stride, kt);
            // ket Hermite density (exact per-component screen in the slack band)
            if (qb * __ldg(ket.tmin + kt) > thr * (1.0 + SCREEN_SLACK)) {
                for (int f = lane; f < NHK; f += 32) sDh[warp][f] = (T)__ldg(ket.Dh + (int64_t)kt * NHK + f);
            } else {
                if (lane < 3) {
                    const double qc = lane == 0 ? k.Ax : (lane == 1 ? k.Ay : k.Az);
                    const double cd = lane == 0 ? k.Rx : (lane == 1 ? k.Ry : k.Rz);
                    herm_e1_flat<LC, LD>(qc, qc + cd, k.i2z, sEk[warp][lane]);
                }
                for (int c = lane; c < NCD; c += 32) {
                    const double qk = __ldg(ket.Qc + c * ket.stride + kt);
                    const double dk = __ldg(ket.Dc + c * ket.stride + kt);
                    sDm[warp][c] = (fabs(qb * qk * dk) > thr) ? __ldg(ket.Dm + c * ket.stride + kt) : 0.0;
                }
                __syncwarp();
                for (int f = lane; f < NHK; f += 32) {
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
                                h = fma(sDm[warp][c * ND + d] *
                                            sEk[warp][0][(cx * (LD + 1) + dx) * (LC + LD + 1) + t] *
                                            sEk[warp][1][(cy * (LD + 1) + dy) * (LC + LD + 1) + u],
                                        sEk[warp][2][(cz * (LD + 1) + dz) * (LC + LD + 1) + v], h);
                        }
                    sDh[warp][f] = (T)(((t + u + v) & 1) ? -h : h);
                }
            }
            // R^{(n)}_{000} = Lambda (-2 rho)^n F_n(T), then the levels n = L-1 .. 0
            const double inv = 1.0 / (b.z + k.z);
            const double rho = b.z * k.z * inv;
            const double PQx = b.Px - k.Px, PQy = b.Py - k.Py, PQz = b.Pz - k.Pz;
            const double T2 = rho * fma(PQx, PQx, fma(PQy, PQy, PQz * PQz));
            T base[L + 1];
            if constexpr (PM == 0) {
                double F[L + 1];
                boys_f64<L>(T2, tabs.f64, F);
                double s = 2.0 * sqrt(rho * INV_PI_D);
#pragma unroll
                for (int n = 0; n <= L; n++) {
                    base[n] = F[n] * s;
                    s *= -2.0 * rho;
                }
            } else {
                float F[L + 1];
                boys_f32<L>(T2, tabs.f64, F);
                float s = (float)(2.0 * sqrt(rho * INV_PI_D));
                const float m2r = (float)(-2.0 * rho);
#pragma unroll
                for (int n = 0; n <= L; n++) {
                    base[n] = F[n] * s;
                    s *= m2r;
                }
            }
            const T X_ = (T)PQx, Y_ = (T)PQy, Z_ = (T)PQz;
            T* R0 = sR[warp][0];
            T* R1 = sR[warp][1];
            if (lane == 0) {
#pragma unroll
                for (int n = 0; n <= L; n++) sBase[warp][n] = base[n];
                R0[0] = base[L];
            }
            __syncwarp();
#pragma unroll 1
            for (int n = L - 1; n >= 0; n--) {
                T* src = ((L - 1 - n) & 1) ? R1 : R0;
                T* dst = ((L - 1 - n) & 1) ? R0 : R1;
                const int cnt = nherm(L - n);
                for (int i = lane; i < cnt; i += 32) {
                    const uint32_t rec = sRec[i];
                    const uint32_t dir = rec >> 28, s2 = (rec >> 10) & 1023u;
                    const T pq = dir == 0 ? X_ : (dir == 1 ? Y_ : Z_);
                    T val = pq * src[rec & 1023u];
                    if (s2 != 1023u) val = fma((T)((rec >> 20) & 255u), src[s2], val);
                    dst[i] = i == 0 ? sBase[warp][n] : val;
                }
                __syncwarp();
            }
            const T* R = (L & 1) ? R1 : R0;  // level 0: written by pass L-1 (R1 when L is odd)
            // contraction over the ket Hermite indices
#pragma unroll
            for (int p = 0; p < NEP; p++) {
                const int e = lane + 32 * p;
                if (e < NHB) {
                    T s = (T)0;
#pragma unroll 7
                    for (int f = 0; f < NHK; f++) s = fma(sDh[warp][f], R[sIdx[f][e]], s);
                    X[p] += (double)s;
                }
            }
            __syncwarp();
        }
        // fixed-order reduction over the warps, then J_ab = S_ab sum_e E^{ab}_e X_e
#pragma unroll
        for (int p = 0; p < NEP; p++) {
            const int e = lane + 32 * p;
            if (e < NHB) sX[warp][e] = X[p];
        }
        __syncthreads();
        for (int e = threadIdx.x; e < NHB; e += MD_THREADS) {
            double s = sX[0][e];
            for (int w = 1; w < NW; w++) s += sX[w][e];
            sX[0][e] = s;
        }
        if (threadIdx.x < 3) {
            const double pa = threadIdx.x == 0 ? b.Ax : (threadIdx.x == 1 ? b.Ay : b.Az);
            const double ab = threadIdx.x == 0 ? b.Rx : (threadIdx.x == 1 ? b.Ry : b.Rz);
            herm_e1_flat<LA, LB>(pa, pa + ab, b.i2z, sEb[threadIdx.x]);
        }
        __syncthreads();
        const uint64_t mask = __ldg(bra.rec_mask + r);
        if (threadIdx.x < NAB && ((mask >> threadIdx.x) & 1ull)) {
            const int c = threadIdx.x;
            const int ai = c / NB, bi = c % NB;
            const int ax = cart_x(LA, ai), ay = cart_y(LA, ai), az = cart_z(LA, ai);
            const int bx = cart_x(LB, bi), by = cart_y(LB, bi), bz = cart_z(LB, bi);
            constexpr int LS = LA + LB + 1, NJ = LB + 1;
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
            const double S = __ldg(bra.pdata + o);
            mat_J[o] += S * hsum(ax, ay, az, bx, by, bz);
        }
        __syncthreads();
    }
}

}  // namespace vlxb
