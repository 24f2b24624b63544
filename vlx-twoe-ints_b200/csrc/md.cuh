// McMurchie-Davidson (Hermite) pieces of the Coulomb path.
//
// A product of two Cartesian Gaussians on A and B is a finite sum of Hermite
// Gaussians on P: x_A^i x_B^j exp(-a x_A^2 - b x_B^2) = K_AB sum_t E^{ij}_t
// Lambda_t(x_P), with the 1-D coefficients E of the recurrence
//   E^{i+1,j}_t = 1/(2p) E^{ij}_{t-1} + X_PA E^{ij}_t + (t+1) E^{ij}_{t+1},
//   E^{i,j+1}_t = 1/(2p) E^{ij}_{t-1} + X_PB E^{ij}_t + (t+1) E^{ij}_{t+1},
// E^{00}_0 = 1 (K_AB, the pair's exponential factor, sits in S_ab of the
// reference's pair data).  The electron-repulsion integral of two such pairs is
//   (ab|cd) = S_ab S_cd Lambda sum_{tuv} sum_{tau nu phi} E^{ab}_{tuv}
//             (-1)^{tau+nu+phi} E^{cd}_{tau nu phi} R_{t+tau, u+nu, v+phi}
// with Lambda = 2 sqrt(rho/pi), rho = pq/(p+q), and the Hermite Coulomb
// integrals R_{tuv} = R^{(0)}_{tuv} of the recurrence (X = P_x - Q_x, ...)
//   R^{(n)}_{000} = (-2 rho)^n F_n(rho |PQ|^2),
//   R^{(n)}_{t+1,u,v} = t R^{(n+1)}_{t-1,u,v} + X R^{(n+1)}_{t,u,v}  (same in u, v).
// For J = sum_cd (ab|cd) D_cd the ket side folds into a Hermite density
//   Dh_{tau nu phi} = (-1)^{tau+nu+phi} sum_cd E^{cd}_{tau nu phi} (w D S)_cd,
// formed once per ket pair, and each quartet only needs the R_{tuv} and one
// contraction X_{tuv} += sum_f R_{tuv+f} Dh_f (the "J engine").
#pragma once
#include "common.cuh"

namespace vlxb {

// Hermite indices (t, u, v) with t + u + v <= n, ordered by level, then by
// u + v, then by v: count and position.
__host__ __device__ constexpr int nherm(int n) { return (n + 1) * (n + 2) * (n + 3) / 6; }
__host__ __device__ constexpr int herm_idx(int t, int u, int v)
{
    return (t + u + v) * (t + u + v + 1) * (t + u + v + 2) / 6 + (u + v) * (u + v + 1) / 2 + v;
}
// exponents of Cartesian component c of angular momentum l (x^l first, the
// reference's order: xx, xy, xz, yy, yz, zz)
__host__ __device__ constexpr int cart_x(int l, int c)
{
    int k = 0;
    for (int a = l; a >= 0; a--)
        for (int b = l - a; b >= 0; b--) {
            if (k == c) return a;
            k++;
        }
    return 0;
}
__host__ __device__ constexpr int cart_y(int l, int c)
{
    int k = 0;
    for (int a = l; a >= 0; a--)
        for (int b = l - a; b >= 0; b--) {
            if (k == c) return b;
            k++;
        }
    return 0;
}
__host__ __device__ constexpr int cart_z(int l, int c) { return l - cart_x(l, c) - cart_y(l, c); }

// 1-D Hermite coefficients E[i][j][t], i <= LI, j <= LJ, t <= i + j.
template <int LI, int LJ, typename T>
__device__ __forceinline__ void herm_e1(T PA, T PB, T i2p, T (&E)[LI + 1][LJ + 1][LI + LJ + 1])
{
#pragma unroll
    for (int i = 0; i <= LI; i++)
#pragma unroll
        for (int j = 0; j <= LJ; j++)
#pragma unroll
            for (int t = 0; t <= LI + LJ; t++) E[i][j][t] = (T)0;
    E[0][0][0] = (T)1;
#pragma unroll
    for (int i = 0; i < LI; i++)
#pragma unroll
        for (int t = 0; t <= i + 1; t++) {
            T v = (t <= i) ? PA * E[i][0][t] : (T)0;
            if (t > 0) v = fma(i2p, E[i][0][t - 1], v);
            if (t + 1 <= i) v = fma((T)(t + 1), E[i][0][t + 1], v);
            E[i + 1][0][t] = v;
        }
#pragma unroll
    for (int i = 0; i <= LI; i++)
#pragma unroll
        for (int j = 0; j < LJ; j++)
#pragma unroll
            for (int t = 0; t <= i + j + 1; t++) {
                T v = (t <= i + j) ? PB * E[i][j][t] : (T)0;
                if (t > 0) v = fma(i2p, E[i][j][t - 1], v);
                if (t + 1 <= i + j) v = fma((T)(t + 1), E[i][j][t + 1], v);
                E[i][j + 1][t] = v;
            }
}

// herm_e1 into a flat array E[(i * (LJ + 1) + j) * (LI + LJ + 1) + t] (shared
// memory, one thread per Cartesian direction).
template <int LI, int LJ>
__device__ __forceinline__ void herm_e1_flat(double PA, double PB, double i2p, double* E)
{
    double e[LI + 1][LJ + 1][LI + LJ + 1];
    herm_e1<LI, LJ, double>(PA, PB, i2p, e);
#pragma unroll
    for (int i = 0; i <= LI; i++)
#pragma unroll
        for (int j = 0; j <= LJ; j++)
#pragma unroll
            for (int t = 0; t <= LI + LJ; t++) E[(i * (LJ + 1) + j) * (LI + LJ + 1) + t] = e[i][j][t];
}

// Signed Hermite density of one ket pair: Dh[f] = (-1)^{|f|} sum_cd
// E^{cd}_f Dm[cd] for the nherm(LC + LD) Hermite indices f; geometry of the
// pair record (QC = Q - C in Ax.., CD = C - D in Rx.., 1/(2 eta) in i2z).
template <int LC, int LD, typename T>
__device__ __forceinline__ void herm_ket_density(const PairGeo& k, const T* Dm, T* Dh)
{
    constexpr int NC = ncart(LC), ND = ncart(LD), LS = LC + LD;
    const T i2e = (T)k.i2z;
    T Ex[LC + 1][LD + 1][LS + 1], Ey[LC + 1][LD + 1][LS + 1], Ez[LC + 1][LD + 1][LS + 1];
    herm_e1<LC, LD, T>((T)k.Ax, (T)(k.Ax + k.Rx), i2e, Ex);
    herm_e1<LC, LD, T>((T)k.Ay, (T)(k.Ay + k.Ry), i2e, Ey);
    herm_e1<LC, LD, T>((T)k.Az, (T)(k.Az + k.Rz), i2e, Ez);
#pragma unroll
    for (int f = 0; f < nherm(LS); f++) Dh[f] = (T)0;
#pragma unroll
    for (int c = 0; c < NC; c++)
#pragma unroll
        for (int d = 0; d < ND; d++) {
            const int cx = cart_x(LC, c), cy = cart_y(LC, c), cz = cart_z(LC, c);
            const int dx = cart_x(LD, d), dy = cart_y(LD, d), dz = cart_z(LD, d);
            const T w = Dm[c * ND + d];
#pragma unroll
            for (int t = 0; t <= cx + dx; t++)
#pragma unroll
                for (int u = 0; u <= cy + dy; u++) {
                    const T wtu = w * Ex[cx][dx][t] * Ey[cy][dy][u];
#pragma unroll
                    for (int v = 0; v <= cz + dz; v++) {
                        const T s = ((t + u + v) & 1) ? (T)-1 : (T)1;
                        Dh[herm_idx(t, u, v)] = fma(s * wtu, Ez[cz][dz][v], Dh[herm_idx(t, u, v)]);
                    }
                }
        }
}

}  // namespace vlxb
