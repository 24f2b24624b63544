// Common device definitions for the vlxb J/K engine (sm_100a).
//
// Quartet scalars follow the conventions of the reference's Obara-Saika engine
// (eri.py:237-355 and the emitted prologue gen_coulomb.py:244-268):
//   PQ = Q - P, W - P = eta/(zeta+eta) PQ, W - Q = -zeta/(zeta+eta) PQ,
//   [00|00]^m = Lambda F_m(T), Lambda = sqrt(4 rho / pi), T = rho |PQ|^2,
// with range separation (gen_exchange.py:278-298):
//   d2 = w^2/(rho+w^2), Lambda *= sqrt(d2), T *= d2, F_m *= d2^m.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace vlxb {

// ---------------------------------------------------------------- Boys table
// F_m(T) at T_k = k * BOYS_H for k in [0, BOYS_NGRID), m in [0, BOYS_NCOL).
// Evaluation: Taylor expansion of F_L about the nearest grid point with
// BOYS_NT terms (|dT| <= BOYS_H/2 = 0.025: truncation < 1e-17 relative),
// then downward recursion F_m = (2T F_{m+1} + e^-T)/(2m+1).  For
// T >= BOYS_TMAX: F_0 = sqrt(pi/T)/2 (error e^-T/sqrt(pi T) < 4e-17
// relative) and exact upward recursion F_{m+1} = ((2m+1)F_m - e^-T)/(2T),
// which is stable for T > m.
constexpr int BOYS_NT = 8;
constexpr double BOYS_H = 0.05;
constexpr double BOYS_INV_H = 20.0;
constexpr double BOYS_TMAX = 36.0;
constexpr int BOYS_NGRID = 721;  // BOYS_TMAX / BOYS_H + 1
constexpr int BOYS_NCOL = 20;    // max m needed: 12 (f shells) + BOYS_NT - 1 = 19
constexpr int MAX_L = 8;

constexpr double PI_D = 3.141592653589793238462643383279502884;
constexpr double INV_PI_D = 0.318309886183790671537767526745028724;
constexpr double SQRT_PI_4 = 0.886226925452758013649083741671;  // sqrt(pi)/2

__device__ __forceinline__ constexpr double inv_odd(int m) { return 1.0 / (2.0 * m + 1.0); }

template <int L>
__device__ __forceinline__ void boys_f64(double T, const double* __restrict__ tab, double* F)
{
    if (T < BOYS_TMAX) {
        const int k = __double2int_rn(T * BOYS_INV_H);
        const double md = (double)k * BOYS_H - T;  // -dT
        const double* row = tab + k * BOYS_NCOL + L;
        double acc = __ldg(row + BOYS_NT - 1);
#pragma unroll
        for (int j = BOYS_NT - 1; j >= 1; j--) acc = fma(acc, md * (1.0 / j), __ldg(row + j - 1));
        F[L] = acc;
        if (L > 0) {
            const double ex = exp(-T);
            const double t2 = 2.0 * T;
#pragma unroll
            for (int m = L - 1; m >= 0; m--) F[m] = fma(t2, F[m + 1], ex) * inv_odd(m);
        }
    } else {
        const double inv_t = 1.0 / T;
        F[0] = SQRT_PI_4 * sqrt(inv_t);
        if (L > 0) {
            const double ex = exp(-T);
            const double h = 0.5 * inv_t;
#pragma unroll
            for (int m = 0; m < L; m++) F[m + 1] = fma((2.0 * m + 1.0), F[m], -ex) * h;
        }
    }
}

// FP32 variant for the mixed-precision path.  F_L and e^-T come from the FP64
// evaluation above (the same table, 8 Taylor terms, FP64 exp), rounded once
// to float, so the Boys values carry no error beyond one float rounding; only
// the short recursion runs in float.  This costs a few FP64 operations per
// quartet and removes the bias a float table and a fast exponential put into
// every FP32 quartet.
template <int L>
__device__ __forceinline__ void boys_f32(double Td, const double* __restrict__ tab, float* F)
{
    if (Td < BOYS_TMAX) {
        const int k = __double2int_rn(Td * BOYS_INV_H);
        const double md = (double)k * BOYS_H - Td;
        const double* row = tab + k * BOYS_NCOL + L;
        double acc = __ldg(row + BOYS_NT - 1);
#pragma unroll
        for (int j = BOYS_NT - 1; j >= 1; j--) acc = fma(acc, md * (1.0 / j), __ldg(row + j - 1));
        F[L] = (float)acc;
        if (L > 0) {
            const float ex = (float)exp(-Td);
            const float t2 = (float)(2.0 * Td);
#pragma unroll
            for (int m = L - 1; m >= 0; m--) F[m] = fmaf(t2, F[m + 1], ex) * (1.0f / (2.0f * m + 1.0f));
        }
    } else {
        F[0] = (float)(SQRT_PI_4 * sqrt(1.0 / Td));
        if (L > 0) {
            const float ex = (float)exp(-Td);
            const float h = (float)(0.5 / Td);
#pragma unroll
            for (int m = 0; m < L; m++) F[m + 1] = fmaf((2.0f * m + 1.0f), F[m], -ex) * h;
        }
    }
}

// ---------------------------------------------------------------- quartet
template <typename T>
struct QVT {
    T PAx, PAy, PAz, WPx, WPy, WPz;
    T QCx, QCy, QCz, WQx, WQy, WQz;
    T ABx, ABy, ABz, CDx, CDy, CDz;
    T inv2z, inv2e, inv2ze, rz, re;
};
using QV = QVT<double>;

// Primitive-pair geometry records (one per primitive shell pair), SoA in HBM.
// Bra: zeta, 0.5/zeta, P[3], PA = P - A [3], AB = A - B [3], alpha (A's exponent).
// Ket: eta,  0.5/eta,  Q[3], QC = Q - C [3], CD = C - D [3], gamma (C's exponent).
// The exponent row is read only by the gradient kernels.
constexpr int GEO_N = 12;
enum GeoField { G_Z = 0, G_I2Z, G_PX, G_PY, G_PZ, G_AX, G_AY, G_AZ, G_RX, G_RY, G_RZ, G_ALPHA };

struct PairGeo {
    double z, i2z, Px, Py, Pz, Ax, Ay, Az, Rx, Ry, Rz;
};

__device__ __forceinline__ PairGeo load_geo(const double* __restrict__ g, int64_t stride, int64_t i)
{
    PairGeo p;
    p.z = __ldg(g + 0 * stride + i);
    p.i2z = __ldg(g + 1 * stride + i);
    p.Px = __ldg(g + 2 * stride + i);
    p.Py = __ldg(g + 3 * stride + i);
    p.Pz = __ldg(g + 4 * stride + i);
    p.Ax = __ldg(g + 5 * stride + i);
    p.Ay = __ldg(g + 6 * stride + i);
    p.Az = __ldg(g + 7 * stride + i);
    p.Rx = __ldg(g + 8 * stride + i);
    p.Ry = __ldg(g + 9 * stride + i);
    p.Rz = __ldg(g + 10 * stride + i);
    return p;
}

// Quartet scalars and the Lambda-scaled Boys values F[0..L].
template <int L>
__device__ __forceinline__ void make_quartet(const PairGeo& b, const PairGeo& k, double omega,
                                             const double* __restrict__ boys_tab, QV& q, double* F)
{
    const double inv = 1.0 / (b.z + k.z);
    const double rho = b.z * k.z * inv;
    const double PQx = k.Px - b.Px, PQy = k.Py - b.Py, PQz = k.Pz - b.Pz;
    const double rz = k.z * inv, re = b.z * inv;
    q.PAx = b.Ax; q.PAy = b.Ay; q.PAz = b.Az;
    q.ABx = b.Rx; q.ABy = b.Ry; q.ABz = b.Rz;
    q.QCx = k.Ax; q.QCy = k.Ay; q.QCz = k.Az;
    q.CDx = k.Rx; q.CDy = k.Ry; q.CDz = k.Rz;
    q.WPx = rz * PQx; q.WPy = rz * PQy; q.WPz = rz * PQz;
    q.WQx = -re * PQx; q.WQy = -re * PQy; q.WQz = -re * PQz;
    q.inv2z = b.i2z; q.inv2e = k.i2z; q.inv2ze = 0.5 * inv;
    q.rz = rz; q.re = re;
    const double r2 = fma(PQx, PQx, fma(PQy, PQy, PQz * PQz));
    double d2 = 1.0;
    if (omega != 0.0) d2 = omega * omega / (rho + omega * omega);
    const double rd = rho * d2;
    boys_f64<L>(rd * r2, boys_tab, F);
    const double lam = 2.0 * sqrt(rd * INV_PI_D);
    if (omega != 0.0) {
        double s = lam;
#pragma unroll
        for (int m = 0; m <= L; m++) { F[m] *= s; s *= d2; }
    } else {
#pragma unroll
        for (int m = 0; m <= L; m++) F[m] *= lam;
    }
}

// Mixed-precision variant of make_quartet: every quartet scalar and the Boys
// argument are formed in FP64 and rounded to float; F_m in float (boys_f32).
template <int L>
__device__ __forceinline__ void make_quartet_f32(const PairGeo& b, const PairGeo& k, double omega,
                                                 const double* __restrict__ boys_tab, QVT<float>& q, float* F)
{
    const double inv = 1.0 / (b.z + k.z);
    const double rho = b.z * k.z * inv;
    const double PQx = k.Px - b.Px, PQy = k.Py - b.Py, PQz = k.Pz - b.Pz;
    const double rz = k.z * inv, re = b.z * inv;
    q.PAx = (float)b.Ax; q.PAy = (float)b.Ay; q.PAz = (float)b.Az;
    q.ABx = (float)b.Rx; q.ABy = (float)b.Ry; q.ABz = (float)b.Rz;
    q.QCx = (float)k.Ax; q.QCy = (float)k.Ay; q.QCz = (float)k.Az;
    q.CDx = (float)k.Rx; q.CDy = (float)k.Ry; q.CDz = (float)k.Rz;
    q.WPx = (float)(rz * PQx); q.WPy = (float)(rz * PQy); q.WPz = (float)(rz * PQz);
    q.WQx = (float)(-re * PQx); q.WQy = (float)(-re * PQy); q.WQz = (float)(-re * PQz);
    q.inv2z = (float)b.i2z; q.inv2e = (float)k.i2z; q.inv2ze = (float)(0.5 * inv);
    q.rz = (float)rz; q.re = (float)re;
    const double r2 = fma(PQx, PQx, fma(PQy, PQy, PQz * PQz));
    double d2 = 1.0;
    if (omega != 0.0) d2 = omega * omega / (rho + omega * omega);
    const double rd = rho * d2;
    boys_f32<L>(rd * r2, boys_tab, F);
    const float lam = (float)(2.0 * sqrt(rd * INV_PI_D));
    float s = lam;
    const float d2f = (float)d2;
#pragma unroll
    for (int m = 0; m <= L; m++) { F[m] *= s; s *= d2f; }
}

// Precision-generic quartet set-up (overloaded on the output type).
template <int L>
__device__ __forceinline__ void make_quartet_t(const PairGeo& b, const PairGeo& k, double omega,
                                               const double* __restrict__ tab64, const float* __restrict__ tab32,
                                               QVT<double>& q, double* F)
{
    make_quartet<L>(b, k, omega, tab64, q, F);
}
template <int L>
__device__ __forceinline__ void make_quartet_t(const PairGeo& b, const PairGeo& k, double omega,
                                               const double* __restrict__ tab64, const float* __restrict__ tab32,
                                               QVT<float>& q, float* F)
{
    make_quartet_f32<L>(b, k, omega, tab64, q, F);
}

template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void eri_full(const QVT<T>& q, const T* F, T* out);
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void j_contract(const QVT<T>& q, const T* F, const T* Dpp, T* X);
template <int LC, int LD, typename T>
__device__ __forceinline__ void hrr_ket_adjoint(T CDx, T CDy, T CDz, const T* Dm, T* Dpp);
template <int LA, int LB, typename T>
__device__ __forceinline__ void hrr_bra_vector(T ABx, T ABy, T ABz, const T* X, T* J);

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
// number of Cartesian components with |e| in [l0, l0 + l1]
__host__ __device__ constexpr int nrange(int l0, int l1)
{
    int n = 0;
    for (int l = l0; l <= l0 + l1; l++) n += ncart(l);
    return n;
}

// Deterministic warp reduction (fixed butterfly order).
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace vlxb
