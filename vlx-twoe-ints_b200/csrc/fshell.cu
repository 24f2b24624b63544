// J and K entry points of the classes with f shells.
//
// The reference's writer maps only p and d letters (eriwriter.py:44-62),
// although its ERI engine takes any number of Cartesian indices (eri.py:59
// labels angular momenta up to I); no f kernel is emitted.  These entry
// points are this library's own, with the argument conventions of the
// generated ones (gen_coulomb.py:74-93, gen_exchange.py:75-115) and the f
// components in the same order as d (x^3 first, then by decreasing y power:
// xxx, xxy, xxz, xyy, xyz, xzz, yyy, yyz, yzz, zzz).
//
// The s/p/d classes run generated straight-line shell-quartet code; doing
// the same for 170 f classes would multiply the library's size and build
// time.  The f classes run one generic kernel per kind instead, with the
// angular momenta as runtime arguments, at the reference's granularity: one
// Cartesian component quartet per work item, evaluated in
// McMurchie-Davidson form,
//   (ab|cd) = S_ab S_cd 2 sqrt(rho'/pi) sum_{tuv} E^ab_t E^ab_u E^ab_v
//             sum_{t'u'v'} (-1)^{t'+u'+v'} E^cd_t' E^cd_u' E^cd_v' R_{t+t',u+u',v+v'}
// with the 1-D Hermite coefficients of each pair and the Hermite Coulomb
// integrals R_{tuv} of the quartet (R^{(n)}_{000} = (-2 rho')^n F_n(rho'|PQ|^2),
// rho' = rho for the Coulomb operator and rho w^2 / (rho + w^2) for the
// attenuated one), built inside the component's own box t <= a_x+b_x+c_x+d_x,
// u <= .., v <= .. .  Screening is the reference's per-component predicate
// (|Q_ij Q_kl D_kl| > thr for J, |Q_ij Q_kl max_D| > thr for K), the J ket
// weights gen_coulomb.py:276-281, the K density gather gen_exchange.py:323.
// A CTA owns one output entry (J bra entry, K (i, k) entry); its threads
// stride over the kets / partner pairs and reduce in a fixed order, so
// results are bit-reproducible.  FP64 only; these classes are not counted
// by vlxb_quartetCounters.
#include "classes.cuh"
#include "md.cuh"

namespace vlxb {

constexpr int FS_THREADS = 128;
constexpr int FS_LMAX = 3;                  // f
constexpr int FS_EMAX = 2 * FS_LMAX + 1;    // 1-D Hermite coefficients per pair and direction
constexpr int FS_BOX = 125;                 // max (tx+1)(ty+1)(tz+1) for tx+ty+tz <= 12

// F_m(T), m = 0..L (runtime L <= 12), from the FP64 table as boys_f64.
__device__ void boys_rt(int L, double T, const double* __restrict__ tab, double* F)
{
    if (T < BOYS_TMAX) {
        const int k = __double2int_rn(T * BOYS_INV_H);
        const double md = (double)k * BOYS_H - T;
        const double* row = tab + k * BOYS_NCOL + L;
        double acc = __ldg(row + BOYS_NT - 1);
        for (int j = BOYS_NT - 1; j >= 1; j--) acc = fma(acc, md * (1.0 / j), __ldg(row + j - 1));
        F[L] = acc;
        const double ex = exp(-T);
        for (int m = L - 1; m >= 0; m--) F[m] = fma(2.0 * T, F[m + 1], ex) / (2.0 * m + 1.0);
    } else {
        F[0] = SQRT_PI_4 * sqrt(1.0 / T);
        const double ex = exp(-T);
        for (int m = 0; m < L; m++) F[m + 1] = fma(2.0 * m + 1.0, F[m], -ex) * (0.5 / T);
    }
}

// 1-D Hermite coefficients E^{ij}_t, t = 0..i+j, of one pair and direction
// (md.cuh's recurrence with runtime i, j <= 3).
__device__ void herm1(int i, int j, double PA, double PB, double i2p, double* E)
{
    double e[FS_LMAX + 1][FS_LMAX + 1][FS_EMAX];
    for (int a = 0; a <= i; a++)
        for (int b = 0; b <= j; b++)
            for (int t = 0; t < FS_EMAX; t++) e[a][b][t] = 0.0;
    e[0][0][0] = 1.0;
    for (int a = 0; a < i; a++)
        for (int t = 0; t <= a + 1; t++) {
            double v = (t <= a) ? PA * e[a][0][t] : 0.0;
            if (t > 0) v = fma(i2p, e[a][0][t - 1], v);
            if (t + 1 <= a) v = fma((double)(t + 1), e[a][0][t + 1], v);
            e[a + 1][0][t] = v;
        }
    for (int b = 0; b < j; b++)
        for (int t = 0; t <= i + b + 1; t++) {
            double v = (t <= i + b) ? PB * e[i][b][t] : 0.0;
            if (t > 0) v = fma(i2p, e[i][b][t - 1], v);
            if (t + 1 <= i + b) v = fma((double)(t + 1), e[i][b][t + 1], v);
            e[i][b + 1][t] = v;
        }
    for (int t = 0; t <= i + j; t++) E[t] = e[i][j][t];
}

struct FPrim {
    double alpha, r[3];
    int c[3];  // Cartesian exponents of the component
};

// prim-cart index -> exponent, centre and component of a type-l primitive
// (prim_info [5][count]: row 0 exponent, rows 2..4 centre).
__device__ __forceinline__ FPrim fprim(const double* __restrict__ info, uint32_t count, int l, uint32_t idx)
{
    const int nc = ncart(l);
    const uint32_t p = idx / (uint32_t)nc;
    const int comp = (int)(idx % (uint32_t)nc);
    FPrim f;
    f.alpha = __ldg(info + p);
    f.r[0] = __ldg(info + p + 2 * (int64_t)count);
    f.r[1] = __ldg(info + p + 3 * (int64_t)count);
    f.r[2] = __ldg(info + p + 4 * (int64_t)count);
    f.c[0] = cart_x(l, comp);
    f.c[1] = cart_y(l, comp);
    f.c[2] = l - f.c[0] - f.c[1];
    return f;
}

// (ab|cd) / (S_ab S_cd) of one Cartesian component quartet.
__device__ double eri_component(const FPrim& A, const FPrim& B, const FPrim& C, const FPrim& D, double omega,
                                const double* __restrict__ tab)
{
    const double p = A.alpha + B.alpha, q = C.alpha + D.alpha;
    double Eab[3][FS_EMAX], Ecd[3][FS_EMAX], PQ[3];
    int tb[3];
    for (int x = 0; x < 3; x++) {
        const double P = (A.alpha * A.r[x] + B.alpha * B.r[x]) / p;
        const double Q = (C.alpha * C.r[x] + D.alpha * D.r[x]) / q;
        herm1(A.c[x], B.c[x], P - A.r[x], P - B.r[x], 0.5 / p, Eab[x]);
        herm1(C.c[x], D.c[x], Q - C.r[x], Q - D.r[x], 0.5 / q, Ecd[x]);
        PQ[x] = P - Q;
        tb[x] = A.c[x] + B.c[x] + C.c[x] + D.c[x];
    }
    const int L = tb[0] + tb[1] + tb[2];
    const double rho = p * q / (p + q);
    const double d2 = omega != 0.0 ? omega * omega / (rho + omega * omega) : 1.0;
    const double rp = rho * d2;
    double F[4 * FS_LMAX + 1];
    boys_rt(L, rp * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]), tab, F);
    // R^{(n)}_{tuv} inside the box, levels n = L .. 0 (two buffers)
    const int nx = tb[0] + 1, ny = tb[1] + 1, nz = tb[2] + 1;
    double Ra[FS_BOX], Rb[FS_BOX];
    double* src = Ra;
    double* dst = Rb;
    double s = 2.0 * sqrt(rp * INV_PI_D);
    double base[4 * FS_LMAX + 1];
    for (int n = 0; n <= L; n++) {
        base[n] = F[n] * s;
        s *= -2.0 * rp;
    }
    src[0] = base[L];
    for (int n = L - 1; n >= 0; n--) {
        const int lev = L - n;  // t + u + v <= lev
        for (int t = 0; t < nx; t++)
            for (int u = 0; u < ny; u++)
                for (int v = 0; v < nz; v++) {
                    if (t + u + v > lev) continue;
                    const int o = (t * ny + u) * nz + v;
                    double val;
                    if (t > 0) {
                        val = PQ[0] * src[((t - 1) * ny + u) * nz + v];
                        if (t > 1) val = fma((double)(t - 1), src[((t - 2) * ny + u) * nz + v], val);
                    } else if (u > 0) {
                        val = PQ[1] * src[(u - 1) * nz + v];
                        if (u > 1) val = fma((double)(u - 1), src[(u - 2) * nz + v], val);
                    } else if (v > 0) {
                        val = PQ[2] * src[v - 1];
                        if (v > 1) val = fma((double)(v - 1), src[v - 2], val);
                    } else {
                        val = base[n];
                    }
                    dst[o] = val;
                }
        double* tmp = src;
        src = dst;
        dst = tmp;
    }
    // src holds R^{(0)}; contract with the bra and (signed) ket coefficients
    double sum = 0.0;
    for (int t = 0; t <= A.c[0] + B.c[0]; t++)
        for (int u = 0; u <= A.c[1] + B.c[1]; u++)
            for (int v = 0; v <= A.c[2] + B.c[2]; v++) {
                const double eb = Eab[0][t] * Eab[1][u] * Eab[2][v];
                double k = 0.0;
                for (int t2 = 0; t2 <= C.c[0] + D.c[0]; t2++)
                    for (int u2 = 0; u2 <= C.c[1] + D.c[1]; u2++)
                        for (int v2 = 0; v2 <= C.c[2] + D.c[2]; v2++) {
                            const double ek = Ecd[0][t2] * Ecd[1][u2] * Ecd[2][v2];
                            const double r = src[((t + t2) * ny + (u + u2)) * nz + (v + v2)];
                            k = fma(((t2 + u2 + v2) & 1) ? -ek : ek, r, k);
                        }
                sum = fma(eb, k, sum);
            }
    return sum;
}

__device__ __forceinline__ double fs_block_sum(double v, double* red)
{
    v = warp_sum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < FS_THREADS / 32; w++) s += red[w];
    __syncthreads();
    return s;
}

struct FShellJ {
    int la, lb, lc, ld;
    const double* info[4];
    uint32_t count[4];
    const double *cd_D, *ab_Q, *cd_Q;
    const uint32_t *ab_first, *ab_second;
    const double* ab_pdata;
    uint32_t n_ab;
    const uint32_t *cd_first, *cd_second;
    const double* cd_pdata;
    uint32_t n_cd;
    double thr;
};

__global__ void __launch_bounds__(FS_THREADS)
coulomb_fshell_kernel(FShellJ a, double* __restrict__ mat_J, const double* __restrict__ tab)
{
    __shared__ double red[FS_THREADS / 32];
    for (uint32_t ij = blockIdx.x; ij < a.n_ab; ij += gridDim.x) {
        const FPrim A = fprim(a.info[a.la], a.count[a.la], a.la, __ldg(a.ab_first + ij));
        const FPrim B = fprim(a.info[a.lb], a.count[a.lb], a.lb, __ldg(a.ab_second + ij));
        const double qij = __ldg(a.ab_Q + ij);
        double acc = 0.0;
        for (uint32_t kl = threadIdx.x; kl < a.n_cd; kl += FS_THREADS) {
            const double dkl = __ldg(a.cd_D + kl);
            if (fabs(qij * __ldg(a.cd_Q + kl) * dkl) <= a.thr) continue;
            const uint32_t k = __ldg(a.cd_first + kl), l = __ldg(a.cd_second + kl);
            const FPrim C = fprim(a.info[a.lc], a.count[a.lc], a.lc, k);
            const FPrim D = fprim(a.info[a.ld], a.count[a.ld], a.ld, l);
            const double w = (a.lc != a.ld || k != l) ? 2.0 : 1.0;
            acc = fma(__ldg(a.cd_pdata + kl) * eri_component(A, B, C, D, 0.0, tab), dkl * w, acc);
        }
        const double s = fs_block_sum(acc, red);
        if (threadIdx.x == 0) mat_J[ij] += __ldg(a.ab_pdata + ij) * s;
    }
}

struct FShellK {
    int la, lb, lc, ld;
    const uint32_t *pair_i, *pair_k;
    uint32_t n_ik;
    const double* info[4];
    const uint32_t* aoinds[4];
    uint32_t count[4];
    double maxD;
    const double* D;
    uint32_t naos;
    const double *Q_ab, *Q_cd;
    const uint32_t *Dinds_ab, *Dinds_cd, *displs_ab, *displs_cd, *counts_ab, *counts_cd;
    const double *pdata_ab, *pdata_cd;
    double omega, thr;
};

__global__ void __launch_bounds__(FS_THREADS)
exchange_fshell_kernel(FShellK a, double* __restrict__ mat_K, const double* __restrict__ tab)
{
    __shared__ double red[FS_THREADS / 32];
    const int ncb = ncart(a.lb), ncd = ncart(a.ld);
    for (uint32_t ik = blockIdx.x; ik < a.n_ik; ik += gridDim.x) {
        const uint32_t i = __ldg(a.pair_i + ik), k = __ldg(a.pair_k + ik);
        const FPrim A = fprim(a.info[a.la], a.count[a.la], a.la, i);
        const FPrim C = fprim(a.info[a.lc], a.count[a.lc], a.lc, k);
        const uint32_t j0 = __ldg(a.displs_ab + i), nj = __ldg(a.counts_ab + i);
        const uint32_t l0 = __ldg(a.displs_cd + k), nl = __ldg(a.counts_cd + k);
        const uint64_t npair = (uint64_t)nj * nl;
        double acc = 0.0;
        for (uint64_t w = threadIdx.x; w < npair; w += FS_THREADS) {
            const uint32_t pj = j0 + (uint32_t)(w / nl), pl = l0 + (uint32_t)(w % nl);
            if (fabs(__ldg(a.Q_ab + pj) * __ldg(a.Q_cd + pl) * a.maxD) <= a.thr) continue;
            const uint32_t jp = __ldg(a.Dinds_ab + pj), lp = __ldg(a.Dinds_cd + pl);
            const FPrim B = fprim(a.info[a.lb], a.count[a.lb], a.lb, jp);
            const FPrim D = fprim(a.info[a.ld], a.count[a.ld], a.ld, lp);
            const uint32_t jao = __ldg(a.aoinds[a.lb] + jp / (uint32_t)ncb + (int64_t)a.count[a.lb] * (jp % ncb));
            const uint32_t lao = __ldg(a.aoinds[a.ld] + lp / (uint32_t)ncd + (int64_t)a.count[a.ld] * (lp % ncd));
            const double eri = __ldg(a.pdata_ab + pj) * __ldg(a.pdata_cd + pl) * eri_component(A, B, C, D, a.omega, tab);
            acc = fma(eri, __ldg(a.D + (int64_t)jao * a.naos + lao), acc);
        }
        const double s = fs_block_sum(acc, red);
        if (threadIdx.x == 0) mat_K[ik] += s;
    }
}

// Schwarz diagonal of primitive shell pairs with an f shell: the largest
// over components (a, b) of sqrt|(ab|ab)| / |S_ab| (vlxb_schwarzBareMax).
__global__ void __launch_bounds__(FS_THREADS)
schwarz_fshell_kernel(int la, int lb, const double* __restrict__ info_a, uint32_t cnt_a,
                      const double* __restrict__ info_b, uint32_t cnt_b, const uint32_t* __restrict__ P,
                      const uint32_t* __restrict__ Q, uint32_t n, double* __restrict__ out,
                      const double* __restrict__ tab)
{
    const int na = ncart(la), nb = ncart(lb);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        double m = 0.0;
        for (int ca = 0; ca < na; ca++)
            for (int cb = 0; cb < nb; cb++) {
                const FPrim A = fprim(info_a, cnt_a, la, P[t] * (uint32_t)na + ca);
                const FPrim B = fprim(info_b, cnt_b, lb, Q[t] * (uint32_t)nb + cb);
                m = fmax(m, fabs(eri_component(A, B, A, B, 0.0, tab)));
            }
        out[t] = sqrt(m);
    }
}

// Pair prefactor S_PQ = c_P c_Q (pi / p)^(3/2) exp(-a b / p |A - B|^2) and
// Q_PQ = |S_PQ| sqrt(max bare diagonal) of pairs with an f shell
// (vlxb_shellPairData).
__global__ void __launch_bounds__(FS_THREADS)
shell_pair_fshell_kernel(int la, int lb, const double* __restrict__ info_a, uint32_t cnt_a,
                         const double* __restrict__ info_b, uint32_t cnt_b, const uint32_t* __restrict__ P,
                         const uint32_t* __restrict__ Q, uint32_t n, double* __restrict__ S_out,
                         double* __restrict__ q_out, const double* __restrict__ tab)
{
    const int na = ncart(la), nb = ncart(lb);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t i = P[t], j = Q[t];
        const FPrim A0 = fprim(info_a, cnt_a, la, i * (uint32_t)na);
        const FPrim B0 = fprim(info_b, cnt_b, lb, j * (uint32_t)nb);
        const double p = A0.alpha + B0.alpha, iz = 1.0 / p;
        double R2 = 0.0;
        for (int x = 0; x < 3; x++) R2 += (A0.r[x] - B0.r[x]) * (A0.r[x] - B0.r[x]);
        const double pi_p = 3.14159265358979323846 * iz;
        const double S = __ldg(info_a + i + (int64_t)cnt_a) * __ldg(info_b + j + (int64_t)cnt_b) * pi_p *
                         sqrt(pi_p) * exp(-A0.alpha * B0.alpha * iz * R2);
        double m = 0.0;
        for (int ca = 0; ca < na; ca++)
            for (int cb = 0; cb < nb; cb++) {
                const FPrim A = fprim(info_a, cnt_a, la, i * (uint32_t)na + ca);
                const FPrim B = fprim(info_b, cnt_b, lb, j * (uint32_t)nb + cb);
                m = fmax(m, fabs(eri_component(A, B, A, B, 0.0, tab)));
            }
        S_out[t] = S;
        q_out[t] = fabs(S) * sqrt(m);
    }
}

int run_shell_pair_f(int la, int lb, const double* info_a, uint32_t cnt_a, const double* info_b, uint32_t cnt_b,
                     const uint32_t* P, const uint32_t* Q, uint32_t n, double* S_out, double* q_out,
                     cudaStream_t st)
{
    const double* tab = boys_table_device();
    if (!tab) return VLXB_ECUDA;
    const uint32_t want = (n + FS_THREADS - 1) / FS_THREADS;
    const int grid = (int)(want < 148u * 64u ? want : 148u * 64u);
    shell_pair_fshell_kernel<<<grid, FS_THREADS, 0, st>>>(la, lb, info_a, cnt_a, info_b, cnt_b, P, Q, n, S_out, q_out,
                                                          tab);
    note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

int run_schwarz_f(int la, int lb, const double* info_a, uint32_t cnt_a, const double* info_b, uint32_t cnt_b,
                  const uint32_t* P, const uint32_t* Q, uint32_t n, double* out, cudaStream_t st)
{
    const double* tab = boys_table_device();
    if (!tab) return VLXB_ECUDA;
    const uint32_t want = (n + FS_THREADS - 1) / FS_THREADS;
    const int grid = (int)(want < 148u * 64u ? want : 148u * 64u);
    schwarz_fshell_kernel<<<grid, FS_THREADS, 0, st>>>(la, lb, info_a, cnt_a, info_b, cnt_b, P, Q, n, out, tab);
    note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

int run_coulomb_f(int la, int lb, int lc, int ld, const CoulombArgs& a, cudaStream_t st)
{
    if (a.n_ab == 0 || a.n_cd == 0) return VLXB_OK;
    if (!a.mat_J || !a.cd_D || !a.ab_Q || !a.cd_Q || !a.ab_first || !a.ab_second || !a.ab_pdata || !a.cd_first ||
        !a.cd_second || !a.cd_pdata)
        return VLXB_EINVAL;
    const int L4[4] = {la, lb, lc, ld};
    for (int t = 0; t < 4; t++)
        if (L4[t] < 0 || L4[t] > FS_LMAX || !a.info[L4[t]] || a.count[L4[t]] == 0) return VLXB_EINVAL;
    if (!(a.thr >= 0.0)) return VLXB_EINVAL;
    const double* tab = boys_table_device();
    if (!tab) return VLXB_ECUDA;
    FShellJ f{la, lb, lc, ld, {a.info[0], a.info[1], a.info[2], a.info[3]},
              {a.count[0], a.count[1], a.count[2], a.count[3]}, a.cd_D, a.ab_Q, a.cd_Q, a.ab_first, a.ab_second,
              a.ab_pdata, a.n_ab, a.cd_first, a.cd_second, a.cd_pdata, a.n_cd, a.thr};
    int grid = launch_grid_limit();
    if ((int64_t)grid > (int64_t)a.n_ab) grid = (int)a.n_ab;
    coulomb_fshell_kernel<<<grid, FS_THREADS, 0, st>>>(f, a.mat_J, tab);
    note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

int run_exchange_f(int la, int lb, int lc, int ld, const ExchangeArgs& a, cudaStream_t st)
{
    if (a.n_ik == 0) return VLXB_OK;
    if (!a.mat_K || !a.pair_i || !a.pair_k || !a.D || !a.Q_ab || !a.Q_cd || !a.Dinds_ab || !a.Dinds_cd ||
        !a.displs_ab || !a.displs_cd || !a.counts_ab || !a.counts_cd || !a.pdata_ab || !a.pdata_cd || a.naos == 0)
        return VLXB_EINVAL;
    const int L4[4] = {la, lb, lc, ld};
    for (int t = 0; t < 4; t++)
        if (L4[t] < 0 || L4[t] > FS_LMAX || !a.info[L4[t]] || !a.aoinds[L4[t]] || a.count[L4[t]] == 0)
            return VLXB_EINVAL;
    if (!(a.thr >= 0.0) || !(a.omega >= 0.0)) return VLXB_EINVAL;
    const double* tab = boys_table_device();
    if (!tab) return VLXB_ECUDA;
    FShellK f{la, lb, lc, ld, a.pair_i, a.pair_k, a.n_ik, {a.info[0], a.info[1], a.info[2], a.info[3]},
              {a.aoinds[0], a.aoinds[1], a.aoinds[2], a.aoinds[3]}, {a.count[0], a.count[1], a.count[2], a.count[3]},
              a.maxD, a.D, a.naos, a.Q_ab, a.Q_cd, a.Dinds_ab, a.Dinds_cd, a.displs_ab, a.displs_cd, a.counts_ab,
              a.counts_cd, a.pdata_ab, a.pdata_cd, a.omega, a.thr};
    int grid = launch_grid_limit();
    if ((int64_t)grid > (int64_t)a.n_ik) grid = (int)a.n_ik;
    exchange_fshell_kernel<<<grid, FS_THREADS, 0, st>>>(f, a.mat_K, tab);
    note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

}  // namespace vlxb
