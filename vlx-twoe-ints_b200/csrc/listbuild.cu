// Device pieces of the caller-side list builder (the step before the class
// entry points).  The reference's caller (VeloxChem, not part of the
// reference) computes the pair data S_ij_00, the Schwarz values Q, the
// density in pair space and the max-|D| block bounds that the emitted kernels
// take as inputs (gen_coulomb.py:80-90, gen_exchange.py:78-110).  These
// kernels compute them on the GPU from the primitive tables and the AO
// density, so that an SCF loop updates its resident lists without a host
// round trip:
//   vlxb_shellPairData     S and Q of primitive shell pairs,
//   vlxb_gatherPairDensity D_AO gathered into list order (J lists' cd_mat_D),
//   vlxb_blockMaxAbs       max |D_AO| over the AO block of two shell types.
#include "common.cuh"
#include "engine.cuh"
#include "generated/q_ssss.cuh"
#include "generated/q_spsp.cuh"
#include "generated/q_sdsd.cuh"
#include "generated/q_pppp.cuh"
#include "generated/q_pdpd.cuh"
#include "generated/q_dddd.cuh"
#include "../../include/vlxb.h"

namespace vlxb {

int run_shell_pair_f(int la, int lb, const double* info_a, uint32_t cnt_a, const double* info_b, uint32_t cnt_b,
                     const uint32_t* P, const uint32_t* Q, uint32_t n, double* S_out, double* q_out,
                     cudaStream_t st);

// S_PQ = c_P c_Q (pi / p)^(3/2) exp(-a b / p |A - B|^2) and
// Q_PQ = |S_PQ| * max over components sqrt|(ab|ab)| / |S_ab| (the bare
// diagonal integral of the pair, as vlxb_schwarzBareMax).
template <int LA, int LB>
__global__ void __launch_bounds__(128)
shell_pair_kernel(const double* __restrict__ info_a, uint32_t cnt_a, const double* __restrict__ info_b,
                  uint32_t cnt_b, const uint32_t* __restrict__ P, const uint32_t* __restrict__ Q, uint32_t n,
                  double* __restrict__ S_out, double* __restrict__ q_out, const double* __restrict__ boys_tab)
{
    constexpr int NA = ncart(LA), NB = ncart(LB), L = 2 * (LA + LB);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t i = P[t], j = Q[t];
        const double ai = info_a[i], aj = info_b[j];
        const double A[3] = {info_a[i + 2 * (int64_t)cnt_a], info_a[i + 3 * (int64_t)cnt_a],
                             info_a[i + 4 * (int64_t)cnt_a]};
        const double B[3] = {info_b[j + 2 * (int64_t)cnt_b], info_b[j + 3 * (int64_t)cnt_b],
                             info_b[j + 4 * (int64_t)cnt_b]};
        PairGeo g;
        g.z = ai + aj;
        const double iz = 1.0 / g.z;
        g.i2z = 0.5 * iz;
        g.Px = (ai * A[0] + aj * B[0]) * iz; g.Py = (ai * A[1] + aj * B[1]) * iz; g.Pz = (ai * A[2] + aj * B[2]) * iz;
        g.Ax = g.Px - A[0]; g.Ay = g.Py - A[1]; g.Az = g.Pz - A[2];
        g.Rx = A[0] - B[0]; g.Ry = A[1] - B[1]; g.Rz = A[2] - B[2];
        const double R2 = g.Rx * g.Rx + g.Ry * g.Ry + g.Rz * g.Rz;
        const double pi_p = 3.14159265358979323846 * iz;
        const double S = info_a[i + (int64_t)cnt_a] * info_b[j + (int64_t)cnt_b] * pi_p * sqrt(pi_p) *
                         exp(-ai * aj * iz * R2);
        QV q;
        double F[L + 1];
        make_quartet<L>(g, g, 0.0, boys_tab, q, F);
        double I[NA * NB * NA * NB];
        eri_full<LA, LB, LA, LB, double>(q, F, I);
        double m = 0.0;
#pragma unroll
        for (int c = 0; c < NA * NB; c++) m = fmax(m, fabs(I[c * NA * NB + c]));
        S_out[t] = S;
        q_out[t] = fabs(S) * sqrt(m);
    }
}

// D_out[t] = D_AO[ao_a(first[t]), ao_b(second[t])], prim-cart index i ->
// primitive i / ncart, component i % ncart, ao = aoinds[component][primitive].
__global__ void gather_pair_density_kernel(const double* __restrict__ D, uint32_t naos,
                                           const uint32_t* __restrict__ first, const uint32_t* __restrict__ second,
                                           const uint32_t* __restrict__ ao_a, int nca, uint32_t cnt_a,
                                           const uint32_t* __restrict__ ao_b, int ncb, uint32_t cnt_b, int64_t n,
                                           double* __restrict__ out)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t i = first[t], j = second[t];
        const uint32_t a = ao_a[(int64_t)(i % nca) * cnt_a + i / nca];
        const uint32_t b = ao_b[(int64_t)(j % ncb) * cnt_b + j / ncb];
        out[t] = D[(int64_t)a * naos + b];
    }
}

// *out = max |D_AO[r][c]| over r in rows, c in cols.  The maximum is exact and
// does not depend on the reduction order; non-negative doubles order like
// their bit patterns, so an integer atomicMax combines the warps.
__global__ void block_max_abs_kernel(const double* __restrict__ D, uint32_t naos, const uint32_t* __restrict__ rows,
                                     int64_t nr, const uint32_t* __restrict__ cols, int64_t nc,
                                     unsigned long long* __restrict__ out_bits)
{
    double m = 0.0;
    const int64_t n = nr * nc;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(D[(int64_t)rows[t / nc] * naos + cols[t % nc]]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, (unsigned long long)__double_as_longlong(m));
}

}  // namespace vlxb

extern "C" int vlxb_shellPairData(int la, int lb, const double* info_a, uint32_t cnt_a, const double* info_b,
                                  uint32_t cnt_b, const uint32_t* P, const uint32_t* Q, uint32_t n, double* S_out,
                                  double* q_out, void* stream)
{
    using namespace vlxb;
    if (n == 0) return VLXB_OK;
    if (!info_a || !info_b || !P || !Q || !S_out || !q_out || la < 0 || lb < la || lb > 3) return VLXB_EINVAL;
    int rc = ensure_pool_configured();
    if (rc) return rc;
    const double* tab = boys_table_device();
    if (!tab) return VLXB_ECUDA;
    cudaStream_t st = (cudaStream_t)stream;
    if (lb == 3) return run_shell_pair_f(la, lb, info_a, cnt_a, info_b, cnt_b, P, Q, n, S_out, q_out, st);
    const int grid = (int)((n + 127) / 128 < 148 * 64 ? (n + 127) / 128 : 148 * 64);
#define VLXB_SPD(A, B)                                                                                        \
    if (la == A && lb == B)                                                                                   \
        shell_pair_kernel<A, B><<<grid, 128, 0, st>>>(info_a, cnt_a, info_b, cnt_b, P, Q, n, S_out, q_out, tab);
    VLXB_SPD(0, 0) VLXB_SPD(0, 1) VLXB_SPD(0, 2) VLXB_SPD(1, 1) VLXB_SPD(1, 2) VLXB_SPD(2, 2)
#undef VLXB_SPD
    note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

extern "C" int vlxb_gatherPairDensity(const double* D_AO, uint32_t naos, const uint32_t* first,
                                      const uint32_t* second, const uint32_t* aoinds_a, int ncart_a, uint32_t cnt_a,
                                      const uint32_t* aoinds_b, int ncart_b, uint32_t cnt_b, int64_t n, double* out,
                                      void* stream)
{
    using namespace vlxb;
    if (n == 0) return VLXB_OK;
    if (!D_AO || !first || !second || !aoinds_a || !aoinds_b || !out || ncart_a <= 0 || ncart_b <= 0 || n < 0)
        return VLXB_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t want = (n + 255) / 256;
    const int grid = (int)(want < 148 * 16 ? want : 148 * 16);
    gather_pair_density_kernel<<<grid, 256, 0, st>>>(D_AO, naos, first, second, aoinds_a, ncart_a, cnt_a, aoinds_b,
                                                      ncart_b, cnt_b, n, out);
    note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

extern "C" int vlxb_blockMaxAbs(const double* D_AO, uint32_t naos, const uint32_t* rows, int64_t nrows,
                                const uint32_t* cols, int64_t ncols, double* out, void* stream)
{
    using namespace vlxb;
    if (!D_AO || !out || nrows < 0 || ncols < 0) return VLXB_EINVAL;
    const int64_t n = nrows * ncols;
    if (n > 0 && (!rows || !cols)) return VLXB_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    VLXB_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
    if (n == 0) return VLXB_OK;
    const int64_t want = (n + 255) / 256;
    const int grid = (int)(want < 148 * 8 ? want : 148 * 8);
    block_max_abs_kernel<<<grid, 256, 0, st>>>(D_AO, naos, rows, nrows, cols, ncols, (unsigned long long*)out);
    note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}
