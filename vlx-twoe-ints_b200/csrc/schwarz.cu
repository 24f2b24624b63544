// Schwarz diagonal of primitive shell pairs: for each pair (P, Q) of types
// (LA, LB), the largest over components of sqrt|(ab|ab)| / |S_ab| (the bare
// diagonal integral, before the pair prefactors).  Used by the caller-side
// list builder; the reference's caller computes its Q outside the generator.
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

int run_schwarz_f(int la, int lb, const double* info_a, uint32_t cnt_a, const double* info_b, uint32_t cnt_b,
                  const uint32_t* P, const uint32_t* Q, uint32_t n, double* out, cudaStream_t st);

template <int LA, int LB>
__global__ void __launch_bounds__(128)
schwarz_kernel(const double* __restrict__ info_a, uint32_t cnt_a, const double* __restrict__ info_b, uint32_t cnt_b,
               const uint32_t* __restrict__ P, const uint32_t* __restrict__ Q, uint32_t n, double* __restrict__ out,
               const double* __restrict__ boys_tab)
{
    constexpr int NA = ncart(LA), NB = ncart(LB), L = 2 * (LA + LB);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const uint32_t i = P[t], j = Q[t];
        const double ai = info_a[i], aj = info_b[j];
        PairGeo g;
        const double A[3] = {info_a[i + 2 * (int64_t)cnt_a], info_a[i + 3 * (int64_t)cnt_a], info_a[i + 4 * (int64_t)cnt_a]};
        const double B[3] = {info_b[j + 2 * (int64_t)cnt_b], info_b[j + 3 * (int64_t)cnt_b], info_b[j + 4 * (int64_t)cnt_b]};
        g.z = ai + aj;
        const double iz = 1.0 / g.z;
        g.i2z = 0.5 * iz;
        g.Px = (ai * A[0] + aj * B[0]) * iz; g.Py = (ai * A[1] + aj * B[1]) * iz; g.Pz = (ai * A[2] + aj * B[2]) * iz;
        g.Ax = g.Px - A[0]; g.Ay = g.Py - A[1]; g.Az = g.Pz - A[2];
        g.Rx = A[0] - B[0]; g.Ry = A[1] - B[1]; g.Rz = A[2] - B[2];
        QV q;
        double F[L + 1];
        make_quartet<L>(g, g, 0.0, boys_tab, q, F);
        double I[NA * NB * NA * NB];
        eri_full<LA, LB, LA, LB, double>(q, F, I);
        double m = 0.0;
#pragma unroll
        for (int c = 0; c < NA * NB; c++) m = fmax(m, fabs(I[c * NA * NB + c]));
        out[t] = sqrt(m);
    }
}

}  // namespace vlxb

extern "C" int vlxb_schwarzBareMax(int la, int lb, const double* info_a, uint32_t cnt_a, const double* info_b,
                                   uint32_t cnt_b, const uint32_t* P, const uint32_t* Q, uint32_t n, double* out,
                                   void* stream)
{
    using namespace vlxb;
    if (n == 0) return VLXB_OK;
    if (!info_a || !info_b || !P || !Q || !out || la < 0 || lb < la || lb > 3) return VLXB_EINVAL;
    int rc = ensure_pool_configured();
    if (rc) return rc;
    if (lb == 3) return run_schwarz_f(la, lb, info_a, cnt_a, info_b, cnt_b, P, Q, n, out, (cudaStream_t)stream);
    const double* tab = boys_table_device();
    if (!tab) return VLXB_ECUDA;
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = (int)((n + 127) / 128 < 148 * 64 ? (n + 127) / 128 : 148 * 64);
#define VLXB_SCHWARZ(A, B) \
    if (la == A && lb == B) schwarz_kernel<A, B><<<grid, 128, 0, st>>>(info_a, cnt_a, info_b, cnt_b, P, Q, n, out, tab);
    VLXB_SCHWARZ(0, 0) VLXB_SCHWARZ(0, 1) VLXB_SCHWARZ(0, 2) VLXB_SCHWARZ(1, 1) VLXB_SCHWARZ(1, 2) VLXB_SCHWARZ(2, 2)
#undef VLXB_SCHWARZ
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

extern "C" int vlxb_quartetCounters(unsigned long long* host_out, int reset, void* stream)
{
    using namespace vlxb;
    unsigned long long* qc = quartet_counters_device();
    if (!qc) return VLXB_ECUDA;
    cudaStream_t st = (cudaStream_t)stream;
    if (host_out) {
        VLXB_CHECK_CUDA(cudaMemcpyAsync(host_out, qc, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        VLXB_CHECK_CUDA(cudaStreamSynchronize(st));
    }
    if (reset) VLXB_CHECK_CUDA(cudaMemsetAsync(qc, 0, 2 * sizeof(unsigned long long), st));
    return VLXB_OK;
}

extern "C" int vlxb_kernelErrors(unsigned long long* host_out, int reset, void* stream)
{
    using namespace vlxb;
    unsigned long long* e = kernel_errors_device();
    if (!e) return VLXB_ECUDA;
    cudaStream_t st = (cudaStream_t)stream;
    if (host_out) {
        VLXB_CHECK_CUDA(cudaMemcpyAsync(host_out, e, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        VLXB_CHECK_CUDA(cudaStreamSynchronize(st));
    }
    if (reset) VLXB_CHECK_CUDA(cudaMemsetAsync(e, 0, sizeof(unsigned long long), st));
    return VLXB_OK;
}
