// Library-level entry points without a reference counterpart.
#include <cuda_runtime.h>

#include "engine.cuh"
#include "../../include/vlxb.h"

namespace vlxb {

unsigned long long launch_count(bool reset);

// FP64 FMA throughput probe: 8 independent fma chains per thread, iters
// steps each (2 * 8 * iters flops per thread); out[thread] keeps the result
// live.  Used to measure the DFMA peak that the roofline divides by.
__global__ void __launch_bounds__(256) fp64_fma_probe(double* out, int iters)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = 1.0 + 1e-9 * (t + k);
    const double b = 0.999999999, c = 1e-9;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    out[t] = s;
}

}  // namespace vlxb

extern "C" {

int vlxb_init(int device)
{
    if (cudaSetDevice(device) != cudaSuccess) return VLXB_ECUDA;
    int rc = vlxb::ensure_pool_configured();
    if (rc) return rc;
    if (!vlxb::quartet_counters_device()) return VLXB_ECUDA;
    return (vlxb::boys_table_device() && vlxb::boys_table32_device()) ? VLXB_OK : VLXB_ECUDA;
}

int vlxb_setFp32Cutoff(double cutoff) { return vlxb::fp32_cut_set(cutoff); }

double vlxb_getFp32Cutoff(void) { return vlxb::fp32_cut_get(); }

int vlxb_setFp32Budget(double budget) { return vlxb::fp32_budget_set(budget); }

double vlxb_getFp32Budget(void) { return vlxb::fp32_budget_get(); }

const char* vlxb_status_string(int status)
{
    switch (status) {
        case VLXB_OK: return "ok";
        case VLXB_EINVAL: return "invalid argument";
        case VLXB_ECUDA: return "CUDA runtime error";
        case VLXB_ENOMEM: return "device memory allocation failed";
        case VLXB_ETOOBIG: return "the call needs more scratch than the fixed no-allocation buffer holds";
        default: return "unknown status";
    }
}

int vlxb_version(void) { return 100; }

int vlxb_setSchedule(int kind, int la, int lb, int lc, int ld, int variant)
{
    return vlxb::schedule_set(kind, la, lb, lc, ld, variant);
}

int vlxb_getSchedule(int kind, int la, int lb, int lc, int ld)
{
    if (kind < 0 || kind > 1 || la < 0 || la > 2 || lb < 0 || lb > 2 || lc < 0 || lc > 2 || ld < 0 || ld > 2)
        return -VLXB_EINVAL;
    return vlxb::schedule_get(kind, la, lb, lc, ld);
}

int vlxb_launchCount(unsigned long long* out, int reset)
{
    if (!out) return VLXB_EINVAL;
    *out = vlxb::launch_count(reset != 0);
    return VLXB_OK;
}

int vlxb_fp64Probe(double* out, int iters, int blocks, void* stream)
{
    if (!out || iters <= 0 || blocks <= 0) return VLXB_EINVAL;
    vlxb::fp64_fma_probe<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters);
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

}  // extern "C"
