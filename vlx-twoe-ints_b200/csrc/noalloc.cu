// An allocation-free variant of the SSSS Coulomb entry point.
//
// Some callers cannot allocate device memory: hosts whose device memory is
// fully reserved by their own allocator, plugins that are not allowed to
// allocate, loops that must never wait on an allocator.  For them this entry
// point takes its scratch from a fixed array in the library's device memory
// instead of the stream-ordered pool the other entry points use, and its Boys
// tables from fixed arrays too, so no call allocates anything.
//
//  * Limit: VLXB_NOALLOC_SCRATCH_BYTES (64 MiB) of scratch per call; a call
//    that needs more is rejected with VLXB_ETOOBIG before any work is queued.
//    The array lives in every GPU that loads the library until process exit.
//  * The first call on a device resolves the arrays' device addresses
//    (cudaGetSymbolAddress) and uploads the Boys tables (cudaMemcpyToSymbol,
//    synchronous); make that first call before any stream capture.
//  * All calls share the array and it keeps the last call's contents; every
//    buffer that must start at zero is cleared by the call itself.  Calls that
//    overlap on the GPU (different streams, or different host threads) race on
//    the array: serialise them.
//  * The per-device quartet counters of the other entry points are allocated
//    on first use, so this path never touches them: its quartets are not
//    counted (the kernels get a null counter pointer).
#include <mutex>
#include <vector>

#include "common.cuh"
#include "generated/q_ssss.cuh"
#include "generated/hrr_pairs.cuh"
#include "col_kernels.cuh"
#include "generated/col_ssss.cuh"
#include "classes.cuh"
#include "../../include/vlxb.h"

namespace vlxb {

constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)VLXB_NOALLOC_SCRATCH_BYTES;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) double g_noalloc_boys64[BOYS_NGRID * BOYS_NCOL];
static __device__ __align__(256) float g_noalloc_boys32[BOYS_NGRID * BOYS_NCOL];

struct NoAllocDevice {
    char* scratch = nullptr;
    const double* boys64 = nullptr;
    const float* boys32 = nullptr;
};

static std::mutex g_noalloc_mu;
static NoAllocDevice g_noalloc_dev[64];

// Per-device set-up, run on the first call with that device current.
static int noalloc_setup(NoAllocDevice& out)
{
    int dev = 0;
    VLXB_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return VLXB_EINVAL;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (!d.scratch) {
        void* p = nullptr;
        void* b64 = nullptr;
        void* b32 = nullptr;
        VLXB_CHECK_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        VLXB_CHECK_CUDA(cudaGetSymbolAddress(&b64, g_noalloc_boys64));
        VLXB_CHECK_CUDA(cudaGetSymbolAddress(&b32, g_noalloc_boys32));
        std::vector<double> host;
        boys_host_table(host);
        std::vector<float> host32(host.begin(), host.end());
        VLXB_CHECK_CUDA(cudaMemcpyToSymbol(g_noalloc_boys64, host.data(), host.size() * sizeof(double)));
        VLXB_CHECK_CUDA(cudaMemcpyToSymbol(g_noalloc_boys32, host32.data(), host32.size() * sizeof(float)));
        d.boys64 = (const double*)b64;
        d.boys32 = (const float*)b32;
        d.scratch = (char*)p;
    }
    out = d;
    return VLXB_OK;
}

}  // namespace vlxb

extern "C" int vlxb_computeCoulombFockSSSS_noalloc(
    double* mat_J, const double* s_prim_info, uint32_t s_prim_count, const double* ss_mat_D,
    const double* ss_mat_Q_local, const double* ss_mat_Q, const uint32_t* ss_first_inds_local,
    const uint32_t* ss_second_inds_local, const double* ss_pair_data_local, uint32_t ss_prim_pair_count_local,
    const uint32_t* ss_first_inds, const uint32_t* ss_second_inds, const double* ss_pair_data,
    uint32_t ss_prim_pair_count, const double* boys_func_table, const double* boys_func_ft, double eri_threshold,
    void* stream)
{
    using namespace vlxb;
    (void)boys_func_table;
    (void)boys_func_ft;
    CoulombArgs A{};
    A.mat_J = mat_J;
    A.info[0] = s_prim_info;
    A.count[0] = s_prim_count;
    A.cd_D = ss_mat_D;
    A.ab_Q = ss_mat_Q_local;
    A.cd_Q = ss_mat_Q;
    A.ab_first = ss_first_inds_local;
    A.ab_second = ss_second_inds_local;
    A.ab_pdata = ss_pair_data_local;
    A.n_ab = ss_prim_pair_count_local;
    A.cd_first = ss_first_inds;
    A.cd_second = ss_second_inds;
    A.cd_pdata = ss_pair_data;
    A.n_cd = ss_prim_pair_count;
    A.thr = eri_threshold;
    if (A.n_ab == 0 || A.n_cd == 0) return VLXB_OK;
    NoAllocDevice d;
    int rc = noalloc_setup(d);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const BoysTabs tab{d.boys64, d.boys32};
    const double cut = fp32_cut_get();
    {
        // size the call first: nothing is launched or allocated
        Arena probe(st, nullptr, NOALLOC_SCRATCH_BYTES, true);
        rc = run_coulomb_impl<0, 0, 0, 0>(A, st, probe, tab, nullptr, cut);
        if (rc) return rc;
        if (probe.used() > NOALLOC_SCRATCH_BYTES) return VLXB_ETOOBIG;
    }
    Arena ar(st, d.scratch, NOALLOC_SCRATCH_BYTES, false);
    return run_coulomb_impl<0, 0, 0, 0>(A, st, ar, tab, nullptr, cut);
}
