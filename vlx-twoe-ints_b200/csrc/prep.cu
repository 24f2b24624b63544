// Host orchestration of the device-side list regrouping (see prep.cuh), the
// per-device Boys table and memory-pool set-up.
#include <cub/cub.cuh>
#include <math.h>

#include <atomic>
#include <mutex>

#include "common.cuh"
#include "engine.cuh"
#include "generated/hrr_pairs.cuh"
#include "prep.cuh"

namespace vlxb {

// ------------------------------------------------------------ Boys table
// F_m(T_k) for T_k = k*BOYS_H, m < BOYS_NCOL, from the convergent series
// F_m(T) = e^{-T} sum_{i>=0} (2T)^i / ((2m+1)(2m+3)...(2m+2i+1)) in long
// double, with downward recursion for the lower orders.
static void build_boys_host(std::vector<double>& tab)
{
    tab.assign((size_t)BOYS_NGRID * BOYS_NCOL, 0.0);
    const int M = BOYS_NCOL - 1;
    for (int k = 0; k < BOYS_NGRID; k++) {
        const long double T = (long double)k * (long double)BOYS_H;
        long double F[BOYS_NCOL];
        long double term = 1.0L / (2.0L * M + 1.0L), sum = term;
        for (int i = 1; i < 4000; i++) {
            term *= 2.0L * T / (2.0L * M + 2.0L * i + 1.0L);
            sum += term;
            if (i > T && term < 1e-25L * sum) break;
        }
        const long double ex = expl(-T);
        F[M] = ex * sum;
        for (int m = M - 1; m >= 0; m--) F[m] = (2.0L * T * F[m + 1] + ex) / (2.0L * m + 1.0L);
        for (int m = 0; m < BOYS_NCOL; m++) tab[(size_t)k * BOYS_NCOL + m] = (double)F[m];
    }
}

void boys_host_table(std::vector<double>& tab) { build_boys_host(tab); }

static std::mutex g_mu;
static const double* g_boys_dev[64] = {nullptr};
static const float* g_boys32_dev[64] = {nullptr};
static std::atomic<double> g_fp32_cut{0.0};
static std::atomic<double> g_fp32_budget{0.2};

double fp32_cut_get() { return g_fp32_cut.load(std::memory_order_relaxed); }

int fp32_cut_set(double cut)
{
    if (!(cut >= 0.0)) return VLXB_EINVAL;
    g_fp32_cut.store(cut);
    return VLXB_OK;
}

double fp32_budget_get() { return g_fp32_budget.load(std::memory_order_relaxed); }

int fp32_budget_set(double budget)
{
    if (!(budget >= 0.0)) return VLXB_EINVAL;
    g_fp32_budget.store(budget);
    return VLXB_OK;
}

const float* boys_table32_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (g_boys32_dev[dev]) return g_boys32_dev[dev];
    }
    std::vector<double> host;
    build_boys_host(host);
    std::vector<float> h32(host.begin(), host.end());
    float* d = nullptr;
    if (cudaMalloc(&d, h32.size() * sizeof(float)) != cudaSuccess) return nullptr;
    if (cudaMemcpy(d, h32.data(), h32.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_boys32_dev[dev]) {
        cudaFree(d);
        return g_boys32_dev[dev];
    }
    g_boys32_dev[dev] = d;
    return d;
}
static bool g_pool_done[64] = {false};
static unsigned long long* g_counters[64] = {nullptr};

unsigned long long* quartet_counters_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_counters[dev]) {
        unsigned long long* p = nullptr;
        if (cudaMalloc(&p, 4 * sizeof(unsigned long long)) != cudaSuccess) return nullptr;
        if (cudaMemset(p, 0, 4 * sizeof(unsigned long long)) != cudaSuccess) return nullptr;
        g_counters[dev] = p;
    }
    return g_counters[dev];
}

unsigned long long* kernel_errors_device()
{
    unsigned long long* p = quartet_counters_device();
    return p ? p + 2 : nullptr;
}

const double* boys_table_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_boys_dev[dev]) return g_boys_dev[dev];
    static std::vector<double> host;
    if (host.empty()) build_boys_host(host);
    double* d = nullptr;
    if (cudaMalloc(&d, host.size() * sizeof(double)) != cudaSuccess) return nullptr;
    if (cudaMemcpy(d, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return nullptr;
    }
    g_boys_dev[dev] = d;
    return d;
}

int ensure_pool_configured()
{
    int dev = 0;
    VLXB_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return VLXB_EINVAL;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_pool_done[dev]) return VLXB_OK;
    cudaMemPool_t pool;
    VLXB_CHECK_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t thr = UINT64_MAX;
    VLXB_CHECK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    g_pool_done[dev] = true;
    return VLXB_OK;
}

#include "generated/schedule_default.inc"

static std::atomic<int> g_sched[2][81];
static std::once_flag g_sched_once;

static void sched_init()
{
    for (int c = 0; c < 81; c++) {
        g_sched[0][c].store(kDefaultScheduleJ[c]);
        g_sched[1][c].store(kDefaultScheduleK[c]);
    }
}

int schedule_get(int kind, int la, int lb, int lc, int ld)
{
    std::call_once(g_sched_once, sched_init);
    return g_sched[kind & 1][la * 27 + lb * 9 + lc * 3 + ld].load(std::memory_order_relaxed);
}

int schedule_set(int kind, int la, int lb, int lc, int ld, int variant)
{
    if (kind < 0 || kind > 1 || la < 0 || la > 2 || lb < 0 || lb > 2 || lc < 0 || lc > 2 || ld < 0 || ld > 2)
        return VLXB_EINVAL;
    if (variant < 0 || variant > (kind == 0 ? 3 : 12)) return VLXB_EINVAL;
    std::call_once(g_sched_once, sched_init);
    g_sched[kind][la * 27 + lb * 9 + lc * 3 + ld].store(variant);
    return VLXB_OK;
}

static std::atomic<unsigned long long> g_launches{0};

void note_launches(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

unsigned long long launch_count(bool reset)
{
    return reset ? g_launches.exchange(0) : g_launches.load();
}

int launch_grid_limit()
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms * 16;
}

// ------------------------------------------------------------ helpers
static int scan_int(Arena& ar, const int* in, int* out, int64_t n)
{
    size_t bytes = 0;
    VLXB_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, ar.stream()));
    void* tmp = ar.alloc<char>((int64_t)bytes);
    if (!tmp) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, (int)n, ar.stream()));
    }
    return VLXB_OK;
}

static int inclusive_sum_f64(Arena& ar, const double* in, double* out, int64_t n)
{
    size_t bytes = 0;
    VLXB_CHECK_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out, (int)n, ar.stream()));
    void* tmp = ar.alloc<char>((int64_t)bytes);
    if (!tmp) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cub::DeviceScan::InclusiveSum(tmp, bytes, in, out, (int)n, ar.stream()));
    }
    return VLXB_OK;
}

static int finish_grouping(Arena& ar, int64_t ntab, int* table, PairGroups& g)
{
    cudaStream_t st = ar.stream();
    g.spidx = ar.alloc<int>(ntab);
    g.n_sp = ar.alloc<int>(1);
    if (!g.spidx || !g.n_sp) return VLXB_ENOMEM;
    int rc = scan_int(ar, table, g.spidx, ntab);
    if (rc) return rc;
    if (!ar.measuring()) {
        k_scan_total<<<1, 1, 0, st>>>(g.spidx, table, ntab, g.n_sp);
    }
    if (!ar.measuring()) note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

static int alloc_sp(Arena& ar, int nxy, PairGroups& g)
{
    g.sp_i = ar.alloc<int32_t>(g.sp_stride);
    g.sp_j = ar.alloc<int32_t>(g.sp_stride);
    g.entry = ar.alloc<int32_t>(g.sp_stride * nxy);
    g.geo = ar.alloc<double>(g.sp_stride * GEO_N);
    if (ar.failed()) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cudaMemsetAsync(g.entry, 0xFF, sizeof(int32_t) * g.sp_stride * nxy, ar.stream()));
    }
    return VLXB_OK;
}

int group_flat(Arena& ar, int na, int nb, int npa, int npb, const uint32_t* first, const uint32_t* second,
               int64_t n, const double* info_a, uint32_t cnt_a, const double* info_b, uint32_t cnt_b,
               PairGroups& g)
{
    cudaStream_t st = ar.stream();
    const int64_t ntab = (int64_t)npa * npb;
    int* table = ar.alloc<int>(ntab);
    if (!table) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cudaMemsetAsync(table, 0, sizeof(int) * ntab, st));
    }
    if (!ar.measuring()) {
        k_mark_pairs<<<prep_blocks(n), PREP_THREADS, 0, st>>>(first, second, n, na, nb, npb, table);
    }
    if (!ar.measuring()) note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    int rc = finish_grouping(ar, ntab, table, g);
    if (rc) return rc;
    g.sp_stride = n < ntab ? n : ntab;
    rc = alloc_sp(ar, na * nb, g);
    if (rc) return rc;
    if (!ar.measuring()) {
        k_fill_pairs<<<prep_blocks(n), PREP_THREADS, 0, st>>>(first, second, n, na, nb, npb, g.spidx, g.entry, g.sp_i,
                                                              g.sp_j, g.sp_stride);
    }
    if (!ar.measuring()) note_launches();
    if (!ar.measuring()) {
        k_pair_geo<<<prep_blocks(g.sp_stride), PREP_THREADS, 0, st>>>(g.n_sp, g.sp_i, g.sp_j, info_a, cnt_a, info_b,
                                                                       cnt_b, g.geo, g.sp_stride);
    }
    if (!ar.measuring()) note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

int group_csr(Arena& ar, int na, int nb, int npa, int npb, const uint32_t* displs, const uint32_t* counts,
              const uint32_t* Dinds, int64_t n_entries_bound, const double* info_a, uint32_t cnt_a,
              const double* info_b, uint32_t cnt_b, PairGroups& g)
{
    cudaStream_t st = ar.stream();
    const int64_t ntab = (int64_t)npa * npb;
    const int n_first = npa * na;
    int* table = ar.alloc<int>(ntab);
    if (!table) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cudaMemsetAsync(table, 0, sizeof(int) * ntab, st));
    }
    if (!ar.measuring()) {
        k_mark_csr<<<prep_blocks(n_first), PREP_THREADS, 0, st>>>(displs, counts, Dinds, n_first, na, nb, npb, table);
    }
    if (!ar.measuring()) note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    int rc = finish_grouping(ar, ntab, table, g);
    if (rc) return rc;
    g.sp_stride = n_entries_bound < ntab ? n_entries_bound : ntab;
    rc = alloc_sp(ar, na * nb, g);
    if (rc) return rc;
    if (!ar.measuring()) {
        k_fill_csr<<<prep_blocks(n_first), PREP_THREADS, 0, st>>>(displs, counts, Dinds, n_first, na, nb, npb, g.spidx,
                                                                  g.entry, g.sp_i, g.sp_j, g.sp_stride);
    }
    if (!ar.measuring()) note_launches();
    if (!ar.measuring()) {
        k_pair_geo<<<prep_blocks(g.sp_stride), PREP_THREADS, 0, st>>>(g.n_sp, g.sp_i, g.sp_j, info_a, cnt_a, info_b,
                                                                       cnt_b, g.geo, g.sp_stride);
    }
    if (!ar.measuring()) note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

template <int NXY>
static void launch_rec_count(const PairGroups& g, const double* Q, int* nrec, cudaStream_t st)
{
    {
        k_rec_count<NXY><<<prep_blocks(g.sp_stride), PREP_THREADS, 0, st>>>(g.n_sp, g.entry, g.sp_stride, Q, nrec);
    }
    note_launches();
}
template <int NXY>
static void launch_rec_fill(const PairGroups& g, const double* Q, const int* recoff, cudaStream_t st)
{
    {
        k_rec_fill<NXY><<<prep_blocks(g.sp_stride), PREP_THREADS, 0, st>>>(g.n_sp, g.entry, g.sp_stride, Q, recoff,
                                                                           g.rec_sp, g.rec_q, g.rec_mask);
    }
    note_launches();
}
template <int NXY>
static void launch_sp_S(const PairGroups& g, const double* pdata, cudaStream_t st)
{
    {
        k_sp_S<NXY><<<prep_blocks(g.sp_stride), PREP_THREADS, 0, st>>>(g.n_sp, g.entry, g.sp_stride, pdata, g.S);
    }
    note_launches();
    {
        k_rec_uniform_s<NXY><<<prep_blocks(g.rec_stride), PREP_THREADS, 0, st>>>(g.n_rec, g.rec_sp, g.rec_mask, g.S,
                                                                                 g.sp_stride, g.su);
    }
    note_launches();
}

#define VLXB_NXY_DISPATCH(nxy, FN, ...)            \
    switch (nxy) {                                 \
        case 1: FN<1>(__VA_ARGS__); break;         \
        case 3: FN<3>(__VA_ARGS__); break;         \
        case 6: FN<6>(__VA_ARGS__); break;         \
        case 9: FN<9>(__VA_ARGS__); break;         \
        case 18: FN<18>(__VA_ARGS__); break;       \
        case 36: FN<36>(__VA_ARGS__); break;       \
        default: return VLXB_EINVAL;               \
    }

int make_records(Arena& ar, int nxy, PairGroups& g, const double* Q, int64_t n_entries)
{
    cudaStream_t st = ar.stream();
    int64_t bound = g.sp_stride * nxy;
    g.rec_stride = bound < n_entries ? bound : n_entries;
    if (g.rec_stride < g.sp_stride) g.rec_stride = g.sp_stride;
    int* nrec = ar.alloc<int>(g.sp_stride + 1);
    int* recoff = ar.alloc<int>(g.sp_stride + 1);
    g.n_rec = ar.alloc<int>(1);
    g.rec_sp = ar.alloc<int32_t>(g.rec_stride);
    g.rec_q = ar.alloc<double>(g.rec_stride);
    g.rec_mask = ar.alloc<uint64_t>(g.rec_stride);
    if (ar.failed()) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cudaMemsetAsync(nrec, 0, sizeof(int) * (g.sp_stride + 1), st));
    }
    if (!ar.measuring()) {
        VLXB_NXY_DISPATCH(nxy, launch_rec_count, g, Q, nrec, st);
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    int rc = scan_int(ar, nrec, recoff, g.sp_stride + 1);
    if (rc) return rc;
    if (!ar.measuring()) {
        k_scan_total<<<1, 1, 0, st>>>(recoff, nrec, g.sp_stride + 1, g.n_rec);
    }
    if (!ar.measuring()) note_launches();
    if (!ar.measuring()) {
        VLXB_NXY_DISPATCH(nxy, launch_rec_fill, g, Q, recoff, st);
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    // keep recoff for segment offsets
    g.seg = recoff;  // temporarily: record offsets per shell pair
    return VLXB_OK;
}

int segment_records(Arena& ar, int nxy, int npa, int npb, PairGroups& g, const double* pdata)
{
    cudaStream_t st = ar.stream();
    const int* recoff = g.seg;
    int* seg = ar.alloc<int>(npa + 1);
    double* q_sorted = ar.alloc<double>(g.rec_stride);
    int* perm_in = ar.alloc<int>(g.rec_stride);
    int* perm = ar.alloc<int>(g.rec_stride);
    int32_t* sp_sorted = ar.alloc<int32_t>(g.rec_stride);
    uint64_t* mask_sorted = ar.alloc<uint64_t>(g.rec_stride);
    g.S = ar.alloc<double>(g.sp_stride * nxy);
    g.su = ar.alloc<double>(g.rec_stride);
    if (ar.failed()) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        k_rec_segments<<<prep_blocks(npa + 1), PREP_THREADS, 0, st>>>(g.spidx, recoff, npa, npb, g.n_rec, seg);
    }
    if (!ar.measuring()) note_launches();
    if (!ar.measuring()) {
        k_iota<<<prep_blocks(g.rec_stride), PREP_THREADS, 0, st>>>(perm_in, g.rec_stride);
    }
    if (!ar.measuring()) note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    size_t bytes = 0;
    VLXB_CHECK_CUDA(cub::DeviceSegmentedRadixSort::SortPairsDescending(
        nullptr, bytes, g.rec_q, q_sorted, perm_in, perm, (int)g.rec_stride, npa, seg, seg + 1, 0, 64, st));
    void* tmp = ar.alloc<char>((int64_t)bytes);
    if (!tmp) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cub::DeviceSegmentedRadixSort::SortPairsDescending(
            tmp, bytes, g.rec_q, q_sorted, perm_in, perm, (int)g.rec_stride, npa, seg, seg + 1, 0, 64, st));
    }
    if (!ar.measuring()) {
        k_gather_recs<<<prep_blocks(g.rec_stride), PREP_THREADS, 0, st>>>(g.n_rec, perm, g.rec_sp, g.rec_mask,
                                                                           sp_sorted, mask_sorted);
    }
    if (!ar.measuring()) note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    g.rec_q = q_sorted;
    g.rec_sp = sp_sorted;
    g.rec_mask = mask_sorted;
    g.seg = seg;
    if (!ar.measuring()) {
        VLXB_NXY_DISPATCH(nxy, launch_sp_S, g, pdata, st);
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

struct MaxOp {
    __device__ __forceinline__ int operator()(int a, int b) const { return a > b ? a : b; }
};

int contract_groups(Arena& ar, int npa, PairGroups& g, const uint32_t* part_aoinds, uint32_t naos)
{
    cudaStream_t st = ar.stream();
    const int64_t R = g.rec_stride;
    uint32_t* key = ar.alloc<uint32_t>(R);
    uint32_t* key_sorted = ar.alloc<uint32_t>(R);
    int* perm_in = ar.alloc<int>(R);
    int* perm = ar.alloc<int>(R);
    int* segflag = ar.alloc<int>(R + 1);
    int* runstart = ar.alloc<int>(R);
    int* runmax = ar.alloc<int>(R);
    int* head = ar.alloc<int>(R + 1);
    int* gid = ar.alloc<int>(R + 1);
    int32_t* gbeg0 = ar.alloc<int32_t>(R);
    double* gq0 = ar.alloc<double>(R);
    int* gperm_in = ar.alloc<int>(R);
    int* gperm = ar.alloc<int>(R);
    g.gseg = ar.alloc<int>(npa + 1);
    g.gq = ar.alloc<double>(R);
    g.gbeg = ar.alloc<int32_t>(R);
    g.gcnt = ar.alloc<int32_t>(R);
    g.msp = ar.alloc<int32_t>(R);
    g.mq = ar.alloc<double>(R);
    g.msu = ar.alloc<double>(R);
    g.mmask = ar.alloc<uint64_t>(R);
    if (ar.failed()) return VLXB_ENOMEM;
    const int nb = prep_blocks(R);
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cudaMemsetAsync(segflag, 0, sizeof(int) * (R + 1), st));
        VLXB_CHECK_CUDA(cudaMemsetAsync(head, 0, sizeof(int) * (R + 1), st));
        k_grp_key<<<nb, PREP_THREADS, 0, st>>>(g.n_rec, g.rec_sp, g.su, g.sp_j, part_aoinds, naos, key);
        k_iota<<<nb, PREP_THREADS, 0, st>>>(perm_in, R);
        k_seg_starts<<<prep_blocks(npa), PREP_THREADS, 0, st>>>(g.seg, npa, segflag);
        note_launches(3);
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    // stable key sort inside each first-shell segment (keeps descending q within a key)
    size_t bytes = 0;
    VLXB_CHECK_CUDA(cub::DeviceSegmentedRadixSort::SortPairs(nullptr, bytes, key, key_sorted, perm_in, perm, (int)R,
                                                             npa, g.seg, g.seg + 1, 0, 32, st));
    void* tmp = ar.alloc<char>((int64_t)bytes);
    if (!tmp) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cub::DeviceSegmentedRadixSort::SortPairs(tmp, bytes, key, key_sorted, perm_in, perm, (int)R,
                                                                 npa, g.seg, g.seg + 1, 0, 32, st));
        k_grp_runs<<<nb, PREP_THREADS, 0, st>>>(g.n_rec, segflag, key_sorted, runstart);
        note_launches();
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    bytes = 0;
    VLXB_CHECK_CUDA(cub::DeviceScan::InclusiveScan(nullptr, bytes, runstart, runmax, MaxOp(), (int)R, st));
    tmp = ar.alloc<char>((int64_t)bytes);
    if (!tmp) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cub::DeviceScan::InclusiveScan(tmp, bytes, runstart, runmax, MaxOp(), (int)R, st));
        k_grp_heads<<<nb, PREP_THREADS, 0, st>>>(g.n_rec, runmax, KGROUP_MAX, head);
        note_launches();
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    int rc = scan_int(ar, head, gid, R + 1);
    if (rc) return rc;
    if (!ar.measuring()) {
        k_grp_fill<<<nb, PREP_THREADS, 0, st>>>(g.n_rec, perm, head, gid, g.rec_sp, g.rec_q, g.su, g.rec_mask, g.msp,
                                                g.mq, g.msu, g.mmask, gbeg0, gq0);
        k_grp_seg<<<prep_blocks(npa + 1), PREP_THREADS, 0, st>>>(g.seg, npa, gid, g.gseg);
        k_iota<<<nb, PREP_THREADS, 0, st>>>(gperm_in, R);
        note_launches(3);
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    // groups by descending max q inside each segment
    bytes = 0;
    VLXB_CHECK_CUDA(cub::DeviceSegmentedRadixSort::SortPairsDescending(nullptr, bytes, gq0, g.gq, gperm_in, gperm,
                                                                       (int)R, npa, g.gseg, g.gseg + 1, 0, 64, st));
    tmp = ar.alloc<char>((int64_t)bytes);
    if (!tmp) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cub::DeviceSegmentedRadixSort::SortPairsDescending(
            tmp, bytes, gq0, g.gq, gperm_in, gperm, (int)R, npa, g.gseg, g.gseg + 1, 0, 64, st));
        k_grp_order<<<nb, PREP_THREADS, 0, st>>>(g.gseg + npa, g.n_rec, gperm, gbeg0, g.gbeg, g.gcnt);
        note_launches();
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

template <int LC, int LD>
int jket_prepare(Arena& ar, const PairGroups& g, const uint32_t* first, const uint32_t* second,
                 const double* D, const double* Q, const double* pdata, JKetData& out,
                 const int32_t* prim_mol_c, int n_mol, bool hermite)
{
    constexpr int NCD = ncart(LC) * ncart(LD), NF = nrange(LC, LD);
    cudaStream_t st = ar.stream();
    const int64_t S = g.sp_stride;
    double* keys = ar.alloc<double>(S);
    double* keys_sorted = ar.alloc<double>(S);
    int* perm_in = ar.alloc<int>(S);
    int* perm = ar.alloc<int>(S);
    double* tmin_u = ar.alloc<double>(S);
    double* Dpp_u = ar.alloc<double>(S * NF);
    double* Dm_u = ar.alloc<double>(S * NCD);
    double* Qc_u = ar.alloc<double>(S * NCD);
    double* Dc_u = ar.alloc<double>(S * NCD);
    // the sorted ket arrays get an even row stride, so that every row of
    // them starts on a 16-byte boundary (bulk copies into shared memory)
    const int64_t SA = (S + 1) & ~(int64_t)1;
    out.geo = ar.alloc<double>(SA * GEO_N);
    out.tmin = ar.alloc<double>(SA);
    out.tmax = ar.alloc<double>(SA);
    out.Dpp = ar.alloc<double>(SA * NF);
    out.Dm = ar.alloc<double>(SA * NCD);
    out.Qc = ar.alloc<double>(SA * NCD);
    out.Dc = ar.alloc<double>(SA * NCD);
    if (ar.failed()) return VLXB_ENOMEM;
    out.stride = SA;
    out.n = g.n_sp;
    if (!ar.measuring()) {
        k_jket_fill<LC, LD><<<prep_blocks(S), PREP_THREADS, 0, st>>>(g.n_sp, g.entry, S, first, second, D, Q, pdata,
                                                                     g.geo, keys, tmin_u, Dpp_u, Dm_u, Qc_u, Dc_u, S);
    }
    if (!ar.measuring()) note_launches();
    if (!ar.measuring()) {
        k_iota<<<prep_blocks(S), PREP_THREADS, 0, st>>>(perm_in, S);
    }
    if (!ar.measuring()) note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    size_t bytes = 0;
    VLXB_CHECK_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, keys, keys_sorted, perm_in, perm,
                                                              (int)S, 0, 64, st));
    void* tmp = ar.alloc<char>((int64_t)bytes);
    if (!tmp) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp, bytes, keys, keys_sorted, perm_in, perm, (int)S,
                                                                  0, 64, st));
    }
    if (prim_mol_c) {
        // stable second sort by molecule: per molecule, descending bound
        int* molkey = ar.alloc<int>(S);
        int* molkey_sorted = ar.alloc<int>(S);
        int* perm2 = ar.alloc<int>(S);
        int* perm_c = ar.alloc<int>(S);
        double* keys_c = ar.alloc<double>(S);
        out.seg = ar.alloc<int>(n_mol + 1);
        if (ar.failed()) return VLXB_ENOMEM;
        int bits = 1;
        while ((1 << bits) <= n_mol) bits++;
        size_t b2 = 0;
        VLXB_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b2, molkey, molkey_sorted, perm_in, perm2, (int)S, 0,
                                                        bits, st));
        void* tmp2 = ar.alloc<char>((int64_t)b2);
        if (!tmp2) return VLXB_ENOMEM;
        if (!ar.measuring()) {
            k_jket_molkey<<<prep_blocks(S), PREP_THREADS, 0, st>>>(g.n_sp, S, perm, g.sp_i, prim_mol_c, n_mol, molkey);
            VLXB_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(tmp2, b2, molkey, molkey_sorted, perm_in, perm2, (int)S,
                                                            0, bits, st));
            k_compose_perm<<<prep_blocks(S), PREP_THREADS, 0, st>>>(g.n_sp, perm, perm2, keys_sorted, perm_c, keys_c);
            k_mol_segments<<<prep_blocks(n_mol + 1), PREP_THREADS, 0, st>>>(g.n_sp, molkey_sorted, n_mol, out.seg);
            note_launches(3);
        }
        VLXB_CHECK_CUDA(cudaGetLastError());
        perm = perm_c;
        keys_sorted = keys_c;
    }
    if (!ar.measuring()) {
        k_jket_gather<LC, LD><<<prep_blocks(S), PREP_THREADS, 0, st>>>(g.n_sp, perm, S, SA, g.geo, keys_sorted, tmin_u,
                                                                       Dpp_u, Dm_u, Qc_u, Dc_u, out.geo, out.tmax,
                                                                       out.tmin, out.Dpp, out.Dm, out.Qc, out.Dc);
    }
    if (!ar.measuring()) note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    if (hermite) {
        out.Dh = ar.alloc<double>(SA * nherm(LC + LD));
        if (!out.Dh) return VLXB_ENOMEM;
        if (!ar.measuring()) {
            k_jket_hermite<LC, LD><<<prep_blocks(S), PREP_THREADS, 0, st>>>(g.n_sp, SA, out.geo, out.Dm, out.Dh);
            note_launches();
        }
        VLXB_CHECK_CUDA(cudaGetLastError());
    }
    return VLXB_OK;
}

template int jket_prepare<0, 0>(Arena&, const PairGroups&, const uint32_t*, const uint32_t*, const double*,
                                const double*, const double*, JKetData&, const int32_t*, int, bool);
template int jket_prepare<0, 1>(Arena&, const PairGroups&, const uint32_t*, const uint32_t*, const double*,
                                const double*, const double*, JKetData&, const int32_t*, int, bool);
template int jket_prepare<0, 2>(Arena&, const PairGroups&, const uint32_t*, const uint32_t*, const double*,
                                const double*, const double*, JKetData&, const int32_t*, int, bool);
template int jket_prepare<1, 1>(Arena&, const PairGroups&, const uint32_t*, const uint32_t*, const double*,
                                const double*, const double*, JKetData&, const int32_t*, int, bool);
template int jket_prepare<1, 2>(Arena&, const PairGroups&, const uint32_t*, const uint32_t*, const double*,
                                const double*, const double*, JKetData&, const int32_t*, int, bool);
template int jket_prepare<2, 2>(Arena&, const PairGroups&, const uint32_t*, const uint32_t*, const double*,
                                const double*, const double*, JKetData&, const int32_t*, int, bool);

template <int NAC>
static void launch_kout(const uint32_t* pi, const uint32_t* pk, int64_t n, int na, int nc, int npc, const int* spidx,
                        KOutData& out, cudaStream_t st)
{
    {
        k_kout_fill<NAC><<<prep_blocks(n), PREP_THREADS, 0, st>>>(pi, pk, n, na, nc, npc, spidx, out.idx, out.ish,
                                                                  out.ksh, out.stride);
    }
    note_launches();
}

int bra_record_mol(Arena& ar, const PairGroups& g, const int32_t* prim_mol_a, int32_t** mol)
{
    *mol = ar.alloc<int32_t>(g.rec_stride);
    if (!*mol) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        k_rec_mol<<<prep_blocks(g.rec_stride), PREP_THREADS, 0, ar.stream()>>>(g.n_rec, g.rec_sp, g.sp_i, prim_mol_a,
                                                                                *mol);
        note_launches();
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

int kout_block_maxd(Arena& ar, const KOutData& ko, const int32_t* prim_mol_a, const double* maxD_mol,
                    double** out)
{
    *out = ar.alloc<double>(ko.stride);
    if (!*out) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        k_kout_maxd<<<prep_blocks(ko.stride), PREP_THREADS, 0, ar.stream()>>>(ko.n, ko.ish, prim_mol_a, maxD_mol,
                                                                               *out);
        note_launches();
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

int kout_prepare(Arena& ar, int na, int nc, int npa, int npc, const uint32_t* pi, const uint32_t* pk, int64_t n,
                 KOutData& out)
{
    cudaStream_t st = ar.stream();
    const int64_t ntab = (int64_t)npa * npc;
    int* table = ar.alloc<int>(ntab);
    if (!table) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cudaMemsetAsync(table, 0, sizeof(int) * ntab, st));
    }
    if (!ar.measuring()) {
        k_mark_pairs<<<prep_blocks(n), PREP_THREADS, 0, st>>>(pi, pk, n, na, nc, npc, table);
    }
    if (!ar.measuring()) note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    PairGroups g;
    int rc = finish_grouping(ar, ntab, table, g);
    if (rc) return rc;
    out.stride = n < ntab ? n : ntab;
    out.n = g.n_sp;
    out.ish = ar.alloc<int32_t>(out.stride);
    out.ksh = ar.alloc<int32_t>(out.stride);
    out.idx = ar.alloc<int32_t>(out.stride * na * nc);
    if (ar.failed()) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        VLXB_CHECK_CUDA(cudaMemsetAsync(out.idx, 0xFF, sizeof(int32_t) * out.stride * na * nc, st));
    }
    if (!ar.measuring()) {
        VLXB_NXY_DISPATCH(na * nc, launch_kout, pi, pk, n, na, nc, npc, g.spidx, out, st);
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

}  // namespace vlxb

namespace vlxb {

int budget_prefix_records(Arena& ar, PairGroups& g, int npa, int lh)
{
    cudaStream_t st = ar.stream();
    g.rec_qa = ar.alloc<double>(g.rec_stride);
    g.rec_qpre = ar.alloc<double>(g.rec_stride);
    if (ar.failed()) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        k_rec_amp<<<prep_blocks(g.rec_stride), PREP_THREADS, 0, st>>>(g.n_rec, g.rec_stride, g.rec_sp, g.rec_q,
                                                                       g.geo, g.sp_stride, lh, g.rec_qa);
        note_launches();
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    int rc = inclusive_sum_f64(ar, g.rec_qa, g.rec_qpre, g.rec_stride);
    if (rc) return rc;
    if (g.gq) {
        g.gqa = ar.alloc<double>(g.rec_stride);
        g.gqpre = ar.alloc<double>(g.rec_stride);
        if (ar.failed()) return VLXB_ENOMEM;
        if (!ar.measuring()) {
            k_grp_amp<<<prep_blocks(g.rec_stride), PREP_THREADS, 0, st>>>(g.gseg + npa, g.rec_stride, g.gbeg, g.gcnt,
                                                                           g.msp, g.mq, g.geo, g.sp_stride, lh,
                                                                           g.gqa);
            note_launches();
        }
        VLXB_CHECK_CUDA(cudaGetLastError());
        rc = inclusive_sum_f64(ar, g.gqa, g.gqpre, g.rec_stride);
        if (rc) return rc;
    }
    return VLXB_OK;
}

int budget_prefix_kets(Arena& ar, JKetData& kd, int lh)
{
    cudaStream_t st = ar.stream();
    double* amp = ar.alloc<double>(kd.stride);
    kd.tpre = ar.alloc<double>(kd.stride);
    if (ar.failed()) return VLXB_ENOMEM;
    if (!ar.measuring()) {
        k_jket_amp<<<prep_blocks(kd.stride), PREP_THREADS, 0, st>>>(kd.n, kd.stride, kd.tmax, kd.geo, lh, amp);
        note_launches();
    }
    VLXB_CHECK_CUDA(cudaGetLastError());
    return inclusive_sum_f64(ar, amp, kd.tpre, kd.stride);
}

}  // namespace vlxb
