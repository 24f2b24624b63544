// Host-side engine pieces shared by all class translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>

#include "common.cuh"

namespace vlxb {

// Status codes returned through the C ABI.
enum Status : int {
    VLXB_OK = 0,
    VLXB_EINVAL = 1,   // invalid argument (null pointer, bad count or class)
    VLXB_ECUDA = 2,    // a CUDA runtime call failed
    VLXB_ENOMEM = 3,   // device allocation failed
    VLXB_ETOOBIG = 4,  // the call needs more scratch than a fixed buffer holds
};

#define VLXB_CHECK_CUDA(call)                              \
    do {                                                   \
        cudaError_t _e = (call);                           \
        if (_e != cudaSuccess) return (_e == cudaErrorMemoryAllocation) ? VLXB_ENOMEM : VLXB_ECUDA; \
    } while (0)

// Scratch arena of one call.  Pool mode (default): every buffer is taken
// from the device's default memory pool with cudaMallocAsync on the call's
// stream and handed back with cudaFreeAsync when the arena goes out of scope,
// so scratch is reused across calls without synchronisation.  Static mode:
// buffers are carved (256-byte aligned) out of a fixed device buffer given by
// the caller, nothing is allocated.  Measure mode: nothing is allocated or
// launched; alloc only adds up the bytes a static-mode call would need (the
// pointers it returns must not be used), and every launch site skips its
// launch (see VLXB_RUN).
class Arena {
  public:
    explicit Arena(cudaStream_t s) : stream_(s) {}
    Arena(cudaStream_t s, char* base, size_t cap, bool measure)
        : stream_(s), base_(base), cap_(cap), static_(true), measure_(measure) {}
    ~Arena()
    {
        for (void* p : ptrs_) cudaFreeAsync(p, stream_);
    }
    Arena(const Arena&) = delete;
    Arena& operator=(const Arena&) = delete;

    template <typename T>
    T* alloc(int64_t n)
    {
        if (failed_) return nullptr;
        size_t bytes = (size_t)(n > 0 ? n : 1) * sizeof(T);
        if (static_) {
            const size_t off = (used_ + 255) & ~(size_t)255;
            used_ = off + bytes;
            if (measure_) return (T*)(uintptr_t)(256 + off);  // placeholder, never dereferenced
            if (used_ > cap_) {
                failed_ = true;
                return nullptr;
            }
            return (T*)(base_ + off);
        }
        void* p = nullptr;
        if (cudaMallocAsync(&p, bytes, stream_) != cudaSuccess) {
            failed_ = true;
            cudaGetLastError();
            return nullptr;
        }
        ptrs_.push_back(p);
        return (T*)p;
    }
    bool failed() const { return failed_; }
    bool measuring() const { return measure_; }
    size_t used() const { return used_; }
    cudaStream_t stream() const { return stream_; }

  private:
    cudaStream_t stream_;
    std::vector<void*> ptrs_;
    char* base_ = nullptr;
    size_t cap_ = 0, used_ = 0;
    bool static_ = false, measure_ = false;
    bool failed_ = false;
};

// Launches, memsets and CUB runs go through VLXB_RUN so that a measuring
// arena only sizes the call.
#define VLXB_RUN(ar, ...)            \
    do {                             \
        if (!(ar).measuring()) {     \
            __VA_ARGS__;             \
        }                            \
    } while (0)

// Per-device FP64 Boys table (BOYS_NGRID x BOYS_NCOL), built on first use.
// Returns nullptr on failure.  The first call on a device synchronises it
// (table upload); call vlxb_init() before any stream capture.
const double* boys_table_device();

// Host copy of the FP64 Boys table (BOYS_NGRID x BOYS_NCOL values).
void boys_host_table(std::vector<double>& tab);

// Float copy of the same table for the mixed-precision path.
const float* boys_table32_device();

// Quartets whose screening bound is below this value are evaluated in FP32
// (0 = plain FP64, the default of the drop-in entry points).
double fp32_cut_get();
int fp32_cut_set(double cut);
// FP32 error budget (0 = none, the cutoff alone decides): among the quartets
// below the cutoff, only the tail of each bra's ket list (J) or of each
// (i, k) block's partner list per j (K) whose summed error proxy (bounds
// times hrr_amp on both pairs) stays within the budget runs in FP32.
double fp32_budget_get();
int fp32_budget_set(double budget);

// Per-device counters of screened-in primitive shell quartets processed by
// the J ([0]) and K ([1]) kernels (device memory, allocated with the table).
unsigned long long* quartet_counters_device();
// Per-device kernel error word (flags VLXB_KERR_*, OR-ed in by kernels whose
// bounded waits ran out); the word after the two counters.
unsigned long long* kernel_errors_device();

// Make the device's default memory pool keep freed scratch (release
// threshold = max) so per-call scratch costs no new cudaMalloc after warm-up.
int ensure_pool_configured();

// ---------------------------------------------------------------- prep API
struct PairGroups {
    int* spidx = nullptr;      // [npa * npb] exclusive scan of the occupancy table
    int* n_sp = nullptr;       // device count of shell pairs
    int64_t sp_stride = 0;     // allocation bound of shell-pair arrays
    int32_t* sp_i = nullptr;   // [sp_stride]
    int32_t* sp_j = nullptr;   // [sp_stride]
    int32_t* entry = nullptr;  // [NXY][sp_stride] caller list position or -1
    double* geo = nullptr;     // [GEO_N][sp_stride]
    int* n_rec = nullptr;      // device count of records
    int64_t rec_stride = 0;
    int32_t* rec_sp = nullptr;
    double* rec_q = nullptr;
    uint64_t* rec_mask = nullptr;
    int* seg = nullptr;        // [npa + 1] (segmented records only)
    double* S = nullptr;       // [NXY][sp_stride] (partner records only)
    double* su = nullptr;      // [rec_stride] uniform S of a record or NaN (partner records only)
    // contracted partner groups (contract_groups): members are the records in
    // group order; groups sorted by descending max member q inside segments
    int* gseg = nullptr;       // [npa + 1] group offsets by first primitive shell
    double* gq = nullptr;      // [rec_stride] max member q
    int32_t* gbeg = nullptr;   // [rec_stride] first member
    int32_t* gcnt = nullptr;   // [rec_stride] member count (1..KGROUP_MAX)
    int32_t* msp = nullptr;    // [rec_stride] member shell pair
    double* mq = nullptr;      // [rec_stride] member q
    double* msu = nullptr;     // [rec_stride] member uniform S or NaN (then alone in its group)
    uint64_t* mmask = nullptr; // [rec_stride] member component mask
    // FP32 error budget (budget_prefix_records; null when no budget is set):
    // per record / group the amplified bound, and its inclusive prefix sum
    double* rec_qa = nullptr;
    double* rec_qpre = nullptr;
    double* gqa = nullptr;
    double* gqpre = nullptr;
};

// Largest number of partner records summed before one HRR.
constexpr int KGROUP_MAX = 8;

// Group a flat list of prim-cart pairs (first[e], second[e]) by shell pair.
int group_flat(Arena& ar, int na, int nb, int npa, int npb, const uint32_t* first, const uint32_t* second,
               int64_t n, const double* info_a, uint32_t cnt_a, const double* info_b, uint32_t cnt_b,
               PairGroups& g);
// Group a CSR partner list (per prim-cart i: displs, counts, Dinds) by shell pair.
int group_csr(Arena& ar, int na, int nb, int npa, int npb, const uint32_t* displs, const uint32_t* counts,
              const uint32_t* Dinds, int64_t n_entries_bound, const double* info_a, uint32_t cnt_a,
              const double* info_b, uint32_t cnt_b, PairGroups& g);
// Split shell pairs into uniform-Q records (Q indexed by caller list position).
int make_records(Arena& ar, int nxy, PairGroups& g, const double* Q, int64_t n_entries);
// Sort records by descending q inside segments of the first primitive shell,
// and fill per-shell-pair S from the caller's pair data.
int segment_records(Arena& ar, int nxy, int npa, int npb, PairGroups& g, const double* pdata);
// Amplified bounds and their prefix sums for the FP32 budget (records, and
// groups when contract_groups ran); lh = angular momentum the pair's HRR moves.
int budget_prefix_records(Arena& ar, PairGroups& g, int npa, int lh);
// The same for the sorted J kets (tpre), lh = the ket's second angular momentum.
struct JKetData;
int budget_prefix_kets(Arena& ar, JKetData& kd, int lh);
// Group segmented partner records by the partner's contracted shell (same AO
// indices, part_aoinds = the partner type's prim_aoinds) for the contracted
// exchange kernels.
int contract_groups(Arena& ar, int npa, PairGroups& g, const uint32_t* part_aoinds, uint32_t naos);

struct JKetData {
    double *geo, *tmax, *tmin, *Dpp, *Dm, *Qc, *Dc;
    int64_t stride;
    int* n;
    int* seg = nullptr;  // [n_mol + 1] ket offsets per molecule (batched calls)
    double* Dh = nullptr;  // [stride][nherm(LC + LD)] Hermite ket density (McMurchie-Davidson kernel)
    double* tpre = nullptr;  // inclusive prefix sum of tmax * hrr_amp over the sorted kets (FP32 budget)
};
// prim_mol_c (batched calls, else null): molecule of every type-c primitive;
// the kets are then sorted by molecule, and by descending bound inside one.
template <int LC, int LD>
int jket_prepare(Arena& ar, const PairGroups& g, const uint32_t* first, const uint32_t* second,
                 const double* D, const double* Q, const double* pdata, JKetData& out,
                 const int32_t* prim_mol_c = nullptr, int n_mol = 0, bool hermite = false);
// Molecule of every bra record (batched Coulomb calls).
int bra_record_mol(Arena& ar, const PairGroups& g, const int32_t* prim_mol_a, int32_t** mol);

struct KOutData {
    int32_t *ish, *ksh, *idx;
    int64_t stride;
    int* n;
};
int kout_prepare(Arena& ar, int na, int nc, int npa, int npc, const uint32_t* pi, const uint32_t* pk, int64_t n,
                 KOutData& out);
// Per-block max |D| of a batched exchange call (molecule of the block's i).
int kout_block_maxd(Arena& ar, const KOutData& ko, const int32_t* prim_mol_a, const double* maxD_mol,
                    double** out);

int launch_grid_limit();

// Kernel variant per class: kind 0 = Coulomb (0 thread-per-quartet, 1 column),
// kind 1 = exchange (0 thread-per-quartet, 1 column with bra lanes, 2 column
// with ket lanes).  Defaults come from the generator; the autotuner
// overrides them through vlxb_setSchedule.
int schedule_get(int kind, int la, int lb, int lc, int ld);
int schedule_set(int kind, int la, int lb, int lc, int ld, int variant);

// Host-side count of this library's own kernel launches (CUB's are not
// counted); read and reset through vlxb_launchCount.
void note_launches(int n = 1);

}  // namespace vlxb
