// Primitive-pair -> AO contraction of J and K, and the SCF energy, on the device.
//
// The class entry points leave mat_J / mat_K in primitive Cartesian pair space,
// one value per entry of the caller's J pair lists and K (i, k) lists, as the
// reference's kernels do (gen_coulomb.py:296 `mat_J[ij] += ...`,
// gen_exchange.py:341 `mat_K[ik] += ...`); the caller then adds those values
// into symmetric AO matrices.  This file does that step on the GPU so that an
// SCF loop keeps J, K and D resident and reads back only the energy.
//
// AO map (built once per list set by the host, resident across iterations):
//   rows r = 0..n_rows-1, one per AO pair (a, b) with a <= b that receives
//   anything; row_ao[r] = a * naos + b;
//   rowptr[r]..rowptr[r+1]-1 index src[], src[t] = position of a pair value
//   in the flat value array (bits 0..30) and a weight flag (bit 31: weight 2,
//   else 1).  The list values are the upper triangle of a symmetric matrix:
//   the AO value is M + M^T, so a value on an AO diagonal counts twice unless
//   it is a diagonal entry of a same-type list (the reference halves those).
//   M[a][b] = M[b][a] = sum over the row in stored order: a fixed order, so
//   the result is bit-reproducible run to run.
#include "engine.cuh"
#include "../../include/vlxb.h"

namespace vlxb {

__global__ void __launch_bounds__(256)
pairs_to_ao_kernel(const double* __restrict__ vals, const int64_t* __restrict__ rowptr,
                   const int32_t* __restrict__ row_ao, const uint32_t* __restrict__ src, int64_t n_rows,
                   double* __restrict__ out, int32_t naos)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t0 = __ldg(rowptr + r), t1 = __ldg(rowptr + r + 1);
        double s = 0.0;
        for (int64_t t = t0; t < t1; t++) {
            const uint32_t e = __ldg(src + t);
            const double v = __ldg(vals + (e & 0x7fffffffu));
            s += (e >> 31) ? 2.0 * v : v;
        }
        const int32_t ab = __ldg(row_ao + r);
        const int32_t a = ab / naos, b = ab % naos;
        out[(int64_t)a * naos + b] = s;
        out[(int64_t)b * naos + a] = s;
    }
}

constexpr int EN_THREADS = 256;
constexpr int EN_BLOCKS = 148 * 4;

// Block-level fixed-order sum of three values into part[3][block].
__device__ __forceinline__ void block_sum3(double v0, double v1, double v2, double* part)
{
    __shared__ double red[3][EN_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v0 = warp_sum(v0);
    v1 = warp_sum(v1);
    v2 = warp_sum(v2);
    if (lane == 0) {
        red[0][warp] = v0;
        red[1][warp] = v1;
        red[2][warp] = v2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int w = 0; w < EN_THREADS / 32; w++) s += red[threadIdx.x][w];
        part[threadIdx.x * gridDim.x + blockIdx.x] = s;
    }
}

// part[0..2][block] = partial sums of D.J, D.K over the block's grid-stride
// share of the naos^2 elements (J or K may be null).
__global__ void __launch_bounds__(EN_THREADS)
energy_partial_kernel(const double* __restrict__ D, const double* __restrict__ J, const double* __restrict__ K,
                      int64_t n, double* __restrict__ part)
{
    double dj = 0.0, dk = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)EN_THREADS + threadIdx.x; t < n; t += (int64_t)gridDim.x * EN_THREADS) {
        const double d = __ldg(D + t);
        if (J) dj = fma(d, __ldg(J + t), dj);
        if (K) dk = fma(d, __ldg(K + t), dk);
    }
    block_sum3(dj, dk, 0.0, part);
}

// out[0] = Tr[D J] - Tr[D K] / 2, out[1] = Tr[D J], out[2] = Tr[D K].
__global__ void __launch_bounds__(EN_THREADS)
energy_final_kernel(const double* __restrict__ part, int nblk, double* __restrict__ out)
{
    __shared__ double red[2][EN_THREADS];
    double dj = 0.0, dk = 0.0;
    for (int b = threadIdx.x; b < nblk; b += EN_THREADS) {
        dj += part[b];
        dk += part[nblk + b];
    }
    red[0][threadIdx.x] = dj;
    red[1][threadIdx.x] = dk;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sj = 0.0, sk = 0.0;
        for (int t = 0; t < EN_THREADS; t++) {
            sj += red[0][t];
            sk += red[1][t];
        }
        out[0] = sj - 0.5 * sk;
        out[1] = sj;
        out[2] = sk;
    }
}

// Nuclear gradient: one block per (atom, Cartesian direction) row; threads
// take the atom's CSR entries in a fixed stride, then a fixed-order block sum.
constexpr int GA_THREADS = 256;

__global__ void __launch_bounds__(GA_THREADS)
pair_grad_atoms_kernel(const double* __restrict__ pg, int64_t gs, const double* __restrict__ w,
                       const int64_t* __restrict__ rowptr, const uint32_t* __restrict__ src,
                       double* __restrict__ out)
{
    __shared__ double red[GA_THREADS / 32];
    const int row = blockIdx.x;
    const int t = row / 3, x = row % 3;
    const int64_t e0 = __ldg(rowptr + t), e1 = __ldg(rowptr + t + 1);
    double s = 0.0;
    for (int64_t e = e0 + threadIdx.x; e < e1; e += GA_THREADS) {
        const uint32_t v = __ldg(src + e);
        const int64_t p = v & 0x7fffffffu;
        const int64_t side = v >> 31;
        s = fma(w ? __ldg(w + p) : 1.0, __ldg(pg + (3 * side + x) * gs + p), s);
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int k = 0; k < GA_THREADS / 32; k++) a += red[k];
        out[row] = a;
    }
}

}  // namespace vlxb

extern "C" int vlxb_pairGradientToAtoms(const double* pair_grad, uint64_t grad_stride, const double* weight,
                                        const int64_t* rowptr, const uint32_t* src, int32_t n_atoms,
                                        double* grad_atoms, void* stream)
{
    using namespace vlxb;
    if (n_atoms <= 0 || !grad_atoms || !rowptr) return VLXB_EINVAL;
    if (grad_stride > (uint64_t)INT64_MAX / 8 || (int64_t)n_atoms * 3 > (int64_t)INT32_MAX) return VLXB_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    if (grad_stride == 0) {  // empty CSR: no pair derivatives to fold
        VLXB_CHECK_CUDA(cudaMemsetAsync(grad_atoms, 0, sizeof(double) * 3 * (size_t)n_atoms, st));
        return VLXB_OK;
    }
    if (!pair_grad || !src) return VLXB_EINVAL;
    pair_grad_atoms_kernel<<<3 * n_atoms, GA_THREADS, 0, st>>>(pair_grad, (int64_t)grad_stride, weight, rowptr,
                                                               src, grad_atoms);
    note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

extern "C" int vlxb_pairsToAO(const double* pair_values, const int64_t* rowptr, const int32_t* row_ao,
                              const uint32_t* src, int64_t n_rows, double* mat_AO, int32_t naos, void* stream)
{
    using namespace vlxb;
    if (naos <= 0 || n_rows < 0 || !mat_AO) return VLXB_EINVAL;
    if (n_rows > 0 && (!pair_values || !rowptr || !row_ao || !src)) return VLXB_EINVAL;
    if ((int64_t)naos * naos > (int64_t)INT32_MAX) return VLXB_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    VLXB_CHECK_CUDA(cudaMemsetAsync(mat_AO, 0, sizeof(double) * (size_t)naos * naos, st));
    if (n_rows == 0) return VLXB_OK;
    const int64_t want = (n_rows + 255) / 256;
    const int grid = (int)(want < 148 * 16 ? want : 148 * 16);
    pairs_to_ao_kernel<<<grid, 256, 0, st>>>(pair_values, rowptr, row_ao, src, n_rows, mat_AO, naos);
    note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}

extern "C" int vlxb_fockEnergy(const double* D_AO, const double* J_AO, const double* K_AO, int32_t naos,
                               double* out3, void* stream)
{
    using namespace vlxb;
    if (!D_AO || !out3 || naos <= 0) return VLXB_EINVAL;
    int rc = ensure_pool_configured();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    Arena ar(st);
    double* part = ar.alloc<double>(3 * EN_BLOCKS);
    if (!part) return VLXB_ENOMEM;
    energy_partial_kernel<<<EN_BLOCKS, EN_THREADS, 0, st>>>(D_AO, J_AO, K_AO, (int64_t)naos * naos, part);
    energy_final_kernel<<<1, EN_THREADS, 0, st>>>(part, EN_BLOCKS, out3);
    note_launches();
    note_launches();
    VLXB_CHECK_CUDA(cudaGetLastError());
    return VLXB_OK;
}
