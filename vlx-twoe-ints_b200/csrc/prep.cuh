// Device-side regrouping of the reference's primitive-Cartesian pair lists
// into primitive-SHELL-pair records (the unit of the integral kernels).
//
// Reference list formats (gen_coulomb.py:80-90, gen_exchange.py:78-110):
//   prim-cart index i of type x -> primitive shell i / ncart(x), component
//   i % ncart(x); prim_info[5][count] (row 0 exponent, rows 2-4 xyz);
//   J lists: first/second prim-cart indices, pair_data S_ij_00, Q, D per pair;
//   K lists: CSR per prim-cart i (displs, counts) of partners D_inds with Q
//   and pair_data; prim_aoinds[ncart][count] maps (primitive, component) to
//   the Cartesian AO index.
//
// Grouping uses a dense table over (shell_i, shell_j) and an exclusive scan,
// so record order is deterministic (shell-major) and no atomics are needed.
// Every count that sizes a later launch stays on the device (grid-stride
// kernels read it), so a whole ABI call issues no host synchronisation.
#pragma once
#include "common.cuh"
#include "md.cuh"

namespace vlxb {

constexpr int PREP_THREADS = 256;

__host__ __forceinline__ int prep_blocks(int64_t n)
{
    int64_t b = (n + PREP_THREADS - 1) / PREP_THREADS;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (int)b;
}

__global__ void k_iota(int* __restrict__ p, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = (int)i;
}

// ------------------------------------------------------------ flat lists

__global__ void k_mark_pairs(const uint32_t* __restrict__ first, const uint32_t* __restrict__ second,
                             int64_t n, int na, int nb, int npb, int* __restrict__ table)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t key = (int64_t)(first[e] / na) * npb + second[e] / nb;
        table[key] = 1;
    }
}

__global__ void k_fill_pairs(const uint32_t* __restrict__ first, const uint32_t* __restrict__ second,
                             int64_t n, int na, int nb, int npb, const int* __restrict__ spidx,
                             int32_t* __restrict__ entry, int32_t* __restrict__ sp_i, int32_t* __restrict__ sp_j,
                             int64_t stride)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t i = first[e], j = second[e];
        const int64_t key = (int64_t)(i / na) * npb + j / nb;
        const int s = spidx[key];
        const int comp = (int)(i % na) * nb + (int)(j % nb);
        entry[comp * stride + s] = (int32_t)e;
        sp_i[s] = (int32_t)(i / na);
        sp_j[s] = (int32_t)(j / nb);
    }
}

// ------------------------------------------------------------ CSR lists

__global__ void k_mark_csr(const uint32_t* __restrict__ displs, const uint32_t* __restrict__ counts,
                           const uint32_t* __restrict__ Dinds, int n_first, int na, int nb, int npb,
                           int* __restrict__ table)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_first; i += gridDim.x * blockDim.x) {
        const uint32_t d0 = displs[i], c = counts[i];
        for (uint32_t t = 0; t < c; t++) {
            const uint32_t j = Dinds[d0 + t];
            table[(int64_t)(i / na) * npb + j / nb] = 1;
        }
    }
}

__global__ void k_fill_csr(const uint32_t* __restrict__ displs, const uint32_t* __restrict__ counts,
                           const uint32_t* __restrict__ Dinds, int n_first, int na, int nb, int npb,
                           const int* __restrict__ spidx, int32_t* __restrict__ entry,
                           int32_t* __restrict__ sp_i, int32_t* __restrict__ sp_j, int64_t stride)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_first; i += gridDim.x * blockDim.x) {
        const uint32_t d0 = displs[i], c = counts[i];
        for (uint32_t t = 0; t < c; t++) {
            const uint32_t j = Dinds[d0 + t];
            const int s = spidx[(int64_t)(i / na) * npb + j / nb];
            const int comp = (i % na) * nb + (int)(j % nb);
            entry[comp * stride + s] = (int32_t)(d0 + t);
            sp_i[s] = i / na;
            sp_j[s] = (int32_t)(j / nb);
        }
    }
}

// n_out[0] = scan[n-1] + flag[n-1]  (exclusive scan total)
__global__ void k_scan_total(const int* __restrict__ scan, const int* __restrict__ flag, int64_t n, int* __restrict__ out)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = (n > 0) ? scan[n - 1] + flag[n - 1] : 0;
}

// Pair geometry (see PairGeo): z, 0.5/z, P, P - A, A - B, and the first
// centre's exponent.
__global__ void k_pair_geo(const int* __restrict__ n_sp, const int32_t* __restrict__ sp_i,
                           const int32_t* __restrict__ sp_j, const double* __restrict__ info_a, uint32_t cnt_a,
                           const double* __restrict__ info_b, uint32_t cnt_b, double* __restrict__ geo,
                           int64_t stride)
{
    const int n = *n_sp;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int i = sp_i[s], j = sp_j[s];
        const double ai = info_a[i], aj = info_b[j];
        const double A[3] = {info_a[i + 2 * (int64_t)cnt_a], info_a[i + 3 * (int64_t)cnt_a], info_a[i + 4 * (int64_t)cnt_a]};
        const double B[3] = {info_b[j + 2 * (int64_t)cnt_b], info_b[j + 3 * (int64_t)cnt_b], info_b[j + 4 * (int64_t)cnt_b]};
        const double z = ai + aj, iz = 1.0 / z;
        geo[G_Z * stride + s] = z;
        geo[G_I2Z * stride + s] = 0.5 * iz;
        geo[G_ALPHA * stride + s] = ai;
#pragma unroll
        for (int x = 0; x < 3; x++) {
            const double P = (ai * A[x] + aj * B[x]) * iz;
            geo[(G_PX + x) * stride + s] = P;
            geo[(G_AX + x) * stride + s] = P - A[x];
            geo[(G_RX + x) * stride + s] = A[x] - B[x];
        }
    }
}

// ------------------------------------------------------------ records
// A record is a subset of one shell pair's components that share one Schwarz
// value q (the caller may give every component its own Q).  Record =
// (shell pair, q, component bitmask).  Records of a shell pair follow the
// first appearance of each distinct q in component order.

template <int NXY>
__global__ void k_rec_count(const int* __restrict__ n_sp, const int32_t* __restrict__ entry, int64_t stride,
                            const double* __restrict__ Q, int* __restrict__ nrec)
{
    const int n = *n_sp;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        double qs[NXY];
        int nd = 0;
        for (int c = 0; c < NXY; c++) {
            const int32_t e = entry[c * stride + s];
            if (e < 0) continue;
            const double v = Q[e];
            bool seen = false;
            for (int t = 0; t < nd; t++) seen |= (qs[t] == v);
            if (!seen) qs[nd++] = v;
        }
        nrec[s] = nd;
    }
}

template <int NXY>
__global__ void k_rec_fill(const int* __restrict__ n_sp, const int32_t* __restrict__ entry, int64_t stride,
                           const double* __restrict__ Q, const int* __restrict__ recoff,
                           int32_t* __restrict__ rec_sp, double* __restrict__ rec_q, uint64_t* __restrict__ rec_mask)
{
    const int n = *n_sp;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        double qs[NXY];
        uint64_t ms[NXY];
        int nd = 0;
        for (int c = 0; c < NXY; c++) {
            const int32_t e = entry[c * stride + s];
            if (e < 0) continue;
            const double v = Q[e];
            int t = 0;
            for (; t < nd; t++) if (qs[t] == v) break;
            if (t == nd) { qs[nd] = v; ms[nd] = 0; nd++; }
            ms[t] |= (1ull << c);
        }
        const int r0 = recoff[s];
        for (int t = 0; t < nd; t++) {
            rec_sp[r0 + t] = s;
            rec_q[r0 + t] = qs[t];
            rec_mask[r0 + t] = ms[t];
        }
    }
}

// S per shell pair and component (0 where the caller has no entry).
template <int NXY>
__global__ void k_sp_S(const int* __restrict__ n_sp, const int32_t* __restrict__ entry, int64_t stride,
                       const double* __restrict__ pdata, double* __restrict__ S)
{
    const int n = *n_sp;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        for (int c = 0; c < NXY; c++) {
            const int32_t e = entry[c * stride + s];
            S[c * stride + s] = (e >= 0) ? pdata[e] : 0.0;
        }
}

// su[r] = the S shared by all components of record r when the record covers
// every component of its shell pair and they share one S value, else NaN
// (the kernels then digest with per-component S).
template <int NXY>
__global__ void k_rec_uniform_s(const int* __restrict__ n_rec, const int32_t* __restrict__ rec_sp,
                                const uint64_t* __restrict__ rec_mask, const double* __restrict__ S, int64_t stride,
                                double* __restrict__ su)
{
    const int n = *n_rec;
    const uint64_t full = (NXY >= 64) ? ~0ull : ((1ull << NXY) - 1ull);
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int sp = rec_sp[r];
        double v = __longlong_as_double(0x7ff8000000000000ll);
        if (rec_mask[r] == full) {
            const double s0 = S[sp];
            bool same = true;
            for (int c = 1; c < NXY; c++) same &= (S[c * stride + sp] == s0);
            if (same) v = s0;
        }
        su[r] = v;
    }
}

// Segment offsets of records by first shell: seg[i] = recoff[spidx[i * npb]],
// seg[np_first] = total records.
__global__ void k_rec_segments(const int* __restrict__ spidx, const int* __restrict__ recoff, int np_first, int npb,
                               const int* __restrict__ n_rec, int* __restrict__ seg)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= np_first; i += gridDim.x * blockDim.x)
        seg[i] = (i < np_first) ? recoff[spidx[(int64_t)i * npb]] : *n_rec;
}

__global__ void k_gather_recs(const int* __restrict__ n_rec, const int* __restrict__ perm,
                              const int32_t* __restrict__ sp_in, const uint64_t* __restrict__ mask_in,
                              int32_t* __restrict__ sp_out, uint64_t* __restrict__ mask_out)
{
    const int n = *n_rec;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int p = perm[r];
        sp_out[r] = sp_in[p];
        mask_out[r] = mask_in[p];
    }
}

// ------------------------------------------------------------ J ket data
// Per ket shell pair: |Q D| bounds, per-component Q and D (for the exact
// screen), Dm = w * D * S with the k<->l weight of gen_coulomb.py:276-281,
// and Dpp = transposed ket HRR of Dm.
template <int LC, int LD>
__global__ void k_jket_fill(const int* __restrict__ n_sp, const int32_t* __restrict__ entry, int64_t stride,
                            const uint32_t* __restrict__ first, const uint32_t* __restrict__ second,
                            const double* __restrict__ Dlist, const double* __restrict__ Qlist,
                            const double* __restrict__ pdata, const double* __restrict__ geo,
                            double* __restrict__ tmax_key, double* __restrict__ tmin,
                            double* __restrict__ Dpp, double* __restrict__ Dm, double* __restrict__ Qc,
                            double* __restrict__ Dc, int64_t key_len)
{
    constexpr int NCD = ncart(LC) * ncart(LD), NF = nrange(LC, LD);
    const int n = *n_sp;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < key_len; s += (int64_t)gridDim.x * blockDim.x) {
        if (s >= n) { tmax_key[s] = -1.0; continue; }
        double dm[NCD];
        double tx = 0.0, tn = 1.0e300;
        for (int c = 0; c < NCD; c++) {
            const int32_t e = entry[c * stride + s];
            double q = 0.0, d = 0.0, m = 0.0;
            if (e >= 0) {
                q = Qlist[e];
                d = Dlist[e];
                const double w = (LC != LD) ? 2.0 : ((first[e] != second[e]) ? 2.0 : 1.0);
                m = w * d * pdata[e];
                const double t = fabs(q * d);
                tx = fmax(tx, t);
                tn = fmin(tn, t);
            }
            dm[c] = m;
            Qc[c * stride + s] = q;
            Dc[c * stride + s] = d;
            Dm[c * stride + s] = m;
        }
        tmax_key[s] = tx;
        tmin[s] = tn;
        double dpp[NF];
        hrr_ket_adjoint<LC, LD>(geo[G_RX * stride + s], geo[G_RY * stride + s], geo[G_RZ * stride + s], dm, dpp);
        for (int f = 0; f < NF; f++) Dpp[f * stride + s] = dpp[f];
    }
}

// Gather ket arrays into the sorted order given by perm.
template <int LC, int LD>
__global__ void k_jket_gather(const int* __restrict__ n_sp, const int* __restrict__ perm, int64_t stride,
                              int64_t ostride, const double* __restrict__ geo_in, const double* __restrict__ tmax_in,
                              const double* __restrict__ tmin_in, const double* __restrict__ Dpp_in,
                              const double* __restrict__ Dm_in, const double* __restrict__ Qc_in,
                              const double* __restrict__ Dc_in, double* __restrict__ geo, double* __restrict__ tmax,
                              double* __restrict__ tmin, double* __restrict__ Dpp, double* __restrict__ Dm,
                              double* __restrict__ Qc, double* __restrict__ Dc)
{
    constexpr int NCD = ncart(LC) * ncart(LD), NF = nrange(LC, LD);
    const int n = *n_sp;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int p = perm[r];
        for (int g = 0; g < GEO_N; g++) geo[g * ostride + r] = geo_in[g * stride + p];
        tmax[r] = tmax_in[r];  // keys are already sorted
        tmin[r] = tmin_in[p];
        for (int f = 0; f < NF; f++) Dpp[f * ostride + r] = Dpp_in[f * stride + p];
        for (int c = 0; c < NCD; c++) {
            Dm[c * ostride + r] = Dm_in[c * stride + p];
            Qc[c * ostride + r] = Qc_in[c * stride + p];
            Dc[c * ostride + r] = Dc_in[c * stride + p];
        }
    }
}

// ------------------------------------------------------------ K outputs
template <int NAC>
__global__ void k_kout_fill(const uint32_t* __restrict__ pi, const uint32_t* __restrict__ pk, int64_t n,
                            int na, int nc, int npc, const int* __restrict__ spidx, int32_t* __restrict__ idx,
                            int32_t* __restrict__ ish, int32_t* __restrict__ ksh, int64_t stride)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t i = pi[e], k = pk[e];
        const int s = spidx[(int64_t)(i / na) * npc + k / nc];
        idx[((i % na) * nc + (k % nc)) * stride + s] = (int32_t)e;
        ish[s] = i / na;
        ksh[s] = k / nc;
    }
}

// ------------------------------------------------------------ contracted partner groups
// Partner records of one first primitive shell whose partners belong to one
// contracted shell share the partner's centre and AO indices, so their
// primitive quartets can be summed before the HRR (Head-Gordon-Pople).  A
// record is groupable when one S covers all its components (su not NaN); its
// key is then the AO index of the partner's first component.  Other records
// get a key of their own (naos + r) and stay alone.
__global__ void k_grp_key(const int* __restrict__ n_rec, const int32_t* __restrict__ rec_sp,
                          const double* __restrict__ su, const int32_t* __restrict__ sp_j,
                          const uint32_t* __restrict__ part_aoinds, uint32_t naos, uint32_t* __restrict__ key)
{
    const int n = *n_rec;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        key[r] = isnan(su[r]) ? naos + (uint32_t)r : part_aoinds[sp_j[rec_sp[r]]];
}

// flag[seg[i]] = 1 for every non-empty segment i (flag zeroed by the caller)
__global__ void k_seg_starts(const int* __restrict__ seg, int nseg, int* __restrict__ flag)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nseg; i += gridDim.x * blockDim.x)
        if (seg[i] < seg[i + 1]) flag[seg[i]] = 1;
}

// After the key sort: a run starts at a segment start or where the key changes;
// runstart[r] = r at run starts, 0 elsewhere (max-scanned by the caller).
__global__ void k_grp_runs(const int* __restrict__ n_rec, const int* __restrict__ segflag,
                           const uint32_t* __restrict__ key_sorted, int* __restrict__ runstart)
{
    const int n = *n_rec;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        runstart[r] = (r == 0 || segflag[r] || key_sorted[r] != key_sorted[r - 1]) ? r : 0;
}

// Group heads: run starts, and every MAXG-th record of a run (groups hold at
// most MAXG members).  head[r] for r >= n_rec stays 0.
__global__ void k_grp_heads(const int* __restrict__ n_rec, const int* __restrict__ runmax, int maxg,
                            int* __restrict__ head)
{
    const int n = *n_rec;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        head[r] = ((r - runmax[r]) % maxg) == 0 ? 1 : 0;
}

// Members in key order (gathered through the sort permutation) and one entry
// per group: first member, member count, max member q (the first member's:
// the key sort is stable and records arrive sorted by descending q).
__global__ void k_grp_fill(const int* __restrict__ n_rec, const int* __restrict__ perm,
                           const int* __restrict__ head, const int* __restrict__ gid,
                           const int32_t* __restrict__ rec_sp, const double* __restrict__ rec_q,
                           const double* __restrict__ su, const uint64_t* __restrict__ rec_mask,
                           int32_t* __restrict__ msp, double* __restrict__ mq, double* __restrict__ msu,
                           uint64_t* __restrict__ mmask, int32_t* __restrict__ gbeg, double* __restrict__ gq)
{
    const int n = *n_rec;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int p = perm[r];
        msp[r] = rec_sp[p];
        mq[r] = rec_q[p];
        msu[r] = su[p];
        mmask[r] = rec_mask[p];
        if (head[r]) {
            gbeg[gid[r]] = r;
            gq[gid[r]] = rec_q[p];
        }
    }
}

// Group segment offsets gseg[i] = gid[seg[i]] (gid exclusive scan of heads,
// n_rec + 1 entries), member counts from consecutive group starts.
__global__ void k_grp_seg(const int* __restrict__ seg, int nseg, const int* __restrict__ gid,
                          int* __restrict__ gseg)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= nseg; i += gridDim.x * blockDim.x)
        gseg[i] = gid[seg[i]];
}

__global__ void k_grp_order(const int* __restrict__ n_grp, const int* __restrict__ n_rec,
                            const int* __restrict__ gperm, const int32_t* __restrict__ gbeg_in,
                            int32_t* __restrict__ gbeg, int32_t* __restrict__ gcnt)
{
    const int n = *n_grp, nr = *n_rec;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int g = gperm[t];
        const int b = gbeg_in[g];
        gbeg[t] = b;
        gcnt[t] = (g + 1 < n ? gbeg_in[g + 1] : nr) - b;
    }
}

// Per-output-block max |D| of batched exchange calls: the block's first
// primitive shell belongs to one molecule, whose own bound screens the block.
__global__ void k_kout_maxd(const int* __restrict__ n_blk, const int32_t* __restrict__ ish,
                            const int32_t* __restrict__ prim_mol, const double* __restrict__ maxD_mol,
                            double* __restrict__ out)
{
    const int n = *n_blk;
    for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < n; o += gridDim.x * blockDim.x)
        out[o] = maxD_mol[prim_mol[ish[o]]];
}

// ------------------------------------------------------------ FP32 error budget
// FP32 error proxy of a primitive shell pair: its bound times the growth the
// horizontal recurrence can put on FP32 rounding errors when it moves lh
// units of angular momentum across the pair, (1 + sqrt(2 zeta) |R|)^lh with
// R = AB (bra) or CD (ket).  Intermediates of the recurrence scale like
// |R|^k against the final integral's sqrt(1 / 2 zeta)^k, so rounding errors
// of the intermediates reach the result multiplied by this factor.
__device__ __forceinline__ double hrr_amp(const double* __restrict__ geo, int64_t stride, int64_t sp, int lh)
{
    if (lh == 0) return 1.0;
    const double z = geo[G_Z * stride + sp];
    const double rx = geo[G_RX * stride + sp], ry = geo[G_RY * stride + sp], rz = geo[G_RZ * stride + sp];
    const double f = 1.0 + sqrt(2.0 * z * (rx * rx + ry * ry + rz * rz));
    double a = f;
    for (int k = 1; k < lh; k++) a *= f;
    return a;
}

// rec_qa[r] = rec_q[r] * hrr_amp(record r); zero past the live records.
__global__ void k_rec_amp(const int* __restrict__ n_rec, int64_t stride, const int32_t* __restrict__ rec_sp,
                          const double* __restrict__ rec_q, const double* __restrict__ geo, int64_t geo_stride,
                          int lh, double* __restrict__ out)
{
    const int n = *n_rec;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < stride; r += (int64_t)gridDim.x * blockDim.x)
        out[r] = r < n ? fabs(rec_q[r]) * hrr_amp(geo, geo_stride, rec_sp[r], lh) : 0.0;
}

// gqa[g] = sum over the group's members of |q| * hrr_amp; zero past the live groups.
__global__ void k_grp_amp(const int* __restrict__ n_grp, int64_t stride, const int32_t* __restrict__ gbeg,
                          const int32_t* __restrict__ gcnt, const int32_t* __restrict__ msp,
                          const double* __restrict__ mq, const double* __restrict__ geo, int64_t geo_stride, int lh,
                          double* __restrict__ out)
{
    const int n = *n_grp;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < stride; t += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        if (t < n) {
            const int b = gbeg[t], c = gcnt[t];
            for (int m = b; m < b + c; m++) s += fabs(mq[m]) * hrr_amp(geo, geo_stride, msp[m], lh);
        }
        out[t] = s;
    }
}

// kamp[t] = tmax[t] * hrr_amp(ket t) over the sorted kets; zero past them.
__global__ void k_jket_amp(const int* __restrict__ n_sp, int64_t stride, const double* __restrict__ tmax,
                           const double* __restrict__ geo, int lh, double* __restrict__ out)
{
    const int n = *n_sp;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < stride; t += (int64_t)gridDim.x * blockDim.x)
        out[t] = t < n ? tmax[t] * hrr_amp(geo, stride, t, lh) : 0.0;
}

// ------------------------------------------------------------ batched Coulomb calls
// Molecule key of every key-sorted ket (n_mol past the live kets, so they
// stay last in the stable molecule sort).
__global__ void k_jket_molkey(const int* __restrict__ n_sp, int64_t S, const int* __restrict__ perm,
                              const int32_t* __restrict__ sp_i, const int32_t* __restrict__ prim_mol, int n_mol,
                              int* __restrict__ molkey)
{
    const int n = *n_sp;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < S; t += (int64_t)gridDim.x * blockDim.x)
        molkey[t] = t < n ? prim_mol[sp_i[perm[t]]] : n_mol;
}

// perm_out[t] = perm[perm2[t]], keys_out[t] = keys[perm2[t]]
__global__ void k_compose_perm(const int* __restrict__ n_sp, const int* __restrict__ perm,
                               const int* __restrict__ perm2, const double* __restrict__ keys,
                               int* __restrict__ perm_out, double* __restrict__ keys_out)
{
    const int n = *n_sp;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        perm_out[t] = perm[perm2[t]];
        keys_out[t] = keys[perm2[t]];
    }
}

// seg[m] = first sorted ket of molecule m (molkey ascending over the n_sp live kets)
__global__ void k_mol_segments(const int* __restrict__ n_sp, const int* __restrict__ molkey, int n_mol,
                               int* __restrict__ seg)
{
    const int n = *n_sp;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m <= n_mol; m += gridDim.x * blockDim.x) {
        int lo = 0, hi = n;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (molkey[mid] < m) lo = mid + 1;
            else hi = mid;
        }
        seg[m] = lo;
    }
}

// molecule of every bra record
__global__ void k_rec_mol(const int* __restrict__ n_rec, const int32_t* __restrict__ rec_sp,
                          const int32_t* __restrict__ sp_i, const int32_t* __restrict__ prim_mol,
                          int32_t* __restrict__ mol)
{
    const int n = *n_rec;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        mol[r] = prim_mol[sp_i[rec_sp[r]]];
}

// Signed Hermite density of every sorted ket pair (McMurchie-Davidson Coulomb
// kernel), stored per ket: Dh[kt * nherm(LC + LD) + f].
template <int LC, int LD>
__global__ void k_jket_hermite(const int* __restrict__ n_sp, int64_t stride, const double* __restrict__ geo,
                               const double* __restrict__ Dm, double* __restrict__ Dh)
{
    constexpr int NCD = ncart(LC) * ncart(LD), NH = nherm(LC + LD);
    const int n = *n_sp;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const PairGeo k = load_geo(geo, stride, r);
        double dm[NCD], dh[NH];
        for (int c = 0; c < NCD; c++) dm[c] = Dm[c * stride + r];
        herm_ket_density<LC, LD, double>(k, dm, dh);
        for (int f = 0; f < NH; f++) Dh[(int64_t)r * NH + f] = dh[f];
    }
}

}  // namespace vlxb
