// Explicit FP32 Schur operator for the mixed-precision CGRAD.
//
// memLS's CGRAD (flowsolver/src/memLS.f90:367-430) iterates on the
// continuity Schur complement without forming it: every iteration computes
// SP = L P - Gt (G P) - (coupled-face terms) as two sparse products, which
// costs two neighbour-gather phases and three grid barriers per iteration in
// the persistent kernel.  In the mixed-precision solve the inner CG only has
// to shape search directions (the FP64 NSSOLVER Gram system and the
// iterative refinement decide the accuracy), so there the operator
// S = L - Gt G is formed once per NSSOLVER call in FP64 (on the 2-ring
// pattern of the node graph) and stored in FP32:
//
//   * pattern (once per lhs): the 2-ring of every row, sorted, as a sliced
//     ELL layout (slices of 32 rows, column-major) with int16 column offsets
//     col - row (the layout requires |col - row| <= 32767 and at most
//     kS2Cap entries per row; otherwise the two-product kernel is used);
//   * values (per NSSOLVER call): S_ij = L_ij - sum_k Gt_ik . G_kj summed in
//     FP64 in a fixed order (L first, then k in CSR order) -- deterministic --
//     and rounded once to FP32;
//   * CG iteration (persistent cooperative kernel, two grid barriers):
//     phase 1 SP_raw = S P with P = R + beta P_prev formed on the fly from
//     an FP32 copy {R, P_prev} of the neighbours, plus <P, SP_raw>, w_f . P
//     and z_f . P; phase 2 the coupled-face (Sherman-Morrison) correction
//     SP = SP_raw - sum_f coef_f (w_f . P) z_f, X += alpha P, R -= alpha SP,
//     |R|^2.  Every product accumulates in FP64; X, R, P and all dot
//     products are FP64, reduced per block and summed in block order.
//
// The coupled-face term is the same exact rank-one form the two-product
// kernel uses: Gt (G P + c valM (valM . G P)) = Gt G P + c (w . P) z with
// w = G^T valM, z = Gt valM built once per NSSOLVER call.
#include <cooperative_groups.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <climits>
#include <vector>

#include "common.cuh"
#include "memls.cuh"

namespace crimson {

constexpr int kS2Cap = 256;        // 2-ring entries per row the formation kernel holds
constexpr int kS2Threads = 1024;   // formation: one warp per row of a 32-row slice
constexpr int kS2U = 8;            // entries per software-pipelined stage of the CG rows
constexpr int kS2CgThreads = 512;
constexpr int kS2MaxFaces = 8;
constexpr int kS2PartStride = 2 * kS2MaxFaces + 1;

// ---------------------------------------------------------------------------
// Pattern
// ---------------------------------------------------------------------------
__global__ void k_s2_count(const int* __restrict__ rowptr, const int* __restrict__ col, int n,
                           long long* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        long long c = 0;
        for (int t = rowptr[i]; t < rowptr[i + 1]; ++t) {
            const int k = col[t];
            c += rowptr[k + 1] - rowptr[k];
        }
        cnt[i] = c;
    }
}

__global__ void k_s2_fill(const int* __restrict__ rowptr, const int* __restrict__ col, int n,
                          const long long* __restrict__ off, unsigned long long* __restrict__ keys) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        long long p = off[i];
        for (int t = rowptr[i]; t < rowptr[i + 1]; ++t) {
            const int k = col[t];
            for (int u = rowptr[k]; u < rowptr[k + 1]; ++u)
                keys[p++] = (unsigned long long)i * (unsigned long long)n + (unsigned long long)col[u];
        }
    }
}

__device__ __forceinline__ long long s2_lower_bound(const unsigned long long* a, long long m, unsigned long long v) {
    long long lo = 0, hi = m;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (a[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void k_s2_csr(const unsigned long long* __restrict__ ukeys, long long m, int n, int* __restrict__ rowptr2,
                         int* __restrict__ col2, int* __restrict__ maxoff) {
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long st = (long long)gridDim.x * blockDim.x;
    for (long long i = t0; i <= n; i += st)
        rowptr2[i] = (int)s2_lower_bound(ukeys, m, (unsigned long long)i * (unsigned long long)n);
    int mo = 0;
    for (long long j = t0; j < m; j += st) {
        const int r = (int)(ukeys[j] / (unsigned long long)n);
        const int c = (int)(ukeys[j] % (unsigned long long)n);
        col2[j] = c;
        mo = max(mo, abs(c - r));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mo = max(mo, __shfl_xor_sync(0xffffffffu, mo, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxoff, mo);
}

// int16 offsets col - row at every sliced position (pads: 0, the row itself)
__global__ void k_s2_offsets(const int* __restrict__ rowptr2, const int* __restrict__ col2, const int* __restrict__ sp,
                             int n, int nrows_pad, short* __restrict__ soff) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows_pad; r += gridDim.x * blockDim.x) {
        const int s = r >> 5;
        const int w = (sp[s + 1] - sp[s]) >> 5;
        const int base = sp[s] + (r & 31);
        const int rs = r < n ? rowptr2[r] : 0;
        const int len = r < n ? rowptr2[r + 1] - rs : 0;
        for (int k = 0; k < w; ++k) soff[base + 32 * k] = k < len ? (short)(col2[rs + k] - r) : (short)0;
    }
}

int schur_pattern(crimson_lhs* L) {
    if (L->s2_state != 0) return CRIMSON_OK;
    cudaStream_t s = L->stream;
    const int n = L->nNo;
    L->s2_state = -1;   // unusable unless every step below succeeds
    DBuf<long long> cnt, koff;
    CR_CHECK(cnt.alloc((size_t)n + 1));
    CR_CHECK(koff.alloc((size_t)n + 1));
    CR_CUDA(cudaMemsetAsync(cnt.p + n, 0, sizeof(long long), s));
    launch(k_s2_count, grid_for(n, 256), 256, 0, s, L->rowptr, L->col, n, cnt.p);
    size_t tb = 0;
    CR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, koff.p, n + 1, s));
    DBuf<unsigned char> tmp;
    CR_CHECK(tmp.alloc(tb));
    CR_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.p, koff.p, n + 1, s));
    long long total = 0;
    CR_CUDA(cudaMemcpyAsync(&total, koff.p + n, sizeof(long long), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    if (total <= 0 || total > (long long)INT_MAX) return CRIMSON_OK;
    const int m = (int)total;
    DBuf<unsigned long long> keys, keys2, ukeys;
    DBuf<int> dcount, dmax;
    CR_CHECK(keys.alloc((size_t)m));
    CR_CHECK(keys2.alloc((size_t)m));
    launch(k_s2_fill, grid_for(n, 256), 256, 0, s, L->rowptr, L->col, n, (const long long*)koff.p, keys.p);
    unsigned long long maxkey = (unsigned long long)n * (unsigned long long)n;
    int end_bit = 1;
    while (end_bit < 64 && (1ull << end_bit) <= maxkey) ++end_bit;
    cub::DoubleBuffer<unsigned long long> dk(keys.p, keys2.p);
    size_t tb_sort = 0, tb_uniq = 0;
    CR_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb_sort, dk, m, 0, end_bit, s));
    CR_CHECK(dcount.alloc(1));
    CR_CHECK(ukeys.alloc((size_t)m));
    CR_CUDA(cub::DeviceSelect::Unique(nullptr, tb_uniq, keys.p, ukeys.p, dcount.p, m, s));
    CR_CHECK(tmp.alloc(std::max(tb_sort, tb_uniq)));
    CR_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb_sort, dk, m, 0, end_bit, s));
    CR_CUDA(cub::DeviceSelect::Unique(tmp.p, tb_uniq, dk.Current(), ukeys.p, dcount.p, m, s));
    int nnz2 = 0;
    CR_CUDA(cudaMemcpyAsync(&nnz2, dcount.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    keys.release();
    keys2.release();
    DBuf<int> rowptr2, col2;
    CR_CHECK(rowptr2.alloc((size_t)n + 1));
    CR_CHECK(col2.alloc((size_t)nnz2));
    CR_CHECK(dmax.alloc(1));
    CR_CUDA(cudaMemsetAsync(dmax.p, 0, sizeof(int), s));
    launch(k_s2_csr, grid_for((long long)nnz2 + n + 1, 256), 256, 0, s, (const unsigned long long*)ukeys.p,
           (long long)nnz2, n, rowptr2.p, col2.p, dmax.p);
    std::vector<int> rp((size_t)n + 1);
    int maxoff = 0;
    CR_CUDA(cudaMemcpyAsync(rp.data(), rowptr2.p, sizeof(int) * rp.size(), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaMemcpyAsync(&maxoff, dmax.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    ukeys.release();
    int maxlen = 0;
    for (int i = 0; i < n; ++i) maxlen = std::max(maxlen, rp[i + 1] - rp[i]);
    if (maxoff > 32767 || maxlen > kS2Cap) return CRIMSON_OK;
    // sliced layout
    const int ns = (n + 31) / 32;
    std::vector<int> sp((size_t)ns + 1, 0);
    long long pos = 0;
    for (int q = 0; q < ns; ++q) {
        int w = 0;
        for (int r = q * 32; r < std::min(n, (q + 1) * 32); ++r) w = std::max(w, rp[r + 1] - rp[r]);
        sp[q] = (int)pos;
        pos += 32LL * w;
        if (pos + 64LL * kS2U > (long long)INT_MAX) return CRIMSON_OK;
    }
    sp[ns] = (int)pos;
    // the CG row loop loads one stage ahead: up to 32 (2 kS2U - 1) entries past
    // the last slice, so the arrays carry 64 kS2U zero entries there
    const size_t np = (size_t)pos + 64 * (size_t)kS2U;
    CR_CHECK(L->s2_sp.upload(sp.data(), sp.size(), s));
    CR_CHECK(L->s2_off.alloc(np));
    CR_CHECK(L->s2_val.alloc(np));
    CR_CUDA(cudaMemsetAsync(L->s2_off.p, 0, sizeof(short) * np, s));
    CR_CUDA(cudaMemsetAsync(L->s2_val.p, 0, sizeof(float) * np, s));
    launch(k_s2_offsets, grid_for((long long)ns * 32, 256), 256, 0, s, (const int*)rowptr2.p, (const int*)col2.p,
           (const int*)L->s2_sp.p, n, ns * 32, L->s2_off.p);
    CR_CUDA(cudaStreamSynchronize(s));
    CR_CUDA(cudaGetLastError());
    L->s2_rowptr = std::move(rowptr2);
    L->s2_col = std::move(col2);
    L->s2_nnz = nnz2;
    L->s2_npad = pos;
    L->s2_nslice = ns;
    L->s2_state = 1;
    return CRIMSON_OK;
}

// ---------------------------------------------------------------------------
// Values: S = L - Gt G in FP64, rounded to FP32.  One block per 32-row slice,
// one warp per row; the row's 2-ring columns and FP64 accumulators sit in
// shared memory.  Within a warp the lanes add distinct columns, and the
// contributions are added in a fixed order (L, then k in CSR order), so the
// result is deterministic.  The slice is written back coalesced.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int s2_find(const int* cols, int len, int j) {
    int lo = 0, hi = len;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (cols[mid] < j)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kS2Threads) k_s2_form(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                        const double* __restrict__ mG, const double* __restrict__ Gt,
                                                        const double* __restrict__ mL, const int* __restrict__ rowptr2,
                                                        const int* __restrict__ col2, const int* __restrict__ sp,
                                                        int n, int nslice, float* __restrict__ val) {
    extern __shared__ double s2_smem[];
    double* acc = s2_smem;                                                 // [32][kS2Cap]
    int* cols = reinterpret_cast<int*>(s2_smem + 32 * kS2Cap);            // [32][kS2Cap]
    __shared__ int lens[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double* a = acc + wid * kS2Cap;
    int* cw = cols + wid * kS2Cap;
    for (int sl = blockIdx.x; sl < nslice; sl += gridDim.x) {
        const int r = sl * 32 + wid;
        int len = 0;
        if (r < n) {
            const int rs2 = rowptr2[r];
            len = rowptr2[r + 1] - rs2;
            for (int e = lane; e < len; e += 32) {
                cw[e] = col2[rs2 + e];
                a[e] = 0.0;
            }
        }
        if (lane == 0) lens[wid] = len;
        __syncwarp();
        if (r < n) {
            const int rs = rowptr[r], re = rowptr[r + 1];
            // every column met here is in the row's 2-ring; the guard only
            // keeps a malformed pattern from writing outside the row
            for (int t = rs + lane; t < re; t += 32) {
                const int j = col[t], q = s2_find(cw, len, j);
                if (q < len && cw[q] == j) a[q] += mL[t];
            }
            __syncwarp();
            for (int t = rs; t < re; ++t) {
                const int k = col[t];
                const double g0 = Gt[3 * (size_t)t], g1 = Gt[3 * (size_t)t + 1], g2 = Gt[3 * (size_t)t + 2];
                const int ks = rowptr[k], ke = rowptr[k + 1];
                for (int u = ks + lane; u < ke; u += 32) {
                    const double* gk = mG + 3 * (size_t)u;
                    const int j = col[u], q = s2_find(cw, len, j);
                    if (q < len && cw[q] == j) a[q] -= g0 * gk[0] + g1 * gk[1] + g2 * gk[2];
                }
                __syncwarp();
            }
        }
        __syncthreads();
        const int p0 = sp[sl], w = (sp[sl + 1] - p0) >> 5;
        for (int p = threadIdx.x; p < 32 * w; p += blockDim.x) {
            const int row = p & 31, e = p >> 5;
            val[p0 + p] = e < lens[row] ? (float)acc[row * kS2Cap + e] : 0.0f;
        }
        __syncthreads();
    }
}

int schur_form(crimson_lhs* L, const double* mG, const double* Gt, const double* mL) {
    if (L->s2_state != 1) return CRIMSON_ERR_STATE;
    cudaStream_t s = L->stream;
    const size_t smem = 32 * (size_t)kS2Cap * (sizeof(double) + sizeof(int));
    // the attribute is per device; setting it again (two host threads racing
    // on the first call) is harmless, so a relaxed flag is enough
    static std::atomic<bool> attr_set[256];
    int dev = 0;
    CR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return CRIMSON_ERR_UNSUPPORTED;
    if (!attr_set[dev].load(std::memory_order_relaxed)) {
        CR_CUDA(cudaFuncSetAttribute(k_s2_form, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set[dev].store(true, std::memory_order_relaxed);
    }
    CR_CUDA(cudaEventRecord(L->s2_ev0, s));
    launch(k_s2_form, std::min(L->s2_nslice, 2 * sm_count()), kS2Threads, smem, s, L->rowptr, L->col, mG, Gt, mL,
           (const int*)L->s2_rowptr.p, (const int*)L->s2_col.p, (const int*)L->s2_sp.p, L->nNo, L->s2_nslice,
           L->s2_val.p);
    CR_CUDA(cudaEventRecord(L->s2_ev1, s));
    CR_CUDA(cudaGetLastError());
    L->s2_form_pending = true;
    return CRIMSON_OK;
}

// ---------------------------------------------------------------------------
// CGRAD on the explicit FP32 operator: one persistent cooperative launch per
// call, two grid barriers per iteration.
// ---------------------------------------------------------------------------
struct CgS2Args {
    const int* sp;
    const short* off;
    const float* val;
    int n;
    double* X;
    double2* recA;   // (n) {R, P_prev}, FP64
    float2* recF;    // (n) {R, P_prev} rounded to FP32: the gathered copy
    double* SPr;     // (n) S P of this iteration, before the coupled-face term
    int nface;
    const double* w;  // (nface, n)
    const double* z;  // (nface, n)
    double coef[kS2MaxFaces];
    double eps;
    double err0;
    int mItr;
    double* part;  // 2 regions of kS2PartStride * gridDim
    double* out;   // err, errO, i, suc
};

__device__ __forceinline__ double s2_sum_partials(const double* part, int k, double* sm) {
    double v = 0.0;
    for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) v += __ldcg(part + (size_t)b * kS2PartStride + k);
    return block_sum(v, sm);
}

template <int NF>
__global__ void __launch_bounds__(kS2CgThreads, 2) k_cg_schur(CgS2Args a) {
    namespace cgrp = cooperative_groups;
    cgrp::grid_group grid = cgrp::this_grid();
    __shared__ double sm[32];
    const int n = a.n;
    double* part1 = a.part;
    double* part2 = a.part + (size_t)gridDim.x * kS2PartStride;
    double err = a.err0, errO = a.err0;
    int suc = 0, i;
    for (i = 1; i <= a.mItr; ++i) {
        if (err < a.eps) {
            suc = 1;
            break;
        }
        const bool first = (i == 1);
        const double beta = first ? 0.0 : err / errO;
        errO = err;
        // ---- phase 1: SP_raw = S P (P on the fly), <P, SP_raw>, w_f . P, z_f . P ----
        double dps = 0.0, wp[NF > 0 ? NF : 1], zp[NF > 0 ? NF : 1];
#pragma unroll
        for (int f = 0; f < (NF > 0 ? NF : 1); ++f) wp[f] = zp[f] = 0.0;
        for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
            const int p0 = __ldg(a.sp + (r >> 5));
            const int w = (__ldg(a.sp + (r >> 5) + 1) - p0) >> 5;
            const int base = p0 + (r & 31);
            float v[kS2U];
            short o[kS2U];
#pragma unroll
            for (int u = 0; u < kS2U; ++u) {
                v[u] = __ldcs(a.val + base + 32 * u);
                o[u] = __ldcs(a.off + base + 32 * u);
            }
            double acc = 0.0;
            for (int k0 = 0; k0 < w; k0 += kS2U) {
                float vn[kS2U];
                short on[kS2U];
#pragma unroll
                for (int u = 0; u < kS2U; ++u) {
                    // the arrays carry 64 kS2U zero entries past the last slice
                    vn[u] = __ldcs(a.val + base + 32 * (k0 + kS2U + u));
                    on[u] = __ldcs(a.off + base + 32 * (k0 + kS2U + u));
                }
#pragma unroll
                for (int u = 0; u < kS2U; ++u) {
                    if (k0 + u < w) {
                        const float2 q = a.recF[r + (int)o[u]];
                        const double pj = first ? (double)q.x : (double)q.x + beta * (double)q.y;
                        acc = acc + (double)v[u] * pj;
                    }
                }
#pragma unroll
                for (int u = 0; u < kS2U; ++u) {
                    v[u] = vn[u];
                    o[u] = on[u];
                }
            }
            const double2 ra = a.recA[r];
            const double pr = first ? ra.x : ra.x + beta * ra.y;
            a.SPr[r] = acc;
            dps += pr * acc;
#pragma unroll
            for (int f = 0; f < NF; ++f)
                if (f < a.nface) {
                    wp[f] += a.w[(size_t)f * n + r] * pr;
                    zp[f] += a.z[(size_t)f * n + r] * pr;
                }
        }
        dps = block_sum(dps, sm);
        if (threadIdx.x == 0) part1[(size_t)blockIdx.x * kS2PartStride] = dps;
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            if (f < a.nface) {
                const double tw = block_sum(wp[f], sm);
                const double tz = block_sum(zp[f], sm);
                if (threadIdx.x == 0) {
                    part1[(size_t)blockIdx.x * kS2PartStride + 1 + f] = tw;
                    part1[(size_t)blockIdx.x * kS2PartStride + 1 + kS2MaxFaces + f] = tz;
                }
            }
        }
        grid.sync();
        double cS[NF > 0 ? NF : 1];
        double den = s2_sum_partials(part1, 0, sm);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            cS[f] = 0.0;
            if (f < a.nface) {
                cS[f] = a.coef[f] * s2_sum_partials(part1, 1 + f, sm);
                den = den - cS[f] * s2_sum_partials(part1, 1 + kS2MaxFaces + f, sm);
            }
        }
        const double alpha = errO / den;
        // ---- phase 2: SP = SP_raw - sum_f cS_f z_f; X += alpha P, R -= alpha SP, |R|^2 ----
        double rs = 0.0;
        for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
            const double2 ra = a.recA[r];
            const double pr = first ? ra.x : ra.x + beta * ra.y;
            double sp = a.SPr[r];
#pragma unroll
            for (int f = 0; f < NF; ++f)
                if (f < a.nface) sp = sp - cS[f] * a.z[(size_t)f * n + r];
            a.X[r] = a.X[r] + alpha * pr;
            const double rv = ra.x - alpha * sp;
            a.recA[r] = make_double2(rv, pr);
            a.recF[r] = make_float2((float)rv, (float)pr);
            rs += rv * rv;
        }
        rs = block_sum(rs, sm);
        if (threadIdx.x == 0) part2[(size_t)blockIdx.x * kS2PartStride] = rs;
        grid.sync();
        const double e2 = sqrt(s2_sum_partials(part2, 0, sm));
        err = e2 * e2;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = err;
        a.out[1] = errO;
        a.out[2] = (double)i;
        a.out[3] = (double)suc;
    }
}

// recA = {R, 0}, recF = {R, 0}
__global__ void k_s2_init(const double* __restrict__ R, double2* __restrict__ recA, float2* __restrict__ recF, int n) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        recA[t] = make_double2(R[t], 0.0);
        recF[t] = make_float2((float)R[t], 0.0f);
    }
}

// One CGRAD call on the explicit operator: R (n) holds the right side and
// receives nothing (the solution is left in L->cgX); out (4 doubles, device)
// receives err, errO, the iteration index and the success flag.
int cg_schur_launch(crimson_lhs* L, const double* R, int nface, const double* coef, const double* w, const double* z,
                    double eps, double err0, int mItr, double* out) {
    if (L->s2_state != 1 || nface > kS2MaxFaces) return CRIMSON_ERR_STATE;
    cudaStream_t s = L->stream;
    const int n = L->nNo;
    const void* kfn[3] = {(const void*)k_cg_schur<0>, (const void*)k_cg_schur<1>,
                          (const void*)k_cg_schur<kS2MaxFaces>};
    const int fi = nface == 0 ? 0 : (nface == 1 ? 1 : 2);
    if (L->s2_grid == 0) {
        int nb = 1 << 30;
        for (const void* f : kfn) {
            int b = 0;
            CR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, kS2CgThreads, 0));
            nb = std::min(nb, b);
        }
        if (nb < 1) return CRIMSON_ERR_UNSUPPORTED;
        L->s2_grid = sm_count() * std::min(nb, 2);
    }
    CR_CHECK(L->s2_part.alloc(2 * (size_t)kS2PartStride * L->s2_grid));
    CR_CHECK(L->cgRecA.alloc(2 * (size_t)n));
    CR_CHECK(L->s2_recF.alloc((size_t)n));
    CR_CHECK(L->cgSP.alloc((size_t)n));
    CR_CUDA(cudaMemsetAsync(L->cgX.p, 0, sizeof(double) * n, s));
    launch(k_s2_init, grid_for(n, 256), 256, 0, s, R, reinterpret_cast<double2*>(L->cgRecA.p), L->s2_recF.p, n);
    CgS2Args a;
    a.sp = L->s2_sp.p;
    a.off = L->s2_off.p;
    a.val = L->s2_val.p;
    a.n = n;
    a.X = L->cgX.p;
    a.recA = reinterpret_cast<double2*>(L->cgRecA.p);
    a.recF = L->s2_recF.p;
    a.SPr = L->cgSP.p;
    a.nface = nface;
    a.w = w;
    a.z = z;
    for (int f = 0; f < kS2MaxFaces; ++f) a.coef[f] = f < nface ? coef[f] : 0.0;
    a.eps = eps;
    a.err0 = err0;
    a.mItr = mItr;
    a.part = L->s2_part.p;
    a.out = out;
    void* kargs[] = {&a};
    note_launch();
    CR_CUDA(cudaLaunchCooperativeKernel(kfn[fi], dim3(L->s2_grid), dim3(kS2CgThreads), kargs, 0, s));
    return CRIMSON_OK;
}

}  // namespace crimson
