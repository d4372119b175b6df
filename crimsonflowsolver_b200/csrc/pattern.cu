// Node-graph CSR pattern on the device.
//
// Replaces genadj/Asadj (flowsolver/src/genadj.f90:20-71, asadj.f90:21-54):
// the reference builds per-node adjacency lists with a linear dedup and
// selection-sorts each row.  Here every element emits its 16 (row, col) pairs
// as 64-bit keys row*nshg + col; one stable radix sort (keys with the pair
// index t = 16 e + 4 a + b as value) + run-length encoding gives exactly the
// sorted, deduplicated rows genadj produces (diagonal included), so the
// pattern is bit-identical.  The same pass precomputes what the reference
// searches for at every assembly and solve:
//   slist/soff - the element pairs of every CSR slot, ascending t (the
//                owner-computes scatter of ElmGMR sums them in this order,
//                which is fillsparseI's serial element order,
//                fillsparse.f90:29-60; replaces sparseloc's searches,
//                fillsparse.f90:210-246)
//   diag  - diagonal slot per row                   (diagPtr, memLS.f90:1121-1131)
//   trans - slot of the transposed block (j,i)      (solfar.f90:225-232, memLS.f90:1664-1675)
#include <cub/cub.cuh>

#include "common.cuh"

namespace crimson {

__global__ void k_pair_keys(const int4* __restrict__ ien, int nelem, unsigned long long nshg,
                            unsigned long long* __restrict__ keys, int* __restrict__ vals) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)nelem * 16;
    for (; t < total; t += (long long)gridDim.x * blockDim.x) {
        int e = (int)(t >> 4), ab = (int)(t & 15);
        int4 n = ien[e];
        int na[4] = {n.x, n.y, n.z, n.w};
        keys[t] = (unsigned long long)na[ab >> 2] * nshg + (unsigned long long)na[ab & 3];
        vals[t] = (int)t;
    }
}

__device__ __forceinline__ long long lower_bound_u64(const unsigned long long* a, long long n,
                                                     unsigned long long v) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if (a[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void k_rowptr_cols(const unsigned long long* __restrict__ ukeys, long long nnz, int nshg,
                              int* __restrict__ rowptr, int* __restrict__ col) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (long long i = t; i <= nshg; i += (long long)gridDim.x * blockDim.x)
        rowptr[i] = (int)lower_bound_u64(ukeys, nnz, (unsigned long long)i * (unsigned long long)nshg);
    for (long long j = t; j < nnz; j += (long long)gridDim.x * blockDim.x)
        col[j] = (int)(ukeys[j] % (unsigned long long)nshg);
}

// Position of column c in row r, or -1.
__device__ __forceinline__ int find_in_row(const int* __restrict__ rowptr, const int* __restrict__ col, int r,
                                           int c) {
    int lo = rowptr[r], hi = rowptr[r + 1];
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (col[mid] < c)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < rowptr[r + 1] && col[lo] == c) ? lo : -1;
}

__global__ void k_diag_trans(const int* __restrict__ rowptr, const int* __restrict__ col, int nshg,
                             int* __restrict__ diag, int* __restrict__ trans, int* __restrict__ bad) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    for (; i < nshg; i += gridDim.x * blockDim.x) {
        int d = find_in_row(rowptr, col, i, i);
        diag[i] = d;
        if (d < 0) atomicAdd(bad, 1);
        for (int j = rowptr[i]; j < rowptr[i + 1]; ++j) {
            int t = find_in_row(rowptr, col, col[j], i);
            trans[j] = t;
            if (t < 0) atomicAdd(bad, 1);
        }
    }
}

__global__ void k_to_one_based(const int* __restrict__ in, int* __restrict__ out, long long n) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (; t < n; t += (long long)gridDim.x * blockDim.x) out[t] = in[t] + 1;
}

int build_pattern(crimson_ctx* c) {
    cudaStream_t s = c->stream;
    const long long npair = (long long)c->nelem * 16;
    if (npair > 0x7fffffffLL) {
        set_last_error("pattern: more than 134M elements (pair count exceeds 32-bit indexing)");
        return CRIMSON_ERR_UNSUPPORTED;
    }
    const int np = (int)npair;
    DBuf<unsigned long long> keys, keys2, ukeys;
    DBuf<int> vals, vals2, counts, dcount, bad;
    CR_CHECK(keys.alloc(npair));
    CR_CHECK(keys2.alloc(npair));
    CR_CHECK(vals.alloc(npair));
    CR_CHECK(vals2.alloc(npair));
    CR_CHECK(ukeys.alloc(npair));
    CR_CHECK(counts.alloc(npair + 1));
    CR_CHECK(dcount.alloc(1));
    CR_CHECK(bad.alloc(1));
    launch(k_pair_keys, grid_for(npair, 256), 256, 0, s, c->ien.p, c->nelem, (unsigned long long)c->nshg, keys.p,
           vals.p);
    CR_CUDA(cudaGetLastError());
    unsigned long long maxkey = (unsigned long long)c->nshg * (unsigned long long)c->nshg;
    int end_bit = 1;
    while (end_bit < 64 && (1ull << end_bit) <= maxkey) ++end_bit;
    size_t tb_sort = 0, tb_rle = 0, tb_scan = 0;
    cub::DoubleBuffer<unsigned long long> dk(keys.p, keys2.p);
    cub::DoubleBuffer<int> dv(vals.p, vals2.p);
    // LSD radix sort is stable: pairs of one slot keep ascending t
    CR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb_sort, dk, dv, np, 0, end_bit, s));
    CR_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, tb_rle, keys.p, ukeys.p, counts.p, dcount.p, np, s));
    CR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, counts.p, counts.p, np + 1, s));
    size_t tb = tb_sort > tb_rle ? tb_sort : tb_rle;
    if (tb_scan > tb) tb = tb_scan;
    DBuf<unsigned char> tmp;
    CR_CHECK(tmp.alloc(tb));
    CR_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb_sort, dk, dv, np, 0, end_bit, s));
    CR_CUDA(cub::DeviceRunLengthEncode::Encode(tmp.p, tb_rle, dk.Current(), ukeys.p, counts.p, dcount.p, np, s));
    int hnnz = 0;
    CR_CUDA(cudaMemcpyAsync(&hnnz, dcount.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    c->nnz = hnnz;
    CR_CHECK(c->rowptr.alloc((size_t)c->nshg + 1));
    CR_CHECK(c->col.alloc((size_t)hnnz));
    CR_CHECK(c->diag.alloc((size_t)c->nshg));
    CR_CHECK(c->trans.alloc((size_t)hnnz));
    CR_CHECK(c->soff.alloc((size_t)hnnz + 1));
    CR_CHECK(c->slist.alloc((size_t)npair));
    // soff = exclusive sum of the run lengths, soff[nnz] = npair
    CR_CUDA(cudaMemsetAsync(counts.p + hnnz, 0, sizeof(int), s));
    CR_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb_scan, counts.p, c->soff.p, hnnz + 1, s));
    CR_CUDA(cudaMemcpyAsync(c->slist.p, dv.Current(), sizeof(int) * (size_t)npair, cudaMemcpyDeviceToDevice, s));
    CR_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    launch(k_rowptr_cols, grid_for((long long)hnnz + c->nshg + 1, 256), 256, 0, s, ukeys.p, hnnz, c->nshg, c->rowptr.p,
                                                                              c->col.p);
    launch(k_diag_trans, grid_for(c->nshg, 128), 128, 0, s, c->rowptr.p, c->col.p, c->nshg, c->diag.p, c->trans.p,
                                                        bad.p);
    CR_CUDA(cudaGetLastError());
    int hbad = 0;
    CR_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    if (hbad) {
        set_last_error("pattern: missing diagonal / transposed block");
        return CRIMSON_ERR_PATTERN;
    }
    return CRIMSON_OK;
}

int pattern_to_host(crimson_ctx* c, int* colm, int* rowp, long long cap) {
    cudaStream_t s = c->stream;
    if (rowp && cap < c->nnz) return CRIMSON_ERR_ARG;
    DBuf<int> tmp;
    if (colm) {
        CR_CHECK(tmp.alloc((size_t)c->nshg + 1));
        launch(k_to_one_based, grid_for(c->nshg + 1, 256), 256, 0, s, c->rowptr.p, tmp.p, c->nshg + 1);
        CR_CUDA(cudaMemcpyAsync(colm, tmp.p, sizeof(int) * ((size_t)c->nshg + 1), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
    }
    if (rowp) {
        CR_CHECK(tmp.alloc((size_t)c->nnz));
        launch(k_to_one_based, grid_for(c->nnz, 256), 256, 0, s, c->col.p, tmp.p, c->nnz);
        CR_CUDA(cudaMemcpyAsync(rowp, tmp.p, sizeof(int) * (size_t)c->nnz, cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
    }
    return CRIMSON_OK;
}

}  // namespace crimson
