// 4x4 block SpMV, SPARMULVV with dof = 4 (flowsolver/src/memLS.f90:2024-2076):
//   KU(:, i) = sum_{j in row i} Val(:, :, j) U(:, col(j))
// on the ElmGMR pattern of a context, in FP64 or FP32.  memLS uses this
// product for the full 4-dof system (the GMRES/CG solvers of non-NS
// LS types); here it is the block-SpMV of the assembly / SpMV
// microbenchmark.
//
// Layout: the same 32-row sliced ELL as the Krylov SpMVs of memls.cu (one
// thread per row, coalesced 128-byte accesses, CSR summation order); each
// slice position holds its whole 4x4 block contiguously (4 rows of 4
// values: 128 B FP64 / 64 B FP32, read as 16-byte vectors), and U / KU are
// node-major 4-vectors (one aligned 32 B / 16 B load per gathered column).
// crimson_spmv4_prepare converts memLS's Val (16, nnz) once; apply then
// streams only the sliced copy.
#include "common.cuh"

namespace crimson {

int sell_build(const int* rowptr, const int* col, int n, cudaStream_t s, DBuf<int>& sell_ptr, DBuf<int>& sell_col,
               long long* npad_out, int* nslice_out);

namespace {

constexpr int kS4Slice = 32;
// entries issued together per thread: all their loads are hoisted ahead of
// the arithmetic (FP64: 160 B per entry in registers, FP32: 80 B)
template <typename T>
struct S4Unroll {
    static constexpr int value = 4;
};
template <>
struct S4Unroll<float> {
    static constexpr int value = 4;
};

template <typename T>
struct Vec4;
template <>
struct Vec4<double> {
    using type = double4;
    static __device__ __forceinline__ double4 load(const double4* p) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        return make_double4(a.x, a.y, b.x, b.y);
    }
    static __device__ __forceinline__ double4 make(double a, double b, double c, double d) {
        return make_double4(a, b, c, d);
    }
};
template <>
struct Vec4<float> {
    using type = float4;
    static __device__ __forceinline__ float4 load(const float4* p) { return __ldg(p); }
    static __device__ __forceinline__ float4 make(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
};

// memLS Val (16, nnz) row-major blocks -> sliced blocks
template <typename T>
__global__ void k_spmv4_to_sell(const int* __restrict__ rowptr, const int* __restrict__ sp, int n,
                                const T* __restrict__ val, typename Vec4<T>::type* __restrict__ out) {
    using V = Vec4<T>;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const size_t base = (size_t)sp[r / kS4Slice] + (r % kS4Slice);
        const int rs = rowptr[r], re = rowptr[r + 1];
        for (int j = rs; j < re; ++j) {
            const size_t pos = base + (size_t)kS4Slice * (j - rs);
            const T* v = val + 16 * (size_t)j;
#pragma unroll
            for (int a = 0; a < 4; ++a) out[4 * pos + a] = V::make(v[4 * a], v[4 * a + 1], v[4 * a + 2], v[4 * a + 3]);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_spmv4(const int* __restrict__ sp, const int* __restrict__ scol,
                                               const typename Vec4<T>::type* __restrict__ blk,
                                               const typename Vec4<T>::type* __restrict__ U,
                                               typename Vec4<T>::type* __restrict__ KU, int n) {
    using V = Vec4<T>;
    using T4 = typename V::type;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int s = r / kS4Slice;
        const int p0 = __ldg(sp + s);
        const int w = (__ldg(sp + s + 1) - p0) / kS4Slice;
        const int base = p0 + (r % kS4Slice);
        T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
        constexpr int UN = S4Unroll<T>::value;
        for (int k0 = 0; k0 < w; k0 += UN) {
            // entries past w are re-read from the row's first position (in
            // bounds) and not accumulated
            T4 x[UN], b0[UN], b1[UN], b2[UN], b3[UN];
#pragma unroll
            for (int u = 0; u < UN; ++u) {
                const size_t pos = (size_t)base + (size_t)kS4Slice * ((k0 + u < w) ? (k0 + u) : 0);
                x[u] = V::load(U + __ldg(scol + pos));
                b0[u] = V::load(blk + 4 * pos + 0);
                b1[u] = V::load(blk + 4 * pos + 1);
                b2[u] = V::load(blk + 4 * pos + 2);
                b3[u] = V::load(blk + 4 * pos + 3);
            }
#pragma unroll
            for (int u = 0; u < UN; ++u) {
                if (k0 + u < w) {
                    a0 = a0 + b0[u].x * x[u].x + b0[u].y * x[u].y + b0[u].z * x[u].z + b0[u].w * x[u].w;
                    a1 = a1 + b1[u].x * x[u].x + b1[u].y * x[u].y + b1[u].z * x[u].z + b1[u].w * x[u].w;
                    a2 = a2 + b2[u].x * x[u].x + b2[u].y * x[u].y + b2[u].z * x[u].z + b2[u].w * x[u].w;
                    a3 = a3 + b3[u].x * x[u].x + b3[u].y * x[u].y + b3[u].z * x[u].z + b3[u].w * x[u].w;
                }
            }
        }
        KU[r] = V::make(a0, a1, a2, a3);
    }
}

}  // namespace

int spmv4_prepare(crimson_ctx* c, int precision, const void* d_val) {
    cudaStream_t s = c->stream;
    if (!c->s4_ptr.p) CR_CHECK(sell_build(c->rowptr.p, c->col.p, c->nshg, s, c->s4_ptr, c->s4_col, &c->s4_npad,
                                          &c->s4_nslice));
    const size_t np = (size_t)c->s4_npad + (size_t)kS4Slice * 8;
    c->s4_prec = precision;
    if (precision == CRIMSON_FP64) {
        CR_CHECK(c->s4_val64.alloc(16 * np));
        CR_CUDA(cudaMemsetAsync(c->s4_val64.p, 0, sizeof(double) * c->s4_val64.n, s));
        launch(k_spmv4_to_sell<double>, grid_for(c->nshg, 256), 256, 0, s, (const int*)c->rowptr.p,
               (const int*)c->s4_ptr.p, c->nshg, (const double*)d_val, reinterpret_cast<double4*>(c->s4_val64.p));
    } else {
        CR_CHECK(c->s4_val32.alloc(16 * np));
        CR_CUDA(cudaMemsetAsync(c->s4_val32.p, 0, sizeof(float) * c->s4_val32.n, s));
        launch(k_spmv4_to_sell<float>, grid_for(c->nshg, 256), 256, 0, s, (const int*)c->rowptr.p,
               (const int*)c->s4_ptr.p, c->nshg, (const float*)d_val, reinterpret_cast<float4*>(c->s4_val32.p));
    }
    CR_CUDA(cudaStreamSynchronize(s));
    CR_CUDA(cudaGetLastError());
    return CRIMSON_OK;
}

int spmv4_apply(crimson_ctx* c, const void* d_u, void* d_ku) {
    cudaStream_t s = c->stream;
    const int grid = grid_for(c->nshg, 256, 8);
    if (c->s4_prec == CRIMSON_FP64) {
        if (!c->s4_val64.p) return CRIMSON_ERR_STATE;
        launch(k_spmv4<double>, grid, 256, 0, s, (const int*)c->s4_ptr.p, (const int*)c->s4_col.p,
               reinterpret_cast<const double4*>(c->s4_val64.p), (const double4*)d_u, (double4*)d_ku, c->nshg);
    } else {
        if (!c->s4_val32.p) return CRIMSON_ERR_STATE;
        launch(k_spmv4<float>, grid, 256, 0, s, (const int*)c->s4_ptr.p, (const int*)c->s4_col.p,
               reinterpret_cast<const float4*>(c->s4_val32.p), (const float4*)d_u, (float4*)d_ku, c->nshg);
    }
    CR_CUDA(cudaGetLastError());
    return CRIMSON_OK;
}

}  // namespace crimson
