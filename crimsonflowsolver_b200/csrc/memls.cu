// memLS NS linear solver on the device (flowsolver/src/memLS.f90).
//
// Layout: node-major vectors (dof, nNo) exactly as memLS's R(dof, nNo); block
// matrices split as DEPART does (memLS.f90:1612-1679) into mK (9, nnz),
// mG (3, nnz), mD (3, nnz), mL (nnz) and Gt (3, nnz).
//
// Two precisions share one implementation, templated on the matrix storage
// type M and the GMRES basis type B:
//   * FP64 (M = B = double): the plain path, same arithmetic as memLS.
//   * mixed (M = B = float): every inner Krylov matvec reads FP32 matrices
//     and the GMRES basis is FP32; FP64 is kept for the NSSOLVER outer
//     vectors and Gram system, every dot product / norm (FP64 accumulation),
//     the Givens rotations and back substitution, the CG recurrences, and a
//     final FP64 defect R - A x with iterative refinement.
//
// Kernels are HBM-bound: block SpMVs use four lanes per block row with four
// blocks per lane issued together; dot products and norms use a single-pass
// grid reduction whose last block sums the per-block partials in a fixed
// order (deterministic).  CGRAD runs as one persistent cooperative kernel per
// call.  The Krylov control flow (Givens rotations, back substitution, the
// 2i x 2i Gram system solved by GE) runs on the host in FP64 on scalars
// copied back per step, as the reference's serial code does.
//
// Modified Gram-Schmidt is fused: kernel j subtracts h(j-1) u_{j-1} from w and
// accumulates <w, u_j> in the same pass.
#include <cooperative_groups.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "memls.cuh"

namespace crimson {

// ---------------------------------------------------------------------------
// Small helpers
// ---------------------------------------------------------------------------
template <typename T>
struct V4;
template <>
struct V4<double> {
    using type = double4;
};
template <>
struct V4<float> {
    using type = float4;
};

__device__ __forceinline__ double4 ldg4(const double4* p) {
    const double2 lo = __ldg(reinterpret_cast<const double2*>(p));
    const double2 hi = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}
__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }
// Streaming (evict-first) loads for matrix streams that are read once per
// pass: they leave the L2 to the vectors and node records the same kernel
// gathers and re-reads (measured: the persistent CG 14% / 9% faster in
// FP32 / FP64 on the 4M-tet cylinder, the GMRES SpMV 8% in FP32).
__device__ __forceinline__ double4 ldcs4(const double4* p) {
    const double2 lo = __ldcs(reinterpret_cast<const double2*>(p));
    const double2 hi = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}
__device__ __forceinline__ float4 ldcs4(const float4* p) { return __ldcs(p); }
template <typename T>
__device__ __forceinline__ typename V4<T>::type mk4(T a, T b, T c, T d);
template <>
__device__ __forceinline__ double4 mk4<double>(double a, double b, double c, double d) {
    return make_double4(a, b, c, d);
}
template <>
__device__ __forceinline__ float4 mk4<float>(float a, float b, float c, float d) {
    return make_float4(a, b, c, d);
}

// ---------------------------------------------------------------------------
// Reductions: partial sums per block -> last block sums them in block order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void grid_reduce_finish(double bsum, double* part, unsigned int* ticket, double* out,
                                                   double* smem) {
    __shared__ bool am_last;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = bsum;
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (am_last) {
        __threadfence();
        double s = 0.0;
        for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) s += ((volatile double*)part)[b];
        s = block_sum(s, smem);
        if (threadIdx.x == 0) {
            *out = s;
            *ticket = 0u;
        }
    }
}

static int red_grid(long long n) {
    int g = grid_for(n, 256, 8);
    return g > RedScratch::kMaxBlocks ? RedScratch::kMaxBlocks : g;
}

// out = <u, v> (FP64 accumulation)
template <typename U, typename V>
__global__ void k_dot(const U* __restrict__ u, const V* __restrict__ v, long long n, double* part,
                      unsigned int* ticket, double* out) {
    __shared__ double sm[32];
    double s = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        s += (double)u[t] * (double)v[t];
    s = block_sum(s, sm);
    grid_reduce_finish(s, part, ticket, out, sm);
}

// MGS step: w -= (*hprev) * uprev (if uprev), then out = <w, uj>  (uj may be w -> squared norm)
template <typename B>
__global__ void k_mgs(B* w, const B* __restrict__ uprev, const double* __restrict__ hprev, const B* uj, long long n,
                      double* part, unsigned int* ticket, double* out) {
    __shared__ double sm[32];
    const double h = uprev ? *hprev : 0.0;
    double s = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        double wv = (double)w[t];
        if (uprev) {
            wv = (double)(B)(wv - h * (double)uprev[t]);
            w[t] = (B)wv;
        }
        s += wv * (uj == w ? wv : (double)uj[t]);
    }
    s = block_sum(s, sm);
    grid_reduce_finish(s, part, ticket, out, sm);
}

// y = y + a*x
template <typename X, typename Y>
__global__ void k_axpy(double a, const X* __restrict__ x, Y* __restrict__ y, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        y[t] = (Y)((double)y[t] + a * (double)x[t]);
}

// y = x / d (d on device; the reference divides)
template <typename B>
__global__ void k_divide(const B* x, const double* __restrict__ dptr, B* y, long long n, int take_sqrt) {
    double d = *dptr;
    if (take_sqrt) d = sqrt(d);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        y[t] = (B)((double)x[t] / d);
}

// z = x - y
template <typename A, typename Bt, typename C>
__global__ void k_sub(const A* x, const Bt* y, C* z, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        z[t] = (C)((double)x[t] - (double)y[t]);
}

// X += sum_j U_j y_j  (U_j at stride n), y on device
template <typename B>
__global__ void k_multi_axpy(double* __restrict__ X, const B* __restrict__ U, const double* __restrict__ yv, int m,
                             long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        double xv = X[t];
        for (int j = 0; j < m; ++j) xv = xv + (double)U[(size_t)j * n + t] * yv[j];
        X[t] = xv;
    }
}

__global__ void k_scale(double a, double* __restrict__ x, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        x[t] = a * x[t];
}

template <typename T, typename S>
__global__ void k_convert(const S* __restrict__ in, T* __restrict__ out, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        out[t] = (T)in[t];
}

// ---------------------------------------------------------------------------
// Block SpMVs (SPARMULVV/VS/SV/SS, memLS.f90:2024-2236).
// Four lanes per block row; each lane handles blocks j = s + lane + 4k and
// issues kUnroll of them together (column index, matrix values, gathered
// vector entries), so 16 independent loads per row are in flight instead of
// one dependent col -> x chain.  Matrix data is read through the read-only
// path (__ldg); evict-first loads measured slower on this pattern.
// ---------------------------------------------------------------------------
constexpr int kLanes = 4;
constexpr int kUnroll = 4;

__device__ __forceinline__ double group_sum(double v) {
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    return v;
}

// Rows handled by this thread's lane group: r = r0 + threadIdx.x / kLanes,
// r0 block-uniform so every lane of a warp reaches the shuffles.
#define CR_ROW_LOOP(n)                                                                          \
    const int lane = threadIdx.x & (kLanes - 1);                                                \
    const long long ngrp = (long long)gridDim.x * (blockDim.x / kLanes);                        \
    for (long long r0 = (long long)blockIdx.x * (blockDim.x / kLanes); r0 < (n); r0 += ngrp) { \
        const long long r = r0 + threadIdx.x / kLanes;                                          \
        const bool rv = r < (n);

// Unrolled visit of the blocks of row r: j and c defined for the body; ok marks valid blocks.
#define CR_ROW_BLOCKS(rowptr, col, ...)                                              \
    if (rv) {                                                                         \
        const int rs_ = (rowptr)[r], re_ = (rowptr)[r + 1];                           \
        for (int b0_ = rs_ + lane; b0_ < re_; b0_ += kLanes * kUnroll) {              \
            int cj_[kUnroll];                                                         \
            _Pragma("unroll") for (int k_ = 0; k_ < kUnroll; ++k_) {                  \
                const int j_ = b0_ + k_ * kLanes;                                     \
                cj_[k_] = __ldg((col) + (j_ < re_ ? j_ : b0_));                       \
            }                                                                         \
            _Pragma("unroll") for (int k_ = 0; k_ < kUnroll; ++k_) {                  \
                const int j0_ = b0_ + k_ * kLanes;                                    \
                const bool ok = j0_ < re_;                                            \
                const size_t j = (size_t)(ok ? j0_ : b0_);                            \
                const int c = cj_[k_];                                                \
                __VA_ARGS__                                                           \
            }                                                                         \
        }                                                                             \
    }

// KU = K U, K (9, nnz), U/KU (3, n)
template <typename M, typename IN, typename OUT>
__global__ void __launch_bounds__(256) k_spmv_vv3(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                  const M* __restrict__ K, const IN* __restrict__ U,
                                                  OUT* __restrict__ KU, int n) {
    CR_ROW_LOOP(n)
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    CR_ROW_BLOCKS(rowptr, col, {
        const M* k = K + 9 * j;
        const IN* u = U + 3 * (size_t)c;
        const double u0 = (double)u[0], u1 = (double)u[1], u2 = (double)u[2];
        const double k0 = (double)__ldg(k + 0), k1 = (double)__ldg(k + 1), k2 = (double)__ldg(k + 2),
                     k3 = (double)__ldg(k + 3), k4 = (double)__ldg(k + 4), k5 = (double)__ldg(k + 5),
                     k6 = (double)__ldg(k + 6), k7 = (double)__ldg(k + 7), k8 = (double)__ldg(k + 8);
        if (ok) {
            a0 += k0 * u0 + k1 * u1 + k2 * u2;
            a1 += k3 * u0 + k4 * u1 + k5 * u2;
            a2 += k6 * u0 + k7 * u1 + k8 * u2;
        }
    })
    a0 = group_sum(a0);
    a1 = group_sum(a1);
    a2 = group_sum(a2);
    if (rv && lane == 0) {
        KU[3 * r + 0] = (OUT)a0;
        KU[3 * r + 1] = (OUT)a1;
        KU[3 * r + 2] = (OUT)a2;
    }
    }
}

// KU(i) = sum K(:,j).U(:,col)  (3 -> 1)
template <typename M, typename IN, typename OUT>
__global__ void __launch_bounds__(256) k_spmv_vs3(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                  const M* __restrict__ K, const IN* __restrict__ U,
                                                  OUT* __restrict__ KU, int n) {
    CR_ROW_LOOP(n)
    double a = 0.0;
    CR_ROW_BLOCKS(rowptr, col, {
        const M* k = K + 3 * j;
        const IN* u = U + 3 * (size_t)c;
        const double t = (double)__ldg(k) * (double)u[0] + (double)__ldg(k + 1) * (double)u[1] +
                         (double)__ldg(k + 2) * (double)u[2];
        if (ok) a += t;
    })
    a = group_sum(a);
    if (rv && lane == 0) KU[r] = (OUT)a;
    }
}

// KU(:,i) = sum K(:,j) U(col)  (1 -> 3)
template <typename M, typename IN, typename OUT>
__global__ void __launch_bounds__(256) k_spmv_sv3(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                  const M* __restrict__ K, const IN* __restrict__ U,
                                                  OUT* __restrict__ KU, int n) {
    CR_ROW_LOOP(n)
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    CR_ROW_BLOCKS(rowptr, col, {
        const M* k = K + 3 * j;
        const double u = (double)U[c];
        const double k0 = (double)__ldg(k), k1 = (double)__ldg(k + 1), k2 = (double)__ldg(k + 2);
        if (ok) {
            a0 += k0 * u;
            a1 += k1 * u;
            a2 += k2 * u;
        }
    })
    a0 = group_sum(a0);
    a1 = group_sum(a1);
    a2 = group_sum(a2);
    if (rv && lane == 0) {
        KU[3 * r + 0] = (OUT)a0;
        KU[3 * r + 1] = (OUT)a1;
        KU[3 * r + 2] = (OUT)a2;
    }
    }
}

// KU = K U, scalar
template <typename M, typename IN, typename OUT>
__global__ void __launch_bounds__(256) k_spmv_ss(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                 const M* __restrict__ K, const IN* __restrict__ U,
                                                 OUT* __restrict__ KU, int n) {
    CR_ROW_LOOP(n)
    double a = 0.0;
    CR_ROW_BLOCKS(rowptr, col, {
        const double t = (double)__ldg(K + j) * (double)U[c];
        if (ok) a += t;
    })
    a = group_sum(a);
    if (rv && lane == 0) KU[r] = (OUT)a;
    }
}

// (G^T v)(c) = sum over row c of G(:, trans j) . v(:, col j)   (transposed SPARMULVS)
template <typename M>
__global__ void __launch_bounds__(256) k_spmv_vs3_trans(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                        const int* __restrict__ trans, const M* __restrict__ G,
                                                        const double* __restrict__ V, double* __restrict__ out, int n) {
    CR_ROW_LOOP(n)
    double acc = 0.0;
    CR_ROW_BLOCKS(rowptr, col, {
        const M* g = G + 3 * (size_t)trans[j];
        const double* v = V + 3 * (size_t)c;
        const double t = (double)g[0] * v[0] + (double)g[1] * v[1] + (double)g[2] * v[2];
        if (ok) acc += t;
    })
    acc = group_sum(acc);
    if (rv && lane == 0) out[r] = acc;
    }
}

// ---------------------------------------------------------------------------
// Sliced ELL copy of the pattern for the SpMVs inside the Krylov loops
// (GMRES's K products and the CG's G / {Gt, L} products).
// Rows are grouped in slices of 32 (one warp); a slice is stored column by
// column with width w = its longest row, so position of entry k of row r is
// sp[r / 32] + r % 32 + 32 k.  One thread per row: every load of column
// indices and matrix values is a fully coalesced 128-byte warp access, with
// no row-pointer -> column dependency; entries are summed in CSR order.
// Padding entries carry zero values and a valid column (the row itself;
// 0 for the rows past n of the last slice), so they add exactly +0.
// K is stored per component (structure of arrays, stride npad); the CG's
// operands as one 4-vector per entry: {G0, G1, G2, column} (one load gives
// the column and the values) and {Gt0, Gt1, Gt2, L}.  Converted once per NSSOLVER call,
// read ~10^3 times.
// ---------------------------------------------------------------------------
constexpr int kSlice = 32;
constexpr int kSellUnroll = 8;

// Visit the entries of row r, U at a time: pos (size_t) and c (int) defined
// for the body.
#define CR_SELL_ROW_U(U, sp, scol, r, ...)                                              \
    {                                                                                    \
        const int s_ = (r) >> 5;                                                         \
        const int p0_ = __ldg((sp) + s_);                                                \
        const int w_ = (__ldg((sp) + s_ + 1) - p0_) >> 5;                                \
        const int base_ = p0_ + ((r) & (kSlice - 1));                                    \
        for (int k0_ = 0; k0_ < w_; k0_ += (U)) {                                        \
            int cc_[(U)];                                                                \
            _Pragma("unroll") for (int u_ = 0; u_ < (U); ++u_) cc_[u_] =                 \
                (k0_ + u_ < w_) ? __ldg((scol) + base_ + kSlice * (k0_ + u_)) : 0;       \
            _Pragma("unroll") for (int u_ = 0; u_ < (U); ++u_) {                         \
                if (k0_ + u_ < w_) {                                                     \
                    const size_t pos = (size_t)base_ + (size_t)kSlice * (k0_ + u_);      \
                    const int c = cc_[u_];                                               \
                    __VA_ARGS__                                                          \
                }                                                                        \
            }                                                                            \
        }                                                                                \
    }
#define CR_SELL_ROW(sp, scol, r, ...) CR_SELL_ROW_U(kSellUnroll, sp, scol, r, __VA_ARGS__)
// Entries per stage of the CG's software-pipelined row loops: the matrix
// records of the next stage are loaded while the current stage's gathers are
// in flight (two stages live: 2 x 5 x 16 B FP32, 2 x 2 x 32 B FP64, within
// the 64 registers of two 512-thread blocks per SM).
template <typename M>
struct CgStage {
    static constexpr int value = 5;
};
template <>
struct CgStage<double> {
    static constexpr int value = 2;
};
// Phase A (G P) uses its own stage width (5 FP32 entries, 2 FP64: FP32
// measured 4% faster per iteration than 4, 6 spills; FP64 3 spills).
template <typename M>
struct CgStageA {
    static constexpr int value = sizeof(M) == 4 ? 5 : 2;
};

// KU = K U on the sliced copy: K as {K0..K3} and {K4..K7} 4-vectors (npad
// each, one 16/32-byte load apiece) and K8 (npad); U / KU (3, n).
template <typename M, typename IN, typename OUT>
__global__ void __launch_bounds__(256) k_sell_vv3(const int* __restrict__ sp, const int* __restrict__ scol,
                                                  const M* __restrict__ Ks, long long npad,
                                                  const IN* __restrict__ U, OUT* __restrict__ KU, int n) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        CR_SELL_ROW(sp, scol, r, {
            const IN* u = U + 3 * (size_t)c;
            const double u0 = (double)__ldg(u), u1 = (double)__ldg(u + 1), u2 = (double)__ldg(u + 2);
            const auto ka = ldcs4(reinterpret_cast<const typename V4<M>::type*>(Ks) + pos);
            const auto kb = ldcs4(reinterpret_cast<const typename V4<M>::type*>(Ks + 4 * npad) + pos);
            const double k0 = (double)ka.x, k1 = (double)ka.y, k2 = (double)ka.z, k3 = (double)ka.w,
                         k4 = (double)kb.x, k5 = (double)kb.y, k6 = (double)kb.z, k7 = (double)kb.w,
                         k8 = (double)__ldcs(Ks + 8 * npad + pos);
            a0 = a0 + k0 * u0 + k1 * u1 + k2 * u2;
            a1 = a1 + k3 * u0 + k4 * u1 + k5 * u2;
            a2 = a2 + k6 * u0 + k7 * u1 + k8 * u2;
        })
        KU[3 * (size_t)r + 0] = (OUT)a0;
        KU[3 * (size_t)r + 1] = (OUT)a1;
        KU[3 * (size_t)r + 2] = (OUT)a2;
    }
}

// Column index of every sliced position (pads: the row, or 0 past n).
__global__ void k_sell_cols(const int* __restrict__ rowptr, const int* __restrict__ col, const int* __restrict__ sp,
                            int n, int nrows_pad, int* __restrict__ scol) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows_pad; r += gridDim.x * blockDim.x) {
        const int s = r >> 5;
        const int w = (sp[s + 1] - sp[s]) >> 5;
        const int base = sp[s] + (r & (kSlice - 1));
        const int rs = r < n ? rowptr[r] : 0;
        const int len = r < n ? rowptr[r + 1] - rs : 0;
        for (int k = 0; k < w; ++k) scol[base + kSlice * k] = k < len ? col[rs + k] : (r < n ? r : 0);
    }
}

// Largest |col - row| of a CSR pattern (atomicMax into *out).
__global__ void k_max_offset(const int* __restrict__ rowptr, const int* __restrict__ col, int n, int* out) {
    int m = 0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        for (int j = rowptr[r]; j < rowptr[r + 1]; ++j) m = max(m, abs(col[j] - r));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Scaled split matrices (CSR, type M) -> sliced copies: K as two 4-vector
// arrays and one scalar array (npad each), G (3, npad) per component,
// {Gt0, Gt1, Gt2, L} (npad).
template <typename M>
__global__ void k_to_sell(const int* __restrict__ rowptr, const int* __restrict__ sp, int n,
                          const double* __restrict__ mK, const double* __restrict__ mG, const double* __restrict__ Gt,
                          const double* __restrict__ mL, long long npad, M* __restrict__ Ks, M* __restrict__ Gs,
                          typename V4<M>::type* __restrict__ GLs) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const size_t base = (size_t)sp[r >> 5] + (r & (kSlice - 1));
        const int rs = rowptr[r], re = rowptr[r + 1];
        for (int j = rs; j < re; ++j) {
            const size_t pos = base + (size_t)kSlice * (j - rs);
            const size_t jj = (size_t)j;
            reinterpret_cast<typename V4<M>::type*>(Ks)[pos] =
                mk4<M>((M)mK[9 * jj], (M)mK[9 * jj + 1], (M)mK[9 * jj + 2], (M)mK[9 * jj + 3]);
            reinterpret_cast<typename V4<M>::type*>(Ks + 4 * npad)[pos] =
                mk4<M>((M)mK[9 * jj + 4], (M)mK[9 * jj + 5], (M)mK[9 * jj + 6], (M)mK[9 * jj + 7]);
            Ks[8 * npad + pos] = (M)mK[9 * jj + 8];
#pragma unroll
            for (int q = 0; q < 3; ++q) Gs[q * npad + pos] = (M)mG[3 * jj + q];
            GLs[pos] = mk4<M>((M)Gt[3 * jj], (M)Gt[3 * jj + 1], (M)Gt[3 * jj + 2], (M)mL[jj]);
        }
    }
}

// ---------------------------------------------------------------------------
// CGRAD as one persistent cooperative kernel (memLS.f90:367-430).
//
// Per iteration three grid-wide barriers: (A) P = R + beta P formed on the
// fly while computing GP = G P, plus the coupled-face dots w_f . P; (B)
// SP = L P - Gt GP - sum_f coef_f (w_f . P) z_f and <P, SP>; (C) X += alpha P,
// R -= alpha SP, |R|^2.  The coupled-face (Sherman-Morrison) term of
// ADDBCMUL(PRE) is applied through the precomputed vectors w_f = G^T valM_f
// and z_f = Gt valM_f: Gt (GP + coef valM (valM . GP)) = Gt GP + coef (w.P) z
// -- exact.  Node records keep every gather to one aligned sector:
// recA = {R, P_prev} (16 B, FP64) read in phase A, recB = {GP, P} read in
// phase B, stored in the matrix type M (32 B FP64 / 16 B FP32: with FP32
// matrices the matvec operands are rounded to FP32 as the matrices are,
// while P itself stays FP64 for the updates); matrix entries G per
// component (three coalesced streams) and {Gt0, Gt1, Gt2, L}; the column
// indices block-resident in shared memory where they fit (CgCols).  Partial sums are written per block
// and summed in block order by every block after the barrier
// (deterministic, identical in all blocks).  Node records written by other
// blocks in an earlier phase are read with ordinary (L1-cached) loads: the
// grid barrier's acquire fence orders them after those writes, and the
// neighbour gathers of one block hit the same lines many times.  The matrix
// streams use evict-first loads (each value is read once per phase), so the
// node records and per-row vectors (~40 MB on the 4M-tet cylinder) stay in
// the 126 MB L2 from one phase to the next.  The loop
// is bounded by mItr.  X, R, P, SP, the recurrences and all dot products
// are FP64 in both precisions; M is the storage type of G, Gt, L and of
// the gathered copy of {GP, P}.
// ---------------------------------------------------------------------------
constexpr int kMaxCoupled = 8;
// 512-thread blocks, two per SM: half the blocks of 256-thread blocks at
// every grid barrier and block-order reduction (measured 2% per iteration).
constexpr int kCgThreads = 512;

template <typename M>
struct CgArgs {
    const int* sp;    // sliced pattern: slice offsets
    const int* scol;  // sliced pattern: columns (read when the columns are not block-resident)
    long long npad;
    int n;
    const M* G;                      // sliced G per component: G0 at [0, npad), G1, G2 (stride npad)
    const typename V4<M>::type* GL;  // sliced (npad) {Gt0, Gt1, Gt2, L}
    double* X;
    double2* recA;  // (n) {R, P of the previous iteration}
    typename V4<M>::type* recB;  // (n) {GP0, GP1, GP2, P} rounded to M: the gathered copy
    double* Pd;                  // (n) P in FP64 for the updates
    double* SP;
    int nface;
    const double* w;  // (nface, n)
    const double* z;  // (nface, n)
    double coef[kMaxCoupled];
    double eps;   // squared tolerance
    double err0;  // squared initial norm
    int mItr;
    double* part;  // 3 regions of kCgPartStride * gridDim
    double* out;   // err, errO, i, suc
};
constexpr int kCgPartStride = kMaxCoupled + 2;

__device__ __forceinline__ double sum_partials(const double* part, int k, double* sm) {
    double s = 0.0;
    for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) s += __ldcg(part + (size_t)b * kCgPartStride + k);
    return block_sum(s, sm);
}

// Column source of the CG row loops.  Block-resident (kRes): every block
// copies the columns of its own rows into shared memory once per launch, as
// 16-bit offsets col - row, and the iterations read no column index from
// HBM (4 B per entry and phase).  A warp's rows are whole slices (32 rows),
// so a warp's columns are the concatenation of its slices' column ranges in
// sliced order; entry k of a row sits at off + 32 k + lane, where off
// advances by the slice's length after each row.  Otherwise the columns are
// read from the sliced pattern.
template <bool kRes>
struct CgCols {
    const int* scol;
    const short* res;  // this warp's resident offsets (kRes)
    int off;           // offset of the current row's slice within res
    int lane;
    __device__ __forceinline__ int col(int r, int base, int k) const {
        if (kRes) return r + (int)res[off + kSlice * k + lane];
        return __ldg(scol + base + kSlice * k);
    }
    __device__ __forceinline__ void next_row(int w) {
        if (kRes) off += kSlice * w;
    }
};

// Fill this block's resident column offsets; returns this warp's base.
__device__ int cg_fill_cols(const int* __restrict__ sp, const int* __restrict__ scol, int n, short* res) {
    __shared__ int woff[kCgThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int s0 = (blockIdx.x * kCgThreads + wid * kSlice) / kSlice;
    const int sstride = gridDim.x * (kCgThreads / kSlice);
    const int nsl = (n + kSlice - 1) / kSlice;
    int tot = 0;
    for (int s = s0 + lane * sstride; s < nsl; s += 32 * sstride) tot += __ldg(sp + s + 1) - __ldg(sp + s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (lane == 0) woff[wid] = tot;
    __syncthreads();
    int base = 0;
    for (int q = 0; q < wid; ++q) base += woff[q];
    int off = base;
    for (int s = s0; s < nsl; s += sstride) {
        const int p0 = __ldg(sp + s), len = __ldg(sp + s + 1) - p0;
        const int row = s * kSlice + lane;  // position p0 + j belongs to row s*32 + j%32
        for (int j = lane; j < len; j += 32) res[off + j] = row < n ? (short)(__ldg(scol + p0 + j) - row) : (short)0;
        off += len;
    }
    __syncthreads();
    return base;
}

template <int NF, typename M, bool kRes>
__global__ void __launch_bounds__(kCgThreads, 2) k_cg_persistent(CgArgs<M> a) {
    namespace cgrp = cooperative_groups;
    cgrp::grid_group grid = cgrp::this_grid();
    extern __shared__ short cg_res[];
    __shared__ double sm[32];
    const int n = a.n;
    const long long npad = a.npad;
    double* partA = a.part;
    double* partB = a.part + (size_t)gridDim.x * kCgPartStride;
    double* partC = a.part + 2 * (size_t)gridDim.x * kCgPartStride;
    const int wbase = kRes ? cg_fill_cols(a.sp, a.scol, n, cg_res) : 0;
    constexpr int U = CgStage<M>::value;
    constexpr int UA = CgStageA<M>::value;
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
        // ---- phase A: P = R + beta P_prev (on the fly), GP = G P, w_f . P ----
        double wp[NF > 0 ? NF : 1];
#pragma unroll
        for (int f = 0; f < (NF > 0 ? NF : 1); ++f) wp[f] = 0.0;
        CgCols<kRes> cs{a.scol, cg_res, wbase, (int)(threadIdx.x & 31)};
        for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
            double a0 = 0.0, a1 = 0.0, a2 = 0.0;
            const int s_ = r >> 5;
            const int p0 = __ldg(a.sp + s_);
            const int w = (__ldg(a.sp + s_ + 1) - p0) >> 5;
            const int base = p0 + (r & (kSlice - 1));
            // stage: G values and columns of U entries; the next stage is
            // loaded before this stage's gathers
            M g0[UA], g1[UA], g2[UA];
            int cc[UA];
#pragma unroll
            for (int u = 0; u < UA; ++u) {
                const bool in = u < w;
                const size_t pos = (size_t)base + kSlice * u;
                g0[u] = in ? __ldcs(a.G + pos) : M(0);
                g1[u] = in ? __ldcs(a.G + npad + pos) : M(0);
                g2[u] = in ? __ldcs(a.G + 2 * npad + pos) : M(0);
                cc[u] = (!kRes && in) ? cs.col(r, base, u) : r;  // resident columns are read at use
            }
            for (int k0 = 0; k0 < w; k0 += UA) {
                M n0[UA], n1[UA], n2[UA];
                int nc[UA];
#pragma unroll
                for (int u = 0; u < UA; ++u) {
                    const bool in = k0 + UA + u < w;
                    const size_t pos = (size_t)base + kSlice * (k0 + UA + u);
                    n0[u] = in ? __ldcs(a.G + pos) : M(0);
                    n1[u] = in ? __ldcs(a.G + npad + pos) : M(0);
                    n2[u] = in ? __ldcs(a.G + 2 * npad + pos) : M(0);
                    nc[u] = (!kRes && in) ? cs.col(r, base, k0 + UA + u) : r;
                }
#pragma unroll
                for (int u = 0; u < UA; ++u) {
                    if (k0 + u < w) {
                        const double2 rp = a.recA[kRes ? cs.col(r, base, k0 + u) : cc[u]];
                        const double pc = first ? rp.x : rp.x + beta * rp.y;
                        a0 = a0 + (double)g0[u] * pc;
                        a1 = a1 + (double)g1[u] * pc;
                        a2 = a2 + (double)g2[u] * pc;
                    }
                }
#pragma unroll
                for (int u = 0; u < UA; ++u) {
                    g0[u] = n0[u];
                    g1[u] = n1[u];
                    g2[u] = n2[u];
                    cc[u] = nc[u];
                }
            }
            cs.next_row(w);
            const double2 rr = a.recA[r];
            const double pr = first ? rr.x : rr.x + beta * rr.y;
            a.recB[r] = mk4<M>((M)a0, (M)a1, (M)a2, (M)pr);
            a.Pd[r] = pr;
#pragma unroll
            for (int f = 0; f < NF; ++f)
                if (f < a.nface) wp[f] += a.w[(size_t)f * n + r] * pr;
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            if (f < a.nface) {
                double t = block_sum(wp[f], sm);
                if (threadIdx.x == 0) partA[(size_t)blockIdx.x * kCgPartStride + f] = t;
            }
        }
        grid.sync();
        double cS[NF > 0 ? NF : 1];
#pragma unroll
        for (int f = 0; f < NF; ++f) cS[f] = f < a.nface ? a.coef[f] * sum_partials(partA, f, sm) : 0.0;
        // ---- phase B: SP = L P - Gt GP - sum_f cS_f z_f ; <P, SP> ----
        double dsum = 0.0;
        CgCols<kRes> cb{a.scol, cg_res, wbase, (int)(threadIdx.x & 31)};
        for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
            double lp = 0.0, gg = 0.0;
            const auto zero4 = mk4<M>(M(0), M(0), M(0), M(0));
            const int s_ = r >> 5;
            const int p0 = __ldg(a.sp + s_);
            const int w = (__ldg(a.sp + s_ + 1) - p0) >> 5;
            const int base = p0 + (r & (kSlice - 1));
            int cc[U];
            typename V4<M>::type gl[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                cc[u] = (!kRes && u < w) ? cb.col(r, base, u) : r;
                gl[u] = (u < w) ? ldcs4(a.GL + base + kSlice * u) : zero4;
            }
            for (int k0 = 0; k0 < w; k0 += U) {
                int ccn[U];  // next stage
                typename V4<M>::type gln[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const bool in = k0 + U + u < w;
                    ccn[u] = (!kRes && in) ? cb.col(r, base, k0 + U + u) : r;
                    gln[u] = in ? ldcs4(a.GL + base + kSlice * (k0 + U + u)) : zero4;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (k0 + u < w) {
                        const auto q = a.recB[kRes ? cb.col(r, base, k0 + u) : cc[u]];
                        lp = lp + (double)gl[u].w * (double)q.w;
                        gg = gg + (double)gl[u].x * (double)q.x + (double)gl[u].y * (double)q.y +
                             (double)gl[u].z * (double)q.z;
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    cc[u] = ccn[u];
                    gl[u] = gln[u];
                }
            }
            cb.next_row(w);
#pragma unroll
            for (int f = 0; f < NF; ++f)
                if (f < a.nface) gg += cS[f] * a.z[(size_t)f * n + r];
            const double v = lp - gg;
            a.SP[r] = v;
            dsum += a.Pd[r] * v;
        }
        dsum = block_sum(dsum, sm);
        if (threadIdx.x == 0) partB[(size_t)blockIdx.x * kCgPartStride] = dsum;
        grid.sync();
        const double alpha = errO / sum_partials(partB, 0, sm);
        // ---- phase C: X += alpha P, R -= alpha SP, |R|^2 ; recA = {R, P} ----
        double rs = 0.0;
        for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
             t += (long long)gridDim.x * blockDim.x) {
            const double pv = a.Pd[t];
            a.X[t] = a.X[t] + alpha * pv;
            const double rv = a.recA[t].x - alpha * a.SP[t];
            a.recA[t] = make_double2(rv, pv);
            rs += rv * rv;
        }
        rs = block_sum(rs, sm);
        if (threadIdx.x == 0) partC[(size_t)blockIdx.x * kCgPartStride] = rs;
        grid.sync();
        const double e2 = sqrt(sum_partials(partC, 0, sm));
        err = e2 * e2;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = err;
        a.out[1] = errO;
        a.out[2] = (double)i;
        a.out[3] = (double)suc;
    }
}

// recA = {R, 0}
__global__ void k_cg_init(const double* __restrict__ R, double2* __restrict__ recA, int n) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) recA[t] = make_double2(R[t], 0.0);
}

// ext = valM scattered into a (3, n) vector
__global__ void k_face_ext(const int* __restrict__ glob, const double* __restrict__ valM, int fdof, int nsd, int nNoF,
                           double* __restrict__ ext) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nNoF; a += gridDim.x * blockDim.x)
        for (int i = 0; i < nsd; ++i) ext[3 * (size_t)glob[a] + i] = valM[(size_t)fdof * a + i];
}

// ---------------------------------------------------------------------------
// ADDBCMUL pieces (memLS.f90:206-268): S = <valM, X> over face nodes; Y += S*coef*valM
// ---------------------------------------------------------------------------
template <typename V>
__global__ void k_face_dot(const int* __restrict__ glob, const double* __restrict__ valM, int fdof, int nsd,
                           int nNoF, const V* __restrict__ X, int dof, double* part, unsigned int* ticket,
                           double* out) {
    __shared__ double sm[32];
    double s = 0.0;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nNoF; a += gridDim.x * blockDim.x) {
        const int Ac = glob[a];
        for (int i = 0; i < nsd; ++i) s += valM[(size_t)fdof * a + i] * (double)X[(size_t)dof * Ac + i];
    }
    s = block_sum(s, sm);
    grid_reduce_finish(s, part, ticket, out, sm);
}

template <typename V>
__global__ void k_face_axpy(const int* __restrict__ glob, const double* __restrict__ valM, int fdof, int nsd,
                            int nNoF, const double* Sptr, double coef, V* __restrict__ Y, int dof) {
    const double S = coef * *Sptr;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nNoF; a += gridDim.x * blockDim.x) {
        const int Ac = glob[a];
        for (int i = 0; i < nsd; ++i)
            Y[(size_t)dof * Ac + i] = (V)((double)Y[(size_t)dof * Ac + i] + valM[(size_t)fdof * a + i] * S);
    }
}

// ---------------------------------------------------------------------------
// PRECOND (memLS.f90:1763-1943) pieces
// ---------------------------------------------------------------------------
// W from the diagonal blocks of Val (dof = 4, row-major 16 per block)
__global__ void k_w_from_val(double* __restrict__ Val, const int* __restrict__ diag, double* __restrict__ W, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double* v = Val + 16 * (size_t)diag[i];
        for (int d = 0; d < 4; ++d) {
            double w = v[5 * d];
            if (w == 0.0) {
                w = 1.0;
                v[5 * d] = 1.0;
            }
            W[4 * (size_t)i + d] = 1.0 / sqrt(fabs(w));
        }
    }
}

// Tangent block j as ElmGMR produced it: FP64 lhsK (9, nnz) / lhsP (4, nnz),
// or FP32 records of 16 floats (K(9), P(4), pads) when rec is not null.
struct TangentIn {
    const double* lhsK;
    const double* lhsP;
    const float* rec;
    __device__ __forceinline__ double K(size_t j, int t) const {
        return rec ? (double)rec[16 * j + t] : lhsK[9 * j + t];
    }
    __device__ __forceinline__ double P(size_t j, int t) const {
        return rec ? (double)rec[16 * j + 9 + t] : lhsP[4 * j + t];
    }
};

// W from lhsK / lhsP diagonals (fused SolFlow path; Val4 diagonal = K11,K22,K33,C)
__global__ void k_w_from_lhs(TangentIn T, const int* __restrict__ diag, double* __restrict__ W, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t k = (size_t)diag[i];
        double w[4] = {T.K(k, 0), T.K(k, 4), T.K(k, 8), T.P(k, 3)};
        for (int d = 0; d < 4; ++d) {
            double v = w[d] == 0.0 ? 1.0 : w[d];
            W[4 * (size_t)i + d] = 1.0 / sqrt(fabs(v));
        }
    }
}

// W(1:i, glob) *= val  (Dirichlet faces)
__global__ void k_w_dirichlet(const int* __restrict__ glob, const double* __restrict__ val, int fdof, int ni, int nNoF,
                              double* __restrict__ W) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nNoF; a += gridDim.x * blockDim.x) {
        const int Ac = glob[a];
        for (int i = 0; i < ni; ++i) W[4 * (size_t)Ac + i] = W[4 * (size_t)Ac + i] * val[(size_t)fdof * a + i];
    }
}

// Row then column scaling of Val (16 per block) + zero-diagonal fix + DEPART split
__global__ void k_scale_split_val(double* __restrict__ Val, const int* __restrict__ rowptr, const int* __restrict__ col,
                                  const int* __restrict__ diag, const double* __restrict__ W, int n,
                                  double* __restrict__ mK, double* __restrict__ mG, double* __restrict__ mD,
                                  double* __restrict__ mL) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const double* wr = W + 4 * (size_t)r;
        for (int j = rowptr[r]; j < rowptr[r + 1]; ++j) {
            const double* wc = W + 4 * (size_t)col[j];
            double* v = Val + 16 * (size_t)j;
            double t[16];
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b) t[4 * a + b] = (v[4 * a + b] * wr[a]) * wc[b];
            if (j == diag[r])
                for (int a = 0; a < 4; ++a)
                    if (t[5 * a] == 0.0) t[5 * a] = 1.0;
            for (int q = 0; q < 16; ++q) v[q] = t[q];
            double* k = mK + 9 * (size_t)j;
            k[0] = t[0]; k[1] = t[1]; k[2] = t[2];
            k[3] = t[4]; k[4] = t[5]; k[5] = t[6];
            k[6] = t[8]; k[7] = t[9]; k[8] = t[10];
            mG[3 * (size_t)j + 0] = t[3];
            mG[3 * (size_t)j + 1] = t[7];
            mG[3 * (size_t)j + 2] = t[11];
            mD[3 * (size_t)j + 0] = t[12];
            mD[3 * (size_t)j + 1] = t[13];
            mD[3 * (size_t)j + 2] = t[14];
            mL[j] = t[15];
        }
    }
}

// Gt(:, l) = -mG(:, trans(l))  (DEPART's transpose search, memLS.f90:1664-1675)
__global__ void k_gt(const double* __restrict__ mG, const int* __restrict__ trans, long long nnz, double* __restrict__ Gt) {
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < nnz; l += (long long)gridDim.x * blockDim.x) {
        const size_t j = (size_t)trans[l];
        Gt[3 * l + 0] = -mG[3 * j + 0];
        Gt[3 * l + 1] = -mG[3 * j + 1];
        Gt[3 * l + 2] = -mG[3 * j + 2];
    }
}

// Fused SolFlow pack + PRECOND scaling + DEPART from lhsK / lhsP:
//   Val4 rows 1-3 cols 1-3 = lhsK, col 4 rows 1-3 = -lhsP(1:3) of the
//   transposed block, row 4 cols 1-3 = lhsP(1:3), (4,4) = lhsP(4)
//   (solfar.f90:217-232), scaled by W(row) W(col) and split.
__global__ void k_scale_split_lhs(TangentIn T, const int* __restrict__ rowptr, const int* __restrict__ col,
                                  const int* __restrict__ diag, const int* __restrict__ trans,
                                  const double* __restrict__ W, int n, double* __restrict__ mK,
                                  double* __restrict__ mG, double* __restrict__ mD, double* __restrict__ mL) {
    // 16 lanes per row, one entry per lane: the block reads and writes of a
    // row are contiguous across the lanes
    const int sub = threadIdx.x & 15;
    const int ngroup = (gridDim.x * blockDim.x) >> 4;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; r < n; r += ngroup) {
        const double* wr = W + 4 * (size_t)r;
        const int dg = diag[r];
        for (int j = rowptr[r] + sub; j < rowptr[r + 1]; j += 16) {
            const double* wc = W + 4 * (size_t)col[j];
            const size_t jj = (size_t)j, jt = (size_t)trans[j];
            const double Pj[4] = {T.P(jj, 0), T.P(jj, 1), T.P(jj, 2), T.P(jj, 3)};
            const double Pt[3] = {T.P(jt, 0), T.P(jt, 1), T.P(jt, 2)};
            double* k = mK + 9 * (size_t)j;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    double v = T.K(jj, 3 * a + b);
                    if (j == dg && a == b && v == 0.0) v = 1.0;
                    double t = (v * wr[a]) * wc[b];
                    if (j == dg && a == b && t == 0.0) t = 1.0;
                    k[3 * a + b] = t;
                }
            for (int a = 0; a < 3; ++a) mG[3 * (size_t)j + a] = (-Pt[a] * wr[a]) * wc[3];
            for (int b = 0; b < 3; ++b) mD[3 * (size_t)j + b] = (Pj[b] * wr[3]) * wc[b];
            double v = Pj[3];
            if (j == dg && v == 0.0) v = 1.0;
            double t = (v * wr[3]) * wc[3];
            if (j == dg && t == 0.0) t = 1.0;
            mL[j] = t;
        }
    }
}

// R = W*R  (node-major, dof 4), and R = R*W afterwards
__global__ void k_mul(double* __restrict__ R, const double* __restrict__ W, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        R[t] = W[t] * R[t];
}

// split (4, n) into (3, n) and (n), and merge back
__global__ void k_split4(const double* __restrict__ R, double* __restrict__ Rm, double* __restrict__ Rc, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Rm[3 * (size_t)i + 0] = R[4 * (size_t)i + 0];
        Rm[3 * (size_t)i + 1] = R[4 * (size_t)i + 1];
        Rm[3 * (size_t)i + 2] = R[4 * (size_t)i + 2];
        Rc[i] = R[4 * (size_t)i + 3];
    }
}
__global__ void k_merge4(double* __restrict__ R, const double* __restrict__ Rm, const double* __restrict__ Rc, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        R[4 * (size_t)i + 0] = Rm[3 * (size_t)i + 0];
        R[4 * (size_t)i + 1] = Rm[3 * (size_t)i + 1];
        R[4 * (size_t)i + 2] = Rm[3 * (size_t)i + 2];
        R[4 * (size_t)i + 3] = Rc[i];
    }
}

// face%valM = face%val * W  (coupled faces)
__global__ void k_valm(const int* __restrict__ glob, const double* __restrict__ val, double* __restrict__ valM, int fdof,
                       int ni, int nNoF, const double* __restrict__ W) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nNoF; a += gridDim.x * blockDim.x)
        for (int i = 0; i < ni; ++i)
            valM[(size_t)fdof * a + i] = val[(size_t)fdof * a + i] * W[4 * (size_t)glob[a] + i];
}

// Defect of the scaled NS system: D4 = R4 - [K u + G p ; D u + L p] given
// KU = K u (+ coupling), GP = G p, DU = D u, LP = L p (all FP64).
__global__ void k_defect4(const double* __restrict__ R4, const double* __restrict__ KU,
                          const double* __restrict__ GPm, const double* __restrict__ DU,
                          const double* __restrict__ LP, double* __restrict__ D4, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int d = 0; d < 3; ++d)
            D4[4 * (size_t)i + d] = R4[4 * (size_t)i + d] - (KU[3 * (size_t)i + d] + GPm[3 * (size_t)i + d]);
        D4[4 * (size_t)i + 3] = R4[4 * (size_t)i + 3] - (DU[i] + LP[i]);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// device scalar slots
enum {
    kSlotDot = 0,
    kSlotNrm = 1,
    kSlotErr = 2,
    kSlotErrO = 3,
    kSlotDen = 4,
    kSlotFace = 8,      // up to 16 faces
    kSlotCg = 24,       // persistent CG outputs (4)
    kSlotH = 64,        // Hessenberg column (sD + 1)
    kSlotY = 64 + 512,  // back-substitution coefficients
    kSlotGram = 64 + 1024,
    kScalTotal = 64 + 1024 + 4096
};

struct Ctx {
    crimson_lhs* L;
    cudaStream_t s;
    double* sc(int i) { return L->scal.p + i; }
    int sync_scal(int first, int count) {
        CR_CUDA(cudaMemcpyAsync(L->hscal + first, L->scal.p + first, sizeof(double) * count, cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        return CRIMSON_OK;
    }
    template <typename U, typename V>
    void dot(const U* u, const V* v, long long n, int slot) {
        launch(k_dot<U, V>, red_grid(n), 256, 0, s, u, v, n, L->red.part.p, L->red.ticket.p, sc(slot));
    }
    int spmv_grid() const { return grid_for((long long)L->nNo * kLanes, 256, 8); }
    template <typename M, typename IN, typename OUT>
    void vv3(const M* K, const IN* U, OUT* KU) {
        launch(k_spmv_vv3<M, IN, OUT>, spmv_grid(), 256, 0, s, L->rowptr, L->col, K, U, KU, L->nNo);
    }
    template <typename M, typename IN, typename OUT>
    void vs3(const M* K, const IN* U, OUT* KU) {
        launch(k_spmv_vs3<M, IN, OUT>, spmv_grid(), 256, 0, s, L->rowptr, L->col, K, U, KU, L->nNo);
    }
    template <typename M, typename IN, typename OUT>
    void sv3(const M* K, const IN* U, OUT* KU) {
        launch(k_spmv_sv3<M, IN, OUT>, spmv_grid(), 256, 0, s, L->rowptr, L->col, K, U, KU, L->nNo);
    }
    template <typename M, typename IN, typename OUT>
    void ss(const M* K, const IN* U, OUT* KU) {
        launch(k_spmv_ss<M, IN, OUT>, spmv_grid(), 256, 0, s, L->rowptr, L->col, K, U, KU, L->nNo);
    }
    template <typename M, typename IN, typename OUT>
    void vv3s(const M* Ks, const IN* U, OUT* KU) {
        launch(k_sell_vv3<M, IN, OUT>, grid_for(L->nNo, 256, 8), 256, 0, s, (const int*)L->sell_ptr.p,
               (const int*)L->sell_col.p, Ks, L->npad, U, KU, L->nNo);
    }
    bool any_coupled() const {
        for (auto& f : L->face)
            if (f.coupledFlag) return true;
        return false;
    }
    // ADDBCMUL on nsd-dof vectors: all face dots first (on X), then all updates of Y
    template <typename VX, typename VY>
    void addbcmul(int op, int dof, const VX* X, VY* Y) {
        int k = 0;
        for (auto& f : L->face) {
            if (f.coupledFlag) {
                int nsd = std::min(f.dof, dof);
                // a few nodes per thread: the face dot is a chain of gathers
                int g = (f.nNo + 4 * 128 - 1) / (4 * 128);
                g = std::max(1, std::min(g, (int)RedScratch::kMaxBlocks));
                launch(k_face_dot<VX>, g, 128, 0, s, f.glob.p, f.valM.p, f.dof, nsd, f.nNo, X, dof, L->red.part.p,
                       L->red.ticket.p, sc(kSlotFace + k));
            }
            ++k;
        }
        k = 0;
        for (auto& f : L->face) {
            if (f.coupledFlag) {
                int nsd = std::min(f.dof, dof);
                double coef = (op == 0) ? f.res : -f.res / (1.0 + f.res * f.nS);
                launch(k_face_axpy<VY>, grid_for(f.nNo, 256), 256, 0, s, f.glob.p, f.valM.p, f.dof, nsd, f.nNo,
                       (const double*)sc(kSlotFace + k), coef, Y, dof);
            }
            ++k;
        }
    }
};

// ---------------------------------------------------------------------------
// One GMRES restart cycle (memLS.f90:715-770) as one persistent cooperative
// kernel: Arnoldi iterations i = 1..sD with the fused modified Gram-Schmidt
// order of the launch-per-step path, until |err_i| < eps.  Per iteration:
// (P1) U(i) = K U(i-1) on the sliced K, with the coupled-face dots
// S0_f = valM_f . U(i-1) and T_f = valM_f . K U(i-1) of ADDBCMUL; (MGS j)
// the face terms of ADDBCMUL (op 0, then op 1 with S1_f = T_f + sum_g
// coef0_g S0_g (valM_f . valM_g)) folded into the first pass, then
// U(i) -= h_{j-1} U(j-2) and h_j = <U(i), U(j-1)>; (norm) U(i) -= h_i U(i-1)
// and |U(i)|^2; every block then applies the Givens rotations to the new
// Hessenberg column (identical arithmetic in every block, so the exit test
// agrees) and block 0 stores the column and err; (normalize) U(i) /= h_{i+1}.
// Every reduction is written per block and summed in block order after the
// grid barrier (two alternating partial regions).  No host round trip per
// iteration; the host does the back substitution and X update per cycle.
// ---------------------------------------------------------------------------
constexpr int kGmThreads = 512;
constexpr int kGmMaxSD = 64;
constexpr int kGmPartStride = 2 * kMaxCoupled + 1;

template <typename M, typename B>
struct GmArgs {
    const int* sp;
    const int* scol;
    long long npad;
    int n;
    const M* Ks;          // sliced K: {K0..K3} (npad), {K4..K7} (npad), K8 (npad)
    B* u;                 // basis, vector k at u + k n3 (k = 0..sD); u[0] normalized on entry
    long long n3;
    int sD;
    int nface;            // coupled faces
    const int* fptr;      // (n + 1) entries of node r: fent[fptr[r] .. fptr[r + 1])
    const int* fent;      // entry ids grouped by node
    const int* fface;     // (entries) face of the entry
    const double* fval;   // (entries, 3) valM of the entry
    const double* gram;   // (nface, nface) valM_f . valM_g (diagonal: nS)
    double coef0[kMaxCoupled], coef1[kMaxCoupled];
    double err0, eps;
    double* part;         // 2 regions of kGmPartStride * gridDim
    double* H;            // (sD + 1, sD) column-major, rotated (written by block 0)
    double* errv;         // (sD + 1)
    double* out;          // iterations done, suc
};

__device__ __forceinline__ double gm_sum(const double* part, int k, double* sm) {
    double s = 0.0;
    for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) s += __ldcg(part + (size_t)b * kGmPartStride + k);
    return block_sum(s, sm);
}

template <typename M, typename B, int NF>
__global__ void __launch_bounds__(kGmThreads, 2) k_gmres_cycle(GmArgs<M, B> a) {
    namespace cgrp = cooperative_groups;
    cgrp::grid_group grid = cgrp::this_grid();
    __shared__ double sm[32];
    __shared__ double sh[kGmMaxSD + 2];  // h_1 .. h_{i+1} of the current column
    __shared__ double sc[kGmMaxSD], ssn[kGmMaxSD], serr[kGmMaxSD + 1];
    __shared__ int sdone;
    const int n = a.n;
    const long long n3 = a.n3, npad = a.npad;
    const int tid0 = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    if (threadIdx.x == 0) {
        serr[0] = a.err0;
        sdone = 0;
    }
    __syncthreads();
    int bar = 0;  // barrier counter: partial region = bar & 1
    auto region = [&]() { return a.part + (size_t)(bar & 1) * kGmPartStride * gridDim.x; };
    int i;
    for (i = 1; i <= a.sD; ++i) {
        const B* uin = a.u + (size_t)(i - 1) * n3;
        B* w = a.u + (size_t)i * n3;
        // ---- P1: w = K U(i-1); face dots S0_f (on U(i-1)) and T_f (on w) ----
        double s0[NF > 0 ? NF : 1], tf[NF > 0 ? NF : 1];
#pragma unroll
        for (int f = 0; f < (NF > 0 ? NF : 1); ++f) s0[f] = tf[f] = 0.0;
        for (int r = tid0; r < n; r += nth) {
            double a0 = 0.0, a1 = 0.0, a2 = 0.0;
            CR_SELL_ROW_U(4, a.sp, a.scol, r, {
                const B* uc = uin + 3 * (size_t)c;
                const double u0 = (double)uc[0], u1 = (double)uc[1], u2 = (double)uc[2];
                const auto ka = ldcs4(reinterpret_cast<const typename V4<M>::type*>(a.Ks) + pos);
                const auto kb = ldcs4(reinterpret_cast<const typename V4<M>::type*>(a.Ks + 4 * npad) + pos);
                const double k8 = (double)__ldcs(a.Ks + 8 * npad + pos);
                a0 = a0 + (double)ka.x * u0 + (double)ka.y * u1 + (double)ka.z * u2;
                a1 = a1 + (double)ka.w * u0 + (double)kb.x * u1 + (double)kb.y * u2;
                a2 = a2 + (double)kb.z * u0 + (double)kb.w * u1 + k8 * u2;
            })
            const B w0 = (B)a0, w1 = (B)a1, w2 = (B)a2;
            w[3 * (size_t)r + 0] = w0;
            w[3 * (size_t)r + 1] = w1;
            w[3 * (size_t)r + 2] = w2;
            if (NF > 0) {
                for (int k = a.fptr[r]; k < a.fptr[r + 1]; ++k) {
                    const int fe = a.fent[k];
                    const int f = a.fface[fe];
                    const double* v = a.fval + 3 * (size_t)fe;
                    const B* ur = uin + 3 * (size_t)r;
#pragma unroll
                    for (int q = 0; q < NF; ++q)
                        if (q == f) {
                            s0[q] += v[0] * (double)ur[0] + v[1] * (double)ur[1] + v[2] * (double)ur[2];
                            tf[q] += v[0] * (double)w0 + v[1] * (double)w1 + v[2] * (double)w2;
                        }
                }
            }
        }
        double cf[NF > 0 ? NF : 1];
        if (NF > 0) {
            double* pr = region();
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                if (f >= a.nface) break;
                const double x0 = block_sum(s0[f], sm), x1 = block_sum(tf[f], sm);
                if (threadIdx.x == 0) {
                    pr[(size_t)blockIdx.x * kGmPartStride + 2 * f] = x0;
                    pr[(size_t)blockIdx.x * kGmPartStride + 2 * f + 1] = x1;
                }
            }
        }
        grid.sync();
        if (NF > 0) {
            const double* pr = region();
            double S0[NF > 0 ? NF : 1], T[NF > 0 ? NF : 1];
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                S0[f] = T[f] = 0.0;
                if (f >= a.nface) continue;
                S0[f] = gm_sum(pr, 2 * f, sm);
                T[f] = gm_sum(pr, 2 * f + 1, sm);
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                cf[f] = 0.0;
                if (f >= a.nface) continue;
                double S1 = T[f];
                for (int g = 0; g < a.nface; ++g) S1 += a.coef0[g] * S0[g] * a.gram[f * a.nface + g];
                cf[f] = a.coef0[f] * S0[f] + a.coef1[f] * S1;
            }
        }
        ++bar;
        // ---- MGS passes j = 1..i: h_j = <w, U(j-1)> after w -= h_{j-1} U(j-2) ----
        for (int j = 1; j <= i; ++j) {
            const B* uj = a.u + (size_t)(j - 1) * n3;
            const B* up = j >= 2 ? a.u + (size_t)(j - 2) * n3 : nullptr;
            const double hp = j >= 2 ? sh[j - 1] : 0.0;
            double d = 0.0;
            for (int r = tid0; r < n; r += nth) {
                int k0 = 0, k1 = 0;
                if (NF > 0 && j == 1) {
                    k0 = a.fptr[r];
                    k1 = a.fptr[r + 1];
                }
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const size_t t = 3 * (size_t)r + k;
                    double wv = (double)w[t];
                    if (j == 1) {
                        if (NF > 0 && k1 > k0) {
                            double add = 0.0;
                            for (int e = k0; e < k1; ++e) {
                                const int fe = a.fent[e];
                                const int f = a.fface[fe];
#pragma unroll
                                for (int q = 0; q < NF; ++q)
                                    if (q == f) add += a.fval[3 * (size_t)fe + k] * cf[q];
                            }
                            wv = (double)(B)(wv + add);
                            w[t] = (B)wv;
                        }
                    } else {
                        wv = (double)(B)(wv - hp * (double)up[t]);
                        w[t] = (B)wv;
                    }
                    d += wv * (double)__ldcs(uj + t);
                }
            }
            d = block_sum(d, sm);
            double* pr = region();
            if (threadIdx.x == 0) pr[(size_t)blockIdx.x * kGmPartStride] = d;
            grid.sync();
            const double hj = gm_sum(region(), 0, sm);
            if (threadIdx.x == 0) sh[j] = hj;
            ++bar;
            __syncthreads();
        }
        // ---- norm: w -= h_i U(i-1); |w|^2 ----
        {
            const double hp = sh[i];
            double d = 0.0;
            for (int r = tid0; r < n; r += nth) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const size_t t = 3 * (size_t)r + k;
                    const double wv = (double)(B)((double)w[t] - hp * (double)uin[t]);
                    w[t] = (B)wv;
                    d += wv * wv;
                }
            }
            d = block_sum(d, sm);
            double* pr = region();
            if (threadIdx.x == 0) pr[(size_t)blockIdx.x * kGmPartStride] = d;
            grid.sync();
            const double hn = gm_sum(region(), 0, sm);
            ++bar;
            // ---- Givens (memLS.f90:750-760), identical in every block ----
            if (threadIdx.x == 0) {
                double hc[kGmMaxSD + 1];
                for (int j = 1; j <= i; ++j) hc[j - 1] = sh[j];
                hc[i] = sqrt(hn);
                sh[i + 1] = hc[i];
                double tmp;
                for (int j = 1; j <= i - 1; ++j) {
                    tmp = sc[j - 1] * hc[j - 1] + ssn[j - 1] * hc[j];
                    hc[j] = -ssn[j - 1] * hc[j - 1] + sc[j - 1] * hc[j];
                    hc[j - 1] = tmp;
                }
                tmp = sqrt(hc[i - 1] * hc[i - 1] + hc[i] * hc[i]);
                sc[i - 1] = hc[i - 1] / tmp;
                ssn[i - 1] = hc[i] / tmp;
                hc[i - 1] = tmp;
                hc[i] = 0.0;
                serr[i] = -ssn[i - 1] * serr[i - 1];
                serr[i - 1] = sc[i - 1] * serr[i - 1];
                if (blockIdx.x == 0) {
                    for (int j = 0; j <= i; ++j) a.H[(size_t)(i - 1) * (a.sD + 1) + j] = hc[j];
                    a.errv[i - 1] = serr[i - 1];
                    a.errv[i] = serr[i];
                }
                sdone = fabs(serr[i]) < a.eps ? 1 : 0;
            }
            __syncthreads();
        }
        if (sdone) break;
        if (i == a.sD) break;
        // ---- normalize: U(i) = w / h_{i+1} ----
        {
            const double hn = sh[i + 1];
            for (long long t = tid0; t < n3; t += nth) w[t] = (B)((double)w[t] / hn);
            grid.sync();
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = (double)(i > a.sD ? a.sD : i);
        a.out[1] = (double)sdone;
    }
}

// valM of the coupled faces gathered into (entries, 3): zero past nsd.
__global__ void k_gm_fval(const double* __restrict__ valM, int fdof, int nsd, int nNoF, double* __restrict__ out) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nNoF; a += gridDim.x * blockDim.x)
        for (int k = 0; k < 3; ++k) out[3 * (size_t)a + k] = k < nsd ? valM[(size_t)fdof * a + k] : 0.0;
}

// Coupled-face map for the persistent cycle, rebuilt when the set of
// coupled faces changes: the entries (face node a of coupled face q, in face
// order) grouped by node (fptr / fent), the face of each entry, and the
// pairs of entries of different faces at one node (faces that share rim
// nodes), from which k_gm_gram forms the off-diagonal valM_f . valM_g.
static int gm_face_map(crimson_lhs* L, int* ok) {
    std::vector<int> cur;
    for (int k = 0; k < (int)L->face.size(); ++k)
        if (L->face[k].coupledFlag) cur.push_back(k);
    if (L->gm_map_ok >= 0 && cur == L->gm_faces) {
        *ok = L->gm_map_ok;
        return CRIMSON_OK;
    }
    L->gm_faces = cur;
    L->gm_map_ok = 0;
    *ok = 0;
    if ((int)cur.size() > kMaxCoupled) return CRIMSON_OK;
    cudaStream_t s = L->stream;
    const int n = L->nNo;
    std::vector<int> node_of, fface;
    for (int q = 0; q < (int)cur.size(); ++q) {
        const MemlsFace& f = L->face[cur[q]];
        std::vector<int> g((size_t)f.nNo);
        CR_CUDA(cudaMemcpyAsync(g.data(), f.glob.p, sizeof(int) * g.size(), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        for (int a = 0; a < f.nNo; ++a) {
            if (g[a] < 0 || g[a] >= n) return CRIMSON_OK;
            node_of.push_back(g[a]);
            fface.push_back(q);
        }
    }
    const int entries = (int)node_of.size();
    std::vector<int> fptr((size_t)n + 1, 0), fent((size_t)std::max(1, entries));
    for (int e = 0; e < entries; ++e) ++fptr[(size_t)node_of[e] + 1];
    for (int r = 0; r < n; ++r) fptr[(size_t)r + 1] += fptr[r];
    std::vector<int> fill(fptr.begin(), fptr.end() - 1);
    for (int e = 0; e < entries; ++e) fent[(size_t)fill[node_of[e]]++] = e;
    std::vector<int> pairs;  // (e1, e2) of different faces at one node
    for (int r = 0; r < n; ++r)
        for (int k1 = fptr[r]; k1 < fptr[(size_t)r + 1]; ++k1)
            for (int k2 = fptr[r]; k2 < fptr[(size_t)r + 1]; ++k2)
                if (k1 != k2 && fface[fent[k1]] != fface[fent[k2]]) {
                    pairs.push_back(fent[k1]);
                    pairs.push_back(fent[k2]);
                }
    CR_CHECK(L->gmFptr.upload(fptr.data(), fptr.size(), s));
    CR_CHECK(L->gmFent.upload(fent.data(), fent.size(), s));
    CR_CHECK(L->gmFface.alloc(std::max<size_t>(1, fface.size())));
    if (!fface.empty())
        CR_CUDA(cudaMemcpyAsync(L->gmFface.p, fface.data(), sizeof(int) * fface.size(), cudaMemcpyHostToDevice, s));
    L->gm_npairs = (int)pairs.size() / 2;
    CR_CHECK(L->gmPairs.alloc(std::max<size_t>(2, pairs.size())));
    if (!pairs.empty())
        CR_CUDA(cudaMemcpyAsync(L->gmPairs.p, pairs.data(), sizeof(int) * pairs.size(), cudaMemcpyHostToDevice, s));
    CR_CHECK(L->gmFval.alloc(3 * (size_t)std::max(1, entries)));
    CR_CHECK(L->gmGram.alloc((size_t)kMaxCoupled * kMaxCoupled));
    CR_CUDA(cudaStreamSynchronize(s));
    L->gm_map_ok = 1;
    *ok = 1;
    return CRIMSON_OK;
}

// valM_f . valM_g of the coupled faces: nS on the diagonal, the shared-node
// pairs off it (one thread, fixed order).
struct FaceNorms {
    double v[kMaxCoupled];
};
__global__ void k_gm_gram(const int* __restrict__ pairs, int npairs, const int* __restrict__ fface,
                          const double* __restrict__ fval, FaceNorms nS, int nface, double* __restrict__ gram) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int f = 0; f < nface; ++f)
        for (int g = 0; g < nface; ++g) gram[f * nface + g] = f == g ? nS.v[f] : 0.0;
    for (int p = 0; p < npairs; ++p) {
        const int e1 = pairs[2 * p], e2 = pairs[2 * p + 1];
        const double* v1 = fval + 3 * (size_t)e1;
        const double* v2 = fval + 3 * (size_t)e2;
        gram[fface[e1] * nface + fface[e2]] += v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
    }
}

// Runs one restart cycle on the device (k_gmres_cycle): U(0) normalized in
// the basis, err0 = its norm before normalizing.  Returns the iterations
// done, whether |err_i| < eps was reached, and the rotated Hessenberg
// columns / err values in the host arrays of gmres().  *used = 0 when the
// persistent cycle does not apply (sD too large, more than 8 coupled faces, or no
// cooperative fit); the caller then runs the launch-per-step loop.
template <typename M, typename B>
static int gmres_cycle(Ctx& C, crimson_subls& ls, const M* Ks, double err0, double eps, std::vector<double>& h,
                       std::vector<double>& err, int* iters, int* suc, int* used) {
    crimson_lhs* L = C.L;
    cudaStream_t s = C.s;
    const int sD = ls.sD;
    *used = 0;
    if (sD < 1 || sD > kGmMaxSD) return CRIMSON_OK;
    int ok = 0;
    CR_CHECK(gm_face_map(L, &ok));
    if (!ok) return CRIMSON_OK;
    const int nface = (int)L->gm_faces.size();
    const void* fns[3] = {(const void*)k_gmres_cycle<M, B, 0>, (const void*)k_gmres_cycle<M, B, 1>,
                          (const void*)k_gmres_cycle<M, B, kMaxCoupled>};
    int& grid = std::is_same<M, float>::value ? L->gm_grid32 : L->gm_grid;
    if (grid == 0) {
        int nb = 1 << 30;
        for (const void* f : fns) {
            int b = 0;
            CR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, kGmThreads, 0));
            nb = std::min(nb, b);
        }
        grid = nb >= 1 ? sm_count() * std::min(nb, 2) : -1;
    }
    if (grid < 1) return CRIMSON_OK;
    CR_CHECK(L->gmH.alloc((size_t)(kGmMaxSD + 1) * kGmMaxSD));
    CR_CHECK(L->gmErr.alloc(kGmMaxSD + 1));
    CR_CHECK(L->gmOut.alloc(2));
    CR_CHECK(L->gmPart.alloc(2 * (size_t)kGmPartStride * std::max(L->gm_grid, L->gm_grid32)));
    GmArgs<M, B> a;
    a.sp = L->sell_ptr.p;
    a.scol = L->sell_col.p;
    a.npad = L->npad;
    a.n = L->nNo;
    a.Ks = Ks;
    a.u = reinterpret_cast<B*>(L->basis.p);
    a.n3 = 3LL * L->nNo;
    a.sD = sD;
    a.nface = nface;
    a.fptr = L->gmFptr.p;
    a.fent = L->gmFent.p;
    a.fface = L->gmFface.p;
    a.fval = L->gmFval.p;
    a.gram = L->gmGram.p;
    FaceNorms nsv{};
    int off = 0;
    for (int q = 0; q < nface; ++q) {
        const MemlsFace& f = L->face[L->gm_faces[q]];
        launch(k_gm_fval, grid_for(f.nNo, 256), 256, 0, s, (const double*)f.valM.p, f.dof, std::min(f.dof, 3), f.nNo,
               L->gmFval.p + 3 * (size_t)off);
        a.coef0[q] = f.res;
        a.coef1[q] = -f.res / (1.0 + f.res * f.nS);
        nsv.v[q] = f.nS;
        off += f.nNo;
    }
    for (int q = nface; q < kMaxCoupled; ++q) a.coef0[q] = a.coef1[q] = 0.0;
    if (nface > 0)
        launch(k_gm_gram, 1, 32, 0, s, (const int*)L->gmPairs.p, L->gm_npairs, (const int*)L->gmFface.p,
               (const double*)L->gmFval.p, nsv, nface, L->gmGram.p);
    a.err0 = err0;
    a.eps = eps;
    a.part = L->gmPart.p;
    a.H = L->gmH.p;
    a.errv = L->gmErr.p;
    a.out = L->gmOut.p;
    void* kargs[] = {&a};
    note_launch();
    const void* kfn = fns[nface == 0 ? 0 : (nface == 1 ? 1 : 2)];
    CR_CUDA(cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(kGmThreads), kargs, 0, s));
    double out[2];
    CR_CUDA(cudaMemcpyAsync(out, L->gmOut.p, sizeof(out), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    const int it = (int)out[0];
    if (it < 1 || it > sD) return CRIMSON_ERR_STATE;
    CR_CUDA(cudaMemcpyAsync(h.data(), L->gmH.p, sizeof(double) * (size_t)(sD + 1) * it, cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaMemcpyAsync(err.data(), L->gmErr.p, sizeof(double) * (it + 1), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    CR_CUDA(cudaGetLastError());
    *iters = it;
    *suc = out[1] != 0.0 ? 1 : 0;
    *used = 1;
    return CRIMSON_OK;
}

// GMRES (memLS.f90:681-788) on dof = 3; K sliced in M, basis in B, R and X FP64; X may not alias R.
template <typename M, typename B>
static int gmres(Ctx& C, crimson_subls& ls, const M* Ks, const double* R, double* X) {
    crimson_lhs* L = C.L;
    cudaStream_t s = C.s;
    const int dof = 3;
    const long long n = (long long)dof * L->nNo;
    const int sD = ls.sD;
    B* u = reinterpret_cast<B*>(L->basis.p);
    auto U = [&](int k) { return u + (size_t)k * n; };
    std::vector<double> h((size_t)(sD + 1) * sD, 0.0), c(sD), sn(sD), err(sD + 1), y(sD);
    auto H = [&](int i, int j) -> double& { return h[(size_t)j * (sD + 1) + i]; };
    const double time = now_s();
    ls.suc = 0;
    CR_CUDA(cudaMemsetAsync(X, 0, sizeof(double) * n, s));
    double eps = 0.0;
    const bool coupled = C.any_coupled();
    int i = 0;
    for (int l = 1; l <= ls.mItr; ++l) {
        if (l == 1) {
            launch(k_convert<B, double>, grid_for(n, 256), 256, 0, s, R, U(0), n);
        } else {
            ls.itr = ls.itr + 1;
            C.vv3s(Ks, (const double*)X, U(0));
            C.addbcmul(0, dof, (const double*)X, U(0));
            launch(k_sub<double, B, B>, grid_for(n, 256), 256, 0, s, R, (const B*)U(0), U(0), n);
        }
        if (coupled) C.addbcmul(1, dof, (const B*)U(0), U(0));  // dots read X before any update: X may alias Y
        C.dot((const B*)U(0), (const B*)U(0), n, kSlotNrm);
        CR_CHECK(C.sync_scal(kSlotNrm, 1));
        err[0] = std::sqrt(L->hscal[kSlotNrm]);
        if (l == 1) {
            eps = err[0];
            if (eps <= ls.absTol) {
                ls.callD = 0.0;
                ls.dB = 0.0;
                return CRIMSON_OK;
            }
            ls.iNorm = eps;
            ls.fNorm = eps;
            eps = std::max(ls.absTol, ls.relTol * eps);
        }
        ls.dB = ls.fNorm;
        launch(k_divide<B>, grid_for(n, 256), 256, 0, s, (const B*)U(0), (const double*)C.sc(kSlotNrm), U(0), n, 1);
        // the cycle as one persistent kernel where it applies, else one launch per step
        int used = 0;
        {
            int it = 0, ok = 0;
            CR_CHECK((gmres_cycle<M, B>(C, ls, Ks, err[0], eps, h, err, &it, &ok, &used)));
            if (used) {
                ls.itr = ls.itr + it;
                i = it;
                if (ok) ls.suc = 1;
            }
        }
        for (i = used ? i : 1; !used && i <= sD; ++i) {
            ls.itr = ls.itr + 1;
            B* w = U(i);
            C.vv3s(Ks, (const B*)U(i - 1), w);
            C.addbcmul(0, dof, (const B*)U(i - 1), w);
            if (coupled) C.addbcmul(1, dof, (const B*)w, w);
            // fused modified Gram-Schmidt
            for (int j = 1; j <= i; ++j) {
                const B* uprev = (j == 1) ? nullptr : U(j - 2);
                launch(k_mgs<B>, red_grid(n), 256, 0, s, w, uprev, (const double*)C.sc(kSlotH + j - 2),
                       (const B*)U(j - 1), n, L->red.part.p, L->red.ticket.p, C.sc(kSlotH + j - 1));
            }
            launch(k_mgs<B>, red_grid(n), 256, 0, s, w, (const B*)U(i - 1), (const double*)C.sc(kSlotH + i - 1),
                   (const B*)w, n, L->red.part.p, L->red.ticket.p, C.sc(kSlotH + i));
            launch(k_divide<B>, grid_for(n, 256), 256, 0, s, (const B*)w, (const double*)C.sc(kSlotH + i), w, n, 1);
            CR_CHECK(C.sync_scal(kSlotH, i + 1));
            for (int j = 1; j <= i; ++j) H(j - 1, i - 1) = L->hscal[kSlotH + j - 1];
            H(i, i - 1) = std::sqrt(L->hscal[kSlotH + i]);
            double tmp;
            for (int j = 1; j <= i - 1; ++j) {
                tmp = c[j - 1] * H(j - 1, i - 1) + sn[j - 1] * H(j, i - 1);
                H(j, i - 1) = -sn[j - 1] * H(j - 1, i - 1) + c[j - 1] * H(j, i - 1);
                H(j - 1, i - 1) = tmp;
            }
            tmp = std::sqrt(H(i - 1, i - 1) * H(i - 1, i - 1) + H(i, i - 1) * H(i, i - 1));
            c[i - 1] = H(i - 1, i - 1) / tmp;
            sn[i - 1] = H(i, i - 1) / tmp;
            H(i - 1, i - 1) = tmp;
            H(i, i - 1) = 0.0;
            err[i] = -sn[i - 1] * err[i - 1];
            err[i - 1] = c[i - 1] * err[i - 1];
            if (std::fabs(err[i]) < eps) {
                ls.suc = 1;
                break;
            }
        }
        if (i > sD) i = sD;
        for (int j = 0; j < i; ++j) y[j] = err[j];
        for (int j = i; j >= 1; --j) {
            for (int k = j + 1; k <= i; ++k) y[j - 1] = y[j - 1] - H(j - 1, k - 1) * y[k - 1];
            y[j - 1] = y[j - 1] / H(j - 1, j - 1);
        }
        std::memcpy(L->hscal + kSlotY, y.data(), sizeof(double) * i);
        CR_CUDA(cudaMemcpyAsync(C.sc(kSlotY), L->hscal + kSlotY, sizeof(double) * i, cudaMemcpyHostToDevice, s));
        launch(k_multi_axpy<B>, grid_for(n, 256), 256, 0, s, X, (const B*)u, (const double*)C.sc(kSlotY), i, n);
        CR_CUDA(cudaStreamSynchronize(s));  // y staging buffer is reused
        ls.fNorm = std::fabs(err[i]);
        if (ls.suc) break;
    }
    ls.callD = now_s() - time + ls.callD;
    ls.dB = 10.0 * std::log(ls.fNorm / ls.dB);
    return CRIMSON_OK;
}

// Coupled-face vectors for the CG's ADDBCMUL(PRE) term: w_f = G^T valM_f and
// z_f = Gt valM_f, with the Sherman-Morrison coefficient -res/(1 + res nS).
// Built once per NSSOLVER call (valM, G, Gt are fixed during it).
template <typename M>
static int cg_faces(Ctx& C, const M* G, const M* Gt, int* nface, double* coef) {
    crimson_lhs* L = C.L;
    cudaStream_t s = C.s;
    const int n = L->nNo;
    int k = 0;
    for (auto& f : L->face) {
        if (!f.coupledFlag) continue;
        if (k >= kMaxCoupled) return CRIMSON_ERR_UNSUPPORTED;
        CR_CHECK(L->cgExt.alloc(3 * (size_t)n));
        CR_CHECK(L->cgW.alloc((size_t)kMaxCoupled * n));
        CR_CHECK(L->cgZ.alloc((size_t)kMaxCoupled * n));
        CR_CUDA(cudaMemsetAsync(L->cgExt.p, 0, sizeof(double) * 3 * (size_t)n, s));
        launch(k_face_ext, grid_for(f.nNo, 256), 256, 0, s, f.glob.p, f.valM.p, f.dof, std::min(f.dof, 3), f.nNo,
               L->cgExt.p);
        launch(k_spmv_vs3_trans<M>, C.spmv_grid(), 256, 0, s, L->rowptr, L->col, L->trans, G, (const double*)L->cgExt.p,
               L->cgW.p + (size_t)k * n, n);
        C.vs3(Gt, (const double*)L->cgExt.p, L->cgZ.p + (size_t)k * n);
        coef[k] = -f.res / (1.0 + f.res * f.nS);
        ++k;
    }
    *nface = k;
    CR_CUDA(cudaGetLastError());
    return CRIMSON_OK;
}

// Shared memory for block-resident CG columns (CgCols) on a grid of two
// blocks per SM: 0 when the pattern's column offsets exceed 16 bits; else
// 2 bytes per sliced entry of the fullest block.  Computed once per pattern.
static int cg_resident_bytes(crimson_lhs* L, size_t* bytes) {
    if (L->cg_res_bytes >= 0) {
        *bytes = (size_t)L->cg_res_bytes;
        return CRIMSON_OK;
    }
    cudaStream_t s = L->stream;
    const int n = L->nNo;
    CR_CHECK(L->cg_tmp.alloc(1));
    CR_CUDA(cudaMemsetAsync(L->cg_tmp.p, 0, sizeof(int), s));
    launch(k_max_offset, grid_for(n, 256), 256, 0, s, (const int*)L->rowptr, (const int*)L->col, n, L->cg_tmp.p);
    int maxoff = 0;
    CR_CUDA(cudaMemcpyAsync(&maxoff, L->cg_tmp.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    std::vector<int> sp((size_t)L->nslice + 1);
    CR_CUDA(cudaMemcpyAsync(sp.data(), L->sell_ptr.p, sizeof(int) * sp.size(), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    long long best = 0;
    if (maxoff <= 32767) {
        const int grid = 2 * sm_count();
        const int wpb = kCgThreads / kSlice;  // slices (warps) per block
        std::vector<long long> per((size_t)grid, 0);
        for (int q = 0; q < L->nslice; ++q) per[(size_t)((q / wpb) % grid)] += sp[q + 1] - sp[q];
        for (long long v : per) best = std::max(best, v);
        best = (2 * best + 15) / 16 * 16;
        if (best == 0) best = 16;
    }
    L->cg_res_bytes = best;
    *bytes = (size_t)best;
    return CRIMSON_OK;
}

// CGRAD (memLS.f90:367-430) on the Schur-like operator L P - Gt G P; R in/out (n).
// Gs / GLs: sliced G and {Gt, L} of this NSSOLVER call.
template <typename M>
static int cgrad(Ctx& C, crimson_subls& ls, const M* Gs, const typename V4<M>::type* GLs,
                 double* R, int nface,
                 const double* coef, bool use_s2 = false) {
    crimson_lhs* L = C.L;
    cudaStream_t s = C.s;
    const int n = L->nNo;
    const double time = now_s();
    ls.suc = 0;
    C.dot((const double*)R, (const double*)R, n, kSlotErr);
    CR_CHECK(C.sync_scal(kSlotErr, 1));
    double errO = std::sqrt(L->hscal[kSlotErr]);
    ls.iNorm = errO;
    double eps = std::max(ls.absTol, ls.relTol * errO);
    eps = eps * eps;
    double err = errO;
    err = err * err;
    if (use_s2) {
        // the same CGRAD on the explicit FP32 Schur operator (schur.cu)
        CR_CUDA(cudaEventRecord(L->ev0, s));
        CR_CHECK(cg_schur_launch(L, R, nface, coef, L->cgW.p, L->cgZ.p, eps, err, ls.mItr, C.sc(kSlotCg)));
        CR_CUDA(cudaEventRecord(L->ev1, s));
        CR_CHECK(C.sync_scal(kSlotCg, 4));
        err = L->hscal[kSlotCg + 0];
        errO = L->hscal[kSlotCg + 1];
        const int i = (int)L->hscal[kSlotCg + 2];
        ls.suc = (int)L->hscal[kSlotCg + 3];
        float ms = 0.f;
        CR_CUDA(cudaEventElapsedTime(&ms, L->ev0, L->ev1));
        L->cg_acc32.ms += ms;
        L->cg_acc32.iters += i - 1;
        L->cg_acc32.launches += 1;
        if (L->s2_form_pending) {
            float fm = 0.f;
            CR_CUDA(cudaEventElapsedTime(&fm, L->s2_ev0, L->s2_ev1));
            L->s2_form_ms += fm;
            L->s2_forms += 1;
            L->s2_form_pending = false;
        }
        CR_CUDA(cudaMemcpyAsync(R, L->cgX.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        CR_CUDA(cudaStreamSynchronize(s));
        ls.fNorm = std::sqrt(err);
        ls.callD = now_s() - time + ls.callD;
        ls.dB = 5.0 * std::log(err / errO);
        ls.itr = ls.itr + i - 1;
        return CRIMSON_OK;
    }
    const void* kres[3] = {(const void*)k_cg_persistent<0, M, true>, (const void*)k_cg_persistent<1, M, true>,
                           (const void*)k_cg_persistent<kMaxCoupled, M, true>};
    const void* kglb[3] = {(const void*)k_cg_persistent<0, M, false>, (const void*)k_cg_persistent<1, M, false>,
                           (const void*)k_cg_persistent<kMaxCoupled, M, false>};
    int& grid = std::is_same<M, float>::value ? L->cg_grid32 : L->cg_grid;
    int& mode = std::is_same<M, float>::value ? L->cg_res32 : L->cg_res64;
    size_t rbytes = 0;
    CR_CHECK(cg_resident_bytes(L, &rbytes));
    if (grid == 0) {
        // block-resident columns when two blocks per SM fit with them
        mode = 0;
        if (rbytes > 0) {
            int ok = 1;
            for (const void* f : kres) {
                int nb = 0;
                if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rbytes) != cudaSuccess ||
                    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, kCgThreads, rbytes) != cudaSuccess || nb < 2)
                    ok = 0;
            }
            (void)cudaGetLastError();  // a refused attribute only selects the other kernel
            mode = ok;
        }
        if (mode) {
            grid = 2 * sm_count();
        } else {
            int nb = 1 << 30;
            for (const void* f : kglb) {
                int b = 0;
                CR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, kCgThreads, 0));
                nb = std::min(nb, b);
            }
            if (nb < 1) return CRIMSON_ERR_UNSUPPORTED;
            grid = sm_count() * std::min(nb, 8);
        }
    }
    const int fi = nface == 0 ? 0 : (nface == 1 ? 1 : 2);
    const void* kfn = mode ? kres[fi] : kglb[fi];
    const size_t dyn = mode ? rbytes : 0;
    CR_CHECK(L->cgPart.alloc(3 * (size_t)kCgPartStride * std::max(L->cg_grid, L->cg_grid32)));
    CR_CHECK(L->cgRecA.alloc(2 * (size_t)n));
    CR_CHECK(L->cgRecB.alloc(4 * (size_t)n));
    CR_CHECK(L->cgPd.alloc((size_t)n));
    CR_CUDA(cudaMemsetAsync(L->cgX.p, 0, sizeof(double) * n, s));
    launch(k_cg_init, grid_for(n, 256), 256, 0, s, (const double*)R, reinterpret_cast<double2*>(L->cgRecA.p), n);
    CgArgs<M> a;
    a.sp = L->sell_ptr.p;
    a.scol = L->sell_col.p;
    a.npad = L->npad;
    a.n = n;
    a.G = Gs;
    a.GL = GLs;
    a.X = L->cgX.p;
    a.recA = reinterpret_cast<double2*>(L->cgRecA.p);
    a.recB = reinterpret_cast<typename V4<M>::type*>(L->cgRecB.p);
    a.Pd = L->cgPd.p;
    a.SP = L->cgSP.p;
    a.nface = nface;
    a.w = L->cgW.p;
    a.z = L->cgZ.p;
    for (int f = 0; f < kMaxCoupled; ++f) a.coef[f] = f < nface ? coef[f] : 0.0;
    a.eps = eps;
    a.err0 = err;
    a.mItr = ls.mItr;
    a.part = L->cgPart.p;
    a.out = C.sc(kSlotCg);
    void* kargs[] = {&a};
    note_launch();
    CR_CUDA(cudaEventRecord(L->ev0, s));
    CR_CUDA(cudaLaunchCooperativeKernel(kfn, dim3(grid), dim3(kCgThreads), kargs, dyn, s));
    CR_CUDA(cudaEventRecord(L->ev1, s));
    CR_CHECK(C.sync_scal(kSlotCg, 4));
    err = L->hscal[kSlotCg + 0];
    errO = L->hscal[kSlotCg + 1];
    const int i = (int)L->hscal[kSlotCg + 2];
    ls.suc = (int)L->hscal[kSlotCg + 3];
    float ms = 0.f;
    CR_CUDA(cudaEventElapsedTime(&ms, L->ev0, L->ev1));
    auto& acc = std::is_same<M, float>::value ? L->cg_acc32 : L->cg_acc64;
    acc.ms += ms;
    acc.iters += i - 1;
    acc.launches += 1;
    CR_CUDA(cudaMemcpyAsync(R, L->cgX.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    CR_CUDA(cudaStreamSynchronize(s));
    ls.fNorm = std::sqrt(err);
    ls.callD = now_s() - time + ls.callD;
    ls.dB = 5.0 * std::log(err / errO);
    ls.itr = ls.itr + i - 1;
    return CRIMSON_OK;
}

// GE (memLS.f90:607-677), A column-major
static int ge_solve(int N, const double* A, double* B) {
    if (N == 2) {
        double pivot = A[0] * A[3] - A[1] * A[2];
        if (pivot == 0.0 || !std::isfinite(pivot)) return CRIMSON_ERR_SINGULAR;
        double saveEl = (B[0] * A[3] - B[1] * A[2]) / pivot;
        B[1] = (B[1] * A[0] - B[0] * A[1]) / pivot;
        B[0] = saveEl;
        return CRIMSON_OK;
    }
    std::vector<double> Cm((size_t)N * (N + 1));
    auto c = [&](int i, int j) -> double& { return Cm[(size_t)j * N + i]; };
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) c(i, j) = A[(size_t)j * N + i];
    for (int i = 0; i < N; ++i) c(i, N) = B[i];
    for (int m = 0; m < N - 1; ++m) {
        int ipv = m;
        double pivot = std::fabs(c(m, m));
        for (int i = m + 1; i < N; ++i)
            if (std::fabs(c(i, m)) > pivot) {
                ipv = i;
                pivot = std::fabs(c(i, m));
            }
        if (pivot < 2.0 * 2.220446049250313e-16) return CRIMSON_ERR_SINGULAR;
        if (ipv != m)
            for (int j = m; j <= N; ++j) std::swap(c(m, j), c(ipv, j));
        for (int i = m + 1; i < N; ++i) {
            double saveEl = c(i, m) / c(m, m);
            c(i, m) = 0.0;
            for (int j = m + 1; j <= N; ++j) c(i, j) = c(i, j) - saveEl * c(m, j);
        }
    }
    for (int j = N - 1; j >= 0; --j) {
        for (int i = j + 1; i < N; ++i) c(j, N) = c(j, N) - c(j, i) * c(i, N);
        c(j, N) = c(j, N) / c(j, j);
    }
    for (int i = 0; i < N; ++i) B[i] = c(i, N);
    return CRIMSON_OK;
}

// Sliced matrix buffers of one precision (zeroed at allocation, so the
// padding entries stay zero: conversions only write real entries).
template <typename M>
static int sell_alloc(crimson_lhs* L, DBuf<M>& K, DBuf<M>& G, DBuf<M>& GL) {
    const size_t np = (size_t)L->npad + (size_t)kSlice * kSellUnroll;
    if (K.n == 9 * np && G.n == 3 * np && GL.n == 4 * np) return CRIMSON_OK;
    CR_CHECK(K.alloc(9 * np));
    CR_CHECK(G.alloc(3 * np));
    CR_CHECK(GL.alloc(4 * np));
    CR_CUDA(cudaMemsetAsync(K.p, 0, sizeof(M) * K.n, L->stream));
    CR_CUDA(cudaMemsetAsync(G.p, 0, sizeof(M) * G.n, L->stream));
    CR_CUDA(cudaMemsetAsync(GL.p, 0, sizeof(M) * GL.n, L->stream));
    return CRIMSON_OK;
}
static int sell_mats(crimson_lhs* L, double** K, double** G, double4** GL) {
    CR_CHECK(sell_alloc(L, L->Ks64, L->Gs64, L->GLs64));
    *K = L->Ks64.p;
    *G = L->Gs64.p;
    *GL = reinterpret_cast<double4*>(L->GLs64.p);
    return CRIMSON_OK;
}
static int sell_mats(crimson_lhs* L, float** K, float** G, float4** GL) {
    CR_CHECK(sell_alloc(L, L->Ks32, L->Gs32, L->GLs32));
    *K = L->Ks32.p;
    *G = L->Gs32.p;
    *GL = reinterpret_cast<float4*>(L->GLs32.p);
    return CRIMSON_OK;
}

// Sliced pattern of a CSR pattern (rowptr, col on the device): slice widths
// from the row lengths (host), columns (device).  The column array carries
// kSlice * kSellUnroll zero entries past npad.
int sell_build(const int* rowptr, const int* col, int n, cudaStream_t s, DBuf<int>& sell_ptr, DBuf<int>& sell_col,
               long long* npad_out, int* nslice_out) {
    std::vector<int> rp((size_t)n + 1);
    CR_CUDA(cudaMemcpyAsync(rp.data(), rowptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    const int ns = (n + kSlice - 1) / kSlice;
    std::vector<int> sp((size_t)ns + 1, 0);
    long long pos = 0;
    for (int q = 0; q < ns; ++q) {
        int w = 0;
        for (int r = q * kSlice; r < std::min(n, (q + 1) * kSlice); ++r) w = std::max(w, rp[r + 1] - rp[r]);
        sp[q] = (int)pos;
        pos += (long long)kSlice * w;
        if (pos + (long long)kSlice * kSellUnroll > 0x7fffffffLL) return CRIMSON_ERR_UNSUPPORTED;
    }
    sp[ns] = (int)pos;
    CR_CHECK(sell_ptr.upload(sp.data(), sp.size(), s));
    const size_t np = (size_t)pos + (size_t)kSlice * kSellUnroll;
    CR_CHECK(sell_col.alloc(np));
    CR_CUDA(cudaMemsetAsync(sell_col.p, 0, sizeof(int) * np, s));
    launch(k_sell_cols, grid_for((long long)ns * kSlice, 256), 256, 0, s, rowptr, col, (const int*)sell_ptr.p, n,
           ns * kSlice, sell_col.p);
    CR_CUDA(cudaStreamSynchronize(s));
    CR_CUDA(cudaGetLastError());
    *npad_out = pos;
    *nslice_out = ns;
    return CRIMSON_OK;
}

static int sell_pattern(crimson_lhs* L) {
    if (L->sell_ptr.p) return CRIMSON_OK;
    CR_CHECK(sell_build(L->rowptr, L->col, L->nNo, L->stream, L->sell_ptr, L->sell_col, &L->npad, &L->nslice));
    return CRIMSON_OK;
}

// NSSOLVER (memLS.f90:1460-1759); R (4, nNo) FP64 in/out.  mK, mG, mD, mL,
// Gt: the scaled split matrices (FP64 CSR).  GMRES and CGRAD run on sliced
// copies in M (FP64, or FP32 for the mixed mode) with a type-B GMRES basis;
// every other product -- the A d of the search directions that enter the
// least-squares (Gram) problem, the Schur right side D u and the
// coupled-face vectors -- uses the FP64 matrices, so the Gram system, the
// residual estimate and the outer residuals are those of the FP64 operator.
template <typename M, typename B>
static int nssolver(crimson_lhs* L, crimson_ls* ls, const double* mK, const double* mG, const double* mD,
                    const double* mL, const double* Gt, double* R) {
    Ctx C{L, L->stream};
    cudaStream_t s = L->stream;
    const int nNo = L->nNo;
    const long long nv = 3LL * nNo;
    int iB = ls->RI.mItr;
    const int nB = 2 * iB;
    auto Ucol = [&](int k) { return L->U.p + (size_t)k * nv; };
    auto Pcol = [&](int k) { return L->P.p + (size_t)k * nNo; };
    auto MUc = [&](int k) { return L->MU.p + (size_t)k * nv; };
    auto MPc = [&](int k) { return L->MP.p + (size_t)k * nNo; };
    launch(k_split4, grid_for(nNo, 256), 256, 0, s, (const double*)R, L->Rmi.p, L->Rci.p, nNo);
    CR_CUDA(cudaMemcpyAsync(L->Rm.p, L->Rmi.p, sizeof(double) * nv, cudaMemcpyDeviceToDevice, s));
    CR_CUDA(cudaMemcpyAsync(L->Rc.p, L->Rci.p, sizeof(double) * nNo, cudaMemcpyDeviceToDevice, s));
    std::vector<double> A((size_t)nB * nB, 0.0), Bv(nB, 0.0), xB(nB, 0.0);
    auto Aa = [&](int i, int j) -> double& { return A[(size_t)j * nB + i]; };
    C.dot((const double*)L->Rm.p, (const double*)L->Rm.p, nv, 0);
    C.dot((const double*)L->Rc.p, (const double*)L->Rc.p, nNo, 1);
    CR_CHECK(C.sync_scal(0, 2));
    double nv1 = std::sqrt(L->hscal[0]), ns1 = std::sqrt(L->hscal[1]);
    double eps = std::sqrt(std::pow(nv1, 2.0) + std::pow(ns1, 2.0));
    if (!std::isfinite(eps)) {
        set_last_error("NSSOLVER: non-finite right-hand side");
        return CRIMSON_ERR_NONFINITE;
    }
    ls->RI.iNorm = eps;
    ls->RI.fNorm = eps;
    ls->CG.callD = 0.0;
    ls->GM.callD = 0.0;
    ls->CG.itr = 0;
    ls->GM.itr = 0;
    const double t0 = now_s();
    ls->RI.suc = 0;
    eps = std::max(ls->RI.absTol, ls->RI.relTol * eps);
    // BCPRE (memLS.f90:1683-1716): nS = |valM|^2 per coupled face, summed on
    // the host in the reference's node order (faces are small).
    for (auto& f : L->face) {
        if (!f.coupledFlag) continue;
        std::vector<double> vm((size_t)f.dof * f.nNo);
        CR_CUDA(cudaMemcpyAsync(vm.data(), f.valM.p, sizeof(double) * vm.size(), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        f.nS = 0.0;
        const int nsd = std::min(f.dof, 3);
        for (int a = 0; a < f.nNo; ++a)
            for (int i = 0; i < nsd; ++i) f.nS = f.nS + std::pow(vm[(size_t)f.dof * a + i], 2.0);
    }
    int cg_nface = 0;
    double cg_coef[kMaxCoupled];
    CR_CHECK(cg_faces(C, mG, Gt, &cg_nface, cg_coef));
    M* Ks = nullptr;
    M* Gs = nullptr;
    typename V4<M>::type* GLs = nullptr;
    CR_CHECK(sell_mats(L, &Ks, &Gs, &GLs));
    launch(k_to_sell<M>, grid_for(nNo, 256), 256, 0, s, L->rowptr, (const int*)L->sell_ptr.p, nNo, mK, mG, Gt, mL,
           L->npad, Ks, Gs, GLs);
    // mixed precision: the CG runs on the explicit FP32 Schur operator
    bool use_s2 = false;
    if (std::is_same<M, float>::value && ls->schur && cg_nface <= kMaxCoupled) {
        CR_CHECK(schur_pattern(L));
        if (L->s2_state == 1) {
            CR_CHECK(schur_form(L, mG, Gt, mL));
            use_s2 = true;
        }
    }
    int i, iBB = 0;
    for (i = 1; i <= ls->RI.mItr; ++i) {
        iB = 2 * i - 1;
        iBB = 2 * i;
        ls->RI.dB = ls->RI.fNorm;
        CR_CHECK((gmres<M, B>(C, ls->GM, (const M*)Ks, L->Rm.p, Ucol(i - 1))));
        C.vs3(mD, (const double*)Ucol(i - 1), Pcol(i - 1));
        launch(k_sub<double, double, double>, grid_for(nNo, 256), 256, 0, s, (const double*)L->Rc.p,
               (const double*)Pcol(i - 1), Pcol(i - 1), (long long)nNo);
        CR_CHECK(cgrad<M>(C, ls->CG, (const M*)Gs, (const typename V4<M>::type*)GLs, Pcol(i - 1),
                          cg_nface,
                          cg_coef, use_s2));
        C.sv3(mG, (const double*)Pcol(i - 1), MUc(iB - 1));
        launch(k_sub<double, double, double>, grid_for(nv, 256), 256, 0, s, (const double*)L->Rm.p,
               (const double*)MUc(iB - 1), MUc(iBB - 1), nv);
        CR_CHECK((gmres<M, B>(C, ls->GM, (const M*)Ks, MUc(iBB - 1), Ucol(i - 1))));
        if (std::is_same<M, double>::value)
            C.vv3s((const M*)Ks, (const double*)Ucol(i - 1), MUc(iBB - 1));  // the sliced copy is FP64
        else
            C.vv3(mK, (const double*)Ucol(i - 1), MUc(iBB - 1));
        C.addbcmul(0, 3, (const double*)Ucol(i - 1), MUc(iBB - 1));
        C.ss(mL, (const double*)Pcol(i - 1), MPc(iB - 1));
        C.vs3(mD, (const double*)Ucol(i - 1), MPc(iBB - 1));
        // Gram matrix entries for columns iB, iBB
        int slot = kSlotGram;
        for (int k = iB; k <= iBB; ++k) {
            for (int j = 1; j <= k - 1; ++j) {
                C.dot((const double*)MUc(j - 1), (const double*)MUc(k - 1), nv, slot++);
                C.dot((const double*)MPc(j - 1), (const double*)MPc(k - 1), nNo, slot++);
            }
            C.dot((const double*)MUc(k - 1), (const double*)MUc(k - 1), nv, slot++);
            C.dot((const double*)MPc(k - 1), (const double*)MPc(k - 1), nNo, slot++);
            C.dot((const double*)MUc(k - 1), (const double*)L->Rmi.p, nv, slot++);
            C.dot((const double*)MPc(k - 1), (const double*)L->Rci.p, nNo, slot++);
        }
        CR_CHECK(C.sync_scal(kSlotGram, slot - kSlotGram));
        slot = kSlotGram;
        for (int k = iB; k <= iBB; ++k) {
            for (int j = 1; j <= k - 1; ++j) {
                Aa(j - 1, k - 1) = L->hscal[slot] + L->hscal[slot + 1];
                slot += 2;
                Aa(k - 1, j - 1) = Aa(j - 1, k - 1);
            }
            Aa(k - 1, k - 1) = std::pow(std::sqrt(L->hscal[slot]), 2.0) + std::pow(std::sqrt(L->hscal[slot + 1]), 2.0);
            slot += 2;
            Bv[k - 1] = L->hscal[slot] + L->hscal[slot + 1];
            slot += 2;
        }
        for (int t = 0; t < iBB; ++t) xB[t] = Bv[t];
        std::vector<double> Asub((size_t)iBB * iBB);
        for (int c = 0; c < iBB; ++c)
            for (int r = 0; r < iBB; ++r) Asub[(size_t)c * iBB + r] = Aa(r, c);
        CR_CHECK(ge_solve(iBB, Asub.data(), xB.data()));
        for (int t = 0; t < iBB; ++t)
            if (!std::isfinite(xB[t])) {
                set_last_error("NSSOLVER: non-finite least-squares coefficients");
                return CRIMSON_ERR_NONFINITE;
            }
        double sxb = 0.0;
        for (int t = 0; t < iBB; ++t) sxb = sxb + xB[t] * Bv[t];
        ls->RI.fNorm = std::sqrt(std::pow(ls->RI.iNorm, 2.0) - sxb);
        if (ls->RI.fNorm < eps) {
            ls->RI.suc = 1;
            break;
        }
        // Rm = Rmi - sum xB_j MU_j ; Rc = Rci - sum xB_j MP_j
        CR_CUDA(cudaMemcpyAsync(L->Rm.p, L->Rmi.p, sizeof(double) * nv, cudaMemcpyDeviceToDevice, s));
        CR_CUDA(cudaMemcpyAsync(L->Rc.p, L->Rci.p, sizeof(double) * nNo, cudaMemcpyDeviceToDevice, s));
        for (int j = 1; j <= iBB; ++j) {
            launch(k_axpy<double, double>, grid_for(nv, 256), 256, 0, s, -xB[j - 1], (const double*)MUc(j - 1),
                   L->Rm.p, nv);
            launch(k_axpy<double, double>, grid_for(nNo, 256), 256, 0, s, -xB[j - 1], (const double*)MPc(j - 1),
                   L->Rc.p, (long long)nNo);
        }
    }
    if (i > ls->RI.mItr) {
        ls->RI.itr = ls->RI.mItr;
    } else {
        ls->RI.itr = i;
        CR_CUDA(cudaMemcpyAsync(L->Rc.p, L->Rci.p, sizeof(double) * nNo, cudaMemcpyDeviceToDevice, s));
        for (int j = 1; j <= iBB; ++j)
            launch(k_axpy<double, double>, grid_for(nNo, 256), 256, 0, s, -xB[j - 1], (const double*)MPc(j - 1),
                   L->Rc.p, (long long)nNo);
    }
    C.dot((const double*)L->Rc.p, (const double*)L->Rc.p, nNo, 0);
    CR_CHECK(C.sync_scal(0, 1));
    ls->Resc = (int)std::lround(100.0 * std::pow(std::sqrt(L->hscal[0]) / ls->RI.fNorm, 2.0));
    ls->Resm = 100 - ls->Resc;
    // solution: Rmi = xB(2) U_1 + sum xB(2i) U_i ; Rci = xB(1) P_1 + sum xB(2i-1) P_i
    CR_CUDA(cudaMemsetAsync(L->Rmi.p, 0, sizeof(double) * nv, s));
    CR_CUDA(cudaMemsetAsync(L->Rci.p, 0, sizeof(double) * nNo, s));
    launch(k_axpy<double, double>, grid_for(nv, 256), 256, 0, s, xB[1], (const double*)Ucol(0), L->Rmi.p, nv);
    launch(k_axpy<double, double>, grid_for(nNo, 256), 256, 0, s, xB[0], (const double*)Pcol(0), L->Rci.p,
           (long long)nNo);
    for (i = 2; i <= ls->RI.itr; ++i) {
        launch(k_axpy<double, double>, grid_for(nv, 256), 256, 0, s, xB[2 * i - 1], (const double*)Ucol(i - 1),
               L->Rmi.p, nv);
        launch(k_axpy<double, double>, grid_for(nNo, 256), 256, 0, s, xB[2 * i - 2], (const double*)Pcol(i - 1),
               L->Rci.p, (long long)nNo);
    }
    launch(k_merge4, grid_for(nNo, 256), 256, 0, s, R, (const double*)L->Rmi.p, (const double*)L->Rci.p, nNo);
    CR_CUDA(cudaStreamSynchronize(s));
    ls->RI.callD = now_s() - t0;
    ls->RI.dB = 10.0 * std::log(ls->RI.fNorm / ls->RI.dB);
    CR_CUDA(cudaGetLastError());
    return CRIMSON_OK;
}

static int lhs_work_alloc(crimson_lhs* L, const crimson_ls* ls) {
    const int nNo = L->nNo;
    const long long nnz = L->nnz;
    const int iB = ls->RI.mItr;
    const int sD = ls->GM.sD;
    if (sD + 1 > 512 || 8 * iB * iB + 64 > 4096) return CRIMSON_ERR_UNSUPPORTED;
    CR_CHECK(L->W.alloc(4 * (size_t)nNo));
    CR_CHECK(L->R.alloc(4 * (size_t)nNo));
    CR_CHECK(L->mK.alloc(9 * (size_t)nnz));
    CR_CHECK(L->mG.alloc(3 * (size_t)nnz));
    CR_CHECK(L->mD.alloc(3 * (size_t)nnz));
    CR_CHECK(L->mL.alloc((size_t)nnz));
    CR_CHECK(L->Rm.alloc(3 * (size_t)nNo));
    CR_CHECK(L->Rc.alloc((size_t)nNo));
    CR_CHECK(L->Rmi.alloc(3 * (size_t)nNo));
    CR_CHECK(L->Rci.alloc((size_t)nNo));
    CR_CHECK(L->U.alloc(3 * (size_t)nNo * iB));
    CR_CHECK(L->P.alloc((size_t)nNo * iB));
    CR_CHECK(L->MU.alloc(3 * (size_t)nNo * 2 * iB));
    CR_CHECK(L->MP.alloc((size_t)nNo * 2 * iB));
    CR_CHECK(L->basis.alloc(3 * (size_t)nNo * (sD + 1)));
    CR_CHECK(L->w3.alloc(3 * (size_t)nNo));
    CR_CHECK(L->cgX.alloc((size_t)nNo));
    CR_CHECK(L->cgSP.alloc((size_t)nNo));
    CR_CHECK(sell_pattern(L));
    if (!L->scal.p) {
        CR_CHECK(L->scal.alloc(kScalTotal));
        CR_CHECK(L->red.init());
        CR_CUDA(cudaMallocHost(&L->hscal, sizeof(double) * kScalTotal));
        CR_CUDA(cudaEventCreate(&L->ev0));
        CR_CUDA(cudaEventCreate(&L->ev1));
        CR_CUDA(cudaEventCreate(&L->s2_ev0));
        CR_CUDA(cudaEventCreate(&L->s2_ev1));
    }
    return CRIMSON_OK;
}

// memLS_SOLVE face flags (memLS.f90:1955-1986)
static void set_face_flags(crimson_lhs* L, const int* incL, const double* res) {
    for (int fa = 0; fa < L->nFaces; ++fa) {
        MemlsFace& f = L->face[fa];
        f.incFlag = !(incL && incL[fa] == 0);
        f.coupledFlag = false;
        if (!f.incFlag) continue;
        if (f.bGrp == CRIMSON_BC_TYPE_NEU && res && res[fa] != 0.0) {
            f.res = res[fa];
            f.coupledFlag = true;
        }
    }
}

// Dirichlet W scaling + valM of coupled faces (tail of PRECOND)
static int precond_faces(crimson_lhs* L, bool after_scale) {
    cudaStream_t s = L->stream;
    for (auto& f : L->face) {
        if (!f.created || f.nNo == 0) continue;
        if (!after_scale) {
            if (f.incFlag && f.bGrp == CRIMSON_BC_TYPE_DIR)
                launch(k_w_dirichlet, grid_for(f.nNo, 256), 256, 0, s, f.glob.p, f.val.p, f.dof, std::min(f.dof, 4),
                       f.nNo, L->W.p);
        } else if (f.coupledFlag) {
            launch(k_valm, grid_for(f.nNo, 256), 256, 0, s, f.glob.p, f.val.p, f.valM.p, f.dof, std::min(f.dof, 4),
                   f.nNo, L->W.p);
        }
    }
    CR_CUDA(cudaGetLastError());
    return CRIMSON_OK;
}

// One line per NS solve in the format of memLS's LOGFILE
// (flowsolver/src/memLS.f90:1720-1757), appended to ls->log_path when set:
// a header "gnNo nTasks nCoupledFaces" when the file is new, then the
// success code (100 RI + 10 GM + CG), RI / GM / CG iterations, the time
// split other / GM / CG in percent, the initial norm, the relative final
// norm, the wall time, Resm, Resc and dB.
static void log_solve(const crimson_lhs* L, const crimson_ls* ls) {
    if (ls->log_path.empty()) return;
    FILE* probe = std::fopen(ls->log_path.c_str(), "r");
    const bool exists = probe != nullptr;
    if (probe) std::fclose(probe);
    FILE* f = std::fopen(ls->log_path.c_str(), "a");
    if (!f) return;
    if (!exists) {
        int nc = 0;
        for (const auto& fc : L->face)
            if (fc.coupledFlag) ++nc;
        std::fprintf(f, "%12d%12d%12d\n", L->gnNo, 1, nc);
    }
    const int code = (ls->RI.suc ? 100 : 0) + (ls->GM.suc ? 10 : 0) + (ls->CG.suc ? 1 : 0);
    const double t = ls->RI.callD > 0.0 ? ls->RI.callD : 1.0;
    std::fprintf(f, "%4.3d%3d%4d%5d%4ld%4ld%4ld%9.2E%9.2E%9.2E%4d%4d%4ld\n", code, ls->RI.itr, ls->GM.itr,
                 ls->CG.itr, std::lround((ls->RI.callD - ls->GM.callD - ls->CG.callD) / t * 1e2),
                 std::lround(ls->GM.callD / t * 1e2), std::lround(ls->CG.callD / t * 1e2), ls->RI.iNorm,
                 ls->RI.iNorm != 0.0 ? ls->RI.fNorm / ls->RI.iNorm : 0.0, ls->RI.callD, ls->Resm, ls->Resc,
                 std::lround(ls->RI.dB));
    std::fclose(f);
}

static void copy_stats(const crimson_ls* ls, crimson_ls_stats* st) {
    if (!st) return;
    st->GM = ls->GM;
    st->CG = ls->CG;
    st->RI = ls->RI;
    st->LS_type = ls->LS_type;
    st->Resm = ls->Resm;
    st->Resc = ls->Resc;
}

// FP64 defect of the scaled system: D4 = R0 - A x (A with the coupled-face
// momentum term of ADDBCMUL(ADD)); returns |D4| and |R0|.
static int defect64(crimson_lhs* L, const double* R0, const double* x4, double* D4, double* nD, double* nR) {
    Ctx C{L, L->stream};
    cudaStream_t s = L->stream;
    const int n = L->nNo;
    // x split into xu (3, n) in Rmi and xp (n) in Rci; products into MU/MP slots 0
    launch(k_split4, grid_for(n, 256), 256, 0, s, x4, L->Rmi.p, L->Rci.p, n);
    double* KU = L->MU.p;
    double* GPm = L->MU.p + 3 * (size_t)n;
    double* DU = L->MP.p;
    double* LP = L->MP.p + (size_t)n;
    C.vv3((const double*)L->mK.p, (const double*)L->Rmi.p, KU);
    C.addbcmul(0, 3, (const double*)L->Rmi.p, KU);
    C.sv3((const double*)L->mG.p, (const double*)L->Rci.p, GPm);
    C.vs3((const double*)L->mD.p, (const double*)L->Rmi.p, DU);
    C.ss((const double*)L->mL.p, (const double*)L->Rci.p, LP);
    launch(k_defect4, grid_for(n, 256), 256, 0, s, R0, (const double*)KU, (const double*)GPm, (const double*)DU,
           (const double*)LP, D4, n);
    C.dot(D4, (const double*)D4, 4LL * n, 0);
    C.dot(R0, R0, 4LL * n, 1);
    CR_CHECK(C.sync_scal(0, 2));
    *nD = std::sqrt(L->hscal[0]);
    *nR = std::sqrt(L->hscal[1]);
    return CRIMSON_OK;
}

// NSSOLVER on the scaled system in L->R (in/out).  FP64: the reference's
// arithmetic.  Mixed: FP32 sliced copies of the scaled split matrices drive
// the Krylov matvecs (GMRES, CGRAD); every other product, in particular the
// A d of the search directions that enter the least-squares problem, uses
// the FP64 matrices, so a sweep's residual estimate is that of the FP64
// operator.  Each sweep solves A d = D, adds d to the FP64 solution and
// forms the FP64 defect D = R0 - A x, until |D| <= refine_tol |R0|
// (RI.relTol when refine_tol <= 0) or max_refine sweeps.  Every sweep's
// NSSOLVER stops at its own relative tolerances, so the sweeps reach a
// defect below what one NSSOLVER's estimate can resolve.  Iteration counts
// are summed over the sweeps.  has_gt: Gt is a separate matrix (host Val path),
// otherwise mD serves as Gt.
static int solve_scaled(crimson_lhs* L, crimson_ls* ls, bool has_gt) {
    cudaStream_t s = L->stream;
    const double* Gt64 = has_gt ? L->Gt.p : L->mD.p;
    if (ls->precision == CRIMSON_FP64)
        return nssolver<double, double>(L, ls, L->mK.p, L->mG.p, L->mD.p, L->mL.p, Gt64, L->R.p);
    const int n = L->nNo;
    CR_CHECK(L->R0.alloc(4 * (size_t)n));
    CR_CHECK(L->X4.alloc(4 * (size_t)n));
    CR_CUDA(cudaMemcpyAsync(L->R0.p, L->R.p, sizeof(double) * 4 * (size_t)n, cudaMemcpyDeviceToDevice, s));
    CR_CUDA(cudaMemsetAsync(L->X4.p, 0, sizeof(double) * 4 * (size_t)n, s));
    crimson_subls gm{}, cg{}, ri{};
    const double tol = ls->refine_tol > 0.0 ? ls->refine_tol : ls->RI.relTol;
    double rel = 1.0;
    L->refine_steps = 0;
    // Each sweep solves for the defect scaled to the norm of the original
    // right side, so the Krylov solvers' absolute tolerances and GE's
    // absolute pivot test see the same magnitudes in every sweep.  A later
    // sweep only has to bring the defect from nD to tol nR: its outer
    // relative tolerance is kRefineSafety * tol nR / nD (never tighter than
    // the first sweep's), so it stops after the reduction it needs.
    constexpr double kRefineSafety = 0.3;
    struct RelTolGuard {
        crimson_subls& ri;
        double v;
        ~RelTolGuard() { ri.relTol = v; }
    } guard{ls->RI, ls->RI.relTol};
    double sigma = 1.0;
    for (int ref = 0; ref < std::max(ls->max_refine, 1); ++ref) {
        CR_CHECK((nssolver<float, float>(L, ls, L->mK.p, L->mG.p, L->mD.p, L->mL.p, Gt64, L->R.p)));
        if (ref == 0) {
            gm = ls->GM;
            cg = ls->CG;
            ri = ls->RI;
        } else {
            gm.itr += ls->GM.itr;
            cg.itr += ls->CG.itr;
            ri.itr += ls->RI.itr;
            gm.callD += ls->GM.callD;
            cg.callD += ls->CG.callD;
            ri.callD += ls->RI.callD;
        }
        launch(k_axpy<double, double>, grid_for(4LL * n, 256), 256, 0, s, 1.0 / sigma, (const double*)L->R.p,
               L->X4.p, 4LL * n);
        double nD = 0.0, nR = 0.0;
        CR_CHECK(defect64(L, L->R0.p, L->X4.p, L->R.p, &nD, &nR));
        rel = nR > 0.0 ? nD / nR : 0.0;
        L->refine_steps = ref + 1;
        L->refine_rel = rel;
        if (!(rel > tol) || nD == 0.0) break;
        if (!std::isfinite(rel)) return CRIMSON_ERR_NONFINITE;
        sigma = nR / nD;
        launch(k_scale, grid_for(4LL * n, 256), 256, 0, s, sigma, L->R.p, 4LL * n);
        ls->RI.relTol = std::min(0.5, std::max(guard.v, kRefineSafety * tol / rel));
    }
    ls->RI.relTol = guard.v;
    ri.relTol = guard.v;
    ri.fNorm = rel * ri.iNorm;
    ri.suc = rel <= tol ? 1 : 0;
    ls->GM = gm;
    ls->CG = cg;
    ls->RI = ri;
    CR_CUDA(cudaMemcpyAsync(L->R.p, L->X4.p, sizeof(double) * 4 * (size_t)n, cudaMemcpyDeviceToDevice, s));
    return CRIMSON_OK;
}

int memls_solve_val(crimson_lhs* L, crimson_ls* ls, double* Ri, double* Val, const int* incL, const double* res,
                    crimson_ls_stats* st) {
    cudaStream_t s = L->stream;
    CR_CHECK(lhs_work_alloc(L, ls));
    CR_CHECK(L->Val.alloc(16 * (size_t)L->nnz));
    CR_CHECK(L->Gt.alloc(3 * (size_t)L->nnz));
    set_face_flags(L, incL, res);
    CR_CUDA(cudaMemcpyAsync(L->R.p, Ri, sizeof(double) * 4 * (size_t)L->nNo, cudaMemcpyHostToDevice, s));
    CR_CUDA(cudaMemcpyAsync(L->Val.p, Val, sizeof(double) * 16 * (size_t)L->nnz, cudaMemcpyHostToDevice, s));
    launch(k_w_from_val, grid_for(L->nNo, 256), 256, 0, s, L->Val.p, L->diag, L->W.p, L->nNo);
    CR_CHECK(precond_faces(L, false));
    launch(k_scale_split_val, grid_for(L->nNo, 128), 128, 0, s, L->Val.p, L->rowptr, L->col, L->diag,
           (const double*)L->W.p, L->nNo, L->mK.p, L->mG.p, L->mD.p, L->mL.p);
    launch(k_gt, grid_for(L->nnz, 256), 256, 0, s, (const double*)L->mG.p, L->trans, L->nnz, L->Gt.p);
    launch(k_mul, grid_for(4LL * L->nNo, 256), 256, 0, s, L->R.p, (const double*)L->W.p, 4LL * L->nNo);
    CR_CHECK(precond_faces(L, true));
    CR_CHECK(solve_scaled(L, ls, true));
    launch(k_mul, grid_for(4LL * L->nNo, 256), 256, 0, s, L->R.p, (const double*)L->W.p, 4LL * L->nNo);
    CR_CUDA(cudaMemcpyAsync(Ri, L->R.p, sizeof(double) * 4 * (size_t)L->nNo, cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaMemcpyAsync(Val, L->Val.p, sizeof(double) * 16 * (size_t)L->nnz, cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    copy_stats(ls, st);
    log_solve(L, ls);
    return CRIMSON_OK;
}

// K_out(j) = K_in(trans(j))^T: the momentum blocks of the transposed system
__global__ void k_transpose_k(const double* __restrict__ Kin, const int* __restrict__ trans, long long nnz,
                              double* __restrict__ Kout) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += (long long)gridDim.x * blockDim.x) {
        const double* k = Kin + 9 * (size_t)trans[j];
        double* o = Kout + 9 * (size_t)j;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) o[3 * a + b] = k[3 * b + a];
    }
}

// R(4, i) = -R(4, i)
__global__ void k_negate_p(double* __restrict__ R, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) R[4 * (size_t)i + 3] = -R[4 * (size_t)i + 3];
}

// transpose: solve with the transposed matrix.  Val4 = [K G; D L] built from
// lhsK / lhsP has G = -D^T (both come from lhsP(1:3)) and a symmetric L
// (the PSPG block is symmetrised per element), so
//   A^T = [K^T  -G; -D  L]  and  A^T [u; p] = [f; g]  <=>  [K^T G; D L] [u; -p] = [f; -g]:
// the same NS solve with the momentum blocks transposed and the pressure
// rows of the right side and of the solution negated.  The diagonal
// scaling, Dirichlet faces and the (symmetric) coupled-face terms carry over.
int memls_solve_lhs_device(crimson_lhs* L, crimson_ls* ls, const double* d_res, const double* d_lhsK,
                           const double* d_lhsP, const int* incL, const double* faceRes, double* d_sol,
                           crimson_ls_stats* st, bool transpose, const float* d_lhs32) {
    const TangentIn T{d_lhsK, d_lhsP, d_lhs32};
    cudaStream_t s = L->stream;
    CR_CHECK(lhs_work_alloc(L, ls));
    set_face_flags(L, incL, faceRes);
    CR_CUDA(cudaMemcpyAsync(L->R.p, d_res, sizeof(double) * 4 * (size_t)L->nNo, cudaMemcpyDeviceToDevice, s));
    launch(k_w_from_lhs, grid_for(L->nNo, 256), 256, 0, s, T, L->diag, L->W.p, L->nNo);
    CR_CHECK(precond_faces(L, false));
    launch(k_scale_split_lhs, grid_for(16LL * L->nNo, 128), 128, 0, s, T, L->rowptr, L->col, L->diag, L->trans,
           (const double*)L->W.p, L->nNo, L->mK.p, L->mG.p, L->mD.p, L->mL.p);
    launch(k_mul, grid_for(4LL * L->nNo, 256), 256, 0, s, L->R.p, (const double*)L->W.p, 4LL * L->nNo);
    CR_CHECK(precond_faces(L, true));
    if (transpose) {
        CR_CHECK(L->mKt.alloc(9 * (size_t)L->nnz));
        launch(k_transpose_k, grid_for(L->nnz, 256), 256, 0, s, (const double*)L->mK.p, L->trans, L->nnz, L->mKt.p);
        std::swap(L->mK, L->mKt);
        launch(k_negate_p, grid_for(L->nNo, 256), 256, 0, s, L->R.p, L->nNo);
    }
    // With Val4 built from lhsK/lhsP, Gt = -mG^T equals mD up to the order of
    // the two scaling products, so mD serves as Gt.
    CR_CHECK(solve_scaled(L, ls, false));
    if (transpose) launch(k_negate_p, grid_for(L->nNo, 256), 256, 0, s, L->R.p, L->nNo);
    launch(k_mul, grid_for(4LL * L->nNo, 256), 256, 0, s, L->R.p, (const double*)L->W.p, 4LL * L->nNo);
    CR_CUDA(cudaMemcpyAsync(d_sol, L->R.p, sizeof(double) * 4 * (size_t)L->nNo, cudaMemcpyDeviceToDevice, s));
    CR_CUDA(cudaStreamSynchronize(s));
    copy_stats(ls, st);
    log_solve(L, ls);
    return CRIMSON_OK;
}

// Diagnostics.  which: 0 = 3x3 block SpMV (K, sliced, FP64, as GMRES runs
// it), 1 = one CG iteration of the persistent FP64 CGRAD kernel (average over
// all launches so far, from CUDA events recorded around each launch),
// 2 = SPARMULSV (G), 3 = fused MGS step, 4 = one CG iteration of the
// FP32-matrix CGRAD kernel, 5 = 3x3 block SpMV with the sliced FP32 K,
// 6 = 3x3 block SpMV on the CSR FP64 K (four lanes per row).
int memls_kernel_time(crimson_lhs* L, int which, int reps, double* ms) {
    if (which == 1 || which == 4) {
        const auto& acc = which == 1 ? L->cg_acc64 : L->cg_acc32;
        if (acc.iters <= 0) return CRIMSON_ERR_STATE;
        *ms = acc.ms / (double)acc.iters;
        return CRIMSON_OK;
    }
    if (!L->mK.p || !L->basis.p || reps <= 0) return CRIMSON_ERR_STATE;
    if ((which == 5 && !L->Ks32.p) || (which == 0 && !L->Ks64.p)) return CRIMSON_ERR_STATE;
    cudaStream_t s = L->stream;
    Ctx C{L, s};
    const long long n3 = 3LL * L->nNo;
    cudaEvent_t e0, e1;
    CR_CUDA(cudaEventCreate(&e0));
    CR_CUDA(cudaEventCreate(&e1));
    auto run = [&]() {
        switch (which) {
            case 0: C.vv3s((const double*)L->Ks64.p, (const double*)L->basis.p, L->basis.p + n3); break;
            case 6: C.vv3((const double*)L->mK.p, (const double*)L->basis.p, L->basis.p + n3); break;
            case 2: C.sv3((const double*)L->mG.p, (const double*)L->cgX.p, L->w3.p); break;
            case 5: C.vv3s((const float*)L->Ks32.p, (const double*)L->basis.p, L->basis.p + n3); break;
            default:
                launch(k_mgs<double>, red_grid(n3), 256, 0, s, L->basis.p + 2 * n3, (const double*)L->basis.p,
                       (const double*)C.sc(kSlotH), (const double*)(L->basis.p + n3), n3, L->red.part.p,
                       L->red.ticket.p, C.sc(kSlotH + 1));
        }
    };
    for (int i = 0; i < 2; ++i) run();
    CR_CUDA(cudaEventRecord(e0, s));
    for (int i = 0; i < reps; ++i) run();
    CR_CUDA(cudaEventRecord(e1, s));
    CR_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    CR_CUDA(cudaEventElapsedTime(&t, e0, e1));
    *ms = (double)t / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CR_CUDA(cudaGetLastError());
    return CRIMSON_OK;
}

}  // namespace crimson
