// Outlet coupling (GetFlowQ + ElmpvsQ right-hand side) without any device
// allocation, for callers that cannot call cudaMalloc.
//
// Who needs it: a host code that couples this solver to its own 0D/lumped
// outlet models from inside a region where it must not allocate device
// memory -- for example while its stream is being captured into a CUDA graph
// (cudaMalloc is not capturable), from a callback running under a framework
// that owns all device memory through its own pool, or in a
// latency-sensitive inner loop where an allocation would synchronise the
// device.  The regular path (crimson_elmgmr_device) keeps the per-surface
// flows in memory the context allocated; this variant keeps them in a
// file-scope static device array instead.
//
// Scratch: g_pvsq_scratch holds one flow value per coupled surface, at most
// kPvsqMaxSurf (64) surfaces = 512 bytes.  Every GPU that loads the library
// holds this array until the process exits.  Host code never dereferences
// the symbol: its device address is obtained once per device with
// cudaGetSymbolAddress (the first call on each device does this set-up, so
// that first call should come before any stream capture) and passed to the
// kernels.  All calls share the array and it keeps the last call's values;
// each call overwrites every slot it uses before reading it, so nothing has
// to start at zero.  Calls that overlap on the GPU (different streams, no
// ordering between them) race on the array.
#include <mutex>

#include "common.cuh"

namespace crimson {

constexpr int kPvsqMaxSurf = 64;

static __device__ __align__(256) double g_pvsq_scratch[kPvsqMaxSurf];

struct PvsqArgs {
    int nsurf;
    int off[kPvsqMaxSurf + 1];
    double coef1[kPvsqMaxSurf];
    double coef2[kPvsqMaxSurf];
};

// Q_k = sum over the surface's nodes of NABI . u   (boundarydata.f90:1157-1196)
__global__ void k_flowq_noalloc(const int* __restrict__ nodes, const double* __restrict__ nabi,
                                const double* __restrict__ y, PvsqArgs a, double* __restrict__ q) {
    __shared__ double sm[32];
    const int k = blockIdx.x;
    double s = 0.0;
    for (int t = a.off[k] + threadIdx.x; t < a.off[k + 1]; t += blockDim.x) {
        const double* nb = nabi + 3 * (size_t)t;
        const double* yv = y + 4 * (size_t)(nodes[t] - 1);
        s += nb[0] * yv[0] + nb[1] * yv[1] + nb[2] * yv[2];
    }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) q[k] = s;
}

// res(i,1:3) += p_k NABI(i,:), p_k = -(Q_k coef1_k) - coef2_k  (elmgmr.f90:1298-1330)
__global__ void k_pvsq_apply_noalloc(const int* __restrict__ nodes, const double* __restrict__ nabi,
                                     const double* __restrict__ q, PvsqArgs a, double* __restrict__ res) {
    const int k = blockIdx.y;
    const double pk = -1.0 * (q[k] * a.coef1[k]) - a.coef2[k];
    for (int t = a.off[k] + blockIdx.x * blockDim.x + threadIdx.x; t < a.off[k + 1]; t += gridDim.x * blockDim.x) {
        const double* nb = nabi + 3 * (size_t)t;
        double* r = res + 4 * (size_t)(nodes[t] - 1);
        // atomic: a caller's lists may name a node under several surfaces
        atomicAdd(r + 0, pk * nb[0]);
        atomicAdd(r + 1, pk * nb[1]);
        atomicAdd(r + 2, pk * nb[2]);
    }
}

// Device address of g_pvsq_scratch for the current device (set up once per device).
static int scratch_ptr(double** out) {
    static std::mutex mu;
    static double* ptrs[64] = {nullptr};
    int dev = 0;
    CR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CRIMSON_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(mu);
    if (!ptrs[dev]) {
        void* p = nullptr;
        CR_CUDA(cudaGetSymbolAddress(&p, g_pvsq_scratch));
        ptrs[dev] = static_cast<double*>(p);
    }
    *out = ptrs[dev];
    return CRIMSON_OK;
}

}  // namespace crimson

extern "C" int crimson_pvsq_noalloc(int nsurf, const int* surf_offsets, const int* d_nodes, const double* d_nabi,
                                    const double* d_y, const double* coef1, const double* coef2, double* d_res,
                                    double* q_out, void* stream) {
    using namespace crimson;
    if (nsurf < 0 || (nsurf > 0 && (!surf_offsets || !d_nodes || !d_nabi || !d_y || !coef1 || !coef2 || !d_res)))
        return CRIMSON_ERR_ARG;
    if (nsurf > kPvsqMaxSurf) {
        set_last_error("crimson_pvsq_noalloc: at most 64 coupled surfaces (static scratch size)");
        return CRIMSON_ERR_UNSUPPORTED;
    }
    if (nsurf == 0) return CRIMSON_OK;
    PvsqArgs a;
    a.nsurf = nsurf;
    if (surf_offsets[0] != 0) {
        set_last_error("crimson_pvsq_noalloc: surf_offsets[0] must be 0");
        return CRIMSON_ERR_ARG;
    }
    for (int k = 0; k <= nsurf; ++k) a.off[k] = surf_offsets[k];
    for (int k = 0; k < nsurf; ++k) {
        if (surf_offsets[k + 1] < surf_offsets[k]) {
            set_last_error("crimson_pvsq_noalloc: surf_offsets must not decrease");
            return CRIMSON_ERR_ARG;
        }
        a.coef1[k] = coef1[k];
        a.coef2[k] = coef2[k];
    }
    for (int k = nsurf + 1; k <= kPvsqMaxSurf; ++k) a.off[k] = a.off[nsurf];
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (q_out) {
        // the copy-back waits for the stream, which a capture forbids
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CR_CUDA(cudaStreamIsCapturing(s, &cs));
        if (cs != cudaStreamCaptureStatusNone) {
            set_last_error("crimson_pvsq_noalloc: q_out must be NULL while the stream is being captured");
            return CRIMSON_ERR_UNSUPPORTED;
        }
    }
    double* q = nullptr;
    CR_CHECK(scratch_ptr(&q));
    launch(k_flowq_noalloc, nsurf, 256, 0, s, d_nodes, d_nabi, d_y, a, q);
    launch(k_pvsq_apply_noalloc, dim3(8, nsurf), 256, 0, s, d_nodes, d_nabi, (const double*)q, a, d_res);
    CR_CUDA(cudaGetLastError());
    if (q_out) {
        CR_CUDA(cudaMemcpyAsync(q_out, q, sizeof(double) * nsurf, cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
    }
    return CRIMSON_OK;
}
