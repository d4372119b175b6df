// Shared device helpers and the internal context layout of crimson_b200.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/crimson_b200.h"

namespace crimson {

// Last error text (per host thread).
void set_last_error(const std::string& s);

#define CR_CUDA(call)                                                                    \
    do {                                                                                 \
        cudaError_t _e = (call);                                                         \
        if (_e != cudaSuccess) {                                                         \
            ::crimson::set_last_error(std::string(#call) + ": " + cudaGetErrorString(_e)); \
            return _e == cudaErrorMemoryAllocation ? CRIMSON_ERR_OOM : CRIMSON_ERR_CUDA;  \
        }                                                                                \
    } while (0)

#define CR_CHECK(expr)                    \
    do {                                  \
        int _rc = (expr);                 \
        if (_rc != CRIMSON_OK) return _rc; \
    } while (0)

// Owning device buffer.
template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            n = o.n;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    int alloc(size_t count) {
        if (count == n && p) return CRIMSON_OK;
        release();
        if (count == 0) return CRIMSON_OK;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            set_last_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
            return CRIMSON_ERR_OOM;
        }
        n = count;
        return CRIMSON_OK;
    }
    int upload(const T* h, size_t count, cudaStream_t s) {
        CR_CHECK(alloc(count));
        if (count) {
            cudaError_t e = cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) {
                set_last_error(cudaGetErrorString(e));
                return CRIMSON_ERR_CUDA;
            }
        }
        return CRIMSON_OK;
    }
};

// Count of kernels this library has launched (diagnostics: crimson_launch_count).
void note_launch();

// Every kernel launch of the library goes through here.
template <typename... KArgs, typename... Args>
inline void launch(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
    note_launch();
    k<<<grid, block, smem, s>>>(static_cast<KArgs>(args)...);
}

// Number of SMs of the current device (148 on B200).
int sm_count();

// Grid size for a grid-stride loop: a multiple of the SM count.
inline int grid_for(long long n, int block, int per_sm = 8) {
    long long want = (n + block - 1) / block;
    long long cap = (long long)sm_count() * per_sm;
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

// ---------------------------------------------------------------------------
// Warp / block reductions (FP64)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum; every thread receives the result.  smem: >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* smem) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) smem[wid] = v;
    __syncthreads();
    double t = (threadIdx.x < nw) ? smem[threadIdx.x] : 0.0;
    if (wid == 0) t = warp_sum(t);
    if (threadIdx.x == 0) smem[0] = t;
    __syncthreads();
    double r = smem[0];
    __syncthreads();
    return r;
}

}  // namespace crimson

// ---------------------------------------------------------------------------
// Internal context.  Device arrays are 0-based and node-major.
// ---------------------------------------------------------------------------
struct crimson_ctx {
    crimson_params p{};
    int nshg = 0, numnp = 0, nelem = 0;
    cudaStream_t stream = nullptr;

    // mesh
    crimson::DBuf<int4> ien;        // (nelem) 0-based node ids
    crimson::DBuf<double4> x;       // (numnp) coordinates, w unused

    // Dirichlet data
    crimson::DBuf<int> iBC;         // (nshg)
    crimson::DBuf<double> BC;       // (ndofBC, nshg) node-major
    std::vector<int> h_iBC;         // the codes on the device (iBC above)
    std::vector<int> h_iBC_orig;    // the codes crimson_set_bc received (iBC_original of itrdrv.f90)
    int npartial = 0;               // nodes with one or two prescribed velocity components
    std::vector<double> h_BC;       // reference layout (nshg, ndofBC)
    std::vector<double> h_x;        // (numnp, 3) reference layout, host copy
    std::vector<int4> h_ienb;       // (nface) host copy of ienb

    // boundary faces (AsBMFG)
    int nface = 0;
    crimson::DBuf<int4> ienb;       // (nface) 0-based, face nodes first
    crimson::DBuf<int> iBCB;        // (nface) flag bits
    crimson::DBuf<double> BCB;      // (nface, 3, 6) as [f*18 + n*6 + c]
    crimson::DBuf<int> fnoff;       // (nshg+1) offsets into flist per node
    crimson::DBuf<int> flist;       // (3 nface) codes 3f + n of the faces at each node, ascending f
    crimson::DBuf<double> frec;     // (nface, 12) face residual records: rl(n, 0:3) of face node n
    std::vector<int> h_iBCB;        // (nface) flag bits, host copy
    std::vector<int> h_face_srf;    // (nface) surface ids, host copy
    // surface-pressure integrals (integrScalar, boundarydata.f90:1101-1140):
    // per coupled surface its nodes (ndsurf) and its edge nodes (ndsurf 1,
    // edsurf the surface), ascending, with their NASC weights
    crimson::DBuf<int> pnodes;
    crimson::DBuf<double> pw;
    std::vector<int> pnode_off;
    crimson::DBuf<int> bcount;      // (nshg) boundary elements (all 4 nodes) containing each node

    // coupled outlets
    int ncoupled = 0;
    std::vector<int> srflist;
    crimson::DBuf<int> onodes;      // outlet node ids grouped by surface
    std::vector<int> onode_off;     // (ncoupled+1) offsets into onodes
    std::vector<double> oarea;      // (ncoupled) surface area: sum of NASC over the surface's nodes
    std::vector<int> h_onodes;      // host copy of onodes
    crimson::DBuf<double> psurf;    // (ncoupled) surface pressure integrals
    crimson::DBuf<int> d_onode_off; // device copy of onode_off
    crimson::DBuf<double4> onabi;   // NABI of those nodes
    crimson::DBuf<double> flowq;    // (ncoupled) device scratch for Q
    crimson::DBuf<double> coefs;    // (2*ncoupled) device copy of coef1, coef2
    std::vector<double> coef_host;  // (2*ncoupled) host staging of coef1, coef2

    // pattern (built by crimson_genadj)
    long long nnz = 0;
    crimson::DBuf<int> rowptr;      // (nshg+1) 0-based
    crimson::DBuf<int> col;         // (nnz) 0-based
    crimson::DBuf<int> diag;        // (nshg) position of the diagonal block
    crimson::DBuf<int> trans;       // (nnz) position of the transposed block
    // Contribution lists of the owner-computes scatter: slist holds the
    // element pairs t = 16 e + 4 a + b grouped by CSR slot, ascending t within
    // a slot; slot s owns slist[soff[s] .. soff[s+1]).  The diagonal slot of
    // node i lists exactly the elements containing i (b == a).
    crimson::DBuf<int> slist;       // (nelem*16)
    crimson::DBuf<int> soff;        // (nnz+1)

    // ElmGMR work space
    crimson::DBuf<double> qres;     // (nshg, 9) node-major: q[9*i + k]
    crimson::DBuf<double> rmass;    // (nshg) 1 / lumped mass (geometry only)
    bool rmass_ready = false;       // rmass holds the inverse lumped mass
    crimson::DBuf<double> qrec;     // (nelem, 8) AsIq element records {W, q11,q12,q13,q22,q23,q33, 0}
    crimson::DBuf<double> erec;     // (nelem, 48) element records of the residual and tangent
    crimson::DBuf<double> y4, ac4, res4;   // (4, nshg) staging for host-pointer calls
    crimson::DBuf<double> lhsK, lhsP;      // (9, nnz), (4, nnz)
    crimson::DBuf<float> lhs32;            // (16, nnz) FP32 tangent records (mixed precision)

    // ElmGMRSclr work space (scalar advection-diffusion)
    crimson::DBuf<double> sclr_qres;       // (nshg, 3) projected diffusive flux, node-major
    crimson::DBuf<double> sclr_qrec;       // (nelem, 4) {diffus grad S, W}
    crimson::DBuf<double> sclr_erec;       // (nelem, 8) {rl(a), xSebe(a, a)}
    crimson::DBuf<double> sclr_xoff;       // (nelem, 12) off-diagonal xSebe
    crimson::DBuf<double> sclr_frec;       // (nface, 3) boundary flux terms
    crimson::DBuf<double> sclr_in, sclr_res, sclr_lhs;  // staging for host-pointer calls

    // time stepping state (crimson_step)
    crimson::DBuf<double> yold, acold, ycur, accur, yalpha, acalpha, solinc, stage;

    // adjoint work space (crimson_elmgmr_vjp)
    crimson::DBuf<double> adj_res, adj_lam, adj_qbar, adj_scal;

    // 4x4 block SpMV (crimson_spmv4_*): sliced pattern and values
    crimson::DBuf<int> s4_ptr, s4_col;
    long long s4_npad = 0;
    int s4_nslice = 0, s4_prec = 0;
    crimson::DBuf<double> s4_val64;
    crimson::DBuf<float> s4_val32;
    crimson::DBuf<int> inlet_nodes;
    crimson::DBuf<double> inlet_profile;   // (ninlet, 3)
    int ninlet = 0;
    std::vector<double> rcr_Rp, rcr_C, rcr_Rd, rcr_Pd, rcr_Pn, rcr_Qn;
    std::vector<crimson_netlist*> netlists;  // per coupled surface; null: the RCR (not owned)
    std::vector<crimson_netlist_loop*> loops;       // closed loops (not owned)
    std::vector<std::vector<int>> loop_surfaces;    // per loop: the coupled surface of each upstream circuit
    std::vector<int> loop_of;                       // per coupled surface: its loop, or -1
    int istep = 0;
    int res_iter = 0;                 // residual control: iterations since the last early exit
    crimson::DBuf<double> sumsq;      // residual control: block partials + total
};
