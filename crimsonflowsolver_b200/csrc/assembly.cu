// ElmGMR on the device: diffusive-flux reconstruction (AsIq/qpbc), interior
// residual + tangent (AsIGMR/e3/e3LHS + fillsparseI), boundary residual
// (AsBMFG/e3b), outlet coupling (ElmpvsQ) and bc3Res.
//
// Reference: flowsolver/src/elmgmr.f90:82-555 and the e3* routines it calls.
//
// Element kernels use four lanes per linear tet.  In the quadrature phase lane
// q evaluates quadrature point q (e3ivar/e3stab/e3Res at that point); in the
// output phase lane a owns row a of the element.  Per-point quantities are
// exchanged through shared memory.  On a linear tet the metrics, gradients
// and div q are element constants, so they are computed once per element
// (the reference recomputes them per point with identical inputs), and the
// sums over quadrature points of the tangent terms are formed algebraically:
//   K_ij(a,b) = d_ij Kd(a,b) + tc dN_b,i dN_a,j + tm dN_b,j dN_a,i
//   Kd(a,b)   = tsFct M_ab + tlW (rho sum_q N_a(q) uBar_q.dN_b + 4 mu dN_a.dN_b
//                                 + sum_q (tauM_q rho (u_q.dN_a)(u_q.dN_b)
//                                          + tauBar_q (L_q.dN_a)(L_q.dN_b)))
//   tc = tlW sum_q tauC_q,  tm = 4 mu tlW
//   G_i(a,b)  = tlW dN_b,i sum_q N_a(q)
//   C(a,b)    = tlW/rho (sum_q tauM_q) dN_a.dN_b
// which equals the reference's per-point accumulation (e3lhs.f90:171-402) in
// exact arithmetic; the FP64 results agree to rounding (~1e-15 relative).
//
// Scatter: owner-computes, deterministic.  The element kernel writes one
// record per element (its residual rows and the tangent's element constants
// above: 52 doubles); it never writes a global sum.  A node pass then forms,
// for every node, the residual row and the diagonal tangent block from the
// records of the elements containing it, and a slot pass forms every
// off-diagonal CSR block from the records of the elements containing that
// edge.  Each sum runs over the pattern pass's contribution list of the
// slot (ascending element order, the order of the reference's serial
// scatter, local.f90:64-75, fillsparse.f90:47-60): the slot pass in that
// order, the node pass over kOwnerLanes lanes per node that take the list
// round-robin and combine in a fixed butterfly -- so every result is the
// same bit for bit on every run.  Records are written once and re-read by
// the 4 (node pass) and 12 (slot pass) owners of their element, mostly from
// L2 on banded node numberings.
#include <mutex>

#include "common.cuh"

namespace crimson {

int build_pattern(crimson_ctx* c);

struct ElmConst {
    double shp[4][4];   // shp[q][n]: shape value of node n at quadrature point q
    double shgl[3][4];  // local gradients (halved), identical at every point
    double Qwt;         // quadrature weight (1/4 * 4/3)
    double M[4][4];     // sum_q N_a(q) N_b(q)
    double SN[4];       // sum_q N_a(q)
    double shpb[3][4];  // boundary rule: shape values at the 3 face points
    double Qwtb;        // boundary weight (2 * 1/3)
};

__constant__ ElmConst c_el;

struct ElmParams {
    double rho, mu, alfi, almi, gami, Delt, Dtgl, dtsfct, taucfct, stabflux;
    int idiff;
};

static ElmConst make_consts() {
    // 4-point rule of flowsolver/src/symtet.c:22-23,72-74; shapes of uniformP.c:22-40
    const double A4 = 0.5854101966249685, B4 = 0.1381966011250150;
    const double rstw4[4][3] = {{A4, B4, B4}, {B4, A4, B4}, {B4, B4, A4}, {B4, B4, B4}};
    ElmConst k{};
    for (int q = 0; q < 4; ++q) {
        const double* par = rstw4[q];
        k.shp[q][0] = par[0];
        k.shp[q][1] = par[1];
        k.shp[q][2] = par[2];
        k.shp[q][3] = 1.0e0 - par[0] - par[1] - par[2];
    }
    for (int n = 0; n < 4; ++n)
        for (int j = 0; j < 3; ++j) k.shgl[j][n] = (n == 3 ? -1.0 : (n == j ? 1.0 : 0.0)) / 2.0;
    k.Qwt = (4.0 / 3.0) * 0.25;
    for (int a = 0; a < 4; ++a) {
        k.SN[a] = 0.0;
        for (int b = 0; b < 4; ++b) {
            k.M[a][b] = 0.0;
            for (int q = 0; q < 4; ++q) k.M[a][b] += k.shp[q][a] * k.shp[q][b];
        }
        for (int q = 0; q < 4; ++q) k.SN[a] += k.shp[q][a];
    }
    // boundary 3-point rule (symtri.c rst3/wt3, genshpb.f90:31-36, genint.f90:86)
    const double B3 = 0.666666666666667, C3 = 0.166666666666667, A3 = 0.3333333333333330000000000000000000;
    const double rst3[3][3] = {{B3, C3, C3}, {C3, B3, C3}, {C3, C3, B3}};
    for (int q = 0; q < 3; ++q) {
        k.shpb[q][0] = rst3[q][0];
        k.shpb[q][1] = rst3[q][1];
        k.shpb[q][2] = rst3[q][2];
        k.shpb[q][3] = 1.0e0 - rst3[q][0] - rst3[q][1] - rst3[q][2];
    }
    k.Qwtb = 2.0 * A3;
    return k;
}

// __constant__ memory is per device: upload the tables once for each device
// that runs an element kernel (the device current on the calling thread,
// which is the device of the context's stream).  Thread-safe.
int upload_elm_consts(cudaStream_t s) {
    static std::mutex mu;
    static bool done[256] = {false};
    int dev = 0;
    CR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) return CRIMSON_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return CRIMSON_OK;
    ElmConst k = make_consts();
    CR_CUDA(cudaMemcpyToSymbolAsync(c_el, &k, sizeof(k), 0, cudaMemcpyHostToDevice, s));
    CR_CUDA(cudaStreamSynchronize(s));
    done[dev] = true;
    return CRIMSON_OK;
}

static ElmParams elm_params(const crimson_params& p) {
    ElmParams e;
    e.rho = p.rho;
    e.mu = p.mu;
    e.alfi = p.alfi;
    e.almi = p.almi;
    e.gami = p.gami;
    e.Delt = p.Delt;
    e.Dtgl = p.Dtgl;
    e.dtsfct = p.dtsfct;
    e.taucfct = p.taucfct;
    e.stabflux = p.stabflux_coeff;
    e.idiff = p.idiff;
    return e;
}

// ---------------------------------------------------------------------------
// Element metrics (e3metric.f90:26-81) from the four vertex coordinates.
// dxidx[i][j] = d xi_i / d x_j ; shg[n][k] = d N_n / d x_k.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void elem_metric(const double xl[4][3], double dxidx[3][3], double shg[4][3],
                                            double* WdetJ) {
    double d[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) d[i][j] = 0.5 * xl[j][i] - 0.5 * xl[3][i];
    dxidx[0][0] = d[1][1] * d[2][2] - d[2][1] * d[1][2];
    dxidx[0][1] = d[2][1] * d[0][2] - d[0][1] * d[2][2];
    dxidx[0][2] = d[0][1] * d[1][2] - d[0][2] * d[1][1];
    double tmp = 1.0 / (dxidx[0][0] * d[0][0] + dxidx[0][1] * d[1][0] + dxidx[0][2] * d[2][0]);
    dxidx[0][0] *= tmp;
    dxidx[0][1] *= tmp;
    dxidx[0][2] *= tmp;
    dxidx[1][0] = (d[1][2] * d[2][0] - d[1][0] * d[2][2]) * tmp;
    dxidx[1][1] = (d[0][0] * d[2][2] - d[2][0] * d[0][2]) * tmp;
    dxidx[1][2] = (d[1][0] * d[0][2] - d[0][0] * d[1][2]) * tmp;
    dxidx[2][0] = (d[1][0] * d[2][1] - d[1][1] * d[2][0]) * tmp;
    dxidx[2][1] = (d[2][0] * d[0][1] - d[0][0] * d[2][1]) * tmp;
    dxidx[2][2] = (d[0][0] * d[1][1] - d[0][1] * d[1][0]) * tmp;
    *WdetJ = c_el.Qwt / tmp;
    // shgl = (e_j/2) for nodes 0..2 and -(1,1,1)/2 for node 3
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        shg[0][k] = 0.5 * dxidx[0][k];
        shg[1][k] = 0.5 * dxidx[1][k];
        shg[2][k] = 0.5 * dxidx[2][k];
        shg[3][k] = -0.5 * dxidx[0][k] - 0.5 * dxidx[1][k] - 0.5 * dxidx[2][k];
    }
}

__device__ __forceinline__ double sel4(const double4& v, int a) {
    return a == 0 ? v.x : (a == 1 ? v.y : (a == 2 ? v.z : v.w));
}
__device__ __forceinline__ float sel4(const float4& v, int a) {
    return a == 0 ? v.x : (a == 1 ? v.y : (a == 2 ? v.z : v.w));
}

// ---------------------------------------------------------------------------
// AsIq + e3q: lumped projection of the viscous flux q = mu (grad u + grad u^T)
// (asiq.f90:52-70, e3q.f90:58-145).  On a linear tet qdi is constant, so
// ql(a,k) = WdetJ sum_q N_a(q) qdi(k) and rmassl(a) = WdetJ sum_q N_a(q).
// Lanes per node in the node passes (k_q_node, k_node_pass).
#ifndef CRIMSON_OWNER_LANES
#define CRIMSON_OWNER_LANES 4
#endif
constexpr int kOwnerLanes = CRIMSON_OWNER_LANES;

// Sum over a node's kOwnerLanes lanes in a fixed butterfly order.
__device__ __forceinline__ double owner_sum(double v) {
#pragma unroll
    for (int o = kOwnerLanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// k_asiq_rec writes one record per element: {WdetJ, q11, q12, q13, q22, q23,
// q33, 0} (qdi is symmetric); k_q_node sums, per node, the records of the
// elements containing it (kOwnerLanes lanes, fixed combining order) and applies qpbc
// (qpbc.f90:67-71).  The lumped mass depends on the geometry only: it is
// summed and inverted on a context's first call and kept (rmass).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_asiq_rec(const int4* __restrict__ ien, const double4* __restrict__ x,
                                                  const double4* __restrict__ y, int nelem, ElmParams P,
                                                  double* __restrict__ qrec) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
        int4 nn = ien[e];
        int nd[4] = {nn.x, nn.y, nn.z, nn.w};
        double xl[4][3], ul[4][3];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            double4 xv = x[nd[a]];
            double4 yv = y[nd[a]];
            xl[a][0] = xv.x;
            xl[a][1] = xv.y;
            xl[a][2] = xv.z;
            ul[a][0] = yv.x;
            ul[a][1] = yv.y;
            ul[a][2] = yv.z;
        }
        double dxidx[3][3], shg[4][3], W;
        elem_metric(xl, dxidx, shg, &W);
        double g[3][3];  // g[k][i] = d u_i / d x_k
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i)
                g[k][i] = shg[0][k] * ul[0][i] + shg[1][k] * ul[1][i] + shg[2][k] * ul[2][i] + shg[3][k] * ul[3][i];
        const double mu = P.mu;
        double4* r = reinterpret_cast<double4*>(qrec + 8 * (size_t)e);
        r[0] = make_double4(W, 2.0 * mu * g[0][0], mu * (g[0][1] + g[1][0]), mu * (g[0][2] + g[2][0]));
        r[1] = make_double4(2.0 * mu * g[1][1], mu * (g[1][2] + g[2][1]), 2.0 * mu * g[2][2], 0.0);
    }
}

__global__ void __launch_bounds__(256) k_q_node(const int* __restrict__ diag, const int* __restrict__ soff,
                                                const int* __restrict__ slist, const double* __restrict__ qrec,
                                                int nshg, int first, double* __restrict__ rmass,
                                                double* __restrict__ qres) {
    constexpr int NPW = 32 / kOwnerLanes;
    const int lane = threadIdx.x & 31, sub = lane % kOwnerLanes;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i0 = warp * NPW; i0 < nshg; i0 += nwarp * NPW) {
        const long long ig = i0 + lane / kOwnerLanes;
        const bool valid = ig < nshg;
        const int i = valid ? (int)ig : nshg - 1;
        const int d = diag[i];
        double q[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, m = 0.0;
        const int p1 = soff[d + 1];
        for (int p = soff[d] + sub; p < p1; p += kOwnerLanes) {
            const int t = slist[p];
            const int e = t >> 4, a = (t >> 2) & 3;
            const double4* r = reinterpret_cast<const double4*>(qrec + 8 * (size_t)e);
            const double4 A = r[0], B = r[1];
            const double wa = A.x * c_el.SN[a];
            // qdi(1:9) column-major 3x3, symmetric
            const double qd[9] = {A.y, A.z, A.w, A.z, B.x, B.y, A.w, B.y, B.z};
#pragma unroll
            for (int k = 0; k < 9; ++k) q[k] += wa * qd[k];
            m += wa;
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) q[k] = owner_sum(q[k]);
        m = owner_sum(m);
        if (!valid || sub != 0) continue;
        double r;
        if (first) {
            r = 1.0 / m;
            rmass[i] = r;
        } else {
            r = rmass[i];
        }
        double* o = qres + 9 * (size_t)i;
#pragma unroll
        for (int k = 0; k < 9; ++k) o[k] = r * q[k];
    }
}

// ---------------------------------------------------------------------------
// AsIGMR / e3 / e3LHS, four lanes per element, writing element records.
//
// Record of element e (RS doubles at erec + RS e, every group 32-byte aligned):
//   kLhs == 1 (FP64 tangent), RS = 52:
//     [0:4)   tc, tm, tlW, cc = tlW/rho sum_q tauM_q
//     [4:20)  grad N_a = (shg[a][0..2], 0) at 4 + 4a: a block (a, b) reads
//             {tc..cc}, grad N_a, grad N_b and Kd(a,b), four sectors
//     [20:36) Kd(a,b) at 20 + 4a + b
//     [36:52) rl(a, 0:4) at 36 + 4a  (momentum 1-3, continuity)
//   kLhs == 2 (FP32 tangent quadrature), RS = 32: rl at [0:16), then 32
//     floats at double offset 16 with the FP32 layout of [0:32) above.
//   kLhs == 0 (residual only), RS = 16: rl at [0:16).
// ---------------------------------------------------------------------------
constexpr int kQ = 28;        // doubles of per-point data exchanged in shared memory
// Shared-memory exchange: element k of a block at k * kQE + q * kQ.  The odd
// element stride (4 kQ + 1 doubles) puts the 8 elements a warp reads at one
// index on 8 different bank pairs (conflict-free broadcast reads), and the
// warp's 32 writes at one index on every bank pair exactly twice.
constexpr int kQE = 4 * kQ + 1;

template <int kLhs>
struct RecLayout {
    static constexpr int RS = kLhs == 1 ? 52 : (kLhs == 2 ? 32 : 16);
    static constexpr int RO = kLhs == 1 ? 36 : 0;
};

// Four blocks of 128 threads per SM (128 registers).
template <int kLhs>
__global__ void __launch_bounds__(128, 4) k_asigmr(const int4* __restrict__ ien, const double4* __restrict__ x,
                                                const double4* __restrict__ y, const double4* __restrict__ ac,
                                                const double* __restrict__ qres, int nelem, ElmParams P,
                                                double* __restrict__ erec) {
    constexpr int RS = RecLayout<kLhs>::RS, RO = RecLayout<kLhs>::RO;
    __shared__ double sq[32 * kQE];
    const int lane4 = threadIdx.x & 3;
    double* const sqe = sq + (threadIdx.x >> 2) * kQE;   // this element's per-point data
    const long long ngroups = (long long)gridDim.x * (blockDim.x >> 2);
    for (long long e0 = (long long)blockIdx.x * (blockDim.x >> 2); e0 < nelem; e0 += ngroups) {
        const long long e = e0 + (threadIdx.x >> 2);
        const bool live = e < nelem;
        int nd[4] = {0, 0, 0, 0};
        double xl[4][3], yl[4][4];
        if (live) {
            int4 nn = ien[e];
            nd[0] = nn.x;
            nd[1] = nn.y;
            nd[2] = nn.z;
            nd[3] = nn.w;
        }
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            double4 xv = live ? x[nd[a]] : make_double4(0, 0, 0, 0);
            double4 yv = live ? y[nd[a]] : make_double4(0, 0, 0, 0);
            xl[a][0] = xv.x;
            xl[a][1] = xv.y;
            xl[a][2] = xv.z;
            // element-local dof order (p, u, v, w) as localy gathers it
            yl[a][0] = yv.w;
            yl[a][1] = yv.x;
            yl[a][2] = yv.y;
            yl[a][3] = yv.z;
        }
        if (!live) {
            // a regular tet so that the dead lanes' arithmetic stays finite
            xl[0][0] = 1.0;
            xl[1][1] = 1.0;
            xl[2][2] = 1.0;
        }
        double dxidx[3][3], shg[4][3], WdetJ;
        elem_metric(xl, dxidx, shg, &WdetJ);
        if (!live) WdetJ = 0.0;
        // global gradients g[k][d] of (p, u, v, w)
        double g[3][4];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int d = 0; d < 4; ++d)
                g[k][d] = shg[0][k] * yl[0][d] + shg[1][k] * yl[1][d] + shg[2][k] * yl[2][d] + shg[3][k] * yl[3][d];
        // div q (e3ivar.f90:354-368): lane a gathers node a's projected flux
        // and the element's 4 lanes sum their terms (fixed butterfly)
        double divq[3] = {0.0, 0.0, 0.0};
        if (P.idiff >= 1) {
            if (live) {
                const double* q = qres + 9 * (size_t)nd[lane4];
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    divq[i] = shg[lane4][0] * q[i] + shg[lane4][1] * q[3 + i] + shg[lane4][2] * q[6 + i];
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                divq[i] += __shfl_xor_sync(0xffffffffu, divq[i], 1);
                divq[i] += __shfl_xor_sync(0xffffffffu, divq[i], 2);
            }
        }
        // metric tensor, tet branch (e3stab.f90:487-528)
        double gij[6];
        {
            const double c1 = 1.259921049894873e+00, c2 = 6.299605249474365e-01;
            double t1, t2, t3;
            t1 = c1 * dxidx[0][0] + c2 * (dxidx[1][0] + dxidx[2][0]);
            t2 = c1 * dxidx[1][0] + c2 * (dxidx[0][0] + dxidx[2][0]);
            t3 = c1 * dxidx[2][0] + c2 * (dxidx[0][0] + dxidx[1][0]);
            gij[0] = dxidx[0][0] * t1 + dxidx[1][0] * t2 + dxidx[2][0] * t3;
            t1 = c1 * dxidx[0][1] + c2 * (dxidx[1][1] + dxidx[2][1]);
            t2 = c1 * dxidx[1][1] + c2 * (dxidx[0][1] + dxidx[2][1]);
            t3 = c1 * dxidx[2][1] + c2 * (dxidx[0][1] + dxidx[1][1]);
            gij[1] = dxidx[0][1] * t1 + dxidx[1][1] * t2 + dxidx[2][1] * t3;
            gij[3] = dxidx[0][0] * t1 + dxidx[1][0] * t2 + dxidx[2][0] * t3;
            t1 = c1 * dxidx[0][2] + c2 * (dxidx[1][2] + dxidx[2][2]);
            t2 = c1 * dxidx[1][2] + c2 * (dxidx[0][2] + dxidx[2][2]);
            t3 = c1 * dxidx[2][2] + c2 * (dxidx[0][2] + dxidx[1][2]);
            gij[2] = dxidx[0][2] * t1 + dxidx[1][2] * t2 + dxidx[2][2] * t3;
            gij[4] = dxidx[0][1] * t1 + dxidx[1][1] * t2 + dxidx[2][1] * t3;
            gij[5] = dxidx[0][0] * t1 + dxidx[1][0] * t2 + dxidx[2][0] * t3;
        }
        // ---- quadrature point q = lane4: e3ivar / e3stab / e3Res ----
        const int q = lane4;
        double pres = 0.0, u[3] = {0.0, 0.0, 0.0}, aci[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            double N = c_el.shp[q][n];
            pres += N * yl[n][0];
            u[0] += N * yl[n][1];
            u[1] += N * yl[n][2];
            u[2] += N * yl[n][3];
            double4 av = live ? ac[nd[n]] : make_double4(0, 0, 0, 0);
            aci[0] += N * av.x;
            aci[1] += N * av.y;
            aci[2] += N * av.z;
        }
        const double rho = P.rho, mu = P.mu;
        double rL[3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
            rL[i] = (aci[i] + u[0] * g[0][i + 1] + u[1] * g[1][i + 1] + u[2] * g[2][i + 1]) * rho + g[i][0] - divq[i];
        const double rnu = mu / rho;
        const double dts = P.Dtgl * P.dtsfct;
        double uGu = u[0] * (gij[0] * u[0] + gij[3] * u[1] + gij[5] * u[2]) +
                     u[1] * (gij[3] * u[0] + gij[1] * u[1] + gij[4] * u[2]) +
                     u[2] * (gij[5] * u[0] + gij[4] * u[1] + gij[2] * u[2]);
        double gg = gij[0] * gij[0] + gij[1] * gij[1] + gij[2] * gij[2] +
                    2.0 * (gij[3] * gij[3] + gij[4] * gij[4] + gij[5] * gij[5]);
        double tauM = (2.0 * dts) * (2.0 * dts) + uGu + 36.0 * (rnu * rnu) * gg;
        double fact = sqrt(tauM);
        double tauC = rho * 0.125 * fact / (gij[0] + gij[1] + gij[2]) * (P.taucfct / P.dtsfct);
        tauM = 1.0 / fact;
        double tauBar = rL[0] * (gij[0] * rL[0] + gij[3] * rL[1] + gij[5] * rL[2]) +
                        rL[1] * (gij[3] * rL[0] + gij[1] * rL[1] + gij[4] * rL[2]) +
                        rL[2] * (gij[5] * rL[0] + gij[4] * rL[1] + gij[2] * rL[2]);
        if (tauBar != 0.0) tauBar = tauM / sqrt(tauBar);
        double uBar[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) uBar[i] = u[i] - tauM * rL[i] / rho;
        // e3Res, advective form (e3res.f90:104-284)
        double rNa[3], rGNa[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
            rNa[i] = (aci[i] + uBar[0] * g[0][i + 1] + uBar[1] * g[1][i + 1] + uBar[2] * g[2][i + 1]) * rho;
        {
            double divu = g[0][1] + g[1][2] + g[2][3];
            double tmp = -pres + tauC * divu;
            double lg[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) lg[i] = tauBar * (rL[0] * g[0][i + 1] + rL[1] * g[1][i + 1] + rL[2] * g[2][i + 1]);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    rGNa[i][j] = mu * (g[j][i + 1] + g[i][j + 1]) + (i == j ? tmp : 0.0) + tauM * rL[i] * u[j] +
                                 lg[i] * rL[j];
        }
        double* s = sqe + kQ * lane4;
        // per-point dot products with every node gradient (reused by all rows)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            s[c] = u[0] * shg[c][0] + u[1] * shg[c][1] + u[2] * shg[c][2];              // alpha_qc
            s[4 + c] = rL[0] * shg[c][0] + rL[1] * shg[c][1] + rL[2] * shg[c][2];       // beta_qc
            s[8 + c] = uBar[0] * shg[c][0] + uBar[1] * shg[c][1] + uBar[2] * shg[c][2]; // gamma_qc
        }
        s[12] = tauM;
        s[13] = tauBar;
        s[14] = tauC;
        s[15] = rNa[0];
        s[16] = rNa[1];
        s[17] = rNa[2];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) s[18 + 3 * i + j] = rGNa[i][j];
        s[27] = 0.0;
        __syncwarp();
        // ---- row a = lane4 ----
        const int a = lane4;
        const double* Sq[4] = {sqe, sqe + kQ, sqe + 2 * kQ, sqe + 3 * kQ};
        double Na[4];
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) Na[qq] = c_el.shp[qq][a];
        double* rec = erec + (size_t)RS * (size_t)(live ? e : 0);
        if (live) {
            // residual row a (e3res.f90:263-284, unpermuted: momentum 1-3, continuity)
            double sG[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, sN[3] = {0, 0, 0};
            double div_ub = 0.0;
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                const double* Sx = Sq[qq];
                div_ub += Sx[8 + a];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    sN[i] += Na[qq] * Sx[15 + i];
#pragma unroll
                    for (int j = 0; j < 3; ++j) sG[i][j] += Sx[18 + 3 * i + j];
                }
            }
            double v[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) v[i] = sN[i] + shg[a][0] * sG[i][0] + shg[a][1] * sG[i][1] + shg[a][2] * sG[i][2];
            reinterpret_cast<double4*>(rec + RO)[a] = make_double4(-WdetJ * v[0], -WdetJ * v[1], -WdetJ * v[2],
                                                                   WdetJ * div_ub);
        }
        if (kLhs == 1 && live) {
            const double lhsFct = P.alfi * P.gami * P.Delt;
            const double tlW = lhsFct * WdetJ;
            const double tsFct = P.almi * WdetJ * rho;
            double TC = 0.0, TM = 0.0, aqa[4], bqa[4], tMq[4], tBq[4];
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                const double* Sx = Sq[qq];
                aqa[qq] = Sx[a];
                bqa[qq] = Sx[4 + a];
                tMq[qq] = Sx[12];
                tBq[qq] = Sx[13];
                TC += Sx[14];
                TM += Sx[12];
            }
            double Kd[4];
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                double conv = 0.0, sym = 0.0;
#pragma unroll
                for (int qq = 0; qq < 4; ++qq) {
                    const double* Sx = Sq[qq];
                    conv += Na[qq] * Sx[8 + b];
                    sym += tMq[qq] * rho * aqa[qq] * Sx[b] + tBq[qq] * bqa[qq] * Sx[4 + b];
                }
                double grad = shg[a][0] * shg[b][0] + shg[a][1] * shg[b][1] + shg[a][2] * shg[b][2];
                Kd[b] = tsFct * c_el.M[a][b] + tlW * (rho * conv + 4.0 * mu * grad + sym);
            }
            double4* r4 = reinterpret_cast<double4*>(rec);
            r4[5 + a] = make_double4(Kd[0], Kd[1], Kd[2], Kd[3]);
            r4[1 + a] = make_double4(shg[a][0], shg[a][1], shg[a][2], 0.0);
            if (a == 3) r4[0] = make_double4(tlW * TC, tlW * 4.0 * mu, tlW, tlW / rho * TM);
        }
        if (kLhs == 2 && live) {
            // FP32 element quadrature of the tangent
            const float rhof = (float)rho, muf = (float)mu;
            const float lhsFct = (float)(P.alfi * P.gami * P.Delt);
            const float tlW = lhsFct * (float)WdetJ;
            const float tsFct = (float)P.almi * (float)WdetJ * rhof;
            float TC = 0.f, TM = 0.f, aqa[4], bqa[4], tMq[4], tBq[4], Naf[4];
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                const double* Sx = Sq[qq];
                aqa[qq] = (float)Sx[a];
                bqa[qq] = (float)Sx[4 + a];
                tMq[qq] = (float)Sx[12];
                tBq[qq] = (float)Sx[13];
                TC += (float)Sx[14];
                TM += (float)Sx[12];
                Naf[qq] = (float)Na[qq];
            }
            float sga[3] = {(float)shg[a][0], (float)shg[a][1], (float)shg[a][2]};
            float Kd[4];
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                float conv = 0.f, sym = 0.f;
#pragma unroll
                for (int qq = 0; qq < 4; ++qq) {
                    const double* Sx = Sq[qq];
                    conv += Naf[qq] * (float)Sx[8 + b];
                    sym += tMq[qq] * rhof * aqa[qq] * (float)Sx[b] + tBq[qq] * bqa[qq] * (float)Sx[4 + b];
                }
                const float grad = sga[0] * (float)shg[b][0] + sga[1] * (float)shg[b][1] + sga[2] * (float)shg[b][2];
                Kd[b] = tsFct * (float)c_el.M[a][b] + tlW * (rhof * conv + 4.0f * muf * grad + sym);
            }
            float4* r4 = reinterpret_cast<float4*>(rec + 16);
            r4[4 + a] = make_float4(Kd[0], Kd[1], Kd[2], Kd[3]);
            if (a < 3)
                r4[1 + a] = make_float4((float)shg[0][a], (float)shg[1][a], (float)shg[2][a], (float)shg[3][a]);
            else
                r4[0] = make_float4(tlW * TC, tlW * 4.0f * muf, tlW, tlW / rhof * TM);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Owner passes: tangent block (a, b) of one element from its record,
// exactly the expressions of the element-local tangent above.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void pair_block(const T sa[3], const T sb[3], T Kd, T tc, T tm, T sn, T cc, T o[13]) {
    const T grad = sa[0] * sb[0] + sa[1] * sb[1] + sa[2] * sb[2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) o[3 * i + j] = (i == j ? Kd : T(0)) + tc * sb[i] * sa[j] + tm * sb[j] * sa[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) o[9 + i] = sn * sb[i];
    o[12] = cc * grad;
}

// Contribution of element pair (a, b) to its slot, in the record's precision.
template <int kLhs>
__device__ __forceinline__ void record_block(const double* __restrict__ rec, int a, int b, double o[13]) {
    if (kLhs == 1) {
        const double4* r4 = reinterpret_cast<const double4*>(rec);
        const double4 sc = r4[0], ga = r4[1 + a], gb = r4[1 + b];
        const double sa[3] = {ga.x, ga.y, ga.z};
        const double sb[3] = {gb.x, gb.y, gb.z};
        const double Kd = rec[20 + 4 * a + b];
        pair_block<double>(sa, sb, Kd, sc.x, sc.y, sc.z * c_el.SN[a], sc.w, o);
    } else {
        const float* rf = reinterpret_cast<const float*>(rec + 16);
        const float4* r4 = reinterpret_cast<const float4*>(rf);
        const float4 sc = r4[0], s0 = r4[1], s1 = r4[2], s2 = r4[3];
        const float sa[3] = {sel4(s0, a), sel4(s1, a), sel4(s2, a)};
        const float sb[3] = {sel4(s0, b), sel4(s1, b), sel4(s2, b)};
        const float Kd = rf[16 + 4 * a + b];
        float of[13];
        pair_block<float>(sa, sb, Kd, sc.x, sc.y, sc.z * (float)c_el.SN[a], sc.w, of);
#pragma unroll
        for (int k = 0; k < 13; ++k) o[k] = (double)of[k];
    }
}

template <int kLhs>
__device__ __forceinline__ void store_block(long long s, const double acc[13], double* __restrict__ lhsK,
                                            double* __restrict__ lhsP, float* __restrict__ lhs32) {
    if (kLhs == 1) {
        double* k = lhsK + 9 * (size_t)s;
#pragma unroll
        for (int c = 0; c < 9; ++c) k[c] = acc[c];
        double* p = lhsP + 4 * (size_t)s;
#pragma unroll
        for (int c = 0; c < 4; ++c) p[c] = acc[9 + c];
    } else {
        float4* r = reinterpret_cast<float4*>(lhs32 + 16 * (size_t)s);
        r[0] = make_float4((float)acc[0], (float)acc[1], (float)acc[2], (float)acc[3]);
        r[1] = make_float4((float)acc[4], (float)acc[5], (float)acc[6], (float)acc[7]);
        r[2] = make_float4((float)acc[8], (float)acc[9], (float)acc[10], (float)acc[11]);
        r[3] = make_float4((float)acc[12], 0.f, 0.f, 0.f);
    }
}

// ---------------------------------------------------------------------------
// bc3LHS (bc3lhs.f90:39-198) on one element's 3x3 momentum block K
// (row-major) for a node with one or two prescribed velocity components
// (m = ibits(iBC,3,3) in 1..6; coefficients BC(:,4..6) = b4, b5, b6).  The
// reference projects, per element and node inod in order, the columns of the
// blocks (i, inod), then the rows of the blocks (inod, i), then sets the
// constrained diagonal entries of block (inod, inod) to 1; G and C are not
// touched.  A block (a, b) therefore gets the row operation of node a and the
// column operation of node b, the one of the smaller local index first.  The
// two-component case m = 6 keeps the reference's own row update (row 3 from
// row 1 and entry 6, rows 1-2 zeroed).
// ---------------------------------------------------------------------------
struct NodeBC {
    int m;   // ibits(iBC,3,3)
    double b4, b5, b6;
};

__device__ __forceinline__ bool bc_partial(int m) { return m != 0 && m != 7; }

__device__ __forceinline__ NodeBC node_bc(const int* __restrict__ iBC, const double* __restrict__ BC, int ndofBC,
                                          int n) {
    NodeBC r;
    r.m = (iBC[n] >> 3) & 7;
    r.b4 = r.b5 = r.b6 = 0.0;
    if (bc_partial(r.m)) {
        const double* b = BC + (size_t)ndofBC * n;
        r.b4 = b[3];
        r.b5 = b[4];
        r.b6 = b[5];
    }
    return r;
}

__device__ __forceinline__ void bc_colop(const NodeBC& n, double K[9]) {
    const int m = n.m;
    if (m == 1 || m == 2 || m == 4) {
        const int c0 = m == 1 ? 0 : (m == 2 ? 1 : 2), f1 = m == 1 ? 1 : 0, f2 = m == 4 ? 1 : 2;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            K[3 * r + f1] = K[3 * r + f1] - n.b4 * K[3 * r + c0];
            K[3 * r + f2] = K[3 * r + f2] - n.b5 * K[3 * r + c0];
            K[3 * r + c0] = 0.0;
        }
    } else if (m == 3 || m == 5 || m == 6) {
        const int f = m == 3 ? 2 : (m == 5 ? 1 : 0), c0 = m == 6 ? 1 : 0, c1 = m == 3 ? 1 : 2;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            K[3 * r + f] = K[3 * r + f] - n.b4 * K[3 * r + c0] - n.b6 * K[3 * r + c1];
            K[3 * r + c0] = 0.0;
            K[3 * r + c1] = 0.0;
        }
    }
}

__device__ __forceinline__ void bc_rowop(const NodeBC& n, double K[9]) {
    const int m = n.m;
    if (m == 1 || m == 2 || m == 4) {
        const int c0 = m == 1 ? 0 : (m == 2 ? 1 : 2), f1 = m == 1 ? 1 : 0, f2 = m == 4 ? 1 : 2;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            K[3 * f1 + q] = K[3 * f1 + q] - n.b4 * K[3 * c0 + q];
            K[3 * f2 + q] = K[3 * f2 + q] - n.b5 * K[3 * c0 + q];
            K[3 * c0 + q] = 0.0;
        }
    } else if (m == 3 || m == 5) {
        const int f = m == 3 ? 2 : 1, c1 = m == 3 ? 1 : 2;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            K[3 * f + q] = K[3 * f + q] - n.b4 * K[q] - n.b6 * K[3 * c1 + q];
            K[q] = 0.0;
            K[3 * c1 + q] = 0.0;
        }
    } else if (m == 6) {
        K[6] = K[6] - n.b4 * K[0];
        K[7] = K[7] - n.b4 * K[1];
        K[8] = K[8] - n.b4 * K[2] - n.b6 * K[5];
#pragma unroll
        for (int q = 0; q < 6; ++q) K[q] = 0.0;
    }
}

// 1 on the constrained diagonal entries (block (inod, inod) only)
__device__ __forceinline__ void bc_diag(const NodeBC& n, double K[9], double v) {
    const int m = n.m;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        if ((m >> c) & 1) K[4 * c] = v;
}

// Node pass: residual row and diagonal tangent block of every node.  The
// elements containing node i are the contributions of its diagonal slot
// (ascending element order); then the boundary faces at i (ascending face
// order, AsBMFG after AsIGMR as in elmgmr.f90).  kOwnerLanes lanes per node
// split the element contributions round-robin (lane l: entries l,
// l + kOwnerLanes, ... in list order) and combine them by a fixed butterfly
// (owner_sum), so the sums are bitwise repeatable; the faces follow.  For a
// partially constrained node every element block gets bc3LHS (columns, rows,
// 1 on the constrained diagonal), and the boundary elements at the node --
// whose rigid-wall tangent is zero -- add 1 each to those entries, as the
// reference's bc3LHS + fillsparseI pass over them does (elmgmr.f90:428-438).
template <int kLhs, bool kProj>
__global__ void __launch_bounds__(256) k_node_pass(const int* __restrict__ diag, const int* __restrict__ soff,
                                                   const int* __restrict__ slist, const double* __restrict__ erec,
                                                   const int* __restrict__ fnoff, const int* __restrict__ flist,
                                                   const double* __restrict__ frec, int nshg,
                                                   const int* __restrict__ iBC, const double* __restrict__ BC,
                                                   int ndofBC, int npartial, const int* __restrict__ bcount,
                                                   double* __restrict__ res, double* __restrict__ lhsK,
                                                   double* __restrict__ lhsP, float* __restrict__ lhs32) {
    constexpr int RS = RecLayout<kLhs>::RS, RO = RecLayout<kLhs>::RO;
    constexpr int NPW = 32 / kOwnerLanes;  // nodes per warp and pass
    const int lane = threadIdx.x & 31, sub = lane % kOwnerLanes;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    // warp-uniform loop: the shuffles of owner_sum always see all 32 lanes
    for (long long i0 = warp * NPW; i0 < nshg; i0 += nwarp * NPW) {
        const long long ig = i0 + lane / kOwnerLanes;
        const bool valid = ig < nshg;
        const int i = valid ? (int)ig : nshg - 1;
        const int d = diag[i];
        double r0 = 0.0, r1 = 0.0, r2 = 0.0, r3 = 0.0;
        double acc[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        NodeBC nb{0, 0.0, 0.0, 0.0};
        if (kLhs && kProj) nb = node_bc(iBC, BC, ndofBC, i);
        const bool proj = kLhs && kProj && bc_partial(nb.m);
        const int p1 = soff[d + 1];
        for (int p = soff[d] + sub; p < p1; p += kOwnerLanes) {
            const int t = slist[p];
            const int e = t >> 4, a = (t >> 2) & 3;
            const double* rec = erec + (size_t)RS * (size_t)e;
            const double4 rl = reinterpret_cast<const double4*>(rec + RO)[a];
            r0 += rl.x;
            r1 += rl.y;
            r2 += rl.z;
            r3 += rl.w;
            if (kLhs) {
                double o[13];
                record_block<kLhs == 2 ? 2 : 1>(rec, a, a, o);
                if (proj) {
                    bc_colop(nb, o);
                    bc_rowop(nb, o);
                    bc_diag(nb, o, 1.0);
                }
#pragma unroll
                for (int c = 0; c < 13; ++c) acc[c] += o[c];
            }
        }
        r0 = owner_sum(r0);
        r1 = owner_sum(r1);
        r2 = owner_sum(r2);
        r3 = owner_sum(r3);
        if (kLhs) {
#pragma unroll
            for (int c = 0; c < 13; ++c) acc[c] = owner_sum(acc[c]);
        }
        if (!valid || sub != 0) continue;
        if (proj && bcount)
            for (int k = 0; k < bcount[i]; ++k)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    if ((nb.m >> c) & 1) acc[4 * c] += 1.0;
        if (fnoff) {
            const int f1 = fnoff[i + 1];
            for (int p = fnoff[i]; p < f1; ++p) {
                const double4 rl = reinterpret_cast<const double4*>(frec)[flist[p]];
                r0 += rl.x;
                r1 += rl.y;
                r2 += rl.z;
                r3 += rl.w;
            }
        }
        reinterpret_cast<double4*>(res)[i] = make_double4(r0, r1, r2, r3);
        if (kLhs) store_block<kLhs == 2 ? 2 : 1>(d, acc, lhsK, lhsP, lhs32);
    }
}

// Slot pass: every off-diagonal CSR block (i, j) from the elements that
// contain the edge (ascending element order).  One thread per slot; the
// diagonal slots (first contribution with a == b) belong to the node pass.
template <int kLhs, bool kProj>
__global__ void __launch_bounds__(256) k_slot_pass(const int* __restrict__ soff, const int* __restrict__ slist,
                                                   const double* __restrict__ erec, long long nnz,
                                                   const int4* __restrict__ ien, const int* __restrict__ iBC,
                                                   const double* __restrict__ BC, int ndofBC, int npartial,
                                                   double* __restrict__ lhsK, double* __restrict__ lhsP,
                                                   float* __restrict__ lhs32) {
    constexpr int RS = RecLayout<kLhs>::RS;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < nnz;
         s += (long long)gridDim.x * blockDim.x) {
        const int p0 = soff[s], p1 = soff[s + 1];
        const int t0 = slist[p0];
        if (((t0 >> 2) & 3) == (t0 & 3)) continue;
        // bc3LHS: row operation of the row node, column operation of the column node
        NodeBC ni{0, 0.0, 0.0, 0.0}, nj{0, 0.0, 0.0, 0.0};
        if (kProj) {
            const int4 nn = ien[t0 >> 4];
            const int na[4] = {nn.x, nn.y, nn.z, nn.w};
            ni = node_bc(iBC, BC, ndofBC, na[(t0 >> 2) & 3]);
            nj = node_bc(iBC, BC, ndofBC, na[t0 & 3]);
        }
        const bool proj = kProj && (bc_partial(ni.m) || bc_partial(nj.m));
        double acc[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int p = p0; p < p1; ++p) {
            const int t = p == p0 ? t0 : slist[p];
            const int e = t >> 4, a = (t >> 2) & 3, b = t & 3;
            double o[13];
            record_block<kLhs>(erec + (size_t)RS * (size_t)e, a, b, o);
            if (proj) {
                if (a < b) {
                    bc_rowop(ni, o);
                    bc_colop(nj, o);
                } else {
                    bc_colop(nj, o);
                    bc_rowop(ni, o);
                }
            }
#pragma unroll
            for (int c = 0; c < 13; ++c) acc[c] += o[c];
        }
        store_block<kLhs>(s, acc, lhsK, lhsP, lhs32);
    }
}

// ---------------------------------------------------------------------------
// AsBMFG / e3b / e3bvar, rigid wall, one thread per boundary face
// (e3b.f90:112-470, e3bvar.f90:140-460).  Residual only: for rigid walls the
// boundary tangent is zero (e3b.f90:338-343).  Writes the face's record
// rl(n, 0:4) of its three face nodes; the node pass sums them.
// ---------------------------------------------------------------------------
__global__ void k_asbmfg(const int4* __restrict__ ienb, const int* __restrict__ iBCB, const double* __restrict__ BCB,
                         const double4* __restrict__ x, const double4* __restrict__ y, int nface, ElmParams P,
                         double* __restrict__ frec) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nface; f += gridDim.x * blockDim.x) {
        int4 nn = ienb[f];
        int nd[4] = {nn.x, nn.y, nn.z, nn.w};
        double xl[4][3], yl[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            double4 xv = x[nd[a]];
            double4 yv = y[nd[a]];
            xl[a][0] = xv.x;
            xl[a][1] = xv.y;
            xl[a][2] = xv.z;
            yl[a][0] = yv.w;
            yl[a][1] = yv.x;
            yl[a][2] = yv.y;
            yl[a][3] = yv.z;
        }
        const int bits = iBCB[f];
        const double* bcb = BCB + 18 * (size_t)f;
        double dxidx[3][3], shg[4][3], Wtmp;
        elem_metric(xl, dxidx, shg, &Wtmp);
        double g[3][4];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int d = 1; d < 4; ++d)
                g[k][d] = shg[0][k] * yl[0][d] + shg[1][k] * yl[1][d] + shg[2][k] * yl[2][d] + shg[3][k] * yl[3][d];
        double v1[3], v2[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            v1[i] = xl[1][i] - xl[0][i];
            v2[i] = xl[2][i] - xl[0][i];
        }
        double t1 = v1[1] * v2[2] - v2[1] * v1[2];
        double t2 = v2[0] * v1[2] - v1[0] * v2[2];
        double t3 = v1[0] * v2[1] - v2[0] * v1[1];
        double temp = 1.0 / sqrt(t1 * t1 + t2 * t2 + t3 * t3);
        double bn[3] = {t1 * temp, t2 * temp, t3 * temp};
        double WdetJb = c_el.Qwtb / (4.0 * temp);
        const double mu = P.mu, rho = P.rho;
        double tau[3];
        tau[0] = bn[0] * 2.0 * mu * g[0][1] + bn[1] * (mu * (g[1][1] + g[0][2])) + bn[2] * (mu * (g[2][1] + g[0][3]));
        tau[1] = bn[0] * (mu * (g[1][1] + g[0][2])) + bn[1] * 2.0 * mu * g[1][2] + bn[2] * (mu * (g[2][2] + g[1][3]));
        tau[2] = bn[0] * (mu * (g[2][1] + g[0][3])) + bn[1] * (mu * (g[2][2] + g[1][3])) + bn[2] * 2.0 * mu * g[2][3];
        double tn = bn[0] * tau[0] + bn[1] * tau[1] + bn[2] * tau[2];
        double rl[3][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
        for (int q = 0; q < 3; ++q) {
            const double* Nb = c_el.shpb[q];
            double pres = 0.0, u[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int n = 0; n < 3; ++n) {
                pres += Nb[n] * yl[n][0];
                u[0] += Nb[n] * yl[n][1];
                u[1] += Nb[n] * yl[n][2];
                u[2] += Nb[n] * yl[n][3];
            }
            double unm = bn[0] * u[0] + bn[1] * u[1] + bn[2] * u[2];
            pres = pres - tn;
            double tt[3] = {tau[0] - bn[0] * tn, tau[1] - bn[1] * tn, tau[2] - bn[2] * tn};
            double unm_copy = 0.0;
            if ((bits >> 1) & 1)
                if (unm < 0.0) unm_copy = unm;
            if (bits & 1) {
                unm = 0.0;
                for (int n = 0; n < 3; ++n) unm += Nb[n] * bcb[6 * n + 0];
            }
            if ((bits >> 1) & 1) {
                pres = 0.0;
                for (int n = 0; n < 3; ++n) pres += Nb[n] * bcb[6 * n + 1];
            }
            if ((bits >> 2) & 1) {
                tt[0] = tt[1] = tt[2] = 0.0;
                for (int n = 0; n < 3; ++n) {
                    tt[0] += Nb[n] * bcb[6 * n + 2];
                    tt[1] += Nb[n] * bcb[6 * n + 3];
                    tt[2] += Nb[n] * bcb[6 * n + 4];
                }
            }
            if ((bits >> 4) & 1) {
                pres = 0.0;
                tt[0] = tt[1] = tt[2] = 0.0;
            }
            double rNa[4];
            const double rou_copy = rho * unm_copy;
#pragma unroll
            for (int i = 0; i < 3; ++i) rNa[i] = (-tt[i] + bn[i] * pres - P.stabflux * rou_copy * u[i]) * WdetJb;
            rNa[3] = unm * WdetJb;
#pragma unroll
            for (int n = 0; n < 3; ++n)
#pragma unroll
                for (int d = 0; d < 4; ++d) rl[n][d] -= Nb[n] * rNa[d];
        }
        double4* r4 = reinterpret_cast<double4*>(frec + 12 * (size_t)f);
#pragma unroll
        for (int n = 0; n < 3; ++n) r4[n] = make_double4(rl[n][0], rl[n][1], rl[n][2], rl[n][3]);
    }
}

// ---------------------------------------------------------------------------
// ElmpvsQ, GRCR branch (elmgmr.f90:1271-1330) with GetFlowQ
// (boundarydata.f90:1157-1196).  One block per coupled surface reduces
// Q_k = sum NABI.u over its nodes (fixed order: deterministic).  The node
// lists of different surfaces are disjoint (built from ndsurf), so the
// residual update touches each node once.
// ---------------------------------------------------------------------------
__global__ void k_flowq(const int* __restrict__ onodes, const int* __restrict__ off, const double4* __restrict__ onabi,
                        const double4* __restrict__ y, double* __restrict__ q) {
    __shared__ double sm[32];
    const int k = blockIdx.x;
    double s = 0.0;
    for (int t = off[k] + threadIdx.x; t < off[k + 1]; t += blockDim.x) {
        double4 nb = onabi[t];
        double4 yv = y[onodes[t]];
        s += nb.x * yv.x + nb.y * yv.y + nb.z * yv.z;
    }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) q[k] = s;
}

__global__ void k_pvsq_add(const int* __restrict__ onodes, const int* __restrict__ off, const double4* __restrict__ onabi,
                           const double* __restrict__ q, const double* __restrict__ coefs, int ncoupled,
                           double* __restrict__ res) {
    const int k = blockIdx.y;
    const double pk = -1.0 * (q[k] * coefs[k]) - coefs[ncoupled + k];
    for (int t = off[k] + blockIdx.x * blockDim.x + threadIdx.x; t < off[k + 1]; t += gridDim.x * blockDim.x) {
        double4 nb = onabi[t];
        double* r = res + 4 * (size_t)onodes[t];
        r[0] += pk * nb.x;
        r[1] += pk * nb.y;
        r[2] += pk * nb.z;
    }
}

// bc3Res (bc3res.f90:30-124): pressure, the velocity components a node's
// iBC prescribes (one or two through the BC coefficients, or all three), and
// the plane condition (bit 11)
__global__ void k_bc3res(const int* __restrict__ iBC, const double* __restrict__ BC, int ndofBC, int nshg,
                         double* __restrict__ res) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nshg; i += gridDim.x * blockDim.x) {
        const int bits = iBC[i];
        double* r = res + 4 * (size_t)i;
        if ((bits >> 2) & 1) r[3] = 0.0;
        const int m = (bits >> 3) & 7;
        if (m != 0) {
            const double* bc = BC + (size_t)ndofBC * i;
            const double b4 = bc[3], b5 = bc[4], b6 = bc[5];
            switch (m) {
                case 1: r[1] = r[1] - b4 * r[0]; r[2] = r[2] - b5 * r[0]; r[0] = 0.0; break;
                case 2: r[0] = r[0] - b4 * r[1]; r[2] = r[2] - b5 * r[1]; r[1] = 0.0; break;
                case 3: r[2] = r[2] - b4 * r[0] - b6 * r[1]; r[0] = 0.0; r[1] = 0.0; break;
                case 4: r[0] = r[0] - b4 * r[2]; r[1] = r[1] - b5 * r[2]; r[2] = 0.0; break;
                case 5: r[1] = r[1] - b4 * r[0] - b6 * r[2]; r[0] = 0.0; r[2] = 0.0; break;
                case 6: r[0] = r[0] - b4 * r[1] - b6 * r[2]; r[1] = 0.0; r[2] = 0.0; break;
                default: r[0] = 0.0; r[1] = 0.0; r[2] = 0.0; break;
            }
        }
        if ((bits >> 11) & 1) {
            r[0] = 0.0;
            r[1] = 0.0;
            r[2] = 0.0;
        }
    }
}

// Grid caps (blocks of 256 per SM) of the owner passes: a grid-stride loop
// over rows / slots in order, so the cap sets how many rows are in flight.
#ifndef CRIMSON_NODE_PASS_BLOCKS_PER_SM
#define CRIMSON_NODE_PASS_BLOCKS_PER_SM 8
#endif
#ifndef CRIMSON_SLOT_PASS_BLOCKS_PER_SM
#define CRIMSON_SLOT_PASS_BLOCKS_PER_SM 32
#endif
constexpr int kNodePassBlocksPerSM = CRIMSON_NODE_PASS_BLOCKS_PER_SM;
constexpr int kSlotPassBlocksPerSM = CRIMSON_SLOT_PASS_BLOCKS_PER_SM;

int elmgmr_device(crimson_ctx* c, const double* d_y, const double* d_ac, const double* coef1, const double* coef2,
                  double* d_res, double* d_lhsK, double* d_lhsP, int lhs, float* d_lhs32) {
    cudaStream_t s = c->stream;
    // every pass below reads the pattern's contribution lists
    if (c->nnz == 0) CR_CHECK(build_pattern(c));
    if (!c->diag.p || !c->soff.p || !c->slist.p) return CRIMSON_ERR_STATE;
    CR_CHECK(upload_elm_consts(s));
    const ElmParams P = elm_params(c->p);
    const double4* y4 = reinterpret_cast<const double4*>(d_y);
    const double4* a4 = reinterpret_cast<const double4*>(d_ac);
    // diffusive flux reconstruction
    if (c->p.idiff == 1) {
        CR_CHECK(c->qres.alloc((size_t)c->nshg * 9));
        CR_CHECK(c->rmass.alloc((size_t)c->nshg));
        CR_CHECK(c->qrec.alloc((size_t)c->nelem * 8));
        const bool first = !c->rmass_ready;
        launch(k_asiq_rec, grid_for(c->nelem, 128, 16), 128, 0, s, c->ien.p, c->x.p, y4, c->nelem, P, c->qrec.p);
        launch(k_q_node, grid_for((long long)kOwnerLanes * c->nshg, 256), 256, 0, s, c->diag.p, c->soff.p, c->slist.p, c->qrec.p, c->nshg,
               first ? 1 : 0, c->rmass.p, c->qres.p);
        c->rmass_ready = true;
    }
    // element records (sized for the FP64 tangent layout, the largest)
    CR_CHECK(c->erec.alloc((size_t)c->nelem * RecLayout<1>::RS));
    const int blk = 128;
    const int grid = grid_for((long long)c->nelem * 4, blk, 16);
    if (lhs == 2)
        launch(k_asigmr<2>, grid, blk, 0, s, c->ien.p, c->x.p, y4, a4, c->qres.p, c->nelem, P, c->erec.p);
    else if (lhs)
        launch(k_asigmr<1>, grid, blk, 0, s, c->ien.p, c->x.p, y4, a4, c->qres.p, c->nelem, P, c->erec.p);
    else
        launch(k_asigmr<0>, grid, blk, 0, s, c->ien.p, c->x.p, y4, a4, c->qres.p, c->nelem, P, c->erec.p);
    CR_CUDA(cudaGetLastError());
    if (c->nface > 0) {
        CR_CHECK(c->frec.alloc((size_t)c->nface * 12));
        launch(k_asbmfg, grid_for(c->nface, 128), 128, 0, s, c->ienb.p, c->iBCB.p, c->BCB.p, c->x.p, y4, c->nface, P,
               c->frec.p);
    }
    const int* fno = c->nface > 0 ? c->fnoff.p : nullptr;
    const int ng = grid_for((long long)kOwnerLanes * c->nshg, 256, kNodePassBlocksPerSM);
    const int gs = grid_for(c->nnz, 256, kSlotPassBlocksPerSM);
    // the bc3LHS projection is compiled into separate pass variants, used only
    // when some node has one or two prescribed velocity components
    const int nb = c->p.ndofBC, np = c->npartial;
    const int* bcnt = c->nface > 0 ? c->bcount.p : nullptr;
    if (lhs == 2) {
        if (np)
            launch(k_node_pass<2, true>, ng, 256, 0, s, c->diag.p, c->soff.p, c->slist.p, c->erec.p, fno, c->flist.p,
                   c->frec.p, c->nshg, c->iBC.p, c->BC.p, nb, np, bcnt, d_res, nullptr, nullptr, d_lhs32);
        else
            launch(k_node_pass<2, false>, ng, 256, 0, s, c->diag.p, c->soff.p, c->slist.p, c->erec.p, fno, c->flist.p,
                   c->frec.p, c->nshg, c->iBC.p, c->BC.p, nb, np, bcnt, d_res, nullptr, nullptr, d_lhs32);
        if (np)
            launch(k_slot_pass<2, true>, gs, 256, 0, s, c->soff.p, c->slist.p, c->erec.p, c->nnz, c->ien.p, c->iBC.p,
                   c->BC.p, nb, np, nullptr, nullptr, d_lhs32);
        else
            launch(k_slot_pass<2, false>, gs, 256, 0, s, c->soff.p, c->slist.p, c->erec.p, c->nnz, c->ien.p, c->iBC.p,
                   c->BC.p, nb, np, nullptr, nullptr, d_lhs32);
    } else if (lhs) {
        if (np)
            launch(k_node_pass<1, true>, ng, 256, 0, s, c->diag.p, c->soff.p, c->slist.p, c->erec.p, fno, c->flist.p,
                   c->frec.p, c->nshg, c->iBC.p, c->BC.p, nb, np, bcnt, d_res, d_lhsK, d_lhsP, nullptr);
        else
            launch(k_node_pass<1, false>, ng, 256, 0, s, c->diag.p, c->soff.p, c->slist.p, c->erec.p, fno, c->flist.p,
                   c->frec.p, c->nshg, c->iBC.p, c->BC.p, nb, np, bcnt, d_res, d_lhsK, d_lhsP, nullptr);
        if (np)
            launch(k_slot_pass<1, true>, gs, 256, 0, s, c->soff.p, c->slist.p, c->erec.p, c->nnz, c->ien.p, c->iBC.p,
                   c->BC.p, nb, np, d_lhsK, d_lhsP, nullptr);
        else
            launch(k_slot_pass<1, false>, gs, 256, 0, s, c->soff.p, c->slist.p, c->erec.p, c->nnz, c->ien.p, c->iBC.p,
                   c->BC.p, nb, np, d_lhsK, d_lhsP, nullptr);
    } else {
        launch(k_node_pass<0, false>, ng, 256, 0, s, c->diag.p, c->soff.p, c->slist.p, c->erec.p, fno, c->flist.p,
               c->frec.p, c->nshg, c->iBC.p, c->BC.p, nb, np, bcnt, d_res, nullptr, nullptr, nullptr);
    }
    if (c->ncoupled > 0) {
        double* hc = c->coef_host.data();
        for (int k = 0; k < c->ncoupled; ++k) {
            hc[k] = coef1 ? coef1[k] : 0.0;
            hc[c->ncoupled + k] = coef2 ? coef2[k] : 0.0;
        }
        CR_CUDA(cudaMemcpyAsync(c->coefs.p, hc, sizeof(double) * 2 * (size_t)c->ncoupled, cudaMemcpyHostToDevice, s));
        launch(k_flowq, c->ncoupled, 256, 0, s, c->onodes.p, c->d_onode_off.p, c->onabi.p, y4, c->flowq.p);
        dim3 g2(8, c->ncoupled);
        launch(k_pvsq_add, g2, 256, 0, s, c->onodes.p, c->d_onode_off.p, c->onabi.p, c->flowq.p, c->coefs.p,
               c->ncoupled, d_res);
    }
    launch(k_bc3res, grid_for(c->nshg, 256), 256, 0, s, c->iBC.p, c->BC.p, nb, c->nshg, d_res);
    CR_CUDA(cudaGetLastError());
    return CRIMSON_OK;
}

}  // namespace crimson
