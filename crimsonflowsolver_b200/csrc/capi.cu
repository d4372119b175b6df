// extern "C" entry points of crimson_b200 (declared in include/crimson_b200.h).
#include <cmath>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "memls.cuh"
#include "netlist.h"

namespace crimson {

thread_local std::string g_last_error;
static std::atomic<unsigned long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void set_last_error(const std::string& s) { g_last_error = s; }

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    }
    return n;
}

int build_pattern(crimson_ctx* c);
int pattern_aux(crimson_lhs* L);
int elmgmr_sclr_device(crimson_ctx* c, int isclr, double diffus, const double* d_y, const double* d_s,
                       const double* d_sdot, const double* d_bcbs, double* d_res, double* d_lhsS, int lhs);
int memls_kernel_time(crimson_lhs* L, int which, int reps, double* ms);
int pattern_to_host(crimson_ctx* c, int* colm, int* rowp, long long cap);
int elmgmr_device(crimson_ctx* c, const double* d_y, const double* d_ac, const double* coef1, const double* coef2,
                  double* d_res, double* d_lhsK, double* d_lhsP, int lhs, float* d_lhs32 = nullptr);
int memls_solve_val(crimson_lhs* L, crimson_ls* ls, double* Ri, double* Val, const int* incL, const double* res,
                    crimson_ls_stats* st);
int memls_solve_lhs_device(crimson_lhs* L, crimson_ls* ls, const double* d_res, const double* d_lhsK,
                           const double* d_lhsP, const int* incL, const double* faceRes, double* d_sol,
                           crimson_ls_stats* st, bool transpose = false, const float* d_lhs32 = nullptr);
int spmv4_prepare(crimson_ctx* c, int precision, const void* d_val);
int spmv4_apply(crimson_ctx* c, const void* d_u, void* d_ku);
int elmgmr_vjp(crimson_ctx* c, const double* d_y, const double* d_ac, const double* coef1, const double* coef2,
               const double* d_lam, double* d_res, double* d_ybar, double* d_abar, double* mubar, double* c1bar,
               double* c2bar);

// ---- layout conversion kernels ----
__global__ void k_soa_to_node4(const double* __restrict__ a, int n, int ld, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int d = 0; d < 4; ++d) out[4 * (size_t)i + d] = a[(size_t)d * ld + i];
}
__global__ void k_node4_to_soa(const double* __restrict__ a, int n, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int d = 0; d < 4; ++d) out[(size_t)d * n + i] = a[4 * (size_t)i + d];
}

// ---- time stepping kernels (itrPC.f90, itrbc.f90) ----
__global__ void k_predict(const double* __restrict__ yold, const double* __restrict__ acold, double* __restrict__ y,
                          double* __restrict__ ac, long long n4, double fct) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n4; t += (long long)gridDim.x * blockDim.x) {
        y[t] = yold[t];
        ac[t] = acold[t] * fct;
    }
}
__global__ void k_yalpha(const double* __restrict__ yold, const double* __restrict__ acold,
                         const double* __restrict__ y, const double* __restrict__ ac, double* __restrict__ ya,
                         double* __restrict__ aa, int n, double alfi, double almi) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t b = 4 * (size_t)i;
        for (int d = 0; d < 3; ++d) {
            ya[b + d] = yold[b + d] + alfi * (y[b + d] - yold[b + d]);
            aa[b + d] = acold[b + d] + almi * (ac[b + d] - acold[b + d]);
        }
        ya[b + 3] = y[b + 3];
        aa[b + 3] = 0.0;
    }
}
__global__ void k_correct(double* __restrict__ y, double* __restrict__ ac, const double* __restrict__ sol, int n,
                          double fct1, double fct2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t b = 4 * (size_t)i;
        for (int d = 0; d < 3; ++d) y[b + d] = y[b + d] + fct1 * sol[b + d];
        y[b + 3] = y[b + 3] + fct2 * sol[b + 3];
        for (int d = 0; d < 3; ++d) ac[b + d] = ac[b + d] + sol[b + d];
    }
}
// BC node-major (ndofBC per node)
__global__ void k_itrbc(const int* __restrict__ iBC, const double* __restrict__ BC, int ndofBC, int n,
                        double* __restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        // itrBC (itrbc.f90:33-101): prescribed velocity components (all
        // three, or one or two through the BC coefficients) and pressure
        const int b = iBC[i];
        const double* bc = BC + (size_t)ndofBC * i;
        double* v = y + 4 * (size_t)i;
        switch ((b >> 3) & 7) {
            case 1: v[0] = bc[2] - bc[3] * v[1] - bc[4] * v[2]; break;
            case 2: v[1] = bc[2] - bc[3] * v[0] - bc[4] * v[2]; break;
            case 3: v[0] = bc[2] - bc[3] * v[2]; v[1] = bc[4] - bc[5] * v[2]; break;
            case 4: v[2] = bc[2] - bc[3] * v[0] - bc[4] * v[1]; break;
            case 5: v[0] = bc[2] - bc[3] * v[1]; v[2] = bc[4] - bc[5] * v[1]; break;
            case 6: v[1] = bc[2] - bc[3] * v[0]; v[2] = bc[4] - bc[5] * v[0]; break;
            case 7: v[0] = bc[2]; v[1] = bc[3]; v[2] = bc[4]; break;
            default: break;
        }
        if ((b >> 2) & 1) v[3] = bc[0];
    }
}
__global__ void k_inflow(const int* __restrict__ nodes, const double* __restrict__ prof, int m, double scale,
                         int ndofBC, double* __restrict__ BC) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        double* bc = BC + (size_t)ndofBC * nodes[t];
        bc[2] = prof[3 * (size_t)t + 0] * scale;
        bc[3] = prof[3 * (size_t)t + 1] * scale;
        bc[4] = prof[3 * (size_t)t + 2] * scale;
    }
}
__global__ void k_flowq_step(const int* __restrict__ onodes, int beg, int end, const double4* __restrict__ onabi,
                             const double4* __restrict__ y, double* __restrict__ q) {
    __shared__ double sm[32];
    double s = 0.0;
    for (int t = beg + threadIdx.x; t < end; t += blockDim.x) {
        double4 nb = onabi[t];
        double4 yv = y[onodes[t]];
        s += nb.x * yv.x + nb.y * yv.y + nb.z * yv.z;
    }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) *q = s;
}

static void rcr_coeffs(double Rp, double C, double Rd, double Pdn, double Pdn1, double Pn, double Qn,
                       double alfi_delt, double* slope, double* offset) {
    // RCR::computeImplicitCoefficients (flowsolver/src/RCR.cxx:49-81)
    double denominator = 1.0 + ((C * Rd) / alfi_delt);
    double num = Rd + Rp * (1.0 + ((C * Rd) / alfi_delt));
    *slope = num / denominator;
    double temp2 = Pn + Pdn1 - Pdn - Rp * Qn;
    temp2 = ((C * Rd) / alfi_delt) * temp2 + Pdn1;
    *offset = temp2 / denominator;
}

static int check_params(const crimson_params* p) {
    if (!p) return CRIMSON_ERR_ARG;
    if (p->itau != 0 || p->flmpl != 0.0 || p->flmpr != 0.0 || p->iconvflow != 2 || (p->idiff != 0 && p->idiff != 1)) {
        set_last_error("unsupported settings: need itau=0, flmpl=flmpr=0, iconvflow=2, idiff in {0,1}");
        return CRIMSON_ERR_UNSUPPORTED;
    }
    return CRIMSON_OK;
}

}  // namespace crimson

using namespace crimson;

extern "C" {

const char* crimson_version(void) { return "crimson_b200 0.1 sm_100a"; }
void* crimson_ctx_stream(crimson_ctx* c) { return c ? (void*)c->stream : nullptr; }
unsigned long long crimson_launch_count(void) { return g_launches.load(); }
int crimson_memls_kernel_time(crimson_lhs* L, int which, int reps, double* ms) {
    if (!L || !ms) return CRIMSON_ERR_ARG;
    return memls_kernel_time(L, which, reps, ms);
}
const char* crimson_last_error(void) { return g_last_error.c_str(); }
int crimson_memls_cg_layout(const crimson_lhs* L, int* resident64, int* resident32, long long* smem_bytes) {
    if (!L) return CRIMSON_ERR_ARG;
    if (L->cg_res_bytes < 0) return CRIMSON_ERR_STATE;
    if (resident64) *resident64 = L->cg_grid ? L->cg_res64 : 0;
    if (resident32) *resident32 = L->cg_grid32 ? L->cg_res32 : 0;
    if (smem_bytes) *smem_bytes = L->cg_res_bytes;
    return CRIMSON_OK;
}

int crimson_ctx_create(crimson_ctx** out, const crimson_params* p, int nshg, int numnp, int nelem, const int* ien,
                       const double* x) {
    if (!out || !ien || !x || nshg <= 0 || numnp < nshg || nelem <= 0) return CRIMSON_ERR_ARG;
    CR_CHECK(check_params(p));
    // The mesh is checked on the host before any device work: node indices in
    // range, finite coordinates, and every tet oriented as e3metric assumes,
    // det[x1 - x4, x2 - x4, x3 - x4] > 0 (a zero or negative volume would give
    // an infinite or sign-flipped WdetJ).
    std::vector<double4> hx(numnp);
    for (int i = 0; i < numnp; ++i) {
        hx[i] = make_double4(x[i], x[(size_t)numnp + i], x[2 * (size_t)numnp + i], 0.0);
        if (!std::isfinite(hx[i].x) || !std::isfinite(hx[i].y) || !std::isfinite(hx[i].z)) {
            set_last_error("non-finite coordinate at node " + std::to_string(i + 1));
            return CRIMSON_ERR_ARG;
        }
    }
    std::vector<int4> hien(nelem);
    for (int i = 0; i < nelem; ++i) {
        int v[4];
        for (int a = 0; a < 4; ++a) {
            v[a] = std::abs(ien[(size_t)a * nelem + i]) - 1;
            if (v[a] < 0 || v[a] >= nshg) {
                set_last_error("ien out of range at element " + std::to_string(i + 1));
                return CRIMSON_ERR_ARG;
            }
        }
        const double4 p4 = hx[v[3]];
        double d[3][3];
        for (int a = 0; a < 3; ++a) {
            d[a][0] = hx[v[a]].x - p4.x;
            d[a][1] = hx[v[a]].y - p4.y;
            d[a][2] = hx[v[a]].z - p4.z;
        }
        const double det = d[0][0] * (d[1][1] * d[2][2] - d[1][2] * d[2][1]) -
                           d[0][1] * (d[1][0] * d[2][2] - d[1][2] * d[2][0]) +
                           d[0][2] * (d[1][0] * d[2][1] - d[1][1] * d[2][0]);
        if (!(det > 0.0)) {
            set_last_error("element " + std::to_string(i + 1) +
                           ": zero or negative volume (nodes must satisfy det[x1-x4, x2-x4, x3-x4] > 0)");
            return CRIMSON_ERR_ARG;
        }
        hien[i] = make_int4(v[0], v[1], v[2], v[3]);
    }
    crimson_ctx* c = new crimson_ctx();
    c->p = *p;
    c->nshg = nshg;
    c->numnp = numnp;
    c->nelem = nelem;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        set_last_error(cudaGetErrorString(e));
        delete c;
        return CRIMSON_ERR_CUDA;
    }
    int rc = c->ien.upload(hien.data(), hien.size(), c->stream);
    if (rc == CRIMSON_OK) rc = c->x.upload(hx.data(), hx.size(), c->stream);
    std::vector<int> zi(nshg, 0);
    if (rc == CRIMSON_OK) rc = c->iBC.upload(zi.data(), zi.size(), c->stream);
    int nbc = p->ndofBC > 0 ? p->ndofBC : 7;
    c->p.ndofBC = nbc;
    std::vector<double> zb((size_t)nshg * nbc, 0.0);
    c->h_BC.assign(zb.begin(), zb.end());
    c->h_iBC.assign(nshg, 0);
    c->h_iBC_orig.assign(nshg, 0);
    c->h_x.assign(x, x + 3 * (size_t)numnp);
    if (rc == CRIMSON_OK) rc = c->BC.upload(zb.data(), zb.size(), c->stream);
    if (rc == CRIMSON_OK) {
        cudaError_t e2 = cudaStreamSynchronize(c->stream);
        if (e2 != cudaSuccess) {
            set_last_error(cudaGetErrorString(e2));
            rc = CRIMSON_ERR_CUDA;
        }
    }
    if (rc != CRIMSON_OK) {
        crimson_ctx_destroy(c);
        return rc;
    }
    *out = c;
    return CRIMSON_OK;
}

int crimson_ctx_destroy(crimson_ctx* c) {
    if (!c) return CRIMSON_ERR_ARG;
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaStream_t s = c->stream;
    delete c;
    if (s) cudaStreamDestroy(s);
    return CRIMSON_OK;
}

int crimson_set_params(crimson_ctx* c, const crimson_params* p) {
    if (!c) return CRIMSON_ERR_ARG;
    CR_CHECK(check_params(p));
    int nbc = c->p.ndofBC;
    c->p = *p;
    c->p.ndofBC = nbc;
    return CRIMSON_OK;
}

int crimson_set_bc(crimson_ctx* c, const int* iBC, const double* BC) {
    if (!c || !iBC || !BC) return CRIMSON_ERR_ARG;
    const int n = c->nshg, nb = c->p.ndofBC;
    if (nb < 6) {
        set_last_error("ndofBC must be at least 6 (BC(:,4:6) hold the velocity constraint coefficients)");
        return CRIMSON_ERR_ARG;
    }
    int np = 0;
    for (int i = 0; i < n; ++i) {
        const int v = (iBC[i] >> 3) & 7;
        if (v != 0 && v != 7) ++np;   // bc3LHS / bc3Res project these (bc3lhs.f90:48-49)
    }
    c->npartial = np;
    std::vector<double> nm((size_t)n * nb);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < nb; ++k) nm[(size_t)nb * i + k] = BC[(size_t)k * n + i];
    c->h_iBC.assign(iBC, iBC + n);
    c->h_iBC_orig.assign(iBC, iBC + n);
    c->h_BC.assign(BC, BC + (size_t)n * nb);
    CR_CHECK(c->iBC.upload(iBC, n, c->stream));
    CR_CHECK(c->BC.upload(nm.data(), nm.size(), c->stream));
    CR_CUDA(cudaStreamSynchronize(c->stream));
    return CRIMSON_OK;
}

int crimson_set_boundary(crimson_ctx* c, int nface, const int* ienb, const int* iBCB, const double* BCB) {
    if (!c || nface < 0 || (nface > 0 && (!ienb || !iBCB))) return CRIMSON_ERR_ARG;
    c->nface = nface;
    if (nface == 0) {
        c->h_iBCB.clear();
        c->h_ienb.clear();
        return CRIMSON_OK;
    }
    std::vector<int4> hb(nface);
    std::vector<int> hbits(nface);
    std::vector<double> hbcb((size_t)nface * 18, 0.0);
    for (int f = 0; f < nface; ++f) {
        int v[4];
        for (int a = 0; a < 4; ++a) {
            v[a] = std::abs(ienb[(size_t)a * nface + f]) - 1;
            if (v[a] < 0 || v[a] >= c->nshg) return CRIMSON_ERR_ARG;
        }
        hb[f] = make_int4(v[0], v[1], v[2], v[3]);
        hbits[f] = iBCB[f];
        if (BCB)
            for (int n = 0; n < 3; ++n)
                for (int k = 0; k < 6; ++k) hbcb[18 * (size_t)f + 6 * n + k] = BCB[((size_t)k * 3 + n) * nface + f];
    }
    // per-node lists of the faces at each face node (ascending face index):
    // the node pass of ElmGMR sums the face residual records in this order
    std::vector<int> fnoff((size_t)c->nshg + 1, 0), flist(3 * (size_t)nface);
    for (int f = 0; f < nface; ++f) {
        const int v[3] = {hb[f].x, hb[f].y, hb[f].z};
        for (int n = 0; n < 3; ++n) fnoff[v[n] + 1] += 1;
    }
    for (int i = 0; i < c->nshg; ++i) fnoff[i + 1] += fnoff[i];
    std::vector<int> fill(fnoff.begin(), fnoff.end() - 1);
    for (int f = 0; f < nface; ++f) {
        const int v[3] = {hb[f].x, hb[f].y, hb[f].z};
        for (int n = 0; n < 3; ++n) flist[fill[v[n]]++] = 3 * f + n;
    }
    CR_CHECK(c->ienb.upload(hb.data(), hb.size(), c->stream));
    CR_CHECK(c->iBCB.upload(hbits.data(), hbits.size(), c->stream));
    c->h_iBCB = hbits;
    c->h_face_srf.assign(iBCB + nface, iBCB + 2 * (size_t)nface);
    c->h_ienb = hb;
    CR_CHECK(c->BCB.upload(hbcb.data(), hbcb.size(), c->stream));
    // boundary elements (all four nodes) at each node: bc3LHS puts 1 on the
    // constrained diagonal entries of a partially constrained node once per
    // boundary element containing it
    std::vector<int> bcount((size_t)c->nshg, 0);
    for (int f = 0; f < nface; ++f) {
        bcount[hb[f].x] += 1;
        bcount[hb[f].y] += 1;
        bcount[hb[f].z] += 1;
        bcount[hb[f].w] += 1;
    }
    CR_CHECK(c->fnoff.upload(fnoff.data(), fnoff.size(), c->stream));
    CR_CHECK(c->flist.upload(flist.data(), flist.size(), c->stream));
    CR_CHECK(c->bcount.upload(bcount.data(), bcount.size(), c->stream));
    CR_CUDA(cudaStreamSynchronize(c->stream));
    return CRIMSON_OK;
}

}  // extern "C"

// NASC (AsBNASC, asbnabi.f90:191-340): per node the integral of its shape
// function over the boundary faces that carry the natural-pressure bit
// (iBCB bit 1), with the 3-point triangle rule; faces in ascending order,
// the points of a face summed first.  The surface integrals of integrScalar
// (boundarydata.f90:1101-1140) weight nodal values with it.
static std::vector<double> node_surface_areas(const crimson_ctx* c) {
    const int n = c->nshg;
    std::vector<double> nasc((size_t)n, 0.0);
    if (c->h_ienb.empty() || c->h_x.size() < 3 * (size_t)c->numnp) return nasc;
    const double B3 = 0.666666666666667, C3 = 0.166666666666667, A3 = 0.3333333333333330000000000000000000;
    const double r3[3][3] = {{B3, C3, C3}, {C3, B3, C3}, {C3, C3, B3}};
    const size_t np = (size_t)c->numnp;
    auto X = [&](int node, int d) { return c->h_x[(size_t)d * np + node]; };
    for (size_t f = 0; f < c->h_ienb.size(); ++f) {
        if (!((c->h_iBCB[f] >> 1) & 1)) continue;
        const int4 e = c->h_ienb[f];
        const int nd[3] = {e.x, e.y, e.z};
        double v1[3], v2[3];
        for (int d = 0; d < 3; ++d) {
            v1[d] = X(nd[1], d) - X(nd[0], d);
            v2[d] = X(nd[2], d) - X(nd[0], d);
        }
        const double t1 = v1[1] * v2[2] - v2[1] * v1[2];
        const double t2 = v2[0] * v1[2] - v1[0] * v2[2];
        const double t3 = v1[0] * v2[1] - v2[0] * v1[1];
        const double temp = 1.0 / std::sqrt(t1 * t1 + t2 * t2 + t3 * t3);
        double rl[3] = {0.0, 0.0, 0.0};
        for (int q = 0; q < 3; ++q) {
            const double wdetjb = (2.0 * A3) / (4.0 * temp);
            for (int a = 0; a < 3; ++a) rl[a] = rl[a] + r3[q][a] * wdetjb;
        }
        for (int a = 0; a < 3; ++a) nasc[nd[a]] = nasc[nd[a]] + rl[a];
    }
    return nasc;
}

// Puts the effective codes on the device: iBC, its host copy and the count
// of partially constrained nodes.
static int upload_codes(crimson_ctx* c, const std::vector<int>& codes) {
    int np = 0;
    for (int v : codes) {
        const int m = (v >> 3) & 7;
        if (m != 0 && m != 7) ++np;
    }
    CR_CHECK(c->iBC.upload(codes.data(), codes.size(), c->stream));
    CR_CUDA(cudaStreamSynchronize(c->stream));
    c->h_iBC = codes;
    c->npartial = np;
    return CRIMSON_OK;
}

// memLS face 1 from the codes (itrdrv.f90:949-992): every node with a
// prescribed velocity component, val 1 on its free components.
static int rebuild_dirichlet_face(crimson_lhs* L, const std::vector<int>& codes) {
    std::vector<int> g;
    std::vector<double> v;
    for (size_t i = 0; i < codes.size(); ++i) {
        if (((codes[i] >> 3) & 7) == 0) continue;
        g.push_back((int)i + 1);
        for (int d = 0; d < 3; ++d) v.push_back(((codes[i] >> (3 + d)) & 1) ? 0.0 : 1.0);
    }
    return crimson_memls_bc_create(L, 1, (int)g.size(), 3, 0, g.data(), v.data());
}

// Surface integral of the pressure weighted by NASC (integrScalar of y(:,4))
// over a surface's nodes and edge nodes.
__global__ void k_surfp_step(const int* __restrict__ pnodes, int beg, int end, const double* __restrict__ pw,
                             const double4* __restrict__ y, double* __restrict__ out) {
    __shared__ double sm[32];
    double s = 0.0;
    for (int t = beg + threadIdx.x; t < end; t += blockDim.x) s += pw[t] * y[pnodes[t]].w;
    s = block_sum(s, sm);
    if (threadIdx.x == 0) *out = s;
}

// Sum of squares of x (n values) per block, then the block partials summed
// in block order by one block: deterministic.  rstatic's totres
// (rstatic.f90:60-118) is sqrt(sum / nshg) over the four dofs of res.
constexpr int kSumsqBlocks = 296;
__global__ void k_sumsq_part(const double* __restrict__ x, long long n, double* __restrict__ part) {
    __shared__ double sm[32];
    double s = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        s += x[t] * x[t];
    s = block_sum(s, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}
__global__ void k_sumsq_final(const double* __restrict__ part, int np, double* __restrict__ out) {
    __shared__ double sm[32];
    double s = 0.0;
    for (int b = threadIdx.x; b < np; b += blockDim.x) s += part[b];
    s = block_sum(s, sm);
    if (threadIdx.x == 0) *out = s;
}

// Residual control (itrdrv.f90:1516-1522, rstatic.f90:117-124): after the
// assembly of a nonlinear iteration, totres = sqrt(|res|^2 / nshg); the
// iteration counter counts the assembled iterations; once totres is below
// the criterion after at least min_iters of them, the step ends without
// this iteration's solve and update (the reference solves and then
// discards the increment) and the counter restarts.  A step that runs all
// its iterations keeps the count for the next step, as the reference does.
static int residual_control(crimson_ctx* c, const crimson_step_args* args, crimson_step_stats* st, int it,
                            bool* done) {
    *done = false;
    if (!args->rescontrol) return CRIMSON_OK;
    cudaStream_t s = c->stream;
    const long long n4 = 4LL * c->nshg;
    launch(k_sumsq_part, kSumsqBlocks, 256, 0, s, (const double*)c->res4.p, n4, c->sumsq.p);
    launch(k_sumsq_final, 1, 256, 0, s, (const double*)c->sumsq.p, kSumsqBlocks, c->sumsq.p + kSumsqBlocks);
    double ss = 0.0;
    CR_CUDA(cudaMemcpyAsync(&ss, c->sumsq.p + kSumsqBlocks, sizeof(double), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    const double totres = std::sqrt(ss / (double)c->nshg);
    if (st && it < 16) st->res_norm[it] = totres;
    c->res_iter += 1;
    if (totres < args->res_criteria && c->res_iter >= args->min_iters) {
        c->res_iter = 0;
        *done = true;
    }
    return CRIMSON_OK;
}

extern "C" {

int crimson_set_outlets(crimson_ctx* c, int ncoupled, const int* srflist, const int* ndsurf, const double* NABI) {
    if (!c || ncoupled < 0 || (ncoupled > 0 && (!srflist || !ndsurf || !NABI))) return CRIMSON_ERR_ARG;
    if (ncoupled > 8) return CRIMSON_ERR_UNSUPPORTED;
    c->ncoupled = ncoupled;
    c->srflist.assign(srflist, srflist + ncoupled);
    std::vector<int> nodes;
    std::vector<double4> nab;
    c->onode_off.assign(1, 0);
    const int n = c->nshg;
    const std::vector<double> nasc = node_surface_areas(c);
    // edsurf (boundarydata.f90:186-253): a node of surface 1 (the wall) on a
    // face of surface s > 1 is an edge node of s (the last such face wins)
    std::vector<int> ed((size_t)n, 0);
    for (size_t f = 0; f < c->h_face_srf.size(); ++f) {
        const int srf = c->h_face_srf[f];
        if (srf <= 1) continue;
        const int v[3] = {c->h_ienb[f].x, c->h_ienb[f].y, c->h_ienb[f].z};
        for (int a = 0; a < 3; ++a)
            if (ndsurf[v[a]] == 1) ed[(size_t)v[a]] = srf;
    }
    std::vector<int> pn;
    std::vector<double> pwt;
    c->pnode_off.assign(1, 0);
    c->oarea.assign((size_t)ncoupled, 0.0);
    for (int k = 0; k < ncoupled; ++k) {
        for (int i = 0; i < n; ++i) {
            if (ndsurf[i] == srflist[k]) {
                nodes.push_back(i);
                nab.push_back(make_double4(NABI[i], NABI[(size_t)n + i], NABI[2 * (size_t)n + i], nasc[i]));
            }
            // integrScalar and calculateArea (boundarydata.f90:259-300,
            // 1101-1140) take the surface's nodes and its edge nodes
            if (ndsurf[i] == srflist[k] || (ndsurf[i] == 1 && ed[(size_t)i] == srflist[k])) {
                pn.push_back(i);
                pwt.push_back(nasc[i]);
                c->oarea[k] += nasc[i];
            }
        }
        c->onode_off.push_back((int)nodes.size());
        c->pnode_off.push_back((int)pn.size());
    }
    CR_CHECK(c->pnodes.upload(pn.data(), pn.size(), c->stream));
    CR_CHECK(c->pw.upload(pwt.data(), pwt.size(), c->stream));
    CR_CHECK(c->onodes.upload(nodes.data(), nodes.size(), c->stream));
    c->h_onodes = nodes;
    CR_CHECK(c->onabi.upload(nab.data(), nab.size(), c->stream));
    CR_CHECK(c->d_onode_off.upload(c->onode_off.data(), c->onode_off.size(), c->stream));
    CR_CHECK(c->flowq.alloc((size_t)ncoupled));
    CR_CHECK(c->coefs.alloc(2 * (size_t)ncoupled));
    c->coef_host.assign(2 * (size_t)ncoupled, 0.0);
    CR_CUDA(cudaStreamSynchronize(c->stream));
    c->rcr_Pn.assign(ncoupled, 0.0);
    c->rcr_Qn.assign(ncoupled, 0.0);
    c->netlists.assign((size_t)ncoupled, nullptr);
    c->loops.clear();
    c->loop_surfaces.clear();
    c->loop_of.assign((size_t)ncoupled, -1);
    return CRIMSON_OK;
}

int crimson_genadj(crimson_ctx* c, int* colm, int* rowp, long long cap, long long* nnz_tot) {
    if (!c) return CRIMSON_ERR_ARG;
    if (c->nnz == 0) CR_CHECK(build_pattern(c));
    if (nnz_tot) *nnz_tot = c->nnz;
    return pattern_to_host(c, colm, rowp, cap);
}

int crimson_elmgmr_device(crimson_ctx* c, const double* d_y, const double* d_ac, const double* coef1,
                          const double* coef2, double* d_res, double* d_lhsK, double* d_lhsP, int lhs) {
    if (!c || !d_y || !d_ac || !d_res) return CRIMSON_ERR_ARG;
    if (lhs && (!d_lhsK || !d_lhsP)) return CRIMSON_ERR_ARG;
    if (c->nnz == 0) CR_CHECK(build_pattern(c));
    return elmgmr_device(c, d_y, d_ac, coef1, coef2, d_res, d_lhsK, d_lhsP, lhs);
}

int crimson_elmgmr(crimson_ctx* c, const double* y, const double* ac, const double* coef1, const double* coef2,
                   double* res, double* lhsK, double* lhsP, int lhs) {
    if (!c || !y || !ac || !res) return CRIMSON_ERR_ARG;
    if (lhs && (!lhsK || !lhsP)) return CRIMSON_ERR_ARG;
    if (c->nnz == 0) CR_CHECK(build_pattern(c));
    cudaStream_t s = c->stream;
    const int n = c->nshg;
    DBuf<double> tmp;
    CR_CHECK(tmp.alloc(4 * (size_t)n));
    CR_CHECK(c->y4.alloc(4 * (size_t)n));
    CR_CHECK(c->ac4.alloc(4 * (size_t)n));
    CR_CHECK(c->res4.alloc(4 * (size_t)n));
    if (lhs) {
        CR_CHECK(c->lhsK.alloc(9 * (size_t)c->nnz));
        CR_CHECK(c->lhsP.alloc(4 * (size_t)c->nnz));
    }
    CR_CUDA(cudaMemcpyAsync(tmp.p, y, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, s));
    launch(k_soa_to_node4, grid_for(n, 256), 256, 0, s, tmp.p, n, n, c->y4.p);
    CR_CUDA(cudaStreamSynchronize(s));
    CR_CUDA(cudaMemcpyAsync(tmp.p, ac, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, s));
    launch(k_soa_to_node4, grid_for(n, 256), 256, 0, s, tmp.p, n, n, c->ac4.p);
    CR_CHECK(elmgmr_device(c, c->y4.p, c->ac4.p, coef1, coef2, c->res4.p, lhs ? c->lhsK.p : nullptr,
                           lhs ? c->lhsP.p : nullptr, lhs));
    launch(k_node4_to_soa, grid_for(n, 256), 256, 0, s, c->res4.p, n, tmp.p);
    CR_CUDA(cudaMemcpyAsync(res, tmp.p, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, s));
    if (lhs) {
        CR_CUDA(cudaMemcpyAsync(lhsK, c->lhsK.p, sizeof(double) * 9 * (size_t)c->nnz, cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaMemcpyAsync(lhsP, c->lhsP.p, sizeof(double) * 4 * (size_t)c->nnz, cudaMemcpyDeviceToHost, s));
    }
    CR_CUDA(cudaStreamSynchronize(s));
    return CRIMSON_OK;
}

int crimson_elmgmr_sclr_device(crimson_ctx* c, int isclr, double diffus, const double* d_y, const double* d_s,
                               const double* d_sdot, const double* d_bcbs, double* d_res, double* d_lhsS, int lhs) {
    if (!c) return CRIMSON_ERR_ARG;
    CR_CHECK(check_params(&c->p));
    if (c->p.flmpl != 0.0 || c->p.flmpr != 0.0 || (c->p.idiff != 0 && c->p.idiff != 1)) {
        set_last_error("ElmGMRSclr: lumped mass fractions and idiff other than 0 or 1 are not supported");
        return CRIMSON_ERR_UNSUPPORTED;
    }
    if (!d_bcbs && isclr >= 1 && isclr <= 4)
        for (int f = 0; f < (int)c->h_iBCB.size(); ++f)
            if ((c->h_iBCB[f] >> (4 + isclr)) & 1) {
                set_last_error("ElmGMRSclr: a face prescribes the scalar flux (iBCB bit 4+isclr) but bcbs is NULL");
                return CRIMSON_ERR_ARG;
            }
    return elmgmr_sclr_device(c, isclr, diffus, d_y, d_s, d_sdot, d_bcbs, d_res, d_lhsS, lhs);
}

int crimson_elmgmr_sclr(crimson_ctx* c, int isclr, double diffus, const double* y, const double* s,
                        const double* sdot, const double* bcbs, double* res, double* lhsS, int lhs) {
    if (!c || !y || !s || !sdot || !res || (lhs && !lhsS)) return CRIMSON_ERR_ARG;
    if (c->nnz == 0) CR_CHECK(build_pattern(c));
    cudaStream_t st = c->stream;
    const int n = c->nshg;
    const int nf = c->nface;
    CR_CHECK(c->y4.alloc(4 * (size_t)n));
    CR_CHECK(c->sclr_in.alloc(4 * (size_t)n + 3 * (size_t)std::max(nf, 1)));
    CR_CHECK(c->sclr_res.alloc((size_t)n));
    if (lhs) CR_CHECK(c->sclr_lhs.alloc((size_t)c->nnz));
    double* d_stage = c->sclr_in.p;  // y (reference layout), then s, sdot, bcbs
    CR_CUDA(cudaMemcpyAsync(d_stage, y, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, st));
    launch(k_soa_to_node4, grid_for(n, 256), 256, 0, st, (const double*)d_stage, n, n, c->y4.p);
    CR_CUDA(cudaStreamSynchronize(st));
    CR_CUDA(cudaMemcpyAsync(d_stage, s, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    CR_CUDA(cudaMemcpyAsync(d_stage + n, sdot, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    double* d_b = nullptr;
    if (bcbs && nf > 0) {
        // reference layout (nface, 3) -> face-major
        std::vector<double> hb(3 * (size_t)nf);
        for (int f = 0; f < nf; ++f)
            for (int k = 0; k < 3; ++k) hb[3 * (size_t)f + k] = bcbs[(size_t)k * nf + f];
        d_b = d_stage + 2 * (size_t)n;
        CR_CUDA(cudaMemcpyAsync(d_b, hb.data(), sizeof(double) * hb.size(), cudaMemcpyHostToDevice, st));
        CR_CUDA(cudaStreamSynchronize(st));
    }
    CR_CHECK(crimson_elmgmr_sclr_device(c, isclr, diffus, c->y4.p, d_stage, d_stage + n, d_b, c->sclr_res.p,
                                        lhs ? c->sclr_lhs.p : nullptr, lhs));
    CR_CUDA(cudaMemcpyAsync(res, c->sclr_res.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    if (lhs) CR_CUDA(cudaMemcpyAsync(lhsS, c->sclr_lhs.p, sizeof(double) * (size_t)c->nnz, cudaMemcpyDeviceToHost, st));
    CR_CUDA(cudaStreamSynchronize(st));
    return CRIMSON_OK;
}

// ---------------------------------------------------------------------------
// memLS objects
// ---------------------------------------------------------------------------
int crimson_memls_ls_create(crimson_ls** out, int LS_type, int present_mask, double relTol, double absTol, int maxItr,
                            int dimKry, const double* relTolIn, const double* absTolIn, const int* maxItrIn) {
    if (!out) return CRIMSON_ERR_ARG;
    if (LS_type != CRIMSON_LS_TYPE_NS) return CRIMSON_ERR_UNSUPPORTED;
    crimson_ls* ls = new crimson_ls();
    // memLS_LS_CREATE defaults (flowsolver/src/memLS.f90:1395-1414)
    ls->RI.relTol = 4e-1;
    ls->GM.relTol = 1e-2;
    ls->CG.relTol = 1e-1;
    ls->RI.mItr = 10;
    ls->GM.mItr = 3;
    ls->CG.mItr = 500;
    ls->GM.sD = 50;
    ls->RI.absTol = 1e-10;
    ls->GM.absTol = 1e-10;
    ls->CG.absTol = 1e-10;
    if (present_mask & 1) ls->RI.relTol = relTol;
    if (present_mask & 2) ls->RI.absTol = absTol;
    if (present_mask & 4) ls->RI.mItr = maxItr;
    if (present_mask & 8) {
        ls->RI.sD = dimKry;
        ls->GM.sD = dimKry;
    }
    if ((present_mask & 16) && relTolIn) {
        ls->GM.relTol = relTolIn[0];
        ls->CG.relTol = relTolIn[1];
    }
    if ((present_mask & 32) && absTolIn) {
        ls->GM.absTol = absTolIn[0];
        ls->CG.absTol = absTolIn[1];
    }
    if ((present_mask & 64) && maxItrIn) {
        ls->GM.mItr = maxItrIn[0];
        ls->CG.mItr = maxItrIn[1];
    }
    *out = ls;
    return CRIMSON_OK;
}

int crimson_memls_ls_free(crimson_ls* ls) {
    delete ls;
    return CRIMSON_OK;
}

int crimson_memls_ls_set_precision(crimson_ls* ls, int precision, int max_refine, double refine_tol) {
    if (!ls || precision < CRIMSON_FP64 || precision > CRIMSON_MIXED_F32_TANGENT || max_refine < 1 || max_refine > 64 ||
        !(refine_tol < 1.0))
        return CRIMSON_ERR_ARG;
    ls->precision = precision;
    ls->max_refine = max_refine;
    ls->refine_tol = refine_tol;
    return CRIMSON_OK;
}

int crimson_memls_ls_set_schur(crimson_ls* ls, int explicit_schur) {
    if (!ls || explicit_schur < 0 || explicit_schur > 1) return CRIMSON_ERR_ARG;
    ls->schur = explicit_schur;
    return CRIMSON_OK;
}

int crimson_memls_schur_info(const crimson_lhs* L, int* state, long long* nnz, long long* npad, double* form_ms) {
    if (!L) return CRIMSON_ERR_ARG;
    if (state) *state = L->s2_state;
    if (nnz) *nnz = L->s2_nnz;
    if (npad) *npad = L->s2_npad;
    if (form_ms) *form_ms = L->s2_forms > 0 ? L->s2_form_ms / L->s2_forms : 0.0;
    return CRIMSON_OK;
}

int crimson_memls_ls_set_log(crimson_ls* ls, const char* path) {
    if (!ls) return CRIMSON_ERR_ARG;
    ls->log_path = path ? std::string(path) : std::string();
    return CRIMSON_OK;
}

int crimson_memls_refine_info(const crimson_lhs* L, int* steps, double* rel) {
    if (!L) return CRIMSON_ERR_ARG;
    if (steps) *steps = L->refine_steps;
    if (rel) *rel = L->refine_rel;
    return CRIMSON_OK;
}

__global__ void k_one_to_zero(const int* __restrict__ in, int* __restrict__ out, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        out[t] = in[t] - 1;
}

int crimson_memls_lhs_create(crimson_lhs** out, int gnNo, int nNo, long long nnz, const int* gNodes,
                             const int* rowPtr, const int* colPtr, int nFaces) {
    if (!out || nNo <= 0 || nnz <= 0 || !rowPtr || !colPtr || nFaces < 0) return CRIMSON_ERR_ARG;
    crimson_lhs* L = new crimson_lhs();
    L->gnNo = gnNo;
    L->nNo = nNo;
    L->nnz = nnz;
    L->nFaces = nFaces;
    L->face.resize(nFaces);
    (void)gNodes;
    if (cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete L;
        return CRIMSON_ERR_CUDA;
    }
    L->own_stream = true;
    int rc = CRIMSON_OK;
    DBuf<int> t1, t2;
    rc = t1.upload(rowPtr, (size_t)nNo + 1, L->stream);
    if (rc == CRIMSON_OK) rc = t2.upload(colPtr, (size_t)nnz, L->stream);
    if (rc == CRIMSON_OK) rc = L->own_rowptr.alloc((size_t)nNo + 1);
    if (rc == CRIMSON_OK) rc = L->own_col.alloc((size_t)nnz);
    if (rc == CRIMSON_OK) {
        launch(k_one_to_zero, grid_for(nNo + 1, 256), 256, 0, L->stream, t1.p, L->own_rowptr.p, nNo + 1);
        launch(k_one_to_zero, grid_for(nnz, 256), 256, 0, L->stream, t2.p, L->own_col.p, nnz);
        L->rowptr = L->own_rowptr.p;
        L->col = L->own_col.p;
        rc = crimson::pattern_aux(L);
        cudaStreamSynchronize(L->stream);
    }
    if (rc != CRIMSON_OK) {
        crimson_memls_lhs_free(L);
        return rc;
    }
    *out = L;
    return CRIMSON_OK;
}

int crimson_memls_lhs_create_from_ctx(crimson_lhs** out, crimson_ctx* c, int nFaces) {
    if (!out || !c || nFaces < 0) return CRIMSON_ERR_ARG;
    if (c->nnz == 0) CR_CHECK(build_pattern(c));
    crimson_lhs* L = new crimson_lhs();
    L->gnNo = c->nshg;
    L->nNo = c->nshg;
    L->nnz = c->nnz;
    L->nFaces = nFaces;
    L->face.resize(nFaces);
    L->stream = c->stream;
    L->own_stream = false;
    L->rowptr = c->rowptr.p;
    L->col = c->col.p;
    L->diag = c->diag.p;
    L->trans = c->trans.p;
    *out = L;
    return CRIMSON_OK;
}

int crimson_memls_lhs_free(crimson_lhs* L) {
    if (!L) return CRIMSON_ERR_ARG;
    // An lhs made from a context borrows that context's stream and must be
    // freed before the context; it never touches the borrowed stream here.
    if (L->own_stream && L->stream) cudaStreamSynchronize(L->stream);
    if (L->hscal) cudaFreeHost(L->hscal);
    if (L->ev0) cudaEventDestroy(L->ev0);
    if (L->ev1) cudaEventDestroy(L->ev1);
    if (L->s2_ev0) cudaEventDestroy(L->s2_ev0);
    if (L->s2_ev1) cudaEventDestroy(L->s2_ev1);
    cudaStream_t s = L->own_stream ? L->stream : nullptr;
    delete L;
    if (s) cudaStreamDestroy(s);
    return CRIMSON_OK;
}

int crimson_memls_bc_create(crimson_lhs* L, int faIn, int nNo, int dof, int BC_type, const int* gNodes,
                            const double* Val) {
    if (!L) return CRIMSON_ERR_ARG;
    if (faIn > L->nFaces || faIn < 1) {
        set_last_error("faIn exceeds the lhs structure's number of faces");
        return CRIMSON_ERR_ARG;
    }
    if (nNo < 0 || dof <= 0 || dof > 4 || (nNo > 0 && !gNodes)) return CRIMSON_ERR_ARG;
    MemlsFace& f = L->face[faIn - 1];
    f.nNo = nNo;
    f.dof = dof;
    f.bGrp = BC_type;
    f.created = true;
    std::vector<int> g(nNo);
    for (int a = 0; a < nNo; ++a) {
        g[a] = gNodes[a] - 1;
        if (g[a] < 0 || g[a] >= L->nNo) return CRIMSON_ERR_ARG;
    }
    std::vector<double> v((size_t)dof * nNo, 0.0);
    if (Val) std::memcpy(v.data(), Val, sizeof(double) * v.size());
    CR_CHECK(f.glob.upload(g.data(), g.size(), L->stream));
    CR_CHECK(f.val.upload(v.data(), v.size(), L->stream));
    CR_CHECK(f.valM.alloc(v.size()));
    CR_CUDA(cudaMemsetAsync(f.valM.p, 0, sizeof(double) * v.size(), L->stream));
    CR_CUDA(cudaStreamSynchronize(L->stream));
    return CRIMSON_OK;
}

int crimson_memls_solve(crimson_lhs* L, crimson_ls* ls, int dof, double* Ri, double* Val, const int* incL,
                        const double* res, crimson_ls_stats* stats) {
    if (!L || !ls || !Ri || !Val) return CRIMSON_ERR_ARG;
    if (dof != 4 || ls->LS_type != CRIMSON_LS_TYPE_NS) return CRIMSON_ERR_UNSUPPORTED;
    return memls_solve_val(L, ls, Ri, Val, incL, res, stats);
}

int crimson_solflow_device(crimson_ctx* c, crimson_lhs* L, crimson_ls* ls, const double* d_res, const double* d_lhsK,
                           const double* d_lhsP, const int* incL, const double* faceRes, double* d_solinc,
                           crimson_ls_stats* stats) {
    if (!c || !L || !ls || !d_res || !d_lhsK || !d_lhsP || !d_solinc) return CRIMSON_ERR_ARG;
    if (L->diag == nullptr || L->trans == nullptr) return CRIMSON_ERR_STATE;
    return memls_solve_lhs_device(L, ls, d_res, d_lhsK, d_lhsP, incL, faceRes, d_solinc, stats);
}

int crimson_solflow_device_transposed(crimson_ctx* c, crimson_lhs* L, crimson_ls* ls, const double* d_rhs,
                                      const double* d_lhsK, const double* d_lhsP, const int* incL,
                                      const double* faceRes, double* d_sol, crimson_ls_stats* stats) {
    if (!c || !L || !ls || !d_rhs || !d_lhsK || !d_lhsP || !d_sol) return CRIMSON_ERR_ARG;
    if (L->diag == nullptr || L->trans == nullptr) return CRIMSON_ERR_STATE;
    return memls_solve_lhs_device(L, ls, d_rhs, d_lhsK, d_lhsP, incL, faceRes, d_sol, stats, true);
}

int crimson_elmgmr_device_f32(crimson_ctx* c, const double* d_y, const double* d_ac, const double* coef1,
                              const double* coef2, double* d_res, float* d_lhs32) {
    if (!c || !d_y || !d_ac || !d_res || !d_lhs32) return CRIMSON_ERR_ARG;
    if (c->ncoupled > 0 && (!coef1 || !coef2)) return CRIMSON_ERR_ARG;
    CR_CHECK(check_params(&c->p));
    if (c->nnz == 0) CR_CHECK(build_pattern(c));
    return elmgmr_device(c, d_y, d_ac, coef1, coef2, d_res, nullptr, nullptr, 2, d_lhs32);
}

int crimson_solflow_device_f32(crimson_ctx* c, crimson_lhs* L, crimson_ls* ls, const double* d_res,
                               const float* d_lhs32, const int* incL, const double* faceRes, double* d_solinc,
                               crimson_ls_stats* stats) {
    if (!c || !L || !ls || !d_res || !d_lhs32 || !d_solinc) return CRIMSON_ERR_ARG;
    if (L->diag == nullptr || L->trans == nullptr) return CRIMSON_ERR_STATE;
    return memls_solve_lhs_device(L, ls, d_res, nullptr, nullptr, incL, faceRes, d_solinc, stats, false, d_lhs32);
}

int crimson_spmv4_prepare(crimson_ctx* c, int precision, const void* d_val) {
    if (!c || !d_val || (precision != CRIMSON_FP64 && precision != CRIMSON_MIXED)) return CRIMSON_ERR_ARG;
    if (c->nnz == 0) CR_CHECK(build_pattern(c));
    return spmv4_prepare(c, precision, d_val);
}

int crimson_spmv4_apply(crimson_ctx* c, const void* d_u, void* d_ku) {
    if (!c || !d_u || !d_ku) return CRIMSON_ERR_ARG;
    if (!c->s4_ptr.p) return CRIMSON_ERR_STATE;
    return spmv4_apply(c, d_u, d_ku);
}

int crimson_elmgmr_vjp(crimson_ctx* c, const double* d_y, const double* d_ac, const double* coef1,
                       const double* coef2, const double* d_lambda, double* d_res, double* d_ybar, double* d_acbar,
                       double* mubar, double* coef1bar, double* coef2bar) {
    if (!c || !d_y || !d_ac || !d_lambda || !d_ybar || !d_acbar) return CRIMSON_ERR_ARG;
    if (c->ncoupled > 0 && (!coef1 || !coef2)) return CRIMSON_ERR_ARG;
    CR_CHECK(check_params(&c->p));
    if (c->npartial > 0) {
        set_last_error("crimson_elmgmr_vjp: partially constrained velocity nodes are not differentiated");
        return CRIMSON_ERR_UNSUPPORTED;
    }
    return elmgmr_vjp(c, d_y, d_ac, coef1, coef2, d_lambda, d_res, d_ybar, d_acbar, mubar, coef1bar, coef2bar);
}

// ---------------------------------------------------------------------------
// Time stepping
// ---------------------------------------------------------------------------
int crimson_set_inflow(crimson_ctx* c, int ninlet, const int* nodes, const double* profile) {
    if (!c || ninlet < 0 || (ninlet > 0 && (!nodes || !profile))) return CRIMSON_ERR_ARG;
    std::vector<int> g(ninlet);
    for (int t = 0; t < ninlet; ++t) {
        g[t] = nodes[t] - 1;
        if (g[t] < 0 || g[t] >= c->nshg) return CRIMSON_ERR_ARG;
    }
    c->ninlet = ninlet;
    CR_CHECK(c->inlet_nodes.upload(g.data(), g.size(), c->stream));
    CR_CHECK(c->inlet_profile.upload(profile, 3 * (size_t)ninlet, c->stream));
    CR_CUDA(cudaStreamSynchronize(c->stream));
    return CRIMSON_OK;
}

int crimson_set_rcr(crimson_ctx* c, int n, const double* Rp, const double* C, const double* Rd, const double* Pd) {
    if (!c || n != c->ncoupled) return CRIMSON_ERR_ARG;
    c->rcr_Rp.assign(Rp, Rp + n);
    c->rcr_C.assign(C, C + n);
    c->rcr_Rd.assign(Rd, Rd + n);
    c->rcr_Pd.assign(Pd, Pd + n);
    c->rcr_Pn.assign(n, 0.0);
    c->rcr_Qn.assign(n, 0.0);
    return CRIMSON_OK;
}

int crimson_set_outlet_netlist(crimson_ctx* c, int k, crimson_netlist* nl) {
    if (!c || k < 0 || k >= c->ncoupled) return CRIMSON_ERR_ARG;
    c->netlists.resize((size_t)c->ncoupled, nullptr);
    c->loop_of.resize((size_t)c->ncoupled, -1);
    if (c->loop_of[(size_t)k] >= 0) {
        set_last_error("crimson_set_outlet_netlist: the surface belongs to a closed loop");
        return CRIMSON_ERR_STATE;
    }
    if (nl && !nl->connect_nodes.empty()) {
        set_last_error("crimson_set_outlet_netlist: a member of a closed loop couples through its loop");
        return CRIMSON_ERR_ARG;
    }
    c->netlists[(size_t)k] = nl;
    return CRIMSON_OK;
}

int crimson_set_outlet_netlist_loop(crimson_ctx* c, crimson_netlist_loop* loop, const int* surfaces) {
    if (!c || !loop || !surfaces) return CRIMSON_ERR_ARG;
    const int nc = c->ncoupled;
    c->netlists.resize((size_t)nc, nullptr);
    c->loop_of.resize((size_t)nc, -1);
    for (crimson_netlist_loop* l : c->loops)
        if (l == loop) return CRIMSON_ERR_ARG;
    for (int j = 0; j < loop->nup; ++j) {
        const int k = surfaces[j];
        if (k < 0 || k >= nc || c->netlists[(size_t)k] || c->loop_of[(size_t)k] >= 0) {
            set_last_error("crimson_set_outlet_netlist_loop: a surface is out of range or already coupled");
            return CRIMSON_ERR_ARG;
        }
        for (int e = 0; e < j; ++e)
            if (surfaces[e] == k) return CRIMSON_ERR_ARG;
    }
    const int l = (int)c->loops.size();
    c->loops.push_back(loop);
    c->loop_surfaces.emplace_back(surfaces, surfaces + loop->nup);
    for (int j = 0; j < loop->nup; ++j) {
        c->netlists[(size_t)surfaces[j]] = loop->member[(size_t)j];
        c->loop_of[(size_t)surfaces[j]] = l;
    }
    return CRIMSON_OK;
}

int crimson_rcr_state(crimson_ctx* c, int n, double* Pn, double* Qn, int set) {
    if (!c || n != c->ncoupled || (n > 0 && (!Pn || !Qn))) return CRIMSON_ERR_ARG;
    if ((int)c->rcr_Pn.size() != n) return CRIMSON_ERR_STATE;
    for (int k = 0; k < n; ++k) {
        if (set) {
            c->rcr_Pn[k] = Pn[k];
            c->rcr_Qn[k] = Qn[k];
        } else {
            Pn[k] = c->rcr_Pn[k];
            Qn[k] = c->rcr_Qn[k];
        }
    }
    return CRIMSON_OK;
}
int crimson_state_set(crimson_ctx* c, const double* y, const double* ac) {
    if (!c || !y || !ac) return CRIMSON_ERR_ARG;
    const int n = c->nshg;
    cudaStream_t s = c->stream;
    for (DBuf<double>* b :
         {&c->yold, &c->acold, &c->ycur, &c->accur, &c->yalpha, &c->acalpha, &c->solinc, &c->res4, &c->stage})
        CR_CHECK(b->alloc(4 * (size_t)n));
    CR_CUDA(cudaMemcpyAsync(c->stage.p, y, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, s));
    launch(k_soa_to_node4, grid_for(n, 256), 256, 0, s, c->stage.p, n, n, c->yold.p);
    CR_CUDA(cudaStreamSynchronize(s));
    CR_CUDA(cudaMemcpyAsync(c->stage.p, ac, sizeof(double) * 4 * n, cudaMemcpyHostToDevice, s));
    launch(k_soa_to_node4, grid_for(n, 256), 256, 0, s, c->stage.p, n, n, c->acold.p);
    CR_CUDA(cudaStreamSynchronize(s));
    return CRIMSON_OK;
}

// GetFlowQ and integrScalar(p) / area (bctcardio.f90:1021-1040's Updcalc)
// of every coupled surface for the current state.
int crimson_outlet_state(crimson_ctx* c, int n, double* q, double* p_mean) {
    if (!c || n != c->ncoupled || (n > 0 && (!q || !p_mean))) return CRIMSON_ERR_ARG;
    if (!c->yold.p) return CRIMSON_ERR_STATE;
    if (n == 0) return CRIMSON_OK;
    cudaStream_t s = c->stream;
    CR_CHECK(c->psurf.alloc((size_t)n));
    for (int k = 0; k < n; ++k) {
        launch(k_flowq_step, 1, 256, 0, s, c->onodes.p, c->onode_off[k], c->onode_off[k + 1], c->onabi.p,
               reinterpret_cast<const double4*>(c->yold.p), c->flowq.p + k);
        launch(k_surfp_step, 1, 256, 0, s, c->pnodes.p, c->pnode_off[k], c->pnode_off[k + 1], c->pw.p,
               reinterpret_cast<const double4*>(c->yold.p), c->psurf.p + k);
    }
    CR_CUDA(cudaMemcpyAsync(q, c->flowq.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaMemcpyAsync(p_mean, c->psurf.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < n; ++k) p_mean[k] = c->oarea[(size_t)k] > 0.0 ? p_mean[k] / c->oarea[(size_t)k] : 0.0;
    return CRIMSON_OK;
}

int crimson_state_get(crimson_ctx* c, double* y, double* ac) {
    if (!c || !c->yold.p || !c->stage.p) return CRIMSON_ERR_STATE;
    const int n = c->nshg;
    cudaStream_t s = c->stream;
    if (y) {
        launch(k_node4_to_soa, grid_for(n, 256), 256, 0, s, c->yold.p, n, c->stage.p);
        CR_CUDA(cudaMemcpyAsync(y, c->stage.p, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
    }
    if (ac) {
        launch(k_node4_to_soa, grid_for(n, 256), 256, 0, s, c->acold.p, n, c->stage.p);
        CR_CUDA(cudaMemcpyAsync(ac, c->stage.p, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
    }
    return CRIMSON_OK;
}

int crimson_step(crimson_ctx* c, crimson_lhs* L, crimson_ls* ls, const crimson_step_args* args,
                 crimson_step_stats* st) {
    if (!c || !L || !ls || !args) return CRIMSON_ERR_ARG;
    if (!c->yold.p) return CRIMSON_ERR_STATE;
    if (args->nitr < 1 || args->nitr > 16) return CRIMSON_ERR_ARG;
    if (L->nFaces != 1 + c->ncoupled) return CRIMSON_ERR_STATE;
    cudaStream_t s = c->stream;
    const crimson_params& P = c->p;
    const int n = c->nshg;
    if (c->nnz == 0) CR_CHECK(build_pattern(c));
    CR_CHECK(c->lhsK.alloc(9 * (size_t)c->nnz));
    CR_CHECK(c->lhsP.alloc(4 * (size_t)c->nnz));
    const int nb = P.ndofBC;
    if (c->ninlet > 0)
        launch(k_inflow, grid_for(c->ninlet, 256), 256, 0, s, c->inlet_nodes.p, c->inlet_profile.p, c->ninlet,
                                                          args->inflow_scale, nb, c->BC.p);
    const int nc = c->ncoupled;
    c->netlists.resize((size_t)nc, nullptr);
    std::vector<double> c1(nc), c2(nc), faceRes(1 + nc, 0.0);
    for (int k = 0; k < nc; ++k)
        if (!c->netlists[(size_t)k] && (int)c->rcr_Rp.size() != nc) {
            set_last_error("crimson_step: coupled surface without an RCR (crimson_set_rcr) or a netlist");
            return CRIMSON_ERR_STATE;
        }
    // Netlists whose closed diodes block the interface (Dirichlet design):
    // the surface keeps its original Dirichlet codes and is not coupled.
    std::vector<char> blocked((size_t)nc, 0);
    for (int k = 0; k < nc; ++k)
        if (crimson_netlist* nl = c->netlists[(size_t)k]) {
            CR_CHECK(netlist_begin_step(nl));  // initialiseAtStartOfTimestep
            blocked[(size_t)k] = nl->flow_permitted ? 0 : 1;
        }
    {
        // iBC = iBC_original with zeros at the nodes of every coupled surface
        // that takes flow (the binary mask of itrdrv.f90:1114-1133,
        // BoundaryConditionManager.cxx:797-811); memLS face 1 follows the
        // codes (rebuildMemLS_lhs, itrdrv.f90:887-1023)
        std::vector<int> codes(c->h_iBC_orig);
        for (int k = 0; k < nc; ++k)
            if (!blocked[(size_t)k])
                for (int t = c->onode_off[k]; t < c->onode_off[k + 1]; ++t) codes[(size_t)c->h_onodes[t]] = 0;
        if (codes != c->h_iBC) {
            CR_CHECK(upload_codes(c, codes));
            CR_CHECK(rebuild_dirichlet_face(L, codes));
        }
    }
    // itrPredict (ipred = 1) and itrBC with the step's codes
    const double fct = (P.gami - 1.0) / P.gami;
    launch(k_predict, grid_for(4LL * n, 256), 256, 0, s, c->yold.p, c->acold.p, c->ycur.p, c->accur.p, 4LL * n, fct);
    launch(k_itrbc, grid_for(n, 256), 256, 0, s, c->iBC.p, c->BC.p, nb, n, c->ycur.p);
    c->loop_of.resize((size_t)nc, -1);
    // closed loops: one solve gives the coefficients of all their surfaces
    for (size_t l = 0; l < c->loops.size(); ++l) {
        const std::vector<int>& sf = c->loop_surfaces[l];
        std::vector<double> a(sf.size()), b(sf.size());
        CR_CHECK(crimson_netlist_loop_implicit_coefficients(c->loops[l], P.alfi * P.Delt, a.data(), b.data()));
        for (size_t j = 0; j < sf.size(); ++j) {
            c1[(size_t)sf[j]] = a[j];
            c2[(size_t)sf[j]] = b[j];
        }
    }
    for (int k = 0; k < nc; ++k) {
        if (crimson_netlist* nl = c->netlists[(size_t)k]) {
            // the implicit coefficients with alfi*Delt
            // (AbstractBoundaryCondition.cxx:32-53); none in the Dirichlet design
            if (blocked[(size_t)k]) {
                c1[k] = c2[k] = 0.0;
                continue;
            }
            if (c->loop_of[(size_t)k] >= 0) continue;
            CR_CHECK(crimson_netlist_implicit_coefficients(nl, P.alfi * P.Delt, &c1[k], &c2[k]));
        } else {
            rcr_coeffs(c->rcr_Rp[k], c->rcr_C[k], c->rcr_Rd[k], c->rcr_Pd[k], c->rcr_Pd[k], c->rcr_Pn[k],
                       c->rcr_Qn[k], P.alfi * P.Delt, &c1[k], &c2[k]);
        }
    }
    for (int k = 0; k < nc; ++k) faceRes[1 + k] = c1[k] * P.alfi * P.gami * P.Delt;
    std::vector<int> incL(1 + nc, 1);
    if (st) std::memset(st, 0, sizeof(*st));
    if (args->rescontrol) CR_CHECK(c->sumsq.alloc(kSumsqBlocks + 1));
    for (int it = 0; it < args->nitr; ++it) {
        launch(k_yalpha, grid_for(n, 256), 256, 0, s, c->yold.p, c->acold.p, c->ycur.p, c->accur.p, c->yalpha.p,
                                                  c->acalpha.p, n, P.alfi, P.almi);
        crimson_ls_stats lst;
        if (ls->precision == CRIMSON_MIXED_F32_TANGENT) {
            // FP32 element quadrature for the tangent, FP64 residual
            CR_CHECK(c->lhs32.alloc(16 * (size_t)c->nnz));
            CR_CHECK(elmgmr_device(c, c->yalpha.p, c->acalpha.p, c1.data(), c2.data(), c->res4.p, nullptr, nullptr, 2,
                                   c->lhs32.p));
            bool done = false;
            CR_CHECK(residual_control(c, args, st, it, &done));
            if (done) break;
            CR_CHECK(memls_solve_lhs_device(L, ls, c->res4.p, nullptr, nullptr, incL.data(), faceRes.data(),
                                            c->solinc.p, &lst, false, c->lhs32.p));
        } else {
            CR_CHECK(elmgmr_device(c, c->yalpha.p, c->acalpha.p, c1.data(), c2.data(), c->res4.p, c->lhsK.p,
                                   c->lhsP.p, 1));
            bool done = false;
            CR_CHECK(residual_control(c, args, st, it, &done));
            if (done) break;
            CR_CHECK(memls_solve_lhs_device(L, ls, c->res4.p, c->lhsK.p, c->lhsP.p, incL.data(), faceRes.data(),
                                            c->solinc.p, &lst));
        }
        launch(k_correct, grid_for(n, 256), 256, 0, s, c->ycur.p, c->accur.p, c->solinc.p, n, P.gami * P.Delt,
                                                   P.gami * P.alfi * P.Delt);
        launch(k_itrbc, grid_for(n, 256), 256, 0, s, c->iBC.p, c->BC.p, nb, n, c->ycur.p);
        if (st) {
            st->ri_itr[it] = lst.RI.itr;
            st->gm_itr[it] = lst.GM.itr;
            st->cg_itr[it] = lst.CG.itr;
            st->ri_inorm[it] = lst.RI.iNorm;
            st->ri_fnorm[it] = lst.RI.fNorm;
            st->refine_steps[it] = ls->precision == CRIMSON_FP64 ? 0 : L->refine_steps;
            st->refine_rel[it] = ls->precision == CRIMSON_FP64 ? 0.0 : L->refine_rel;
            st->nsolves = it + 1;
        }
    }
    // RCR history update at t_{n+1} (AbstractBoundaryCondition.cxx:55-91)
    if (nc > 0) {
        for (int k = 0; k < nc; ++k)
            launch(k_flowq_step, 1, 256, 0, s, c->onodes.p, c->onode_off[k], c->onode_off[k + 1], c->onabi.p,
                                           reinterpret_cast<const double4*>(c->ycur.p), c->flowq.p + k);
        // surface pressures of the blocked netlist surfaces (updmultidomaincontainer,
        // elmgmr.f90:1733-1743: integrScalar of p / area, at t_{n+1})
        CR_CHECK(c->psurf.alloc((size_t)nc));
        for (int k = 0; k < nc; ++k)
            if (blocked[(size_t)k])
                launch(k_surfp_step, 1, 256, 0, s, c->pnodes.p, c->pnode_off[k], c->pnode_off[k + 1], c->pw.p,
                                              reinterpret_cast<const double4*>(c->ycur.p), c->psurf.p + k);
        std::vector<double> hq(nc), hp(nc, 0.0);
        CR_CUDA(cudaMemcpyAsync(hq.data(), c->flowq.p, sizeof(double) * nc, cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaMemcpyAsync(hp.data(), c->psurf.p, sizeof(double) * nc, cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        for (int k = 0; k < nc; ++k)
            if (blocked[(size_t)k] && !(c->oarea[(size_t)k] > 0.0)) {
                set_last_error("crimson_step: a blocked netlist surface has no area (set the boundary faces "
                               "before crimson_set_outlets)");
                return CRIMSON_ERR_STATE;
            }
        // closed loops: one update of every member with the flows (or, blocked,
        // the surface pressures) of their surfaces, then the finalisation
        for (size_t l = 0; l < c->loops.size(); ++l) {
            const std::vector<int>& sf = c->loop_surfaces[l];
            std::vector<double> lq(sf.size()), lp(sf.size(), 0.0);
            for (size_t j = 0; j < sf.size(); ++j) {
                lq[j] = hq[(size_t)sf[j]];
                if (blocked[(size_t)sf[j]]) lp[j] = hp[(size_t)sf[j]] / c->oarea[(size_t)sf[j]];
            }
            CR_CHECK(crimson_netlist_loop_update(c->loops[l], P.Delt, lq.data(), lp.data()));
            CR_CHECK(crimson_netlist_loop_finalize_step(c->loops[l]));
        }
        for (int k = 0; k < nc; ++k) {
            if (crimson_netlist* nl = c->netlists[(size_t)k]) {
                // updateLPN with the end-of-step flow (or, blocked, the surface
                // pressure), then finalizeLPNAtEndOfTimestep (itrdrv.f90:1686-1688)
                if (c->loop_of[(size_t)k] < 0) {
                    if (blocked[(size_t)k])
                        CR_CHECK(crimson_netlist_update_pressure(nl, P.Delt, hp[k] / c->oarea[(size_t)k]));
                    else
                        CR_CHECK(crimson_netlist_update(nl, P.Delt, hq[k]));
                    CR_CHECK(crimson_netlist_finalize_step(nl));
                }
                c->rcr_Pn[k] = nl->node[(size_t)nl->iface_node - 1].p;
                c->rcr_Qn[k] = hq[k];
                if (st && k < 8) {
                    st->q_out[k] = hq[k];
                    st->p_out[k] = c->rcr_Pn[k];
                }
                continue;
            }
            double d1, h1;
            rcr_coeffs(c->rcr_Rp[k], c->rcr_C[k], c->rcr_Rd[k], c->rcr_Pd[k], c->rcr_Pd[k], c->rcr_Pn[k], c->rcr_Qn[k],
                       P.Delt, &d1, &h1);
            c->rcr_Pn[k] = d1 * hq[k] + h1;
            c->rcr_Qn[k] = hq[k];
            if (st && k < 8) {
                st->q_out[k] = hq[k];
                st->p_out[k] = c->rcr_Pn[k];
            }
        }
    }
    CR_CUDA(cudaMemcpyAsync(c->yold.p, c->ycur.p, sizeof(double) * 4 * n, cudaMemcpyDeviceToDevice, s));
    CR_CUDA(cudaMemcpyAsync(c->acold.p, c->accur.p, sizeof(double) * 4 * n, cudaMemcpyDeviceToDevice, s));
    CR_CUDA(cudaStreamSynchronize(s));
    CR_CUDA(cudaGetLastError());
    c->istep += 1;
    return CRIMSON_OK;
}

}  // extern "C"

namespace crimson {

__global__ void k_diag_trans_only(const int* __restrict__ rowptr, const int* __restrict__ col, int n,
                                  int* __restrict__ diag, int* __restrict__ trans, int* __restrict__ bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int d = -1;
        for (int j = rowptr[i]; j < rowptr[i + 1]; ++j) {
            if (col[j] == i) d = j;
            const int c = col[j];
            int t = -1, lo = rowptr[c], hi = rowptr[c + 1];
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (col[mid] < i)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            if (lo < rowptr[c + 1] && col[lo] == i) t = lo;
            trans[j] = t;
            if (t < 0) atomicAdd(bad, 1);
        }
        diag[i] = d;
        if (d < 0) atomicAdd(bad, 1);
    }
}

// diagPtr (memLS.f90:1121-1131) and the transpose map for a caller-given pattern
int pattern_aux(crimson_lhs* L) {
    CR_CHECK(L->own_diag.alloc((size_t)L->nNo));
    CR_CHECK(L->own_trans.alloc((size_t)L->nnz));
    DBuf<int> bad;
    CR_CHECK(bad.alloc(1));
    CR_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), L->stream));
    launch(k_diag_trans_only, grid_for(L->nNo, 128), 128, 0, L->stream, L->rowptr, L->col, L->nNo, L->own_diag.p,
                                                                     L->own_trans.p, bad.p);
    int hb = 0;
    CR_CUDA(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, L->stream));
    CR_CUDA(cudaStreamSynchronize(L->stream));
    if (hb) {
        set_last_error("pattern without diagonal or not structurally symmetric");
        return CRIMSON_ERR_PATTERN;
    }
    L->diag = L->own_diag.p;
    L->trans = L->own_trans.p;
    return CRIMSON_OK;
}

}  // namespace crimson
