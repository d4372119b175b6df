// Adjoint of ElmGMR's residual: lambda^T d res / d(y_alpha, ac_alpha, mu,
// coef1, coef2), exact (no counterpart in the reference, which has no
// adjoint).
//
// res is the vector ElmGMR assembles (flowsolver/src/elmgmr.f90:82-555):
// the interior SUPG/PSPG residual (e3ivar/e3stab/e3Res, e3ivar.f90:99-198,
// e3stab.f90:83-133, e3res.f90:94-286) with the viscous-flux projection
// qres (AsIq/qpbc, asiq.f90:52-70, qpbc.f90:67-71), the boundary residual
// (e3b/e3bvar, e3b.f90:112-470), the outlet coupling p_k NABI with
// p_k = -(Q_k coef1_k) - coef2_k (elmgmr.f90:1271-1330) and bc3Res.
//
// The element tangent ElmGMR assembles (e3LHS) is the reference's
// approximate Jacobian: it omits the derivatives of tauM, tauC, tauBar and
// of uBar and the viscous-flux projection.  The adjoint needs the exact
// transposed Jacobian, so each element's residual is re-evaluated in
// forward-mode dual arithmetic: one thread per element, K derivative
// directions per pass, and the contraction with the element's lambda is
// scattered to the nodes.  Per tet the residual depends on 32 local inputs:
// y_alpha (4 nodes x p,u,v,w), ac_alpha (4 x 3), div q (3: on a linear tet
// div q = sum_n dN_n . q_n is an element constant) and mu.  The cotangent of
// div q goes to the nodal qres through dN, and from qres through the
// transposed lumped projection back to u and mu.
#include <vector>

#include "common.cuh"

namespace crimson {

int elmgmr_device(crimson_ctx* c, const double* d_y, const double* d_ac, const double* coef1, const double* coef2,
                  double* d_res, double* d_lhsK, double* d_lhsP, int lhs, float* d_lhs32 = nullptr);

// ---------------------------------------------------------------------------
// Forward-mode dual numbers
// ---------------------------------------------------------------------------
template <int K>
struct Dual {
    double v;
    double d[K];
};

template <int K>
__device__ __forceinline__ Dual<K> dconst(double x) {
    Dual<K> r;
    r.v = x;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = 0.0;
    return r;
}
// input value x, seeded with unit derivative in slot `slot` (none if out of range)
template <int K>
__device__ __forceinline__ Dual<K> dseed(double x, int slot) {
    Dual<K> r;
    r.v = x;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (k == slot) ? 1.0 : 0.0;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator+(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator-(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator-(const Dual<K>& a) {
    Dual<K> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator/(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator+(const Dual<K>& a, double b) {
    Dual<K> r = a;
    r.v += b;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator+(double a, const Dual<K>& b) {
    return b + a;
}
template <int K>
__device__ __forceinline__ Dual<K> operator-(const Dual<K>& a, double b) {
    Dual<K> r = a;
    r.v -= b;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator-(double a, const Dual<K>& b) {
    return -b + a;
}
template <int K>
__device__ __forceinline__ Dual<K> operator*(const Dual<K>& a, double b) {
    Dual<K> r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator*(double a, const Dual<K>& b) {
    return b * a;
}
template <int K>
__device__ __forceinline__ Dual<K> operator/(const Dual<K>& a, double b) {
    Dual<K> r;
    r.v = a.v / b;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] / b;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator/(double a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -r.v * b.d[k] / b.v;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> dsqrt(const Dual<K>& a) {
    Dual<K> r;
    r.v = sqrt(a.v);
    const double h = 0.5 / r.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * h;
    return r;
}
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
template <int K>
__device__ __forceinline__ double val(const Dual<K>& a) {
    return a.v;
}
__device__ __forceinline__ double val(double a) { return a; }

// ---------------------------------------------------------------------------
// Element tables and settings
// ---------------------------------------------------------------------------
struct AdjConst {
    double shp[4][4];   // shp[q][n] at the 4-point rule (symtet.c, uniformP.c:22-40)
    double Qwt;         // (1/4) * (4/3) (genint.f90:85)
    double SN[4];       // sum_q shp[q][n]
    double shpb[3][4];  // boundary 3-point rule
    double Qwtb;
};

struct AdjParams {
    double rho, Dtgl, dtsfct, taucfct, stabflux;
    int idiff;
};

static AdjConst make_adj_consts() {
    const double A4 = 0.5854101966249685, B4 = 0.1381966011250150;
    const double rstw4[4][3] = {{A4, B4, B4}, {B4, A4, B4}, {B4, B4, A4}, {B4, B4, B4}};
    AdjConst k{};
    for (int q = 0; q < 4; ++q) {
        k.shp[q][0] = rstw4[q][0];
        k.shp[q][1] = rstw4[q][1];
        k.shp[q][2] = rstw4[q][2];
        k.shp[q][3] = 1.0e0 - rstw4[q][0] - rstw4[q][1] - rstw4[q][2];
    }
    k.Qwt = (4.0 / 3.0) * 0.25;
    for (int a = 0; a < 4; ++a) {
        k.SN[a] = 0.0;
        for (int q = 0; q < 4; ++q) k.SN[a] += k.shp[q][a];
    }
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

// e3metric for a linear tet (e3metric.f90:26-81): dxidx, shg = dN/dx, WdetJ
__device__ __forceinline__ void adj_metric(const double xl[4][3], double Qwt, double dxidx[3][3], double shg[4][3],
                                           double* WdetJ) {
    double d[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) d[i][j] = 0.5 * xl[j][i] - 0.5 * xl[3][i];
    dxidx[0][0] = d[1][1] * d[2][2] - d[2][1] * d[1][2];
    dxidx[0][1] = d[2][1] * d[0][2] - d[0][1] * d[2][2];
    dxidx[0][2] = d[0][1] * d[1][2] - d[0][2] * d[1][1];
    const double tmp = 1.0 / (dxidx[0][0] * d[0][0] + dxidx[0][1] * d[1][0] + dxidx[0][2] * d[2][0]);
    dxidx[0][0] *= tmp;
    dxidx[0][1] *= tmp;
    dxidx[0][2] *= tmp;
    dxidx[1][0] = (d[1][2] * d[2][0] - d[1][0] * d[2][2]) * tmp;
    dxidx[1][1] = (d[0][0] * d[2][2] - d[2][0] * d[0][2]) * tmp;
    dxidx[1][2] = (d[1][0] * d[0][2] - d[0][0] * d[1][2]) * tmp;
    dxidx[2][0] = (d[1][0] * d[2][1] - d[1][1] * d[2][0]) * tmp;
    dxidx[2][1] = (d[2][0] * d[0][1] - d[0][0] * d[2][1]) * tmp;
    dxidx[2][2] = (d[0][0] * d[1][1] - d[0][1] * d[1][0]) * tmp;
    *WdetJ = Qwt / tmp;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        shg[0][k] = 0.5 * dxidx[0][k];
        shg[1][k] = 0.5 * dxidx[1][k];
        shg[2][k] = 0.5 * dxidx[2][k];
        shg[3][k] = -0.5 * dxidx[0][k] - 0.5 * dxidx[1][k] - 0.5 * dxidx[2][k];
    }
}

// e3gijd, tet branch (e3stab.f90:487-528)
__device__ __forceinline__ void adj_gijd(const double dx[3][3], double g[6]) {
    const double c1 = 1.259921049894873e+00;
    const double c2 = 6.299605249474365e-01;
    double t1, t2, t3;
    t1 = c1 * dx[0][0] + c2 * (dx[1][0] + dx[2][0]);
    t2 = c1 * dx[1][0] + c2 * (dx[0][0] + dx[2][0]);
    t3 = c1 * dx[2][0] + c2 * (dx[0][0] + dx[1][0]);
    g[0] = dx[0][0] * t1 + dx[1][0] * t2 + dx[2][0] * t3;
    t1 = c1 * dx[0][1] + c2 * (dx[1][1] + dx[2][1]);
    t2 = c1 * dx[1][1] + c2 * (dx[0][1] + dx[2][1]);
    t3 = c1 * dx[2][1] + c2 * (dx[0][1] + dx[1][1]);
    g[1] = dx[0][1] * t1 + dx[1][1] * t2 + dx[2][1] * t3;
    g[3] = dx[0][0] * t1 + dx[1][0] * t2 + dx[2][0] * t3;
    t1 = c1 * dx[0][2] + c2 * (dx[1][2] + dx[2][2]);
    t2 = c1 * dx[1][2] + c2 * (dx[0][2] + dx[2][2]);
    t3 = c1 * dx[2][2] + c2 * (dx[0][2] + dx[1][2]);
    g[2] = dx[0][2] * t1 + dx[1][2] * t2 + dx[2][2] * t3;
    g[4] = dx[0][1] * t1 + dx[1][1] * t2 + dx[2][1] * t3;
    g[5] = dx[0][0] * t1 + dx[1][0] * t2 + dx[2][0] * t3;
}

// ---------------------------------------------------------------------------
// Interior residual of one tet contracted with lambda:
//   sum_a lambda_a . rl_a, rl as e3_elem forms it (itau = 0, iconvflow = 2,
//   no body force, no ALE, flmpr = 0).  yl[n] = (p, u, v, w); acl[n] = (ax,
//   ay, az); lam[n] = (momentum x, y, z, continuity) rows of node n.
// ---------------------------------------------------------------------------
template <typename T>
__device__ T e3_res_dot(const AdjConst& C, const AdjParams& P, const double shg[4][3], double W, const double gijd[6],
                        const T yl[4][4], const T acl[4][3], const T divqi[3], const T& mu, const double lam[4][4]) {
    const double rho = P.rho;
    const double rhoinv = 1.0 / rho;
    T g[3][4];  // g[k][d] = d yl(:, d) / d x_k
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int d = 0; d < 4; ++d)
            g[k][d] = shg[0][k] * yl[0][d] + shg[1][k] * yl[1][d] + shg[2][k] * yl[2][d] + shg[3][k] * yl[3][d];
    const T rnu = mu * rhoinv;
    const double dts = P.Dtgl * P.dtsfct;
    const double gg = gijd[0] * gijd[0] + gijd[1] * gijd[1] + gijd[2] * gijd[2] +
                      2.0 * (gijd[3] * gijd[3] + gijd[4] * gijd[4] + gijd[5] * gijd[5]);
    const T visc = 36.0 * (rnu * rnu) * gg;
    const double ff = P.taucfct / P.dtsfct;
    const double trG = gijd[0] + gijd[1] + gijd[2];
    const T divu = g[0][1] + g[1][2] + g[2][3];
    T acc = 0.0 * rnu;
    for (int q = 0; q < 4; ++q) {
        const double* N = C.shp[q];
        const T pres = N[0] * yl[0][0] + N[1] * yl[1][0] + N[2] * yl[2][0] + N[3] * yl[3][0];
        T u[3], ac[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            u[i] = N[0] * yl[0][i + 1] + N[1] * yl[1][i + 1] + N[2] * yl[2][i + 1] + N[3] * yl[3][i + 1];
            ac[i] = N[0] * acl[0][i] + N[1] * acl[1][i] + N[2] * acl[2][i] + N[3] * acl[3][i];
        }
        T rL[3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
            rL[i] = (ac[i] + u[0] * g[0][i + 1] + u[1] * g[1][i + 1] + u[2] * g[2][i + 1]) * rho + g[i][0] - divqi[i];
        const T uGu = u[0] * (gijd[0] * u[0] + gijd[3] * u[1] + gijd[5] * u[2]) +
                      u[1] * (gijd[3] * u[0] + gijd[1] * u[1] + gijd[4] * u[2]) +
                      u[2] * (gijd[5] * u[0] + gijd[4] * u[1] + gijd[2] * u[2]);
        const T fact = dsqrt((2.0 * dts) * (2.0 * dts) + uGu + visc);
        const T tauC = rho * 0.125 * fact / trG * ff;
        const T tauM = 1.0 / fact;
        T tauBar = rL[0] * (gijd[0] * rL[0] + gijd[3] * rL[1] + gijd[5] * rL[2]) +
                   rL[1] * (gijd[3] * rL[0] + gijd[1] * rL[1] + gijd[4] * rL[2]) +
                   rL[2] * (gijd[5] * rL[0] + gijd[4] * rL[1] + gijd[2] * rL[2]);
        if (val(tauBar) != 0.0) tauBar = tauM / dsqrt(tauBar);
        T uB[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) uB[i] = u[i] - tauM * rL[i] * rhoinv;
        const T tmp = tauC * divu - pres;
        T rNa[3], rG[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            rNa[i] = (ac[i] + uB[0] * g[0][i + 1] + uB[1] * g[1][i + 1] + uB[2] * g[2][i + 1]) * rho;
            const T tb = tauBar * (rL[0] * g[0][i + 1] + rL[1] * g[1][i + 1] + rL[2] * g[2][i + 1]);
            const T tm = tauM * rL[i];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                rG[i][j] = mu * (g[j][i + 1] + g[i][j + 1]) + tm * u[j] + tb * rL[j];
                if (i == j) rG[i][j] = rG[i][j] + tmp;
            }
        }
        // rl(a, 4) += W dN_a . uBar ; rl(a, i) -= W (N_a rNa_i + dN_a . rGNa_i)
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            T c = (shg[a][0] * uB[0] + shg[a][1] * uB[1] + shg[a][2] * uB[2]) * (W * lam[a][3]);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const T ri = N[a] * rNa[i] + shg[a][0] * rG[i][0] + shg[a][1] * rG[i][1] + shg[a][2] * rG[i][2];
                c = c - ri * (W * lam[a][i]);
            }
            acc = acc + c;
        }
    }
    return acc;
}

// Boundary residual of one face contracted with lambda (e3b/e3bvar rigid
// wall, as k_asbmfg forms it).  Nodes 0..2 on the face, node 3 interior.
template <typename T>
__device__ T e3b_res_dot(const AdjConst& C, const AdjParams& P, const double shg[4][3], const double bn[3],
                         double WdetJb, int bits, const double* bcb, const T yl[4][4], const T& mu,
                         const double lam[3][4]) {
    T g[3][4];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int d = 0; d < 4; ++d)
            g[k][d] = shg[0][k] * yl[0][d] + shg[1][k] * yl[1][d] + shg[2][k] * yl[2][d] + shg[3][k] * yl[3][d];
    T tau[3];
    tau[0] = bn[0] * 2.0 * mu * g[0][1] + bn[1] * (mu * (g[1][1] + g[0][2])) + bn[2] * (mu * (g[2][1] + g[0][3]));
    tau[1] = bn[0] * (mu * (g[1][1] + g[0][2])) + bn[1] * 2.0 * mu * g[1][2] + bn[2] * (mu * (g[2][2] + g[1][3]));
    tau[2] = bn[0] * (mu * (g[2][1] + g[0][3])) + bn[1] * (mu * (g[2][2] + g[1][3])) + bn[2] * 2.0 * mu * g[2][3];
    const T tn = bn[0] * tau[0] + bn[1] * tau[1] + bn[2] * tau[2];
    T acc = 0.0 * mu;
    for (int q = 0; q < 3; ++q) {
        const double* Nb = C.shpb[q];
        T pres = Nb[0] * yl[0][0] + Nb[1] * yl[1][0] + Nb[2] * yl[2][0];
        T u[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) u[i] = Nb[0] * yl[0][i + 1] + Nb[1] * yl[1][i + 1] + Nb[2] * yl[2][i + 1];
        T unm = bn[0] * u[0] + bn[1] * u[1] + bn[2] * u[2];
        pres = pres - tn;
        T tt[3] = {tau[0] - bn[0] * tn, tau[1] - bn[1] * tn, tau[2] - bn[2] * tn};
        T unm_copy = 0.0 * unm;
        if ((bits >> 1) & 1)
            if (val(unm) < 0.0) unm_copy = unm;
        if (bits & 1) {
            double s = 0.0;
            for (int n = 0; n < 3; ++n) s += Nb[n] * bcb[6 * n + 0];
            unm = 0.0 * unm + s;
        }
        if ((bits >> 1) & 1) {
            double s = 0.0;
            for (int n = 0; n < 3; ++n) s += Nb[n] * bcb[6 * n + 1];
            pres = 0.0 * pres + s;
        }
        if ((bits >> 2) & 1) {
            double s[3] = {0.0, 0.0, 0.0};
            for (int n = 0; n < 3; ++n) {
                s[0] += Nb[n] * bcb[6 * n + 2];
                s[1] += Nb[n] * bcb[6 * n + 3];
                s[2] += Nb[n] * bcb[6 * n + 4];
            }
            for (int i = 0; i < 3; ++i) tt[i] = 0.0 * tt[i] + s[i];
        }
        if ((bits >> 4) & 1) {
            pres = 0.0 * pres;
            for (int i = 0; i < 3; ++i) tt[i] = 0.0 * tt[i];
        }
        const T rou_copy = P.rho * unm_copy;
        T rNa[4];
#pragma unroll
        for (int i = 0; i < 3; ++i) rNa[i] = (bn[i] * pres - tt[i] - P.stabflux * rou_copy * u[i]) * WdetJb;
        rNa[3] = unm * WdetJb;
#pragma unroll
        for (int n = 0; n < 3; ++n)
#pragma unroll
            for (int d = 0; d < 4; ++d) acc = acc - rNa[d] * (Nb[n] * lam[n][d]);
    }
    return acc;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
constexpr int kAdjK = 8;  // derivative directions per pass

// lambda with the rows bc3Res zeroes set to zero (node-major (4, n))
__global__ void k_adj_mask(const int* __restrict__ iBC, const double* __restrict__ lam, double* __restrict__ out,
                           int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int b = iBC[i];
        const double* l = lam + 4 * (size_t)i;
        double* o = out + 4 * (size_t)i;
        const bool vel = ((b >> 3) & 7) == 7 || ((b >> 11) & 1);
        o[0] = vel ? 0.0 : l[0];
        o[1] = vel ? 0.0 : l[1];
        o[2] = vel ? 0.0 : l[2];
        o[3] = ((b >> 2) & 1) ? 0.0 : l[3];
    }
}

__device__ __forceinline__ void warp_atomic_add(double v, double* dst) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(dst, v);
}

// Interior VJP: one thread per tet, all 32 local directions in 32/K passes.
// Directions: 0..15 y (node n = k/4, dof (p,u,v,w) = k%4), 16..27 ac
// (node (k-16)/3, comp (k-16)%3), 28..30 div q, 31 mu.
__global__ void __launch_bounds__(64) k_adj_interior(const int4* __restrict__ ien, const double4* __restrict__ x,
                                                     const double4* __restrict__ y, const double4* __restrict__ ac,
                                                     const double* __restrict__ qres, const double4* __restrict__ lam,
                                                     int nelem, AdjConst C, AdjParams P, double mu,
                                                     double* __restrict__ ybar, double* __restrict__ abar,
                                                     double* __restrict__ qbar, double* __restrict__ mubar) {
    using D = Dual<kAdjK>;
    double mub = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
        const int4 nn = ien[e];
        const int nd[4] = {nn.x, nn.y, nn.z, nn.w};
        double xl[4][3], yv[4][4], av[4][3], lm[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double4 xx = x[nd[a]];
            const double4 yy = y[nd[a]];
            const double4 aa = ac[nd[a]];
            const double4 ll = lam[nd[a]];
            xl[a][0] = xx.x;
            xl[a][1] = xx.y;
            xl[a][2] = xx.z;
            yv[a][0] = yy.w;
            yv[a][1] = yy.x;
            yv[a][2] = yy.y;
            yv[a][3] = yy.z;
            av[a][0] = aa.x;
            av[a][1] = aa.y;
            av[a][2] = aa.z;
            lm[a][0] = ll.x;
            lm[a][1] = ll.y;
            lm[a][2] = ll.z;
            lm[a][3] = ll.w;
        }
        double dxidx[3][3], shg[4][3], W, gijd[6];
        adj_metric(xl, C.Qwt, dxidx, shg, &W);
        adj_gijd(dxidx, gijd);
        double dq[3] = {0.0, 0.0, 0.0};
        if (P.idiff >= 1) {
            for (int a = 0; a < 4; ++a) {
                const double* q = qres + 9 * (size_t)nd[a];
                for (int i = 0; i < 3; ++i) dq[i] += shg[a][0] * q[i] + shg[a][1] * q[i + 3] + shg[a][2] * q[i + 6];
            }
        }
        for (int pass = 0; pass < 32 / kAdjK; ++pass) {
            const int base = pass * kAdjK;
            D yl[4][4], acl[4][3], dqi[3];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
#pragma unroll
                for (int d = 0; d < 4; ++d) yl[a][d] = dseed<kAdjK>(yv[a][d], 4 * a + d - base);
#pragma unroll
                for (int i = 0; i < 3; ++i) acl[a][i] = dseed<kAdjK>(av[a][i], 16 + 3 * a + i - base);
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) dqi[i] = dseed<kAdjK>(dq[i], 28 + i - base);
            const D m = dseed<kAdjK>(mu, 31 - base);
            const D r = e3_res_dot(C, P, shg, W, gijd, yl, acl, dqi, m, lm);
#pragma unroll
            for (int k = 0; k < kAdjK; ++k) {
                const int dir = base + k;
                const double v = r.d[k];
                if (v == 0.0) continue;
                if (dir < 16) {
                    const int a = dir / 4, d = dir % 4;
                    atomicAdd(ybar + 4 * (size_t)nd[a] + (d == 0 ? 3 : d - 1), v);
                } else if (dir < 28) {
                    const int a = (dir - 16) / 3, i = (dir - 16) % 3;
                    atomicAdd(abar + 4 * (size_t)nd[a] + i, v);
                } else if (dir < 31) {
                    // div q_i = sum_a sum_j dN_a,j q_a(i + 3j)
                    const int i = dir - 28;
                    for (int a = 0; a < 4; ++a)
                        for (int j = 0; j < 3; ++j) atomicAdd(qbar + 9 * (size_t)nd[a] + i + 3 * j, shg[a][j] * v);
                } else {
                    mub += v;
                }
            }
        }
    }
    warp_atomic_add(mub, mubar);
}

// Transposed lumped projection (AsIq + qpbc): qres_a = (sum_e W SN_a qdi_e) /
// rmass_a with qdi = mu (grad u + grad u^T); given qbar, add its cotangent to
// u and mu.  rinv = 1 / rmass (as qpbc leaves it).
__global__ void __launch_bounds__(128) k_adj_asiq(const int4* __restrict__ ien, const double4* __restrict__ x,
                                                  const double4* __restrict__ y, const double* __restrict__ qbar,
                                                  const double* __restrict__ rinv, int nelem, AdjConst C, double mu,
                                                  double* __restrict__ ybar, double* __restrict__ mubar) {
    double mub = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
        const int4 nn = ien[e];
        const int nd[4] = {nn.x, nn.y, nn.z, nn.w};
        double xl[4][3], ul[4][3];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double4 xx = x[nd[a]];
            const double4 yy = y[nd[a]];
            xl[a][0] = xx.x;
            xl[a][1] = xx.y;
            xl[a][2] = xx.z;
            ul[a][0] = yy.x;
            ul[a][1] = yy.y;
            ul[a][2] = yy.z;
        }
        double dxidx[3][3], shg[4][3], W;
        adj_metric(xl, C.Qwt, dxidx, shg, &W);
        double qb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double w = W * C.SN[a] * rinv[nd[a]];
            const double* q = qbar + 9 * (size_t)nd[a];
#pragma unroll
            for (int k = 0; k < 9; ++k) qb[k] += w * q[k];
        }
        double g[3][3];  // g[k][i] = d u_i / d x_k
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i)
                g[k][i] = shg[0][k] * ul[0][i] + shg[1][k] * ul[1][i] + shg[2][k] * ul[2][i] + shg[3][k] * ul[3][i];
        // qdi / mu for the mu cotangent
        const double s[9] = {2.0 * g[0][0], g[0][1] + g[1][0], g[0][2] + g[2][0], g[0][1] + g[1][0], 2.0 * g[1][1],
                             g[1][2] + g[2][1], g[0][2] + g[2][0], g[1][2] + g[2][1], 2.0 * g[2][2]};
#pragma unroll
        for (int k = 0; k < 9; ++k) mub += qb[k] * s[k];
        // cotangent of g[k][i]
        double gb[3][3];
        gb[0][0] = 2.0 * mu * qb[0];
        gb[1][1] = 2.0 * mu * qb[4];
        gb[2][2] = 2.0 * mu * qb[8];
        gb[0][1] = gb[1][0] = mu * (qb[1] + qb[3]);
        gb[0][2] = gb[2][0] = mu * (qb[2] + qb[6]);
        gb[1][2] = gb[2][1] = mu * (qb[5] + qb[7]);
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const double v = shg[b][0] * gb[0][i] + shg[b][1] * gb[1][i] + shg[b][2] * gb[2][i];
                atomicAdd(ybar + 4 * (size_t)nd[b] + i, v);
            }
    }
    warp_atomic_add(mub, mubar);
}

// Boundary-face VJP: 17 local directions (16 y + mu) in 3 passes.
__global__ void __launch_bounds__(64) k_adj_faces(const int4* __restrict__ ienb, const int* __restrict__ iBCB,
                                                  const double* __restrict__ BCB, const double4* __restrict__ x,
                                                  const double4* __restrict__ y, const double4* __restrict__ lam,
                                                  int nface, AdjConst C, AdjParams P, double mu,
                                                  double* __restrict__ ybar, double* __restrict__ mubar) {
    using D = Dual<kAdjK>;
    double mub = 0.0;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nface; f += gridDim.x * blockDim.x) {
        const int4 nn = ienb[f];
        const int nd[4] = {nn.x, nn.y, nn.z, nn.w};
        double xl[4][3], yv[4][4], lm[3][4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double4 xx = x[nd[a]];
            const double4 yy = y[nd[a]];
            xl[a][0] = xx.x;
            xl[a][1] = xx.y;
            xl[a][2] = xx.z;
            yv[a][0] = yy.w;
            yv[a][1] = yy.x;
            yv[a][2] = yy.y;
            yv[a][3] = yy.z;
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double4 ll = lam[nd[a]];
            lm[a][0] = ll.x;
            lm[a][1] = ll.y;
            lm[a][2] = ll.z;
            lm[a][3] = ll.w;
        }
        const int bits = iBCB[f];
        const double* bcb = BCB + 18 * (size_t)f;
        double dxidx[3][3], shg[4][3], Wtmp;
        adj_metric(xl, C.Qwt, dxidx, shg, &Wtmp);
        double v1[3], v2[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            v1[i] = xl[1][i] - xl[0][i];
            v2[i] = xl[2][i] - xl[0][i];
        }
        const double t1 = v1[1] * v2[2] - v2[1] * v1[2];
        const double t2 = v2[0] * v1[2] - v1[0] * v2[2];
        const double t3 = v1[0] * v2[1] - v2[0] * v1[1];
        const double temp = 1.0 / sqrt(t1 * t1 + t2 * t2 + t3 * t3);
        const double bn[3] = {t1 * temp, t2 * temp, t3 * temp};
        const double WdetJb = C.Qwtb / (4.0 * temp);
        for (int pass = 0; pass < 3; ++pass) {
            const int base = pass * kAdjK;
            D yl[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int d = 0; d < 4; ++d) yl[a][d] = dseed<kAdjK>(yv[a][d], 4 * a + d - base);
            const D m = dseed<kAdjK>(mu, 16 - base);
            const D r = e3b_res_dot(C, P, shg, bn, WdetJb, bits, bcb, yl, m, lm);
#pragma unroll
            for (int k = 0; k < kAdjK; ++k) {
                const int dir = base + k;
                const double v = r.d[k];
                if (v == 0.0 || dir > 16) continue;
                if (dir < 16) {
                    const int a = dir / 4, d = dir % 4;
                    atomicAdd(ybar + 4 * (size_t)nd[a] + (d == 0 ? 3 : d - 1), v);
                } else {
                    mub += v;
                }
            }
        }
    }
    warp_atomic_add(mub, mubar);
}

// s_k = sum over outlet k's nodes of NABI . v (v = y or lambda), fixed order
__global__ void k_adj_flow(const int* __restrict__ onodes, const int* __restrict__ off,
                           const double4* __restrict__ onabi, const double4* __restrict__ v, double* __restrict__ s) {
    __shared__ double sm[32];
    const int k = blockIdx.x;
    double t = 0.0;
    for (int j = off[k] + threadIdx.x; j < off[k + 1]; j += blockDim.x) {
        const double4 nb = onabi[j];
        const double4 vv = v[onodes[j]];
        t += nb.x * vv.x + nb.y * vv.y + nb.z * vv.z;
    }
    t = block_sum(t, sm);
    if (threadIdx.x == 0) s[k] = t;
}

// ybar(vel) -= coef1_k s_k NABI over outlet k's nodes (d p_k / d u)
__global__ void k_adj_pvsq(const int* __restrict__ onodes, const int* __restrict__ off,
                           const double4* __restrict__ onabi, const double* __restrict__ s,
                           const double* __restrict__ coef1, int ncoupled, double* __restrict__ ybar) {
    const int k = blockIdx.y;
    const double f = -coef1[k] * s[k];
    for (int j = off[k] + blockIdx.x * blockDim.x + threadIdx.x; j < off[k + 1]; j += gridDim.x * blockDim.x) {
        const double4 nb = onabi[j];
        double* r = ybar + 4 * (size_t)onodes[j];
        atomicAdd(r + 0, f * nb.x);
        atomicAdd(r + 1, f * nb.y);
        atomicAdd(r + 2, f * nb.z);
    }
}

int elmgmr_vjp(crimson_ctx* c, const double* d_y, const double* d_ac, const double* coef1, const double* coef2,
               const double* d_lam, double* d_res, double* d_ybar, double* d_abar, double* mubar, double* c1bar,
               double* c2bar) {
    cudaStream_t s = c->stream;
    const int n = c->nshg;
    const crimson_params& p = c->p;
    // primal residual at (y, ac): also leaves qres and 1/rmass in the context
    CR_CHECK(c->adj_res.alloc(4 * (size_t)n));
    CR_CHECK(elmgmr_device(c, d_y, d_ac, coef1, coef2, d_res ? d_res : c->adj_res.p, nullptr, nullptr, 0));
    CR_CHECK(c->adj_lam.alloc(4 * (size_t)n));
    CR_CHECK(c->adj_qbar.alloc(9 * (size_t)n));
    CR_CHECK(c->adj_scal.alloc(4 + 2 * (size_t)std::max(c->ncoupled, 1)));
    CR_CUDA(cudaMemsetAsync(d_ybar, 0, sizeof(double) * 4 * (size_t)n, s));
    CR_CUDA(cudaMemsetAsync(d_abar, 0, sizeof(double) * 4 * (size_t)n, s));
    CR_CUDA(cudaMemsetAsync(c->adj_qbar.p, 0, sizeof(double) * 9 * (size_t)n, s));
    CR_CUDA(cudaMemsetAsync(c->adj_scal.p, 0, sizeof(double) * c->adj_scal.n, s));
    launch(k_adj_mask, grid_for(n, 256), 256, 0, s, (const int*)c->iBC.p, d_lam, c->adj_lam.p, n);
    const AdjConst C = make_adj_consts();
    AdjParams P;
    P.rho = p.rho;
    P.Dtgl = p.Dtgl;
    P.dtsfct = p.dtsfct;
    P.taucfct = p.taucfct;
    P.stabflux = p.stabflux_coeff;
    P.idiff = p.idiff;
    const double4* x4 = c->x.p;
    const double4* y4 = reinterpret_cast<const double4*>(d_y);
    const double4* a4 = reinterpret_cast<const double4*>(d_ac);
    const double4* l4 = reinterpret_cast<const double4*>(c->adj_lam.p);
    double* mub = c->adj_scal.p;
    launch(k_adj_interior, grid_for(c->nelem, 64, 16), 64, 0, s, (const int4*)c->ien.p, x4, y4, a4,
           (const double*)c->qres.p, l4, c->nelem, C, P, p.mu, d_ybar, d_abar, c->adj_qbar.p, mub);
    if (p.idiff == 1)
        launch(k_adj_asiq, grid_for(c->nelem, 128, 16), 128, 0, s, (const int4*)c->ien.p, x4, y4,
               (const double*)c->adj_qbar.p, (const double*)c->rmass.p, c->nelem, C, p.mu, d_ybar, mub);
    if (c->nface > 0)
        launch(k_adj_faces, grid_for(c->nface, 64, 16), 64, 0, s, (const int4*)c->ienb.p, (const int*)c->iBCB.p,
               (const double*)c->BCB.p, x4, y4, l4, c->nface, C, P, p.mu, d_ybar, mub);
    const int nc = c->ncoupled;
    std::vector<double> hs(2 * (size_t)std::max(nc, 1), 0.0);
    if (nc > 0) {
        const int* doff = c->d_onode_off.p;
        DBuf<double> dc1;
        std::vector<double> h1(nc);
        for (int k = 0; k < nc; ++k) h1[k] = coef1 ? coef1[k] : 0.0;
        CR_CHECK(dc1.upload(h1.data(), nc, s));
        double* sl = c->adj_scal.p + 4;        // s_k = lambda . NABI
        double* qf = c->adj_scal.p + 4 + nc;   // Q_k = y . NABI
        launch(k_adj_flow, nc, 256, 0, s, (const int*)c->onodes.p, doff, (const double4*)c->onabi.p, l4,
               sl);
        launch(k_adj_flow, nc, 256, 0, s, (const int*)c->onodes.p, doff, (const double4*)c->onabi.p, y4,
               qf);
        launch(k_adj_pvsq, dim3(8, nc), 256, 0, s, (const int*)c->onodes.p, doff,
               (const double4*)c->onabi.p, (const double*)sl, (const double*)dc1.p, nc, d_ybar);
        CR_CUDA(cudaMemcpyAsync(hs.data(), sl, sizeof(double) * 2 * nc, cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));  // dc1 is released at scope exit
    }
    double hm = 0.0;
    CR_CUDA(cudaMemcpyAsync(&hm, mub, sizeof(double), cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    CR_CUDA(cudaGetLastError());
    if (mubar) *mubar = hm;
    for (int k = 0; k < nc; ++k) {
        // p_k = -(Q_k coef1_k) - coef2_k; res(vel) += p_k NABI
        if (c1bar) c1bar[k] = -hs[nc + k] * hs[k];
        if (c2bar) c2bar[k] = -hs[k];
    }
    return CRIMSON_OK;
}

}  // namespace crimson
