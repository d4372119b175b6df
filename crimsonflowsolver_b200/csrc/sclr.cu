// ElmGMRSclr on the device (flowsolver/src/elmgmr.f90:599-822): residual and
// tangent of the advection-diffusion equation of one scalar, assembled with
// the same deterministic owner-computes scheme as ElmGMR.
//
//   k_sclr_q      AsIqSclr / e3qSclr (asiq.f90:89-125, e3q.f90:215-300) per
//                 element: q = diffus grad S and W, the same at every point
//   k_sclr_qnode  per node: the lumped-projection contributions of q and of
//                 the lumped mass of the elements containing it, then
//                 qpbcSclr (qpbc.f90:118-175): qres = q / rmass
//   k_sclr_elem   AsIGMRSclr / e3Sclr (asigmr.f90:141-190, e3.f90:183-330):
//                 per element the residual rows rl(a) and the 4x4 tangent
//                 xSebe (e3ivarSclr, e3StabSclr, e3ResSclr, e3LHSSclr)
//   k_sclr_face   AsBSclr / e3bSclr (asbmfg.f90:114-150, e3b.f90:626-720):
//                 the boundary flux term of each face node
//   k_sclr_node   per node: residual row (elements, then faces) and the
//                 diagonal tangent entry; bc3ResSclr (bc3res.f90:138-160)
//   k_sclr_slot   per off-diagonal CSR entry: fillsparseSclr's sum
//                 (fillsparse.f90:167-200) in ascending element order
//
// The node passes give each node kNodeLanes lanes and combine their sums in
// a fixed order; the slot pass sums each entry's short list in element
// order.  Every result is bitwise repeatable.
//
// Settings as the reference's defaults for a passive scalar: diffusivity
// scdiff(isclr) (getdiff.f90:145-174), the flow velocity as convection
// velocity (consrv_sclr_conv_vel = 0), SUPG (ivart = 2), no discontinuity
// capturing (idcsclr = 0), no source terms (nosource = 1: with nosource = 0
// the reference reads uninitialised source arrays, its source call being
// commented out, e3ivar.f90:670-680), Navier = 1, linear tets.
#include "common.cuh"

namespace crimson {

int build_pattern(crimson_ctx* c);

namespace {

// Quadrature tables built on the host with the oracle's arithmetic
// (symtet.c / genint.f90:85 interior rule, symtri.c through genshpb.f90
// boundary rule, shape gradients halved as genshp.f90:35-36).
struct SclrTables {
    double shp[4][4];    // [intp][n]
    double M[4][4];      // sum over the points of shp[q][a] shp[q][b]
    double shgl[3][4];   // [dir][n], the same at every point of a linear tet
    double Qwt[4];
    double shpb[3][4];   // boundary points
    double Qwtb[3];
};

SclrTables sclr_tables() {
    SclrTables t;
    const double A4 = 0.5854101966249685, B4 = 0.1381966011250150;
    const double r4[4][3] = {{A4, B4, B4}, {B4, A4, B4}, {B4, B4, A4}, {B4, B4, B4}};
    for (int q = 0; q < 4; ++q) {
        t.shp[q][0] = r4[q][0];
        t.shp[q][1] = r4[q][1];
        t.shp[q][2] = r4[q][2];
        t.shp[q][3] = 1.0e0 - r4[q][0] - r4[q][1] - r4[q][2];
        t.Qwt[q] = (4.0 / 3.0) * 0.25;
    }
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
            t.M[a][b] = 0.0;
            for (int q = 0; q < 4; ++q) t.M[a][b] += t.shp[q][a] * t.shp[q][b];
        }
    for (int j = 0; j < 3; ++j)
        for (int n = 0; n < 4; ++n) t.shgl[j][n] = (n == 3 ? -1.0e0 : (n == j ? 1.0e0 : 0.0e0)) / 2.0;
    const double B3 = 0.666666666666667, C3 = 0.166666666666667, A3 = 0.3333333333333330000000000000000000;
    const double r3[3][3] = {{B3, C3, C3}, {C3, B3, C3}, {C3, C3, B3}};
    for (int q = 0; q < 3; ++q) {
        t.shpb[q][0] = r3[q][0];
        t.shpb[q][1] = r3[q][1];
        t.shpb[q][2] = r3[q][2];
        t.shpb[q][3] = 1.0e0 - r3[q][0] - r3[q][1] - r3[q][2];
        t.Qwtb[q] = 2.0 * A3;
    }
    // the kernels rely on equal weights per rule (metric and W hoisted out
    // of the quadrature loops)
    return t;
}

struct SclrParams {
    double alfi, almi, gami, Delt, Dtgl, dtsfct, diffus;
    int idiff, isclr, lhs;
};

// e3metric (e3metric.f90:26-81) for a linear tet
__device__ __forceinline__ void sclr_metric(const double xl[4][3], const double shgl[3][4], double Qwt,
                                            double dxidx[3][3], double shg[4][3], double* W) {
    double d[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) d[i][j] = d[i][j] + xl[n][i] * shgl[j][n];
    dxidx[0][0] = d[1][1] * d[2][2] - d[2][1] * d[1][2];
    dxidx[0][1] = d[2][1] * d[0][2] - d[0][1] * d[2][2];
    dxidx[0][2] = d[0][1] * d[1][2] - d[0][2] * d[1][1];
    const double tmp = 1.0 / (dxidx[0][0] * d[0][0] + dxidx[0][1] * d[1][0] + dxidx[0][2] * d[2][0]);
    dxidx[0][0] = dxidx[0][0] * tmp;
    dxidx[0][1] = dxidx[0][1] * tmp;
    dxidx[0][2] = dxidx[0][2] * tmp;
    dxidx[1][0] = (d[1][2] * d[2][0] - d[1][0] * d[2][2]) * tmp;
    dxidx[1][1] = (d[0][0] * d[2][2] - d[2][0] * d[0][2]) * tmp;
    dxidx[1][2] = (d[1][0] * d[0][2] - d[0][0] * d[1][2]) * tmp;
    dxidx[2][0] = (d[1][0] * d[2][1] - d[1][1] * d[2][0]) * tmp;
    dxidx[2][1] = (d[2][0] * d[0][1] - d[0][0] * d[2][1]) * tmp;
    dxidx[2][2] = (d[0][0] * d[1][1] - d[0][1] * d[1][0]) * tmp;
    *W = Qwt / tmp;
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            shg[n][k] = shgl[0][n] * dxidx[0][k] + shgl[1][n] * dxidx[1][k] + shgl[2][n] * dxidx[2][k];
}

// e3gijd, tet branch (e3stab.f90:487-528)
__device__ __forceinline__ void sclr_gijd(const double dx[3][3], double g[6]) {
    const double c1 = 1.259921049894873e+00, c2 = 6.299605249474365e-01;
    double t1 = c1 * dx[0][0] + c2 * (dx[1][0] + dx[2][0]);
    double t2 = c1 * dx[1][0] + c2 * (dx[0][0] + dx[2][0]);
    double t3 = c1 * dx[2][0] + c2 * (dx[0][0] + dx[1][0]);
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

__device__ __forceinline__ void sclr_gather_x(const int4 nn, const double4* __restrict__ x, double xl[4][3]) {
    const int nd[4] = {nn.x, nn.y, nn.z, nn.w};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const double4 v = x[nd[a]];
        xl[a][0] = v.x;
        xl[a][1] = v.y;
        xl[a][2] = v.z;
    }
}

// Offset of off-diagonal xSebe(a, b), a != b, in an element's xoff record.
__host__ __device__ __forceinline__ int sclr_off(int a, int b) { return 3 * a + (b < a ? b : b - 1); }

// Lanes per node in the node passes: the contributions of a node are split
// round-robin over kNodeLanes lanes (lane l sums entries l, l + kNodeLanes,
// ... in list order), then combined by a fixed butterfly, so every result is
// the same bit for bit on every run.
constexpr int kNodeLanes = 8;

__device__ __forceinline__ double lanes_sum(double v) {
#pragma unroll
    for (int o = kNodeLanes / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// AsIqSclr / e3qSclr per element: the point-independent part of the flux
// projection, {qdi = diffus grad S, W} (32 bytes); a linear tet's metric, W
// and grad S are the same at the 4 points.
__global__ void __launch_bounds__(128) k_sclr_q(const int4* __restrict__ ien, const double4* __restrict__ x,
                                                const double* __restrict__ s, int nelem, SclrTables T,
                                                double diffus, double4* __restrict__ qrec) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
        const int4 nn = ien[e];
        double xl[4][3];
        sclr_gather_x(nn, x, xl);
        const double sl[4] = {s[nn.x], s[nn.y], s[nn.z], s[nn.w]};
        double dxidx[3][3], shg[4][3], W;
        sclr_metric(xl, T.shgl, T.Qwt[0], dxidx, shg, &W);
        double gT[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
            for (int k = 0; k < 3; ++k) gT[k] = gT[k] + shg[n][k] * sl[n];
        qrec[e] = make_double4(diffus * gT[0], diffus * gT[1], diffus * gT[2], W);
    }
}

// Per node: the lumped-projection sums over the elements containing it (the
// contributions of its diagonal slot), each contribution
// ql(a) = sum_q N_a(q) W qdi and rmassl(a) = sum_q N_a(q) W as e3qSclr
// accumulates them, then qpbcSclr: qres = (1 / rmass) q.
__global__ void __launch_bounds__(256) k_sclr_qnode(const int* __restrict__ diag, const int* __restrict__ soff,
                                                    const int* __restrict__ slist, const double4* __restrict__ qrec,
                                                    int nshg, SclrTables T, double* __restrict__ qres) {
    constexpr int NPW = 32 / kNodeLanes;   // nodes per warp and pass
    const int lane = threadIdx.x & 31, sub = lane % kNodeLanes;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    // warp-uniform loop: the shuffles below always see all 32 lanes
    for (long long i0 = warp * NPW; i0 < nshg; i0 += nwarp * NPW) {
        const long long ig = i0 + lane / kNodeLanes;
        const bool valid = ig < nshg;
        const int i = valid ? (int)ig : nshg - 1;
        const int d = diag[i];
        double q0 = 0.0, q1 = 0.0, q2 = 0.0, m = 0.0;
        const int p1 = soff[d + 1];
        for (int p = soff[d] + sub; p < p1; p += kNodeLanes) {
            const int t = slist[p];
            const int a = (t >> 2) & 3;
            const double4 r = qrec[t >> 4];
            double ql0 = 0.0, ql1 = 0.0, ql2 = 0.0, rm = 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double sw = T.shp[q][a] * r.w;
                ql0 = ql0 + sw * r.x;
                ql1 = ql1 + sw * r.y;
                ql2 = ql2 + sw * r.z;
                rm = rm + sw;
            }
            q0 += ql0;
            q1 += ql1;
            q2 += ql2;
            m += rm;
        }
        q0 = lanes_sum(q0);
        q1 = lanes_sum(q1);
        q2 = lanes_sum(q2);
        m = lanes_sum(m);
        if (valid && sub == 0) {
            const double rinv = 1.0 / m;
            qres[3 * (size_t)i] = rinv * q0;
            qres[3 * (size_t)i + 1] = rinv * q1;
            qres[3 * (size_t)i + 2] = rinv * q2;
        }
    }
}

// e3Sclr per element.  Two records: erec (8 doubles) holds {rl(a),
// xSebe(a, a)} at 2 a, so a node's residual and diagonal entry are one
// 16-byte load and the node pass streams only these; xoff (12 doubles, with
// the tangent only) holds the off-diagonal xSebe(a, b) at sclr_off(a, b)
// for the slot pass.
__global__ void __launch_bounds__(128, 3) k_sclr_elem(const int4* __restrict__ ien, const double4* __restrict__ x,
                                                   const double4* __restrict__ y, const double* __restrict__ s,
                                                   const double* __restrict__ sdot, const double* __restrict__ qres,
                                                   int nelem, SclrTables T, SclrParams P, double* __restrict__ erec,
                                                   double* __restrict__ xoff) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += gridDim.x * blockDim.x) {
        const int4 nn = ien[e];
        const int nd[4] = {nn.x, nn.y, nn.z, nn.w};
        double xl[4][3], ul[4][3], sl[4], sdl[4], ql[4][3];
        sclr_gather_x(nn, x, xl);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double4 v = y[nd[a]];
            ul[a][0] = v.x;
            ul[a][1] = v.y;
            ul[a][2] = v.z;
            sl[a] = s[nd[a]];
            sdl[a] = sdot[nd[a]];
#pragma unroll
            for (int k = 0; k < 3; ++k) ql[a][k] = P.idiff >= 1 ? qres[3 * (size_t)nd[a] + k] : 0.0;
        }
        const double lhsFct = P.alfi * P.gami * P.Delt;
        const double dts = P.Dtgl * P.dtsfct;
        // linear tet, equal weights: metric, W, grad S, div q and g_ij are
        // the same at the 4 points
        double dxidx[3][3], shg[4][3], W;
        sclr_metric(xl, T.shgl, T.Qwt[0], dxidx, shg, &W);
        double gS[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int n = 0; n < 4; ++n)
#pragma unroll
            for (int k = 0; k < 3; ++k) gS[k] = gS[k] + shg[n][k] * sl[n];
        double divS = 0.0;
        if (P.idiff >= 1)
#pragma unroll
            for (int n = 0; n < 4; ++n)
                divS = divS + shg[n][0] * ql[n][0] + shg[n][1] * ql[n][1] + shg[n][2] * ql[n][2];
        double g[6];
        sclr_gijd(dxidx, g);
        const double tauDiff = 9.0 * (P.diffus * P.diffus) *
                               (g[0] * g[0] + g[1] * g[1] + g[2] * g[2] +
                                2.0 * (g[3] * g[3] + g[4] * g[4] + g[5] * g[5]));
        // Per point only what depends on the interpolated u and Sdot: the
        // stabilisation tauS (e3StabSclr, ivart = 2, ipord = 1, no sources)
        // and the sums it enters.  With c_a = u . grad N_a:
        //   V       = sum_q tauS rLS u           (SUPG residual flux)
        //   A(a, b) = sum_q tauS c_a N_b         (SUPG mass, e3LHSSclr's flipped term)
        //   B(a, b) = sum_q tauS c_a c_b         (SUPG convection)
        double V[3] = {0.0, 0.0, 0.0}, A[4][4], B[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) A[a][b] = B[a][b] = 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double* shp = T.shp[q];
            double u1 = 0.0, u2 = 0.0, u3 = 0.0, Sdot = 0.0;
#pragma unroll
            for (int n = 0; n < 4; ++n) {
                u1 = u1 + shp[n] * ul[n][0];
                u2 = u2 + shp[n] * ul[n][1];
                u3 = u3 + shp[n] * ul[n][2];
                Sdot = Sdot + shp[n] * sdl[n];
            }
            const double rLS = (Sdot + (u1 * gS[0] + u2 * gS[1] + u3 * gS[2])) - divS;
            const double tauT = (2.0 * dts) * (2.0 * dts) + u1 * (g[0] * u1 + g[3] * u2 + g[5] * u3) +
                                u2 * (g[3] * u1 + g[1] * u2 + g[4] * u3) + u3 * (g[5] * u1 + g[4] * u2 + g[2] * u3) +
                                tauDiff;
            const double tauS = 1.0 / sqrt(tauT);
            const double tmp = tauS * rLS;
            V[0] = V[0] + tmp * u1;
            V[1] = V[1] + tmp * u2;
            V[2] = V[2] + tmp * u3;
            if (P.lhs) {
                double c[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) c[a] = u1 * shg[a][0] + u2 * shg[a][1] + u3 * shg[a][2];
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const double tc = tauS * c[a];
#pragma unroll
                    for (int b = 0; b < 4; ++b) A[a][b] = A[a][b] + tc * shp[b];
#pragma unroll
                    for (int b = a; b < 4; ++b) B[a][b] = B[a][b] + tc * c[b];
                }
            }
        }
        // the point sums of the q-independent terms: sum_q N_a X_q = (M X)_a
        double Mu[4][3], Msd[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            Mu[a][0] = Mu[a][1] = Mu[a][2] = Msd[a] = 0.0;
#pragma unroll
            for (int n = 0; n < 4; ++n) {
                Mu[a][0] = Mu[a][0] + T.M[a][n] * ul[n][0];
                Mu[a][1] = Mu[a][1] + T.M[a][n] * ul[n][1];
                Mu[a][2] = Mu[a][2] + T.M[a][n] * ul[n][2];
                Msd[a] = Msd[a] + T.M[a][n] * sdl[n];
            }
        }
        // e3ResSclr summed over the points (flmpr = 0):
        //   rl(a) = -W [ (M Sdot)_a + (M u)_a . grad S + 4 diffus grad N_a . grad S + grad N_a . V ]
        double rl[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double gg = shg[a][0] * gS[0] + shg[a][1] * gS[1] + shg[a][2] * gS[2];
            const double gv = shg[a][0] * V[0] + shg[a][1] * V[1] + shg[a][2] * V[2];
            const double mg = Mu[a][0] * gS[0] + Mu[a][1] * gS[1] + Mu[a][2] * gS[2];
            rl[a] = -W * (Msd[a] + mg + 4.0 * P.diffus * gg + gv);
        }
        // e3LHSSclr summed over the points (flmpl = 0, no sources):
        //   xS(a, b) = almi W M_ab + lhsFct W (M u)_a . grad N_b + W A(a, b)
        //            + lhsFct W (4 diffus grad N_a . grad N_b + B(a, b))
        double xS[4][4];
        if (P.lhs) {
            const double lw = lhsFct * W, mw = P.almi * W, d4 = 4.0 * P.diffus;
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const double conv = Mu[a][0] * shg[b][0] + Mu[a][1] * shg[b][1] + Mu[a][2] * shg[b][2];
                    const double gab = shg[a][0] * shg[b][0] + shg[a][1] * shg[b][1] + shg[a][2] * shg[b][2];
                    const double bab = a <= b ? B[a][b] : B[b][a];
                    xS[a][b] = mw * T.M[a][b] + lw * conv + W * A[a][b] + lw * (d4 * gab + bab);
                }
        } else {
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) xS[a][b] = 0.0;
        }
        double4* r = reinterpret_cast<double4*>(erec + 8 * (size_t)e);
        r[0] = make_double4(rl[0], xS[0][0], rl[1], xS[1][1]);
        r[1] = make_double4(rl[2], xS[2][2], rl[3], xS[3][3]);
        if (P.lhs) {
            double4* o = reinterpret_cast<double4*>(xoff + 12 * (size_t)e);
            o[0] = make_double4(xS[0][1], xS[0][2], xS[0][3], xS[1][0]);
            o[1] = make_double4(xS[1][2], xS[1][3], xS[2][0], xS[2][1]);
            o[2] = make_double4(xS[2][3], xS[3][0], xS[3][1], xS[3][2]);
        }
    }
}

// e3bSclr per face: the flux term of face nodes 0..2 (frec 3 f + n).
__global__ void __launch_bounds__(128) k_sclr_face(const int4* __restrict__ ienb, const int* __restrict__ iBCB,
                                                   const double* __restrict__ bcbs, const double4* __restrict__ x,
                                                   const double* __restrict__ s, int nface, SclrTables T,
                                                   SclrParams P, double* __restrict__ frec) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nface; f += gridDim.x * blockDim.x) {
        const int4 nn = ienb[f];
        double xl[4][3];
        sclr_gather_x(nn, x, xl);
        const double sl[4] = {s[nn.x], s[nn.y], s[nn.z], s[nn.w]};
        // the host entry checks that bcbs is given where a face prescribes the flux
        const bool given = bcbs != nullptr && ((iBCB[f] >> (4 + P.isclr)) & 1);
        double rl[3] = {0.0, 0.0, 0.0};
        // the face normal, WdetJb (equal weights) and the tet's gradient are
        // the same at the 3 boundary points
        const double v1[3] = {xl[1][0] - xl[0][0], xl[1][1] - xl[0][1], xl[1][2] - xl[0][2]};
        const double v2[3] = {xl[2][0] - xl[0][0], xl[2][1] - xl[0][1], xl[2][2] - xl[0][2]};
        const double te1 = v1[1] * v2[2] - v2[1] * v1[2];
        const double te2 = v2[0] * v1[2] - v1[0] * v2[2];
        const double te3 = v1[0] * v2[1] - v2[0] * v1[1];
        const double temp = 1.0 / sqrt(te1 * te1 + te2 * te2 + te3 * te3);
        const double bn[3] = {te1 * temp, te2 * temp, te3 * temp};
        const double WdetJb = T.Qwtb[0] / (4.0 * temp);
        double cflux = 0.0;
        if (!given) {
            double d[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
            for (int n = 0; n < 4; ++n)
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) d[i][j] = d[i][j] + xl[n][i] * T.shgl[j][n];
            double dx[3][3];
            dx[0][0] = d[1][1] * d[2][2] - d[2][1] * d[1][2];
            dx[0][1] = d[2][1] * d[0][2] - d[0][1] * d[2][2];
            dx[0][2] = d[0][1] * d[1][2] - d[0][2] * d[1][1];
            const double tmp = 1.0 / (dx[0][0] * d[0][0] + dx[0][1] * d[1][0] + dx[0][2] * d[2][0]);
            dx[0][0] = dx[0][0] * tmp;
            dx[0][1] = dx[0][1] * tmp;
            dx[0][2] = dx[0][2] * tmp;
            dx[1][0] = (d[1][2] * d[2][0] - d[1][0] * d[2][2]) * tmp;
            dx[1][1] = (d[0][0] * d[2][2] - d[2][0] * d[0][2]) * tmp;
            dx[1][2] = (d[1][0] * d[0][2] - d[0][0] * d[1][2]) * tmp;
            dx[2][0] = (d[1][0] * d[2][1] - d[1][1] * d[2][0]) * tmp;
            dx[2][1] = (d[2][0] * d[0][1] - d[0][0] * d[2][1]) * tmp;
            dx[2][2] = (d[0][0] * d[1][1] - d[0][1] * d[1][0]) * tmp;
            double gl[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int n = 0; n < 4; ++n)
#pragma unroll
                for (int k = 0; k < 3; ++k) gl[k] = gl[k] + T.shgl[k][n] * sl[n];
            double gS[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) gS[k] = dx[0][k] * gl[0] + dx[1][k] * gl[1] + dx[2][k] * gl[2];
            cflux = P.diffus * (gS[0] * bn[0] + gS[1] * bn[1] + gS[2] * bn[2]);
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            double flux = cflux;
            if (given) {
                flux = 0.0;
#pragma unroll
                for (int n = 0; n < 3; ++n) flux = flux + T.shpb[q][n] * bcbs[3 * (size_t)f + n];
            }
            const double rNa = -WdetJb * flux;
#pragma unroll
            for (int n = 0; n < 3; ++n) rl[n] = rl[n] - T.shpb[q][n] * rNa;
        }
#pragma unroll
        for (int n = 0; n < 3; ++n) frec[3 * (size_t)f + n] = rl[n];
    }
}

// Per node: residual row from its elements (ascending) and its boundary
// faces (ascending), bc3ResSclr, and the diagonal tangent entry.
__global__ void __launch_bounds__(256) k_sclr_node(const int* __restrict__ diag, const int* __restrict__ soff,
                                                   const int* __restrict__ slist, const double* __restrict__ erec,
                                                   const int* __restrict__ fnoff, const int* __restrict__ flist,
                                                   const double* __restrict__ frec, int nshg,
                                                   const int* __restrict__ iBC, int isclr, int lhs,
                                                   double* __restrict__ res, double* __restrict__ lhsS) {
    constexpr int NPW = 32 / kNodeLanes;
    const double2* rec = reinterpret_cast<const double2*>(erec);
    const int lane = threadIdx.x & 31, sub = lane % kNodeLanes;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarp = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long i0 = warp * NPW; i0 < nshg; i0 += nwarp * NPW) {
        const long long ig = i0 + lane / kNodeLanes;
        const bool valid = ig < nshg;
        const int i = valid ? (int)ig : nshg - 1;
        const int d = diag[i];
        double r = 0.0, k = 0.0;
        const int p1 = soff[d + 1];
        for (int p = soff[d] + sub; p < p1; p += kNodeLanes) {
            const int t = slist[p];
            const double2 v = rec[4 * (size_t)(t >> 4) + ((t >> 2) & 3)];
            r += v.x;
            k += v.y;
        }
        // faces after the elements, on the node's first lane
        if (fnoff && sub == 0) {
            double rf = 0.0;
            const int f1 = fnoff[i + 1];
            for (int pf = fnoff[i]; pf < f1; ++pf) rf += frec[flist[pf]];
            r = r + rf;
        }
        r = lanes_sum(r);
        k = lanes_sum(k);
        if (valid && sub == 0) {
            if ((iBC[i] >> (isclr + 5)) & 1) r = 0.0;
            res[i] = r;
            if (lhs) lhsS[d] = k;
        }
    }
}

// Per off-diagonal CSR entry: the elements' xSebe(a, b) in ascending element order.
__global__ void __launch_bounds__(256) k_sclr_slot(const int* __restrict__ soff, const int* __restrict__ slist,
                                                   const double* __restrict__ xoff, long long nnz,
                                                   double* __restrict__ lhsS) {
    for (long long sl = (long long)blockIdx.x * blockDim.x + threadIdx.x; sl < nnz;
         sl += (long long)gridDim.x * blockDim.x) {
        const int p0 = soff[sl], p1 = soff[sl + 1];
        const int t0 = slist[p0];
        if (((t0 >> 2) & 3) == (t0 & 3)) continue;
        double k = 0.0;
        for (int p = p0; p < p1; ++p) {
            const int t = slist[p];
            const int e = t >> 4, a = (t >> 2) & 3, b = t & 3;
            k += xoff[12 * (size_t)e + sclr_off(a, b)];
        }
        lhsS[sl] = k;
    }
}

}  // namespace

// Device entry: d_y (4, nshg) node-major (u, v, w, p), d_s / d_sdot (nshg),
// d_bcbs (nface, 3) face-major or null; d_res (nshg), d_lhsS (nnz).
int elmgmr_sclr_device(crimson_ctx* c, int isclr, double diffus, const double* d_y, const double* d_s,
                       const double* d_sdot, const double* d_bcbs, double* d_res, double* d_lhsS, int lhs) {
    if (isclr < 1 || isclr > 4 || !(diffus >= 0.0) || !d_y || !d_s || !d_sdot || !d_res || (lhs && !d_lhsS))
        return CRIMSON_ERR_ARG;
    cudaStream_t s = c->stream;
    if (c->nnz == 0) CR_CHECK(build_pattern(c));
    if (!c->diag.p || !c->soff.p || !c->slist.p) return CRIMSON_ERR_STATE;
    static const SclrTables T = sclr_tables();
    SclrParams P;
    P.alfi = c->p.alfi;
    P.almi = c->p.almi;
    P.gami = c->p.gami;
    P.Delt = c->p.Delt;
    P.Dtgl = c->p.Dtgl;
    P.dtsfct = c->p.dtsfct;
    P.diffus = diffus;
    P.idiff = c->p.idiff;
    P.isclr = isclr;
    P.lhs = lhs ? 1 : 0;
    CR_CHECK(c->sclr_qres.alloc(3 * (size_t)c->nshg));
    if (c->p.idiff == 1) {
        CR_CHECK(c->sclr_qrec.alloc(4 * (size_t)c->nelem));
        double4* qrec = reinterpret_cast<double4*>(c->sclr_qrec.p);
        launch(k_sclr_q, grid_for(c->nelem, 128, 16), 128, 0, s, c->ien.p, c->x.p, d_s, c->nelem, T, diffus, qrec);
        launch(k_sclr_qnode, grid_for((long long)kNodeLanes * c->nshg, 256), 256, 0, s, c->diag.p, c->soff.p,
               c->slist.p, (const double4*)qrec, c->nshg, T, c->sclr_qres.p);
    }
    CR_CHECK(c->sclr_erec.alloc(8 * (size_t)c->nelem));
    if (lhs) CR_CHECK(c->sclr_xoff.alloc(12 * (size_t)c->nelem));
    launch(k_sclr_elem, grid_for(c->nelem, 128, 16), 128, 0, s, c->ien.p, c->x.p,
           reinterpret_cast<const double4*>(d_y), d_s, d_sdot, (const double*)c->sclr_qres.p, c->nelem, T, P,
           c->sclr_erec.p, lhs ? c->sclr_xoff.p : nullptr);
    const bool faces = c->nface > 0 && c->fnoff.p;
    if (faces) {
        CR_CHECK(c->sclr_frec.alloc(3 * (size_t)c->nface));
        launch(k_sclr_face, grid_for(c->nface, 128, 16), 128, 0, s, c->ienb.p, c->iBCB.p, d_bcbs, c->x.p, d_s,
               c->nface, T, P, c->sclr_frec.p);
    }
    launch(k_sclr_node, grid_for((long long)kNodeLanes * c->nshg, 256), 256, 0, s, c->diag.p, c->soff.p, c->slist.p,
           (const double*)c->sclr_erec.p, faces ? (const int*)c->fnoff.p : nullptr, (const int*)c->flist.p,
           (const double*)c->sclr_frec.p, c->nshg, c->iBC.p, isclr, P.lhs, d_res, d_lhsS);
    if (lhs)
        launch(k_sclr_slot, grid_for(c->nnz, 256), 256, 0, s, c->soff.p, c->slist.p, (const double*)c->sclr_xoff.p,
               c->nnz, d_lhsS);
    CR_CUDA(cudaGetLastError());
    return CRIMSON_OK;
}

}  // namespace crimson
