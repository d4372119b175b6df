// CPU FP64 oracle for the CRIMSON ElmGMR / memLS hot path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
// baseline.  Product code never links or calls this file.
//
// Every routine restates the cited reference Fortran (paths relative to the
// carthurs/CRIMSONFlowsolver tree) with the same loop order and the same order
// of floating-point operations inside each element / each memLS kernel.
// Fortran evaluates a+b+c left to right; the C++ below keeps that
// association explicitly.  Build with -ffp-contract=off so no FMA contraction
// changes the rounding (the reference build uses plain -O2/-O3 gfortran).
//
// Parity status: pinned end to end by the values the reference's own test
// checkClosedLoopWithHeart (flowsolver/test/testMain.cxx:266-345) asserts for
// testbin/mainTests/netlist/closedLoopHeart, which this restatement, driven
// by oracle/pyoracle.py's time stepper, reproduces
// (tests/test_reference_closed_loop_heart.py); no Fortran/MPI toolchain
// exists here to run the reference itself, and no golden vector exists at the
// single-call boundary.  tests/test_oracle_*.py hold the analytic
// self-checks.
#include "crimson_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// Quadrature and shape tables
// ---------------------------------------------------------------------------
// 4-point tet rule, flowsolver/src/symtet.c:22-23, 72-74 (weights 1/4),
// scaled by 4/3 in genint.f90:85.
const double A4 = 0.5854101966249685;
const double B4 = 0.1381966011250150;

struct Tables {
    double shp[4][4];        // shp[intp][n]          (genshp.f90 / uniformP.c:22-40)
    double shgl[4][3][4];    // shgl[intp][dir][n]    halved (genshp.f90:35-36)
    double Qwt[4];
    double shpb[3][4];       // boundary: tri rule (symtri.c rst3) through shpTet (genshpb.f90:31-36)
    double shglb[3][3][4];
    double Qwtb[3];
};

void tet_shape(const double par[3], double N[4], double dN[4][3]) {
    // TetShapeAndDrv for p = 1 (flowsolver/src/uniformP.c:22-40)
    double L[4];
    L[0] = par[0];
    L[1] = par[1];
    L[2] = par[2];
    L[3] = 1.0e0 - par[0] - par[1] - par[2];
    for (int i = 0; i < 4; ++i) {
        N[i] = L[i];
        if (i == 3) {
            dN[i][0] = dN[i][1] = dN[i][2] = -1.0e0;
        } else {
            for (int j = 0; j < 3; ++j) dN[i][j] = (i == j) ? 1.0e0 : 0.0e0;
        }
    }
}

Tables make_tables() {
    Tables t;
    const double rstw4[4][4] = {{A4, B4, B4, B4}, {B4, A4, B4, B4}, {B4, B4, A4, B4}, {B4, B4, B4, A4}};
    for (int q = 0; q < 4; ++q) {
        double N[4], dN[4][3];
        double par[3] = {rstw4[q][0], rstw4[q][1], rstw4[q][2]};
        tet_shape(par, N, dN);
        for (int n = 0; n < 4; ++n) {
            t.shp[q][n] = N[n];
            for (int j = 0; j < 3; ++j) t.shgl[q][j][n] = dN[n][j] / 2.0;
        }
        t.Qwt[q] = (4.0 / 3.0) * 0.25;
    }
    const double B3 = 0.666666666666667, C3 = 0.166666666666667, A3 = 0.3333333333333330000000000000000000;
    const double rst3[3][3] = {{B3, C3, C3}, {C3, B3, C3}, {C3, C3, B3}};
    for (int q = 0; q < 3; ++q) {
        double N[4], dN[4][3];
        double par[3] = {rst3[q][0], rst3[q][1], rst3[q][2]};
        tet_shape(par, N, dN);
        for (int n = 0; n < 4; ++n) {
            t.shpb[q][n] = N[n];
            for (int j = 0; j < 3; ++j) t.shglb[q][j][n] = dN[n][j] / 2.0;
        }
        t.Qwtb[q] = 2.0 * A3;
    }
    return t;
}

const Tables& tables() {
    static Tables t = make_tables();
    return t;
}

// ---------------------------------------------------------------------------
// e3metric (flowsolver/src/e3metric.f90:26-81); dxidx[i][j] = dxidx(:,i,j)
// ---------------------------------------------------------------------------
void e3metric(const double xl[4][3], const double shgl[3][4], double Qwt, double dxidx[3][3],
              double shg[4][3], double* WdetJ) {
    double d[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int n = 0; n < 4; ++n) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) d[i][j] = d[i][j] + xl[n][i] * shgl[j][n];
    }
    dxidx[0][0] = d[1][1] * d[2][2] - d[2][1] * d[1][2];
    dxidx[0][1] = d[2][1] * d[0][2] - d[0][1] * d[2][2];
    dxidx[0][2] = d[0][1] * d[1][2] - d[0][2] * d[1][1];
    double tmp = 1.0 / (dxidx[0][0] * d[0][0] + dxidx[0][1] * d[1][0] + dxidx[0][2] * d[2][0]);
    dxidx[0][0] = dxidx[0][0] * tmp;
    dxidx[0][1] = dxidx[0][1] * tmp;
    dxidx[0][2] = dxidx[0][2] * tmp;
    dxidx[1][0] = (d[1][2] * d[2][0] - d[1][0] * d[2][2]) * tmp;
    dxidx[1][1] = (d[0][0] * d[2][2] - d[2][0] * d[0][2]) * tmp;
    dxidx[1][2] = (d[1][0] * d[0][2] - d[0][0] * d[1][2]) * tmp;
    dxidx[2][0] = (d[1][0] * d[2][1] - d[1][1] * d[2][0]) * tmp;
    dxidx[2][1] = (d[2][0] * d[0][1] - d[0][0] * d[2][1]) * tmp;
    dxidx[2][2] = (d[0][0] * d[1][1] - d[0][1] * d[1][0]) * tmp;
    *WdetJ = Qwt / tmp;
    for (int n = 0; n < 4; ++n) {
        for (int k = 0; k < 3; ++k)
            shg[n][k] = shgl[0][n] * dxidx[0][k] + shgl[1][n] * dxidx[1][k] + shgl[2][n] * dxidx[2][k];
    }
}

// e3gijd, tet branch (flowsolver/src/e3stab.f90:487-528); gijd[0..5] = gijd(:,1..6)
void e3gijd(const double dx[3][3], double g[6]) {
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
// e3q for one element (flowsolver/src/e3q.f90:58-145, e3qvar.f90:58-131)
// yl[n][0..3] = (p, u, v, w) as gathered by localy.
// ---------------------------------------------------------------------------
void e3q_elem(const orc_params* p, const double yl[4][4], const double xl[4][3], double ql[4][9],
              double rmassl[4]) {
    const Tables& T = tables();
    for (int n = 0; n < 4; ++n) {
        for (int k = 0; k < 9; ++k) ql[n][k] = 0.0;
        rmassl[n] = 0.0;
    }
    for (int intp = 0; intp < 4; ++intp) {
        const double* shapeVar = T.shp[intp];
        double dxidx[3][3], shg[4][3], WdetJ;
        e3metric(xl, T.shgl[intp], T.Qwt[intp], dxidx, shg, &WdetJ);
        double g[3][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};   // g[k][d] = g{k+1}yi(:,d+1)
        for (int n = 0; n < 4; ++n) {
            for (int k = 0; k < 3; ++k)
                for (int d = 1; d < 4; ++d) g[k][d] = g[k][d] + shg[n][k] * yl[n][d];
        }
        const double rmu = p->mu;
        double qdi[9];
        qdi[0] = 2.0 * rmu * g[0][1];
        qdi[3] = rmu * (g[0][2] + g[1][1]);
        qdi[6] = rmu * (g[0][3] + g[2][1]);
        qdi[1] = rmu * (g[0][2] + g[1][1]);
        qdi[4] = 2.0 * rmu * g[1][2];
        qdi[7] = rmu * (g[1][3] + g[2][2]);
        qdi[2] = rmu * (g[0][3] + g[2][1]);
        qdi[5] = rmu * (g[1][3] + g[2][2]);
        qdi[8] = 2.0 * rmu * g[2][3];
        for (int i = 0; i < 4; ++i)
            for (int k = 0; k < 9; ++k) ql[i][k] = ql[i][k] + shapeVar[i] * WdetJ * qdi[k];
        if (p->idiff == 1) {
            for (int i = 0; i < 4; ++i) rmassl[i] = rmassl[i] + shapeVar[i] * WdetJ;
        }
    }
}

// ---------------------------------------------------------------------------
// e3 for one element: e3ivar, e3stab, e3Res, e3LHS over 4 quadrature points
// (flowsolver/src/e3.f90:96-169).  rl[a][0..3] = momentum x,y,z, continuity.
// xKebe[c][a][b] = xKebe(:,c+1,a+1,b+1); xGoC[c][a][b] likewise.
// ---------------------------------------------------------------------------
void e3_elem(const orc_params* p, const double yl[4][4], const double acl[4][4], const double xl[4][3],
             const double ql[4][9], int lhs, double rl[4][4], double xKebe[9][4][4], double xGoC[4][4][4]) {
    const Tables& T = tables();
    for (int intp = 0; intp < 4; ++intp) {
        const double* shpfun = T.shp[intp];
        // getDiff (getdiff.f90:44-53)
        double rho = p->rho;
        double rmu = p->mu;
        // ---- e3ivar (e3ivar.f90:99-198, 348-370, 424-429) ----
        double pres = 0.0, u1 = 0.0, u2 = 0.0, u3 = 0.0;
        for (int n = 0; n < 4; ++n) {
            pres = pres + shpfun[n] * yl[n][0];
            u1 = u1 + shpfun[n] * yl[n][1];
            u2 = u2 + shpfun[n] * yl[n][2];
            u3 = u3 + shpfun[n] * yl[n][3];
        }
        double aci[3] = {0.0, 0.0, 0.0};
        for (int n = 0; n < 4; ++n) {
            aci[0] = aci[0] + shpfun[n] * acl[n][1];
            aci[1] = aci[1] + shpfun[n] * acl[n][2];
            aci[2] = aci[2] + shpfun[n] * acl[n][3];
        }
        double dxidx[3][3], shg[4][3], WdetJ;
        e3metric(xl, T.shgl[intp], T.Qwt[intp], dxidx, shg, &WdetJ);
        double g1[4] = {0, 0, 0, 0}, g2[4] = {0, 0, 0, 0}, g3[4] = {0, 0, 0, 0};
        for (int n = 0; n < 4; ++n) {
            for (int d = 0; d < 4; ++d) g1[d] = g1[d] + shg[n][0] * yl[n][d];
            for (int d = 0; d < 4; ++d) g2[d] = g2[d] + shg[n][1] * yl[n][d];
            for (int d = 0; d < 4; ++d) g3[d] = g3[d] + shg[n][2] * yl[n][d];
        }
        double divqi[3] = {0.0, 0.0, 0.0};
        if (p->idiff >= 1) {
            for (int n = 0; n < 4; ++n) {
                divqi[0] = divqi[0] + shg[n][0] * ql[n][0] + shg[n][1] * ql[n][3] + shg[n][2] * ql[n][6];
                divqi[1] = divqi[1] + shg[n][0] * ql[n][1] + shg[n][1] * ql[n][4] + shg[n][2] * ql[n][7];
                divqi[2] = divqi[2] + shg[n][0] * ql[n][2] + shg[n][1] * ql[n][5] + shg[n][2] * ql[n][8];
            }
        }
        // e3resStrongPDE_ALE (e3res.f90:718-797), no body force, uMesh = 0
        const double src[3] = {0.0, 0.0, 0.0};
        double rLui[3];
        rLui[0] = (aci[0] + u1 * g1[1] + u2 * g2[1] + u3 * g3[1] - src[0]) * rho + g1[0] - divqi[0];
        rLui[1] = (aci[1] + u1 * g1[2] + u2 * g2[2] + u3 * g3[2] - src[1]) * rho + g2[0] - divqi[1];
        rLui[2] = (aci[2] + u1 * g1[3] + u2 * g2[3] + u3 * g3[3] - src[2]) * rho + g3[0] - divqi[2];
        if (p->iconvflow == 1) {
            double divu = (g1[1] + g2[2] + g3[3]) * rho;
            rLui[0] = rLui[0] + u1 * divu;
            rLui[1] = rLui[1] + u2 * divu;
            rLui[2] = rLui[2] + u3 * divu;
        }
        // ---- e3stab, itau = 0 (e3stab.f90:83-133, 356-374) ----
        double gijd[6];
        e3gijd(dxidx, gijd);
        const double fff = 36.0;
        const double omegasq = 0.0;
        double rhoinv = 1.0 / rho;
        double rnu = rmu * rhoinv;
        double dts = p->Dtgl * p->dtsfct;
        double tauM = ((2.0 * dts) * (2.0 * dts)
                       + (u1 * (gijd[0] * u1 + gijd[3] * u2 + gijd[5] * u3)
                          + u2 * (gijd[3] * u1 + gijd[1] * u2 + gijd[4] * u3)
                          + u3 * (gijd[5] * u1 + gijd[4] * u2 + gijd[2] * u3)))
                      + fff * (rnu * rnu)
                            * (gijd[0] * gijd[0] + gijd[1] * gijd[1] + gijd[2] * gijd[2]
                               + 2.0 * (gijd[3] * gijd[3] + gijd[4] * gijd[4] + gijd[5] * gijd[5]) + omegasq);
        double fact = std::sqrt(tauM);
        double ff = p->taucfct / p->dtsfct;
        double tauC = rho * 0.125 * fact / (gijd[0] + gijd[1] + gijd[2]) * ff;
        tauM = 1.0 / fact;
        double tauBar = rLui[0] * (gijd[0] * rLui[0] + gijd[3] * rLui[1] + gijd[5] * rLui[2])
                        + rLui[1] * (gijd[3] * rLui[0] + gijd[1] * rLui[1] + gijd[4] * rLui[2])
                        + rLui[2] * (gijd[5] * rLui[0] + gijd[4] * rLui[1] + gijd[2] * rLui[2]);
        if (tauBar != 0.0) tauBar = tauM / std::sqrt(tauBar);
        double uBar[3];
        uBar[0] = u1 - tauM * rLui[0] * rhoinv;
        uBar[1] = u2 - tauM * rLui[1] * rhoinv;
        uBar[2] = u3 - tauM * rLui[2] * rhoinv;
        // ---- e3Res (e3res.f90:94-286) ----
        double rNa[3], rGNa[3][3];
        double tmps = 1.0 - p->flmpr;
        rNa[0] = aci[0] * tmps - src[0];
        rNa[1] = aci[1] * tmps - src[1];
        rNa[2] = aci[2] * tmps - src[2];
        double tmp = -pres + tauC * (g1[1] + g2[2] + g3[3]);
        double tmp1 = rmu * (g2[1] + g1[2]);
        double tmp2 = rmu * (g3[2] + g2[3]);
        double tmp3 = rmu * (g1[3] + g3[1]);
        if (p->iconvflow == 2) {
            rNa[0] = rNa[0] + uBar[0] * g1[1] + uBar[1] * g2[1] + uBar[2] * g3[1];
            rNa[1] = rNa[1] + uBar[0] * g1[2] + uBar[1] * g2[2] + uBar[2] * g3[2];
            rNa[2] = rNa[2] + uBar[0] * g1[3] + uBar[1] * g2[3] + uBar[2] * g3[3];
            rGNa[0][0] = 2.0 * rmu * g1[1] + tmp;
            rGNa[0][1] = tmp1;
            rGNa[0][2] = tmp3;
            rGNa[1][0] = tmp1;
            rGNa[1][1] = 2.0 * rmu * g2[2] + tmp;
            rGNa[1][2] = tmp2;
            rGNa[2][0] = tmp3;
            rGNa[2][1] = tmp2;
            rGNa[2][2] = 2.0 * rmu * g3[3] + tmp;
        } else {
            rGNa[0][0] = 2.0 * rmu * g1[1] + tmp - u1 * u1 * rho;
            rGNa[0][1] = tmp1 - u1 * u2 * rho;
            rGNa[0][2] = tmp3 - u1 * u3 * rho;
            rGNa[1][0] = tmp1 - u1 * u2 * rho;
            rGNa[1][1] = 2.0 * rmu * g2[2] + tmp - u2 * u2 * rho;
            rGNa[1][2] = tmp2 - u3 * u2 * rho;
            rGNa[2][0] = tmp3 - u1 * u3 * rho;
            rGNa[2][1] = tmp2 - u3 * u2 * rho;
            rGNa[2][2] = 2.0 * rmu * g3[3] + tmp - u3 * u3 * rho;
        }
        tmp1 = tauM * rLui[0];
        tmp2 = tauM * rLui[1];
        tmp3 = tauM * rLui[2];
        rGNa[0][0] = rGNa[0][0] + tmp1 * u1;
        rGNa[0][1] = rGNa[0][1] + tmp1 * u2;
        rGNa[0][2] = rGNa[0][2] + tmp1 * u3;
        rGNa[1][0] = rGNa[1][0] + tmp2 * u1;
        rGNa[1][1] = rGNa[1][1] + tmp2 * u2;
        rGNa[1][2] = rGNa[1][2] + tmp2 * u3;
        rGNa[2][0] = rGNa[2][0] + tmp3 * u1;
        rGNa[2][1] = rGNa[2][1] + tmp3 * u2;
        rGNa[2][2] = rGNa[2][2] + tmp3 * u3;
        if (p->iconvflow == 1) {
            rGNa[0][0] = rGNa[0][0] + tmp1 * u1;
            rGNa[0][1] = rGNa[0][1] + tmp2 * u1;
            rGNa[0][2] = rGNa[0][2] + tmp3 * u1;
            rGNa[1][0] = rGNa[1][0] + tmp1 * u2;
            rGNa[1][1] = rGNa[1][1] + tmp2 * u2;
            rGNa[1][2] = rGNa[1][2] + tmp3 * u2;
            rGNa[2][0] = rGNa[2][0] + tmp1 * u3;
            rGNa[2][1] = rGNa[2][1] + tmp2 * u3;
            rGNa[2][2] = rGNa[2][2] + tmp3 * u3;
        }
        if (p->iconvflow == 2) {
            tmp1 = tauBar * (rLui[0] * g1[1] + rLui[1] * g2[1] + rLui[2] * g3[1]);
            tmp2 = tauBar * (rLui[0] * g1[2] + rLui[1] * g2[2] + rLui[2] * g3[2]);
            tmp3 = tauBar * (rLui[0] * g1[3] + rLui[1] * g2[3] + rLui[2] * g3[3]);
            rGNa[0][0] = rGNa[0][0] + tmp1 * rLui[0];
            rGNa[0][1] = rGNa[0][1] + tmp1 * rLui[1];
            rGNa[0][2] = rGNa[0][2] + tmp1 * rLui[2];
            rGNa[1][0] = rGNa[1][0] + tmp2 * rLui[0];
            rGNa[1][1] = rGNa[1][1] + tmp2 * rLui[1];
            rGNa[1][2] = rGNa[1][2] + tmp2 * rLui[2];
            rGNa[2][0] = rGNa[2][0] + tmp3 * rLui[0];
            rGNa[2][1] = rGNa[2][1] + tmp3 * rLui[1];
            rGNa[2][2] = rGNa[2][2] + tmp3 * rLui[2];
        }
        rNa[0] = rNa[0] * rho;
        rNa[1] = rNa[1] * rho;
        rNa[2] = rNa[2] * rho;
        for (int aa = 0; aa < 4; ++aa) {
            rl[aa][3] = rl[aa][3] + WdetJ * (shg[aa][0] * uBar[0] + shg[aa][1] * uBar[1] + shg[aa][2] * uBar[2]);
            for (int i = 0; i < 3; ++i)
                rl[aa][i] = rl[aa][i] - WdetJ * (shpfun[aa] * rNa[i] + shg[aa][0] * rGNa[i][0]
                                                 + shg[aa][1] * rGNa[i][1] + shg[aa][2] * rGNa[i][2]);
        }
        if (!lhs) continue;
        // ---- e3LHS (e3lhs.f90:85-402) ----
        double lhsFct = p->alfi * p->gami * p->Delt;
        double lhmFct = p->almi * (1.0 - p->flmpl);
        double tlW = lhsFct * WdetJ;
        double tmp1s = tlW * rho;
        tauM = tlW * tauM;
        tauC = tlW * tauC;
        double rmuW = tlW * rmu;
        double tsFct = lhmFct * WdetJ * rho;
        double ub[3];
        if (p->iconvflow == 2) {
            tauBar = lhsFct * WdetJ * tauBar;
            ub[0] = tmp1s * uBar[0];
            ub[1] = tmp1s * uBar[1];
            ub[2] = tmp1s * uBar[2];
        } else {
            tauBar = 0.0;
            ub[0] = tmp1s * u1;
            ub[1] = tmp1s * u2;
            ub[2] = tmp1s * u3;
        }
        for (int b = 0; b < 4; ++b) {
            double t1 = ub[0] * shg[b][0] + ub[1] * shg[b][1] + ub[2] * shg[b][2];
            for (int aa = 0; aa < 4; ++aa) {
                double m1 = tsFct * shpfun[aa] * shpfun[b];
                double m2 = m1 + t1 * shpfun[aa];
                xKebe[0][aa][b] = xKebe[0][aa][b] + m2;
                xKebe[4][aa][b] = xKebe[4][aa][b] + m2;
                xKebe[8][aa][b] = xKebe[8][aa][b] + m2;
            }
        }
        for (int b = 0; b < 4; ++b) {
            double t1[3], t2[3], t3[3];
            t1[0] = tauC * shg[b][0];
            t1[1] = tauC * shg[b][1];
            t1[2] = tauC * shg[b][2];
            t2[0] = rmuW * shg[b][0];
            t2[1] = rmuW * shg[b][1];
            t2[2] = rmuW * shg[b][2];
            double s1 = tauM * (u1 * shg[b][0] + u2 * shg[b][1] + u3 * shg[b][2]) * rho;
            double s2 = tauBar * (rLui[0] * shg[b][0] + rLui[1] * shg[b][1] + rLui[2] * shg[b][2]);
            t3[0] = t2[0] + s1 * u1 + s2 * rLui[0];
            t3[1] = t2[1] + s1 * u2 + s2 * rLui[1];
            t3[2] = t2[2] + s1 * u3 + s2 * rLui[2];
            int aa = b;
            double tt = t3[0] * shg[aa][0] + t3[1] * shg[aa][1] + t3[2] * shg[aa][2];
            xKebe[0][aa][b] = xKebe[0][aa][b] + tt + t1[0] * shg[aa][0] + t2[0] * shg[aa][0];
            xKebe[4][aa][b] = xKebe[4][aa][b] + tt + t1[1] * shg[aa][1] + t2[1] * shg[aa][1];
            xKebe[8][aa][b] = xKebe[8][aa][b] + tt + t1[2] * shg[aa][2] + t2[2] * shg[aa][2];
            double q;
            q = t1[0] * shg[aa][1] + t2[1] * shg[aa][0];
            xKebe[1][aa][b] = xKebe[1][aa][b] + q;
            xKebe[3][b][aa] = xKebe[3][b][aa] + q;
            q = t1[0] * shg[aa][2] + t2[2] * shg[aa][0];
            xKebe[2][aa][b] = xKebe[2][aa][b] + q;
            xKebe[6][b][aa] = xKebe[6][b][aa] + q;
            q = t1[1] * shg[aa][2] + t2[2] * shg[aa][1];
            xKebe[5][aa][b] = xKebe[5][aa][b] + q;
            xKebe[7][b][aa] = xKebe[7][b][aa] + q;
            for (aa = b + 1; aa < 4; ++aa) {
                tt = t3[0] * shg[aa][0] + t3[1] * shg[aa][1] + t3[2] * shg[aa][2];
                q = tt + t1[0] * shg[aa][0] + t2[0] * shg[aa][0];
                xKebe[0][aa][b] = xKebe[0][aa][b] + q;
                xKebe[0][b][aa] = xKebe[0][b][aa] + q;
                q = tt + t1[1] * shg[aa][1] + t2[1] * shg[aa][1];
                xKebe[4][aa][b] = xKebe[4][aa][b] + q;
                xKebe[4][b][aa] = xKebe[4][b][aa] + q;
                q = tt + t1[2] * shg[aa][2] + t2[2] * shg[aa][2];
                xKebe[8][aa][b] = xKebe[8][aa][b] + q;
                xKebe[8][b][aa] = xKebe[8][b][aa] + q;
                q = t1[0] * shg[aa][1] + t2[1] * shg[aa][0];
                xKebe[1][aa][b] = xKebe[1][aa][b] + q;
                xKebe[3][b][aa] = xKebe[3][b][aa] + q;
                q = t1[0] * shg[aa][2] + t2[2] * shg[aa][0];
                xKebe[2][aa][b] = xKebe[2][aa][b] + q;
                xKebe[6][b][aa] = xKebe[6][b][aa] + q;
                q = t1[1] * shg[aa][0] + t2[0] * shg[aa][1];
                xKebe[3][aa][b] = xKebe[3][aa][b] + q;
                xKebe[1][b][aa] = xKebe[1][b][aa] + q;
                q = t1[1] * shg[aa][2] + t2[2] * shg[aa][1];
                xKebe[5][aa][b] = xKebe[5][aa][b] + q;
                xKebe[7][b][aa] = xKebe[7][b][aa] + q;
                q = t1[2] * shg[aa][0] + t2[0] * shg[aa][2];
                xKebe[6][aa][b] = xKebe[6][aa][b] + q;
                xKebe[2][b][aa] = xKebe[2][b][aa] + q;
                q = t1[2] * shg[aa][1] + t2[1] * shg[aa][2];
                xKebe[7][aa][b] = xKebe[7][aa][b] + q;
                xKebe[5][b][aa] = xKebe[5][b][aa] + q;
            }
        }
        for (int b = 0; b < 4; ++b) {
            double t1[3] = {tlW * shg[b][0], tlW * shg[b][1], tlW * shg[b][2]};
            for (int aa = 0; aa < 4; ++aa) {
                xGoC[0][aa][b] = xGoC[0][aa][b] + t1[0] * shpfun[aa];
                xGoC[1][aa][b] = xGoC[1][aa][b] + t1[1] * shpfun[aa];
                xGoC[2][aa][b] = xGoC[2][aa][b] + t1[2] * shpfun[aa];
            }
        }
        tauM = tauM / rho;
        for (int b = 0; b < 4; ++b) {
            double t1[3] = {tauM * shg[b][0], tauM * shg[b][1], tauM * shg[b][2]};
            for (int aa = b; aa < 4; ++aa)
                xGoC[3][aa][b] = xGoC[3][aa][b] + t1[0] * shg[aa][0] + t1[1] * shg[aa][1] + t1[2] * shg[aa][2];
        }
    }
    if (lhs) {
        // symmetrize C (e3.f90:163-169)
        for (int ib = 0; ib < 4; ++ib)
            for (int iaa = 0; iaa < ib; ++iaa) xGoC[3][iaa][ib] = xGoC[3][ib][iaa];
    }
}

// ---------------------------------------------------------------------------
// e3b + e3bvar for one linear-tet boundary face, rigid wall
// (flowsolver/src/e3b.f90:112-470, e3bvar.f90:140-460).  rl[n][0..3].
// ---------------------------------------------------------------------------
void e3b_face(const orc_params* p, const double yl[4][4], const double xlb[4][3], int ibcb_bits,
              const double bcb[3][6], double rl[4][4]) {
    const Tables& T = tables();
    for (int intp = 0; intp < 3; ++intp) {
        const double* shapeVar = T.shpb[intp];
        double rmu = p->mu;
        double rho = p->rho;
        // e3bvar
        double pres = 0.0, u1 = 0.0, u2 = 0.0, u3 = 0.0;
        for (int n = 0; n < 3; ++n) {
            pres = pres + shapeVar[n] * yl[n][0];
            u1 = u1 + shapeVar[n] * yl[n][1];
            u2 = u2 + shapeVar[n] * yl[n][2];
            u3 = u3 + shapeVar[n] * yl[n][3];
        }
        double d[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int n = 0; n < 4; ++n)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) d[i][j] = d[i][j] + xlb[n][i] * T.shglb[intp][j][n];
        double v1[3], v2[3];
        for (int i = 0; i < 3; ++i) {
            v1[i] = xlb[1][i] - xlb[0][i];
            v2[i] = xlb[2][i] - xlb[0][i];
        }
        double temp1 = v1[1] * v2[2] - v2[1] * v1[2];
        double temp2 = v2[0] * v1[2] - v1[0] * v2[2];
        double temp3 = v1[0] * v2[1] - v2[0] * v1[1];
        double temp = 1.0 / std::sqrt(temp1 * temp1 + temp2 * temp2 + temp3 * temp3);
        double bn[3] = {temp1 * temp, temp2 * temp, temp3 * temp};
        double WdetJb = T.Qwtb[intp] / (4.0 * temp);
        double dx[3][3];
        dx[0][0] = d[1][1] * d[2][2] - d[2][1] * d[1][2];
        dx[0][1] = d[2][1] * d[0][2] - d[0][1] * d[2][2];
        dx[0][2] = d[0][1] * d[1][2] - d[0][2] * d[1][1];
        double tmp = 1.0 / (dx[0][0] * d[0][0] + dx[0][1] * d[1][0] + dx[0][2] * d[2][0]);
        dx[0][0] = dx[0][0] * tmp;
        dx[0][1] = dx[0][1] * tmp;
        dx[0][2] = dx[0][2] * tmp;
        dx[1][0] = (d[1][2] * d[2][0] - d[1][0] * d[2][2]) * tmp;
        dx[1][1] = (d[0][0] * d[2][2] - d[2][0] * d[0][2]) * tmp;
        dx[1][2] = (d[1][0] * d[0][2] - d[0][0] * d[1][2]) * tmp;
        dx[2][0] = (d[1][0] * d[2][1] - d[1][1] * d[2][0]) * tmp;
        dx[2][1] = (d[2][0] * d[0][1] - d[0][0] * d[2][1]) * tmp;
        dx[2][2] = (d[0][0] * d[1][1] - d[0][1] * d[1][0]) * tmp;
        double gl[3][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
        for (int n = 0; n < 4; ++n)
            for (int k = 0; k < 3; ++k)
                for (int dd = 0; dd < 4; ++dd) gl[k][dd] = gl[k][dd] + T.shglb[intp][k][n] * yl[n][dd];
        double g[3][4];   // g[k][dd] = g{k+1}yi(:,dd+1), dd = 1..3
        for (int dd = 1; dd < 4; ++dd)
            for (int k = 0; k < 3; ++k)
                g[k][dd] = dx[0][k] * gl[0][dd] + dx[1][k] * gl[1][dd] + dx[2][k] * gl[2][dd];
        double unm = bn[0] * u1 + bn[1] * u2 + bn[2] * u3;
        double tau1n = bn[0] * 2.0 * rmu * g[0][1] + bn[1] * (rmu * (g[1][1] + g[0][2])) + bn[2] * (rmu * (g[2][1] + g[0][3]));
        double tau2n = bn[0] * (rmu * (g[1][1] + g[0][2])) + bn[1] * 2.0 * rmu * g[1][2] + bn[2] * (rmu * (g[2][2] + g[1][3]));
        double tau3n = bn[0] * (rmu * (g[2][1] + g[0][3])) + bn[1] * (rmu * (g[2][2] + g[1][3])) + bn[2] * 2.0 * rmu * g[2][3];
        double tn = bn[0] * tau1n + bn[1] * tau2n + bn[2] * tau3n;
        pres = pres - tn;
        tau1n = tau1n - bn[0] * tn;
        tau2n = tau2n - bn[1] * tn;
        tau3n = tau3n - bn[2] * tn;
        // e3b boundary conditions
        double unm_copy = 0.0;
        if ((ibcb_bits >> 1) & 1) {
            if (unm < 0.0) unm_copy = unm;
        }
        if (ibcb_bits & 1) {
            unm = 0.0;
            for (int n = 0; n < 3; ++n) unm = unm + shapeVar[n] * bcb[n][0];
        }
        if ((ibcb_bits >> 1) & 1) {
            pres = 0.0;
            for (int n = 0; n < 3; ++n) pres = pres + shapeVar[n] * bcb[n][1];
        }
        if ((ibcb_bits >> 2) & 1) {
            tau1n = 0.0;
            tau2n = 0.0;
            tau3n = 0.0;
            for (int n = 0; n < 3; ++n) {
                tau1n = tau1n + shapeVar[n] * bcb[n][2];
                tau2n = tau2n + shapeVar[n] * bcb[n][3];
                tau3n = tau3n + shapeVar[n] * bcb[n][4];
            }
        }
        if ((ibcb_bits >> 4) & 1) {
            pres = 0.0;
            tau1n = 0.0;
            tau2n = 0.0;
            tau3n = 0.0;
        }
        double rNa[4];
        rNa[0] = -tau1n + bn[0] * pres;
        rNa[1] = -tau2n + bn[1] * pres;
        rNa[2] = -tau3n + bn[2] * pres;
        rNa[3] = unm;
        if (p->iconvflow == 1) {
            double rou = rho * unm;
            rNa[0] = rNa[0] + rou * u1;
            rNa[1] = rNa[1] + rou * u2;
            rNa[2] = rNa[2] + rou * u3;
        }
        double rou_copy = rho * unm_copy;
        rNa[0] = rNa[0] - p->stabflux_coeff * rou_copy * u1;
        rNa[1] = rNa[1] - p->stabflux_coeff * rou_copy * u2;
        rNa[2] = rNa[2] - p->stabflux_coeff * rou_copy * u3;
        for (int k = 0; k < 4; ++k) rNa[k] = rNa[k] * WdetJb;
        for (int n = 0; n < 3; ++n)
            for (int k = 0; k < 4; ++k) rl[n][k] = rl[n][k] - shapeVar[n] * rNa[k];
    }
}

// sparseloc binary search (flowsolver/src/fillsparse.f90:210-246); list 1-based semantics
inline long long sparseloc(const int* list, int n, int target) {
    int rowvl = 1, rowvh = n + 1;
    while (rowvh - rowvl > 1) {
        int rowv = (rowvh + rowvl) / 2;
        if (list[rowv - 1] > target)
            rowvh = rowv;
        else
            rowvl = rowv;
    }
    return rowvl;
}

int nthreads_of(const orc_params* p) { return p->nthreads > 0 ? p->nthreads : 1; }

// CPUT (memLS.f90:2382-2400): wall-clock seconds
double CPUT() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// ===========================================================================
// genadj + Asadj (flowsolver/src/genadj.f90:20-71, asadj.f90:21-54)
// ===========================================================================
extern "C" int orc_genadj(int nshg, int nelem, const int* ien, int* colm, int* rowp, long long cap,
                          long long* nnz_tot) {
    if (nshg <= 0 || nelem < 0 || !ien || !colm) return ORC_ERR_ARG;
    std::vector<std::vector<int>> row_fill_list(nshg);
    for (int i = 0; i < nelem; ++i) {
        int ndlist[4];
        for (int j = 0; j < 4; ++j) ndlist[j] = std::abs(ien[j * nelem + i]);
        for (int j = 0; j < 4; ++j) {
            int jnd = ndlist[j];
            std::vector<int>& lst = row_fill_list[jnd - 1];
            int jlngth = (int)lst.size();
            for (int k = 0; k < 4; ++k) {
                int knd = ndlist[k];
                bool ibroke = false;
                for (int l = 0; l < jlngth; ++l) {
                    if (lst[l] == knd) {
                        ibroke = true;
                        break;
                    }
                }
                if (!ibroke) {
                    lst.push_back(knd);
                    ++jlngth;
                }
            }
        }
    }
    colm[0] = 1;
    for (int i = 0; i < nshg; ++i) colm[i + 1] = colm[i] + (int)row_fill_list[i].size();
    long long icnt = 0;
    const double ibig = 10.0 * nshg;
    std::vector<double> tmpr;
    for (int i = 0; i < nshg; ++i) {
        int ncol = (int)row_fill_list[i].size();
        tmpr.assign(row_fill_list[i].begin(), row_fill_list[i].end());
        for (int j = 0; j < ncol; ++j) {
            // minval + minloc (first occurrence)
            int mloc = 0;
            double imin = tmpr[0];
            for (int t = 1; t < ncol; ++t)
                if (tmpr[t] < imin) {
                    imin = tmpr[t];
                    mloc = t;
                }
            if (rowp) {
                if (icnt >= cap) return ORC_ERR_PATTERN;
                rowp[icnt] = (int)imin;
            }
            ++icnt;
            tmpr[mloc] = ibig;
        }
    }
    *nnz_tot = icnt;
    return ORC_OK;
}

// ===========================================================================
// bc3LHS (flowsolver/src/bc3lhs.f90:39-198): for every element node with one
// or two prescribed velocity components (ibits(iBC,3,3) in 1..6), project
// the constraint out of the element tangent xK (xK[cc*16 + a*4 + b], cc the
// row-major 3x3 component): the columns of blocks (i, inod), then the rows
// of blocks (inod, i), then 1 on the constrained diagonal entries of block
// (inod, inod).  BC column-major (nshg, ndofBC): BC(:,4..6) are k = 3..5.
// The two-component case ibits = 6 keeps the reference's own row update
// (row 3 from row 1 and entry 6, rows 1-2 zeroed) exactly as bc3lhs.f90
// writes it.
// ===========================================================================
static void bc3lhs_elem(int nshg, const int* iBC, const double* BC, const int nd[4], double* xK) {
    for (int inod = 0; inod < 4; ++inod) {
        const int in = nd[inod];
        const int m = (iBC[in] >> 3) & 7;
        if (m == 0 || m == 7) continue;
        const double b4 = BC[3 * (size_t)nshg + in], b5 = BC[4 * (size_t)nshg + in], b6 = BC[5 * (size_t)nshg + in];
        auto K = [&](int cc, int a, int b) -> double& { return xK[cc * 16 + a * 4 + b]; };
        if (m == 1 || m == 2 || m == 4) {
            const int c0 = m == 1 ? 0 : (m == 2 ? 1 : 2);
            const int f1 = m == 1 ? 1 : 0, f2 = m == 4 ? 1 : 2;
            for (int i = 0; i < 4; ++i)
                for (int r = 0; r < 3; ++r) K(3 * r + f1, i, inod) = K(3 * r + f1, i, inod) - b4 * K(3 * r + c0, i, inod);
            for (int i = 0; i < 4; ++i)
                for (int r = 0; r < 3; ++r) K(3 * r + f2, i, inod) = K(3 * r + f2, i, inod) - b5 * K(3 * r + c0, i, inod);
            for (int i = 0; i < 4; ++i)
                for (int r = 0; r < 3; ++r) K(3 * r + c0, i, inod) = 0.0;
            for (int i = 0; i < 4; ++i)
                for (int q = 0; q < 3; ++q) K(3 * f1 + q, inod, i) = K(3 * f1 + q, inod, i) - b4 * K(3 * c0 + q, inod, i);
            for (int i = 0; i < 4; ++i)
                for (int q = 0; q < 3; ++q) K(3 * f2 + q, inod, i) = K(3 * f2 + q, inod, i) - b5 * K(3 * c0 + q, inod, i);
            for (int i = 0; i < 4; ++i)
                for (int q = 0; q < 3; ++q) K(3 * c0 + q, inod, i) = 0.0;
            K(4 * c0, inod, inod) = 1.0;
        } else {
            const int f = m == 3 ? 2 : (m == 5 ? 1 : 0);
            const int c0 = m == 6 ? 1 : 0, c1 = m == 3 ? 1 : 2;
            for (int i = 0; i < 4; ++i)
                for (int r = 0; r < 3; ++r)
                    K(3 * r + f, i, inod) = K(3 * r + f, i, inod) - b4 * K(3 * r + c0, i, inod) - b6 * K(3 * r + c1, i, inod);
            for (int i = 0; i < 4; ++i)
                for (int r = 0; r < 3; ++r) {
                    K(3 * r + c0, i, inod) = 0.0;
                    K(3 * r + c1, i, inod) = 0.0;
                }
            if (m != 6) {
                for (int i = 0; i < 4; ++i)
                    for (int q = 0; q < 3; ++q)
                        K(3 * f + q, inod, i) = K(3 * f + q, inod, i) - b4 * K(3 * c0 + q, inod, i) - b6 * K(3 * c1 + q, inod, i);
                for (int i = 0; i < 4; ++i)
                    for (int q = 0; q < 3; ++q) {
                        K(3 * c0 + q, inod, i) = 0.0;
                        K(3 * c1 + q, inod, i) = 0.0;
                    }
            } else {
                // bc3lhs.f90:643-672: row 3 updated from row 1 (and entry 6), rows 1-2 zeroed
                for (int i = 0; i < 4; ++i) {
                    K(6, inod, i) = K(6, inod, i) - b4 * K(0, inod, i);
                    K(7, inod, i) = K(7, inod, i) - b4 * K(1, inod, i);
                    K(8, inod, i) = K(8, inod, i) - b4 * K(2, inod, i) - b6 * K(5, inod, i);
                }
                for (int i = 0; i < 4; ++i)
                    for (int q = 0; q < 6; ++q) K(q, inod, i) = 0.0;
            }
            K(4 * c0, inod, inod) = 1.0;
            K(4 * c1, inod, inod) = 1.0;
        }
    }
}

// bc3Res velocity branches (bc3res.f90:53-103) for node i, res column-major
static void bc3res_partial(int nshg, const int* iBC, const double* BC, int i, double* res) {
    const int m = (iBC[i] >> 3) & 7;
    double* r0 = res + i;
    double* r1 = res + (size_t)nshg + i;
    double* r2 = res + 2 * (size_t)nshg + i;
    const double b4 = BC[3 * (size_t)nshg + i], b5 = BC[4 * (size_t)nshg + i], b6 = BC[5 * (size_t)nshg + i];
    switch (m) {
        case 1: *r1 = *r1 - b4 * *r0; *r2 = *r2 - b5 * *r0; *r0 = 0.0; break;
        case 2: *r0 = *r0 - b4 * *r1; *r2 = *r2 - b5 * *r1; *r1 = 0.0; break;
        case 3: *r2 = *r2 - b4 * *r0 - b6 * *r1; *r0 = 0.0; *r1 = 0.0; break;
        case 4: *r0 = *r0 - b4 * *r2; *r1 = *r1 - b5 * *r2; *r2 = 0.0; break;
        case 5: *r1 = *r1 - b4 * *r0 - b6 * *r2; *r0 = 0.0; *r2 = 0.0; break;
        case 6: *r0 = *r0 - b4 * *r1 - b6 * *r2; *r1 = 0.0; *r2 = 0.0; break;
        case 7: *r0 = 0.0; *r1 = 0.0; *r2 = 0.0; break;
        default: break;
    }
}

// ===========================================================================
// ElmGMR (flowsolver/src/elmgmr.f90:82-555)
// ===========================================================================
extern "C" int orc_elmgmr(const orc_params* p, int nshg, int numnp, int nelem, const int* ien, const double* x,
                          const double* y, const double* ac, const int* iBC, const double* BC,
                          int nface, const int* ienb, const int* iBCB, const double* BCB,
                          int ncoupled, const int* srflist, const double* coef1, const double* coef2,
                          const int* ndsurf, const double* NABI,
                          const int* colm, const int* rowp, long long nnz,
                          double* res, double* lhsK, double* lhsP, int lhs,
                          double* qres_out, double* rmass_out) {
    if (!p || !ien || !x || !y || !ac || !res) return ORC_ERR_ARG;
    if (p->itau != 0 || p->flmpl != 0.0 || p->flmpr != 0.0 || (p->iconvflow != 1 && p->iconvflow != 2) ||
        (p->idiff != 0 && p->idiff != 1))
        return ORC_ERR_UNSUPPORTED;
    const int ibksiz = p->ibksiz > 0 ? p->ibksiz : 255;
    const int nthr = nthreads_of(p);
    // ---- diffusive-flux reconstruction: AsIq + qpbc (elmgmr.f90:82-118) ----
    std::vector<double> qres((size_t)nshg * 9, 0.0), rmass(nshg, 0.0);
    auto gather = [&](int e, const double* arr, double yl[4][4], double xl[4][3], double acl[4][4]) {
        for (int a = 0; a < 4; ++a) {
            int nd = ien[a * nelem + e] - 1;
            if (yl) {
                // localy: yl(:,:,1) = y(:,4), yl(:,:,2:4) = y(:,1:3) (localy.f90:54-64)
                yl[a][0] = arr[3 * (size_t)nshg + nd];
                yl[a][1] = arr[0 * (size_t)nshg + nd];
                yl[a][2] = arr[1 * (size_t)nshg + nd];
                yl[a][3] = arr[2 * (size_t)nshg + nd];
            }
            if (acl) {
                acl[a][0] = ac[3 * (size_t)nshg + nd];
                acl[a][1] = ac[0 * (size_t)nshg + nd];
                acl[a][2] = ac[1 * (size_t)nshg + nd];
                acl[a][3] = ac[2 * (size_t)nshg + nd];
            }
            if (xl)
                for (int d = 0; d < 3; ++d) xl[a][d] = x[d * (size_t)numnp + nd];
        }
    };
    const int nblk = (nelem + ibksiz - 1) / ibksiz;
    if (p->idiff == 1) {
        // blocks are computed in parallel into block buffers, scattered in block order
        const int chunk = 64;
        std::vector<double> qlbuf((size_t)chunk * ibksiz * 36), rmbuf((size_t)chunk * ibksiz * 4);
        for (int b0 = 0; b0 < nblk; b0 += chunk) {
            int b1 = std::min(nblk, b0 + chunk);
#pragma omp parallel for num_threads(nthr) schedule(static)
            for (int b = b0; b < b1; ++b) {
                int e0 = b * ibksiz, e1 = std::min(nelem, e0 + ibksiz);
                for (int e = e0; e < e1; ++e) {
                    double yl[4][4], xl[4][3], ql[4][9], rm[4];
                    gather(e, y, yl, xl, nullptr);
                    e3q_elem(p, yl, xl, ql, rm);
                    size_t off = ((size_t)(b - b0) * ibksiz + (e - e0));
                    for (int a = 0; a < 4; ++a) {
                        for (int k = 0; k < 9; ++k) qlbuf[off * 36 + a * 9 + k] = ql[a][k];
                        rmbuf[off * 4 + a] = rm[a];
                    }
                }
            }
            for (int b = b0; b < b1; ++b) {
                int e0 = b * ibksiz, e1 = std::min(nelem, e0 + ibksiz);
                // local scatter order: dof j, node i, element (local.f90:68-75)
                for (int k = 0; k < 9; ++k)
                    for (int a = 0; a < 4; ++a)
                        for (int e = e0; e < e1; ++e) {
                            size_t off = ((size_t)(b - b0) * ibksiz + (e - e0));
                            int nd = ien[a * nelem + e] - 1;
                            qres[(size_t)k * nshg + nd] = qres[(size_t)k * nshg + nd] + qlbuf[off * 36 + a * 9 + k];
                        }
                for (int a = 0; a < 4; ++a)
                    for (int e = e0; e < e1; ++e) {
                        size_t off = ((size_t)(b - b0) * ibksiz + (e - e0));
                        int nd = ien[a * nelem + e] - 1;
                        rmass[nd] = rmass[nd] + rmbuf[off * 4 + a];
                    }
            }
        }
        // qpbc (qpbc.f90:46-71), no periodic nodes on this path
        for (int i = 0; i < nshg; ++i) rmass[i] = 1.0 / rmass[i];
        for (int k = 0; k < 9; ++k)
            for (int i = 0; i < nshg; ++i) qres[(size_t)k * nshg + i] = rmass[i] * qres[(size_t)k * nshg + i];
    }
    if (qres_out) std::memcpy(qres_out, qres.data(), sizeof(double) * (size_t)nshg * 9);
    if (rmass_out) std::memcpy(rmass_out, rmass.data(), sizeof(double) * (size_t)nshg);
    // ---- interior elements (elmgmr.f90:122-255) ----
    std::fill(res, res + (size_t)nshg * 4, 0.0);
    if (lhs) {
        std::fill(lhsK, lhsK + (size_t)9 * nnz, 0.0);
        std::fill(lhsP, lhsP + (size_t)4 * nnz, 0.0);
    }
    {
        const int chunk = 32;
        const size_t per = 16 + (lhs ? (144 + 64) : 0);
        std::vector<double> buf((size_t)chunk * ibksiz * per);
        for (int b0 = 0; b0 < nblk; b0 += chunk) {
            int b1 = std::min(nblk, b0 + chunk);
#pragma omp parallel for num_threads(nthr) schedule(static)
            for (int b = b0; b < b1; ++b) {
                int e0 = b * ibksiz, e1 = std::min(nelem, e0 + ibksiz);
                for (int e = e0; e < e1; ++e) {
                    double yl[4][4], acl[4][4], xl[4][3], ql[4][9];
                    gather(e, y, yl, xl, acl);
                    for (int a = 0; a < 4; ++a) {
                        int nd = ien[a * nelem + e] - 1;
                        for (int k = 0; k < 9; ++k) ql[a][k] = qres[(size_t)k * nshg + nd];
                    }
                    double rl[4][4] = {{0}}, xK[9][4][4] = {{{0}}}, xG[4][4][4] = {{{0}}};
                    e3_elem(p, yl, acl, xl, ql, lhs, rl, xK, xG);
                    double* o = &buf[((size_t)(b - b0) * ibksiz + (e - e0)) * per];
                    std::memcpy(o, rl, sizeof(rl));
                    if (lhs) {
                        std::memcpy(o + 16, xK, sizeof(xK));
                        std::memcpy(o + 16 + 144, xG, sizeof(xG));
                    }
                }
            }
            for (int b = b0; b < b1; ++b) {
                int e0 = b * ibksiz, e1 = std::min(nelem, e0 + ibksiz);
                auto O = [&](int e) { return &buf[((size_t)(b - b0) * ibksiz + (e - e0)) * per]; };
                for (int j = 0; j < 4; ++j)
                    for (int a = 0; a < 4; ++a)
                        for (int e = e0; e < e1; ++e) {
                            int nd = ien[a * nelem + e] - 1;
                            res[(size_t)j * nshg + nd] = res[(size_t)j * nshg + nd] + O(e)[a * 4 + j];
                        }
                if (!lhs) continue;
                // bc3LHS (elmgmr.f90:224-225), then fillsparseI (fillsparse.f90:29-60)
                for (int e = e0; e < e1; ++e) {
                    double* xK = O(e) + 16;
                    const double* xG = O(e) + 16 + 144;
                    const int ndl[4] = {ien[e] - 1, ien[nelem + e] - 1, ien[2 * nelem + e] - 1, ien[3 * nelem + e] - 1};
                    bc3lhs_elem(nshg, iBC, BC, ndl, xK);
                    for (int aa = 0; aa < 4; ++aa) {
                        int i = ien[aa * nelem + e];
                        int c = colm[i - 1];
                        int n = colm[i] - c;
                        for (int bb = 0; bb < 4; ++bb) {
                            long long k = sparseloc(&rowp[c - 1], n, ien[bb * nelem + e]) + c - 1;   // 1-based
                            double* K = &lhsK[9 * (k - 1)];
                            double* P = &lhsP[4 * (k - 1)];
                            for (int cc = 0; cc < 9; ++cc) K[cc] = K[cc] + xK[cc * 16 + aa * 4 + bb];
                            for (int cc = 0; cc < 4; ++cc) P[cc] = P[cc] + xG[cc * 16 + aa * 4 + bb];
                        }
                    }
                }
            }
        }
    }
    // ---- boundary elements: AsBMFG (elmgmr.f90:325-460), residual only for rigid walls ----
    {
        const int nbblk = (nface + ibksiz - 1) / ibksiz;
        for (int b = 0; b < nbblk; ++b) {
            int f0 = b * ibksiz, f1 = std::min(nface, f0 + ibksiz);
            std::vector<double> rlb((size_t)(f1 - f0) * 16);
            for (int f = f0; f < f1; ++f) {
                double yl[4][4], xlb[4][3], bcb[3][6];
                for (int a = 0; a < 4; ++a) {
                    int nd = ienb[a * nface + f] - 1;
                    yl[a][0] = y[3 * (size_t)nshg + nd];
                    yl[a][1] = y[0 * (size_t)nshg + nd];
                    yl[a][2] = y[1 * (size_t)nshg + nd];
                    yl[a][3] = y[2 * (size_t)nshg + nd];
                    for (int d = 0; d < 3; ++d) xlb[a][d] = x[d * (size_t)numnp + nd];
                }
                for (int n = 0; n < 3; ++n)
                    for (int c = 0; c < 6; ++c) bcb[n][c] = BCB ? BCB[((size_t)c * 3 + n) * nface + f] : 0.0;
                double rl[4][4] = {{0}};
                e3b_face(p, yl, xlb, iBCB[f], bcb, rl);
                std::memcpy(&rlb[(size_t)(f - f0) * 16], rl, sizeof(rl));
            }
            for (int j = 0; j < 4; ++j)
                for (int a = 0; a < 4; ++a)
                    for (int f = f0; f < f1; ++f) {
                        int nd = ienb[a * nface + f] - 1;
                        res[(size_t)j * nshg + nd] = res[(size_t)j * nshg + nd] + rlb[(size_t)(f - f0) * 16 + a * 4 + j];
                    }
            // rigid wall: zero boundary tangent; bc3LHS still puts 1 on the
            // constrained diagonal entries of partially constrained nodes
            // before fillsparseI (elmgmr.f90:428-438)
            if (lhs) {
                for (int f = f0; f < f1; ++f) {
                    double xK[144] = {0.0};
                    int ndl[4];
                    for (int a = 0; a < 4; ++a) ndl[a] = ienb[a * nface + f] - 1;
                    bc3lhs_elem(nshg, iBC, BC, ndl, xK);
                    for (int aa = 0; aa < 4; ++aa) {
                        int i = ndl[aa] + 1;
                        int c = colm[i - 1];
                        int n = colm[i] - c;
                        for (int bb = 0; bb < 4; ++bb) {
                            long long k = sparseloc(&rowp[c - 1], n, ndl[bb] + 1) + c - 1;
                            double* K = &lhsK[9 * (k - 1)];
                            for (int cc = 0; cc < 9; ++cc) K[cc] = K[cc] + xK[cc * 16 + aa * 4 + bb];
                        }
                    }
                }
            }
        }
    }
    // ---- ElmpvsQ, GRCR branch (elmgmr.f90:1271-1330) with sign = -1 ----
    if (ncoupled > 0) {
        std::vector<double> pk(ncoupled);
        orc_getflowq(nshg, y, ncoupled, srflist, ndsurf, NABI, pk.data());
        for (int j = 0; j < ncoupled; ++j) {
            double pj = -1.0 * (pk[j] * coef1[j]);
            pj = pj - coef2[j];
            pk[j] = pj;
        }
        for (int i = 0; i < nshg; ++i)
            for (int k = 0; k < ncoupled; ++k)
                if (srflist[k] == ndsurf[i])
                    for (int d = 0; d < 3; ++d)
                        res[(size_t)d * nshg + i] = res[(size_t)d * nshg + i] + pk[k] * NABI[(size_t)d * nshg + i];
    }
    // ---- bc3Res (bc3res.f90:30-124) ----
    for (int i = 0; i < nshg; ++i) {
        if ((iBC[i] >> 2) & 1) res[3 * (size_t)nshg + i] = 0.0;
        bc3res_partial(nshg, iBC, BC, i, res);
        if ((iBC[i] >> 11) & 1) {
            res[0 * (size_t)nshg + i] = 0.0;
            res[1 * (size_t)nshg + i] = 0.0;
            res[2 * (size_t)nshg + i] = 0.0;
        }
    }
    return ORC_OK;
}

// ===========================================================================
// ElmGMRSclr (flowsolver/src/elmgmr.f90:599-822): residual and tangent of the
// advection-diffusion equation of scalar isclr with diffusivity diffus
// (getdiffsclr, getdiff.f90:145-174), no sources (nosource = 1: the source
// call in e3ivarSclr is commented out in the reference, e3ivar.f90:670-680),
// convective form with the flow velocity (consrv_sclr_conv_vel = 0), SUPG
// weak form (ivart = 2), no discontinuity capturing (idcsclr = 0).
//   s, sdot (nshg): the scalar and its time derivative (y(:,5+isclr),
//   ac(:,5+isclr)); y (nshg, 4) supplies the velocity.
//   bcbs (nface, 3): prescribed scalar flux per face node, read where
//   ibits(iBCB(:,1), 4+isclr) is set (e3b.f90:700-715); may be NULL.
// ===========================================================================

// e3qSclr + e3qvarSclr for one element (e3q.f90:215-300, e3qvar.f90:149-180)
void e3q_sclr_elem(double diffus, int idiff, const double sl[4], const double xl[4][3], double ql[4][3],
                   double rm[4]) {
    const Tables& T = tables();
    for (int a = 0; a < 4; ++a) {
        ql[a][0] = ql[a][1] = ql[a][2] = 0.0;
        rm[a] = 0.0;
    }
    for (int intp = 0; intp < 4; ++intp) {
        const double* shapeVar = T.shp[intp];
        double dxidx[3][3], shg[4][3], W;
        e3metric(xl, T.shgl[intp], T.Qwt[intp], dxidx, shg, &W);
        double gradT[3] = {0.0, 0.0, 0.0};
        for (int n = 0; n < 4; ++n)
            for (int k = 0; k < 3; ++k) gradT[k] = gradT[k] + shg[n][k] * sl[n];
        double qdi[3];
        for (int k = 0; k < 3; ++k) qdi[k] = diffus * gradT[k];
        for (int i = 0; i < 4; ++i)
            for (int k = 0; k < 3; ++k) ql[i][k] = ql[i][k] + shapeVar[i] * W * qdi[k];
        if (idiff == 1)
            for (int i = 0; i < 4; ++i) rm[i] = rm[i] + shapeVar[i] * W;
    }
}

// e3Sclr for one element (e3.f90:183-330): e3ivarSclr (e3ivar.f90:492-700),
// e3StabSclr (e3stab.f90:542-600), e3ResSclr (e3res.f90:300-370), e3LHSSclr
// (e3lhs.f90:416-528).  ul[n] = (u, v, w); rl[a]; xS[a][b] = xSebe(:,a,b).
void e3_sclr_elem(const orc_params* p, double diffus, const double ul[4][3], const double sl[4],
                  const double sdl[4], const double xl[4][3], const double ql[4][3], int lhs, double rl[4],
                  double xS[4][4]) {
    const Tables& T = tables();
    for (int intp = 0; intp < 4; ++intp) {
        const double* shpfun = T.shp[intp];
        // e3ivarSclr
        double u1 = 0.0, u2 = 0.0, u3 = 0.0, Sclr = 0.0;
        for (int n = 0; n < 4; ++n) {
            u1 = u1 + shpfun[n] * ul[n][0];
            u2 = u2 + shpfun[n] * ul[n][1];
            u3 = u3 + shpfun[n] * ul[n][2];
            Sclr = Sclr + shpfun[n] * sl[n];
        }
        double Sdot = 0.0;
        for (int n = 0; n < 4; ++n) Sdot = Sdot + shpfun[n] * sdl[n];
        double dxidx[3][3], shg[4][3], W;
        e3metric(xl, T.shgl[intp], T.Qwt[intp], dxidx, shg, &W);
        double gradS[3] = {0.0, 0.0, 0.0};
        for (int n = 0; n < 4; ++n)
            for (int k = 0; k < 3; ++k) gradS[k] = gradS[k] + shg[n][k] * sl[n];
        double divS = 0.0;
        if (p->idiff >= 1)
            for (int n = 0; n < 4; ++n)
                divS = divS + shg[n][0] * ql[n][0] + shg[n][1] * ql[n][1] + shg[n][2] * ql[n][2];
        const double srcR = 0.0, srcL = 0.0, srcRat = 0.0;  // nosource
        const double rLS = (Sdot + (u1 * gradS[0] + u2 * gradS[1] + u3 * gradS[2])) - divS;
        // e3StabSclr, ivart = 2, ipord = 1
        double g[6];
        e3gijd(dxidx, g);
        const double fff = 9.0;
        const double dts = p->Dtgl * p->dtsfct;
        double tauT = (2.0 * dts) * (2.0 * dts) + srcRat * srcRat + u1 * (g[0] * u1 + g[3] * u2 + g[5] * u3) +
                      u2 * (g[3] * u1 + g[1] * u2 + g[4] * u3) + u3 * (g[5] * u1 + g[4] * u2 + g[2] * u3) +
                      fff * (diffus * diffus) *
                          (g[0] * g[0] + g[1] * g[1] + g[2] * g[2] + 2.0 * (g[3] * g[3] + g[4] * g[4] + g[5] * g[5]));
        const double tauS = 1.0 / std::sqrt(tauT);
        // e3ResSclr
        const double tmps = 1.0 - p->flmpr, rcp = 1.0;
        const double rNa = rcp * (tmps * Sdot + u1 * gradS[0] + u2 * gradS[1] + u3 * gradS[2]) - srcR;
        const double tmp = rcp * tauS * (rLS - srcR);
        const double rGNa[3] = {diffus * gradS[0] + u1 * tmp, diffus * gradS[1] + u2 * tmp, diffus * gradS[2] + u3 * tmp};
        for (int aa = 0; aa < 4; ++aa)
            rl[aa] = rl[aa] - W * (shpfun[aa] * rNa + shg[aa][0] * rGNa[0] + shg[aa][1] * rGNa[1] + shg[aa][2] * rGNa[2]);
        // e3LHSSclr
        if (!lhs) continue;
        const double lhsFct = p->alfi * p->gami * p->Delt;
        const double tauSo = tauS;
        const double tauSl = lhsFct * W * tauS;
        const double kptmp = lhsFct * W * diffus;
        const double tsFct = p->almi * W * (1.0 - p->flmpl);
        const double src = srcL * W * lhsFct;
        for (int b = 0; b < 4; ++b) {
            const double t1 = W * (u1 * shg[b][0] + u2 * shg[b][1] + u3 * shg[b][2]);
            const double t2 = t1 * tauSo;
            for (int aa = 0; aa < 4; ++aa) {
                const double tmp1 = shpfun[aa] * shpfun[b];
                const double tmp2 = shpfun[aa] * lhsFct;
                xS[aa][b] = xS[aa][b] + tmp1 * (tsFct + src) + tmp2 * t1;
                xS[b][aa] = xS[b][aa] + t2 * shpfun[aa];
            }
        }
        for (int b = 0; b < 4; ++b) {
            const double tb = tauSl * (u1 * shg[b][0] + u2 * shg[b][1] + u3 * shg[b][2]);
            const double t1[3] = {kptmp * shg[b][0] + u1 * tb, kptmp * shg[b][1] + u2 * tb, kptmp * shg[b][2] + u3 * tb};
            xS[b][b] = xS[b][b] + t1[0] * shg[b][0] + t1[1] * shg[b][1] + t1[2] * shg[b][2];
            for (int aa = b + 1; aa < 4; ++aa) {
                const double v = t1[0] * shg[aa][0] + t1[1] * shg[aa][1] + t1[2] * shg[aa][2];
                xS[aa][b] = xS[aa][b] + v;
                xS[b][aa] = xS[b][aa] + v;
            }
        }
    }
}

// e3bSclr + e3bvarSclr for one linear-tet boundary face (e3b.f90:626-720,
// e3bvar.f90:1033-1200), Navier = 1; rl[0..2] for the three face nodes.
void e3b_sclr_face(double diffus, int isclr, const double sl[4], const double xlb[4][3], int ibcb_bits,
                   const double bcbs[3], double rl[4]) {
    const Tables& T = tables();
    for (int intp = 0; intp < 3; ++intp) {
        const double* shapeVar = T.shpb[intp];
        double d[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int n = 0; n < 4; ++n)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) d[i][j] = d[i][j] + xlb[n][i] * T.shglb[intp][j][n];
        double v1[3], v2[3];
        for (int i = 0; i < 3; ++i) {
            v1[i] = xlb[1][i] - xlb[0][i];
            v2[i] = xlb[2][i] - xlb[0][i];
        }
        const double temp1 = v1[1] * v2[2] - v2[1] * v1[2];
        const double temp2 = v2[0] * v1[2] - v1[0] * v2[2];
        const double temp3 = v1[0] * v2[1] - v2[0] * v1[1];
        const double temp = 1.0 / std::sqrt(temp1 * temp1 + temp2 * temp2 + temp3 * temp3);
        const double bn[3] = {temp1 * temp, temp2 * temp, temp3 * temp};
        const double WdetJb = T.Qwtb[intp] / (4.0 * temp);
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
        for (int n = 0; n < 4; ++n)
            for (int k = 0; k < 3; ++k) gl[k] = gl[k] + T.shglb[intp][k][n] * sl[n];
        double gS[3];
        for (int k = 0; k < 3; ++k) gS[k] = dx[0][k] * gl[0] + dx[1][k] * gl[1] + dx[2][k] * gl[2];
        double flux = diffus * (gS[0] * bn[0] + gS[1] * bn[1] + gS[2] * bn[2]);
        if ((ibcb_bits >> (4 + isclr)) & 1) {
            flux = 0.0;
            for (int n = 0; n < 3; ++n) flux = flux + shapeVar[n] * bcbs[n];
        }
        const double rNa = -WdetJb * flux;
        for (int n = 0; n < 3; ++n) rl[n] = rl[n] - shapeVar[n] * rNa;
    }
}

extern "C" int orc_elmgmr_sclr(const orc_params* p, int isclr, double diffus, int nshg, int numnp, int nelem,
                               const int* ien, const double* x, const double* y, const double* s,
                               const double* sdot, const int* iBC, int nface, const int* ienb, const int* iBCB,
                               const double* bcbs, const int* colm, const int* rowp, long long nnz, double* res,
                               double* lhsS, int lhs, double* qres_out) {
    if (!p || !ien || !x || !y || !s || !sdot || !res || isclr < 1 || isclr > 4) return ORC_ERR_ARG;
    if (p->flmpl != 0.0 || p->flmpr != 0.0 || (p->idiff != 0 && p->idiff != 1)) return ORC_ERR_UNSUPPORTED;
    const int ibksiz = p->ibksiz > 0 ? p->ibksiz : 255;
    const int nblk = (nelem + ibksiz - 1) / ibksiz;
    auto node = [&](int e, int a) { return ien[a * nelem + e] - 1; };
    auto gather = [&](int e, double ul[4][3], double sl[4], double sdl[4], double xl[4][3]) {
        for (int a = 0; a < 4; ++a) {
            const int nd = node(e, a);
            for (int d = 0; d < 3; ++d) {
                ul[a][d] = y[(size_t)d * nshg + nd];
                xl[a][d] = x[(size_t)d * numnp + nd];
            }
            sl[a] = s[nd];
            sdl[a] = sdot[nd];
        }
    };
    // ---- diffusive flux: AsIqSclr + qpbcSclr (elmgmr.f90:650-683; qpbc.f90:118-175) ----
    std::vector<double> qres((size_t)nshg * 3, 0.0), rmass(nshg, 0.0);
    if (p->idiff == 1) {
        for (int b = 0; b < nblk; ++b) {
            const int e0 = b * ibksiz, e1 = std::min(nelem, e0 + ibksiz);
            std::vector<double> qb((size_t)(e1 - e0) * 12), rb((size_t)(e1 - e0) * 4);
            for (int e = e0; e < e1; ++e) {
                double ul[4][3], sl[4], sdl[4], xl[4][3], ql[4][3], rm[4];
                gather(e, ul, sl, sdl, xl);
                e3q_sclr_elem(diffus, p->idiff, sl, xl, ql, rm);
                for (int a = 0; a < 4; ++a) {
                    for (int k = 0; k < 3; ++k) qb[(size_t)(e - e0) * 12 + a * 3 + k] = ql[a][k];
                    rb[(size_t)(e - e0) * 4 + a] = rm[a];
                }
            }
            // local scatter order: dof k, node a, element e (local.f90:68-75)
            for (int k = 0; k < 3; ++k)
                for (int a = 0; a < 4; ++a)
                    for (int e = e0; e < e1; ++e) {
                        const int nd = node(e, a);
                        qres[(size_t)k * nshg + nd] = qres[(size_t)k * nshg + nd] + qb[(size_t)(e - e0) * 12 + a * 3 + k];
                    }
            for (int a = 0; a < 4; ++a)
                for (int e = e0; e < e1; ++e) {
                    const int nd = node(e, a);
                    rmass[nd] = rmass[nd] + rb[(size_t)(e - e0) * 4 + a];
                }
        }
        for (int i = 0; i < nshg; ++i) rmass[i] = 1.0 / rmass[i];
        for (int k = 0; k < 3; ++k)
            for (int i = 0; i < nshg; ++i) qres[(size_t)k * nshg + i] = rmass[i] * qres[(size_t)k * nshg + i];
    }
    if (qres_out) std::memcpy(qres_out, qres.data(), sizeof(double) * (size_t)nshg * 3);
    // ---- interior elements: AsIGMRSclr + fillsparseSclr (elmgmr.f90:698-745) ----
    std::fill(res, res + nshg, 0.0);
    if (lhs) std::fill(lhsS, lhsS + nnz, 0.0);
    for (int b = 0; b < nblk; ++b) {
        const int e0 = b * ibksiz, e1 = std::min(nelem, e0 + ibksiz);
        std::vector<double> rb((size_t)(e1 - e0) * 4), xb((size_t)(e1 - e0) * 16);
        for (int e = e0; e < e1; ++e) {
            double ul[4][3], sl[4], sdl[4], xl[4][3], ql[4][3];
            gather(e, ul, sl, sdl, xl);
            for (int a = 0; a < 4; ++a)
                for (int k = 0; k < 3; ++k) ql[a][k] = qres[(size_t)k * nshg + node(e, a)];
            double rl[4] = {0, 0, 0, 0}, xS[4][4] = {{0}};
            e3_sclr_elem(p, diffus, ul, sl, sdl, xl, ql, lhs, rl, xS);
            for (int a = 0; a < 4; ++a) {
                rb[(size_t)(e - e0) * 4 + a] = rl[a];
                for (int c = 0; c < 4; ++c) xb[(size_t)(e - e0) * 16 + a * 4 + c] = xS[a][c];
            }
        }
        for (int a = 0; a < 4; ++a)
            for (int e = e0; e < e1; ++e) {
                const int nd = node(e, a);
                res[nd] = res[nd] + rb[(size_t)(e - e0) * 4 + a];
            }
        if (!lhs) continue;
        // fillsparseSclr (fillsparse.f90:167-200)
        for (int e = e0; e < e1; ++e)
            for (int aa = 0; aa < 4; ++aa) {
                const int i = ien[aa * nelem + e];
                const int c = colm[i - 1];
                const int n = colm[i] - c;
                for (int bb = 0; bb < 4; ++bb) {
                    const long long k = sparseloc(&rowp[c - 1], n, ien[bb * nelem + e]) + c - 1;
                    lhsS[k - 1] = lhsS[k - 1] + xb[(size_t)(e - e0) * 16 + aa * 4 + bb];
                }
            }
    }
    // ---- boundary elements: AsBSclr (elmgmr.f90:772-800) ----
    const int nbblk = (nface + ibksiz - 1) / ibksiz;
    for (int b = 0; b < nbblk; ++b) {
        const int f0 = b * ibksiz, f1 = std::min(nface, f0 + ibksiz);
        std::vector<double> rb((size_t)(f1 - f0) * 4);
        for (int f = f0; f < f1; ++f) {
            double sl[4], xlb[4][3], bc[3] = {0.0, 0.0, 0.0};
            for (int a = 0; a < 4; ++a) {
                const int nd = ienb[a * nface + f] - 1;
                sl[a] = s[nd];
                for (int d = 0; d < 3; ++d) xlb[a][d] = x[(size_t)d * numnp + nd];
            }
            if (bcbs)
                for (int n = 0; n < 3; ++n) bc[n] = bcbs[(size_t)n * nface + f];
            double rl[4] = {0, 0, 0, 0};
            e3b_sclr_face(diffus, isclr, sl, xlb, iBCB[f], bc, rl);
            for (int a = 0; a < 4; ++a) rb[(size_t)(f - f0) * 4 + a] = rl[a];
        }
        for (int a = 0; a < 4; ++a)
            for (int f = f0; f < f1; ++f) {
                const int nd = ienb[a * nface + f] - 1;
                res[nd] = res[nd] + rb[(size_t)(f - f0) * 4 + a];
            }
    }
    // ---- bc3ResSclr (bc3res.f90:138-160) ----
    for (int i = 0; i < nshg; ++i)
        if ((iBC[i] >> (isclr + 5)) & 1) res[i] = 0.0;
    return ORC_OK;
}

extern "C" int orc_getflowq(int nshg, const double* y, int nsrf, const int* srflist, const int* ndsurf,
                            const double* NABI, double* q) {
    for (int k = 0; k < nsrf; ++k) q[k] = 0.0;
    for (int i = 0; i < nshg; ++i)
        for (int k = 0; k < nsrf; ++k)
            if (srflist[k] == ndsurf[i])
                for (int j = 0; j < 3; ++j) q[k] = q[k] + NABI[(size_t)j * nshg + i] * y[(size_t)j * nshg + i];
    return ORC_OK;
}

// ===========================================================================
// SolFlow packing (flowsolver/src/solfar.f90:210-232)
// ===========================================================================
extern "C" int orc_solflow_pack(int nshg, long long nnz, const int* colm, const int* rowp, const double* res,
                                const double* lhsK, const double* lhsP, double* Res4, double* Val4) {
    for (int i = 0; i < nshg; ++i)
        for (int d = 0; d < 4; ++d) Res4[4 * (size_t)i + d] = res[(size_t)d * nshg + i];
    for (long long i = 0; i < nnz; ++i) {
        double* V = &Val4[16 * i];
        const double* K = &lhsK[9 * i];
        const double* P = &lhsP[4 * i];
        V[0] = K[0]; V[1] = K[1]; V[2] = K[2];
        V[4] = K[3]; V[5] = K[4]; V[6] = K[5];
        V[8] = K[6]; V[9] = K[7]; V[10] = K[8];
        V[12] = P[0]; V[13] = P[1]; V[14] = P[2];
        V[15] = P[3];
    }
    for (int i = 1; i <= nshg; ++i) {
        for (int j = colm[i - 1]; j <= colm[i] - 1; ++j) {
            int k = rowp[j - 1];
            for (int l = colm[k - 1]; l <= colm[k] - 1; ++l) {
                if (rowp[l - 1] == i) {
                    Val4[16 * (size_t)(l - 1) + 3] = -lhsP[4 * (size_t)(j - 1) + 0];
                    Val4[16 * (size_t)(l - 1) + 7] = -lhsP[4 * (size_t)(j - 1) + 1];
                    Val4[16 * (size_t)(l - 1) + 11] = -lhsP[4 * (size_t)(j - 1) + 2];
                    break;
                }
            }
        }
    }
    return ORC_OK;
}

// ===========================================================================
// memLS (flowsolver/src/memLS.f90)
// ===========================================================================
namespace {

const int LS_TYPE_CG = 1, LS_TYPE_GMRES = 2, LS_TYPE_NS = 3;
const int BC_TYPE_Dir = 0, BC_TYPE_Neu = 1;
const int BCOP_TYPE_ADD = 0, BCOP_TYPE_PRE = 1;
int g_memls_threads = 1;

struct Face {
    double nS = 0, res = 0;
    std::vector<double> val, valM;   // (dof, nNo)
    bool foC = false, coupledFlag = false, sharedFlag = false, incFlag = true;
    int nNo = 0, dof = 0, bGrp = BC_TYPE_Dir;
    std::vector<int> glob;   // 0-based
};

struct Lhs {
    int gnNo = 0, nNo = 0, nFaces = 0, mynNo = 0;
    long long nnz = 0;
    std::vector<int> colPtr;         // 0-based column index
    std::vector<long long> rowS, rowE;   // 0-based inclusive range
    std::vector<long long> diagPtr;
    std::vector<int> map;
    std::vector<Face> face;
};

struct Ls {
    orc_subls GM, CG, RI;
    int LS_type = LS_TYPE_NS, Resm = 0, Resc = 0;
};

// ---- vector kernels: node-order sums as in NORMV/NORMS/DOTV/DOTS (memLS.f90:2240-2378) ----
double DOTV(int dof, int nNo, const double* U, const double* V) {
    double s = 0.0;
    if (g_memls_threads > 1) {
#pragma omp parallel for reduction(+ : s) num_threads(g_memls_threads) schedule(static)
        for (int i = 0; i < nNo; ++i) {
            double t = 0.0;
            for (int d = 0; d < dof; ++d) t = t + U[(size_t)dof * i + d] * V[(size_t)dof * i + d];
            s += t;
        }
        return s;
    }
    for (int i = 0; i < nNo; ++i) {
        const double* u = &U[(size_t)dof * i];
        const double* v = &V[(size_t)dof * i];
        switch (dof) {
            case 1: s = s + u[0] * v[0]; break;
            case 2: s = s + u[0] * v[0] + u[1] * v[1]; break;
            case 3: s = s + u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; break;
            case 4: s = s + u[0] * v[0] + u[1] * v[1] + u[2] * v[2] + u[3] * v[3]; break;
            default: {
                double t = 0.0;
                for (int d = 0; d < dof; ++d) t = t + u[d] * v[d];
                s = s + t;
            }
        }
    }
    return s;
}
double NORMV(int dof, int nNo, const double* U) { return std::sqrt(DOTV(dof, nNo, U, U)); }
double DOTS(int nNo, const double* U, const double* V) { return DOTV(1, nNo, U, V); }
double NORMS(int nNo, const double* U) { return std::sqrt(DOTV(1, nNo, U, U)); }

// SPARMULVV/VS/SV/SS (memLS.f90:2024-2236)
void SPARMULVV(int dof, const Lhs& L, const double* K, const double* U, double* KU) {
#pragma omp parallel for num_threads(g_memls_threads) schedule(static)
    for (int i = 0; i < L.nNo; ++i) {
        double ku[4] = {0, 0, 0, 0};
        for (long long j = L.rowS[i]; j <= L.rowE[i]; ++j) {
            const double* k = &K[(size_t)dof * dof * j];
            const double* u = &U[(size_t)dof * L.colPtr[j]];
            if (dof == 3) {
                ku[0] = ku[0] + k[0] * u[0] + k[1] * u[1] + k[2] * u[2];
                ku[1] = ku[1] + k[3] * u[0] + k[4] * u[1] + k[5] * u[2];
                ku[2] = ku[2] + k[6] * u[0] + k[7] * u[1] + k[8] * u[2];
            } else if (dof == 4) {
                ku[0] = ku[0] + k[0] * u[0] + k[1] * u[1] + k[2] * u[2] + k[3] * u[3];
                ku[1] = ku[1] + k[4] * u[0] + k[5] * u[1] + k[6] * u[2] + k[7] * u[3];
                ku[2] = ku[2] + k[8] * u[0] + k[9] * u[1] + k[10] * u[2] + k[11] * u[3];
                ku[3] = ku[3] + k[12] * u[0] + k[13] * u[1] + k[14] * u[2] + k[15] * u[3];
            } else if (dof == 2) {
                ku[0] = ku[0] + k[0] * u[0] + k[1] * u[1];
                ku[1] = ku[1] + k[2] * u[0] + k[3] * u[1];
            } else {
                ku[0] = ku[0] + k[0] * u[0];
            }
        }
        for (int d = 0; d < dof; ++d) KU[(size_t)dof * i + d] = ku[d];
    }
}
void SPARMULVS(int dof, const Lhs& L, const double* K, const double* U, double* KU) {
#pragma omp parallel for num_threads(g_memls_threads) schedule(static)
    for (int i = 0; i < L.nNo; ++i) {
        double s = 0.0;
        for (long long j = L.rowS[i]; j <= L.rowE[i]; ++j) {
            const double* k = &K[(size_t)dof * j];
            const double* u = &U[(size_t)dof * L.colPtr[j]];
            if (dof == 3)
                s = s + k[0] * u[0] + k[1] * u[1] + k[2] * u[2];
            else if (dof == 2)
                s = s + k[0] * u[0] + k[1] * u[1];
            else
                s = s + k[0] * u[0];
        }
        KU[i] = s;
    }
}
void SPARMULSV(int dof, const Lhs& L, const double* K, const double* U, double* KU) {
#pragma omp parallel for num_threads(g_memls_threads) schedule(static)
    for (int i = 0; i < L.nNo; ++i) {
        double ku[3] = {0, 0, 0};
        for (long long j = L.rowS[i]; j <= L.rowE[i]; ++j) {
            double u = U[L.colPtr[j]];
            for (int d = 0; d < dof; ++d) ku[d] = ku[d] + K[(size_t)dof * j + d] * u;
        }
        for (int d = 0; d < dof; ++d) KU[(size_t)dof * i + d] = ku[d];
    }
}
void SPARMULSS(const Lhs& L, const double* K, const double* U, double* KU) {
#pragma omp parallel for num_threads(g_memls_threads) schedule(static)
    for (int i = 0; i < L.nNo; ++i) {
        double s = 0.0;
        for (long long j = L.rowS[i]; j <= L.rowE[i]; ++j) s = s + K[j] * U[L.colPtr[j]];
        KU[i] = s;
    }
}

// ADDBCMUL (memLS.f90:206-268), unshared faces
void ADDBCMUL(int op_type, int dof, Lhs& L, const double* X, double* Y) {
    for (int faIn = 0; faIn < L.nFaces; ++faIn) {
        Face& f = L.face[faIn];
        double coef = (op_type == BCOP_TYPE_ADD) ? f.res : -f.res / (1.0 + f.res * f.nS);
        int nsd = std::min(f.dof, dof);
        if (!f.coupledFlag) continue;
        double S = 0.0;
        for (int a = 0; a < f.nNo; ++a) {
            int Ac = f.glob[a];
            for (int i = 0; i < nsd; ++i) S = S + f.valM[(size_t)f.dof * a + i] * X[(size_t)dof * Ac + i];
        }
        S = coef * S;
        for (int a = 0; a < f.nNo; ++a) {
            int Ac = f.glob[a];
            for (int i = 0; i < nsd; ++i) Y[(size_t)dof * Ac + i] = Y[(size_t)dof * Ac + i] + f.valM[(size_t)f.dof * a + i] * S;
        }
    }
}

bool any_coupled(const Lhs& L) {
    for (const Face& f : L.face)
        if (f.coupledFlag) return true;
    return false;
}

// GE (memLS.f90:607-677); A column-major N x N
int GE(int N, const double* A, double* B) {
    if (N == 2) {
        double pivot = A[0] * A[3] - A[1] * A[2];
        double saveEl = (B[0] * A[3] - B[1] * A[2]) / pivot;
        B[1] = (B[1] * A[0] - B[0] * A[1]) / pivot;
        B[0] = saveEl;
        return ORC_OK;
    }
    std::vector<double> C((size_t)N * (N + 1));
    auto c = [&](int i, int j) -> double& { return C[(size_t)j * N + i]; };
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
        if (pivot < 2.0 * 2.220446049250313e-16) return ORC_ERR_SINGULAR;
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
    return ORC_OK;
}

// GMRES (memLS.f90:681-788); Val dof*dof per block, R/X (dof, nNo)
void GMRES(int dof, Lhs& L, orc_subls& ls, const double* Val, const double* R, double* X) {
    const int nNo = L.nNo;
    const size_t n = (size_t)dof * nNo;
    const int sD = ls.sD;
    std::vector<double> h((size_t)(sD + 1) * sD), u(n * (sD + 1)), unCondU(n);
    std::vector<double> y(sD), c(sD), s(sD), err(sD + 1);
    auto H = [&](int i, int j) -> double& { return h[(size_t)j * (sD + 1) + i]; };
    auto U = [&](int k) { return &u[n * k]; };
    double eps = 0.0, tmp;
    const double time = CPUT();
    ls.suc = 0;
    bool coupled = any_coupled(L);
    std::fill(X, X + n, 0.0);
    int i = 0;
    for (int l = 1; l <= ls.mItr; ++l) {
        if (l == 1) {
            std::memcpy(U(0), R, n * sizeof(double));
        } else {
            ls.itr = ls.itr + 1;
            SPARMULVV(dof, L, Val, X, U(0));
            ADDBCMUL(BCOP_TYPE_ADD, dof, L, X, U(0));
            for (size_t t = 0; t < n; ++t) U(0)[t] = R[t] - U(0)[t];
        }
        if (coupled) {
            std::memcpy(unCondU.data(), U(0), n * sizeof(double));
            ADDBCMUL(BCOP_TYPE_PRE, dof, L, unCondU.data(), U(0));
        }
        err[0] = NORMV(dof, nNo, U(0));
        if (l == 1) {
            eps = err[0];
            if (eps <= ls.absTol) {
                ls.callD = 0.0;
                ls.dB = 0.0;
                return;
            }
            ls.iNorm = eps;
            ls.fNorm = eps;
            eps = std::max(ls.absTol, ls.relTol * eps);
        }
        ls.dB = ls.fNorm;
        for (size_t t = 0; t < n; ++t) U(0)[t] = U(0)[t] / err[0];
        for (i = 1; i <= sD; ++i) {
            ls.itr = ls.itr + 1;
            double* ui = U(i - 1);
            double* un = U(i);
            SPARMULVV(dof, L, Val, ui, un);
            ADDBCMUL(BCOP_TYPE_ADD, dof, L, ui, un);
            if (coupled) {
                std::memcpy(unCondU.data(), un, n * sizeof(double));
                ADDBCMUL(BCOP_TYPE_PRE, dof, L, unCondU.data(), un);
            }
            for (int j = 1; j <= i; ++j) {
                double hj = DOTV(dof, nNo, un, U(j - 1));
                H(j - 1, i - 1) = hj;
                const double* uj = U(j - 1);
                for (size_t t = 0; t < n; ++t) un[t] = un[t] - hj * uj[t];
            }
            H(i, i - 1) = NORMV(dof, nNo, un);
            for (size_t t = 0; t < n; ++t) un[t] = un[t] / H(i, i - 1);
            for (int j = 1; j <= i - 1; ++j) {
                tmp = c[j - 1] * H(j - 1, i - 1) + s[j - 1] * H(j, i - 1);
                H(j, i - 1) = -s[j - 1] * H(j - 1, i - 1) + c[j - 1] * H(j, i - 1);
                H(j - 1, i - 1) = tmp;
            }
            tmp = std::sqrt(H(i - 1, i - 1) * H(i - 1, i - 1) + H(i, i - 1) * H(i, i - 1));
            c[i - 1] = H(i - 1, i - 1) / tmp;
            s[i - 1] = H(i, i - 1) / tmp;
            H(i - 1, i - 1) = tmp;
            H(i, i - 1) = 0.0;
            err[i] = -s[i - 1] * err[i - 1];
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
        for (int j = 1; j <= i; ++j) {
            const double* uj = U(j - 1);
            double yj = y[j - 1];
            for (size_t t = 0; t < n; ++t) X[t] = X[t] + uj[t] * yj;
        }
        ls.fNorm = std::fabs(err[i]);
        if (ls.suc) break;
    }
    ls.callD = CPUT() - time + ls.callD;
    ls.dB = 10.0 * std::log(ls.fNorm / ls.dB);
}

// CGRAD (memLS.f90:367-430)
void CGRAD(int dof, Lhs& L, orc_subls& ls, const double* D, const double* G, const double* Lm, double* R) {
    const int nNo = L.nNo;
    std::vector<double> X(nNo, 0.0), P(nNo), SP(nNo), DGP(nNo), GP((size_t)dof * nNo), unCondU((size_t)dof * nNo);
    bool coupled = any_coupled(L);
    const double time = CPUT();
    ls.suc = 0;
    double errO = NORMS(nNo, R);
    ls.iNorm = errO;
    double eps = std::max(ls.absTol, ls.relTol * errO);
    eps = eps * eps;
    double err = errO;
    err = err * err;
    std::memcpy(P.data(), R, nNo * sizeof(double));
    int i;
    for (i = 1; i <= ls.mItr; ++i) {
        if (err < eps) {
            ls.suc = 1;
            break;
        }
        errO = err;
        SPARMULSV(dof, L, G, P.data(), GP.data());
        if (coupled) {
            unCondU = GP;
            ADDBCMUL(BCOP_TYPE_PRE, dof, L, unCondU.data(), GP.data());
        }
        SPARMULVS(dof, L, D, GP.data(), DGP.data());
        SPARMULSS(L, Lm, P.data(), SP.data());
        for (int t = 0; t < nNo; ++t) SP[t] = SP[t] - DGP[t];
        double alpha = errO / DOTS(nNo, P.data(), SP.data());
        for (int t = 0; t < nNo; ++t) X[t] = X[t] + alpha * P[t];
        for (int t = 0; t < nNo; ++t) R[t] = R[t] - alpha * SP[t];
        err = NORMS(nNo, R);
        err = err * err;
        for (int t = 0; t < nNo; ++t) P[t] = R[t] + err / errO * P[t];
    }
    std::memcpy(R, X.data(), nNo * sizeof(double));
    ls.fNorm = std::sqrt(err);
    ls.callD = CPUT() - time + ls.callD;
    ls.dB = 5.0 * std::log(err / errO);
    ls.itr = ls.itr + i - 1;
}

// PRECOND (memLS.f90:1763-1943) for dof = 4
void PRECOND(int dof, Lhs& L, double* Val, double* R, double* W) {
    const int nNo = L.nNo;
    for (int Ac = 0; Ac < nNo; ++Ac) {
        long long d = L.diagPtr[Ac];
        for (int i = 0; i < dof; ++i) W[(size_t)dof * Ac + i] = Val[(size_t)dof * dof * d + i * dof + i];
    }
    for (int Ac = 0; Ac < nNo; ++Ac) {
        long long d = L.diagPtr[Ac];
        for (int i = 0; i < dof; ++i)
            if (W[(size_t)dof * Ac + i] == 0.0) {
                W[(size_t)dof * Ac + i] = 1.0;
                Val[(size_t)dof * dof * d + i * dof + i] = 1.0;
            }
    }
    for (size_t t = 0; t < (size_t)dof * nNo; ++t) W[t] = 1.0 / std::sqrt(std::fabs(W[t]));
    for (int faIn = 0; faIn < L.nFaces; ++faIn) {
        Face& f = L.face[faIn];
        if (!f.incFlag) continue;
        int i = std::min(f.dof, dof);
        if (f.bGrp == BC_TYPE_Dir)
            for (int a = 0; a < f.nNo; ++a) {
                int Ac = f.glob[a];
                for (int k = 0; k < i; ++k) W[(size_t)dof * Ac + k] = W[(size_t)dof * Ac + k] * f.val[(size_t)f.dof * a + k];
            }
    }
    // row scaling
    for (int Ac = 0; Ac < nNo; ++Ac)
        for (long long j = L.rowS[Ac]; j <= L.rowE[Ac]; ++j)
            for (int r = 0; r < dof; ++r)
                for (int c = 0; c < dof; ++c)
                    Val[(size_t)dof * dof * j + r * dof + c] = Val[(size_t)dof * dof * j + r * dof + c] * W[(size_t)dof * Ac + r];
    for (size_t t = 0; t < (size_t)dof * nNo; ++t) R[t] = W[t] * R[t];
    // column scaling
    for (int Ac = 0; Ac < nNo; ++Ac)
        for (long long j = L.rowS[Ac]; j <= L.rowE[Ac]; ++j) {
            int a = L.colPtr[j];
            for (int r = 0; r < dof; ++r)
                for (int c = 0; c < dof; ++c)
                    Val[(size_t)dof * dof * j + r * dof + c] = Val[(size_t)dof * dof * j + r * dof + c] * W[(size_t)dof * a + c];
        }
    for (int Ac = 0; Ac < nNo; ++Ac) {
        long long i = L.diagPtr[Ac];
        for (int a = 0; a < dof; ++a) {
            size_t b = (size_t)dof * dof * i + a * dof + a;
            if (Val[b] == 0.0) Val[b] = 1.0;
        }
    }
    for (int faIn = 0; faIn < L.nFaces; ++faIn) {
        Face& f = L.face[faIn];
        if (f.coupledFlag)
            for (int a = 0; a < f.nNo; ++a) {
                int Ac = f.glob[a];
                for (int i = 0; i < std::min(f.dof, dof); ++i)
                    f.valM[(size_t)f.dof * a + i] = f.val[(size_t)f.dof * a + i] * W[(size_t)dof * Ac + i];
            }
    }
}

// NSSOLVER (memLS.f90:1460-1759), dof = 4
int NSSOLVER(int dof, Lhs& L, Ls& ls, const double* Val, double* Ri) {
    const int nNo = L.nNo;
    const long long nnz = L.nnz;
    const int nsd = dof - 1;
    int iB = ls.RI.mItr;
    int nB = 2 * iB;
    const size_t nv = (size_t)nsd * nNo;
    std::vector<double> Rm(nv), Rc(nNo), Rmi(nv), Rci(nNo), U(nv * iB), P((size_t)nNo * iB), MU(nv * nB),
        MP((size_t)nNo * nB), A((size_t)nB * nB), B(nB), xB(nB);
    for (int a = 0; a < nNo; ++a) {
        for (int d = 0; d < nsd; ++d) Rmi[(size_t)nsd * a + d] = Ri[(size_t)dof * a + d];
        Rci[a] = Ri[(size_t)dof * a + nsd];
    }
    std::fill(xB.begin(), xB.end(), 0.0);
    std::fill(B.begin(), B.end(), 0.0);
    Rm = Rmi;
    Rc = Rci;
    double nv1 = NORMV(nsd, nNo, Rm.data()), ns1 = NORMS(nNo, Rc.data());
    double eps = std::sqrt(std::pow(nv1, 2.0) + std::pow(ns1, 2.0));
    ls.RI.iNorm = eps;
    ls.RI.fNorm = eps;
    ls.CG.callD = 0.0;
    ls.GM.callD = 0.0;
    ls.CG.itr = 0;
    ls.GM.itr = 0;
    ls.RI.callD = CPUT();
    ls.RI.suc = 0;
    eps = std::max(ls.RI.absTol, ls.RI.relTol * eps);
    // DEPART (memLS.f90:1612-1679)
    std::vector<double> mK((size_t)nsd * nsd * nnz), mG((size_t)nsd * nnz), mD((size_t)nsd * nnz), mL(nnz),
        Gt((size_t)nsd * nnz);
    for (long long i = 0; i < nnz; ++i) {
        const double* t = &Val[16 * i];
        double* k = &mK[9 * i];
        k[0] = t[0]; k[1] = t[1]; k[2] = t[2];
        k[3] = t[4]; k[4] = t[5]; k[5] = t[6];
        k[6] = t[8]; k[7] = t[9]; k[8] = t[10];
        mG[3 * i + 0] = t[3]; mG[3 * i + 1] = t[7]; mG[3 * i + 2] = t[11];
        mD[3 * i + 0] = t[12]; mD[3 * i + 1] = t[13]; mD[3 * i + 2] = t[14];
        mL[i] = t[15];
    }
    for (int i = 0; i < nNo; ++i)
        for (long long j = L.rowS[i]; j <= L.rowE[i]; ++j) {
            int k = L.colPtr[j];
            for (long long l = L.rowS[k]; l <= L.rowE[k]; ++l)
                if (L.colPtr[l] == i) {
                    for (int d = 0; d < 3; ++d) Gt[3 * l + d] = -mG[3 * j + d];
                    break;
                }
        }
    // BCPRE (memLS.f90:1683-1716)
    for (Face& f : L.face)
        if (f.coupledFlag) {
            f.nS = 0.0;
            for (int a = 0; a < f.nNo; ++a)
                for (int i = 0; i < nsd; ++i) f.nS = f.nS + std::pow(f.valM[(size_t)f.dof * a + i], 2.0);
        }
    auto Ucol = [&](int k) { return &U[nv * k]; };
    auto Pcol = [&](int k) { return &P[(size_t)nNo * k]; };
    auto MUc = [&](int k) { return &MU[nv * k]; };
    auto MPc = [&](int k) { return &MP[(size_t)nNo * k]; };
    auto Aa = [&](int i, int j) -> double& { return A[(size_t)j * nB + i]; };
    int i, iBB = 0;
    for (i = 1; i <= ls.RI.mItr; ++i) {
        iB = 2 * i - 1;
        iBB = 2 * i;
        ls.RI.dB = ls.RI.fNorm;
        GMRES(nsd, L, ls.GM, mK.data(), Rm.data(), Ucol(i - 1));
        SPARMULVS(nsd, L, mD.data(), Ucol(i - 1), Pcol(i - 1));
        for (int t = 0; t < nNo; ++t) Pcol(i - 1)[t] = Rc[t] - Pcol(i - 1)[t];
        CGRAD(nsd, L, ls.CG, Gt.data(), mG.data(), mL.data(), Pcol(i - 1));
        SPARMULSV(nsd, L, mG.data(), Pcol(i - 1), MUc(iB - 1));
        for (size_t t = 0; t < nv; ++t) MUc(iBB - 1)[t] = Rm[t] - MUc(iB - 1)[t];
        GMRES(nsd, L, ls.GM, mK.data(), MUc(iBB - 1), Ucol(i - 1));
        SPARMULVV(nsd, L, mK.data(), Ucol(i - 1), MUc(iBB - 1));
        ADDBCMUL(BCOP_TYPE_ADD, nsd, L, Ucol(i - 1), MUc(iBB - 1));
        SPARMULSS(L, mL.data(), Pcol(i - 1), MPc(iB - 1));
        SPARMULVS(nsd, L, mD.data(), Ucol(i - 1), MPc(iBB - 1));
        for (int k = iB; k <= iBB; ++k) {
            for (int j = 1; j <= k - 1; ++j) {
                Aa(j - 1, k - 1) = DOTV(nsd, nNo, MUc(j - 1), MUc(k - 1)) + DOTS(nNo, MPc(j - 1), MPc(k - 1));
                Aa(k - 1, j - 1) = Aa(j - 1, k - 1);
            }
            Aa(k - 1, k - 1) = std::pow(NORMV(nsd, nNo, MUc(k - 1)), 2.0) + std::pow(NORMS(nNo, MPc(k - 1)), 2.0);
            B[k - 1] = DOTV(nsd, nNo, MUc(k - 1), Rmi.data()) + DOTS(nNo, MPc(k - 1), Rci.data());
        }
        for (int t = 0; t < iBB; ++t) xB[t] = B[t];
        std::vector<double> Asub((size_t)iBB * iBB);
        for (int c = 0; c < iBB; ++c)
            for (int r = 0; r < iBB; ++r) Asub[(size_t)c * iBB + r] = Aa(r, c);
        if (GE(iBB, Asub.data(), xB.data()) != ORC_OK) return ORC_ERR_SINGULAR;
        double sxb = 0.0;
        for (int t = 0; t < iBB; ++t) sxb = sxb + xB[t] * B[t];
        ls.RI.fNorm = std::sqrt(std::pow(ls.RI.iNorm, 2.0) - sxb);
        if (std::getenv("CRIMSON_ORACLE_VERBOSE"))
            std::fprintf(stderr, "NSSOLVER i=%d fNorm/iNorm=%.6e GM.itr=%d CG.itr=%d\n", i, ls.RI.fNorm / ls.RI.iNorm,
                         ls.GM.itr, ls.CG.itr);
        if (ls.RI.fNorm < eps) {
            ls.RI.suc = 1;
            break;
        }
        for (size_t t = 0; t < nv; ++t) Rm[t] = Rmi[t] - xB[0] * MUc(0)[t];
        for (int t = 0; t < nNo; ++t) Rc[t] = Rci[t] - xB[0] * MPc(0)[t];
        for (int j = 2; j <= iBB; ++j) {
            for (size_t t = 0; t < nv; ++t) Rm[t] = Rm[t] - xB[j - 1] * MUc(j - 1)[t];
            for (int t = 0; t < nNo; ++t) Rc[t] = Rc[t] - xB[j - 1] * MPc(j - 1)[t];
        }
    }
    if (i > ls.RI.mItr) {
        ls.RI.itr = ls.RI.mItr;
    } else {
        ls.RI.itr = i;
        for (int t = 0; t < nNo; ++t) Rc[t] = Rci[t] - xB[0] * MPc(0)[t];
        for (int j = 2; j <= iBB; ++j)
            for (int t = 0; t < nNo; ++t) Rc[t] = Rc[t] - xB[j - 1] * MPc(j - 1)[t];
    }
    ls.Resc = (int)std::lround(100.0 * std::pow(NORMS(nNo, Rc.data()) / ls.RI.fNorm, 2.0));
    ls.Resm = 100 - ls.Resc;
    for (size_t t = 0; t < nv; ++t) Rmi[t] = xB[1] * Ucol(0)[t];
    for (int t = 0; t < nNo; ++t) Rci[t] = xB[0] * Pcol(0)[t];
    for (i = 2; i <= ls.RI.itr; ++i) {
        iB = 2 * i - 1;
        iBB = 2 * i;
        for (size_t t = 0; t < nv; ++t) Rmi[t] = Rmi[t] + xB[iBB - 1] * Ucol(i - 1)[t];
        for (int t = 0; t < nNo; ++t) Rci[t] = Rci[t] + xB[iB - 1] * Pcol(i - 1)[t];
    }
    ls.RI.callD = CPUT() - ls.RI.callD;
    ls.RI.dB = 10.0 * std::log(ls.RI.fNorm / ls.RI.dB);
    for (int a = 0; a < nNo; ++a) {
        for (int d = 0; d < nsd; ++d) Ri[(size_t)dof * a + d] = Rmi[(size_t)nsd * a + d];
        Ri[(size_t)dof * a + nsd] = Rci[a];
    }
    return ORC_OK;
}

}  // namespace

extern "C" void orc_memls_set_threads(int n) { g_memls_threads = n > 0 ? n : 1; }

extern "C" void* orc_memls_ls_create(int LS_type, int present_mask, double relTol, double absTol, int maxItr,
                                     int dimKry, const double* relTolIn, const double* absTolIn,
                                     const int* maxItrIn) {
    // memLS_LS_CREATE (memLS.f90:1379-1440); present_mask bits:
    // 1 relTol, 2 absTol, 4 maxItr, 8 dimKry, 16 relTolIn, 32 absTolIn, 64 maxItrIn
    if (LS_type != LS_TYPE_NS) return nullptr;
    Ls* ls = new Ls();
    std::memset(&ls->GM, 0, sizeof(orc_subls));
    std::memset(&ls->CG, 0, sizeof(orc_subls));
    std::memset(&ls->RI, 0, sizeof(orc_subls));
    ls->LS_type = LS_type;
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
    if (present_mask & 16) {
        ls->GM.relTol = relTolIn[0];
        ls->CG.relTol = relTolIn[1];
    }
    if (present_mask & 32) {
        ls->GM.absTol = absTolIn[0];
        ls->CG.absTol = absTolIn[1];
    }
    if (present_mask & 64) {
        ls->GM.mItr = maxItrIn[0];
        ls->CG.mItr = maxItrIn[1];
    }
    return ls;
}

extern "C" void orc_memls_ls_free(void* ls) { delete static_cast<Ls*>(ls); }

extern "C" void* orc_memls_lhs_create(int gnNo, int nNo, long long nnz, const int* gNodes, const int* rowPtr,
                                      const int* colPtr, int nFaces) {
    // memLS_LHS_CREATE, nTasks = 1 branch (memLS.f90:1113-1143)
    Lhs* L = new Lhs();
    L->gnNo = gnNo;
    L->nNo = nNo;
    L->nnz = nnz;
    L->nFaces = nFaces;
    L->colPtr.resize(nnz);
    L->rowS.resize(nNo);
    L->rowE.resize(nNo);
    L->diagPtr.assign(nNo, -1);
    L->map.resize(nNo);
    L->face.resize(nFaces);
    for (long long i = 0; i < nnz; ++i) L->colPtr[i] = colPtr[i] - 1;
    for (int Ac = 0; Ac < nNo; ++Ac) {
        long long s = rowPtr[Ac] - 1, e = rowPtr[Ac + 1] - 2;
        for (long long i = s; i <= e; ++i)
            if (L->colPtr[i] == Ac) {
                L->diagPtr[Ac] = i;
                break;
            }
        L->rowS[Ac] = s;
        L->rowE[Ac] = e;
        L->map[Ac] = Ac;
    }
    L->mynNo = nNo;
    (void)gNodes;
    return L;
}

extern "C" void orc_memls_lhs_free(void* lhs) { delete static_cast<Lhs*>(lhs); }

extern "C" int orc_memls_bc_create(void* lhs, int faIn, int nNo, int dof, int BC_type, const int* gNodes,
                                   const double* Val) {
    // memLS_BC_CREATE (memLS.f90:272-340), single task
    Lhs* L = static_cast<Lhs*>(lhs);
    if (faIn > L->nFaces || faIn < 1) return ORC_ERR_ARG;
    Face& f = L->face[faIn - 1];
    f.nNo = nNo;
    f.dof = dof;
    f.bGrp = BC_type;
    f.glob.resize(nNo);
    f.val.assign((size_t)dof * nNo, 0.0);
    f.valM.assign((size_t)dof * nNo, 0.0);
    for (int a = 0; a < nNo; ++a) f.glob[a] = L->map[gNodes[a] - 1];
    if (Val)
        for (size_t t = 0; t < (size_t)dof * nNo; ++t) f.val[t] = Val[t];
    f.foC = true;
    return ORC_OK;
}

extern "C" int orc_memls_solve(void* lhs, void* lsv, int dof, double* Ri, double* Val, const int* incL,
                               const double* res, orc_ls_stats* stats) {
    // memLS_SOLVE (memLS.f90:1947-2020)
    Lhs* L = static_cast<Lhs*>(lhs);
    Ls* ls = static_cast<Ls*>(lsv);
    if (!L || !ls || dof != 4) return ORC_ERR_UNSUPPORTED;
    const int nNo = L->nNo;
    if (L->nFaces != 0) {
        for (int faIn = 0; faIn < L->nFaces; ++faIn) {
            L->face[faIn].incFlag = true;
            if (incL && incL[faIn] == 0) L->face[faIn].incFlag = false;
        }
        for (int faIn = 0; faIn < L->nFaces; ++faIn) {
            Face& f = L->face[faIn];
            f.coupledFlag = false;
            if (!f.incFlag) continue;
            bool flag = f.bGrp == BC_TYPE_Neu;
            if (flag && res && res[faIn] != 0.0) {
                f.res = res[faIn];
                f.coupledFlag = true;
            }
        }
    }
    std::vector<double> R((size_t)dof * nNo), W((size_t)dof * nNo);
    for (int a = 0; a < nNo; ++a)
        for (int d = 0; d < dof; ++d) R[(size_t)dof * L->map[a] + d] = Ri[(size_t)dof * a + d];
    PRECOND(dof, *L, Val, R.data(), W.data());
    int rc = NSSOLVER(dof, *L, *ls, Val, R.data());
    for (size_t t = 0; t < R.size(); ++t) R[t] = R[t] * W[t];
    for (int a = 0; a < nNo; ++a)
        for (int d = 0; d < dof; ++d) Ri[(size_t)dof * a + d] = R[(size_t)dof * L->map[a] + d];
    if (stats) {
        stats->GM = ls->GM;
        stats->CG = ls->CG;
        stats->RI = ls->RI;
        stats->LS_type = ls->LS_type;
        stats->Resm = ls->Resm;
        stats->Resc = ls->Resc;
    }
    return rc;
}

// ===========================================================================
// Generalized-alpha (flowsolver/src/itrPC.f90)
// ===========================================================================
extern "C" void orc_time_params(double rhoinf, double* almi, double* alfi, double* gami) {
    // setupTimeParameters (itrPC.f90:16-37)
    if (rhoinf < 0.0 || rhoinf > 1.0) {
        *almi = 1.0;
        *alfi = 1.0;
        *gami = 1.0;
    } else {
        *almi = (3.0 - rhoinf) / (1.0 + rhoinf) / 2.0;
        *alfi = 1.0 / (1.0 + rhoinf);
        *gami = 0.5 + *almi - *alfi;
    }
}

extern "C" void orc_itr_predict(int nshg, double gami, const double* yold, const double* acold, double* y,
                                double* ac) {
    // itrPredict, ipred = 1 (itrPC.f90:106-110)
    double fct = (gami - 1.0) / gami;
    for (size_t t = 0; t < (size_t)nshg * 4; ++t) {
        y[t] = yold[t];
        ac[t] = acold[t] * fct;
    }
}

extern "C" void orc_itr_yalpha(int nshg, double alfi, double almi, const double* yold, const double* acold,
                               const double* y, const double* ac, double* yAlpha, double* acAlpha) {
    // itrYAlpha (itrPC.f90:326-336)
    for (int i = 0; i < nshg; ++i) acAlpha[3 * (size_t)nshg + i] = 0.0;
    for (int d = 0; d < 3; ++d)
        for (int i = 0; i < nshg; ++i) {
            size_t t = (size_t)d * nshg + i;
            yAlpha[t] = yold[t] + alfi * (y[t] - yold[t]);
            acAlpha[t] = acold[t] + almi * (ac[t] - acold[t]);
        }
    for (int i = 0; i < nshg; ++i) yAlpha[3 * (size_t)nshg + i] = y[3 * (size_t)nshg + i];
}

extern "C" void orc_itr_correct(int nshg, double gami, double alfi, double Delt, const double* solinc, double* y,
                                double* ac) {
    // itrCorrect (itrPC.f90:176-182); solinc (nshg, 4) column-major
    double fct1 = gami * Delt;
    double fct2 = gami * alfi * Delt;
    for (int d = 0; d < 3; ++d)
        for (int i = 0; i < nshg; ++i) {
            size_t t = (size_t)d * nshg + i;
            y[t] = y[t] + fct1 * solinc[t];
        }
    for (int i = 0; i < nshg; ++i) y[3 * (size_t)nshg + i] = y[3 * (size_t)nshg + i] + fct2 * solinc[3 * (size_t)nshg + i];
    for (int d = 0; d < 3; ++d)
        for (int i = 0; i < nshg; ++i) {
            size_t t = (size_t)d * nshg + i;
            ac[t] = ac[t] + solinc[t];
        }
}

extern "C" void orc_itr_bc(int nshg, const int* iBC, const double* BC, double* y) {
    // itrBC velocity and pressure branches (itrbc.f90:33-101)
    for (int i = 0; i < nshg; ++i) {
        const double* B = BC + i;
        auto bc = [&](int k) { return B[(size_t)k * nshg]; };   // BC(:, k+1)
        double* y1 = y + i;
        double* y2 = y + (size_t)nshg + i;
        double* y3 = y + 2 * (size_t)nshg + i;
        switch ((iBC[i] >> 3) & 7) {
            case 1: *y1 = bc(2) - bc(3) * *y2 - bc(4) * *y3; break;
            case 2: *y2 = bc(2) - bc(3) * *y1 - bc(4) * *y3; break;
            case 3: *y1 = bc(2) - bc(3) * *y3; *y2 = bc(4) - bc(5) * *y3; break;
            case 4: *y3 = bc(2) - bc(3) * *y1 - bc(4) * *y2; break;
            case 5: *y1 = bc(2) - bc(3) * *y2; *y3 = bc(4) - bc(5) * *y2; break;
            case 6: *y2 = bc(2) - bc(3) * *y1; *y3 = bc(4) - bc(5) * *y1; break;
            case 7: *y1 = bc(2); *y2 = bc(3); *y3 = bc(4); break;
            default: break;
        }
        if ((iBC[i] >> 2) & 1) y[3 * (size_t)nshg + i] = bc(0);
    }
}

extern "C" void orc_rcr_coeffs(double Rp, double C, double Rd, double Pdn, double Pdn1, double Pn, double Qn,
                               double alfi_delt, double* slope, double* offset) {
    // RCR::computeImplicitCoefficients (RCR.cxx:49-81)
    double denominator = 1.0 + ((C * Rd) / alfi_delt);
    double firstCoefficientNumerator = Rd + Rp * (1.0 + ((C * Rd) / alfi_delt));
    *slope = firstCoefficientNumerator / denominator;
    double temp2 = Pn + Pdn1 - Pdn - Rp * Qn;
    temp2 = ((C * Rd) / alfi_delt) * temp2 + Pdn1;
    *offset = temp2 / denominator;
}
