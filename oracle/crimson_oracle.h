/*
 * CPU FP64 oracle for the CRIMSON ElmGMR / memLS hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates the reference Fortran
 * (carthurs/CRIMSONFlowsolver, the Fortran under flowsolver/src) in C++ with the same
 * loop and summation order inside each element and each memLS kernel.  It is
 * the checker for the CUDA path and the timed CPU baseline; the product never
 * links, loads or calls it.
 *
 * Parity status: pinned end to end.  The reference is Fortran 90 + MPI and
 * no Fortran compiler or MPI exists in this environment, and its own tests
 * pin only whole-run history values, so no golden vector exists at the
 * single-call boundary.  One of those whole runs is a rigid-wall memLS case
 * whose mesh ships with it (testbin/mainTests/netlist/closedLoopHeart,
 * asserted by flowsolver/test/testMain.cxx:266-345); this restatement,
 * sequenced by oracle/pyoracle.py, reproduces the asserted flows and
 * pressures (tests/test_reference_closed_loop_heart.py).  Analytic
 * self-checks in tests/test_oracle_*.py cover the single calls.
 *
 * Conventions mirror the Fortran arrays: column-major, 1-based node and CSR
 * indices (ien, colm, rowp, ienb, gNodes).
 *   y, ac, res     (nshg, 4)      y[d*nshg + i]      dofs (u, v, w, p)
 *   x              (numnp, 3)     x[d*numnp + i]
 *   ien            (nelem, 4)     ien[a*nelem + e]   1-based
 *   qres           (nshg, 9)      qres[k*nshg + i]
 *   BC             (nshg, ndofBC) BC[c*nshg + i]
 *   lhsK           (9, nnz)       lhsK[9*k + c]
 *   lhsP           (4, nnz)       lhsP[4*k + c]
 *   ienb           (nface, 4)     face nodes 1..3 first, opposite node 4th
 *   iBCB           (nface, 2)     iBCB[c*nface + f]  (flag bits, surface id)
 *   BCB            (nface, 3, 6)  BCB[(c*3 + n)*nface + f]
 *   NABI           (nshg, 3)      NABI[d*nshg + i]
 */
#ifndef CRIMSON_ORACLE_H
#define CRIMSON_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double rho;            /* datmat(1,1,1) */
    double mu;             /* datmat(1,2,1) */
    double alfi, almi, gami;
    double Delt;           /* Delt(itseq) */
    double Dtgl;           /* 1/Delt */
    double dtsfct;         /* Tau Time Constant */
    double taucfct;        /* Tau C Scale Factor */
    double flmpl, flmpr;   /* lumped-mass fractions; this path requires 0 */
    double stabflux_coeff; /* Influx Coefficient */
    int idiff;             /* 0 or 1 */
    int iconvflow;         /* 2 advective, 1 conservative */
    int itau;              /* 0 (Diagonal-Shakib) */
    int ibksiz;            /* elements per block (255) */
    int ndofBC;            /* columns of BC */
    int nthreads;          /* 1 = reference summation order; >1 = OpenMP */
} orc_params;

/* Return codes */
#define ORC_OK 0
#define ORC_ERR_ARG 1
#define ORC_ERR_UNSUPPORTED 2
#define ORC_ERR_PATTERN 3
#define ORC_ERR_SINGULAR 4

/* genadj + Asadj (flowsolver/src/genadj.f90:1-84, asadj.f90:1-60) */
int orc_genadj(int nshg, int nelem, const int* ien, int* colm, int* rowp, long long cap, long long* nnz_tot);

/* ElmGMR interior + boundary + ElmpvsQ + bc3Res (flowsolver/src/elmgmr.f90:1-555) */
int orc_elmgmr(const orc_params* p, int nshg, int numnp, int nelem, const int* ien, const double* x,
               const double* y, const double* ac, const int* iBC, const double* BC,
               int nface, const int* ienb, const int* iBCB, const double* BCB,
               int ncoupled, const int* srflist, const double* coef1, const double* coef2,
               const int* ndsurf, const double* NABI,
               const int* colm, const int* rowp, long long nnz,
               double* res, double* lhsK, double* lhsP, int lhs,
               double* qres_out, double* rmass_out);

/* GetFlowQ (flowsolver/src/boundarydata.f90:1157-1196) */
/* ElmGMRSclr (flowsolver/src/elmgmr.f90:599-822) for scalar isclr (1..4)
 * with diffusivity diffus: s, sdot (nshg) the scalar and its rate, y (nshg,4)
 * the velocity, bcbs (nface, 3) prescribed face fluxes (may be NULL);
 * res (nshg), lhsS (nnz); qres_out (nshg, 3) the projected flux. */
int orc_elmgmr_sclr(const orc_params* p, int isclr, double diffus, int nshg, int numnp, int nelem,
                    const int* ien, const double* x, const double* y, const double* s, const double* sdot,
                    const int* iBC, int nface, const int* ienb, const int* iBCB, const double* bcbs,
                    const int* colm, const int* rowp, long long nnz, double* res, double* lhsS, int lhs,
                    double* qres_out);
int orc_getflowq(int nshg, const double* y, int nsrf, const int* srflist, const int* ndsurf,
                 const double* NABI, double* q);

/* SolFlow packing (flowsolver/src/solfar.f90:210-232) */
int orc_solflow_pack(int nshg, long long nnz, const int* colm, const int* rowp, const double* res,
                     const double* lhsK, const double* lhsP, double* Res4, double* Val4);

/* memLS (flowsolver/src/memLS.f90) */
typedef struct {
    double absTol, relTol, iNorm, fNorm, dB, callD;
    int suc, mItr, sD, itr, cM, cN, cD, reserve;
} orc_subls;

typedef struct {
    orc_subls GM, CG, RI;
    int LS_type, Resm, Resc;
} orc_ls_stats;

void* orc_memls_ls_create(int LS_type, int present_mask, double relTol, double absTol, int maxItr, int dimKry,
                          const double* relTolIn, const double* absTolIn, const int* maxItrIn);
void orc_memls_ls_free(void* ls);
void* orc_memls_lhs_create(int gnNo, int nNo, long long nnz, const int* gNodes, const int* rowPtr,
                           const int* colPtr, int nFaces);
void orc_memls_lhs_free(void* lhs);
int orc_memls_bc_create(void* lhs, int faIn, int nNo, int dof, int BC_type, const int* gNodes, const double* Val);
int orc_memls_solve(void* lhs, void* ls, int dof, double* Ri, double* Val, const int* incL, const double* res,
                    orc_ls_stats* stats);
void orc_memls_set_threads(int n);

/* Generalized-alpha (flowsolver/src/itrPC.f90) */
void orc_time_params(double rhoinf, double* almi, double* alfi, double* gami);
void orc_itr_predict(int nshg, double gami, const double* yold, const double* acold, double* y, double* ac);
void orc_itr_yalpha(int nshg, double alfi, double almi, const double* yold, const double* acold,
                    const double* y, const double* ac, double* yAlpha, double* acAlpha);
void orc_itr_correct(int nshg, double gami, double alfi, double Delt, const double* solinc, double* y, double* ac);
void orc_itr_bc(int nshg, const int* iBC, const double* BC, double* y);

/* RCR implicit coefficients (flowsolver/src/RCR.cxx:49-81) */
void orc_rcr_coeffs(double Rp, double C, double Rd, double Pdn, double Pdn1, double Pn, double Qn,
                    double alfi_delt, double* slope, double* offset);

#ifdef __cplusplus
}
#endif
#endif
