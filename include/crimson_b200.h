/*
 * crimson_b200 -- B200 (sm_100a) implementation of the CRIMSON flow solver's
 * element assembly (ElmGMR) and memLS Navier-Stokes linear solve.
 *
 * C ABI: plain pointers and sizes only.  Every entry point returns an int
 * status (CRIMSON_OK = 0) instead of the reference's PRINT + STOP.
 *
 * Array conventions follow the reference's Fortran arrays (column-major,
 * 1-based node and CSR indices) on every host-pointer entry point:
 *   ien   (nelem, 4)     int    ien[a*nelem + e], 1-based node numbers
 *   x     (numnp, 3)     double x[d*numnp + i]
 *   y, ac, res (nshg, 4) double y[d*nshg + i], dofs (u, v, w, p)
 *   iBC   (nshg)         int    bit 2 pressure, bits 3,4,5 velocity, bit 11 plane
 *   BC    (nshg, ndofBC) double BC[c*nshg + i]
 *   colm  (nshg+1)       int    row pointer, 1-based   (the reference's naming)
 *   rowp  (nnz)          int    column indices, 1-based, sorted in each row
 *   lhsK  (9, nnz)       double row-major 3x3 momentum blocks
 *   lhsP  (4, nnz)       double (G^T row D, PSPG C) per block
 *   ienb  (nface, 4)     int    boundary face nodes first, opposite node last
 *   iBCB  (nface, 2)     int    (flag bits, surface id)
 *   BCB   (nface, 3, 6)  double BCB[(c*3 + n)*nface + f]
 *   NABI  (nshg, 3)      double integral of N_a n over coupled outlets
 *   Ri    (dof, nNo)     double memLS right-hand side / solution
 *   Val   (dof*dof, nnz) double memLS block matrix, row-major blocks
 *
 * Entry points with the suffix _device take device pointers in the solver's
 * node-major layout (dof, nshg) -- the layout of memLS's R(dof, nNo) -- and
 * launch on the context's CUDA stream.
 *
 * Threading: one host thread per context; calls on a context are ordered on
 * its stream.  All mutable state lives in the context and lhs handles,
 * except two process-wide items: the element kernels' constant tables are
 * uploaded once per device (guarded by a mutex), and crimson_pvsq_noalloc
 * keeps its flows in one static device array per device (below).
 */
#ifndef CRIMSON_B200_H
#define CRIMSON_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CRIMSON_OK 0
#define CRIMSON_ERR_ARG 1
#define CRIMSON_ERR_UNSUPPORTED 2
#define CRIMSON_ERR_CUDA 3
#define CRIMSON_ERR_OOM 4
#define CRIMSON_ERR_PATTERN 5
#define CRIMSON_ERR_SINGULAR 6
#define CRIMSON_ERR_NONFINITE 7
#define CRIMSON_ERR_STATE 8

/* Precision of the element quadrature and inner Krylov arithmetic. */
#define CRIMSON_FP64 0
#define CRIMSON_MIXED 1          /* FP32 inner Krylov matvecs, FP64 refinement */
#define CRIMSON_MIXED_F32_TANGENT 2  /* CRIMSON_MIXED + FP32 quadrature of the tangent in crimson_step */

typedef struct crimson_ctx crimson_ctx;
typedef struct crimson_lhs crimson_lhs;
typedef struct crimson_ls crimson_ls;

/* Flow / time-integration / stabilisation settings.  The fields are the
 * module variables ElmGMR reads implicitly (phcommonvars: datmat, alfi, almi,
 * gami, Delt, Dtgl, dtsfct, taucfct, flmpl, flmpr, stabflux_coeff, idiff,
 * iconvflow, itau, ibksiz) -- flowsolver/src/elmgmr.f90:21-30. */
typedef struct {
    double rho, mu;
    double alfi, almi, gami;
    double Delt, Dtgl;
    double dtsfct, taucfct;
    double flmpl, flmpr;
    double stabflux_coeff;
    int idiff, iconvflow, itau, ibksiz, ndofBC, nthreads;
} crimson_params;

/* memLS statistics, field for field memLS_subLsType
 * (flowsolver/src/memLS.f90:159-188). */
typedef struct {
    double absTol, relTol, iNorm, fNorm, dB, callD;
    int suc, mItr, sD, itr, cM, cN, cD, reserve;
} crimson_subls;

typedef struct {
    crimson_subls GM, CG, RI;
    int LS_type, Resm, Resc;
} crimson_ls_stats;

/* ---------------------------------------------------------------------------
 * Context: mesh, boundary data and device work space.
 * Replaces the state the reference builds in input/proces/genblk and keeps in
 * pointer_data (mien blocks, x) -- flowsolver/src/genblk.f90:33-62,
 * flowsolver/src/readnblk.f90:33.
 * ------------------------------------------------------------------------- */
int crimson_ctx_create(crimson_ctx** ctx, const crimson_params* p, int nshg, int numnp, int nelem,
                       const int* ien, const double* x);
int crimson_ctx_destroy(crimson_ctx* ctx);
int crimson_set_params(crimson_ctx* ctx, const crimson_params* p);
/* iBC / BC as passed to ElmGMR (flowsolver/src/elmgmr.f90:1-8).  Velocity
 * constraints on none, one, two or all three components (ibits(iBC,3,3)):
 * itrBC, bc3Res and bc3LHS (itrbc.f90:33-101, bc3res.f90:30-124,
 * bc3lhs.f90:39-198) use BC(:,3:6) as the reference does; ndofBC >= 6. */
int crimson_set_bc(crimson_ctx* ctx, const int* iBC, const double* BC);
/* boundary element blocks mienb / miBCB / mBCB used by AsBMFG
 * (flowsolver/src/elmgmr.f90:325-460) */
int crimson_set_boundary(crimson_ctx* ctx, int nface, const int* ienb, const int* iBCB, const double* BCB);
/* coupled outlet surfaces: nsrflistGRCR, ndsurf, NABI (flowsolver/src/pvsqbi.f90:28,
 * flowsolver/src/elmgmr.f90:1271-1330) */
int crimson_set_outlets(crimson_ctx* ctx, int ncoupled, const int* srflist, const int* ndsurf, const double* NABI);

/* ---------------------------------------------------------------------------
 * Sparse pattern: genadj(colm, rowp, icnt) -- flowsolver/src/genadj.f90:1.
 * Builds the node-graph CSR pattern on the device (bit-identical to genadj:
 * sorted columns, diagonal included, 1-based).  colm/rowp may be NULL to only
 * build it and query nnz_tot; rowp needs room for cap entries.
 * ------------------------------------------------------------------------- */
int crimson_genadj(crimson_ctx* ctx, int* colm, int* rowp, long long cap, long long* nnz_tot);

/* ---------------------------------------------------------------------------
 * Assembly: ElmGMR(u, y, ac, x, ..., iBC, BC, ..., res, ..., rowp, colm, lhsK,
 * lhsP, ...) -- flowsolver/src/elmgmr.f90:1-8, called from SolFlow
 * (flowsolver/src/solfar.f90:148).  Host arrays in the reference layout.
 * coef1/coef2 are the implicit coefficients (dp/dq, Hop) of the coupled
 * surfaces (callCppGetImplicitCoeff_rcr, flowsolver/src/elmgmr.f90:1298).
 * lhs = 1 forms lhsK/lhsP (the reference's lhs flag).
 * ------------------------------------------------------------------------- */
int crimson_elmgmr(crimson_ctx* ctx, const double* y, const double* ac, const double* coef1, const double* coef2,
                   double* res, double* lhsK, double* lhsP, int lhs);
/* Device-resident ElmGMR: y, ac, res node-major (4, nshg); lhsK (9, nnz),
 * lhsP (4, nnz) on the device. */
int crimson_elmgmr_device(crimson_ctx* ctx, const double* d_y, const double* d_ac, const double* coef1,
                          const double* coef2, double* d_res, double* d_lhsK, double* d_lhsP, int lhs);

/* ---------------------------------------------------------------------------
 * memLS (flowsolver/src/memLS.f90): NS solver type only.
 * ------------------------------------------------------------------------- */
#define CRIMSON_LS_TYPE_NS 3
#define CRIMSON_BC_TYPE_DIR 0
#define CRIMSON_BC_TYPE_NEU 1
/* memLS_LS_CREATE(ls, LS_type, relTol, absTol, maxItr, dimKry, relTolIn,
 * absTolIn, maxItrIn) -- flowsolver/src/memLS.f90:1379.  present_mask bits mark
 * the optional arguments given: 1 relTol, 2 absTol, 4 maxItr, 8 dimKry,
 * 16 relTolIn, 32 absTolIn, 64 maxItrIn. */
int crimson_memls_ls_create(crimson_ls** ls, int LS_type, int present_mask, double relTol, double absTol,
                            int maxItr, int dimKry, const double* relTolIn, const double* absTolIn,
                            const int* maxItrIn);
int crimson_memls_ls_free(crimson_ls* ls);
/* Arithmetic of the NS solve; no counterpart in the reference (memLS is FP64
 * throughout).  CRIMSON_FP64 (default): memLS's arithmetic.  CRIMSON_MIXED:
 * FP32 copies of the scaled block matrices in every GMRES and CG matvec and
 * an FP32 GMRES basis; FP64 for every other product (the least-squares
 * products A d, so the NSSOLVER residual estimate is the FP64 operator's),
 * outer vectors, dot products, Givens rotations, Gram system and CG
 * recurrences; FP64 iterative refinement on the defect
 * R - A x until |R - A x| <= refine_tol |R| (relTol of memLS_LS_CREATE when
 * refine_tol <= 0) or max_refine sweeps (1..64).
 * Applies to crimson_memls_solve, crimson_solflow_device and crimson_step.
 * CRIMSON_MIXED_F32_TANGENT: as CRIMSON_MIXED, and crimson_step assembles the
 * tangent with FP32 element quadrature (the residual stays FP64).  The
 * converged solution is unchanged, but with a fixed number of nonlinear
 * iterations per step the iterates follow a slightly different Newton path
 * (on a small cylinder after 2 steps of 3 iterations: 1e-6 velocity, 4e-5
 * pressure relative to the FP64 tangent). */
int crimson_memls_ls_set_precision(crimson_ls* ls, int precision, int max_refine, double refine_tol);
/* Inner CG form of the mixed-precision solve (no counterpart in the
 * reference, which has only FP64).  explicit_schur = 1: each
 * NSSOLVER call forms the continuity Schur operator S = L - Gt G in FP64 on
 * the 2-ring pattern, rounds it to FP32, and CGRAD multiplies by S (one
 * sparse product and two grid barriers per iteration); the pattern is built
 * on the first mixed solve of an lhs and is used when every |col - row| of
 * the 2-ring fits 16 bits and no row has more than 256 entries.
 * explicit_schur = 0 (the default): CGRAD multiplies by L and Gt G as two
 * FP32 products, as memLS does in FP64.  On the 4M-tet cylinder one CG
 * iteration takes 0.0765 ms with the explicit operator and 0.0739 ms with the
 * two products: S has about 4 times the entries of the block pattern, which
 * cancels its single product per iteration.  FP64 solves are unaffected. */
int crimson_memls_ls_set_schur(crimson_ls* ls, int explicit_schur);
/* Per-solve log in the format of memLS's memLS_NS.log (LOGFILE,
 * flowsolver/src/memLS.f90:1720-1757), appended to path after every solve
 * with this ls; path = "memLS_NS.log" gives the reference's file.  NULL or ""
 * turns it off (the default). */
int crimson_memls_ls_set_log(crimson_ls* ls, const char* path);
/* Refinement sweeps taken by the last mixed solve on lhs and its final
 * relative FP64 defect |R - A x| / |R| (scaled system). */
int crimson_memls_refine_info(const crimson_lhs* lhs, int* steps, double* rel);
/* memLS_LHS_CREATE(lhs, commu, gnNo, nNo, nnz, gNodes, rowPtr, colPtr, nFaces)
 * -- flowsolver/src/memLS.f90:1080 (single task; rowPtr = colm, colPtr = rowp) */
int crimson_memls_lhs_create(crimson_lhs** lhs, int gnNo, int nNo, long long nnz, const int* gNodes,
                             const int* rowPtr, const int* colPtr, int nFaces);
/* Same, sharing the pattern already built on the device by crimson_genadj and
 * the context's stream; free such an lhs before its context. */
int crimson_memls_lhs_create_from_ctx(crimson_lhs** lhs, crimson_ctx* ctx, int nFaces);
int crimson_memls_lhs_free(crimson_lhs* lhs);
/* memLS_BC_CREATE(lhs, faIn, nNo, dof, BC_type, gNodes, Val) -- memLS.f90:272 */
int crimson_memls_bc_create(crimson_lhs* lhs, int faIn, int nNo, int dof, int BC_type, const int* gNodes,
                            const double* Val);
/* memLS_SOLVE(lhs, ls, dof, Ri, Val, incL, res) -- flowsolver/src/memLS.f90:1947.
 * Host arrays.  As in the reference, Ri returns the solution and Val returns
 * scaled in place by the diagonal preconditioner. */
int crimson_memls_solve(crimson_lhs* lhs, crimson_ls* ls, int dof, double* Ri, double* Val, const int* incL,
                        const double* res, crimson_ls_stats* stats);

/* ---------------------------------------------------------------------------
 * SolFlow's pack + solve on the device (flowsolver/src/solfar.f90:210-280):
 * Res4 = res, Val4 from lhsK/lhsP (with the transposed -G blocks found by a
 * precomputed transpose map instead of the search), memLS_SOLVE, solinc.
 * d_res (4, nshg) node-major in, d_solinc (4, nshg) out.  lhs must come from
 * crimson_memls_lhs_create_from_ctx.  faceRes has nFaces entries.
 * ------------------------------------------------------------------------- */
int crimson_solflow_device(crimson_ctx* ctx, crimson_lhs* lhs, crimson_ls* ls, const double* d_res,
                           const double* d_lhsK, const double* d_lhsP, const int* incL, const double* faceRes,
                           double* d_solinc, crimson_ls_stats* stats);

/* ---------------------------------------------------------------------------
 * FP32 element quadrature for the tangent (mixed precision; no counterpart
 * in the reference).  crimson_elmgmr_device_f32 forms res exactly as
 * crimson_elmgmr_device (FP64 arithmetic and scatter) and the tangent in
 * FP32: d_lhs32 (16, nnz) floats per block = lhsK(1:9), lhsP(1:4), 3 zero
 * pads (16-byte aligned records scattered with 4-wide vector reductions).
 * crimson_solflow_device_f32 is crimson_solflow_device taking those
 * records.  crimson_step uses both when the ls handle is
 * CRIMSON_MIXED_F32_TANGENT.
 * ------------------------------------------------------------------------- */
int crimson_elmgmr_device_f32(crimson_ctx* ctx, const double* d_y, const double* d_ac, const double* coef1,
                              const double* coef2, double* d_res, float* d_lhs32);
int crimson_solflow_device_f32(crimson_ctx* ctx, crimson_lhs* lhs, crimson_ls* ls, const double* d_res,
                               const float* d_lhs32, const int* incL, const double* faceRes, double* d_solinc,
                               crimson_ls_stats* stats);

/* ---------------------------------------------------------------------------
 * 4x4 block SpMV, SPARMULVV with dof = 4 (flowsolver/src/memLS.f90:2024-2076):
 * KU(:, i) = sum_j Val(:, :, j) U(:, col(j)) on the context's pattern.
 * prepare: d_val is memLS's Val (16, nnz), row-major 4x4 blocks, on the
 * device, FP64 (precision CRIMSON_FP64) or FP32 (CRIMSON_MIXED); it is
 * copied into a sliced layout.  apply: d_u, d_ku (4, nshg) node-major on the
 * device, in the prepared precision; launches on the context's stream.
 * ------------------------------------------------------------------------- */
int crimson_spmv4_prepare(crimson_ctx* ctx, int precision, const void* d_val);
int crimson_spmv4_apply(crimson_ctx* ctx, const void* d_u, void* d_ku);

/* ---------------------------------------------------------------------------
 * Adjoint building blocks.  No counterpart in the reference (it has no
 * adjoint).
 * ------------------------------------------------------------------------- */
/* Transposed solve: same arguments and preconditioning as
 * crimson_solflow_device, but solves A^T z = rhs, A the Val4 matrix SolFlow
 * packs from lhsK/lhsP (plus the coupled-face terms).  d_rhs, d_sol (4, nshg)
 * node-major on the device. */
int crimson_solflow_device_transposed(crimson_ctx* ctx, crimson_lhs* lhs, crimson_ls* ls, const double* d_rhs,
                                      const double* d_lhsK, const double* d_lhsP, const int* incL,
                                      const double* faceRes, double* d_sol, crimson_ls_stats* stats);
/* Exact vector-Jacobian product of ElmGMR's residual res(y, ac; mu, coef1,
 * coef2) -- the same vector crimson_elmgmr_device assembles, with the
 * viscous-flux projection, boundary faces, outlet coupling and bc3Res --
 * for a cotangent lambda (4, nshg) node-major on the device:
 *   d_ybar  = (d res / d y)^T lambda      (4, nshg) node-major (u, v, w, p)
 *   d_acbar = (d res / d ac)^T lambda     (4, nshg) node-major (pressure slot 0)
 *   *mubar = lambda . d res / d mu; coef1bar[k], coef2bar[k] likewise (host).
 * d_res (optional) receives res itself.  Unlike the assembled tangent (the
 * reference's approximate Jacobian), this differentiates tauM, tauC, tauBar,
 * uBar and the flux projection as well.  Returns CRIMSON_ERR_UNSUPPORTED when
 * some node has one or two prescribed velocity components. */
int crimson_elmgmr_vjp(crimson_ctx* ctx, const double* d_y, const double* d_ac, const double* coef1,
                       const double* coef2, const double* d_lambda, double* d_res, double* d_ybar, double* d_acbar,
                       double* mubar, double* coef1bar, double* coef2bar);

/* ---------------------------------------------------------------------------
 * Device-resident time step: itrdrv_iter_step (flowsolver/src/itrdrv.f90:1239)
 * = itrPredict, itrBC, nitr x [itrYAlpha, ElmGMR, SolFlow pack + memLS_SOLVE,
 * itrCorrect, itrBC], with RCR outlets (flowsolver/src/RCR.cxx:49-81).
 * ------------------------------------------------------------------------- */
typedef struct {
    int nitr;               /* solve/update pairs per step (Step Construction) */
    double inflow_scale;    /* multiplies the registered inlet profile at t_{n+1} */
    /* Residual Control / Residual Criteria / Minimum Required Iterations
     * (itrdrv.f90:1516-1522): with rescontrol != 0 the step ends after the
     * assembly of the first iteration whose totres = sqrt(|res|^2 / nshg)
     * (rstatic.f90) is below res_criteria once at least min_iters
     * iterations have been assembled, without that iteration's solve; the
     * count carries over a step that ends without such an exit.  Zero
     * (off) in a zero-initialised struct. */
    int rescontrol;
    double res_criteria;
    int min_iters;
} crimson_step_args;

typedef struct {
    int nsolves;
    int ri_itr[16], gm_itr[16], cg_itr[16];
    double ri_inorm[16], ri_fnorm[16];
    double q_out[8], p_out[8];   /* outlet flow and pressure at t_{n+1} */
    int refine_steps[16];        /* mixed precision: refinement sweeps per solve */
    double refine_rel[16];       /* mixed precision: final |R - A x| / |R| per solve */
    double res_norm[16];         /* residual control: totres of each assembled iteration */
} crimson_step_stats;

/* register the inlet profile: BC(node, 3:5) = profile * inflow_scale */
int crimson_set_inflow(crimson_ctx* ctx, int ninlet, const int* nodes, const double* profile);
/* RCR outlets on the coupled surfaces, in srflist order */
int crimson_set_rcr(crimson_ctx* ctx, int n, const double* Rp, const double* C, const double* Rd, const double* Pd);
/* RCR history (P_n, Q_n per coupled surface, the AbstractBoundaryCondition
 * state, flowsolver/src/AbstractBoundaryCondition.cxx:55-91): read (set = 0)
 * or write (set = 1), e.g. to restart from a checkpoint. */
int crimson_rcr_state(crimson_ctx* ctx, int n, double* Pn, double* Qn, int set);
/* ElmGMRSclr (flowsolver/src/elmgmr.f90:599-822): residual res (nshg) and
 * tangent lhsS (nnz, the CSR pattern of crimson_genadj) of the
 * advection-diffusion equation of scalar isclr (1..4) with diffusivity
 * diffus (scdiff(isclr)), after AsIqSclr/qpbcSclr (the lumped projection of
 * diffus grad S when idiff = 1), AsIGMRSclr/e3Sclr, fillsparseSclr,
 * AsBSclr/e3bSclr (the boundary flux term; faces whose iBCB bit 4+isclr is
 * set take the prescribed flux bcbs (nface, 3) instead, bcbs may be NULL
 * otherwise) and bc3ResSclr (rows with iBC bit isclr+5 zeroed).  y (nshg, 4)
 * supplies the velocity; s and sdot (nshg) are the scalar and its rate at
 * the alpha levels (y(:,5+isclr), ac(:,5+isclr) in the reference).  The
 * reference's defaults for a passive scalar: SUPG, no discontinuity
 * capturing, the flow velocity as convection velocity, no source terms
 * (the reference's source call is commented out; its nosource = 0 reads
 * uninitialised arrays).  Summation in ascending element order per entry,
 * bitwise repeatable.  The reference solves this system with ACUSIM
 * LesLib, which it does not contain; hosts pass res and lhsS to their
 * own solver.  Returns CRIMSON_ERR_UNSUPPORTED for lumped-mass fractions. */
int crimson_elmgmr_sclr(crimson_ctx* ctx, int isclr, double diffus, const double* y, const double* s,
                        const double* sdot, const double* bcbs, double* res, double* lhsS, int lhs);
/* Device pointers: d_y (4, nshg) node-major, d_s, d_sdot, d_res (nshg),
 * d_bcbs (nface, 3) face-major or NULL, d_lhsS (nnz); on the context's stream. */
int crimson_elmgmr_sclr_device(crimson_ctx* ctx, int isclr, double diffus, const double* d_y, const double* d_s,
                               const double* d_sdot, const double* d_bcbs, double* d_res, double* d_lhsS, int lhs);

/* ---------------------------------------------------------------------------
 * Netlist (lumped-parameter 0D) outlet circuits: NetlistCircuit
 * (flowsolver/src/NetlistCircuit.cxx, CircuitData.cxx, CircuitComponent.cxx)
 * for circuits of resistors, capacitors, inductors and diodes, with fixed
 * nodal pressures ('f'), fixed component flows ('f') and exactly one
 * component carrying the 3D interface flow ('t'), coupled to the 3D domain
 * through p = dp/dQ * Q + H as the ElmpvsQ netlist branch does
 * (flowsolver/src/elmgmr.f90:1430-1452).  Volume-tracking components and
 * pressure chambers (elastance E, initial and unstressed volume) carry a
 * volume unknown.  Host-only calls (no GPU needed).
 *
 * Nodes are numbered 1..nnodes and each belongs to at least one component;
 * the 3D interface node is node 1 (the reference reads the coupling
 * coefficients from the system's first unknown, node 1's pressure) and
 * belongs to exactly one component.  Diodes start closed and switch at the
 * end of each step (open while the pressure drop is >= -1e-8 or the flow
 * >= 1e-8).  While closed diodes block every path from the interface the
 * circuit is in the reference's Dirichlet design (CircuitData.cxx:482-540):
 * the interface node takes the 3D surface pressure as a prescribed pressure
 * and the interface component's flow is solved for; the flow solver then
 * holds the surface at its Dirichlet codes (itrdrv.f90:1114-1133).
 * Control systems act through crimson_netlist_set_parameter: the Python
 * controllers of crimsonflowsolver_b200.controllers drive it, the
 * reference's built-in left-ventricular elastance and bleed controllers
 * among them; left-ventricular pressure prescriptions are not built.
 * --------------------------------------------------------------------------- */
typedef struct crimson_netlist crimson_netlist;
#define CRIMSON_NETLIST_RESISTOR 0
#define CRIMSON_NETLIST_CAPACITOR 1
#define CRIMSON_NETLIST_INDUCTOR 2
#define CRIMSON_NETLIST_DIODE 3   /* value = open resistance */
#define CRIMSON_NETLIST_VOLUME_TRACKING 4   /* dV/dt = q */
#define CRIMSON_NETLIST_PRESSURE_CHAMBER 5  /* dV/dt = q, p_start = value * (V - V_unstressed) */
#define CRIMSON_NETLIST_FLOW_FIXED 0
#define CRIMSON_NETLIST_FLOW_3D 1
/* createBasicCircuitDescription + initialiseCircuit
 * (NetlistCircuit.cxx:131-297, 787-834): component j (0-based arrays) joins
 * start_node[j] -> end_node[j]; initial_volume / unstressed_volume (ncomp,
 * read for volume-tracking components only; may be NULL without them, and
 * unstressed_volume NULL means 0); initial_pressure (nnodes) is the state
 * the histories start from. */
int crimson_netlist_create(crimson_netlist** nl, int ncomp, const int* kind, const int* start_node,
                           const int* end_node, const double* value, const double* initial_volume,
                           const double* unstressed_volume, int nnodes, const double* initial_pressure, int npres,
                           const int* pres_node, const double* pres_value, int nflow, const int* flow_comp,
                           const int* flow_kind, const double* flow_value, int interface_node);
/* A member of a closed loop (NetlistBoundaryCircuitWhenDownstreamCircuitsExist,
 * NetlistClosedLoopDownstreamCircuit): as crimson_netlist_create, with the
 * nodes shared with the loop's other circuits (shared_nodes, nshared; their
 * Kirchhoff equations are the loop's) and interface_node 1 for an upstream
 * circuit coupled to a 3D surface or 0 for the loop-closing (downstream)
 * circuit, which has no 3D interface and no 3D-flow component.  A member is
 * solved only through its crimson_netlist_loop; crimson_netlist_get,
 * _get/_set_parameter, _state and _flow_permitted work on it as on any
 * circuit. */
int crimson_netlist_create_member(crimson_netlist** nl, int ncomp, const int* kind, const int* start_node,
                                  const int* end_node, const double* value, const double* initial_volume,
                                  const double* unstressed_volume, int nnodes, const double* initial_pressure,
                                  int npres, const int* pres_node, const double* pres_value, int nflow,
                                  const int* flow_comp, const int* flow_kind, const double* flow_value,
                                  int interface_node, int nshared, const int* shared_nodes);
void crimson_netlist_free(crimson_netlist* nl);
/* detectWhetherClosedDiodesStopAllFlowAt3DInterface (CircuitData.cxx:388-470):
 * 1 in the Neumann design, 0 in the Dirichlet design. */
int crimson_netlist_flow_permitted(crimson_netlist* nl, int* permitted);
/* computeImplicitCoefficients (NetlistCircuit.cxx:1764-1800) with the
 * step's alfi*Delt: the interface pressure p = dp_dq * Q + hop.
 * CRIMSON_ERR_STATE in the Dirichlet design (the reference sets them to NaN
 * there, AbstractBoundaryCondition.cxx:32-53). */
int crimson_netlist_implicit_coefficients(crimson_netlist* nl, double alfi_delt, double* dp_dq, double* hop);
/* updateLPN (NetlistCircuit.cxx:1582-1594): solve with Delt and the
 * interface flow at the end of the step (Neumann design; CRIMSON_ERR_STATE
 * in the Dirichlet design). */
int crimson_netlist_update(crimson_netlist* nl, double delt, double interface_flow);
/* updateLPN in the Dirichlet design: the interface node's prescribed
 * pressure is the 3D surface's mean pressure at the end of the step
 * (integrScalar of p over the surface / its area, elmgmr.f90:1733-1743);
 * CRIMSON_ERR_STATE in the Neumann design. */
int crimson_netlist_update_pressure(crimson_netlist* nl, double delt, double interface_pressure);
/* finalizeLPNAtEndOfTimestep (NetlistCircuit.cxx:732-737): histories and
 * diode states for the next step. */
int crimson_netlist_finalize_step(crimson_netlist* nl);
/* Current nodal pressures (nnodes), component flows (ncomp), diode states
 * (ncomp, 1 = open) and volumes (ncomp, 0 for components without one); any
 * pointer may be NULL. */
int crimson_netlist_get(const crimson_netlist* nl, double* pressures, double* flows, int* open, double* volumes);
/* The parameters control systems adjust between steps
 * (ControlSystemsManager.cxx:125-330; itrdrv.f90:2100 updates them after
 * the step's finalisation): a component's value (R, C, L, a diode's open
 * resistance, a chamber's elastance), a pressure chamber's unstressed
 * volume, a node's pressure (the prescribed value of a fixed-pressure node;
 * for other nodes the current value, which the next solve replaces) or a
 * component's fixed prescribed flow.  index is 1-based; CRIMSON_ERR_ARG
 * when the circuit has no such parameter. */
#define CRIMSON_NETLIST_PARAM_COMPONENT 0
#define CRIMSON_NETLIST_PARAM_UNSTRESSED_VOLUME 1
#define CRIMSON_NETLIST_PARAM_PRESSURE 2
#define CRIMSON_NETLIST_PARAM_FLOW 3
int crimson_netlist_get_parameter(crimson_netlist* nl, int what, int index, double* value);
int crimson_netlist_set_parameter(crimson_netlist* nl, int what, int index, double value);
/* Checkpoint of the circuit state: state_size doubles, read (set = 0) or
 * written (set = 1). */
int crimson_netlist_state_size(const crimson_netlist* nl, int* n);
int crimson_netlist_state(crimson_netlist* nl, double* buf, int set);
/* Closed loops (ClosedLoopDownstreamSubsection.cxx:101-500, 609-940): the
 * upstream circuits (in input order) and one loop-closing circuit solved as
 * one system.  Connection c (file order of the downstream input) joins node
 * conn_down_node[c] of the loop-closing circuit to node conn_upstream_node[c]
 * of upstream circuit conn_upstream[c] (0-based); each member's shared nodes
 * must be exactly its connected nodes.  The loop does not own its members:
 * free the loop first. */
typedef struct crimson_netlist_loop crimson_netlist_loop;
int crimson_netlist_loop_create(crimson_netlist_loop** loop, int nupstream, crimson_netlist* const* upstream,
                                crimson_netlist* downstream, int nconn, const int* conn_down_node,
                                const int* conn_upstream, const int* conn_upstream_node);
void crimson_netlist_loop_free(crimson_netlist_loop* loop);
/* getImplicitCoefficients: per upstream circuit k, p_k = dp_dq[k] * Q_k +
 * hop[k] from one solve with alfi*Delt; NaN for a circuit in the Dirichlet
 * design. */
int crimson_netlist_loop_implicit_coefficients(crimson_netlist_loop* loop, double alfi_delt, double* dp_dq,
                                               double* hop);
/* updateLPN for every member: one solve with Delt; upstream circuit k takes
 * interface_flow[k] in the Neumann design, interface_pressure[k] (the 3D
 * surface's mean pressure) in the Dirichlet design. */
int crimson_netlist_loop_update(crimson_netlist_loop* loop, double delt, const double* interface_flow,
                                const double* interface_pressure);
/* crimson_netlist_finalize_step of every member. */
int crimson_netlist_loop_finalize_step(crimson_netlist_loop* loop);
/* Couple surface k (0-based, srflist order) through nl instead of its RCR
 * in crimson_step: the coefficients come from nl at the start of each step,
 * and nl is updated and finalised with the surface's flow at its end; the
 * step's p_out is the interface node's pressure.  While nl's closed valves
 * block the interface, the surface keeps the codes crimson_set_bc gave it
 * (the reference's iBC_original; the coupled surfaces that take flow get
 * zeros, itrdrv.f90:1114-1133), memLS face 1 of the step's lhs is rebuilt
 * from the codes when they change, the surface is not coupled, and nl is
 * updated with the surface's NASC-weighted mean pressure.  nl == NULL
 * restores the RCR.  The context does not own nl: free the context first. */
int crimson_set_outlet_netlist(crimson_ctx* ctx, int k, crimson_netlist* nl);

/* Couple the upstream circuits of loop through it: upstream circuit j
 * couples surface surfaces[j] (0-based, srflist order).  Each step takes
 * the loop's implicit coefficients once, updates the loop with the flows
 * (blocked circuits: the NASC-weighted mean pressures) of its surfaces and
 * finalises every member; the Dirichlet-design rules of
 * crimson_set_outlet_netlist hold per upstream circuit.  The context does
 * not own the loop. */
int crimson_set_outlet_netlist_loop(crimson_ctx* ctx, crimson_netlist_loop* loop, const int* surfaces);

/* yold/acold in the reference layout (nshg, 4) */
int crimson_state_set(crimson_ctx* ctx, const double* y, const double* ac);
int crimson_state_get(crimson_ctx* ctx, double* y, double* ac);
/* Per coupled surface (n = the number given to crimson_set_outlets) the
 * flow GetFlowQ and the mean pressure integrScalar(p) / area of the current
 * state, the values Updcalc writes to FlowHist.dat and PressHist.dat
 * (bctcardio.f90:1021-1040); the mean pressure is 0 for a surface whose
 * faces carry no natural-pressure bit. */
int crimson_outlet_state(crimson_ctx* ctx, int n, double* q, double* p_mean);
int crimson_step(crimson_ctx* ctx, crimson_lhs* lhs, crimson_ls* ls, const crimson_step_args* args,
                 crimson_step_stats* stats);

/* The CUDA stream (cudaStream_t) every call on this context launches on. */
void* crimson_ctx_stream(crimson_ctx* ctx);

/* ---------------------------------------------------------------------------
 * Outlet coupling without device allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc (a stream
 * being captured into a CUDA graph, a host framework that owns all device
 * memory through its own pool, a latency-bound coupling loop where an
 * allocation would synchronise the device).
 * Computes the flows Q_k = sum NABI . u over each coupled surface and adds
 * p_k NABI to the momentum rows of res with p_k = -(Q_k coef1_k) - coef2_k,
 * as ElmGMR's outlet coupling does.  Device inputs: d_nodes (1-based node
 * numbers of the surfaces, grouped by surface), d_nabi (3, n) NABI of those
 * nodes, d_y (4, nshg) node-major; d_res (4, nshg) updated in place.  Host
 * inputs: surf_offsets (nsurf+1) into d_nodes with surf_offsets[0] == 0 and
 * non-decreasing entries, coef1/coef2 (nsurf).  q_out (host, nsurf) receives
 * the flows when not NULL (the call then copies them back and waits for the
 * stream, so q_out must be NULL while the stream is being captured: the call
 * returns CRIMSON_ERR_UNSUPPORTED otherwise).  stream is a cudaStream_t
 * (NULL = default stream).
 * Preconditions the call cannot check (it is given no nshg): every node
 * number lies in 1..nshg of d_y / d_res.  A node listed under several
 * surfaces receives each surface's term (the update is atomic per value).
 * Unlike crimson_elmgmr_device, this call applies no bc3Res afterwards:
 * zero the constrained rows yourself if the coupling runs after it.
 * At most 64 surfaces: the flows live in a 512-byte static device array
 * shared by every call (overlapping calls on the GPU race on it); the first
 * call on a device looks up that array's address, so make it before any
 * stream capture.  Returns CRIMSON_ERR_UNSUPPORTED for nsurf > 64.
 * ------------------------------------------------------------------------- */
int crimson_pvsq_noalloc(int nsurf, const int* surf_offsets, const int* d_nodes, const double* d_nabi,
                         const double* d_y, const double* coef1, const double* coef2, double* d_res, double* q_out,
                         void* stream);

/* Diagnostics: average device time (ms) of one launch of a memLS kernel on the
 * lhs's current split matrices, timed with CUDA events on the lhs stream.
 * which: 0 = 3x3 block SpMV (SPARMULVV, K) on the sliced-ELL copy GMRES
 * uses, 2 = SPARMULSV (G), 3 = fused MGS step, 5 = the sliced 3x3 block SpMV
 * with FP32 K (after a mixed solve), 6 = the 3x3 block SpMV on CSR K.
 * which 1 / 4: time of one CGRAD iteration of the persistent CG kernel with
 * FP64 / FP32 matrices, averaged over every launch on this lhs so far (CUDA
 * events recorded around each cooperative launch; reps is ignored).
 * Valid after a solve on the lhs. */
int crimson_memls_kernel_time(crimson_lhs* lhs, int which, int reps, double* ms);

/* Diagnostics: column layout of the persistent CG kernel on this lhs.
 * resident64 / resident32 = 1 when the kernel with FP64 / FP32 matrices keeps
 * every block's column indices in shared memory for the whole launch (16-bit
 * offsets col - row; chosen when the offsets fit and two blocks per SM fit
 * with them), 0 when it reads them from the sliced pattern each phase;
 * smem_bytes = shared memory per block of the resident layout (0: offsets
 * exceed 16 bits).  Valid after a solve on the lhs. */
int crimson_memls_cg_layout(const crimson_lhs* lhs, int* resident64, int* resident32, long long* smem_bytes);

/* Diagnostics of the explicit FP32 Schur operator (crimson_memls_ls_set_schur)
 * on this lhs: state 1 = built and used by mixed solves, 0 = not built yet,
 * -1 = the pattern does not allow it; nnz / npad = its entries and sliced
 * positions (padding included); form_ms = average time of one formation
 * (CUDA events).  Valid after a mixed solve on the lhs. */
int crimson_memls_schur_info(const crimson_lhs* lhs, int* state, long long* nnz, long long* npad, double* form_ms);

/* Number of CUDA kernels this library has launched since it was loaded. */
unsigned long long crimson_launch_count(void);

/* Library version and build target, for diagnostics. */
const char* crimson_version(void);
/* Last CUDA error string seen by this library (diagnostics). */
const char* crimson_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
