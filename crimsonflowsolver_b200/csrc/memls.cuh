// memLS handles shared by memls.cu and capi.cu.
#pragma once

#include <string>
#include <vector>

#include "common.cuh"

struct crimson_lhs;

namespace crimson {

struct RedScratch {
    DBuf<double> part;          // partial sums, kMaxBlocks per concurrent slot
    DBuf<unsigned int> ticket;  // one counter per slot
    static constexpr int kMaxBlocks = 1184;   // 148 SMs x 8
    static constexpr int kSlots = 4;
    int init() {
        CR_CHECK(part.alloc((size_t)kMaxBlocks * kSlots));
        CR_CHECK(ticket.alloc(kSlots));
        CR_CUDA(cudaMemset(ticket.p, 0, sizeof(unsigned int) * kSlots));
        return CRIMSON_OK;
    }
};

int schur_pattern(crimson_lhs* L);
int schur_form(crimson_lhs* L, const double* mG, const double* Gt, const double* mL);
int cg_schur_launch(crimson_lhs* L, const double* R, int nface, const double* coef, const double* w, const double* z,
                    double eps, double err0, int mItr, double* out);

}  // namespace crimson

using crimson::DBuf;
using crimson::RedScratch;

struct MemlsFace {
    int nNo = 0, dof = 0, bGrp = CRIMSON_BC_TYPE_DIR;
    bool incFlag = true, coupledFlag = false, created = false;
    double res = 0.0, nS = 0.0;
    DBuf<int> glob;
    DBuf<double> val, valM;
};

struct crimson_lhs {
    int gnNo = 0, nNo = 0, nFaces = 0;
    long long nnz = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // pattern (owned or borrowed from a ctx)
    DBuf<int> own_rowptr, own_col, own_diag, own_trans;
    const int* rowptr = nullptr;
    const int* col = nullptr;
    const int* diag = nullptr;
    const int* trans = nullptr;
    std::vector<MemlsFace> face;
    // work space
    DBuf<double> W, R, Val, mK, mG, mD, mL, Gt, mKt;
    DBuf<double> Rm, Rc, Rmi, Rci, U, P, MU, MP, X3, basis, w3;
    DBuf<double> cgX, cgP, cgSP, cgGP, cgR, cgP2;
    DBuf<double> cgW, cgZ, cgExt;     // coupled-face vectors w = G^T valM, z = Gt valM (per face)
    DBuf<double> cgPart;              // persistent CG partial sums (3 regions)
    DBuf<double> cgRecA, cgRecB, cgPd; // {R, P} and {GP, P} node records; P (FP64)
    // sliced ELL copy of the pattern (32 rows per slice) and of the matrices
    // the Krylov loops multiply by, per storage precision
    int nslice = 0;
    long long npad = 0;
    DBuf<int> sell_ptr, sell_col;
    DBuf<double> Ks64, Gs64, GLs64;
    DBuf<float> Ks32, Gs32, GLs32;
    int cg_grid = 0, cg_grid32 = 0;
    int cg_res64 = 0, cg_res32 = 0;    // CG kernel with block-resident columns (per matrix type)
    long long cg_res_bytes = -1;       // its shared memory per block (0: offsets exceed 16 bits); -1 unknown
    DBuf<int> cg_tmp;
    // persistent GMRES cycle: Hessenberg / err outputs, partial sums and the
    // coupled-face node map (built for the coupled faces in gm_faces)
    DBuf<double> gmH, gmErr, gmOut, gmPart, gmFval, gmGram;
    DBuf<int> gmFptr, gmFent, gmFface, gmPairs;
    std::vector<int> gm_faces;
    int gm_npairs = 0;
    int gm_map_ok = -1;   // 1: map built, 0: not usable (more than 8 coupled faces), -1: not built
    int gm_grid = 0, gm_grid32 = 0;
    // mixed precision: FP64 right side and accumulated solution of the
    // iterative refinement
    DBuf<double> R0, X4;
    int refine_steps = 0;
    double refine_rel = 0.0;
    // CUDA-event time of the persistent CG launches (per matrix precision)
    struct CgAcc {
        double ms = 0.0;
        long long iters = 0, launches = 0;
    } cg_acc64, cg_acc32;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // explicit FP32 Schur operator S = L - Gt G of the mixed-precision CG
    // (schur.cu): 2-ring pattern (CSR and sliced int16 offsets), FP32 values
    int s2_state = 0;       // 0: pattern not built, 1: usable, -1: not usable on this pattern
    DBuf<int> s2_rowptr, s2_col, s2_sp;
    DBuf<short> s2_off;
    DBuf<float> s2_val;
    DBuf<float2> s2_recF;
    DBuf<double> s2_part;
    long long s2_nnz = 0, s2_npad = 0;
    int s2_nslice = 0, s2_grid = 0;
    cudaEvent_t s2_ev0 = nullptr, s2_ev1 = nullptr;
    bool s2_form_pending = false;   // a formation was recorded between s2_ev0 and s2_ev1
    double s2_form_ms = 0.0;
    int s2_forms = 0;
    DBuf<double> scal;      // device scalars
    RedScratch red;
    double* hscal = nullptr;   // pinned host mirror of scal
    int sD = 0, iBcap = 0;
};

struct crimson_ls {
    crimson_subls GM{}, CG{}, RI{};
    int LS_type = CRIMSON_LS_TYPE_NS, Resm = 0, Resc = 0;
    int precision = CRIMSON_FP64;  // CRIMSON_FP64, CRIMSON_MIXED or CRIMSON_MIXED_F32_TANGENT
    int max_refine = 4;            // FP64 refinement sweeps of the mixed solve
    double refine_tol = 0.0;       // target |R - A x| / |R|; <= 0: RI.relTol
    int schur = 0;                 // mixed precision: 1 = CG on the explicit FP32 Schur operator when the pattern allows
    std::string log_path;          // per-solve log (memLS_NS.log format); empty: off
};

