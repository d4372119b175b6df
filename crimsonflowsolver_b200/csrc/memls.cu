// memLS NS linear solver on the device (flowsolver/src/memLS.f90).
//
// Layout: node-major vectors (dof, nNo) exactly as memLS's R(dof, nNo); block
// matrices split as DEPART does (memLS.f90:1612-1679) into mK (9, nnz),
// mG (3, nnz), mD (3, nnz), mL (nnz) and Gt (3, nnz).
//
// Kernels are HBM-bound: block SpMVs use 8 lanes per block row with lanes
// striding the row's blocks, so each warp streams 4 rows' blocks contiguously;
// dot products and norms use a single-pass grid reduction whose last block
// sums the per-block partials in a fixed order (deterministic).  The Krylov
// control flow (Givens rotations, back substitution, the 2i x 2i Gram system
// solved by GE) runs on the host in FP64 on scalars copied back per step, as
// the reference's serial code does.
//
// Modified Gram-Schmidt is fused: kernel j subtracts h(j-1) u_{j-1} from w and
// accumulates <w, u_j> in the same pass, so orthogonalising against i basis
// vectors streams w i+1 times instead of 2i times.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "memls.cuh"

namespace crimson {

// ---------------------------------------------------------------------------
// Reductions: partial sums per block -> last block sums them in block order.
// ---------------------------------------------------------------------------


// Finish a grid reduction: every block calls this with its block-summed value.
__device__ __forceinline__ void grid_reduce_finish(double bsum, double* part, unsigned int* ticket, double* out,
                                                   double* smem) {
    __shared__ bool am_last;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = bsum;
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (am_last) {
        __threadfence();
        double s = 0.0;
        for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) s += ((volatile double*)part)[b];
        s = block_sum(s, smem);
        if (threadIdx.x == 0) {
            *out = s;
            *ticket = 0u;
        }
    }
}

static int red_grid(long long n) {
    int g = grid_for(n, 256, 8);
    return g > RedScratch::kMaxBlocks ? RedScratch::kMaxBlocks : g;
}

// out = <u, v>
__global__ void k_dot(const double* __restrict__ u, const double* __restrict__ v, long long n, double* part,
                      unsigned int* ticket, double* out) {
    __shared__ double sm[32];
    double s = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        s += u[t] * v[t];
    s = block_sum(s, sm);
    grid_reduce_finish(s, part, ticket, out, sm);
}

// MGS step: w -= (*hprev) * uprev (if uprev), then out = <w, uj>  (uj may be w -> squared norm)
__global__ void k_mgs(double* w, const double* __restrict__ uprev, const double* __restrict__ hprev,
                      const double* uj, long long n, double* part, unsigned int* ticket, double* out) {
    __shared__ double sm[32];
    const double h = uprev ? *hprev : 0.0;
    double s = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        double wv = w[t];
        if (uprev) {
            wv = wv - h * uprev[t];
            w[t] = wv;
        }
        s += wv * (uj == w ? wv : uj[t]);
    }
    s = block_sum(s, sm);
    grid_reduce_finish(s, part, ticket, out, sm);
}

// y = a*x + y with a from host
__global__ void k_axpy(double a, const double* __restrict__ x, double* __restrict__ y, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        y[t] = y[t] + a * x[t];
}

// y = x / d (d on device, the reference divides)
__global__ void k_divide(const double* x, const double* __restrict__ dptr, double* y,
                         long long n, int take_sqrt) {
    double d = *dptr;
    if (take_sqrt) d = sqrt(d);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        y[t] = x[t] / d;
}

// z = x - y
__global__ void k_sub(const double* x, const double* y, double* z, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        z[t] = x[t] - y[t];
}

// X += sum_j U_j y_j  (U_j at stride n), y on device
__global__ void k_multi_axpy(double* __restrict__ X, const double* __restrict__ U, const double* __restrict__ yv,
                             int m, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        double xv = X[t];
        for (int j = 0; j < m; ++j) xv = xv + U[(size_t)j * n + t] * yv[j];
        X[t] = xv;
    }
}

// ---------------------------------------------------------------------------
// Block SpMVs (SPARMULVV/VS/SV/SS, memLS.f90:2024-2236), 8 lanes per row.
// ---------------------------------------------------------------------------
constexpr int kLanes = 8;

__device__ __forceinline__ double group_sum8(double v) {
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    return v;
}

// KU = K U, K (9, nnz), U/KU (3, n)
__global__ void __launch_bounds__(256) k_spmv_vv3(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                  const double* __restrict__ K, const double* __restrict__ U,
                                                  double* __restrict__ KU, int n) {
    const int lane = threadIdx.x & (kLanes - 1);
    const long long ng = (long long)gridDim.x * (blockDim.x / kLanes);
    for (long long r0 = (long long)blockIdx.x * (blockDim.x / kLanes); r0 < n; r0 += ng) {
        const long long r = r0 + threadIdx.x / kLanes;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        if (r < n) {
            const int s = rowptr[r], e = rowptr[r + 1];
            for (int j = s + lane; j < e; j += kLanes) {
                const double* k = K + 9 * (size_t)j;
                const double* u = U + 3 * (size_t)col[j];
                const double u0 = u[0], u1 = u[1], u2 = u[2];
                a0 += k[0] * u0 + k[1] * u1 + k[2] * u2;
                a1 += k[3] * u0 + k[4] * u1 + k[5] * u2;
                a2 += k[6] * u0 + k[7] * u1 + k[8] * u2;
            }
        }
        a0 = group_sum8(a0);
        a1 = group_sum8(a1);
        a2 = group_sum8(a2);
        if (r < n && lane == 0) {
            KU[3 * r + 0] = a0;
            KU[3 * r + 1] = a1;
            KU[3 * r + 2] = a2;
        }
    }
}

// KU(i) = sum K(:,j).U(:,col)  (3 -> 1)
__global__ void __launch_bounds__(256) k_spmv_vs3(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                  const double* __restrict__ K, const double* __restrict__ U,
                                                  double* __restrict__ KU, int n) {
    const int lane = threadIdx.x & (kLanes - 1);
    const long long ng = (long long)gridDim.x * (blockDim.x / kLanes);
    for (long long r0 = (long long)blockIdx.x * (blockDim.x / kLanes); r0 < n; r0 += ng) {
        const long long r = r0 + threadIdx.x / kLanes;
        double a = 0.0;
        if (r < n) {
            const int s = rowptr[r], e = rowptr[r + 1];
            for (int j = s + lane; j < e; j += kLanes) {
                const double* k = K + 3 * (size_t)j;
                const double* u = U + 3 * (size_t)col[j];
                a += k[0] * u[0] + k[1] * u[1] + k[2] * u[2];
            }
        }
        a = group_sum8(a);
        if (r < n && lane == 0) KU[r] = a;
    }
}

// KU(:,i) = sum K(:,j) U(col)  (1 -> 3)
__global__ void __launch_bounds__(256) k_spmv_sv3(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                  const double* __restrict__ K, const double* __restrict__ U,
                                                  double* __restrict__ KU, int n) {
    const int lane = threadIdx.x & (kLanes - 1);
    const long long ng = (long long)gridDim.x * (blockDim.x / kLanes);
    for (long long r0 = (long long)blockIdx.x * (blockDim.x / kLanes); r0 < n; r0 += ng) {
        const long long r = r0 + threadIdx.x / kLanes;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        if (r < n) {
            const int s = rowptr[r], e = rowptr[r + 1];
            for (int j = s + lane; j < e; j += kLanes) {
                const double* k = K + 3 * (size_t)j;
                const double u = U[col[j]];
                a0 += k[0] * u;
                a1 += k[1] * u;
                a2 += k[2] * u;
            }
        }
        a0 = group_sum8(a0);
        a1 = group_sum8(a1);
        a2 = group_sum8(a2);
        if (r < n && lane == 0) {
            KU[3 * r + 0] = a0;
            KU[3 * r + 1] = a1;
            KU[3 * r + 2] = a2;
        }
    }
}

// CG operator: SP = L P - Gt GP, and out = <P, SP> (fused SPARMULSS, SPARMULVS, DOTS)
__global__ void __launch_bounds__(256) k_cg_op(const int* __restrict__ rowptr, const int* __restrict__ col,
                                               const double* __restrict__ L, const double* __restrict__ Gt,
                                               const double* __restrict__ P, const double* __restrict__ GP,
                                               double* __restrict__ SP, int n, double* part, unsigned int* ticket,
                                               double* out) {
    __shared__ double sm[32];
    const int lane = threadIdx.x & (kLanes - 1);
    const long long ng = (long long)gridDim.x * (blockDim.x / kLanes);
    double dsum = 0.0;
    for (long long r0 = (long long)blockIdx.x * (blockDim.x / kLanes); r0 < n; r0 += ng) {
        const long long r = r0 + threadIdx.x / kLanes;
        double a = 0.0, b = 0.0;
        if (r < n) {
            const int s = rowptr[r], e = rowptr[r + 1];
            for (int j = s + lane; j < e; j += kLanes) {
                const int c = col[j];
                a += L[j] * P[c];
                const double* g = Gt + 3 * (size_t)j;
                const double* gp = GP + 3 * (size_t)c;
                b += g[0] * gp[0] + g[1] * gp[1] + g[2] * gp[2];
            }
        }
        a = group_sum8(a);
        b = group_sum8(b);
        if (r < n && lane == 0) {
            const double v = a - b;
            SP[r] = v;
            dsum += P[r] * v;
        }
    }
    dsum = block_sum(dsum, sm);
    grid_reduce_finish(dsum, part, ticket, out, sm);
}

// X += alpha P, R -= alpha SP, out = <R, R>, alpha = (*errO)/(*den)
__global__ void k_cg_update(double* __restrict__ X, double* __restrict__ R, const double* __restrict__ P,
                            const double* __restrict__ SP, int n, const double* errO, const double* den, double* part,
                            unsigned int* ticket, double* out) {
    __shared__ double sm[32];
    const double alpha = *errO / *den;
    double s = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        X[t] = X[t] + alpha * P[t];
        double r = R[t] - alpha * SP[t];
        R[t] = r;
        s += r * r;
    }
    s = block_sum(s, sm);
    grid_reduce_finish(s, part, ticket, out, sm);
}

// P = R + (err/errO) P
__global__ void k_cg_dir(double* __restrict__ P, const double* __restrict__ R, int n, const double* err,
                         const double* errO) {
    const double f = *err / *errO;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) P[t] = R[t] + f * P[t];
}

// ---------------------------------------------------------------------------
// ADDBCMUL pieces (memLS.f90:206-268): S = <valM, X> over face nodes; Y += S*coef*valM
// ---------------------------------------------------------------------------
__global__ void k_face_dot(const int* __restrict__ glob, const double* __restrict__ valM, int fdof, int nsd,
                           int nNoF, const double* __restrict__ X, int dof, double* out) {
    __shared__ double sm[32];
    double s = 0.0;
    for (int a = threadIdx.x; a < nNoF; a += blockDim.x) {
        const int Ac = glob[a];
        for (int i = 0; i < nsd; ++i) s += valM[(size_t)fdof * a + i] * X[(size_t)dof * Ac + i];
    }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) *out = s;
}

__global__ void k_face_axpy(const int* __restrict__ glob, const double* __restrict__ valM, int fdof, int nsd,
                            int nNoF, const double* Sptr, double coef, double* __restrict__ Y, int dof) {
    const double S = coef * *Sptr;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nNoF; a += gridDim.x * blockDim.x) {
        const int Ac = glob[a];
        for (int i = 0; i < nsd; ++i) Y[(size_t)dof * Ac + i] = Y[(size_t)dof * Ac + i] + valM[(size_t)fdof * a + i] * S;
    }
}

// ---------------------------------------------------------------------------
// PRECOND (memLS.f90:1763-1943) pieces
// ---------------------------------------------------------------------------
// W from the diagonal blocks of Val (dof = 4, row-major 16 per block)
__global__ void k_w_from_val(double* __restrict__ Val, const int* __restrict__ diag, double* __restrict__ W, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double* v = Val + 16 * (size_t)diag[i];
        for (int d = 0; d < 4; ++d) {
            double w = v[5 * d];
            if (w == 0.0) {
                w = 1.0;
                v[5 * d] = 1.0;
            }
            W[4 * (size_t)i + d] = 1.0 / sqrt(fabs(w));
        }
    }
}

// W from lhsK / lhsP diagonals (fused SolFlow path; Val4 diagonal = K11,K22,K33,C)
__global__ void k_w_from_lhs(const double* __restrict__ lhsK, const double* __restrict__ lhsP,
                             const int* __restrict__ diag, double* __restrict__ W, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t k = (size_t)diag[i];
        double w[4] = {lhsK[9 * k + 0], lhsK[9 * k + 4], lhsK[9 * k + 8], lhsP[4 * k + 3]};
        for (int d = 0; d < 4; ++d) {
            double v = w[d] == 0.0 ? 1.0 : w[d];
            W[4 * (size_t)i + d] = 1.0 / sqrt(fabs(v));
        }
    }
}

// W(1:i, glob) *= val  (Dirichlet faces)
__global__ void k_w_dirichlet(const int* __restrict__ glob, const double* __restrict__ val, int fdof, int ni, int nNoF,
                              double* __restrict__ W) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nNoF; a += gridDim.x * blockDim.x) {
        const int Ac = glob[a];
        for (int i = 0; i < ni; ++i) W[4 * (size_t)Ac + i] = W[4 * (size_t)Ac + i] * val[(size_t)fdof * a + i];
    }
}

// Row then column scaling of Val (16 per block) + zero-diagonal fix + DEPART split
__global__ void k_scale_split_val(double* __restrict__ Val, const int* __restrict__ rowptr, const int* __restrict__ col,
                                  const int* __restrict__ diag, const int* __restrict__ trans,
                                  const double* __restrict__ W, int n, double* __restrict__ mK,
                                  double* __restrict__ mG, double* __restrict__ mD, double* __restrict__ mL) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const double* wr = W + 4 * (size_t)r;
        for (int j = rowptr[r]; j < rowptr[r + 1]; ++j) {
            const double* wc = W + 4 * (size_t)col[j];
            double* v = Val + 16 * (size_t)j;
            double t[16];
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b) t[4 * a + b] = (v[4 * a + b] * wr[a]) * wc[b];
            if (j == diag[r])
                for (int a = 0; a < 4; ++a)
                    if (t[5 * a] == 0.0) t[5 * a] = 1.0;
            for (int q = 0; q < 16; ++q) v[q] = t[q];
            double* k = mK + 9 * (size_t)j;
            k[0] = t[0]; k[1] = t[1]; k[2] = t[2];
            k[3] = t[4]; k[4] = t[5]; k[5] = t[6];
            k[6] = t[8]; k[7] = t[9]; k[8] = t[10];
            mG[3 * (size_t)j + 0] = t[3];
            mG[3 * (size_t)j + 1] = t[7];
            mG[3 * (size_t)j + 2] = t[11];
            mD[3 * (size_t)j + 0] = t[12];
            mD[3 * (size_t)j + 1] = t[13];
            mD[3 * (size_t)j + 2] = t[14];
            mL[j] = t[15];
        }
    }
}

// Gt(:, l) = -mG(:, trans(l))  (DEPART's transpose search, memLS.f90:1664-1675)
__global__ void k_gt(const double* __restrict__ mG, const int* __restrict__ trans, long long nnz, double* __restrict__ Gt) {
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < nnz; l += (long long)gridDim.x * blockDim.x) {
        const size_t j = (size_t)trans[l];
        Gt[3 * l + 0] = -mG[3 * j + 0];
        Gt[3 * l + 1] = -mG[3 * j + 1];
        Gt[3 * l + 2] = -mG[3 * j + 2];
    }
}

// Fused SolFlow pack + PRECOND scaling + DEPART from lhsK / lhsP:
//   Val4 rows 1-3 cols 1-3 = lhsK, col 4 rows 1-3 = -lhsP(1:3) of the
//   transposed block, row 4 cols 1-3 = lhsP(1:3), (4,4) = lhsP(4)
//   (solfar.f90:217-232), scaled by W(row) W(col) and split.
__global__ void k_scale_split_lhs(const double* __restrict__ lhsK, const double* __restrict__ lhsP,
                                  const int* __restrict__ rowptr, const int* __restrict__ col,
                                  const int* __restrict__ diag, const int* __restrict__ trans,
                                  const double* __restrict__ W, int n, double* __restrict__ mK,
                                  double* __restrict__ mG, double* __restrict__ mD, double* __restrict__ mL) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const double* wr = W + 4 * (size_t)r;
        const int dg = diag[r];
        for (int j = rowptr[r]; j < rowptr[r + 1]; ++j) {
            const double* wc = W + 4 * (size_t)col[j];
            const double* K = lhsK + 9 * (size_t)j;
            const double* Pj = lhsP + 4 * (size_t)j;
            const double* Pt = lhsP + 4 * (size_t)trans[j];
            double* k = mK + 9 * (size_t)j;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    double v = K[3 * a + b];
                    if (j == dg && a == b && v == 0.0) v = 1.0;
                    double t = (v * wr[a]) * wc[b];
                    if (j == dg && a == b && t == 0.0) t = 1.0;
                    k[3 * a + b] = t;
                }
            for (int a = 0; a < 3; ++a) mG[3 * (size_t)j + a] = (-Pt[a] * wr[a]) * wc[3];
            for (int b = 0; b < 3; ++b) mD[3 * (size_t)j + b] = (Pj[b] * wr[3]) * wc[b];
            double v = Pj[3];
            if (j == dg && v == 0.0) v = 1.0;
            double t = (v * wr[3]) * wc[3];
            if (j == dg && t == 0.0) t = 1.0;
            mL[j] = t;
        }
    }
}

// R = W*R  (node-major, dof 4), and R = R*W afterwards
__global__ void k_mul(double* __restrict__ R, const double* __restrict__ W, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        R[t] = W[t] * R[t];
}

// split (4, n) into (3, n) and (n), and merge back
__global__ void k_split4(const double* __restrict__ R, double* __restrict__ Rm, double* __restrict__ Rc, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Rm[3 * (size_t)i + 0] = R[4 * (size_t)i + 0];
        Rm[3 * (size_t)i + 1] = R[4 * (size_t)i + 1];
        Rm[3 * (size_t)i + 2] = R[4 * (size_t)i + 2];
        Rc[i] = R[4 * (size_t)i + 3];
    }
}
__global__ void k_merge4(double* __restrict__ R, const double* __restrict__ Rm, const double* __restrict__ Rc, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        R[4 * (size_t)i + 0] = Rm[3 * (size_t)i + 0];
        R[4 * (size_t)i + 1] = Rm[3 * (size_t)i + 1];
        R[4 * (size_t)i + 2] = Rm[3 * (size_t)i + 2];
        R[4 * (size_t)i + 3] = Rc[i];
    }
}

// face%valM = face%val * W  (coupled faces)
__global__ void k_valm(const int* __restrict__ glob, const double* __restrict__ val, double* __restrict__ valM, int fdof,
                       int ni, int nNoF, const double* __restrict__ W) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nNoF; a += gridDim.x * blockDim.x)
        for (int i = 0; i < ni; ++i)
            valM[(size_t)fdof * a + i] = val[(size_t)fdof * a + i] * W[4 * (size_t)glob[a] + i];
}

}  // namespace crimson

namespace crimson {

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// device scalar slots
enum {
    kSlotDot = 0,
    kSlotNrm = 1,
    kSlotErr = 2,
    kSlotErrO = 3,
    kSlotDen = 4,
    kSlotFace = 8,      // up to 32 faces
    kSlotH = 64,        // Hessenberg column (sD + 1)
    kSlotY = 64 + 512,  // back-substitution coefficients
    kSlotGram = 64 + 1024,
    kScalTotal = 64 + 1024 + 4096
};

struct Ctx {
    crimson_lhs* L;
    cudaStream_t s;
    double* sc(int i) { return L->scal.p + i; }
    int sync_scal(int first, int count) {
        CR_CUDA(cudaMemcpyAsync(L->hscal + first, L->scal.p + first, sizeof(double) * count, cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        return CRIMSON_OK;
    }
    void dot(const double* u, const double* v, long long n, int slot) {
        launch(k_dot, red_grid(n), 256, 0, s, u, v, n, L->red.part.p, L->red.ticket.p, sc(slot));
    }
    void spmv_vv3(const double* K, const double* U, double* KU) {
        launch(k_spmv_vv3, grid_for((long long)L->nNo * kLanes, 256, 8), 256, 0, s, L->rowptr, L->col, K, U, KU, L->nNo);
    }
    void spmv_vs3(const double* K, const double* U, double* KU) {
        launch(k_spmv_vs3, grid_for((long long)L->nNo * kLanes, 256, 8), 256, 0, s, L->rowptr, L->col, K, U, KU, L->nNo);
    }
    void spmv_sv3(const double* K, const double* U, double* KU) {
        launch(k_spmv_sv3, grid_for((long long)L->nNo * kLanes, 256, 8), 256, 0, s, L->rowptr, L->col, K, U, KU, L->nNo);
    }
    void spmv_ss_into(const double* Kd, const double* U, double* KU);
    bool any_coupled() const {
        for (auto& f : L->face)
            if (f.coupledFlag) return true;
        return false;
    }
    // ADDBCMUL on nsd-dof vectors: all face dots first (on X), then all updates of Y
    void addbcmul(int op, int dof, const double* X, double* Y) {
        int k = 0;
        for (auto& f : L->face) {
            if (f.coupledFlag) {
                int nsd = std::min(f.dof, dof);
                launch(k_face_dot, 1, 512, 0, s, f.glob.p, f.valM.p, f.dof, nsd, f.nNo, X, dof, sc(kSlotFace + k));
            }
            ++k;
        }
        k = 0;
        for (auto& f : L->face) {
            if (f.coupledFlag) {
                int nsd = std::min(f.dof, dof);
                double coef = (op == 0) ? f.res : -f.res / (1.0 + f.res * f.nS);
                launch(k_face_axpy, grid_for(f.nNo, 256), 256, 0, s, f.glob.p, f.valM.p, f.dof, nsd, f.nNo,
                                                                 sc(kSlotFace + k), coef, Y, dof);
            }
            ++k;
        }
    }
};

__global__ void k_spmv_ss(const int* __restrict__ rowptr, const int* __restrict__ col, const double* __restrict__ K,
                          const double* __restrict__ U, double* __restrict__ KU, int n) {
    const int lane = threadIdx.x & (kLanes - 1);
    const long long ng = (long long)gridDim.x * (blockDim.x / kLanes);
    for (long long r0 = (long long)blockIdx.x * (blockDim.x / kLanes); r0 < n; r0 += ng) {
        const long long r = r0 + threadIdx.x / kLanes;
        double a = 0.0;
        if (r < n) {
            const int s = rowptr[r], e = rowptr[r + 1];
            for (int j = s + lane; j < e; j += kLanes) a += K[j] * U[col[j]];
        }
        a = group_sum8(a);
        if (r < n && lane == 0) KU[r] = a;
    }
}

void Ctx::spmv_ss_into(const double* Kd, const double* U, double* KU) {
    launch(k_spmv_ss, grid_for((long long)L->nNo * kLanes, 256, 8), 256, 0, s, L->rowptr, L->col, Kd, U, KU, L->nNo);
}

// GMRES (memLS.f90:681-788) on dof = 3 with K = mK; X may not alias R.
static int gmres(Ctx& C, crimson_subls& ls, const double* K, const double* R, double* X) {
    crimson_lhs* L = C.L;
    cudaStream_t s = C.s;
    const int dof = 3;
    const long long n = (long long)dof * L->nNo;
    const int sD = ls.sD;
    double* u = L->basis.p;
    auto U = [&](int k) { return u + (size_t)k * n; };
    std::vector<double> h((size_t)(sD + 1) * sD, 0.0), c(sD), sn(sD), err(sD + 1), y(sD);
    auto H = [&](int i, int j) -> double& { return h[(size_t)j * (sD + 1) + i]; };
    const double time = now_s();
    ls.suc = 0;
    CR_CUDA(cudaMemsetAsync(X, 0, sizeof(double) * n, s));
    double eps = 0.0;
    const bool coupled = C.any_coupled();
    int i = 0;
    for (int l = 1; l <= ls.mItr; ++l) {
        if (l == 1) {
            CR_CUDA(cudaMemcpyAsync(U(0), R, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        } else {
            ls.itr = ls.itr + 1;
            C.spmv_vv3(K, X, U(0));
            C.addbcmul(0, dof, X, U(0));
            launch(k_sub, grid_for(n, 256), 256, 0, s, R, U(0), U(0), n);
        }
        if (coupled) {
            CR_CUDA(cudaMemcpyAsync(L->w3.p, U(0), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
            C.addbcmul(1, dof, L->w3.p, U(0));
        }
        C.dot(U(0), U(0), n, kSlotNrm);
        CR_CHECK(C.sync_scal(kSlotNrm, 1));
        err[0] = std::sqrt(L->hscal[kSlotNrm]);
        if (l == 1) {
            eps = err[0];
            if (eps <= ls.absTol) {
                ls.callD = 0.0;
                ls.dB = 0.0;
                return CRIMSON_OK;
            }
            ls.iNorm = eps;
            ls.fNorm = eps;
            eps = std::max(ls.absTol, ls.relTol * eps);
        }
        ls.dB = ls.fNorm;
        launch(k_divide, grid_for(n, 256), 256, 0, s, U(0), C.sc(kSlotNrm), U(0), n, 1);
        for (i = 1; i <= sD; ++i) {
            ls.itr = ls.itr + 1;
            double* w = U(i);
            C.spmv_vv3(K, U(i - 1), w);
            C.addbcmul(0, dof, U(i - 1), w);
            if (coupled) {
                CR_CUDA(cudaMemcpyAsync(L->w3.p, w, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
                C.addbcmul(1, dof, L->w3.p, w);
            }
            // fused modified Gram-Schmidt
            for (int j = 1; j <= i; ++j) {
                const double* uprev = (j == 1) ? nullptr : U(j - 2);
                launch(k_mgs, red_grid(n), 256, 0, s, w, uprev, C.sc(kSlotH + j - 2), U(j - 1), n, L->red.part.p,
                                                  L->red.ticket.p, C.sc(kSlotH + j - 1));
            }
            launch(k_mgs, red_grid(n), 256, 0, s, w, U(i - 1), C.sc(kSlotH + i - 1), w, n, L->red.part.p, L->red.ticket.p,
                                              C.sc(kSlotH + i));
            launch(k_divide, grid_for(n, 256), 256, 0, s, w, C.sc(kSlotH + i), w, n, 1);
            CR_CHECK(C.sync_scal(kSlotH, i + 1));
            for (int j = 1; j <= i; ++j) H(j - 1, i - 1) = L->hscal[kSlotH + j - 1];
            H(i, i - 1) = std::sqrt(L->hscal[kSlotH + i]);
            double tmp;
            for (int j = 1; j <= i - 1; ++j) {
                tmp = c[j - 1] * H(j - 1, i - 1) + sn[j - 1] * H(j, i - 1);
                H(j, i - 1) = -sn[j - 1] * H(j - 1, i - 1) + c[j - 1] * H(j, i - 1);
                H(j - 1, i - 1) = tmp;
            }
            tmp = std::sqrt(H(i - 1, i - 1) * H(i - 1, i - 1) + H(i, i - 1) * H(i, i - 1));
            c[i - 1] = H(i - 1, i - 1) / tmp;
            sn[i - 1] = H(i, i - 1) / tmp;
            H(i - 1, i - 1) = tmp;
            H(i, i - 1) = 0.0;
            err[i] = -sn[i - 1] * err[i - 1];
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
        std::memcpy(L->hscal + kSlotY, y.data(), sizeof(double) * i);
        CR_CUDA(cudaMemcpyAsync(C.sc(kSlotY), L->hscal + kSlotY, sizeof(double) * i, cudaMemcpyHostToDevice, s));
        launch(k_multi_axpy, grid_for(n, 256), 256, 0, s, X, u, C.sc(kSlotY), i, n);
        CR_CUDA(cudaStreamSynchronize(s));   // y staging buffer is reused
        ls.fNorm = std::fabs(err[i]);
        if (ls.suc) break;
    }
    ls.callD = now_s() - time + ls.callD;
    ls.dB = 10.0 * std::log(ls.fNorm / ls.dB);
    return CRIMSON_OK;
}

// CGRAD (memLS.f90:367-430) on the Schur-like operator L P - Gt G P; R in/out (n)
static int cgrad(Ctx& C, crimson_subls& ls, const double* Gt, const double* G, const double* Lm, double* R) {
    crimson_lhs* L = C.L;
    cudaStream_t s = C.s;
    const int n = L->nNo;
    const double time = now_s();
    const bool coupled = C.any_coupled();
    double* X = L->cgX.p;
    double* P = L->cgP.p;
    double* SP = L->cgSP.p;
    double* GP = L->cgGP.p;
    ls.suc = 0;
    C.dot(R, R, n, kSlotErr);
    CR_CHECK(C.sync_scal(kSlotErr, 1));
    double errO = std::sqrt(L->hscal[kSlotErr]);
    ls.iNorm = errO;
    double eps = std::max(ls.absTol, ls.relTol * errO);
    eps = eps * eps;
    double err = errO;
    err = err * err;
    // the device err slot holds the squared norm; the reference re-squares sqrt(sum)
    L->hscal[kSlotErr] = err;
    CR_CUDA(cudaMemcpyAsync(C.sc(kSlotErr), L->hscal + kSlotErr, sizeof(double), cudaMemcpyHostToDevice, s));
    CR_CUDA(cudaMemsetAsync(X, 0, sizeof(double) * n, s));
    CR_CUDA(cudaMemcpyAsync(P, R, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    int i;
    for (i = 1; i <= ls.mItr; ++i) {
        if (err < eps) {
            ls.suc = 1;
            break;
        }
        errO = err;
        CR_CUDA(cudaMemcpyAsync(C.sc(kSlotErrO), C.sc(kSlotErr), sizeof(double), cudaMemcpyDeviceToDevice, s));
        C.spmv_sv3(G, P, GP);
        if (coupled) {
            CR_CUDA(cudaMemcpyAsync(L->w3.p, GP, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToDevice, s));
            C.addbcmul(1, 3, L->w3.p, GP);
        }
        launch(k_cg_op, red_grid((long long)n * kLanes), 256, 0, s, L->rowptr, L->col, Lm, Gt, P, GP, SP, n,
                                                                L->red.part.p, L->red.ticket.p, C.sc(kSlotDen));
        launch(k_cg_update, red_grid(n), 256, 0, s, X, R, P, SP, n, C.sc(kSlotErrO), C.sc(kSlotDen), L->red.part.p,
                                                L->red.ticket.p, C.sc(kSlotErr));
        CR_CHECK(C.sync_scal(kSlotErr, 1));
        double e2 = std::sqrt(L->hscal[kSlotErr]);
        err = e2 * e2;
        L->hscal[kSlotErr] = err;
        CR_CUDA(cudaMemcpyAsync(C.sc(kSlotErr), L->hscal + kSlotErr, sizeof(double), cudaMemcpyHostToDevice, s));
        launch(k_cg_dir, grid_for(n, 256), 256, 0, s, P, R, n, C.sc(kSlotErr), C.sc(kSlotErrO));
    }
    CR_CUDA(cudaMemcpyAsync(R, X, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    CR_CUDA(cudaStreamSynchronize(s));
    ls.fNorm = std::sqrt(err);
    ls.callD = now_s() - time + ls.callD;
    ls.dB = 5.0 * std::log(err / errO);
    ls.itr = ls.itr + i - 1;
    return CRIMSON_OK;
}

// GE (memLS.f90:607-677), A column-major
static int ge_solve(int N, const double* A, double* B) {
    if (N == 2) {
        double pivot = A[0] * A[3] - A[1] * A[2];
        double saveEl = (B[0] * A[3] - B[1] * A[2]) / pivot;
        B[1] = (B[1] * A[0] - B[0] * A[1]) / pivot;
        B[0] = saveEl;
        return CRIMSON_OK;
    }
    std::vector<double> Cm((size_t)N * (N + 1));
    auto c = [&](int i, int j) -> double& { return Cm[(size_t)j * N + i]; };
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
        if (pivot < 2.0 * 2.220446049250313e-16) return CRIMSON_ERR_SINGULAR;
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
    return CRIMSON_OK;
}

// NSSOLVER (memLS.f90:1460-1759); R (4, nNo) in/out
static int nssolver(crimson_lhs* L, crimson_ls* ls, const double* mK, const double* mG, const double* mD,
                    const double* mL, const double* Gt, double* R) {
    Ctx C{L, L->stream};
    cudaStream_t s = L->stream;
    const int nNo = L->nNo;
    const long long nv = 3LL * nNo;
    int iB = ls->RI.mItr;
    const int nB = 2 * iB;
    auto Ucol = [&](int k) { return L->U.p + (size_t)k * nv; };
    auto Pcol = [&](int k) { return L->P.p + (size_t)k * nNo; };
    auto MUc = [&](int k) { return L->MU.p + (size_t)k * nv; };
    auto MPc = [&](int k) { return L->MP.p + (size_t)k * nNo; };
    launch(k_split4, grid_for(nNo, 256), 256, 0, s, R, L->Rmi.p, L->Rci.p, nNo);
    CR_CUDA(cudaMemcpyAsync(L->Rm.p, L->Rmi.p, sizeof(double) * nv, cudaMemcpyDeviceToDevice, s));
    CR_CUDA(cudaMemcpyAsync(L->Rc.p, L->Rci.p, sizeof(double) * nNo, cudaMemcpyDeviceToDevice, s));
    std::vector<double> A((size_t)nB * nB, 0.0), B(nB, 0.0), xB(nB, 0.0);
    auto Aa = [&](int i, int j) -> double& { return A[(size_t)j * nB + i]; };
    C.dot(L->Rm.p, L->Rm.p, nv, 0);
    C.dot(L->Rc.p, L->Rc.p, nNo, 1);
    CR_CHECK(C.sync_scal(0, 2));
    double nv1 = std::sqrt(L->hscal[0]), ns1 = std::sqrt(L->hscal[1]);
    double eps = std::sqrt(std::pow(nv1, 2.0) + std::pow(ns1, 2.0));
    ls->RI.iNorm = eps;
    ls->RI.fNorm = eps;
    ls->CG.callD = 0.0;
    ls->GM.callD = 0.0;
    ls->CG.itr = 0;
    ls->GM.itr = 0;
    const double t0 = now_s();
    ls->RI.suc = 0;
    eps = std::max(ls->RI.absTol, ls->RI.relTol * eps);
    // BCPRE (memLS.f90:1683-1716): nS = |valM|^2 per coupled face, summed on
    // the host in the reference's node order (faces are small).
    for (auto& f : L->face) {
        if (!f.coupledFlag) continue;
        std::vector<double> vm((size_t)f.dof * f.nNo);
        CR_CUDA(cudaMemcpyAsync(vm.data(), f.valM.p, sizeof(double) * vm.size(), cudaMemcpyDeviceToHost, s));
        CR_CUDA(cudaStreamSynchronize(s));
        f.nS = 0.0;
        const int nsd = std::min(f.dof, 3);
        for (int a = 0; a < f.nNo; ++a)
            for (int i = 0; i < nsd; ++i) f.nS = f.nS + std::pow(vm[(size_t)f.dof * a + i], 2.0);
    }
    int i, iBB = 0;
    for (i = 1; i <= ls->RI.mItr; ++i) {
        iB = 2 * i - 1;
        iBB = 2 * i;
        ls->RI.dB = ls->RI.fNorm;
        CR_CHECK(gmres(C, ls->GM, mK, L->Rm.p, Ucol(i - 1)));
        C.spmv_vs3(mD, Ucol(i - 1), Pcol(i - 1));
        launch(k_sub, grid_for(nNo, 256), 256, 0, s, L->Rc.p, Pcol(i - 1), Pcol(i - 1), nNo);
        CR_CHECK(cgrad(C, ls->CG, Gt, mG, mL, Pcol(i - 1)));
        C.spmv_sv3(mG, Pcol(i - 1), MUc(iB - 1));
        launch(k_sub, grid_for(nv, 256), 256, 0, s, L->Rm.p, MUc(iB - 1), MUc(iBB - 1), nv);
        CR_CHECK(gmres(C, ls->GM, mK, MUc(iBB - 1), Ucol(i - 1)));
        C.spmv_vv3(mK, Ucol(i - 1), MUc(iBB - 1));
        C.addbcmul(0, 3, Ucol(i - 1), MUc(iBB - 1));
        C.spmv_ss_into(mL, Pcol(i - 1), MPc(iB - 1));
        C.spmv_vs3(mD, Ucol(i - 1), MPc(iBB - 1));
        // Gram matrix entries for columns iB, iBB
        int slot = kSlotGram;
        for (int k = iB; k <= iBB; ++k) {
            for (int j = 1; j <= k - 1; ++j) {
                C.dot(MUc(j - 1), MUc(k - 1), nv, slot++);
                C.dot(MPc(j - 1), MPc(k - 1), nNo, slot++);
            }
            C.dot(MUc(k - 1), MUc(k - 1), nv, slot++);
            C.dot(MPc(k - 1), MPc(k - 1), nNo, slot++);
            C.dot(MUc(k - 1), L->Rmi.p, nv, slot++);
            C.dot(MPc(k - 1), L->Rci.p, nNo, slot++);
        }
        CR_CHECK(C.sync_scal(kSlotGram, slot - kSlotGram));
        slot = kSlotGram;
        for (int k = iB; k <= iBB; ++k) {
            for (int j = 1; j <= k - 1; ++j) {
                Aa(j - 1, k - 1) = L->hscal[slot] + L->hscal[slot + 1];
                slot += 2;
                Aa(k - 1, j - 1) = Aa(j - 1, k - 1);
            }
            Aa(k - 1, k - 1) = std::pow(std::sqrt(L->hscal[slot]), 2.0) + std::pow(std::sqrt(L->hscal[slot + 1]), 2.0);
            slot += 2;
            B[k - 1] = L->hscal[slot] + L->hscal[slot + 1];
            slot += 2;
        }
        for (int t = 0; t < iBB; ++t) xB[t] = B[t];
        std::vector<double> Asub((size_t)iBB * iBB);
        for (int c = 0; c < iBB; ++c)
            for (int r = 0; r < iBB; ++r) Asub[(size_t)c * iBB + r] = Aa(r, c);
        CR_CHECK(ge_solve(iBB, Asub.data(), xB.data()));
        double sxb = 0.0;
        for (int t = 0; t < iBB; ++t) sxb = sxb + xB[t] * B[t];
        ls->RI.fNorm = std::sqrt(std::pow(ls->RI.iNorm, 2.0) - sxb);
        if (ls->RI.fNorm < eps) {
            ls->RI.suc = 1;
            break;
        }
        // Rm = Rmi - sum xB_j MU_j ; Rc = Rci - sum xB_j MP_j
        CR_CUDA(cudaMemcpyAsync(L->Rm.p, L->Rmi.p, sizeof(double) * nv, cudaMemcpyDeviceToDevice, s));
        CR_CUDA(cudaMemcpyAsync(L->Rc.p, L->Rci.p, sizeof(double) * nNo, cudaMemcpyDeviceToDevice, s));
        for (int j = 1; j <= iBB; ++j) {
            launch(k_axpy, grid_for(nv, 256), 256, 0, s, -xB[j - 1], MUc(j - 1), L->Rm.p, nv);
            launch(k_axpy, grid_for(nNo, 256), 256, 0, s, -xB[j - 1], MPc(j - 1), L->Rc.p, nNo);
        }
    }
    if (i > ls->RI.mItr) {
        ls->RI.itr = ls->RI.mItr;
    } else {
        ls->RI.itr = i;
        CR_CUDA(cudaMemcpyAsync(L->Rc.p, L->Rci.p, sizeof(double) * nNo, cudaMemcpyDeviceToDevice, s));
        for (int j = 1; j <= iBB; ++j) launch(k_axpy, grid_for(nNo, 256), 256, 0, s, -xB[j - 1], MPc(j - 1), L->Rc.p, nNo);
    }
    C.dot(L->Rc.p, L->Rc.p, nNo, 0);
    CR_CHECK(C.sync_scal(0, 1));
    ls->Resc = (int)std::lround(100.0 * std::pow(std::sqrt(L->hscal[0]) / ls->RI.fNorm, 2.0));
    ls->Resm = 100 - ls->Resc;
    // solution: Rmi = xB(2) U_1 + sum xB(2i) U_i ; Rci = xB(1) P_1 + sum xB(2i-1) P_i
    CR_CUDA(cudaMemsetAsync(L->Rmi.p, 0, sizeof(double) * nv, s));
    CR_CUDA(cudaMemsetAsync(L->Rci.p, 0, sizeof(double) * nNo, s));
    launch(k_axpy, grid_for(nv, 256), 256, 0, s, xB[1], Ucol(0), L->Rmi.p, nv);
    launch(k_axpy, grid_for(nNo, 256), 256, 0, s, xB[0], Pcol(0), L->Rci.p, nNo);
    for (i = 2; i <= ls->RI.itr; ++i) {
        launch(k_axpy, grid_for(nv, 256), 256, 0, s, xB[2 * i - 1], Ucol(i - 1), L->Rmi.p, nv);
        launch(k_axpy, grid_for(nNo, 256), 256, 0, s, xB[2 * i - 2], Pcol(i - 1), L->Rci.p, nNo);
    }
    launch(k_merge4, grid_for(nNo, 256), 256, 0, s, R, L->Rmi.p, L->Rci.p, nNo);
    CR_CUDA(cudaStreamSynchronize(s));
    ls->RI.callD = now_s() - t0;
    ls->RI.dB = 10.0 * std::log(ls->RI.fNorm / ls->RI.dB);
    CR_CUDA(cudaGetLastError());
    return CRIMSON_OK;
}

static int lhs_work_alloc(crimson_lhs* L, const crimson_ls* ls) {
    const int nNo = L->nNo;
    const long long nnz = L->nnz;
    const int iB = ls->RI.mItr;
    const int sD = ls->GM.sD;
    CR_CHECK(L->W.alloc(4 * (size_t)nNo));
    CR_CHECK(L->R.alloc(4 * (size_t)nNo));
    CR_CHECK(L->mK.alloc(9 * (size_t)nnz));
    CR_CHECK(L->mG.alloc(3 * (size_t)nnz));
    CR_CHECK(L->mD.alloc(3 * (size_t)nnz));
    CR_CHECK(L->mL.alloc((size_t)nnz));
    CR_CHECK(L->Rm.alloc(3 * (size_t)nNo));
    CR_CHECK(L->Rc.alloc((size_t)nNo));
    CR_CHECK(L->Rmi.alloc(3 * (size_t)nNo));
    CR_CHECK(L->Rci.alloc((size_t)nNo));
    CR_CHECK(L->U.alloc(3 * (size_t)nNo * iB));
    CR_CHECK(L->P.alloc((size_t)nNo * iB));
    CR_CHECK(L->MU.alloc(3 * (size_t)nNo * 2 * iB));
    CR_CHECK(L->MP.alloc((size_t)nNo * 2 * iB));
    CR_CHECK(L->basis.alloc(3 * (size_t)nNo * (sD + 1)));
    CR_CHECK(L->w3.alloc(3 * (size_t)nNo));
    CR_CHECK(L->cgX.alloc((size_t)nNo));
    CR_CHECK(L->cgP.alloc((size_t)nNo));
    CR_CHECK(L->cgSP.alloc((size_t)nNo));
    CR_CHECK(L->cgGP.alloc(3 * (size_t)nNo));
    if (!L->scal.p) {
        CR_CHECK(L->scal.alloc(kScalTotal));
        CR_CHECK(L->red.init());
        CR_CUDA(cudaMallocHost(&L->hscal, sizeof(double) * kScalTotal));
    }
    if (sD + 1 > 512 || iB * 8 * iB + 64 > 4096) return CRIMSON_ERR_UNSUPPORTED;
    return CRIMSON_OK;
}

// memLS_SOLVE face flags (memLS.f90:1955-1986)
static void set_face_flags(crimson_lhs* L, const int* incL, const double* res) {
    for (int fa = 0; fa < L->nFaces; ++fa) {
        MemlsFace& f = L->face[fa];
        f.incFlag = !(incL && incL[fa] == 0);
        f.coupledFlag = false;
        if (!f.incFlag) continue;
        if (f.bGrp == CRIMSON_BC_TYPE_NEU && res && res[fa] != 0.0) {
            f.res = res[fa];
            f.coupledFlag = true;
        }
    }
}

// Dirichlet W scaling + valM of coupled faces (tail of PRECOND)
static int precond_faces(crimson_lhs* L, bool after_scale) {
    cudaStream_t s = L->stream;
    for (auto& f : L->face) {
        if (!f.created || f.nNo == 0) continue;
        if (!after_scale) {
            if (f.incFlag && f.bGrp == CRIMSON_BC_TYPE_DIR)
                launch(k_w_dirichlet, grid_for(f.nNo, 256), 256, 0, s, f.glob.p, f.val.p, f.dof, std::min(f.dof, 4), f.nNo,
                                                                   L->W.p);
        } else if (f.coupledFlag) {
            launch(k_valm, grid_for(f.nNo, 256), 256, 0, s, f.glob.p, f.val.p, f.valM.p, f.dof, std::min(f.dof, 4), f.nNo,
                                                        L->W.p);
        }
    }
    CR_CUDA(cudaGetLastError());
    return CRIMSON_OK;
}

int memls_solve_val(crimson_lhs* L, crimson_ls* ls, double* Ri, double* Val, const int* incL, const double* res,
                    crimson_ls_stats* st) {
    cudaStream_t s = L->stream;
    CR_CHECK(lhs_work_alloc(L, ls));
    CR_CHECK(L->Val.alloc(16 * (size_t)L->nnz));
    CR_CHECK(L->Gt.alloc(3 * (size_t)L->nnz));
    set_face_flags(L, incL, res);
    CR_CUDA(cudaMemcpyAsync(L->R.p, Ri, sizeof(double) * 4 * (size_t)L->nNo, cudaMemcpyHostToDevice, s));
    CR_CUDA(cudaMemcpyAsync(L->Val.p, Val, sizeof(double) * 16 * (size_t)L->nnz, cudaMemcpyHostToDevice, s));
    launch(k_w_from_val, grid_for(L->nNo, 256), 256, 0, s, L->Val.p, L->diag, L->W.p, L->nNo);
    CR_CHECK(precond_faces(L, false));
    launch(k_scale_split_val, grid_for(L->nNo, 128), 128, 0, s, L->Val.p, L->rowptr, L->col, L->diag, L->trans, L->W.p,
                                                           L->nNo, L->mK.p, L->mG.p, L->mD.p, L->mL.p);
    launch(k_gt, grid_for(L->nnz, 256), 256, 0, s, L->mG.p, L->trans, L->nnz, L->Gt.p);
    launch(k_mul, grid_for(4LL * L->nNo, 256), 256, 0, s, L->R.p, L->W.p, 4LL * L->nNo);
    CR_CHECK(precond_faces(L, true));
    CR_CHECK(nssolver(L, ls, L->mK.p, L->mG.p, L->mD.p, L->mL.p, L->Gt.p, L->R.p));
    launch(k_mul, grid_for(4LL * L->nNo, 256), 256, 0, s, L->R.p, L->W.p, 4LL * L->nNo);
    CR_CUDA(cudaMemcpyAsync(Ri, L->R.p, sizeof(double) * 4 * (size_t)L->nNo, cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaMemcpyAsync(Val, L->Val.p, sizeof(double) * 16 * (size_t)L->nnz, cudaMemcpyDeviceToHost, s));
    CR_CUDA(cudaStreamSynchronize(s));
    if (st) {
        st->GM = ls->GM;
        st->CG = ls->CG;
        st->RI = ls->RI;
        st->LS_type = ls->LS_type;
        st->Resm = ls->Resm;
        st->Resc = ls->Resc;
    }
    return CRIMSON_OK;
}

int memls_solve_lhs_device(crimson_lhs* L, crimson_ls* ls, const double* d_res, const double* d_lhsK,
                           const double* d_lhsP, const int* incL, const double* faceRes, double* d_sol,
                           crimson_ls_stats* st) {
    cudaStream_t s = L->stream;
    CR_CHECK(lhs_work_alloc(L, ls));
    set_face_flags(L, incL, faceRes);
    CR_CUDA(cudaMemcpyAsync(L->R.p, d_res, sizeof(double) * 4 * (size_t)L->nNo, cudaMemcpyDeviceToDevice, s));
    launch(k_w_from_lhs, grid_for(L->nNo, 256), 256, 0, s, d_lhsK, d_lhsP, L->diag, L->W.p, L->nNo);
    CR_CHECK(precond_faces(L, false));
    launch(k_scale_split_lhs, grid_for(L->nNo, 128), 128, 0, s, d_lhsK, d_lhsP, L->rowptr, L->col, L->diag, L->trans,
                                                           L->W.p, L->nNo, L->mK.p, L->mG.p, L->mD.p, L->mL.p);
    launch(k_mul, grid_for(4LL * L->nNo, 256), 256, 0, s, L->R.p, L->W.p, 4LL * L->nNo);
    CR_CHECK(precond_faces(L, true));
    // With Val4 built from lhsK/lhsP, Gt = -mG^T equals mD up to the order of
    // the two scaling products, so mD serves as Gt.
    CR_CHECK(nssolver(L, ls, L->mK.p, L->mG.p, L->mD.p, L->mL.p, L->mD.p, L->R.p));
    launch(k_mul, grid_for(4LL * L->nNo, 256), 256, 0, s, L->R.p, L->W.p, 4LL * L->nNo);
    CR_CUDA(cudaMemcpyAsync(d_sol, L->R.p, sizeof(double) * 4 * (size_t)L->nNo, cudaMemcpyDeviceToDevice, s));
    CR_CUDA(cudaStreamSynchronize(s));
    if (st) {
        st->GM = ls->GM;
        st->CG = ls->CG;
        st->RI = ls->RI;
        st->LS_type = ls->LS_type;
        st->Resm = ls->Resm;
        st->Resc = ls->Resc;
    }
    return CRIMSON_OK;
}

}  // namespace crimson

namespace crimson {

// Average device time of one launch of a memLS kernel on the lhs's current
// split matrices (events recorded on the lhs stream around reps launches).
int memls_kernel_time(crimson_lhs* L, int which, int reps, double* ms) {
    if (!L->mK.p || !L->basis.p || reps <= 0) return CRIMSON_ERR_STATE;
    cudaStream_t s = L->stream;
    Ctx C{L, s};
    const long long n3 = 3LL * L->nNo;
    cudaEvent_t e0, e1;
    CR_CUDA(cudaEventCreate(&e0));
    CR_CUDA(cudaEventCreate(&e1));
    auto run = [&]() {
        switch (which) {
            case 0: C.spmv_vv3(L->mK.p, L->basis.p, L->basis.p + n3); break;
            case 1:
                launch(k_cg_op, red_grid((long long)L->nNo * kLanes), 256, 0, s, L->rowptr, L->col, L->mL.p, L->mD.p,
                       L->cgP.p, L->cgGP.p, L->cgSP.p, L->nNo, L->red.part.p, L->red.ticket.p, C.sc(kSlotDen));
                break;
            case 2: C.spmv_sv3(L->mG.p, L->cgP.p, L->cgGP.p); break;
            default:
                launch(k_mgs, red_grid(n3), 256, 0, s, L->basis.p + 2 * n3, L->basis.p, C.sc(kSlotH),
                       L->basis.p + n3, n3, L->red.part.p, L->red.ticket.p, C.sc(kSlotH + 1));
        }
    };
    for (int i = 0; i < 2; ++i) run();
    CR_CUDA(cudaEventRecord(e0, s));
    for (int i = 0; i < reps; ++i) run();
    CR_CUDA(cudaEventRecord(e1, s));
    CR_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    CR_CUDA(cudaEventElapsedTime(&t, e0, e1));
    *ms = (double)t / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CR_CUDA(cudaGetLastError());
    return CRIMSON_OK;
}

}  // namespace crimson
