"""Discrete adjoint of the time stepping (no counterpart in the reference).

Objective (the multi-outlet cylinder workload): the squared misfit of the
time-averaged outlet pressures,

    J(theta) = sum_k ( (1/N) sum_{n=1..N} P_k(t_n) - T_k )^2,

with theta = (mu, Rp_1, C_1, Rd_1, ..., Rp_m, C_m, Rd_m).  The gradient is
the exact discrete adjoint of the converged time steps that
``crimson_step`` computes (itrdrv_iter_step, flowsolver/src/itrdrv.f90:1239,
with RCR outlets, flowsolver/src/RCR.cxx:49-81):

* per step the unknowns are x = (a_{n+1} on the free velocity dofs, p_{n+1})
  with y = y_n + gamma dt a - (gamma - 1) dt a_n, and the equations are
  res(y_alpha, a_alpha; mu, c1, c2) = 0 on the free rows (res is what ElmGMR
  assembles; c1, c2 the RCR implicit coefficients from P_n, Q_n);
* the adjoint solve J^T lambda = xbar is flexible GMRES on the exact
  transposed Jacobian product ``crimson_elmgmr_vjp``, right-preconditioned
  by the transposed memLS solve with the assembled (approximate) tangent,
  ``crimson_solflow_device_transposed`` (-A^-T ~ J^-T: A ~ -J, as the
  forward Newton step uses it);
* the RCR update P_{n+1} = d1 Q_{n+1} + h1(P_n, Q_n) and the coupling
  coefficients are differentiated by hand (``rcr_coeffs``).

Multi-step gradients use timestep checkpointing: the forward pass keeps the
state every ``checkpoint_every`` steps; the reverse pass recomputes each
segment from its checkpoint, then runs the adjoint steps of the segment
backwards.  ``CrimsonObjective`` wraps J and its gradient as a
``torch.autograd.Function``.  All accumulation is FP64.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, replace
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _native as N
from .problem import RCR, FlowParams
from .solver import FlowSolver


# ---------------------------------------------------------------------------
# RCR implicit coefficients and their partial derivatives
# ---------------------------------------------------------------------------
def rcr_coeffs(Rp: float, C: float, Rd: float, Pd: float, Pn: float, Qn: float, tau: float):
    """(slope, offset) of P = slope Q + offset, RCR::computeImplicitCoefficients
    (flowsolver/src/RCR.cxx:49-81) with a constant distal pressure Pd, and
    their partials: d slope / d(Rp, C, Rd), d offset / d(Rp, C, Rd, Pn, Qn)."""
    a = C * Rd / tau
    den = 1.0 + a
    slope = (Rd + Rp * den) / den
    T2 = Pn - Rp * Qn
    offset = (a * T2 + Pd) / den
    ds = np.array([1.0, -(Rd * Rd / tau) / den ** 2, 1.0 / den ** 2])          # Rp, C, Rd
    dof_da = (T2 - Pd) / den ** 2
    do = np.array([-Qn * a / den, dof_da * Rd / tau, dof_da * C / tau])         # Rp, C, Rd
    do_P = a / den
    do_Q = -Rp * a / den
    return slope, offset, ds, do, do_P, do_Q


@dataclass
class Record:
    """One time step as the reverse pass needs it (host arrays, node-major)."""
    y0: np.ndarray   # y_n   (nshg, 4) before the step
    a0: np.ndarray   # a_n
    P0: np.ndarray   # P_n   per outlet
    Q0: np.ndarray
    y1: np.ndarray   # y_{n+1} after the step
    a1: np.ndarray
    P1: np.ndarray
    Q1: np.ndarray


class AdjointProblem:
    """Objective and gradient of the outlet-pressure misfit over ``nsteps``."""

    def __init__(self, mesh, P: FlowParams, targets: Sequence[float], nsteps: int,
                 inflow: Optional[Callable[[float], float]] = None, checkpoint_every: int = 10,
                 adj_tol: float = 1e-10, adj_maxit: int = 40):
        if not P.rcr:
            raise ValueError("the objective needs at least one RCR outlet")
        if P.netlists:
            raise ValueError("netlist outlets are not differentiated (RCR outlets only)")
        self.mesh = mesh
        self.P0 = P
        self.targets = np.asarray(targets, dtype=np.float64)
        self.nc = len(P.rcr)
        if self.targets.shape != (self.nc,):
            raise ValueError("one target pressure per RCR outlet")
        self.nsteps = int(nsteps)
        self.inflow = inflow if inflow is not None else (lambda t: 10.0)
        self.ce = max(1, int(checkpoint_every))
        self.adj_tol = adj_tol
        self.adj_maxit = adj_maxit
        self.last_stats = {}

    # ---- parameters ----
    def theta0(self) -> np.ndarray:
        th = [self.P0.mu]
        for r in self.P0.rcr:
            th += [r.Rp, r.C, r.Rd]
        return np.asarray(th, dtype=np.float64)

    def params(self, theta) -> FlowParams:
        th = np.asarray(theta, dtype=np.float64)
        rcr = [RCR(srfid=r.srfid, Rp=float(th[1 + 3 * k]), C=float(th[2 + 3 * k]), Rd=float(th[3 + 3 * k]), Pd=r.Pd)
               for k, r in enumerate(self.P0.rcr)]
        return replace(self.P0, mu=float(th[0]), rcr=rcr)

    # ---- forward ----
    def _rcr_get(self, F: FlowSolver):
        P = np.zeros(self.nc)
        Q = np.zeros(self.nc)
        N.check(N.lib().crimson_rcr_state(F.elm.h, self.nc, N.dp(P), N.dp(Q), 0), "crimson_rcr_state")
        return P, Q

    def _rcr_set(self, F: FlowSolver, P, Q):
        P = np.ascontiguousarray(P, dtype=np.float64)
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        N.check(N.lib().crimson_rcr_state(F.elm.h, self.nc, N.dp(P), N.dp(Q), 1), "crimson_rcr_state")

    def _objective(self, Ps: np.ndarray) -> float:
        return float(np.sum((Ps.mean(axis=0) - self.targets) ** 2))

    def objective(self, theta) -> float:
        """J(theta): one forward run (no checkpoints kept)."""
        F = FlowSolver(self.mesh, self.params(theta), inflow=self.inflow)
        try:
            Ps = np.zeros((self.nsteps, self.nc))
            for n in range(self.nsteps):
                st = F.step()
                Ps[n] = st.p_out[:self.nc]
            return self._objective(Ps)
        finally:
            F.close()

    # ---- gradient ----
    def gradient(self, theta):
        """(J, dJ/dtheta) by the checkpointed discrete adjoint."""
        import torch

        Pp = self.params(theta)
        F = FlowSolver(self.mesh, Pp, inflow=self.inflow)
        try:
            # forward pass: checkpoints and the outlet pressures
            ckpt = {}
            Ps = np.zeros((self.nsteps, self.nc))
            for n in range(self.nsteps):
                if n % self.ce == 0:
                    y, a = F.state()
                    Pn, Qn = self._rcr_get(F)
                    ckpt[n] = (y, a, Pn, Qn)
                st = F.step()
                Ps[n] = st.p_out[:self.nc]
            J = self._objective(Ps)
            Pbar_obj = 2.0 * (Ps.mean(axis=0) - self.targets) / self.nsteps
            ctx = _AdjointContext(F, Pp, torch)
            yb = torch.zeros((self.mesh.nshg, 4), dtype=torch.float64, device="cuda")
            ab = torch.zeros_like(yb)
            Pb = np.zeros(self.nc)
            Qb = np.zeros(self.nc)
            thb = np.zeros(1 + 3 * self.nc)
            iters = []
            for s in sorted(ckpt.keys(), reverse=True):
                e = min(s + self.ce, self.nsteps)
                y, a, Pn, Qn = ckpt[s]
                F.set_state(y, a)
                self._rcr_set(F, Pn, Qn)
                F.istep = s
                recs: List[Record] = []
                for n in range(s, e):
                    y0, a0 = F.state()
                    P0, Q0 = self._rcr_get(F)
                    F.step()
                    y1, a1 = F.state()
                    P1, Q1 = self._rcr_get(F)
                    recs.append(Record(y0, a0, P0, Q0, y1, a1, P1, Q1))
                for rec in reversed(recs):
                    Pb = Pb + Pbar_obj
                    yb, ab, Pb, Qb, it = ctx.step_back(rec, yb, ab, Pb, Qb, thb, self.adj_tol, self.adj_maxit)
                    iters.append(it)
            self.last_stats = {"adjoint_iterations": iters}
            return J, thb
        finally:
            F.close()


class _AdjointContext:
    """Per-problem device buffers and the adjoint of one time step."""

    def __init__(self, F: FlowSolver, P: FlowParams, torch):
        self.F = F
        self.P = P
        self.t = torch
        m = F.mesh
        n = m.nshg
        dev = "cuda"
        self.n = n
        self.nnz = F.elm._nnz()
        self.lhsK = torch.empty((self.nnz, 9), dtype=torch.float64, device=dev)
        self.lhsP = torch.empty((self.nnz, 4), dtype=torch.float64, device=dev)
        self.res = torch.empty((n, 4), dtype=torch.float64, device=dev)
        self.ybar = torch.empty((n, 4), dtype=torch.float64, device=dev)
        self.abar = torch.empty((n, 4), dtype=torch.float64, device=dev)
        self.sol = torch.empty((n, 4), dtype=torch.float64, device=dev)
        iBC = np.asarray(m.iBC)
        vel_fixed = (((iBC >> 3) & 7) == 7) | (((iBC >> 11) & 1) == 1)
        p_fixed = ((iBC >> 2) & 1) == 1
        free = np.ones((n, 4), dtype=bool)
        free[vel_fixed, 0:3] = False
        free[p_fixed, 3] = False
        self.free = torch.tensor(free, device=dev)
        self.dirv = torch.tensor(np.repeat(vel_fixed[:, None], 3, axis=1), device=dev)
        # outlet node groups in srflist order (Q_k = sum NABI . u over ndsurf == srfid)
        self.onodes = []
        self.onabi = []
        for r in P.rcr:
            nodes = np.nonzero(m.ndsurf == r.srfid)[0]
            self.onodes.append(torch.tensor(nodes, device=dev))
            self.onabi.append(torch.tensor(m.NABI[nodes], dtype=torch.float64, device=dev))
        self.af, self.am, self.g, self.dt = P.alfi, P.almi, P.gami, P.Delt
        self.cp = P.gami * P.alfi * P.Delt
        self.incL = np.ones(1 + len(P.rcr), dtype=np.int32)

    def _vjp(self, ya, aa, c1, c2, lam):
        mub = ctypes.c_double()
        nc = len(c1)
        c1b = np.zeros(max(nc, 1))
        c2b = np.zeros(max(nc, 1))
        c1a = np.ascontiguousarray(c1, dtype=np.float64)
        c2a = np.ascontiguousarray(c2, dtype=np.float64)
        self.t.cuda.synchronize()
        N.check(N.lib().crimson_elmgmr_vjp(self.F.elm.h, ya.data_ptr(), aa.data_ptr(), N.dp(c1a), N.dp(c2a),
                                           lam.data_ptr(), self.res.data_ptr(), self.ybar.data_ptr(),
                                           self.abar.data_ptr(), ctypes.byref(mub), N.dp(c1b), N.dp(c2b)),
                "crimson_elmgmr_vjp")
        self.t.cuda.synchronize()
        return mub.value, c1b[:nc].copy(), c2b[:nc].copy()

    def _jt(self, ya, aa, c1, c2, lam):
        """J~^T lambda on x~ = (a on free velocity dofs, p / cp), plus the VJP outputs."""
        mub, c1b, c2b = self._vjp(ya, aa, c1, c2, lam)
        jt = self.t.empty_like(lam)
        jt[:, 0:3] = self.af * self.g * self.dt * self.ybar[:, 0:3] + self.am * self.abar[:, 0:3]
        jt[:, 3] = self.cp * self.ybar[:, 3]
        jt = self.t.where(self.free, jt, self.t.zeros_like(jt))
        return jt, mub, c1b, c2b

    def _solve_t(self, rhs, faceRes):
        """A^-T rhs.  The right side is scaled to unit norm first: memLS's
        Krylov absolute tolerances and GE's absolute pivot test assume
        right sides of the size of a residual, and the adjoint's corrections
        shrink by orders of magnitude."""
        nr = float(self.t.linalg.norm(rhs))
        if nr == 0.0:
            return self.t.zeros_like(rhs)
        st = N.LsStats()
        fr = np.ascontiguousarray(faceRes, dtype=np.float64)
        scaled = (rhs / nr).contiguous()
        self.t.cuda.synchronize()
        N.check(N.lib().crimson_solflow_device_transposed(self.F.elm.h, self.F.memls.lhs, self.F.memls.ls,
                                                          scaled.data_ptr(), self.lhsK.data_ptr(),
                                                          self.lhsP.data_ptr(), N.ip(self.incL), N.dp(fr),
                                                          self.sol.data_ptr(), ctypes.byref(st)),
                "crimson_solflow_device_transposed")
        self.t.cuda.synchronize()
        return self.sol * nr

    def step_back(self, rec: Record, yb, ab, Pb, Qb, thb, tol, maxit):
        """Cotangents of S_{n+1} -> cotangents of S_n; adds dJ/dtheta terms to thb."""
        t = self.t
        P = self.P
        dev = "cuda"
        nc = len(P.rcr)
        af, am, g, dt, cp = self.af, self.am, self.g, self.dt, self.cp
        Pb = np.array(Pb, dtype=np.float64)
        Qb = np.array(Qb, dtype=np.float64)
        Pb_prev = np.zeros(nc)
        Qb_prev = np.zeros(nc)
        # 1. RCR history update P_{n+1} = d1 Q_{n+1} + h1(P_n, Q_n), tau = dt
        for k, r in enumerate(P.rcr):
            d1, h1, ds, do, doP, doQ = rcr_coeffs(r.Rp, r.C, r.Rd, r.Pd, rec.P0[k], rec.Q0[k], dt)
            Qb[k] += d1 * Pb[k]
            Pb_prev[k] += doP * Pb[k]
            Qb_prev[k] += doQ * Pb[k]
            thb[1 + 3 * k:4 + 3 * k] += (ds * rec.Q1[k] + do) * Pb[k]
        # 2. Q_{n+1} = sum NABI . u_{n+1}
        yb = yb.clone()
        for k in range(nc):
            yb[self.onodes[k], 0:3] += self.onabi[k] * Qb[k]
        # 3. explicit relations of the update
        free_v = self.free[:, 0:3]
        yb_prev = t.zeros_like(yb)
        ab_prev = t.zeros_like(ab)
        yb_prev[:, 0:3] = t.where(free_v, yb[:, 0:3], t.zeros_like(yb[:, 0:3]))
        ab_prev[:, 0:3] = t.where(free_v, -(g - 1.0) * dt * yb[:, 0:3], ((g - 1.0) / g) * ab[:, 0:3])
        xbar = t.zeros_like(yb)
        xbar[:, 0:3] = ab[:, 0:3] + g * dt * yb[:, 0:3]
        xbar[:, 3] = cp * yb[:, 3]
        xbar = t.where(self.free, xbar, t.zeros_like(xbar))
        # 4. the converged step's alpha-level state and coupling coefficients
        y0 = t.tensor(rec.y0, device=dev)
        a0 = t.tensor(rec.a0, device=dev)
        y1 = t.tensor(rec.y1, device=dev)
        a1 = t.tensor(rec.a1, device=dev)
        ya = y1.clone()
        ya[:, 0:3] = y0[:, 0:3] + af * (y1[:, 0:3] - y0[:, 0:3])
        aa = t.zeros_like(a1)
        aa[:, 0:3] = a0[:, 0:3] + am * (a1[:, 0:3] - a0[:, 0:3])
        c1 = np.zeros(nc)
        c2 = np.zeros(nc)
        dc = []
        for k, r in enumerate(P.rcr):
            c1[k], c2[k], ds, do, doP, doQ = rcr_coeffs(r.Rp, r.C, r.Rd, r.Pd, rec.P0[k], rec.Q0[k], af * dt)
            dc.append((ds, do, doP, doQ))
        faceRes = np.concatenate([[0.0], c1 * af * g * dt])
        # assembled tangent at the converged state (the preconditioner)
        self.F.elm.device(ya, aa, self.res, self.lhsK, self.lhsP, list(c1), list(c2), lhs=True)
        t.cuda.synchronize()
        # 5. J~^T lambda = xbar: flexible GMRES on the exact J~^T, right
        #    preconditioned by the transposed memLS solve (-A^-T ~ J~^-T)
        bn = float(t.linalg.norm(xbar))
        its = 0
        if bn > 0.0:
            lam, its = _fgmres(lambda v: self._jt(ya, aa, c1, c2, v)[0], lambda v: -self._solve_t(v, faceRes),
                               xbar, tol, maxit, t)
            jt, mub, c1b, c2b = self._jt(ya, aa, c1, c2, lam)
            # 6. z_bar -= (d G / d z)^T lambda
            yba = self.ybar
            aba = self.abar
            yb_prev[:, 0:3] -= t.where(free_v, yba[:, 0:3], (1.0 - af) * yba[:, 0:3])
            ab_prev[:, 0:3] -= t.where(free_v, -af * (g - 1.0) * dt * yba[:, 0:3] + (1.0 - am) * aba[:, 0:3],
                                       (1.0 - am / g) * aba[:, 0:3])
            thb[0] -= mub
            for k in range(nc):
                ds, do, doP, doQ = dc[k]
                c1bar = -c1b[k]
                c2bar = -c2b[k]
                thb[1 + 3 * k:4 + 3 * k] += c1bar * ds + c2bar * do
                Pb_prev[k] += c2bar * doP
                Qb_prev[k] += c2bar * doQ
        return yb_prev, ab_prev, Pb_prev, Qb_prev, its


def _fgmres(apply_a, apply_m, b, tol, maxit, t):
    """Flexible GMRES (right preconditioning that may change per step: the
    preconditioner is itself an iterative solve) for a(x) = b, from x = 0.
    Orthogonalisation by modified Gram-Schmidt; the small least-squares
    problem is solved on the host in FP64.  Restarts every 30 steps; stops at
    |b - a(x)| <= tol |b| or after maxit steps.  Returns (x, steps)."""
    bn = float(t.linalg.norm(b))
    x = t.zeros_like(b)
    steps = 0
    restart = 30
    r = b.clone()
    while steps < maxit:
        beta = float(t.linalg.norm(r))
        if beta <= tol * bn:
            break
        V = [r / beta]
        Z = []
        m = min(restart, maxit - steps)
        H = np.zeros((m + 1, m))
        y = None
        for j in range(m):
            z = apply_m(V[j])
            Z.append(z)
            w = apply_a(z)
            for i in range(j + 1):
                H[i, j] = float((w * V[i]).sum())
                w = w - H[i, j] * V[i]
            H[j + 1, j] = float(t.linalg.norm(w))
            steps += 1
            e1 = np.zeros(j + 2)
            e1[0] = beta
            y, *_ = np.linalg.lstsq(H[:j + 2, :j + 1], e1, rcond=None)
            res = float(np.linalg.norm(e1 - H[:j + 2, :j + 1] @ y))
            if res <= tol * bn or H[j + 1, j] == 0.0:
                break
            V.append(w / H[j + 1, j])
        for i in range(len(y)):
            x = x + float(y[i]) * Z[i]
        r = b - apply_a(x)
    return x, steps


def make_objective_function():
    """``CrimsonObjective``: J(theta) as a torch.autograd.Function whose
    backward runs the checkpointed adjoint."""
    import torch

    class CrimsonObjective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, problem: AdjointProblem):
            th = theta.detach().cpu().numpy().astype(np.float64)
            J, g = problem.gradient(th)
            ctx.save_for_backward(torch.tensor(g, dtype=theta.dtype, device=theta.device))
            return torch.tensor(J, dtype=theta.dtype, device=theta.device)

        @staticmethod
        def backward(ctx, gJ):
            (g,) = ctx.saved_tensors
            return gJ * g, None

    return CrimsonObjective
