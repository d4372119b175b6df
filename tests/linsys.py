"""Shared test helper: the first Newton system of a small cylinder and an
independent sparse direct solve of it (scipy SuperLU, FP64).

The system is what SolFlow hands memLS (flowsolver/src/solfar.f90:210-264):
Res4 / Val4 packed from ElmGMR's res, lhsK, lhsP, a Dirichlet face from iBC
and one coupled (resistance) outlet face whose faceRes adds
faceRes * v v^T (v = NABI of the face nodes) to the momentum block
(ADDBCMUL, flowsolver/src/memLS.f90:206-268).  Constrained dofs (val 0 on
the Dirichlet face) have solution 0, as memLS's W scaling gives them.
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from crimsonflowsolver_b200 import solver
from oracle import pyoracle as po


def first_system(m, P, colm, rowp, srfid=3):
    F = po.OracleFlow(m, P)
    F.y = F.yold.copy()
    F.ac = F.acold * ((P.gami - 1) / P.gami)
    F._itr_bc(F.y)
    c1, c2 = F.implicit_coeffs(0)
    yA = F.y.copy()
    acA = F.ac.copy()
    acA[:, 3] = 0
    out = F.elm(yA, acA, srflist=[srfid], coef1=c1, coef2=c2)
    Res4, Val4 = po.solflow_pack(m.nshg, colm, rowp, out["res"], out["lhsK"], out["lhsP"])
    faceRes = np.array([0.0, c1[0]]) * P.alfi * P.gami * P.Delt
    return F, Res4, Val4, faceRes, out, (yA, acA, c1, c2)


def assembled_matrix(m, colm, rowp, Val4, faceRes, srfid=3):
    """The unscaled 4 nshg x 4 nshg operator memLS applies (node-major dofs)."""
    n = m.nshg
    A = sp.bsr_matrix((Val4.reshape(-1, 4, 4), rowp - 1, colm - 1), shape=(4 * n, 4 * n)).tocsr()
    nodes, v = solver.neumann_face(m, srfid)
    idx = (4 * nodes[:, None] + np.arange(3)[None, :]).ravel()
    vv = v.ravel()
    cpl = sp.csr_matrix((np.outer(vv, vv).ravel() * faceRes[1],
                         (np.repeat(idx, idx.size), np.tile(idx, idx.size))), shape=(4 * n, 4 * n))
    return (A + cpl).tocsr()


def free_dofs(m):
    nodes, sv = solver.dirichlet_face(m)
    mask = np.ones((m.nshg, 4), dtype=bool)
    mask[nodes, 0:3] = sv != 0
    return mask.ravel()


def direct_solve(m, colm, rowp, Res4, Val4, faceRes, srfid=3):
    A = assembled_matrix(m, colm, rowp, Val4, faceRes, srfid)
    f = free_dofs(m)
    x = np.zeros(4 * m.nshg)
    x[f] = spla.spsolve(A[f][:, f].tocsc(), Res4.ravel()[f])
    return x.reshape(m.nshg, 4), A, f


def defect(A, f, x, Res4):
    """|R - A x| / |R| over the free dofs (2-norms)."""
    r = Res4.ravel()[f] - (A[f][:, f] @ x.ravel()[f])
    return float(np.linalg.norm(r) / np.linalg.norm(Res4.ravel()[f]))
