"""Self-checks of the oracle that need no reference output (CPU).

* A uniform velocity with zero pressure and acceleration is an exact
  solution of the discrete interior equations: every residual row of a node
  that touches no boundary face vanishes (convective and viscous terms are
  zero, and the patch sum of grad N_a is zero for interior nodes).
* Continuity row sum: sum_a grad N_a = 0 on every tet, so the continuity
  residual summed over all nodes is minus the boundary flux of the boundary
  residual term, sum over the boundary faces of int u.n (rigid wall and
  natural-pressure faces carry u.n, here computed independently).
* The PSPG block C (lhsP(4, :)) is symmetric, block (i,j) = block (j,i)
  (flowsolver/src/e3.f90:163-169 symmetrises it per element).
* RCR implicit coefficients (flowsolver/src/RCR.cxx:49-81) reproduce an
  implicit-Euler integration of the Windkessel C dPc/dt = Q - (Pc - Pd)/Rd,
  P = Rp Q + Pc, for a prescribed flow.
"""
import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, RCR, mesh
from oracle import pyoracle as po


@pytest.fixture(scope="module")
def cyl():
    m = mesh.cylinder(ncross=8, naxial=8)
    P = FlowParams(rcr=[RCR(srfid=3)])
    colm, rowp = po.genadj(m.ien, m.nshg)
    return m, P, colm, rowp


def test_uniform_flow_interior_residual_vanishes(cyl):
    m, P, colm, rowp = cyl
    y = np.zeros((m.nshg, 4))
    y[:, 0:3] = [3.0, -2.0, 12.0]
    ac = np.zeros((m.nshg, 4))
    out = po.Elm(m, P, colm, rowp)(y, ac, srflist=[3], coef1=[0.0], coef2=[0.0], lhs=False)
    res = np.asarray(out["res"])
    interior = np.ones(m.nshg, dtype=bool)
    interior[np.unique(m.ienb[:, :3])] = False
    # scale: the residual of a sheared field on the same mesh
    y2 = y.copy()
    y2[:, 2] += 5.0 * m.x[:, 0]
    r2 = np.asarray(po.Elm(m, P, colm, rowp)(y2, ac, srflist=[3], coef1=[0.0], coef2=[0.0], lhs=False)["res"])
    scale = np.abs(r2[interior]).max()
    assert interior.sum() > 50
    assert np.abs(res[interior]).max() <= 1e-12 * scale


def test_continuity_row_sum_is_boundary_flux(cyl):
    m, P, colm, rowp = cyl
    rng = np.random.default_rng(5)
    y = rng.standard_normal((m.nshg, 4))
    ac = rng.standard_normal((m.nshg, 4))
    iBC0 = m.iBC.copy()
    m.iBC[:] = 0        # no bc3Res zeroing: every row counts
    try:
        out = po.Elm(m, P, colm, rowp)(y, ac, srflist=[3], coef1=[0.0], coef2=[0.0], lhs=False)
    finally:
        m.iBC[:] = iBC0
    res = np.asarray(out["res"])
    # boundary term of e3b: rl(n, 4) -= N_n unm WdetJb, unm = u.n at the face
    # points (3-point rule, weights 1/3 x area) for every face of the mesh
    x = m.x
    fb = m.ienb
    v1 = x[fb[:, 1]] - x[fb[:, 0]]
    v2 = x[fb[:, 2]] - x[fb[:, 0]]
    cr = np.cross(v1, v2)
    area = 0.5 * np.linalg.norm(cr, axis=1)
    nrm = cr / np.linalg.norm(cr, axis=1)[:, None]
    B, C = 0.666666666666667, 0.166666666666667
    pts = [(B, C, C), (C, B, C), (C, C, B)]
    flux = 0.0
    for wts in pts:
        u = sum(w * y[fb[:, k], 0:3] for k, w in enumerate(wts))
        flux += np.sum(area / 3.0 * np.einsum("ij,ij->i", u, nrm))
    total = res[:, 3].sum()
    assert abs(total + flux) <= 1e-9 * np.abs(res[:, 3]).sum()


def test_pspg_block_symmetric(cyl):
    m, P, colm, rowp = cyl
    rng = np.random.default_rng(6)
    y = rng.standard_normal((m.nshg, 4))
    ac = rng.standard_normal((m.nshg, 4))
    out = po.Elm(m, P, colm, rowp)(y, ac, srflist=[3], coef1=[50.0], coef2=[1.0])
    C = np.asarray(out["lhsP"])[:, 3]
    rows = np.repeat(np.arange(m.nshg), np.diff(colm))
    cols = rowp - 1
    pos = {(r, c): k for k, (r, c) in enumerate(zip(rows.tolist(), cols.tolist()))}
    tr = np.array([pos[(c, r)] for r, c in zip(rows.tolist(), cols.tolist())])
    assert np.abs(C - C[tr]).max() <= 1e-13 * np.abs(C).max()


def test_rcr_coefficients_match_implicit_euler_windkessel():
    Rp, Cc, Rd, Pd, tau = 100.0, 1e-4, 1000.0, 5.0, 1e-3
    n = 400
    Q = 10.0 + 5.0 * np.sin(2 * np.pi * np.arange(1, n + 1) * tau / 0.8)
    # direct implicit Euler on the capacitor pressure
    Pc = 0.0
    P_direct = np.zeros(n)
    for k in range(n):
        Pc = (Pc + tau / Cc * Q[k] + tau * Pd / (Cc * Rd)) / (1.0 + tau / (Cc * Rd))
        P_direct[k] = Rp * Q[k] + Pc
    # the coefficient recursion P_{n+1} = slope Q_{n+1} + offset(P_n, Q_n)
    Pn, Qn = 0.0, 0.0   # Pc_0 = 0 <=> P_0 = Rp Q_0 with Q_0 = 0
    P_coef = np.zeros(n)
    for k in range(n):
        s, o = po.rcr_coeffs(Rp, Cc, Rd, Pd, Pd, Pn, Qn, tau)
        Pn, Qn = s * Q[k] + o, Q[k]
        P_coef[k] = Pn
    assert np.abs(P_coef - P_direct).max() <= 1e-10 * np.abs(P_direct).max()
