"""CPU: the oracle's ElmGMRSclr (flowsolver/src/elmgmr.f90:599-822) against
properties of the discrete advection-diffusion operator that hold whatever
the summation order:

* patch test: with zero velocity and a linear scalar field, the projected
  flux is diffus * grad S at every node and the residual (interior terms
  plus the consistent boundary flux of e3bSclr) vanishes;
* with zero velocity the tangent is the symmetric mass + stiffness matrix;
* without the flux projection (idiff = 0) the residual is affine in (S, Sdot)
  and its change along (alfi gami Delt d, almi d) -- an increment d of the
  scalar's rate -- is -lhsS d on interior rows.  e3LHSSclr
  (e3lhs.f90:452-475) leaves almi off the SUPG mass term, so the identity is
  exact for zero velocity or almi = 1 (rhoinf = 1/3) and off by that term
  otherwise;
* the Dirichlet bit isclr + 5 zeroes its rows; the flux bit 4 + isclr swaps
  the consistent flux for the prescribed one.
"""
import copy

import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, mesh
from oracle import pyoracle as po


@pytest.fixture(scope="module")
def cyl():
    m = mesh.cylinder(ncross=6, naxial=6)
    m.set_inflow(10.0)
    colm, rowp = po.genadj(m.ien, m.nshg)
    return m, colm, rowp


def _dense(colm, rowp, v, n):
    A = np.zeros((n, n))
    for i in range(n):
        for k in range(colm[i] - 1, colm[i + 1] - 1):
            A[i, rowp[k] - 1] = v[k]
    return A


def test_patch_linear_scalar(cyl):
    m, colm, rowp = cyl
    elm = po.Elm(m, FlowParams(idiff=1), colm, rowp)
    g = np.array([0.3, -1.2, 0.7])
    s = m.x @ g + 2.0
    y = np.zeros((m.nshg, 4))
    out = po.elmgmr_sclr(elm, y, s, np.zeros(m.nshg), isclr=1, diffus=0.25)
    assert np.abs(out["qres"] - 0.25 * g).max() < 1e-12
    assert np.abs(out["res"]).max() < 1e-11


def test_zero_velocity_tangent_symmetric(cyl):
    m, colm, rowp = cyl
    elm = po.Elm(m, FlowParams(), colm, rowp)
    rng = np.random.default_rng(3)
    out = po.elmgmr_sclr(elm, np.zeros((m.nshg, 4)), rng.standard_normal(m.nshg), rng.standard_normal(m.nshg),
                         diffus=0.1)
    A = _dense(colm, rowp, out["lhsS"], m.nshg)
    assert np.abs(A - A.T).max() <= 1e-13 * np.abs(A).max()
    assert np.all(np.linalg.eigvalsh(0.5 * (A + A.T)) > 0)


@pytest.mark.parametrize("rhoinf,moving", [(0.0, False), (1.0 / 3.0, True), (0.0, True)])
def test_affine_in_scalar_without_projection(cyl, rhoinf, moving):
    m, colm, rowp = cyl
    P = FlowParams(idiff=0, rhoinf=rhoinf)
    elm = po.Elm(m, P, colm, rowp)
    rng = np.random.default_rng(4)
    y = rng.standard_normal((m.nshg, 4)) * (1.0 if moving else 0.0)
    s, sd, d = (rng.standard_normal(m.nshg) for _ in range(3))
    a = P.alfi * P.gami * P.Delt
    r0 = po.elmgmr_sclr(elm, y, s, sd, diffus=0.05)
    r1 = po.elmgmr_sclr(elm, y, s + a * d, sd + P.almi * d, diffus=0.05, lhs=False)
    A = _dense(colm, rowp, r0["lhsS"], m.nshg)
    interior = np.ones(m.nshg, bool)
    interior[np.unique(m.ienb[:, :3])] = False
    assert interior.sum() > 10
    lhs_d = (A @ d)[interior]
    err = np.abs((r1["res"] - r0["res"])[interior] + lhs_d).max() / np.abs(lhs_d).max()
    if moving and abs(P.almi - 1.0) > 1e-12:
        assert err > 1e-6   # the SUPG mass term without almi
    else:
        assert err <= 1e-11


def test_dirichlet_and_flux_bits(cyl):
    m0, colm, rowp = cyl
    m = copy.copy(m0)
    isclr = 2
    m.iBC = m0.iBC.copy()
    inlet = np.unique(m.ienb[m.iBCB[:, 1] == 1, :3])
    m.iBC[inlet] |= 1 << (isclr + 5)
    m.iBCB = m0.iBCB.copy()
    flux_faces = np.nonzero(m.iBCB[:, 1] >= 3)[0]
    m.iBCB[flux_faces, 0] |= 1 << (4 + isclr)
    rng = np.random.default_rng(5)
    y = rng.standard_normal((m.nshg, 4))
    s, sd = rng.standard_normal(m.nshg), rng.standard_normal(m.nshg)
    bcbs = np.zeros((m.ienb.shape[0], 3))
    bcbs[flux_faces] = rng.standard_normal((flux_faces.size, 3))
    ref = po.elmgmr_sclr(po.Elm(m0, FlowParams(), colm, rowp), y, s, sd, isclr=isclr, diffus=0.1)
    out = po.elmgmr_sclr(po.Elm(m, FlowParams(), colm, rowp), y, s, sd, isclr=isclr, diffus=0.1, bcbs=bcbs)
    assert np.all(out["res"][inlet] == 0.0)
    assert np.array_equal(out["lhsS"], ref["lhsS"])
    # the prescribed flux only moves rows of the flux faces' nodes
    free = np.ones(m.nshg, bool)
    free[inlet] = False
    moved = np.nonzero((out["res"] != ref["res"]) & free)[0]
    assert moved.size and set(moved) <= set(np.unique(m.ienb[flux_faces, :3]))
    # a zero prescribed flux leaves exactly the interior terms
    out0 = po.elmgmr_sclr(po.Elm(m, FlowParams(), colm, rowp), y, s, sd, isclr=isclr, diffus=0.1,
                          bcbs=np.zeros_like(bcbs))
    assert np.abs(out["res"] - out0["res"]).max() > 0


def test_unsupported_settings(cyl):
    m, colm, rowp = cyl
    with pytest.raises(RuntimeError):
        po.elmgmr_sclr(po.Elm(m, FlowParams(idiff=2), colm, rowp), np.zeros((m.nshg, 4)), np.zeros(m.nshg),
                       np.zeros(m.nshg))
    with pytest.raises(RuntimeError):
        po.elmgmr_sclr(po.Elm(m, FlowParams(), colm, rowp), np.zeros((m.nshg, 4)), np.zeros(m.nshg),
                       np.zeros(m.nshg), isclr=0)
