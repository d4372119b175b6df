"""The oracle's memLS NS solve against an independent sparse direct solve.

Pins the oracle's NSSOLVER (flowsolver/src/memLS.f90:1460-1759) to the system
it is meant to solve: SuperLU on the assembled operator
[K + faceRes v v^T, G; D, L] restricted to the unconstrained dofs.  memLS
stops at an estimated relative residual of epstol_ns = 1e-5, so the solutions
agree to the conditioning times that (measured 1.7e-7 on this mesh); the
bound used is 1e-5.
"""
import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, RCR, mesh
from oracle import pyoracle as po
from tests.conftest import relerr
from tests.linsys import defect, direct_solve, first_system


@pytest.fixture(scope="module")
def system():
    m = mesh.cylinder(ncross=8, naxial=10)
    m.set_inflow(10.0)
    P = FlowParams(rcr=[RCR(srfid=3)])
    colm, rowp = po.genadj(m.ien, m.nshg)
    F, Res4, Val4, faceRes, _, _ = first_system(m, P, colm, rowp)
    xd, A, f = direct_solve(m, colm, rowp, Res4, Val4, faceRes)
    return m, P, F, Res4, Val4, faceRes, xd, A, f


def test_direct_solve_is_exact(system):
    m, P, F, Res4, Val4, faceRes, xd, A, f = system
    assert defect(A, f, xd, Res4) < 1e-10


def test_oracle_memls_matches_direct(system):
    m, P, F, Res4, Val4, faceRes, xd, A, f = system
    osol, ost = F.memls.solve(Res4, Val4.copy(), faceRes)
    assert ost.RI.suc == 1
    assert relerr(osol, xd) < 1e-5, relerr(osol, xd)
    assert defect(A, f, osol, Res4) < 1e-4
    # constrained dofs come back exactly zero
    assert np.all(osol.ravel()[~f] == 0.0)
