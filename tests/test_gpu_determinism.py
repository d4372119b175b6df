"""Determinism of the GPU path.

ElmGMR's scatter is owner-computes: every residual row and CSR block is
summed by one thread over its contribution list in ascending element order
(the reference's serial order, local.f90:64-75, fillsparse.f90:47-60), and
every memLS reduction sums its per-block partials in block order.  So the
same inputs give the same bits: on one context called twice, on two
contexts, and through whole time steps of two solvers.
"""
import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, RCR, mesh, solver

pytestmark = pytest.mark.gpu


def _same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b))


def test_elmgmr_bitwise_repeatable():
    from tests.fixtures import basic_mesh

    m, y, ac = basic_mesh()
    rng = np.random.default_rng(3)
    y[:, 0:3] = 10.0 * rng.standard_normal((m.nshg, 3))
    srf = m.outlets
    P = FlowParams(rcr=[RCR(srfid=s) for s in srf])
    c1 = [110.0 + 5 * k for k in range(len(srf))]
    c2 = [-3.0 + k for k in range(len(srf))]
    with solver.ElmGMR(m, P) as e1, solver.ElmGMR(m, P) as e2:
        a = e1(y, ac, c1, c2)
        b = e1(y, ac, c1, c2)
        c = e2(y, ac, c1, c2)
    for k in ("res", "lhsK", "lhsP"):
        assert _same(a[k], b[k]) and _same(a[k], c[k]), k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_time_steps_bitwise_repeatable(precision):
    P = FlowParams(rcr=[RCR(srfid=3)], precision=precision)
    inflow = lambda t: 10.0 + 5.0 * np.sin(2 * np.pi * t / 0.8)
    F = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10), P, inflow=inflow)
    G = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10), P, inflow=inflow)
    try:
        for _ in range(2):
            sf = F.step()
            sg = G.step()
            assert [sf.cg_itr[i] for i in range(sf.nsolves)] == [sg.cg_itr[i] for i in range(sg.nsolves)]
        yf, af = F.state()
        yg, ag = G.state()
    finally:
        F.close()
        G.close()
    assert _same(yf, yg) and _same(af, ag)
    assert sf.p_out[0] == sg.p_out[0]
