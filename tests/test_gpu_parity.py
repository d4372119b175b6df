"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Tolerances (normwise, max|gpu - oracle| / max|oracle| per array):
  * CSR pattern (colm, rowp): bit-exact.
  * res, lhsK, lhsP: 1e-12.  The GPU sums element contributions with FP64
    atomics in a nondeterministic order and forms the quadrature sums
    algebraically, so results agree to rounding, not bit for bit.
  * memLS solution: 1e-10 relative to the solution norm on the same
    Res4/Val4, with identical outer/inner iteration counts.
"""
import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, RCR, mesh, solver
from oracle import pyoracle as po
from tests.conftest import relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    m = mesh.cylinder(ncross=8, naxial=10)
    m.set_inflow(10.0)
    P = FlowParams(rcr=[RCR(srfid=3)])
    elm = solver.ElmGMR(m, P)
    colm, rowp = elm.genadj()
    return m, P, elm, colm, rowp


def test_pattern_bit_exact(case):
    m, P, elm, colm, rowp = case
    ocolm, orowp = po.genadj(m.ien, m.nshg)
    assert np.array_equal(colm, ocolm)
    assert np.array_equal(rowp, orowp)


def test_pattern_lattice_bit_exact():
    m = mesh.lattice(6)
    elm = solver.ElmGMR(m, FlowParams())
    colm, rowp = elm.genadj()
    ocolm, orowp = po.genadj(m.ien, m.nshg)
    assert np.array_equal(colm, ocolm) and np.array_equal(rowp, orowp)


@pytest.mark.parametrize("state", ["random", "flow"])
def test_elmgmr_parity(case, state):
    m, P, elm, colm, rowp = case
    rng = np.random.default_rng(7)
    if state == "random":
        y = rng.standard_normal((m.nshg, 4))
        ac = rng.standard_normal((m.nshg, 4))
    else:
        y = np.zeros((m.nshg, 4))
        r2 = m.x[:, 0] ** 2 + m.x[:, 1] ** 2
        y[:, 2] = 20.0 * np.clip(1 - r2, 0, None)
        y[:, 3] = 3.2 * (10.0 - m.x[:, 2])
        ac = 0.1 * rng.standard_normal((m.nshg, 4))
    c1, c2 = [123.0], [-7.5]
    g = elm(y, ac, c1, c2)
    o = po.Elm(m, P, colm, rowp)(y, ac, srflist=[3], coef1=c1, coef2=c2)
    for k in ("res", "lhsK", "lhsP"):
        assert relerr(g[k], o[k]) < 1e-12, (k, relerr(g[k], o[k]))


def test_elmgmr_residual_only(case):
    m, P, elm, colm, rowp = case
    rng = np.random.default_rng(8)
    y = rng.standard_normal((m.nshg, 4))
    ac = rng.standard_normal((m.nshg, 4))
    g = elm(y, ac, [1.0], [2.0], lhs=False)
    o = po.Elm(m, P, colm, rowp)(y, ac, lhs=False, srflist=[3], coef1=[1.0], coef2=[2.0])
    assert g["lhsK"] is None
    assert relerr(g["res"], o["res"]) < 1e-12


def test_elmgmr_no_diffusive_flux(case):
    m, P0, elm0, colm, rowp = case
    P = FlowParams(idiff=0, rcr=[RCR(srfid=3)])
    elm = solver.ElmGMR(m, P)
    rng = np.random.default_rng(9)
    y = rng.standard_normal((m.nshg, 4))
    ac = rng.standard_normal((m.nshg, 4))
    g = elm(y, ac, [5.0], [1.0])
    o = po.Elm(m, P, colm, rowp)(y, ac, srflist=[3], coef1=[5.0], coef2=[1.0])
    for k in ("res", "lhsK", "lhsP"):
        assert relerr(g[k], o[k]) < 1e-12, k


def _system(case):
    m, P, elm, colm, rowp = case
    F = po.OracleFlow(m, P)
    F.y = F.yold.copy()
    F.ac = F.acold * ((P.gami - 1) / P.gami)
    F._itr_bc(F.y)
    c1, c2 = F.implicit_coeffs(0)
    yA = F.y.copy()
    acA = F.ac.copy()
    acA[:, 3] = 0
    out = F.elm(yA, acA, srflist=[3], coef1=c1, coef2=c2)
    Res4, Val4 = po.solflow_pack(m.nshg, colm, rowp, out["res"], out["lhsK"], out["lhsP"])
    faceRes = np.array([0.0, c1[0]]) * P.alfi * P.gami * P.Delt
    return F, Res4, Val4, faceRes, out, (yA, acA, c1, c2)


def test_memls_solve_parity(case):
    m, P, elm, colm, rowp = case
    F, Res4, Val4, faceRes, _, _ = _system(case)
    osol, ost = F.memls.solve(Res4, Val4.copy(), faceRes)
    ms = solver.MemLS(P, 2, nshg=m.nshg, colm=colm, rowp=rowp)
    nodes, sv = solver.dirichlet_face(m)
    ms.bc_create(1, nodes, 3, 0, sv)
    nn, vv = solver.neumann_face(m, 3)
    ms.bc_create(2, nn, 3, 1, vv)
    V = Val4.copy()
    gsol, gst = ms.solve(Res4, V, faceRes)
    assert (gst.RI.itr, gst.GM.itr, gst.CG.itr) == (ost.RI.itr, ost.GM.itr, ost.CG.itr)
    assert relerr(gsol, osol) < 1e-10, relerr(gsol, osol)


def test_solflow_device_parity(case):
    import torch

    m, P, elm, colm, rowp = case
    F, Res4, Val4, faceRes, out, (yA, acA, c1, c2) = _system(case)
    osol, ost = F.memls.solve(Res4, Val4.copy(), faceRes)
    ms = solver.MemLS(P, 2, ctx=elm)
    nodes, sv = solver.dirichlet_face(m)
    ms.bc_create(1, nodes, 3, 0, sv)
    nn, vv = solver.neumann_face(m, 3)
    ms.bc_create(2, nn, 3, 1, vv)
    dev = torch.device("cuda:0")
    dy = torch.tensor(yA, device=dev)
    dac = torch.tensor(acA, device=dev)
    dres = torch.zeros((m.nshg, 4), dtype=torch.float64, device=dev)
    dK = torch.zeros((len(rowp), 9), dtype=torch.float64, device=dev)
    dP = torch.zeros((len(rowp), 4), dtype=torch.float64, device=dev)
    dsol = torch.zeros((m.nshg, 4), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    elm.device(dy, dac, dres, dK, dP, c1, c2)
    st = ms.solflow_device(elm, dres, dK, dP, faceRes, dsol)
    torch.cuda.synchronize()
    assert relerr(dres.cpu().numpy(), Res4) < 1e-12
    assert (st.RI.itr, st.GM.itr, st.CG.itr) == (ost.RI.itr, ost.GM.itr, ost.CG.itr)
    assert relerr(dsol.cpu().numpy(), osol) < 1e-10, relerr(dsol.cpu().numpy(), osol)


def test_time_steps_parity():
    m = mesh.cylinder(ncross=8, naxial=10)
    P = FlowParams(rcr=[RCR(srfid=3)])
    inflow = lambda t: 10.0 + 5.0 * np.sin(2 * np.pi * t / 0.8)
    F = po.OracleFlow(m, P, inflow=inflow)
    G = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10), P, inflow=inflow)
    for _ in range(2):
        F.step()
        st = G.step()
    y, ac = G.state()
    assert relerr(y[:, 0:3], F.y[:, 0:3]) < 1e-10, relerr(y[:, 0:3], F.y[:, 0:3])
    assert relerr(y[:, 3], F.y[:, 3]) < 1e-10, relerr(y[:, 3], F.y[:, 3])
    assert abs(st.p_out[0] - F.Pn[0]) <= 1e-10 * abs(F.Pn[0])


def test_bifurcation_time_steps_parity():
    """Two time steps on a small Y-bifurcation (two RCR outlets, +-20% seeded
    values) against the oracle: the multi-outlet coupling path."""
    m = mesh.bifurcation(h=0.25)
    P = FlowParams(rcr=[RCR(**d) for d in mesh.bifurcation_rcr()])
    inflow = lambda t: 10.0 + 5.0 * np.sin(2 * np.pi * t / 0.8)
    F = po.OracleFlow(m, P, inflow=inflow)
    G = solver.FlowSolver(mesh.bifurcation(h=0.25), P, inflow=inflow)
    try:
        for _ in range(2):
            F.step()
            st = G.step()
        y, ac = G.state()
    finally:
        G.close()
    assert relerr(y[:, 0:3], F.y[:, 0:3]) < 1e-10, relerr(y[:, 0:3], F.y[:, 0:3])
    assert relerr(y[:, 3], F.y[:, 3]) < 1e-10, relerr(y[:, 3], F.y[:, 3])
    for k in range(2):
        assert abs(st.p_out[k] - F.Pn[k]) <= 1e-10 * abs(F.Pn[k])


@pytest.mark.parametrize("state", ["restart", "seeded"])
def test_reference_mesh_parity(state):
    """The reference's own test mesh (testbin/mainTests/basic) with its
    restart state, and with a seeded velocity field on the same mesh: CSR
    pattern bit-exact and ElmGMR (its boundary faces and outlets included)
    within 1e-12 of the oracle."""
    from tests.fixtures import basic_mesh

    m, y, ac = basic_mesh()
    if state == "seeded":
        rng = np.random.default_rng(17)
        y[:, 0:3] = 10.0 * rng.standard_normal((m.nshg, 3))
        ac = rng.standard_normal((m.nshg, 4))
    srf = m.outlets
    P = FlowParams(rcr=[RCR(srfid=s) for s in srf])
    elm = solver.ElmGMR(m, P)
    try:
        colm, rowp = elm.genadj()
        oc, orp = po.genadj(m.ien, m.nshg)
        assert np.array_equal(colm, oc) and np.array_equal(rowp, orp)
        c1 = [110.0 + 5 * k for k in range(len(srf))]
        c2 = [-3.0 + k for k in range(len(srf))]
        g = elm(y, ac, c1, c2)
        o = po.Elm(m, P, colm, rowp)(y, ac, srflist=srf, coef1=c1, coef2=c2)
    finally:
        elm.close()
    for k in ("res", "lhsK", "lhsP"):
        assert relerr(g[k], o[k]) < 1e-12, (k, relerr(g[k], o[k]))


def test_time_steps_parity_launch_per_step_gmres():
    """Krylov space 80 (> 64) runs GMRES through the launch-per-step loop
    instead of the persistent cycle kernel: the same parity bar."""
    m = mesh.cylinder(ncross=8, naxial=10)
    P = FlowParams(rcr=[RCR(srfid=3)], kspace=80)
    inflow = lambda t: 10.0 + 5.0 * np.sin(2 * np.pi * t / 0.8)
    F = po.OracleFlow(m, P, inflow=inflow)
    G = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10), P, inflow=inflow)
    try:
        for _ in range(2):
            F.step()
            st = G.step()
        y, ac = G.state()
    finally:
        G.close()
    assert relerr(y[:, 0:3], F.y[:, 0:3]) < 1e-10, relerr(y[:, 0:3], F.y[:, 0:3])
    assert relerr(y[:, 3], F.y[:, 3]) < 1e-10, relerr(y[:, 3], F.y[:, 3])
    assert abs(st.p_out[0] - F.Pn[0]) <= 1e-10 * abs(F.Pn[0])


def test_multi_outlet_time_steps_parity():
    """Three RCR outlets splitting one cap: the outlet surfaces share their
    rim nodes, so the two ADDBCMUL passes of every GMRES product couple the
    faces (the persistent GMRES cycle carries their valM Gram matrix)."""
    m = mesh.cylinder(ncross=8, naxial=8, n_outlets=3)
    P = FlowParams(rcr=[RCR(srfid=3), RCR(srfid=4, Rp=120.0, C=1.2e-4), RCR(srfid=5, Rd=900.0)])
    inflow = lambda t: 10.0 + 5.0 * np.sin(2 * np.pi * t / 0.8)
    F = po.OracleFlow(m, P, inflow=inflow)
    G = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=8, n_outlets=3), P, inflow=inflow)
    try:
        for _ in range(2):
            F.step()
            st = G.step()
        y, ac = G.state()
    finally:
        G.close()
    assert relerr(y[:, 0:3], F.y[:, 0:3]) < 1e-10, relerr(y[:, 0:3], F.y[:, 0:3])
    assert relerr(y[:, 3], F.y[:, 3]) < 1e-10, relerr(y[:, 3], F.y[:, 3])
    for k in range(3):
        assert abs(st.p_out[k] - F.Pn[k]) <= 1e-10 * abs(F.Pn[k])


def test_elmgmr_partial_constraints_parity():
    """Wall nodes with one or two prescribed velocity components (ibits 1-6,
    random BC(:,4:6) coefficients): bc3LHS on every element block, the
    boundary elements' unit diagonal entries, and bc3Res -- res, lhsK, lhsP
    within 1e-12 of the oracle."""
    from tests.partial_bc import with_partial_constraints

    m = mesh.cylinder(ncross=8, naxial=10)
    m.set_inflow(10.0)
    with_partial_constraints(m)
    P = FlowParams(rcr=[RCR(srfid=3)])
    elm = solver.ElmGMR(m, P)
    try:
        colm, rowp = elm.genadj()
        rng = np.random.default_rng(21)
        y = rng.standard_normal((m.nshg, 4))
        ac = rng.standard_normal((m.nshg, 4))
        g = elm(y, ac, [80.0], [-4.0])
        o = po.Elm(m, P, colm, rowp)(y, ac, srflist=[3], coef1=[80.0], coef2=[-4.0])
    finally:
        elm.close()
    for k in ("res", "lhsK", "lhsP"):
        assert relerr(g[k], o[k]) < 1e-12, (k, relerr(g[k], o[k]))


def test_time_steps_partial_constraints_parity():
    """Two time steps with slip-type constraints (ibits 1-5) on half of the
    wall nodes: itrBC, bc3Res and bc3LHS in the step against the oracle."""
    from tests.partial_bc import with_partial_constraints

    inflow = lambda t: 10.0 + 5.0 * np.sin(2 * np.pi * t / 0.8)
    P = FlowParams(rcr=[RCR(srfid=3)])
    meshes = []
    for _ in range(2):
        m = mesh.cylinder(ncross=8, naxial=10)
        with_partial_constraints(m, masks=(1, 2, 3, 4, 5))
        meshes.append(m)
    F = po.OracleFlow(meshes[0], P, inflow=inflow)
    G = solver.FlowSolver(meshes[1], P, inflow=inflow)
    try:
        its = []
        for _ in range(2):
            F.step()
            st = G.step()
            its += [(st.ri_itr[i], st.gm_itr[i], st.cg_itr[i]) for i in range(st.nsolves)]
        y, ac = G.state()
    finally:
        G.close()
    assert its == [s[:3] for s in F.stats]
    assert relerr(y[:, 0:3], F.y[:, 0:3]) < 1e-10, relerr(y[:, 0:3], F.y[:, 0:3])
    assert relerr(y[:, 3], F.y[:, 3]) < 1e-10, relerr(y[:, 3], F.y[:, 3])
