"""Mixed-precision NS solve (FP32 inner matvecs + FP64 iterative refinement).

Checks, on the first Newton system of a small cylinder with a coupled
resistance outlet:
  * the FP64 defect |R - A x| / |R| of the scaled system reported by the
    library is at most the refinement tolerance;
  * the solution agrees with an independent FP64 sparse direct solve:
    1e-5 (normwise) at the default refinement tolerance epstol_ns = 1e-5,
    1e-7 at a refinement tolerance of 1e-10 (where FP64 memLS alone cannot
    go: its residual estimate sqrt(|R|^2 - x_B . B) loses all digits below
    about 1e-8);
  * host (Val4) and device (lhsK/lhsP) entry points agree;
  * two device time steps in mixed precision track a tightly converged FP64
    oracle run to 1e-6 on velocity, pressure and outlet pressure.
"""
import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, RCR, mesh, solver
from oracle import pyoracle as po
from tests.conftest import relerr
from tests.linsys import defect, direct_solve, first_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system():
    m = mesh.cylinder(ncross=8, naxial=10)
    m.set_inflow(10.0)
    P = FlowParams(rcr=[RCR(srfid=3)])
    elm = solver.ElmGMR(m, P)
    colm, rowp = elm.genadj()
    F, Res4, Val4, faceRes, out, state = first_system(m, P, colm, rowp)
    xd, A, f = direct_solve(m, colm, rowp, Res4, Val4, faceRes)
    yield m, P, elm, colm, rowp, Res4, Val4, faceRes, state, xd, A, f
    elm.close()


def _host_memls(m, P, colm, rowp):
    ms = solver.MemLS(P, 2, nshg=m.nshg, colm=colm, rowp=rowp)
    nodes, sv = solver.dirichlet_face(m)
    ms.bc_create(1, nodes, 3, 0, sv)
    nn, vv = solver.neumann_face(m, 3)
    ms.bc_create(2, nn, 3, 1, vv)
    return ms


@pytest.mark.parametrize("refine_tol,bound", [(0.0, 1e-5), (1e-10, 1e-7)])
def test_mixed_solve_vs_direct(system, refine_tol, bound):
    m, P, elm, colm, rowp, Res4, Val4, faceRes, state, xd, A, f = system
    Pm = FlowParams(rcr=P.rcr, precision="mixed", max_refine=8, refine_tol=refine_tol)
    with_tol = refine_tol if refine_tol > 0 else P.epstol_ns
    ms = _host_memls(m, Pm, colm, rowp)
    try:
        sol, st = ms.solve(Res4, Val4.copy(), faceRes)
        steps, rel = ms.refine_info()
    finally:
        ms.close()
    assert 1 <= steps <= 8
    assert rel <= with_tol, (steps, rel)
    assert st.RI.suc == 1
    e = relerr(sol, xd)
    assert e < bound, (e, steps, rel)
    assert defect(A, f, sol, Res4) < 10 * with_tol
    assert np.all(sol.ravel()[~f] == 0.0)


def test_mixed_device_matches_host(system):
    import torch

    m, P, elm, colm, rowp, Res4, Val4, faceRes, (yA, acA, c1, c2), xd, A, f = system
    Pm = FlowParams(rcr=P.rcr, precision="mixed", max_refine=8, refine_tol=1e-10)
    ms = solver.MemLS(Pm, 2, ctx=elm)
    try:
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
        steps, rel = ms.refine_info()
    finally:
        ms.close()
    assert rel <= 1e-10 and st.RI.suc == 1
    assert relerr(dsol.cpu().numpy(), xd) < 1e-7


def test_mixed_time_steps_track_fp64_oracle():
    """Two mixed-precision time steps against FP64 oracle runs.

    The FP64 oracle at the default tolerances (epstol_ns 1e-5) differs from
    itself run at epstol_ns 3e-7 by 2.4e-6 (velocity) / 8e-6 (pressure) after
    two steps: that is the size of the linear-solve tolerance, not of the
    arithmetic.  So the mixed run (refinement to 1e-9) is checked at 1e-6
    against the tightly converged FP64 oracle, and against the default one at
    the default tolerance's own spread (1e-5 velocity, 3e-5 pressure).
    """
    inflow = lambda t: 10.0 + 5.0 * np.sin(2 * np.pi * t / 0.8)
    m = mesh.cylinder(ncross=8, naxial=10)
    Pm = FlowParams(rcr=[RCR(srfid=3)], precision="mixed", max_refine=8, refine_tol=1e-9)
    G = solver.FlowSolver(m, Pm, inflow=inflow)
    try:
        for _ in range(2):
            st = G.step()
        y, ac = G.state()
    finally:
        G.close()
    for P, bv, bp in ((FlowParams(rcr=[RCR(srfid=3)], epstol_ns=3e-7, epstol_mom=3e-6, epstol_cont=3e-6), 1e-6, 1e-6),
                      (FlowParams(rcr=[RCR(srfid=3)]), 1e-5, 3e-5)):
        F = po.OracleFlow(mesh.cylinder(ncross=8, naxial=10), P, inflow=inflow)
        for _ in range(2):
            F.step()
        ev = relerr(y[:, 0:3], F.y[:, 0:3])
        ep = relerr(y[:, 3], F.y[:, 3])
        eo = abs(st.p_out[0] - F.Pn[0]) / abs(F.Pn[0])
        print(f"mixed vs fp64 oracle (epstol_ns {P.epstol_ns:g}): vel {ev:.3e} p {ep:.3e} Pout {eo:.3e}")
        assert ev < bv, ev
        assert ep < bp, ep
        assert eo < bp, eo


def test_fp32_tangent_records_match_fp64(system):
    """FP32 element quadrature of the tangent: the 16-float records equal the
    FP64 lhsK / lhsP to FP32 rounding (1e-6 normwise) and the residual formed
    alongside is the FP64 one (1e-12)."""
    import ctypes

    import torch

    from crimsonflowsolver_b200 import _native as N

    m, P, elm, colm, rowp, Res4, Val4, faceRes, (yA, acA, c1, c2), xd, A, f = system
    dev = torch.device("cuda:0")
    dy = torch.tensor(yA, device=dev)
    dac = torch.tensor(acA, device=dev)
    nnz = len(rowp)
    r64 = torch.zeros((m.nshg, 4), dtype=torch.float64, device=dev)
    K = torch.zeros((nnz, 9), dtype=torch.float64, device=dev)
    Pm = torch.zeros((nnz, 4), dtype=torch.float64, device=dev)
    elm.device(dy, dac, r64, K, Pm, c1, c2)
    r32 = torch.zeros_like(r64)
    rec = torch.zeros((nnz, 16), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    N.check(N.lib().crimson_elmgmr_device_f32(elm.h, dy.data_ptr(), dac.data_ptr(), N.dp(np.asarray(c1, float)),
                                              N.dp(np.asarray(c2, float)), r32.data_ptr(), rec.data_ptr()), "f32")
    torch.cuda.synchronize()
    rec = rec.double().cpu().numpy()
    assert relerr(r32.cpu().numpy(), r64.cpu().numpy()) < 1e-12
    assert relerr(rec[:, 0:9], K.cpu().numpy()) < 1e-6
    assert relerr(rec[:, 9:13], Pm.cpu().numpy()) < 1e-6
    assert np.all(rec[:, 13:16] == 0.0)


def test_f32_tangent_converged_steps_match_fp64():
    """FP32 element quadrature of the tangent (mixed_f32_tangent) changes the
    Newton path, not its limit: with the nonlinear iterations converged (8
    per step) two steps agree with the FP64 path to 1e-6."""
    inflow = lambda t: 10.0 + 5.0 * np.sin(2 * np.pi * t / 0.8)
    out = {}
    for prec, extra in (("fp64", dict(epstol_ns=3e-7, epstol_mom=3e-6, epstol_cont=3e-6)),
                        ("mixed_f32_tangent", dict(max_refine=8, refine_tol=1e-9))):
        P = FlowParams(rcr=[RCR(srfid=3)], nitr=8, precision=prec, **extra)
        G = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10), P, inflow=inflow)
        try:
            for _ in range(2):
                st = G.step()
            out[prec] = (G.state()[0], st.p_out[0])
        finally:
            G.close()
    y64, p64 = out["fp64"]
    y32, p32 = out["mixed_f32_tangent"]
    ev = relerr(y32[:, 0:3], y64[:, 0:3])
    ep = relerr(y32[:, 3], y64[:, 3])
    print(f"f32 tangent, converged steps: vel {ev:.3e} p {ep:.3e} Pout {abs(p32 - p64) / abs(p64):.3e}")
    assert ev < 1e-6 and ep < 1e-6 and abs(p32 - p64) <= 1e-6 * abs(p64)

def test_mixed_first_sweep_meets_tolerance():
    """The least-squares products of the mixed NSSOLVER are FP64, so its
    residual estimate is that of the FP64 operator: one sweep reaches the
    NSSOLVER tolerance in the FP64 defect, with the iteration counts of the
    FP64 solve (the FP32 Krylov directions differ only in rounding), and the
    time steps agree with the FP64 library run far below the tolerance.
    """
    inflow = lambda t: 10.0 + 5.0 * np.sin(2 * np.pi * t / 0.8)
    m = mesh.cylinder(ncross=8, naxial=10)
    runs = {}
    for prec in ("fp64", "mixed"):
        P = FlowParams(rcr=[RCR(srfid=3)], precision=prec, max_refine=8)
        F = solver.FlowSolver(m, P, inflow=inflow)
        try:
            stats = [F.step() for _ in range(3)]
            runs[prec] = (F.state(), stats, P.epstol_ns)
        finally:
            F.close()
    (y64, _), s64, tol = runs["fp64"]
    (ym, _), sm, _ = runs["mixed"]
    for a, b in zip(s64, sm):
        assert a.nsolves == b.nsolves
        for i in range(b.nsolves):
            assert b.refine_steps[i] == 1, (i, b.refine_steps[i], b.refine_rel[i])
            assert b.refine_rel[i] <= tol
            assert a.ri_itr[i] == b.ri_itr[i]
            assert abs(a.cg_itr[i] - b.cg_itr[i]) <= 0.02 * a.cg_itr[i]
    ev = relerr(ym[:, 0:3], y64[:, 0:3])
    ep = relerr(ym[:, 3], y64[:, 3])
    print(f"mixed vs FP64 library after 3 steps: vel {ev:.3e} p {ep:.3e}")
    assert ev < 1e-7 and ep < 1e-7, (ev, ep)


def test_explicit_schur_cg(system):
    """The mixed solve's inner CG on the explicit FP32 Schur operator
    S = L - Gt G (2-ring pattern) against the two-product FP32 CG: both meet
    the refinement tolerance and the direct solve's bound, the operator has
    the node graph's 2-ring as its pattern, and two solves give the same bits."""
    import scipy.sparse as sp

    m, P, elm, colm, rowp, Res4, Val4, faceRes, state, xd, A, f = system
    sols = {}
    for schur in (1, 0):
        Pm = FlowParams(rcr=P.rcr, precision="mixed", max_refine=8, refine_tol=1e-10, explicit_schur=schur)
        ms = _host_memls(m, Pm, colm, rowp)
        try:
            sol, st = ms.solve(Res4, Val4.copy(), faceRes)
            steps, rel = ms.refine_info()
            info = ms.schur_info()
            if schur:
                sol2, _ = ms.solve(Res4, Val4.copy(), faceRes)
                assert np.array_equal(sol, sol2)
        finally:
            ms.close()
        assert rel <= 1e-10 and st.RI.suc == 1, (schur, steps, rel)
        assert relerr(sol, xd) < 1e-7, (schur, relerr(sol, xd))
        sols[schur] = sol
        if schur:
            n = m.nshg
            r = np.repeat(np.arange(n), np.diff(colm))
            G1 = sp.csr_matrix((np.ones(len(rowp)), (r, rowp - 1)), shape=(n, n))
            assert info[0] == 1 and info[1] == (G1 @ G1).nnz, info
        else:
            assert info[0] == 0, info
    assert relerr(sols[1], sols[0]) < 1e-7
