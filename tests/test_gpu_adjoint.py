"""Adjoint building blocks and the checkpointed gradient, through the C ABI.

* crimson_elmgmr_vjp against central differences of crimson_elmgmr_device
  (the production residual) in random directions of y, ac, mu and the
  coupling coefficients: relative error <= 1e-6.
* crimson_solflow_device_transposed against a sparse direct solve of the
  transposed system: <= 1e-4 (memLS stops at an estimated relative
  residual of epstol_ns = 1e-5 in the scaled norm).
* dJ/dtheta of the outlet-pressure misfit (theta = mu and the 3 RCR
  parameters of each of 3 outlets) against central finite differences of the
  forward solver with relative step 1e-6: <= 1e-4 relative, component by
  component; the checkpoint interval does not change the gradient.
"""
import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, RCR, mesh, solver
from crimsonflowsolver_b200.adjoint import AdjointProblem, make_objective_function
from tests.conftest import relerr
from tests.linsys import assembled_matrix, first_system, free_dofs

pytestmark = pytest.mark.gpu


def _inflow(t):
    return 10.0 + 5.0 * np.sin(2 * np.pi * t / 0.8)


@pytest.fixture(scope="module")
def flowstate():
    import torch

    m = mesh.cylinder(ncross=8, naxial=10, n_outlets=3)
    P = FlowParams(rcr=[RCR(srfid=3), RCR(srfid=4, Rp=120.0), RCR(srfid=5, Rd=900.0)])
    F = solver.FlowSolver(m, P, inflow=_inflow)
    for _ in range(2):
        F.step()
    y, ac = F.state()
    F.close()
    dev = torch.device("cuda:0")
    return m, P, torch.tensor(y, device=dev), torch.tensor(ac, device=dev)


def _res(elm, y, ac, c1, c2):
    import torch

    r = torch.zeros_like(y)
    elm.device(y, ac, r, None, None, c1, c2, lhs=False)
    torch.cuda.synchronize()
    return r


def _vjp(elm, y, ac, c1, c2, lam):
    import ctypes

    import torch

    from crimsonflowsolver_b200 import _native as N

    yb = torch.zeros_like(y)
    ab = torch.zeros_like(y)
    res = torch.zeros_like(y)
    mub = ctypes.c_double()
    nc = len(c1)
    c1b = np.zeros(nc)
    c2b = np.zeros(nc)
    torch.cuda.synchronize()
    N.check(N.lib().crimson_elmgmr_vjp(elm.h, y.data_ptr(), ac.data_ptr(), N.dp(np.asarray(c1, float)),
                                       N.dp(np.asarray(c2, float)), lam.data_ptr(), res.data_ptr(), yb.data_ptr(),
                                       ab.data_ptr(), ctypes.byref(mub), N.dp(c1b), N.dp(c2b)), "vjp")
    torch.cuda.synchronize()
    return res, yb, ab, mub.value, c1b, c2b


def test_vjp_matches_central_differences(flowstate):
    import torch

    m, P, y, ac = flowstate
    elm = solver.ElmGMR(m, P)
    try:
        c1 = [95.0, 120.0, 88.0]
        c2 = [3.0, -2.0, 1.5]
        g = torch.Generator(device="cpu").manual_seed(7)
        lam = torch.randn(y.shape, generator=g, dtype=torch.float64).to(y.device)
        res, yb, ab, mub, c1b, c2b = _vjp(elm, y, ac, c1, c2, lam)
        r0 = _res(elm, y, ac, c1, c2)
        assert relerr(res.cpu().numpy(), r0.cpu().numpy()) < 1e-12
        # state directions
        for trial in range(3):
            dy = torch.randn(y.shape, generator=g, dtype=torch.float64).to(y.device)
            da = torch.randn(y.shape, generator=g, dtype=torch.float64).to(y.device)
            da[:, 3] = 0.0
            dy *= float(y[:, 0:3].abs().max())
            da *= float(ac[:, 0:3].abs().max() + 1.0)
            h = 1e-6
            fp = float((lam * _res(elm, y + h * dy, ac + h * da, c1, c2)).sum())
            fm = float((lam * _res(elm, y - h * dy, ac - h * da, c1, c2)).sum())
            fd = (fp - fm) / (2 * h)
            an = float((yb * dy).sum() + (ab * da).sum())
            assert abs(fd - an) <= 1e-6 * abs(an), (trial, fd, an)
        # coupling coefficients
        for k in range(3):
            for which, bar in ((0, c1b), (1, c2b)):
                cc = [list(c1), list(c2)]
                hk = 1e-2 * max(abs(cc[which][k]), 1.0)   # res is linear in coef1, coef2
                cp = [list(c1), list(c2)]
                cm = [list(c1), list(c2)]
                cp[which][k] += hk
                cm[which][k] -= hk
                fd = float((lam * (_res(elm, y, ac, *cp) - _res(elm, y, ac, *cm))).sum()) / (2 * hk)
                assert abs(fd - bar[k]) <= 1e-6 * max(abs(bar[k]), 1e-300), (which, k, fd, bar[k])
    finally:
        elm.close()
    # viscosity: residual of contexts built with mu (1 +- h)
    h = 1e-6
    fs = []
    for s in (1.0, -1.0):
        Pm = FlowParams(rcr=P.rcr, mu=P.mu * (1.0 + s * h))
        e2 = solver.ElmGMR(m, Pm)
        try:
            fs.append(float((lam * _res(e2, y, ac, c1, c2)).sum()))
        finally:
            e2.close()
    fd = (fs[0] - fs[1]) / (2 * h * P.mu)
    assert abs(fd - mub) <= 1e-6 * abs(mub), (fd, mub)


def test_transposed_solve_matches_direct():
    import torch

    m = mesh.cylinder(ncross=8, naxial=10)
    m.set_inflow(10.0)
    P = FlowParams(rcr=[RCR(srfid=3)])
    elm = solver.ElmGMR(m, P)
    colm, rowp = elm.genadj()
    F, Res4, Val4, faceRes, out, (yA, acA, c1, c2) = first_system(m, P, colm, rowp)
    ms = solver.MemLS(P, 2, ctx=elm)
    try:
        nodes, sv = solver.dirichlet_face(m)
        ms.bc_create(1, nodes, 3, 0, sv)
        nn, vv = solver.neumann_face(m, 3)
        ms.bc_create(2, nn, 3, 1, vv)
        dev = torch.device("cuda:0")
        dres = torch.zeros((m.nshg, 4), dtype=torch.float64, device=dev)
        dK = torch.zeros((len(rowp), 9), dtype=torch.float64, device=dev)
        dP = torch.zeros((len(rowp), 4), dtype=torch.float64, device=dev)
        elm.device(torch.tensor(yA, device=dev), torch.tensor(acA, device=dev), dres, dK, dP, c1, c2)
        rng = np.random.default_rng(3)
        r = rng.standard_normal((m.nshg, 4))
        sol = torch.zeros_like(dres)
        import ctypes

        from crimsonflowsolver_b200 import _native as N

        st = N.LsStats()
        inc = np.ones(2, dtype=np.int32)
        fr = np.ascontiguousarray(faceRes, dtype=np.float64)
        rd = torch.tensor(r, device=dev)
        torch.cuda.synchronize()
        N.check(N.lib().crimson_solflow_device_transposed(elm.h, ms.lhs, ms.ls, rd.data_ptr(), dK.data_ptr(),
                                                          dP.data_ptr(), N.ip(inc), N.dp(fr), sol.data_ptr(),
                                                          ctypes.byref(st)), "transposed")
        torch.cuda.synchronize()
        z = sol.cpu().numpy()
    finally:
        ms.close()
        elm.close()
    import scipy.sparse.linalg as spla

    A = assembled_matrix(m, colm, rowp, Val4, faceRes)
    f = free_dofs(m)
    AT = A[f][:, f].T.tocsc()
    zd = np.zeros(4 * m.nshg)
    zd[f] = spla.spsolve(AT, r.ravel()[f])
    assert st.RI.suc == 1
    assert np.all(z.ravel()[~f] == 0.0)
    assert relerr(z.ravel(), zd) < 1e-4, relerr(z.ravel(), zd)


def _problem(ce):
    m = mesh.cylinder(ncross=8, naxial=8, n_outlets=3)
    # 10 nonlinear iterations per step: the adjoint differentiates the
    # converged step, so the forward map must be converged for central
    # differences to see the same derivative (with 6, J itself still moves by
    # 1e-6 relative and the mu component by 1.7e-4)
    P = FlowParams(rcr=[RCR(srfid=3), RCR(srfid=4, Rp=120.0, C=1.2e-4), RCR(srfid=5, Rd=900.0)], nitr=10)
    return AdjointProblem(m, P, targets=[2.0, 3.0, 1.5], nsteps=4, inflow=_inflow, checkpoint_every=ce)


def test_adjoint_gradient_matches_central_fd():
    prob = _problem(ce=2)
    th = prob.theta0()
    J, g = prob.gradient(th)
    its = prob.last_stats["adjoint_iterations"]
    assert max(its) < prob.adj_maxit, its
    fd = np.zeros_like(th)
    for i in range(len(th)):
        h = 1e-6 * abs(th[i])
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        fd[i] = (prob.objective(tp) - prob.objective(tm)) / (2 * h)
    sens_ad = th * g
    sens_fd = th * fd
    err = np.abs(sens_ad - sens_fd) / np.abs(sens_fd)
    print("J", J, "adjoint iterations per step", its, "\nlog-sensitivities adjoint", sens_ad, "\nfd", sens_fd,
          "\nerr", err)
    assert err.max() < 1e-4, err


def _oracle_objective(prob, theta):
    """J(theta) from the FP64 CPU oracle's own time stepping (the reference
    algorithm restated), one thread so that every evaluation rounds alike."""
    from oracle import pyoracle as po

    F = po.OracleFlow(prob.mesh, prob.params(theta), nthreads=1, inflow=prob.inflow)
    Ps = np.zeros((prob.nsteps, prob.nc))
    for n in range(prob.nsteps):
        F.step()
        Ps[n] = F.Pn
    return prob._objective(Ps)


def test_adjoint_gradient_matches_central_fd_of_oracle():
    """The GPU adjoint gradient against central differences (relative step
    1e-6) of the reference solver restated on the CPU, for mu and the 9 RCR
    parameters: within 1e-4 relative per component (log-sensitivities)."""
    prob = _problem(ce=2)
    th = prob.theta0()
    J, g = prob.gradient(th)
    J_oracle = _oracle_objective(prob, th)
    assert abs(J - J_oracle) <= 1e-8 * abs(J_oracle), (J, J_oracle)
    fd = np.zeros_like(th)
    for i in range(len(th)):
        h = 1e-6 * abs(th[i])
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        fd[i] = (_oracle_objective(prob, tp) - _oracle_objective(prob, tm)) / (2 * h)
    err = np.abs(th * g - th * fd) / np.abs(th * fd)
    print("oracle central FD: J", J_oracle, "\nlog-sensitivities adjoint", th * g, "\nfd", th * fd, "\nerr", err)
    assert err.max() < 1e-4, err


def test_checkpoint_interval_and_autograd():
    import torch

    p1 = _problem(ce=1)
    p4 = _problem(ce=4)
    th = p1.theta0()
    J1, g1 = p1.gradient(th)
    J4, g4 = p4.gradient(th)
    assert abs(J1 - J4) <= 1e-12 * abs(J1)
    assert np.abs(g1 - g4).max() <= 1e-9 * np.abs(g1).max()
    Obj = make_objective_function()
    t = torch.tensor(th, dtype=torch.float64, requires_grad=True)
    J = Obj.apply(t, p4)
    J.backward()
    assert abs(float(J.detach()) - J4) <= 1e-12 * abs(J4)
    assert np.abs(t.grad.numpy() - g4).max() <= 1e-9 * np.abs(g4).max()
