"""GPU: the allocation-free outlet coupling entry point (crimson_pvsq_noalloc).

Some callers cannot call cudaMalloc -- a stream being captured into a CUDA
graph, a host framework that owns all device memory through its own pool, a
latency-bound coupling loop where an allocation would synchronise the device.
crimson_pvsq_noalloc performs ElmGMR's outlet coupling (GetFlowQ + the
p_k NABI right-hand side) with its per-surface flows in a static device array
instead of memory the library allocates.  This test calls it through the C
ABI, twice in a row (the shared array keeps the previous call's contents),
and checks each result against the regular entry point, crimson_elmgmr_device,
which applies the same coupling inside ElmGMR: res_noalloc(coef) applied to
the uncoupled residual must equal the coupled residual within 1e-12
(normwise), and the returned flows must equal sum NABI . u.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_pvsq_noalloc_matches_elmgmr_coupling():
    import torch

    from crimsonflowsolver_b200 import FlowParams, RCR, mesh, solver
    from crimsonflowsolver_b200 import _native as N
    from tests.conftest import relerr

    m = mesh.cylinder(ncross=8, naxial=10)
    m.set_inflow(10.0)
    P = FlowParams(rcr=[RCR(srfid=3)])
    elm = solver.ElmGMR(m, P)
    nnz = elm._nnz()
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(11)
    nodes = np.nonzero(m.ndsurf == 3)[0]
    offsets = np.array([0, len(nodes)], dtype=np.int32)
    d_nodes = torch.tensor(nodes + 1, dtype=torch.int32, device=dev)
    d_nabi = torch.tensor(np.ascontiguousarray(m.NABI[nodes]), dtype=torch.float64, device=dev)
    for call in range(2):
        y = torch.tensor(rng.standard_normal((m.nshg, 4)), device=dev)
        ac = torch.tensor(rng.standard_normal((m.nshg, 4)), device=dev)
        dK = torch.zeros((nnz, 9), dtype=torch.float64, device=dev)
        dP = torch.zeros((nnz, 4), dtype=torch.float64, device=dev)
        c1 = [100.0 + 50.0 * call]
        c2 = [25.0 - 10.0 * call]
        coupled = torch.zeros((m.nshg, 4), dtype=torch.float64, device=dev)
        plain = torch.zeros((m.nshg, 4), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        elm.device(y, ac, coupled, dK, dP, c1, c2, lhs=False)
        elm.device(y, ac, plain, dK, dP, [0.0], [0.0], lhs=False)
        torch.cuda.synchronize()
        q = np.zeros(1)
        rc = N.lib().crimson_pvsq_noalloc(1, N.ip(offsets), d_nodes.data_ptr(), d_nabi.data_ptr(), y.data_ptr(),
                                          N.dp(np.array(c1)), N.dp(np.array(c2)), plain.data_ptr(), N.dp(q), None)
        N.check(rc, "crimson_pvsq_noalloc")
        torch.cuda.synchronize()
        assert relerr(plain.cpu().numpy(), coupled.cpu().numpy()) < 1e-12
        yh = y.cpu().numpy()
        q_ref = float(np.sum(m.NABI[nodes] * yh[nodes, 0:3]))
        assert abs(q[0] - q_ref) <= 1e-12 * max(1.0, np.abs(m.NABI[nodes] * yh[nodes, 0:3]).sum())


def test_pvsq_noalloc_rejects_too_many_surfaces():
    from crimsonflowsolver_b200 import _native as N

    off = np.zeros(66, dtype=np.int32)
    c = np.zeros(65)
    rc = N.lib().crimson_pvsq_noalloc(65, N.ip(off), ctypes.c_void_p(8), ctypes.c_void_p(8), ctypes.c_void_p(8),
                                      N.dp(c), N.dp(c), ctypes.c_void_p(8), None, None)
    assert rc == 2  # CRIMSON_ERR_UNSUPPORTED: checked before any device work
