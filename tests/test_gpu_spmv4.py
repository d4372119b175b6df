"""4x4 block SpMV (SPARMULVV, dof 4) against scipy's BSR product on the
ElmGMR pattern of a small jittered lattice: FP64 to 1e-13, FP32 to 1e-5
(normwise, FP32 values and vectors with FP32 accumulation)."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from crimsonflowsolver_b200 import FlowParams, mesh, solver
from crimsonflowsolver_b200 import _native as N
from tests.conftest import relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,tol", [(0, 1e-13), (1, 1e-5)])
def test_spmv4_matches_bsr(prec, tol):
    import torch

    m = mesh.lattice(6)
    elm = solver.ElmGMR(m, FlowParams())
    try:
        colm, rowp = elm.genadj()
        nnz = len(rowp)
        rng = np.random.default_rng(11)
        val = rng.standard_normal((nnz, 16))
        u = rng.standard_normal((m.nshg, 4))
        A = sp.bsr_matrix((val.reshape(-1, 4, 4), rowp - 1, colm - 1), shape=(4 * m.nshg, 4 * m.nshg))
        ref = (A @ u.ravel()).reshape(-1, 4)
        dt = torch.float64 if prec == 0 else torch.float32
        dv = torch.tensor(val, dtype=dt, device="cuda")
        du = torch.tensor(u, dtype=dt, device="cuda")
        dk = torch.zeros_like(du)
        torch.cuda.synchronize()
        L = N.lib()
        N.check(L.crimson_spmv4_prepare(elm.h, prec, ctypes.c_void_p(dv.data_ptr())), "prepare")
        for _ in range(2):   # twice: the sliced copy is reused
            N.check(L.crimson_spmv4_apply(elm.h, ctypes.c_void_p(du.data_ptr()), ctypes.c_void_p(dk.data_ptr())),
                    "apply")
        torch.cuda.synchronize()
        got = dk.double().cpu().numpy()
    finally:
        elm.close()
    assert relerr(got, ref) < tol, relerr(got, ref)
