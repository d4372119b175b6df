"""GPU parity of ElmGMRSclr (flowsolver/src/elmgmr.f90:599-822): the CUDA
path through crimson_elmgmr_sclr / crimson_elmgmr_sclr_device against the
oracle's orc_elmgmr_sclr on the same inputs.

Tolerance: res and lhsS within 1e-12 normwise (max |gpu - oracle| / max
|oracle|).  The device kernels evaluate the same quadrature formulas in the
same order per element and sum per entry in ascending element order (faces
after elements), but the compiler may contract multiply-adds differently, so
the bar is rounding, not bits.  Repeated GPU calls are bitwise identical.
"""
import copy

import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, mesh, solver
from oracle import pyoracle as po
from tests.conftest import relerr
from tests.fixtures import basic_mesh

pytestmark = pytest.mark.gpu


def _with_scalar_bits(m0, isclr):
    """Dirichlet bit isclr + 5 on the inlet nodes, flux bit 4 + isclr on the outlet faces."""
    m = copy.copy(m0)
    m.iBC = m0.iBC.copy()
    inlet = np.unique(m.ienb[m.iBCB[:, 1] == 1, :3])
    m.iBC[inlet] |= 1 << (isclr + 5)
    m.iBCB = m0.iBCB.copy()
    flux = np.nonzero(m.iBCB[:, 1] >= 3)[0]
    m.iBCB[flux, 0] |= 1 << (4 + isclr)
    return m, inlet, flux


def _state(m, seed):
    rng = np.random.default_rng(seed)
    y = rng.standard_normal((m.nshg, 4))
    return y, rng.standard_normal(m.nshg), rng.standard_normal(m.nshg)


@pytest.fixture(scope="module")
def cyl():
    m = mesh.cylinder(ncross=8, naxial=10)
    m.set_inflow(10.0)
    return m


@pytest.mark.parametrize("idiff", [1, 0])
@pytest.mark.parametrize("lhs", [True, False])
def test_sclr_parity(cyl, idiff, lhs):
    P = FlowParams(idiff=idiff)
    elm = solver.ElmGMR(cyl, P)
    colm, rowp = elm.genadj()
    y, s, sd = _state(cyl, 11)
    g = elm.sclr(y, s, sd, isclr=1, diffus=0.2, lhs=lhs)
    o = po.elmgmr_sclr(po.Elm(cyl, P, colm, rowp), y, s, sd, isclr=1, diffus=0.2, lhs=lhs)
    assert relerr(g["res"], o["res"]) < 1e-12
    if lhs:
        assert relerr(g["lhsS"], o["lhsS"]) < 1e-12
    else:
        assert g["lhsS"] is None
    elm.close()


@pytest.mark.parametrize("isclr", [1, 3])
def test_sclr_bits_parity(cyl, isclr):
    m, inlet, flux = _with_scalar_bits(cyl, isclr)
    P = FlowParams()
    elm = solver.ElmGMR(m, P)
    colm, rowp = elm.genadj()
    y, s, sd = _state(m, 12)
    bcbs = np.zeros((m.ienb.shape[0], 3))
    bcbs[flux] = np.random.default_rng(13).standard_normal((flux.size, 3))
    g = elm.sclr(y, s, sd, isclr=isclr, diffus=0.05, bcbs=bcbs)
    o = po.elmgmr_sclr(po.Elm(m, P, colm, rowp), y, s, sd, isclr=isclr, diffus=0.05, bcbs=bcbs)
    assert np.all(g["res"][inlet] == 0.0)
    assert relerr(g["res"], o["res"]) < 1e-12
    assert relerr(g["lhsS"], o["lhsS"]) < 1e-12
    # a face that prescribes the flux needs bcbs
    with pytest.raises(RuntimeError):
        elm.sclr(y, s, sd, isclr=isclr, diffus=0.05)
    # the flux bit of another scalar is not this scalar's
    o2 = po.elmgmr_sclr(po.Elm(m, P, colm, rowp), y, s, sd, isclr=2, diffus=0.05)
    assert relerr(elm.sclr(y, s, sd, isclr=2, diffus=0.05)["res"], o2["res"]) < 1e-12
    elm.close()


def test_sclr_reference_basic_mesh_parity():
    m, y, _ = basic_mesh()
    P = FlowParams()
    elm = solver.ElmGMR(m, P)
    colm, rowp = elm.genadj()
    _, s, sd = _state(m, 14)
    y = np.asarray(y[:, :4], dtype=np.float64)
    g = elm.sclr(y, s, sd, isclr=1, diffus=0.04)
    o = po.elmgmr_sclr(po.Elm(m, P, colm, rowp), y, s, sd, isclr=1, diffus=0.04)
    assert relerr(g["res"], o["res"]) < 1e-12
    assert relerr(g["lhsS"], o["lhsS"]) < 1e-12
    elm.close()


def test_sclr_patch_and_repeatability(cyl):
    elm = solver.ElmGMR(cyl, FlowParams(idiff=1))
    grad = np.array([0.3, -1.2, 0.7])
    s = cyl.x @ grad + 2.0
    g = elm.sclr(np.zeros((cyl.nshg, 4)), s, np.zeros(cyl.nshg), diffus=0.25)
    assert np.abs(g["res"]).max() < 1e-11
    y, s, sd = _state(cyl, 15)
    a = elm.sclr(y, s, sd, diffus=0.1)
    b = elm.sclr(y, s, sd, diffus=0.1)
    assert np.array_equal(a["res"], b["res"]) and np.array_equal(a["lhsS"], b["lhsS"])
    elm.close()


def test_sclr_device_entry_matches_host(cyl):
    import torch

    P = FlowParams()
    elm = solver.ElmGMR(cyl, P)
    nnz = elm._nnz()
    y, s, sd = _state(cyl, 16)
    h = elm.sclr(y, s, sd, isclr=1, diffus=0.1)
    dev = torch.device("cuda:0")
    d_y = torch.from_numpy(np.ascontiguousarray(y)).to(dev)          # (nshg, 4) row-major = node-major
    d_s = torch.from_numpy(s).to(dev)
    d_sd = torch.from_numpy(sd).to(dev)
    d_res = torch.zeros(cyl.nshg, dtype=torch.float64, device=dev)
    d_lhs = torch.zeros(nnz, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    elm.sclr_device(d_y, d_s, d_sd, d_res, d_lhs, isclr=1, diffus=0.1)
    torch.cuda.synchronize()
    assert np.array_equal(d_res.cpu().numpy(), h["res"])
    assert np.array_equal(d_lhs.cpu().numpy(), h["lhsS"])
    elm.close()


def test_sclr_rejects_bad_arguments(cyl):
    elm = solver.ElmGMR(cyl, FlowParams())
    y, s, sd = _state(cyl, 17)
    for isclr in (0, 5):
        with pytest.raises(RuntimeError):
            elm.sclr(y, s, sd, isclr=isclr, diffus=0.1)
    with pytest.raises(RuntimeError):
        elm.sclr(y, s, sd, isclr=1, diffus=-1.0)
    elm.close()
    with pytest.raises(RuntimeError):
        with solver.ElmGMR(cyl, FlowParams(idiff=2)) as elm:
            elm.sclr(y, s, sd, isclr=1, diffus=0.1)
