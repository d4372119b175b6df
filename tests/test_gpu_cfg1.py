"""Parity on the plain-method configuration as built: the 24x24 x 40 jittered
cylinder (107,520 tets, 20,377 nodes), steady parabolic inflow of mean
10 cm/s, zero-traction outlet, no-slip wall, rho 1.06, mu 0.04, dt 1e-3,
10 time steps of 3 nonlinear iterations, FP64, NSSOLVER tolerance 1e-5 (the
tightest setting the reference's outer residual estimate decides
independently of rounding: at 1e-6 the oracle's own first solve takes 8
outer iterations with 8 threads and 10 with 1).

* FP64 GPU vs the FP64 oracle: identical outer / GMRES / CG iteration counts
  in every one of the 30 solves, velocity and pressure within 1e-10
  (normwise relative) after 10 steps.
* Mixed precision (FP32 inner Krylov matvecs, FP64 refinement to the same
  tolerance) vs the FP64 oracle: velocity and pressure within 1e-6.
"""
import os

import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, mesh, solver
from oracle import pyoracle as po
from tests.conftest import relerr

pytestmark = pytest.mark.gpu

NSTEPS = 10


def _params(**kw):
    return FlowParams(epstol_ns=1e-5, **kw)


@pytest.fixture(scope="module")
def oracle_run():
    m = mesh.cylinder(ncross=24, naxial=40, seed=1)
    assert (m.nelem, m.nshg) == (107520, 20377)
    F = po.OracleFlow(m, _params(), nthreads=os.cpu_count() or 1, inflow=lambda t: 10.0)
    for _ in range(NSTEPS):
        F.step()
    return F


def _gpu_run(precision):
    G = solver.FlowSolver(mesh.cylinder(ncross=24, naxial=40, seed=1), _params(precision=precision),
                          inflow=lambda t: 10.0)
    its = []
    try:
        for _ in range(NSTEPS):
            st = G.step()
            its += [(st.ri_itr[i], st.gm_itr[i], st.cg_itr[i]) for i in range(st.nsolves)]
        y, _ = G.state()
    finally:
        G.close()
    return y, its


def test_cfg1_fp64_matches_oracle(oracle_run):
    F = oracle_run
    y, its = _gpu_run("fp64")
    assert its == [s[:3] for s in F.stats]
    ev, ep = relerr(y[:, 0:3], F.y[:, 0:3]), relerr(y[:, 3], F.y[:, 3])
    print(f"cfg1 FP64 GPU vs oracle after {NSTEPS} steps: velocity {ev:.2e} pressure {ep:.2e}")
    assert ev < 1e-10 and ep < 1e-10, (ev, ep)


def test_cfg1_mixed_within_1e6_of_oracle(oracle_run):
    F = oracle_run
    y, _ = _gpu_run("mixed")
    ev, ep = relerr(y[:, 0:3], F.y[:, 0:3]), relerr(y[:, 3], F.y[:, 3])
    print(f"cfg1 mixed GPU vs FP64 oracle after {NSTEPS} steps: velocity {ev:.2e} pressure {ep:.2e}")
    assert ev < 1e-6 and ep < 1e-6, (ev, ep)
