"""Failure detection on the GPU path without a GPU fault.

A time step from a state holding a NaN returns CRIMSON_ERR_NONFINITE (the
NSSOLVER right-hand side is checked before any Krylov work; every device
loop is bounded), and the context stays usable: after the state is reset, the
next step equals a fresh solver's step from the same state bit for bit (the
whole path is deterministic, so nothing the failed step left behind may
change a result).
"""
import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, RCR, mesh, solver
from crimsonflowsolver_b200 import _native as N
from tests.conftest import relerr


def _rcr(F, set_to=None):
    """Read (or write) the RCR history (P_n, Q_n) of a solver's context."""
    P = np.zeros(1) if set_to is None else np.array(set_to[0], dtype=np.float64)
    Q = np.zeros(1) if set_to is None else np.array(set_to[1], dtype=np.float64)
    N.check(N.lib().crimson_rcr_state(F.elm.h, 1, N.dp(P), N.dp(Q), 0 if set_to is None else 1), "crimson_rcr_state")
    return P.copy(), Q.copy()

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nonfinite_state_returns_status_and_context_recovers(precision):
    m = mesh.cylinder(ncross=8, naxial=10)
    P = FlowParams(rcr=[RCR(srfid=3)], precision=precision)
    F = solver.FlowSolver(m, P, inflow=lambda t: 10.0)
    G = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10), P, inflow=lambda t: 10.0)
    try:
        F.step()
        y, ac = F.state()
        bad = y.copy()
        bad[m.nshg // 2, 0] = np.nan
        F.set_state(bad, ac)
        with pytest.raises(RuntimeError, match="NONFINITE"):
            F.step()
        F.set_state(y, ac)
        G.set_state(y, ac)
        _rcr(G, _rcr(F))   # the failed step left F's outlet history as it was after step 1
        F.istep = G.istep = 1
        F.step()
        G.step()
        y1, _ = F.state()
        y2, _ = G.state()
        assert np.all(np.isfinite(y1))
        assert np.array_equal(y1, y2), relerr(y1, y2)
    finally:
        F.close()
        G.close()
