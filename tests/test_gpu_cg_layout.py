"""Both column layouts of the persistent CG kernel give the same solve.

The kernel keeps the column indices of its rows in shared memory as 16-bit
offsets col - row when every offset fits (meshes numbered with locality, as
generated); otherwise it reads them from the sliced pattern in each phase.
A randomly renumbered copy of a 41k-node cylinder has offsets up to the node
count and takes the second layout.  One time step on both numberings, FP64
and mixed (the two-product CG, explicit_schur=0): the same iteration counts
and states equal to rounding (the CSR rows sum their entries in a different
order after renumbering).  The mixed solve's explicit FP32 Schur operator
needs 16-bit 2-ring offsets too: on the renumbered mesh it is not built and
the solve falls back to the two-product CG, bit for bit.
"""
import ctypes

import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, RCR, mesh, solver
from crimsonflowsolver_b200 import _native as N
from tests.conftest import relerr

pytestmark = pytest.mark.gpu


def _renumber(m, seed=11):
    """Copy of m with node i renamed perm[i]."""
    rng = np.random.default_rng(seed)
    n = m.nshg
    perm = rng.permutation(n)
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n)

    def nodal(a):
        return None if a is None else a[inv]

    return mesh.Mesh(x=m.x[inv].copy(), ien=perm[m.ien].astype(np.int32), name=m.name + "-renumbered",
                     ienb=perm[m.ienb].astype(np.int32), iBCB=m.iBCB.copy(), BCB=m.BCB.copy(), iBC=nodal(m.iBC),
                     BC=nodal(m.BC), ndsurf=nodal(m.ndsurf), NABI=nodal(m.NABI),
                     inlet_nodes=perm[m.inlet_nodes], inlet_profile=m.inlet_profile.copy(),
                     outlets=list(m.outlets)), perm


def _run(m, precision, explicit_schur=0):
    P = FlowParams(rcr=[RCR(srfid=3)], precision=precision, max_refine=8, explicit_schur=explicit_schur)
    F = solver.FlowSolver(m, P, inflow=lambda t: 10.0)
    try:
        st = F.step()
        y, _ = F.state()
        if explicit_schur:
            return y, st, F.memls.schur_info()[0], None
        r64, r32, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        N.check(N.lib().crimson_memls_cg_layout(F.memls.lhs, ctypes.byref(r64), ctypes.byref(r32), ctypes.byref(nb)),
                "crimson_memls_cg_layout")
        res = r64.value if precision == "fp64" else r32.value
        return y, st, res, nb.value
    finally:
        F.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_resident_and_streamed_columns_agree(precision):
    m = mesh.cylinder(ncross=32, naxial=48)
    assert m.nshg > 32768
    mr, perm = _renumber(m)
    y0, s0, res0, nb0 = _run(m, precision)
    y1, s1, res1, nb1 = _run(mr, precision)
    assert res0 == 1 and nb0 > 0
    assert res1 == 0 and nb1 == 0
    assert s0.nsolves == s1.nsolves
    for i in range(s0.nsolves):
        assert s0.ri_itr[i] == s1.ri_itr[i]
        assert abs(s0.cg_itr[i] - s1.cg_itr[i]) <= 1 + 0.01 * s0.cg_itr[i]
    e = relerr(y1[perm], y0)
    assert e < 1e-8, e


def test_explicit_schur_falls_back_on_wide_offsets():
    mr, _ = _renumber(mesh.cylinder(ncross=32, naxial=48))
    y0, s0, _, _ = _run(mr, "mixed", explicit_schur=0)
    y1, s1, state, _ = _run(mr, "mixed", explicit_schur=1)
    assert state == -1
    assert np.array_equal(y0, y1)
