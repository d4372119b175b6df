"""CPU: crimson_ctx_create rejects invalid meshes on the host with a clean
error status, before any device work (runs without a GPU).

A zero-volume tet, a tet ordered against the orientation e3metric assumes
(det[x1-x4, x2-x4, x3-x4] > 0), a non-finite coordinate and an out-of-range
node index each return CRIMSON_ERR_ARG with a message naming the element or
node.  The generated meshes pass the same check.
"""
import ctypes

import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, mesh
from crimsonflowsolver_b200 import _native as N
from crimsonflowsolver_b200.solver import make_params


def _create(x, ien):
    """Call crimson_ctx_create with column-major 1-based arrays; returns (rc, message)."""
    L = N.lib()
    prm = make_params(FlowParams())
    h = ctypes.c_void_p()
    xf = np.asfortranarray(x, dtype=np.float64)
    ienf = np.asfortranarray(ien + 1, dtype=np.int32)
    rc = L.crimson_ctx_create(ctypes.byref(h), ctypes.byref(prm), x.shape[0], x.shape[0], ien.shape[0],
                              ienf.ctypes.data_as(N.c_int_p), xf.ctypes.data_as(N.c_dbl_p))
    msg = L.crimson_last_error().decode()
    if rc == N.OK:
        L.crimson_ctx_destroy(h)
    return rc, msg


def _two_tets():
    x = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [1.0, 1.0, 1.0]])
    ien = np.array([[0, 1, 2, 3], [1, 2, 3, 4]])
    # order each tet as e3metric needs
    for e in range(2):
        d = x[ien[e, :3]] - x[ien[e, 3]]
        if np.linalg.det(d) < 0:
            ien[e, [1, 2]] = ien[e, [2, 1]]
    return x, ien


def test_generated_meshes_pass_orientation_check():
    for m in (mesh.cylinder(ncross=6, naxial=4), mesh.lattice(4), mesh.bifurcation(h=0.4)):
        ien = m.ien
        d = m.x[ien[:, :3]] - m.x[ien[:, 3:4]]
        assert np.all(np.linalg.det(d) > 0), m.name


@pytest.mark.parametrize("case", ["zero_volume", "inverted", "nan_coordinate", "node_out_of_range"])
def test_invalid_mesh_rejected_on_host(case):
    x, ien = _two_tets()
    if case == "zero_volume":
        x[4] = (x[1] + x[2] + x[3]) / 3.0     # node 5 in the plane of nodes 2, 3, 4: tet 2 flat
    elif case == "inverted":
        ien[1, [1, 2]] = ien[1, [2, 1]]
    elif case == "nan_coordinate":
        x[3, 2] = np.nan
    else:
        ien[1, 3] = 7
    rc, msg = _create(x, ien)
    assert rc == 1, (rc, msg)                   # CRIMSON_ERR_ARG
    if case in ("zero_volume", "inverted"):
        assert "element 2" in msg and "volume" in msg, msg
    elif case == "nan_coordinate":
        assert "node 4" in msg, msg
    else:
        assert "element 2" in msg, msg
