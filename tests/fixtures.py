"""The reference's own test mesh (testbin/mainTests/basic: 1072 nodes, 4157
tets, 1092 boundary faces, PHASTA restart state) as a Mesh, from the
committed fixture tests/golden/basic_mesh.npz (see make_phasta_fixture.py)."""
import os

import numpy as np

from crimsonflowsolver_b200 import mesh as meshmod

HERE = os.path.dirname(os.path.abspath(__file__))


def basic_mesh():
    d = np.load(os.path.join(HERE, "golden", "basic_mesh.npz"))
    m = meshmod.Mesh(x=d["x"].copy(), ien=d["ien"].copy(), name="reference basic")
    m.ienb = d["ienb"].copy()
    m.iBCB = d["iBCB"].copy()
    m.BCB = np.repeat(d["BCB"][:, None, :], 3, axis=1).copy()   # per face node
    m.iBC = d["iBC"].copy()
    m.BC = np.zeros((m.nshg, meshmod.NDOFBC))
    m.NABI, m.ndsurf = meshmod.compute_nabi(m.x, m.ienb, m.iBCB, m.nshg)
    m.outlets = sorted(int(s) for s in np.unique(m.iBCB[:, 1]) if s >= meshmod.SRF_OUTLET0)
    return m, d["y"].copy(), d["ac"].copy()
