"""Synthetic workload meshes: orientation, surfaces and outlet geometry (CPU)."""
import numpy as np

from crimsonflowsolver_b200 import mesh


def _signed_volumes(m):
    x, ien = m.x, m.ien
    a = x[ien[:, 1]] - x[ien[:, 0]]
    b = x[ien[:, 2]] - x[ien[:, 0]]
    c = x[ien[:, 3]] - x[ien[:, 0]]
    return np.einsum("ij,ij->i", a, np.cross(b, c)) / 6.0


def test_bifurcation_geometry():
    m = mesh.bifurcation(h=0.2)
    v = _signed_volumes(m)
    assert np.all(v < 0) or np.all(v > 0)          # one orientation (the reference's)
    vol = np.abs(v).sum()
    exact = np.pi * 1.0 * 5.5 + 2 * np.pi * 0.49 * 5.0   # parent to B + R/2, two daughters (overlap ignored)
    assert 0.8 * exact < vol < 1.1 * exact
    assert m.outlets == [3, 4]
    for s, sx in ((3, 1.0), (4, -1.0)):
        a = m.NABI[m.ndsurf == s].sum(axis=0)
        ang = np.degrees(np.arctan2(sx * a[0], a[2]))
        assert abs(ang - 30.0) < 3.0, ang          # outlet normal along the daughter axis
        assert abs(a[1]) < 1e-9
    assert len(m.inlet_nodes) > 0 and np.all(m.x[m.inlet_nodes, 2] == 0.0)
    rcr = mesh.bifurcation_rcr()
    assert [r["srfid"] for r in rcr] == [3, 4]
    for r in rcr:
        assert 80.0 <= r["Rp"] <= 120.0 and 0.8e-4 <= r["C"] <= 1.2e-4 and 800.0 <= r["Rd"] <= 1200.0


def test_cylinder_sector_outlets():
    m = mesh.cylinder(ncross=8, naxial=6, n_outlets=3)
    assert m.outlets == [3, 4, 5]
    tot = sum(m.NABI[m.ndsurf == s].sum(axis=0) for s in m.outlets)
    assert tot[2] > 0 and abs(tot[0]) < 0.2 * tot[2] and abs(tot[1]) < 0.2 * tot[2]
