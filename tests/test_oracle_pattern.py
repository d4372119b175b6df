"""CPU: the oracle's genadj restatement against an independent sort+unique."""
import numpy as np

from oracle import pyoracle as po
from crimsonflowsolver_b200 import mesh


def _ref_pattern(ien, nshg):
    ie = ien.astype(np.int64)
    keys = np.unique((ie[:, :, None] * nshg + ie[:, None, :]).ravel())
    rows, cols = keys // nshg, keys % nshg
    colm = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=nshg))]) + 1
    return colm.astype(np.int32), (cols + 1).astype(np.int32)


def test_genadj_cylinder(small_cyl):
    colm, rowp = po.genadj(small_cyl.ien, small_cyl.nshg)
    c2, r2 = _ref_pattern(small_cyl.ien, small_cyl.nshg)
    assert np.array_equal(colm, c2) and np.array_equal(rowp, r2)


def test_genadj_lattice_shuffled():
    m = mesh.lattice(4)
    ien = m.ien[np.random.default_rng(3).permutation(m.nelem)]
    colm, rowp = po.genadj(ien, m.nshg)
    c2, r2 = _ref_pattern(ien, m.nshg)
    assert np.array_equal(colm, c2) and np.array_equal(rowp, r2)
    # every row holds its diagonal and is sorted
    for i in range(m.nshg):
        row = rowp[colm[i] - 1:colm[i + 1] - 1]
        assert np.all(np.diff(row) > 0) and (i + 1) in row


def test_genadj_single_element():
    ien = np.array([[0, 1, 2, 3]], dtype=np.int32)
    colm, rowp = po.genadj(ien, 4)
    assert list(colm) == [1, 5, 9, 13, 17]
    assert list(rowp) == [1, 2, 3, 4] * 4


def test_reference_mesh_fixture_loads_and_is_oriented():
    """The reference's own mesh: every tet has det[x1-x4, x2-x4, x3-x4] > 0
    (the orientation e3metric's WdetJ > 0 needs), and genadj's pattern is
    symmetric with the diagonal in every row."""
    from tests.fixtures import basic_mesh

    m, y, ac = basic_mesh()
    x, ien = m.x, m.ien
    det = np.einsum("ij,ij->i", x[ien[:, 0]] - x[ien[:, 3]],
                    np.cross(x[ien[:, 1]] - x[ien[:, 3]], x[ien[:, 2]] - x[ien[:, 3]]))
    assert np.all(det > 0)
    colm, rowp = po.genadj(m.ien, m.nshg)
    rows = np.repeat(np.arange(m.nshg), np.diff(colm))
    pairs = set(zip(rows.tolist(), (rowp - 1).tolist()))
    assert all((c, r) in pairs for r, c in pairs)
    assert all((i, i) in pairs for i in range(m.nshg))
    assert y.shape == (1072, 4) and np.all(np.isfinite(y))
