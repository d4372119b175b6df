"""PHASTA reader / writer (CPU)."""
import os

import numpy as np
import pytest

from crimsonflowsolver_b200 import phasta

REF_BASIC = os.path.join(os.environ.get("CRIMSON_REFERENCE", "/nonexistent"), "testbin", "mainTests", "basic")


def test_restart_round_trip(tmp_path):
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "basic_mesh.npz"))
    y, ac = d["y"], d["ac"]
    rng = np.random.default_rng(2)
    y = y + rng.standard_normal(y.shape)
    p = str(tmp_path / "restart.7.1")
    phasta.write_restart(p, y, ac, step=7)
    y2, ac2, step = phasta.read_restart(p)
    assert step == 7
    assert np.array_equal(y2, y) and np.array_equal(ac2, ac)
    blocks, order = phasta.read_blocks(p)
    assert order == "<" and blocks["solution"][0] == [y.shape[0], 5, 7]


@pytest.mark.skipif(not os.path.isdir(REF_BASIC), reason="set CRIMSON_REFERENCE to a reference checkout")
def test_reader_matches_committed_fixture():
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "basic_mesh.npz"))
    m = phasta.read_geombc(os.path.join(REF_BASIC, "geombc.dat.1"))
    y, ac, _ = phasta.read_restart(os.path.join(REF_BASIC, "restart.0.1"))
    assert np.array_equal(m.x, d["x"]) and np.array_equal(m.ien, d["ien"])
    assert np.array_equal(m.ienb, d["ienb"]) and np.array_equal(m.iBCB, d["iBCB"])
    assert np.array_equal(m.iBC, d["iBC"]) and np.array_equal(y, d["y"])
