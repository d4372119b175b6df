"""PHASTA reader / writer (CPU).

Fixtures from the reference's own case testbin/mainTests/basic
(tests/golden/make_phasta_fixture.py): basic_mesh.npz holds the arrays this
path reads; basic_headers.json holds the text lines of geombc.dat.1 and
restart.0.1 (comments and block headers, no binary data).  The reader is
checked on a file assembled from those header lines and the fixture's arrays,
and the writer's headers against the reference restart's, so both run
without a reference checkout.
"""
import json
import os

import numpy as np
import pytest

from crimsonflowsolver_b200 import phasta

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
REF_BASIC = os.path.join(os.environ.get("CRIMSON_REFERENCE", "/nonexistent"), "testbin", "mainTests", "basic")


def _fixture():
    return np.load(os.path.join(GOLDEN, "basic_mesh.npz"))


def _headers():
    with open(os.path.join(GOLDEN, "basic_headers.json")) as f:
        return json.load(f)


def test_restart_round_trip(tmp_path):
    d = _fixture()
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


def test_reference_headers_parse():
    """Every block header of the reference's geombc/restart follows the grammar
    the reader parses, and the sizes agree with the fixture's arrays."""
    d = _fixture()
    nn, ne, nb = d["x"].shape[0], d["ien"].shape[0], d["ienb"].shape[0]
    for name, lines in _headers().items():
        blocks = {}
        for line in lines:
            if line.startswith("#") or not line.strip():
                continue
            key, nbytes, ints = phasta.parse_header(line)
            blocks[key] = (nbytes, ints)
        if name == "geombc.dat.1":
            assert blocks["co-ordinates"] == (nn * 3 * 8 + 1, [nn, 3])
            assert blocks["connectivity interior linear tetrahedron"][0] == ne * 4 * 4 + 1
            assert blocks["connectivity interior linear tetrahedron"][1][:2] == [ne, 4]
            assert blocks["connectivity boundary linear tetrahedron"][0] == nb * 4 * 4 + 1
            assert blocks["nbc codes linear tetrahedron"][0] == nb * 2 * 4 + 1
            assert blocks["nbc values linear tetrahedron"][0] == nb * 6 * 8 + 1
            nd = len(d["dirichlet_nodes"])
            assert blocks["bc codes array"] == (nd * 4 + 1, [nd])
            assert blocks["boundary condition array"] == (d["dirichlet_values"].size * 8 + 1,
                                                          [d["dirichlet_values"].size])
        else:
            assert blocks["solution"] == (nn * 5 * 8 + 1, [nn, 5, 0])
            assert blocks["time derivative of solution"] == (nn * 5 * 8 + 1, [nn, 5, 0])


def test_reader_on_reference_headers(tmp_path):
    """A geombc assembled from the reference's header lines (keys, byte counts,
    header integers) with the fixture's arrays as data reads back to them."""
    d = _fixture()
    nn = d["x"].shape[0]
    dn = d["dirichlet_nodes"]
    nbc = np.zeros(nn, dtype=np.int32)
    nbc[dn] = np.arange(1, len(dn) + 1)
    data = {
        "co-ordinates": d["x"].astype("<f8"),
        "connectivity interior linear tetrahedron": (d["ien"] + 1).astype("<i4"),
        "connectivity boundary linear tetrahedron": (d["ienb"] + 1).astype("<i4"),
        "nbc codes linear tetrahedron": d["iBCB"].astype("<i4"),
        "nbc values linear tetrahedron": d["BCB"].astype("<f8"),
        "bc mapping array": nbc.astype("<i4"),
        "bc codes array": d["iBC"][dn].astype("<i4"),
        "boundary condition array": d["dirichlet_values"].astype("<f8"),
    }
    out = bytearray()
    for line in _headers()["geombc.dat.1"]:
        out += (line + "\n").encode("latin1")
        if line.startswith("#") or not line.strip():
            continue
        key, nbytes, ints = phasta.parse_header(line)
        if key == "byteorder magic number":
            payload = np.array([phasta.MAGIC], "<i4").tobytes()
        elif key in data:
            payload = np.asfortranarray(data[key]).tobytes(order="F")
        else:
            payload = bytes(max(nbytes - 1, 0))   # blocks this path does not read
        assert len(payload) + (1 if nbytes else 0) == nbytes, key
        out += payload + (b"\n" if nbytes else b"")
    p = tmp_path / "geombc.dat.1"
    p.write_bytes(bytes(out))
    m = phasta.read_geombc(str(p))
    assert np.array_equal(m.x, d["x"]) and np.array_equal(m.ien, d["ien"])
    assert np.array_equal(m.ienb, d["ienb"]) and np.array_equal(m.iBCB, d["iBCB"])
    assert np.array_equal(m.iBC, d["iBC"]) and np.array_equal(m.dirichlet_values, d["dirichlet_values"])


def test_writer_headers_match_reference_restart(tmp_path):
    """write_restart emits the reference restart's magic-number, size and
    solution / time-derivative headers (same keys, byte counts, integers)."""
    d = _fixture()
    p = str(tmp_path / "restart.0.1")
    phasta.write_restart(p, d["y"], d["ac"], step=0)
    ours = [phasta.parse_header(s) for s in phasta.header_lines(p) if s.strip() and not s.startswith("#")]
    ref = [phasta.parse_header(s) for s in _headers()["restart.0.1"] if s.strip() and not s.startswith("#")]
    ref_by_key = {k: (nb, ints) for k, nb, ints in ref}
    assert [k for k, _, _ in ours] == [k for k, _, _ in ref][:len(ours)]
    for k, nb, ints in ours:
        assert ref_by_key[k] == (nb, ints), k
    y, ac, step = phasta.read_restart(p)
    assert step == 0 and np.array_equal(y, d["y"]) and np.array_equal(ac, d["ac"])


@pytest.mark.skipif(not os.path.isdir(REF_BASIC), reason="set CRIMSON_REFERENCE to a reference checkout")
def test_reader_matches_committed_fixture():
    d = _fixture()
    m = phasta.read_geombc(os.path.join(REF_BASIC, "geombc.dat.1"))
    y, ac, _ = phasta.read_restart(os.path.join(REF_BASIC, "restart.0.1"))
    assert np.array_equal(m.x, d["x"]) and np.array_equal(m.ien, d["ien"])
    assert np.array_equal(m.ienb, d["ienb"]) and np.array_equal(m.iBCB, d["iBCB"])
    assert np.array_equal(m.iBC, d["iBC"]) and np.array_equal(y, d["y"])
