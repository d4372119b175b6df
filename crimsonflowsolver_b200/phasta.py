"""PHASTA geombc / restart files (the reference's mesh and state format).

A PHASTA file is a sequence of text headers ``key : < nbytes > ints``, each
followed by ``nbytes`` bytes of binary data whose last byte is a newline; the
file starts with a byte-order magic number (362436) and ``#`` comment lines.
Arrays are Fortran column-major.  This module reads the blocks this path
needs (flowsolver/src/readnblk.f90:83-600 reads the same keys) and writes
restart files the reference can read back.

* :func:`read_geombc` -> :class:`~crimsonflowsolver_b200.mesh.Mesh`:
  coordinates, interior and boundary tet connectivity (0-based here),
  boundary codes / values (``iBCB``, ``BCB`` per face node), Dirichlet codes
  mapped to nodes (``iBC``; values in ``dirichlet_values``), NABI / ndsurf.
* :func:`read_restart` -> (y, ac) in this package's (u, v, w, p) order; the
  file stores (p, u, v, w, ...) per node, reordered as the reference's
  restart reader does (readnblk.f90:516-541).
* :func:`write_restart` writes ``solution`` and ``time derivative of
  solution`` with 5 variables per node (the scalar slot zero), the layout
  the reference reads.
"""
from __future__ import annotations

import re
from typing import Dict, Tuple

import numpy as np

from . import mesh as meshmod

MAGIC = 362436


_HEADER = re.compile(r"(.*?)\s*:\s*<\s*(\d+)\s*>(.*)")


def parse_header(line: str) -> Tuple[str, int, list]:
    """One block header ``key : < nbytes > ints`` -> (key, nbytes, ints)
    (the grammar cvSolverIO writes and reads, solverio/src/cvSolverIO.cxx)."""
    m = _HEADER.match(line)
    if not m:
        raise ValueError(f"bad header line {line!r}")
    return m.group(1).strip(), int(m.group(2)), [int(t) for t in m.group(3).split()]


def header_lines(path: str) -> list:
    """The text lines of a PHASTA file (comments and block headers, no data)."""
    b = open(path, "rb").read()
    pos, out = 0, []
    while pos < len(b):
        e = b.index(b"\n", pos)
        line = b[pos:e].decode("latin1")
        pos = e + 1
        out.append(line)
        if line.startswith("#") or not line.strip():
            continue
        pos += parse_header(line)[1]
    return out


def read_blocks(path: str) -> Tuple[Dict[str, Tuple[list, bytes]], str]:
    """All blocks of a PHASTA file: key -> (header ints, raw data), and the byte order."""
    b = open(path, "rb").read()
    pos = 0
    blocks = {}
    order = "<"
    while pos < len(b):
        e = b.index(b"\n", pos)
        line = b[pos:e].decode("latin1")
        pos = e + 1
        if line.startswith("#") or not line.strip():
            continue
        try:
            key, nb, ints = parse_header(line)
        except ValueError:
            raise ValueError(f"{path}: bad header line {line!r}") from None
        data = b[pos:pos + nb]
        if len(data) != nb:
            raise ValueError(f"{path}: block {key!r} is truncated")
        pos += nb
        if key == "byteorder magic number":
            order = "<" if np.frombuffer(data[:4], "<i4")[0] == MAGIC else ">"
        blocks[key] = (ints, data[:-1] if nb > 0 else b"")
    return blocks, order


def _arr(blocks, order, key, dtype, shape):
    ints, data = blocks[key]
    return np.frombuffer(data, order + dtype).reshape(shape, order="F").copy()


def read_geombc(path: str) -> meshmod.Mesh:
    g, o = read_blocks(path)
    nn = g["co-ordinates"][0][0]
    x = _arr(g, o, "co-ordinates", "f8", (nn, 3))
    ne, nshl = g["connectivity interior linear tetrahedron"][0][:2]
    if nshl != 4:
        raise ValueError("only linear tetrahedra are supported")
    ien = _arr(g, o, "connectivity interior linear tetrahedron", "i4", (ne, 4)) - 1
    m = meshmod.Mesh(x=x, ien=ien.astype(np.int32), name=path)
    key_b = "connectivity boundary linear tetrahedron"
    if key_b in g:
        nb = g[key_b][0][0]
        m.ienb = (_arr(g, o, key_b, "i4", (nb, 4)) - 1).astype(np.int32)
        m.iBCB = _arr(g, o, "nbc codes linear tetrahedron", "i4", (nb, 2)).astype(np.int32)
        bcb = _arr(g, o, "nbc values linear tetrahedron", "f8", (nb, 6))
        m.BCB = np.repeat(bcb[:, None, :], 3, axis=1).copy()
    m.iBC = np.zeros(nn, dtype=np.int32)
    m.BC = np.zeros((nn, meshmod.NDOFBC))
    if "bc mapping array" in g:
        nbc = _arr(g, o, "bc mapping array", "i4", (nn,))
        nd = g["bc codes array"][0][0]
        codes = _arr(g, o, "bc codes array", "i4", (nd,))
        nv = g["boundary condition array"][0][0]
        vals = _arr(g, o, "boundary condition array", "f8", (nd, nv // nd)) if nd else np.zeros((0, 1))
        dn = np.nonzero(nbc > 0)[0]
        m.iBC[dn] = codes[nbc[dn] - 1]
        m.dirichlet_nodes = dn.astype(np.int32)
        m.dirichlet_values = vals[nbc[dn] - 1]
    if m.ienb is not None:
        m.NABI, m.ndsurf = meshmod.compute_nabi(m.x, m.ienb, m.iBCB, nn)
        m.outlets = sorted(int(s) for s in np.unique(m.iBCB[:, 1]) if s >= meshmod.SRF_OUTLET0)
    return m


def read_restart(path: str) -> Tuple[np.ndarray, np.ndarray, int]:
    """(y, ac, step): y, ac (nshg, 4) in (u, v, w, p) order."""
    r, o = read_blocks(path)
    ints = r["solution"][0]
    nn, nv = ints[0], ints[1]
    step = ints[2] if len(ints) > 2 else 0
    q = _arr(r, o, "solution", "f8", (nn, nv))
    y = np.zeros((nn, 4))
    y[:, 0:3] = q[:, 1:4]
    y[:, 3] = q[:, 0]
    ac = np.zeros((nn, 4))
    if "time derivative of solution" in r and r["time derivative of solution"][0][0]:
        qa = _arr(r, o, "time derivative of solution", "f8", (nn, r["time derivative of solution"][0][1]))
        ac[:, 0:3] = qa[:, 1:4]
        ac[:, 3] = qa[:, 0]
    return y, ac, step


def _block(key: str, arr: np.ndarray, ints) -> bytes:
    data = np.asfortranarray(arr).astype("<f8").tobytes(order="F") + b"\n"
    head = f"{key} : < {len(data)} > {' '.join(str(i) for i in ints)} \n".encode("latin1")
    return head + data


def write_restart(path: str, y: np.ndarray, ac: np.ndarray, step: int = 0) -> None:
    """restart file with (p, u, v, w, 0) per node, readable by the reference."""
    nn = y.shape[0]

    def q(v):
        out = np.zeros((nn, 5))
        out[:, 0] = v[:, 3]
        out[:, 1:4] = v[:, 0:3]
        return out

    head = (b"# PHASTA Input File Version 2.0\n# Byte Order Magic Number : 362436 \n"
            b"byteorder magic number  : < 5 > 1 \n" + np.array([MAGIC], "<i4").tobytes() + b"\n"
            b"number of modes : < 0 > " + str(nn).encode() + b" \n"
            b"number of variables : < 0 > 5 \n")
    with open(path, "wb") as f:
        f.write(head)
        f.write(_block("solution", q(y), [nn, 5, step]))
        f.write(_block("time derivative of solution", q(ac), [nn, 5, step]))
