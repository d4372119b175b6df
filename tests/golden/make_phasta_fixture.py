"""Build tests/golden/basic_mesh.npz from the reference's own test case
testbin/mainTests/basic (geombc.dat.1 + restart.0.1, PHASTA format).

Run once where the reference checkout is available:

    python tests/golden/make_phasta_fixture.py /path/to/reference

The PHASTA files are a sequence of text headers ``key : < nbytes > ints``,
each followed by ``nbytes`` bytes of binary data (the last one a newline);
the file starts with a byte-order magic number (362436).  Arrays are
Fortran column-major.  Kept: coordinates, interior and boundary tet
connectivity (0-based here), boundary codes / values, the Dirichlet code and
value arrays mapped to nodes, and the restart solution reordered as the
reference's restart reader does (y(:,1:3) = q(:,2:4), y(:,4) = q(:,1);
flowsolver/src/readnblk.f90:516-541).
"""
import os
import re
import sys

import numpy as np


def read_phasta(path):
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
        m = re.match(r"(.*?)\s*:\s*<\s*(\d+)\s*>(.*)", line)
        if not m:
            raise ValueError(f"bad header line {line!r}")
        key, nb, ints = m.group(1).strip(), int(m.group(2)), [int(t) for t in m.group(3).split()]
        data = b[pos:pos + nb]
        pos += nb
        if key == "byteorder magic number":
            magic = np.frombuffer(data[:4], "<i4")[0]
            order = "<" if magic == 362436 else ">"
        blocks[key] = (ints, data[:-1] if nb > 0 else b"")
    return blocks, order


def arr(blocks, order, key, dtype, shape):
    ints, data = blocks[key]
    a = np.frombuffer(data, order + dtype)
    return a.reshape(shape, order="F")


def main(ref):
    base = os.path.join(ref, "testbin", "mainTests", "basic")
    g, o = read_phasta(os.path.join(base, "geombc.dat.1"))
    nn = g["co-ordinates"][0][0]
    x = arr(g, o, "co-ordinates", "f8", (nn, 3))
    ne, nshl = g["connectivity interior linear tetrahedron"][0][:2]
    ien = arr(g, o, "connectivity interior linear tetrahedron", "i4", (ne, nshl)) - 1
    nb = g["connectivity boundary linear tetrahedron"][0][0]
    ienb = arr(g, o, "connectivity boundary linear tetrahedron", "i4", (nb, 4)) - 1
    ibcb = arr(g, o, "nbc codes linear tetrahedron", "i4", (nb, 2))
    bcb = arr(g, o, "nbc values linear tetrahedron", "f8", (nb, 6))
    nbc = arr(g, o, "bc mapping array", "i4", (nn,))
    nd = g["bc codes array"][0][0]
    ibc_codes = arr(g, o, "bc codes array", "i4", (nd,))
    nv = g["boundary condition array"][0][0]
    bc_vals = arr(g, o, "boundary condition array", "f8", (nd, nv // nd))
    r, ro = read_phasta(os.path.join(base, "restart.0.1"))
    q = arr(r, ro, "solution", "f8", (nn, r["solution"][0][1]))
    qa = arr(r, ro, "time derivative of solution", "f8", (nn, r["time derivative of solution"][0][1]))
    y = np.zeros((nn, 4))
    y[:, 0:3] = q[:, 1:4]
    y[:, 3] = q[:, 0]
    ac = np.zeros((nn, 4))
    ac[:, 0:3] = qa[:, 1:4]
    ac[:, 3] = qa[:, 0]
    iBC = np.zeros(nn, dtype=np.int32)
    dn = np.nonzero(nbc > 0)[0]
    iBC[dn] = ibc_codes[nbc[dn] - 1]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basic_mesh.npz")
    np.savez_compressed(out, x=x, ien=ien.astype(np.int32), ienb=ienb.astype(np.int32), iBCB=ibcb.astype(np.int32),
                        BCB=bcb, iBC=iBC, dirichlet_nodes=dn.astype(np.int32),
                        dirichlet_values=bc_vals[nbc[dn] - 1], y=y, ac=ac)
    print(out, "nodes", nn, "tets", ne, "boundary", nb, "dirichlet", len(dn))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
