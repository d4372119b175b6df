"""Build tests/golden/basic_mesh.npz from the reference's own test case
testbin/mainTests/basic (geombc.dat.1 + restart.0.1, PHASTA format), with
the package's PHASTA reader.  Run once where a reference checkout exists:

    python tests/golden/make_phasta_fixture.py /path/to/reference
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from crimsonflowsolver_b200 import phasta  # noqa: E402


def main(ref):
    base = os.path.join(ref, "testbin", "mainTests", "basic")
    m = phasta.read_geombc(os.path.join(base, "geombc.dat.1"))
    y, ac, _ = phasta.read_restart(os.path.join(base, "restart.0.1"))
    out = os.path.join(HERE, "basic_mesh.npz")
    np.savez_compressed(out, x=m.x, ien=m.ien, ienb=m.ienb, iBCB=m.iBCB, BCB=m.BCB[:, 0, :], iBC=m.iBC,
                        dirichlet_nodes=m.dirichlet_nodes, dirichlet_values=m.dirichlet_values, y=y, ac=ac)
    print(out, "nodes", m.nshg, "tets", m.nelem, "boundary", len(m.ienb), "dirichlet", len(m.dirichlet_nodes))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
