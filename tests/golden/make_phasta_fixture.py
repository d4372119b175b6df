"""Build the PHASTA fixtures from the reference's own test cases
testbin/mainTests/basic, netlist/closedLoopHeart and legacy/netlistWithRCRTs
(geombc.dat.1 + restart.0.1), with the package's PHASTA reader.  Run once
where a reference checkout exists:

    python tests/golden/make_phasta_fixture.py /path/to/reference/checkout

Writes
  basic_mesh.npz      the arrays this path reads (coordinates, connectivity,
                      boundary codes/values, Dirichlet codes, restart state);
  basic_headers.json  the text lines (comments and block headers, no binary
                      data) of both files, so the reader and the writer can
                      be checked against the reference's header grammar and
                      block sizes without the reference checkout;
  closed_loop_heart_mesh.npz  the same arrays for the closedLoopHeart case
                      (4205 nodes, 18022 tets; outlets 5, 6, 7 coupled
                      through netlist circuits and a closed loop);
  case_inputs.json    the solver.inp, rcrt.dat and netlist_surfaces.xml of
                      closedLoopHeart and of legacy/netlistWithRCRTs (a
                      heart circuit on surface 5, RCR outlets 6 and 7, on
                      the same mesh and restart state).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from crimsonflowsolver_b200 import phasta  # noqa: E402


def main(ref):
    base = os.path.join(ref, "testbin", "mainTests", "basic")
    geo, rst = os.path.join(base, "geombc.dat.1"), os.path.join(base, "restart.0.1")
    m = phasta.read_geombc(geo)
    y, ac, _ = phasta.read_restart(rst)
    out = os.path.join(HERE, "basic_mesh.npz")
    np.savez_compressed(out, x=m.x, ien=m.ien, ienb=m.ienb, iBCB=m.iBCB, BCB=m.BCB[:, 0, :], iBC=m.iBC,
                        dirichlet_nodes=m.dirichlet_nodes, dirichlet_values=m.dirichlet_values, y=y, ac=ac)
    heads = {"geombc.dat.1": phasta.header_lines(geo), "restart.0.1": phasta.header_lines(rst)}
    with open(os.path.join(HERE, "basic_headers.json"), "w") as f:
        json.dump(heads, f, indent=1)
    print(out, "nodes", m.nshg, "tets", m.nelem, "boundary", len(m.ienb), "dirichlet", len(m.dirichlet_nodes))
    texts = {}
    # legacy/netlistWithRCRTs runs on the same geombc.dat.1 and restart.0.1
    for case, name in (("netlist/closedLoopHeart", "closed_loop_heart_mesh.npz"),
                       ("legacy/netlistWithRCRTs", None)):
        base = os.path.join(ref, "testbin", "mainTests", *case.split("/"))
        m = phasta.read_geombc(os.path.join(base, "geombc.dat.1"))
        y, ac, _ = phasta.read_restart(os.path.join(base, "restart.0.1"))
        texts[case] = {}
        if name is not None:
            out = os.path.join(HERE, name)
            np.savez_compressed(out, x=m.x, ien=m.ien, ienb=m.ienb, iBCB=m.iBCB, BCB=m.BCB[:, 0, :], iBC=m.iBC,
                                dirichlet_nodes=m.dirichlet_nodes, dirichlet_values=m.dirichlet_values, y=y,
                                ac=ac)
        for f in ("solver.inp", "rcrt.dat", "netlist_surfaces.xml"):
            if os.path.exists(os.path.join(base, f)):
                with open(os.path.join(base, f)) as fh:
                    texts[case][f] = fh.read()
    with open(os.path.join(HERE, "case_inputs.json"), "w") as f:
        json.dump(texts, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_phasta_fixture.py /path/to/reference/checkout")
    main(sys.argv[1])
