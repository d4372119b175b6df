"""The reference's own test mesh (testbin/mainTests/basic: 1072 nodes, 4157
tets, 1092 boundary faces, PHASTA restart state) as a Mesh, from the
committed fixture tests/golden/basic_mesh.npz (see make_phasta_fixture.py)."""
import os

import numpy as np

from crimsonflowsolver_b200 import mesh as meshmod

HERE = os.path.dirname(os.path.abspath(__file__))


def basic_mesh():
    return _load("basic_mesh.npz", "reference basic")


def closed_loop_heart_mesh():
    """The mesh and restart state of the reference's netlist/closedLoopHeart
    case (4205 nodes, 18022 tets, netlist surfaces 5, 6, 7)."""
    return _load("closed_loop_heart_mesh.npz", "reference closedLoopHeart")


def _load(name, label):
    d = np.load(os.path.join(HERE, "golden", name))
    m = meshmod.Mesh(x=d["x"].copy(), ien=d["ien"].copy(), name=label)
    m.ienb = d["ienb"].copy()
    m.iBCB = d["iBCB"].copy()
    m.BCB = np.repeat(d["BCB"][:, None, :], 3, axis=1).copy()   # per face node
    m.iBC = d["iBC"].copy()
    m.dirichlet_nodes = d["dirichlet_nodes"].copy()
    m.dirichlet_values = d["dirichlet_values"].copy()
    m.BC = np.zeros((m.nshg, meshmod.NDOFBC))
    m.NABI, m.ndsurf = meshmod.compute_nabi(m.x, m.ienb, m.iBCB, m.nshg)
    m.outlets = sorted(int(s) for s in np.unique(m.iBCB[:, 1]) if s >= meshmod.SRF_OUTLET0)
    return m, d["y"].copy(), d["ac"].copy()


# The reference's test checkClosedLoopWithHeart (flowsolver/test/testMain.cxx:
# 266-345) runs testbin/mainTests/netlist/closedLoopHeart for five steps and
# checks these values.  FlowHist.dat / PressHist.dat row 6 is the state after
# step 5 (row 1 holds the initial state); the netlist files' row 5 is the
# circuits' state after step 4.
CLOSED_LOOP_HEART_GOLDEN = {
    "flow_step5": (-307.419802901504, 270.813353397073, 37.8070383450010),
    "pressure_step5": (553.277617338762, 548.211423767513, 541.282726604241),
    "heart_interface_flow_step4": -287.802631760359,
    "downstream_pressures_step4": (533.100216837156, 533.100216837156, 0.0, 535.821025669528),
    "downstream_flows_step4": (0.0, 27.2080883237159, -27.2080883237159),
}


def closed_loop_heart_case():
    """(mesh, y, ac, FlowParams) of the closedLoopHeart case: its solver.inp
    (density 0.00106, viscosity 0.004, Delt 1e-3, first-order time
    integration, "0 1" x 5 = five solve/update pairs, influx coefficient
    0.5, residual control at 1e-3 after at least 2 iterations, memLS) with configs/input.config's memLS defaults (Kspace 50,
    nGMRES 1, maxIters 200, nPrjs 10, epstol 0.01 / 0.2 / 0.4), and its
    netlist inputs: surfaces 5, 6, 7 joined by the loop-closing circuit, the
    heart's LV elastance control bound.  The loop is built afresh on every
    call (controllers keep state)."""
    import json

    from crimsonflowsolver_b200 import FlowParams
    from crimsonflowsolver_b200 import netlist_io as nio

    m, y, ac = closed_loop_heart_mesh()
    with open(os.path.join(HERE, "golden", "netlist_closed_loops.json")) as f:
        v = json.load(f)["netlist/closedLoopHeart"]
    _, loops = nio.closed_loops(nio.parse_netlist_xml(v["surfaces"]), v["srfids"],
                                nio.parse_netlist_xml(v["downstream"]))
    P = FlowParams(rho=0.00106, mu=0.004, rhoinf=-1.0, Delt=1e-3, nitr=5, epstol_mom=0.01, epstol_cont=0.2,
                   epstol_ns=0.4, kspace=50, ngmres=1, maxiters=200, nprjs=10, stabflux_coeff=0.5, loops=loops,
                   rescontrol=True, res_criteria=1e-3, min_iters=2)
    return m, y, ac, P
