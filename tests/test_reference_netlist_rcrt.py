"""CPU: the reference's legacy/netlistWithRCRTs case (its test
checkMixedNetlistAndRCRT, flowsolver/test/testMain.cxx:362-420): the
closedLoopHeart mesh and restart state (the case ships the same
geombc.dat.1 and restart.0.1), a heart circuit without valves on surface
5 (LV chamber under the built-in elastance control) and RCR outlets 6, 7
from rcrt.dat, five first-order steps with memLS and residual control.  The
RCRs start from their surfaces' initial mean pressure and flow
(callCPPSetPressureFromFortran, itrdrv.f90:748-760).  Inputs:
tests/golden/case_inputs.json (solver.inp, rcrt.dat, netlist_surfaces.xml)
read with crimsonflowsolver_b200.case; the oracle's time stepper checked
against the values the reference's test asserts."""
import json
import os

import numpy as np
import pytest

from crimsonflowsolver_b200 import case
from crimsonflowsolver_b200 import netlist_io as nio
from oracle import pyoracle as po
from tests.fixtures import closed_loop_heart_mesh

HERE = os.path.dirname(os.path.abspath(__file__))
# FlowHist.dat / PressHist.dat row 6 (after step 5) for surfaces 5, 6, 7;
# netlistPressures_surface_5.dat row 5 (after step 4), node 1
GOLD_Q = {5: 137208.420657606, 6: -97144.4580441544, 7: -40084.8691875509}
GOLD_P = {5: 790.498746283900, 6: 7653.31439101382, 7: 9376.67945078140}
GOLD_NODE1_STEP4 = 798.293386775323


def rcrt_case():
    """(mesh, y, ac, settings, netlists, rcr) of the case."""
    with open(os.path.join(HERE, "golden", "case_inputs.json")) as f:
        t = json.load(f)["legacy/netlistWithRCRTs"]
    s = case.parse_solver_inp(t["solver.inp"])
    netlists = [nio.to_netlistbc(c, srf) for c, srf in
                zip(nio.parse_netlist_xml(t["netlist_surfaces.xml"]),
                    [int(v) for v in s["list of netlist lpn surfaces"].split()])]
    rcr = case.parse_rcrt(t["rcrt.dat"], [int(v) for v in s["list of experimental rcr surfaces"].split()])
    m, y, ac = closed_loop_heart_mesh()
    return m, y, ac, s, netlists, rcr


def run_oracle(steps=5):
    m, y, ac, s, netlists, rcr = rcrt_case()
    F = po.OracleFlow(m, case.flow_params(s, rcr=rcr, netlists=netlists), nthreads=4)
    F.yold, F.acold = y.copy(), ac.copy()
    F._itr_bc(F.yold)
    q0 = po.getflowq(F.m, F.yold, F.srflist)
    for j, r in enumerate(F.rcr):
        if not hasattr(r, "components"):
            w = F.nasc[F.pnodes[j]]
            F.Pn[j] = float(np.sum(w * F.yold[F.pnodes[j], 3]) / np.sum(w))
            F.Qn[j] = q0[j]
    hist = []
    for _ in range(steps):
        F.step()
        p = {}
        for j, srf in enumerate(F.srflist):
            w = F.nasc[F.pnodes[j]]
            p[srf] = float(np.sum(w * F.yold[F.pnodes[j], 3]) / np.sum(w))
        hist.append({"Q": dict(zip(F.srflist, F.Qn)), "p": p,
                     "node1": float(F.netlists[F.srflist.index(5)].pressure(1))})
    return F, hist


@pytest.fixture(scope="module")
def oracle_run():
    return run_oracle()


def test_inputs():
    m, y, ac, s, netlists, rcr = rcrt_case()
    assert [(r.srfid, r.Rp, r.C, r.Rd, r.Pd) for r in rcr] == [(6, 0.03, 5.74, 0.3, 0.0), (7, 0.03, 5.74, 0.3, 0.0)]
    assert [n.srfid for n in netlists] == [5] and netlists[0].controllers
    with pytest.raises(NotImplementedError):
        case.parse_rcrt("2 2 1 2 3 0 0 1 5", [6])        # time-varying distal pressure
    with pytest.raises(NotImplementedError):
        case.flow_params(s, netlists=netlists)              # the RCR surfaces not given


def test_reference_values(oracle_run):
    """Flows after step 5 within 1e-6 relative (measured 4e-8, 2e-8, 1e-7),
    surface mean pressures within 2e-7 (1.4e-8, 2.7e-8, 5.2e-8), the heart
    circuit's node-1 pressure after step 4 within 1e-7 (1.2e-8)."""
    _, hist = oracle_run
    for srf in (5, 6, 7):
        assert abs(hist[4]["Q"][srf] - GOLD_Q[srf]) <= 1e-6 * abs(GOLD_Q[srf]), (srf, hist[4]["Q"][srf])
        assert abs(hist[4]["p"][srf] - GOLD_P[srf]) <= 2e-7 * abs(GOLD_P[srf]), (srf, hist[4]["p"][srf])
    assert abs(hist[3]["node1"] - GOLD_NODE1_STEP4) <= 1e-7 * GOLD_NODE1_STEP4
