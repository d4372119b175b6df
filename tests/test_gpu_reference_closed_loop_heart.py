"""GPU: the reference's closedLoopHeart case (testbin/mainTests/netlist/
closedLoopHeart; flowsolver/test/testMain.cxx:266-345) through the device
time step (FlowSolver: crimson_step with the closed loop coupled by
crimson_set_outlet_netlist_loop), against the oracle's time stepper step by
step -- the design of each surface, memLS iteration counts, outlet flows and
pressures, and at the end velocity and pressure within 1e-9 -- and against
the values the reference's test asserts, with the bars of
tests/test_reference_closed_loop_heart.py."""
import numpy as np
import pytest

from crimsonflowsolver_b200 import solver
from oracle import pyoracle as po
from tests.conftest import relerr
from tests.fixtures import CLOSED_LOOP_HEART_GOLDEN as GOLD
from tests.fixtures import closed_loop_heart_case
from tests.test_reference_closed_loop_heart import run_oracle

pytestmark = pytest.mark.gpu


def test_closed_loop_heart_case_on_device():
    F, hist = run_oracle()
    m, y, ac, P = closed_loop_heart_case()
    y0 = y.copy()
    po.itr_bc(m, y0)
    G = solver.FlowSolver(m, P, inflow=lambda t: 0.0)
    nasc = po.surface_areas(m)
    onodes = [po.pressure_nodes(m, s) for s in (5, 6, 7)]
    try:
        G.set_state(y0, ac)
        for k in range(5):
            assert G.loops[0].flow_permitted() == hist[k]["permitted"], k
            st = G.step()
            for j in range(3):
                assert abs(st.q_out[j] - hist[k]["Q"][j]) <= 1e-9 * max(1.0, abs(hist[k]["Q"][j])), (k, j)
            yk, _ = G.state()
            p = np.array([np.sum(nasc[o] * yk[o, 3]) / np.sum(nasc[o]) for o in onodes])
            assert np.all(np.abs(p - hist[k]["p"]) <= 1e-9 * np.abs(hist[k]["p"])), (k, p, hist[k]["p"])
            down = G.loops[0].downstream.get()[0]
            assert np.abs(down - hist[k]["down_p"]).max() <= 1e-9 * np.abs(hist[k]["down_p"]).max(), k
        yG, _ = G.state()
    finally:
        G.close()
    assert relerr(yG[:, 0:3], F.yold[:, 0:3]) < 1e-9, relerr(yG[:, 0:3], F.yold[:, 0:3])
    assert relerr(yG[:, 3], F.yold[:, 3]) < 1e-9, relerr(yG[:, 3], F.yold[:, 3])
    gold_q, gold_p = np.array(GOLD["flow_step5"]), np.array(GOLD["pressure_step5"])
    assert np.all(np.abs(np.array([st.q_out[j] for j in range(3)]) - gold_q) <= 2e-5 * np.abs(gold_q))
    assert np.all(np.abs(p - gold_p) <= 5e-8 * np.abs(gold_p))


def test_residual_control_on_device():
    """Residual control firing (criterion 5, at least two iterations): the
    device step's totres per assembled iteration, its number of solves per
    step and the state after three steps match the oracle's."""
    import dataclasses

    m, y, ac, P = closed_loop_heart_case()
    P = dataclasses.replace(P, res_criteria=5.0)
    F = po.OracleFlow(m, P, nthreads=4)
    F.yold, F.acold = y.copy(), ac.copy()
    F._itr_bc(F.yold)
    m2, _, _, P2 = closed_loop_heart_case()
    G = solver.FlowSolver(m2, dataclasses.replace(P2, res_criteria=5.0), inflow=lambda t: 0.0)
    y0 = y.copy()
    po.itr_bc(m2, y0)
    try:
        G.set_state(y0, ac)
        for k in range(3):
            n0, r0 = len(F.stats), len(F.res_norms)
            F.step()
            st = G.step()
            assert st.nsolves == len(F.stats) - n0, k
            norms = F.res_norms[r0:]
            for i, v in enumerate(norms):
                assert abs(st.res_norm[i] - v) <= 1e-9 * v, (k, i, st.res_norm[i], v)
        yG, _ = G.state()
    finally:
        G.close()
    assert relerr(yG, F.yold) < 1e-9


def test_case_driver_runs_the_reference_case(tmp_path):
    """crimsonflowsolver_b200.case.Case with closedLoopHeart's own solver.inp
    (parsed, input.config defaults) and netlist inputs: five steps on the
    device, the FlowHist.dat / PressHist.dat rows (initial state + 5 steps,
    from crimson_outlet_state) against the reference test's values."""
    import json
    import os

    from crimsonflowsolver_b200 import case

    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "netlist_closed_loops.json")) as f:
        inp = json.load(f)["netlist/closedLoopHeart"]["solver_inp"]
    m, y, ac, ref = closed_loop_heart_case()
    c = case.Case(case.parse_solver_inp(inp), m, y, ac, loops=ref.loops)
    h = c.run(out_dir=str(tmp_path))
    assert h["flow"].shape == (6, 3) and h["pressure"].shape == (6, 3)
    gold_q, gold_p = np.array(GOLD["flow_step5"]), np.array(GOLD["pressure_step5"])
    assert np.all(np.abs(h["flow"][5] - gold_q) <= 2e-5 * np.abs(gold_q)), h["flow"][5]
    assert np.all(np.abs(h["pressure"][5] - gold_p) <= 5e-8 * np.abs(gold_p)), h["pressure"][5]
    assert abs(h["pressure"][0][0] - 10664.0) < 1e-6   # the restart's uniform pressure
    rows = open(tmp_path / "PressHist.dat").read().split("\n")
    assert int(rows[0]) == 6 and len(rows[6].split()) == 3


def test_case_driver_runs_the_rcrt_case():
    """legacy/netlistWithRCRTs through crimsonflowsolver_b200.case.Case (RCR
    outlets from rcrt.dat starting from the initial surface state, the heart
    circuit on surface 5): five device steps against the oracle's run and the
    reference test's values, with the bars of
    tests/test_reference_netlist_rcrt.py."""
    from crimsonflowsolver_b200 import case
    from tests import test_reference_netlist_rcrt as T

    _, hist = T.run_oracle()
    m, y, ac, s, netlists, rcr = T.rcrt_case()
    c = case.Case(s, m, y, ac, netlists=netlists, rcr=rcr)
    h = c.run()
    order = [o.srfid for o in c.P.outlets()]
    for j, srf in enumerate(order):
        for k in range(5):
            assert abs(h["flow"][k + 1][j] - hist[k]["Q"][srf]) <= 1e-9 * abs(hist[k]["Q"][srf]), (k, srf)
            assert abs(h["pressure"][k + 1][j] - hist[k]["p"][srf]) <= 1e-9 * abs(hist[k]["p"][srf]), (k, srf)
        assert abs(h["flow"][5][j] - T.GOLD_Q[srf]) <= 1e-6 * abs(T.GOLD_Q[srf])
        assert abs(h["pressure"][5][j] - T.GOLD_P[srf]) <= 2e-7 * abs(T.GOLD_P[srf])
