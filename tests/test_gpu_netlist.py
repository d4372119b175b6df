"""Netlist outlets in the device time step (crimson_set_outlet_netlist) against
the oracle's time stepper with the same circuit (OracleFlow +
oracle/netlist_oracle.py), closed loops of circuits
(crimson_set_outlet_netlist_loop) likewise, and the Windkessel written as a
netlist against the built-in RCR outlet.  Parity bar as for the RCR time steps: velocity,
pressure and outlet pressure within 1e-10, identical iteration counts."""
import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, NetlistBC, NetlistLoopBC, RCR, mesh, solver
from oracle import pyoracle as po
from tests.conftest import relerr

pytestmark = pytest.mark.gpu


def _inflow(t):
    return 10.0 + 5.0 * np.sin(2 * np.pi * t / 0.8)


def test_rcr_netlist_matches_rcr_outlet():
    """The circuit 1 -Rp- 2, 2 -C- ground, 2 -Rd- Pd coupled through the
    netlist path gives the RCR outlet's steps (coefficients equal to
    rounding)."""
    Pr = FlowParams(rcr=[RCR(srfid=3, Rp=100.0, C=1e-4, Rd=1000.0, Pd=0.0)])
    Pn = FlowParams(netlists=[NetlistBC.rcr(3, Rp=100.0, C=1e-4, Rd=1000.0, Pd=0.0)])
    A = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10), Pr, inflow=_inflow)
    B = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10), Pn, inflow=_inflow)
    try:
        for _ in range(3):
            sa = A.step()
            sb = B.step()
            assert [sa.cg_itr[i] for i in range(sa.nsolves)] == [sb.cg_itr[i] for i in range(sb.nsolves)]
        ya, _ = A.state()
        yb, _ = B.state()
    finally:
        A.close()
        B.close()
    assert relerr(yb, ya) < 1e-10, relerr(yb, ya)
    assert abs(sb.p_out[0] - sa.p_out[0]) <= 1e-10 * abs(sa.p_out[0])
    assert abs(sb.q_out[0] - sa.q_out[0]) <= 1e-10 * abs(sa.q_out[0])


def _circuit():
    # proximal resistance and inertance, a compliance, a diode-guarded
    # compliant branch and a distal resistance to a venous pressure
    return NetlistBC(srfid=3, components=[("r", 1, 2, 80.0), ("l", 2, 3, 2.0), ("c", 3, 4, 1.5e-4),
                                          ("d", 3, 5, 10.0), ("c", 5, 6, 5e-5), ("r", 3, 7, 900.0)],
                     prescribed_pressures={4: 0.0, 6: 0.0, 7: 5.0}, interface_component=1,
                     initial_pressures={2: 5.0, 3: 5.0, 5: 0.0})


def test_netlist_time_steps_parity():
    """Three steps with a five-element circuit (inductor, two capacitors, a
    diode) on the outlet, device vs oracle."""
    P = FlowParams(netlists=[_circuit()])
    F = po.OracleFlow(mesh.cylinder(ncross=8, naxial=10), P, inflow=_inflow)
    G = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10), P, inflow=_inflow)
    try:
        for _ in range(3):
            F.step()
            st = G.step()
        y, _ = G.state()
        p, q, op, _ = G.netlists[0].get()
    finally:
        G.close()
    its = [(r, g, c) for r, g, c, _, _ in F.stats[-st.nsolves:]]
    assert its == [(st.ri_itr[i], st.gm_itr[i], st.cg_itr[i]) for i in range(st.nsolves)]
    assert relerr(y[:, 0:3], F.y[:, 0:3]) < 1e-10, relerr(y[:, 0:3], F.y[:, 0:3])
    assert relerr(y[:, 3], F.y[:, 3]) < 1e-10, relerr(y[:, 3], F.y[:, 3])
    o = F.netlists[0]
    assert abs(st.p_out[0] - F.Pn[0]) <= 1e-10 * abs(F.Pn[0])
    assert relerr(p, [o.pressure(i + 1) for i in range(len(p))]) < 1e-10
    assert relerr(q, o.q) < 1e-10
    assert list(op) == list(o.open)


def test_valve_switches_surface_between_dirichlet_and_neumann():
    """A diode on the only path from a netlist outlet (the circuit of the
    reference's simpleDiodeTest case, a second outlet with an RCR): the
    valve starts closed, so the surface starts at its Dirichlet codes and
    the circuit takes the 3D surface pressure; it opens, closes under
    backflow and opens again within six steps.  Device vs oracle: the
    design of every step, velocity and pressure within 1e-10, outlet
    pressures and flows, identical iteration counts."""
    m = mesh.cylinder(ncross=8, naxial=10, n_outlets=2)
    spec = NetlistBC(srfid=m.outlets[1], components=[("r", 1, 2, 1.0), ("d", 2, 3, 0.1)],
                     prescribed_pressures={3: 1250.0}, interface_component=1,
                     initial_pressures={1: 1058.5, 2: 1058.5, 3: 1250.0})
    P = FlowParams(rcr=[RCR(srfid=m.outlets[0])], netlists=[spec], nitr=2)
    F = po.OracleFlow(mesh.cylinder(ncross=8, naxial=10, n_outlets=2), P, inflow=lambda t: 10.0)
    G = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10, n_outlets=2), P, inflow=lambda t: 10.0)
    modes = ""
    try:
        for _ in range(6):
            modes += "N" if F.netlists[1].permitted else "D"
            assert G.netlists[0].flow_permitted() == F.netlists[1].permitted
            F.step()
            st = G.step()
            its = [(r, g, c) for r, g, c, _, _ in F.stats[-st.nsolves:]]
            assert its == [(st.ri_itr[i], st.gm_itr[i], st.cg_itr[i]) for i in range(st.nsolves)]
            for k in range(2):
                assert abs(st.p_out[k] - F.Pn[k]) <= 1e-9 * abs(F.Pn[k]), (k, st.p_out[k], F.Pn[k])
                assert abs(st.q_out[k] - F.Qn[k]) <= 1e-9 * max(1.0, abs(F.Qn[k])), (k, st.q_out[k], F.Qn[k])
        y, _ = G.state()
        p, q, op, _ = G.netlists[0].get()
    finally:
        G.close()
    assert "DN" in modes and "ND" in modes, modes
    assert relerr(y[:, 0:3], F.y[:, 0:3]) < 1e-10, relerr(y[:, 0:3], F.y[:, 0:3])
    assert relerr(y[:, 3], F.y[:, 3]) < 1e-10, relerr(y[:, 3], F.y[:, 3])
    o = F.netlists[1]
    assert relerr(p, [o.pressure(i + 1) for i in range(len(p))]) < 1e-10
    assert list(op) == list(o.open)


def test_controllers_in_time_steps_parity():
    """Control systems between steps (itrdrv.f90:2100): a sensor controller
    publishes a signal from the outlet pressure and a second one scales the
    distal resistance by it.  Four steps, device vs oracle (each with its
    own controller instances): state, outlet pressure and the controlled
    resistance."""
    from crimsonflowsolver_b200.controllers import ParameterController

    class Sensor(ParameterController):
        controllerPriority = 1

        def updateControl(self, value, delt, pressures, flows, volumes):
            self.clearBroadcastData()
            self.addBroadcastVariable("signal", 1.0 + 1e-4 * pressures[1])
            return value

    class Distal(ParameterController):
        controllerPriority = 2

        def __init__(self, name):
            super().__init__(name)
            self.base = None

        def updateControl(self, value, delt, pressures, flows, volumes):
            self.base = value if self.base is None else self.base
            return self.base * self.getRecievedBroadcastValue("sensor", "signal")

    def spec():
        s = NetlistBC.rcr(3, Rp=100.0, C=1e-4, Rd=1000.0, Pd=0.0)
        s.controllers = [("component", 3, Distal("distal")), ("pressure", 1, Sensor("sensor"))]
        return s

    Pg, Po = FlowParams(netlists=[spec()]), FlowParams(netlists=[spec()])
    F = po.OracleFlow(mesh.cylinder(ncross=8, naxial=10), Po, inflow=_inflow)
    G = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10), Pg, inflow=_inflow)
    try:
        for _ in range(4):
            F.step()
            st = G.step()
            assert abs(st.p_out[0] - F.Pn[0]) <= 1e-10 * abs(F.Pn[0])
            rg = G.netlists[0].get_parameter("component", 3)
            ro = F.netlists[0].get_parameter("component", 3)
            assert abs(rg - ro) <= 1e-10 * abs(ro) and rg != 1000.0
        y, _ = G.state()
    finally:
        G.close()
    assert relerr(y[:, 0:3], F.y[:, 0:3]) < 1e-10, relerr(y[:, 0:3], F.y[:, 0:3])
    assert relerr(y[:, 3], F.y[:, 3]) < 1e-10, relerr(y[:, 3], F.y[:, 3])


def _loop(m):
    """Two outlets joined by a loop-closing circuit: outlet 1 through an
    RC branch, outlet 2 through a valve (the simpleDiodeTest circuit, which
    starts closed), both ending at node 1 of a circuit that drains through a
    compliance and a resistance to a venous pressure."""
    s0, s1 = m.outlets
    a = NetlistBC(srfid=s0, components=[("r", 1, 2, 60.0), ("c", 2, 3, 1e-4), ("r", 2, 4, 400.0)],
                  prescribed_pressures={3: 0.0}, interface_component=1, initial_pressures={2: 5.0, 4: 5.0},
                  shared_nodes=(4,))
    b = NetlistBC(srfid=s1, components=[("r", 1, 2, 1.0), ("d", 2, 3, 0.1)], interface_component=1,
                  initial_pressures={1: 1058.5, 2: 1058.5, 3: 1000.0}, shared_nodes=(3,))
    d = NetlistBC(srfid=0, components=[("r", 1, 2, 300.0), ("c", 1, 3, 5e-4), ("r", 2, 4, 10.0)],
                  prescribed_pressures={3: 0.0, 4: 1250.0}, interface_component=0,
                  initial_pressures={1: 5.0, 2: 1200.0}, shared_nodes=(1,))
    return NetlistLoopBC(upstream=[a, b], downstream=d, connections=[(1, s0, 4), (1, s1, 3)])


def test_closed_loop_time_steps_parity():
    """A closed loop over both outlets (crimson_set_outlet_netlist_loop):
    one loop solve gives both surfaces' coefficients, the valved outlet
    switches between the Dirichlet and the Neumann design, and every step's
    designs, iteration counts, outlet pressures and flows, and at the end
    velocity, pressure and every member's state match the oracle's time
    stepper (OracleFlow with OracleLoop)."""
    m = mesh.cylinder(ncross=8, naxial=10, n_outlets=2)
    P = FlowParams(loops=[_loop(m)], nitr=2)
    F = po.OracleFlow(mesh.cylinder(ncross=8, naxial=10, n_outlets=2), P, inflow=lambda t: 10.0)
    G = solver.FlowSolver(mesh.cylinder(ncross=8, naxial=10, n_outlets=2), P, inflow=lambda t: 10.0)
    modes = ""
    try:
        for _ in range(6):
            designs = [u.permitted for u in F.loops[0].up]
            assert G.loops[0].flow_permitted() == designs
            modes += "".join("N" if x else "D" for x in designs) + " "
            F.step()
            st = G.step()
            its = [(r, g, c) for r, g, c, _, _ in F.stats[-st.nsolves:]]
            assert its == [(st.ri_itr[i], st.gm_itr[i], st.cg_itr[i]) for i in range(st.nsolves)]
            for k in range(2):
                assert abs(st.p_out[k] - F.Pn[k]) <= 1e-9 * abs(F.Pn[k]), (k, st.p_out[k], F.Pn[k])
                assert abs(st.q_out[k] - F.Qn[k]) <= 1e-9 * max(1.0, abs(F.Qn[k])), (k, st.q_out[k], F.Qn[k])
        y, _ = G.state()
        members = [mm.get() for mm in G.loops[0].members]
    finally:
        G.close()
    assert "ND" in modes and "NN" in modes, modes
    assert relerr(y[:, 0:3], F.y[:, 0:3]) < 1e-10, relerr(y[:, 0:3], F.y[:, 0:3])
    assert relerr(y[:, 3], F.y[:, 3]) < 1e-10, relerr(y[:, 3], F.y[:, 3])
    for (p, q, op, _), o in zip(members, F.loops[0].members):
        assert relerr(p, [o.pressure(i + 1) for i in range(len(p))]) < 1e-10
        assert relerr(q, o.q) < 1e-10
        assert list(op) == list(o.open)
