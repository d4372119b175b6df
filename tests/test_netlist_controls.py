"""Netlist control systems (CPU): the parameter calls of the library
(crimson_netlist_get/set_parameter) and the per-step controller driver
(crimsonflowsolver_b200.controllers) against the oracle restatement, and the
control declarations of the reference's own netlist inputs."""
import numpy as np
import pytest

from crimsonflowsolver_b200 import NetlistBC, netlist_io as nio
from crimsonflowsolver_b200.controllers import ParameterController, run_controllers
from crimsonflowsolver_b200.netlist import Netlist
from oracle.netlist_oracle import OracleNetlist
from oracle.netlist_oracle import run_controllers as oracle_run_controllers
from tests.test_netlist_io import _inputs, _parse

ALFI, DT = 0.5, 1e-3


def _close(a, b, tol):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max())


def _circuit(controllers=()):
    # interface resistor, a valve into a pressure chamber, a compliance, a
    # distal resistance to a controlled venous pressure, a fixed side flow
    return NetlistBC(srfid=3, components=[("r", 1, 2, 50.0), ("d", 2, 3, 5.0), ("v", 3, 4, 2000.0),
                                          ("c", 2, 5, 1e-4), ("r", 2, 6, 900.0), ("r", 2, 7, 4000.0)],
                     prescribed_pressures={4: 0.0, 5: 0.0, 6: 10.0}, prescribed_flows={6: 0.5},
                     interface_component=1, initial_pressures={2: 10.0, 3: 10.0},
                     volumes={3: (8.0, 2.0)}, controllers=list(controllers))


def test_parameters_match_oracle():
    g, o = Netlist(_circuit()), OracleNetlist(_circuit())
    cases = [("component", 5, 1200.0), ("component", 3, 2500.0), ("unstressed_volume", 3, 1.5),
             ("pressure", 6, 12.0), ("pressure", 2, 33.0), ("flow", 6, 0.25)]
    for target, index, value in cases:
        assert g.get_parameter(target, index) == pytest.approx(o.get_parameter(target, index))
        g.set_parameter(target, index, value)
        o.set_parameter(target, index, value)
        assert g.get_parameter(target, index) == value == o.get_parameter(target, index)
    for bad in [("unstressed_volume", 1), ("flow", 1), ("component", 7), ("pressure", 8)]:
        with pytest.raises((RuntimeError, KeyError, AssertionError)):
            g.get_parameter(*bad)
    with pytest.raises(RuntimeError):
        g.set_parameter("component", 4, 0.0)  # a capacitance of 0
    for step in range(6):
        assert g.flow_permitted() == o.permitted
        if o.permitted:
            assert _close(g.implicit_coefficients(ALFI * DT), o.implicit_coefficients(ALFI * DT), 1e-10)
            g.update(DT, 40.0 + 10.0 * step)
            o.update(DT, 40.0 + 10.0 * step)
        else:
            g.update_pressure(DT, 200.0)
            o.update_pressure(DT, 200.0)
        p, q, _, v = g.get()
        assert _close(p, [o.pressure(i + 1) for i in range(len(p))], 1e-10)
        assert _close(q, o.q, 1e-10)
        assert _close(v[2], o.vol[2], 1e-10)
        g.finalize_step()
        o.finalize_step()
    g.close()


class PressureSensor(ParameterController):
    """Publishes a signal from the interface pressure; controls nothing of
    its own (returns the node pressure it observes)."""
    controllerPriority = 1

    def updateControl(self, value, delt, pressures, flows, volumes):
        self.clearBroadcastData()
        self.addBroadcastVariable("signal", 1.0 + 0.01 * (pressures[1] - 40.0))
        return value


class DistalResistance(ParameterController):
    """Scales the distal resistance by the sensor's signal, relative to the
    value it first saw."""
    controllerPriority = 2

    def __init__(self, name):
        super().__init__(name)
        self.baseline = None

    def updateControl(self, value, delt, pressures, flows, volumes):
        if self.baseline is None:
            self.baseline = value
        return self.baseline * self.getRecievedBroadcastValue("sensor", "signal")


class VenousPressure(ParameterController):
    """Drives the prescribed venous pressure from the chamber volume."""
    controllerPriority = 3

    def updateControl(self, value, delt, pressures, flows, volumes):
        return 5.0 + 0.5 * volumes[3]


def _controlled():
    # listed out of priority order on purpose: the driver sorts them
    return [("component", 5, DistalResistance("distal")), ("pressure", 1, PressureSensor("sensor")),
            ("pressure", 6, VenousPressure("venous"))]


def test_controllers_drive_library_and_oracle_alike():
    gspec, ospec = _circuit(_controlled()), _circuit(_controlled())
    g, o = Netlist(gspec), OracleNetlist(ospec)
    g_bound = [(g, t, i, c) for t, i, c in gspec.controllers]
    o_bound = [(o, t, i, c) for t, i, c in ospec.controllers]
    r5 = []
    for step in range(10):
        q = 40.0 + 30.0 * np.sin(2 * np.pi * step / 10)
        if o.permitted:
            assert _close(g.implicit_coefficients(ALFI * DT), o.implicit_coefficients(ALFI * DT), 1e-10)
            g.update(DT, q)
            o.update(DT, q)
        else:
            g.update_pressure(DT, 10.0 * q)
            o.update_pressure(DT, 10.0 * q)
        g.finalize_step()
        o.finalize_step()
        run_controllers(g_bound, DT)
        oracle_run_controllers(o_bound, DT)
        p, f, _, _ = g.get()
        assert _close(p, [o.pressure(i + 1) for i in range(len(p))], 1e-10)
        assert _close(f, o.q, 1e-10)
        for t, i, _ in gspec.controllers:
            assert g.get_parameter(t, i) == pytest.approx(o.get_parameter(t, i), rel=1e-12)
        r5.append(g.get_parameter("component", 5))
    # the distal resistance followed the sensor, the venous pressure the volume
    assert len(set(np.round(r5, 9))) > 3
    assert g.get_parameter("pressure", 6) != 10.0
    g.close()


def test_reference_control_declarations_parse_and_bind():
    """The customPython controls of the reference's baroreflex case (the
    .dat's coronary circuit: two component controllers and a node
    controller) bind to user controllers, the built-in LV elastance control
    to its built-in controller; a file-driven prescription given neither its
    table's directory nor a controller raises."""
    coronary = _parse("x.dat", _inputs()["netlist/baroreflexPython/netlist_surfaces.dat"])[1]
    assert coronary["control_specs"] == [("component", 3, "customPython", "coronaryRpController"),
                                         ("component", 5, "customPython", "coronaryRdController"),
                                         ("node", 5, "customPython", "leftVentricularPressureReceiver")]
    ctl = {n: PressureSensor(n) for n in ("coronaryRpController", "coronaryRdController",
                                          "leftVentricularPressureReceiver")}
    spec = nio.to_netlistbc(coronary, 4, controllers=ctl)
    assert [(t, i) for t, i, _ in spec.controllers] == [("component", 3), ("component", 5), ("pressure", 5)]
    with pytest.raises(NotImplementedError):
        nio.to_netlistbc(coronary, 4)            # no controllers given
    lv = _parse("x.xml", _inputs()["netlist/heart/netlist_surfaces.xml"])[0]
    spec = nio.to_netlistbc(lv, 3, controllers={})
    assert [(t, i, type(c).__name__) for t, i, c in spec.controllers] == [
        ("component", 5, "LeftVentricularElastanceController")]
    assert spec.components[4][3] == pytest.approx(4.10246e-3)   # the set-up elastance
    files = _parse("x.xml", _inputs()["zeroDDomain/pythonFlowPrescriptions/netlist_surfaces.xml"])[2]
    with pytest.raises(NotImplementedError):
        nio.to_netlistbc(files, 3, controllers={})


def _tables():
    import json
    import os

    with open(os.path.join(os.path.dirname(__file__), "golden", "netlist_periodic_tables.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case,target,index", [("pythonFlowPrescriptions", "flow", 2),
                                               ("pythonPressurePrescriptions", "pressure", 3)])
def test_periodic_table_controls(tmp_path, case, target, index):
    """The reference's periodic prescriptions (its zeroDDomain
    pythonFlowPrescriptions / pythonPressurePrescriptions inputs, third
    circuit): the table beside the input drives a component's fixed flow or
    a node's fixed pressure, advancing by delt per step and wrapping at the
    table's last time; library and oracle take the same values."""
    name = f"zeroDDomain/{case}/netlist_surfaces.xml"
    circuit = _parse("x.xml", _inputs()[name])[2]
    (item, idx, ctype, source), = circuit["control_specs"]
    assert idx == index and ctype.startswith("prescribedPeriodic")
    table = _tables()[f"zeroDDomain/{case}/{source}.dat"]
    (tmp_path / f"{source}.dat").write_text(table)
    gspec = nio.to_netlistbc(circuit, 3, data_dir=str(tmp_path))
    ospec = nio.to_netlistbc(circuit, 3, data_dir=str(tmp_path))
    assert [(t, i) for t, i, _ in gspec.controllers] == [(target, index)]
    data = np.loadtxt(str(tmp_path / f"{source}.dat"))
    g, o = Netlist(gspec), OracleNetlist(ospec)
    time = 0.0
    for step in range(130):
        q = 20.0 + 10.0 * np.sin(2 * np.pi * step / 50)
        g.update(DT, q)
        o.update(DT, q)
        g.finalize_step()
        o.finalize_step()
        run_controllers([(g, t, i, c) for t, i, c in gspec.controllers], DT)
        oracle_run_controllers([(o, t, i, c) for t, i, c in ospec.controllers], DT)
        time += DT
        if time >= data[-1, 0]:
            time -= data[-1, 0]
        want = np.interp(time, data[:, 0], data[:, 1])
        assert g.get_parameter(target, index) == pytest.approx(want, rel=1e-12, abs=1e-9)
        assert o.get_parameter(target, index) == pytest.approx(want, rel=1e-12, abs=1e-9)
        p, f, _, _ = g.get()
        assert _close(p, [o.pressure(i + 1) for i in range(len(p))], 1e-10) and _close(f, o.q, 1e-10)
    g.close()


def test_bleed_controller_and_builtin_order():
    """The built-in bleed control sets its component to 0.001 from its
    trigger step on (1600 steps in the reference), after every Python
    controller of the step."""
    from crimsonflowsolver_b200.controllers import BleedController

    seen = []

    class Watch(ParameterController):
        controllerPriority = 5

        def updateControl(self, value, delt, pressures, flows, volumes):
            seen.append(g.get_parameter("component", 5))
            return value

    g = Netlist(_circuit())
    bound = [(g, "component", 5, BleedController("bleed", trigger_step=3)), (g, "pressure", 1, Watch("w"))]
    values = []
    for step in range(6):
        if g.flow_permitted():
            g.update(DT, 40.0)
        else:
            g.update_pressure(DT, 400.0)
        g.finalize_step()
        run_controllers(bound, DT)
        values.append(g.get_parameter("component", 5))
    assert values == [900.0, 900.0, 900.0, 0.001, 0.001, 0.001]
    assert seen == [900.0, 900.0, 900.0, 900.0, 0.001, 0.001]   # the Python controller ran first each step
    assert BleedController().trigger_step == 1600
    g.close()


def test_lv_elastance_curve():
    """The built-in LV elastance follows the raised-cosine curve: e_min at
    the cycle start, e_max at t_max, halfway down at t_max + t_relax / 2,
    e_min after the relaxation, periodic in the heart period."""
    from crimsonflowsolver_b200.controllers import LeftVentricularElastanceController as LV

    c = LV()
    assert c.elastance() == pytest.approx(c.e_min)
    for t, want in [(c.t_max, c.e_max), (c.t_max + 0.5 * c.t_relax, 0.5 * (c.e_min + c.e_max)),
                    (c.t_max + c.t_relax + 0.1, c.e_min), (0.25 * c.t_max, c.e_min + 0.5 * (c.e_max - c.e_min)
                                                          * (1 - np.cos(np.pi / 4)))]:
        c.time = t
        assert c.elastance() == pytest.approx(want, rel=1e-12)
    c = LV()
    dt = 1e-3
    vals = [c.updateControl(0.0, dt) for _ in range(2 * 860)]
    assert vals[859] == pytest.approx(c.e_min, rel=1e-9) and vals[:860] == pytest.approx(vals[860:], rel=1e-9)
    assert max(vals) == pytest.approx(c.e_max, rel=1e-4)
