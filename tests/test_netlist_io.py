"""Netlist input files (CPU): the reference's own netlist_surfaces.dat / .xml
test inputs (tests/golden/netlist_inputs.json, made by
make_netlist_fixture.py) through the readers, and the circuits they describe
through the library's netlist calls against the oracle restatement."""
import json
import os

import numpy as np
import pytest

from crimsonflowsolver_b200 import netlist_io as nio
from crimsonflowsolver_b200.netlist import Netlist
from oracle import pyoracle as po
from oracle.netlist_oracle import OracleNetlist

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "netlist_inputs.json")
ALFI, DT = 0.5, 1e-3


def _inputs():
    with open(GOLDEN) as f:
        return json.load(f)


def _parse(name, text):
    return nio.parse_netlist_xml(text) if name.endswith(".xml") else nio.parse_netlist_dat(text)


def _close(a, b, tol):
    a, b = np.asarray(a, float), np.asarray(b, float)
    if a.size == 0:
        return True
    return np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max())


def test_every_reference_input_parses():
    n = 0
    for name, text in _inputs().items():
        circuits = _parse(name, text)
        assert circuits, name
        for c in circuits:
            assert c["components"] and c["initial_pressures"]
            assert sum(1 for t in c["flow_types"].values() if t == "t") == 1, name
            nodes = {s for _, s, _, _ in c["components"]} | {e for _, _, e, _ in c["components"]}
            assert nodes == set(range(1, max(nodes) + 1)) == set(c["initial_pressures"]), name
            n += 1
    assert n >= 40


def _q3d(step):
    """Interface flow of the Neumann steps."""
    return 50.0 + 40.0 * np.sin(2 * np.pi * step / 12)


def _p3d(step):
    """3D surface pressure of the Dirichlet steps: swings both ways, so the
    heart circuits' valves open and close within twelve steps."""
    return 20000.0 * np.sin(2 * np.pi * step / 12)


def _circuits():
    out = []
    for name, text in sorted(_inputs().items()):
        for k, c in enumerate(_parse(name, text)):
            out.append(pytest.param(name, k, id=f"{name}#{k + 1}"))
    return out


def _square(c):
    """The reference's well-formedness test (NetlistCircuit.cxx:1285-1289):
    Kirchhoff nodes + chamber rows + prescribed pressures and flows must
    equal the nodal pressures + tracked volumes."""
    deg = {}
    for _, s, e, _ in c["components"]:
        deg[s] = deg.get(s, 0) + 1
        deg[e] = deg.get(e, 0) + 1
    nk = sum(1 for v in deg.values() if v > 1)
    nch = sum(1 for x in c["components"] if x[0] == "v")
    return nk + nch + len(c["prescribed_pressures"]) + len(c["prescribed_flows"]) == len(deg) + len(c["volumes"])


@pytest.mark.parametrize("name,k", _circuits())
def test_reference_circuit_matches_oracle(name, k):
    """Each circuit of the reference's inputs (control scripts held at their
    input values) over twelve steps: implicit coefficients, pressures,
    flows, volumes and diode states, library vs oracle, with a pulsatile
    interface flow while flow can cross the interface (Neumann design) and
    a pulsatile 3D surface pressure while closed valves block it (Dirichlet
    design).  Circuits of closed-loop cases, whose boundary nodes belong to
    a downstream circuit in another file, are not square on their own and
    are rejected, as the reference rejects them without that circuit."""
    c = _parse(name, _inputs()[name])[k]
    spec = nio.to_netlistbc(c, 3, ignore_controls=True)
    if not _square(c):
        with pytest.raises(RuntimeError, match="not square"):
            Netlist(spec)
        return
    g = Netlist(spec)
    o = OracleNetlist(spec)
    try:
        for step in range(12):
            assert g.flow_permitted() == o.permitted, step
            if o.permitted:
                a = g.implicit_coefficients(ALFI * DT)
                b = o.implicit_coefficients(ALFI * DT)
                assert _close(a, b, 1e-9), (step, a, b)
                q = _q3d(step)
                g.update(DT, q)
                o.update(DT, q)
            else:
                with pytest.raises(RuntimeError):
                    g.implicit_coefficients(ALFI * DT)
                p3d = _p3d(step)
                g.update_pressure(DT, p3d)
                o.update_pressure(DT, p3d)
            p, f, _, vol = g.get()
            assert _close(p, [o.pressure(i + 1) for i in range(len(p))], 1e-9)
            assert _close(f, o.q, 1e-9)
            assert _close([vol[j] for j in o.vol_comps], [o.vol[j] for j in o.vol_comps], 1e-9)
            g.finalize_step()
            o.finalize_step()
            assert list(g.get()[2]) == list(o.open)
    finally:
        g.close()


def test_designs_switch_both_ways():
    """The Dirichlet steps above are not idle: 11 of the reference's square
    circuits start with closed valves blocking the interface, and 9 of them
    switch to the Neumann design and back within the twelve steps."""
    starts_blocked = switches = 0
    for name, text in sorted(_inputs().items()):
        for c in _parse(name, text):
            if not _square(c):
                continue
            o = OracleNetlist(nio.to_netlistbc(c, 3, ignore_controls=True))
            modes = ""
            for step in range(12):
                modes += "N" if o.permitted else "D"
                if o.permitted:
                    o.update(DT, _q3d(step))
                else:
                    o.update_pressure(DT, _p3d(step))
                o.finalize_step()
            starts_blocked += modes[0] == "D"
            switches += "DN" in modes and "ND" in modes
    assert starts_blocked == 11 and switches == 9


def test_emulate_rcr_input_is_the_rcr_model():
    """The reference's emulateRCR case (a Windkessel written as a netlist)
    gives the RCR.cxx coefficients and pressures for its own values."""
    (c,) = _parse("x.xml", _inputs()["netlist/emulateRCR/netlist_surfaces.xml"])
    spec = nio.to_netlistbc(c, 3)
    (_, _, _, Rp), (_, _, _, C), (_, _, _, Rd) = spec.components
    g = Netlist(spec)
    Pn, Qn = spec.initial_pressures[1], 0.0
    for step in range(10):
        ref = po.rcr_coeffs(Rp, C, Rd, 0.0, 0.0, Pn, Qn, ALFI * DT)
        assert _close(g.implicit_coefficients(ALFI * DT), ref, 1e-12)
        q = 30.0 + 10.0 * step
        g.update(DT, q)
        g.finalize_step()
        d1, h1 = po.rcr_coeffs(Rp, C, Rd, 0.0, 0.0, Pn, Qn, DT)
        Pn, Qn = d1 * q + h1, q
        assert _close(g.get()[0][0], Pn, 1e-12)
    g.close()


def test_unsupported_features_raise():
    """Left-ventricular pressure prescriptions (the reference itself exits
    on them without its heart model, NetlistCircuit.cxx:1391-1395) and
    unknown control types raise; the built-in LV elastance control binds."""
    heart = _parse("x.dat", _inputs()["netlist/netlist_surfaces.dat"])[0]
    spec = nio.to_netlistbc(heart, 3)
    assert [(t, i, type(c).__name__) for t, i, c in spec.controllers] == [
        ("component", 5, "LeftVentricularElastanceController")]
    lv = dict(heart, controls=0, pressure_types={6: "l"})
    with pytest.raises(NotImplementedError):
        nio.to_netlistbc(lv, 3)
    odd = dict(heart, control_specs=[("component", 5, "pc", "")])
    with pytest.raises(NotImplementedError):
        nio.to_netlistbc(odd, 3)


def _builtin_controlled():
    out = []
    for name, text in sorted(_inputs().items()):
        for k, c in enumerate(_parse(name, text)):
            types = {t.lower() for _, _, t, _ in c["control_specs"]}
            if types and types <= {"l", "leftventricularelastance", "bleed", "bleedresistance"} and _square(c):
                out.append(pytest.param(name, k, id=f"{name}#{k + 1}"))
    return out


@pytest.mark.parametrize("name,k", _builtin_controlled())
def test_reference_circuit_with_builtin_controls(name, k):
    """The reference's heart circuits with their built-in LV elastance
    control bound (the chamber's elastance follows the Pope et al. curve,
    set after every step): twelve steps through both designs, library vs
    oracle, each side with its own controller instances."""
    from crimsonflowsolver_b200.controllers import run_controllers
    from oracle.netlist_oracle import run_controllers as oracle_run

    c = _parse(name, _inputs()[name])[k]
    gs, os_ = nio.to_netlistbc(c, 3), nio.to_netlistbc(c, 3)
    g, o = Netlist(gs), OracleNetlist(os_)
    gb = [(g, t, i, ctl) for t, i, ctl in gs.controllers]
    ob = [(o, t, i, ctl) for t, i, ctl in os_.controllers]
    try:
        for step in range(12):
            assert g.flow_permitted() == o.permitted, step
            if o.permitted:
                assert _close(g.implicit_coefficients(ALFI * DT), o.implicit_coefficients(ALFI * DT), 1e-9)
                g.update(DT, _q3d(step))
                o.update(DT, _q3d(step))
            else:
                g.update_pressure(DT, _p3d(step))
                o.update_pressure(DT, _p3d(step))
            g.finalize_step()
            o.finalize_step()
            run_controllers(gb, DT)
            oracle_run(ob, DT)
            p, f, _, vol = g.get()
            assert _close(p, [o.pressure(i + 1) for i in range(len(p))], 1e-9)
            assert _close(f, o.q, 1e-9)
            for t, i, _ in gs.controllers:
                assert g.get_parameter(t, i) == pytest.approx(o.get_parameter(t, i), rel=1e-12)
    finally:
        g.close()


def test_read_netlists_assigns_surfaces(tmp_path):
    p = tmp_path / "netlist_surfaces.dat"
    p.write_text(_inputs()["netlist/simpleDiodeTest/netlist_surfaces.dat"])
    a, b = nio.read_netlists(str(p), [3, 4])
    assert (a.srfid, b.srfid) == (3, 4)
    assert [x[0] for x in a.components] == ["r", "d"] and [x[0] for x in b.components] == ["r", "c", "r"]
    with pytest.raises(ValueError):
        nio.read_netlists(str(p), [3])
