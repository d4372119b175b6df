"""CPU: closed loops of netlist circuits (ClosedLoopDownstreamSubsection,
flowsolver/src/ClosedLoopDownstreamSubsection.cxx:101-940;
NetlistBoundaryCircuitWhenDownstreamCircuitsExist.cxx;
NetlistClosedLoopDownstreamCircuit.cxx) through crimson_netlist_loop_*,
against the oracle's restatement (oracle/netlist_oracle.py, OracleLoop).

* every closed-loop case of the reference's inputs (fixture
  tests/golden/netlist_closed_loops.json: the downstream XML, the
  netlist_surfaces file and the solver.inp surface list) reads into square
  loops, and twelve steps of coefficients, updates and finalisations match
  the oracle to 1e-9 in both interface designs;
* pin of the loop assembly: a loop with one upstream circuit is the same
  circuit as the standalone netlist with the shared nodes merged, so its
  coefficients, pressures and flows equal that circuit's (library and
  oracle, whose standalone path the reference's circuits pin);
* the readers, and the rejections of malformed loops.
"""
import json
import math
import os

import numpy as np
import pytest

from crimsonflowsolver_b200 import NetlistBC, NetlistLoopBC
from crimsonflowsolver_b200 import netlist_io as nio
from crimsonflowsolver_b200.netlist import Netlist, NetlistLoop
from oracle.netlist_oracle import OracleLoop, OracleNetlist

HERE = os.path.dirname(os.path.abspath(__file__))
DT, ALFI = 1e-3, 0.5


def _cases():
    with open(os.path.join(HERE, "golden", "netlist_closed_loops.json")) as f:
        return json.load(f)


def _loops(case):
    v = _cases()[case]
    parse = nio.parse_netlist_xml if v["surfaces_file"].endswith(".xml") else nio.parse_netlist_dat
    return nio.closed_loops(parse(v["surfaces"]), v["srfids"], nio.parse_netlist_xml(v["downstream"]),
                            ignore_controls=True)


def _oracle(spec):
    return OracleLoop([OracleNetlist(c) for c in spec.upstream], OracleNetlist(spec.downstream),
                      [(d, spec.upstream_index(s), u) for d, s, u in spec.connections])


def _close(a, b, tol):
    a, b = np.asarray(a, float), np.asarray(b, float)
    same_nan = np.isnan(a) == np.isnan(b)
    ok = np.abs(np.nan_to_num(a) - np.nan_to_num(b)) <= tol * np.maximum(1.0, np.abs(np.nan_to_num(b)))
    return bool(np.all(same_nan) and np.all(ok))


def test_reader_closed_loop_heart():
    """netlist/closedLoopHeart: surfaces 5 6 7, one loop-closing circuit
    whose node 1 joins node 5 of surface 5's circuit and whose node 4 joins
    node 4 of surface 6's and node 3 of surface 7's."""
    standalone, loops = _loops("netlist/closedLoopHeart")
    assert standalone == [] and len(loops) == 1
    L = loops[0]
    assert [c.srfid for c in L.upstream] == [5, 6, 7]
    assert L.connections == [(1, 5, 5), (4, 6, 4), (4, 7, 3)]
    assert [c.shared_nodes for c in L.upstream] == [(5,), (4,), (3,)]
    assert L.downstream.shared_nodes == (1, 4) and L.downstream.interface_component == 0
    assert L.downstream.prescribed_pressures == {3: 0.0}


def test_reader_two_loops():
    """zeroDDomain/twoDomainsClosedLoop: surfaces 4 6 5 7 and two
    loop-closing circuits, each joining two of them (input order kept)."""
    standalone, loops = _loops("zeroDDomain/twoDomainsClosedLoop")
    assert standalone == []
    assert [[c.srfid for c in L.upstream] for L in loops] == [[4, 7], [6, 5]]


def test_solver_inp_surface_list():
    assert nio.netlist_surfaces_of_solver_inp("a : 1\n    List of Netlist LPN Surfaces : 4 6 5 7 # x\n") == [4, 6, 5, 7]
    assert nio.netlist_surfaces_of_solver_inp("Number of Coupled Surfaces : 2\n") == []


def _case_loops():
    out = []
    for case in sorted(_cases()):
        _, loops = _loops(case)
        out += [(case, i) for i in range(len(loops))]
    return out


@pytest.mark.parametrize("case,i", _case_loops())
def test_reference_loop_matches_oracle(case, i):
    """Twelve steps of each loop of the reference's closed-loop inputs
    (control scripts held at their input values): coefficients (NaN for a
    circuit in the Dirichlet design), every member's pressures, flows,
    volumes and diode states, library vs oracle, with pulsatile interface
    flows and surface pressures."""
    spec = _loops(case)[1][i]
    g = NetlistLoop(spec)
    o = _oracle(spec)
    designs = set()
    try:
        for step in range(12):
            assert g.flow_permitted() == [m.permitted for m in o.up]
            designs.add(tuple(g.flow_permitted()))
            assert _close(g.implicit_coefficients(ALFI * DT), o.implicit_coefficients(ALFI * DT), 1e-9), step
            n = len(spec.upstream)
            q = [3.0 * math.sin(0.7 * step + k) for k in range(n)]
            p = [1000.0 + 300.0 * math.cos(0.5 * step + k) for k in range(n)]
            g.update(DT, q, p)
            o.update(DT, q, p)
            for gm, om in zip(g.members, o.members):
                pp, f, _, vol = gm.get()
                assert _close(pp, [om.pressure(j + 1) for j in range(len(pp))], 1e-9), step
                assert _close(f, om.q, 1e-9), step
                assert _close([vol[j] for j in om.vol_comps], [om.vol[j] for j in om.vol_comps], 1e-9)
            g.finalize_step()
            o.finalize_step()
            for gm, om in zip(g.members, o.members):
                assert list(gm.get()[2]) == list(om.open)
    finally:
        g.close()
    # every reference loop has a heart (valved) circuit that starts blocked
    assert any(not all(d) for d in designs)


def _pin_loop():
    """Upstream: 1 -R- 2 (3D flow), 2 -C- 3 (ground), 2 -L- 4, 4 -D- 5; node
    5 is shared.  Loop-closing: 1 -R- 2, 1 -C- 3 (ground), 2 -R- 4 (venous
    pressure); its node 1 is the upstream node 5."""
    up = NetlistBC(srfid=3, components=[("r", 1, 2, 50.0), ("c", 2, 3, 2e-4), ("l", 2, 4, 3.0), ("d", 4, 5, 5.0)],
                   prescribed_pressures={3: 0.0}, interface_component=1,
                   initial_pressures={1: 90.0, 2: 90.0, 4: 80.0, 5: 70.0}, shared_nodes=(5,))
    down = NetlistBC(srfid=0, components=[("r", 1, 2, 400.0), ("c", 1, 3, 1e-3), ("r", 2, 4, 20.0)],
                     prescribed_pressures={3: 0.0, 4: 8.0}, interface_component=0,
                     initial_pressures={1: 70.0, 2: 40.0}, shared_nodes=(1,))
    loop = NetlistLoopBC(upstream=[up], downstream=down, connections=[(1, 3, 5)])
    # the same circuit with downstream node d numbered 4 + d (node 1 -> 5)
    ren = {1: 5, 2: 6, 3: 7, 4: 8}
    merged = NetlistBC(srfid=3, components=up.components[:] + [(k, ren[s], ren[e], v) for k, s, e, v in down.components],
                       prescribed_pressures={3: 0.0, 7: 0.0, 8: 8.0}, interface_component=1,
                       initial_pressures={1: 90.0, 2: 90.0, 4: 80.0, 5: 70.0, 6: 40.0})
    return loop, merged


def test_loop_of_one_circuit_equals_merged_circuit():
    """Library and oracle: the loop's coefficients, pressures (the shared
    node's on both sides), flows and diode states equal those of the merged
    standalone circuit over twelve steps whose diode opens."""
    spec, merged = _pin_loop()
    g, gm = NetlistLoop(spec), Netlist(merged)
    o, om = _oracle(spec), OracleNetlist(merged)
    opened = False
    try:
        for step in range(12):
            q = 2.0 + math.sin(step)
            (a, b), = g.implicit_coefficients(ALFI * DT)
            (oa, ob), = o.implicit_coefficients(ALFI * DT)
            ma, mb = gm.implicit_coefficients(ALFI * DT)
            oma, omb = om.implicit_coefficients(ALFI * DT)
            assert _close([a, b], [ma, mb], 1e-10) and _close([oa, ob], [oma, omb], 1e-10), step
            g.update(DT, [q])
            gm.update(DT, q)
            o.update(DT, [q], [0.0])
            om.update(DT, q)
            pu, fu, ou, _ = g.upstream[0].get()
            pd, fd, od, _ = g.downstream.get()
            pm, fm, omo, _ = gm.get()
            assert _close(np.r_[pu, pd[1:]], pm, 1e-10) and abs(pd[0] - pu[4]) <= 1e-10 * abs(pu[4]), step
            assert _close(np.r_[fu, fd], fm, 1e-10), step
            assert _close(np.r_[o.up[0].p, o.down.p[1:]], om.p, 1e-10), step
            g.finalize_step()
            gm.finalize_step()
            o.finalize_step()
            om.finalize_step()
            assert list(np.r_[g.upstream[0].get()[2], g.downstream.get()[2]]) == list(gm.get()[2])
            opened |= bool(g.upstream[0].get()[2][3])
    finally:
        g.close()
        gm.close()
    assert opened


def test_member_is_solved_through_its_loop():
    spec, _ = _pin_loop()
    m = Netlist(spec.upstream[0])
    d = Netlist(spec.downstream)
    try:
        with pytest.raises(RuntimeError):
            m.implicit_coefficients(ALFI * DT)
        with pytest.raises(RuntimeError):
            d.update(DT, 1.0)
        assert d.flow_permitted()
    finally:
        m.close()
        d.close()


def test_malformed_loops_rejected():
    spec, _ = _pin_loop()
    up, down = spec.upstream[0], spec.downstream
    # the connections name a node the circuit does not share
    with pytest.raises(RuntimeError):
        NetlistLoop(NetlistLoopBC(upstream=[up], downstream=down, connections=[(1, 3, 4)]))
    # the loop-closing circuit's shared nodes differ from its connections
    down2 = NetlistBC(**{**down.__dict__, "shared_nodes": (1, 2)})
    with pytest.raises(RuntimeError):
        NetlistLoop(NetlistLoopBC(upstream=[up], downstream=down2, connections=[(1, 3, 5)]))
    # a circuit whose rows and shared nodes do not make up its unknowns (the
    # shared node also has a prescribed pressure)
    up3 = NetlistBC(**{**up.__dict__, "prescribed_pressures": {3: 0.0, 5: 1.0}})
    with pytest.raises(RuntimeError, match="shared nodes"):
        Netlist(up3)
    # a loop-closing circuit cannot carry the 3D flow
    with pytest.raises(RuntimeError):
        Netlist(NetlistBC(**{**down.__dict__, "interface_component": 1}))
    # the reader: a loop-closing circuit without a 3D interface only
    circ = nio.parse_netlist_xml(_cases()["netlist/closedLoopHeart"]["surfaces"])[0]
    with pytest.raises(ValueError):
        nio.to_netlistbc(circ, 5, ignore_controls=True, loop_closing=True)


def test_reader_rejects_circuit_in_two_loops():
    v = _cases()["netlist/closedLoopHeart"]
    circuits = nio.parse_netlist_xml(v["surfaces"])
    down = nio.parse_netlist_xml(v["downstream"])
    with pytest.raises(NotImplementedError):
        nio.closed_loops(circuits, v["srfids"], down + down, ignore_controls=True)
    with pytest.raises(ValueError):
        nio.closed_loops(circuits, [5, 6, 8], down, ignore_controls=True)


def test_closed_loop_heart_with_lv_control():
    """netlist/closedLoopHeart with its circuits' controls bound (the heart's
    built-in LV elastance): twelve steps, library vs oracle, each side with
    its own controller instances run after the finalisation."""
    from crimsonflowsolver_b200.controllers import run_controllers
    from oracle.netlist_oracle import run_controllers as oracle_run

    v = _cases()["netlist/closedLoopHeart"]

    def read():
        return nio.closed_loops(nio.parse_netlist_xml(v["surfaces"]), v["srfids"],
                                nio.parse_netlist_xml(v["downstream"]))[1][0]

    gs, os_ = read(), read()
    assert any(c.controllers for c in gs.upstream)
    g, o = NetlistLoop(gs), _oracle(os_)
    gb = [(m, t, i, c) for m, spec in zip(g.members, gs.upstream + [gs.downstream]) for t, i, c in spec.controllers]
    ob = [(m, t, i, c) for m, spec in zip(o.members, os_.upstream + [os_.downstream]) for t, i, c in spec.controllers]
    try:
        for step in range(12):
            assert g.flow_permitted() == [m.permitted for m in o.up]
            assert _close(g.implicit_coefficients(ALFI * DT), o.implicit_coefficients(ALFI * DT), 1e-9), step
            q = [2.0 * math.sin(0.9 * step + k) for k in range(3)]
            p = [9000.0 + 2000.0 * math.cos(0.4 * step + k) for k in range(3)]
            g.update(DT, q, p)
            o.update(DT, q, p)
            g.finalize_step()
            o.finalize_step()
            run_controllers(gb, DT)
            oracle_run(ob, DT)
            for gm, om in zip(g.members, o.members):
                pp, f, _, _ = gm.get()
                assert _close(pp, [om.pressure(j + 1) for j in range(len(pp))], 1e-9), step
                assert _close(f, om.q, 1e-9), step
            for (gm, t, i, _), (om, _, _, _) in zip(gb, ob):
                assert gm.get_parameter(t, i) == pytest.approx(om.get_parameter(t, i), rel=1e-12)
    finally:
        g.close()


def test_loop_checkpoint_restart():
    """Every member's state written after five steps and read into a fresh
    loop: the next five steps of both loops are identical."""
    spec = _loops("netlist/closedLoopHeart")[1][0]
    a = NetlistLoop(spec)
    b = NetlistLoop(spec)

    def run(loop, steps):
        for step in steps:
            loop.flow_permitted()
            loop.implicit_coefficients(ALFI * DT)
            loop.update(DT, [1.5 * math.sin(step + k) for k in range(3)], [9000.0 + 100.0 * step] * 3)
            loop.finalize_step()

    try:
        run(a, range(5))
        for ma, mb in zip(a.members, b.members):
            mb.set_state(ma.state())
        run(a, range(5, 10))
        run(b, range(5, 10))
        for ma, mb in zip(a.members, b.members):
            assert np.array_equal(ma.state(), mb.state())
    finally:
        a.close()
        b.close()
