"""Netlist outlet circuits (CPU): the library's crimson_netlist_* calls against
the oracle restatement of NetlistCircuit (oracle/netlist_oracle.py), and both
against the reference's own three-element Windkessel (RCR.cxx:49-81, the
oracle's orc_rcr_coeffs) for the circuit 1 -Rp- 2, 2 -C- ground, 2 -Rd- Pd.
The netlist calls are host code: no GPU is needed."""
import ctypes

import numpy as np
import pytest

from crimsonflowsolver_b200 import NetlistBC
from crimsonflowsolver_b200 import _native as N
from crimsonflowsolver_b200.netlist import Netlist
from oracle import pyoracle as po
from oracle.netlist_oracle import OracleNetlist

ALFI, DT = 0.5, 1e-3


def _close(a, b, tol=1e-12):
    a, b = np.asarray(a, float), np.asarray(b, float)
    if a.size == 0 and b.size == 0:
        return True
    return np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max())


@pytest.mark.parametrize("Pd", [0.0, 7.5])
def test_rcr_circuit_matches_reference_rcr(Pd):
    """The netlist form of the Windkessel gives the RCR.cxx coefficients and
    end-of-step pressures (library and oracle), step after step."""
    Rp, C, Rd = 100.0, 1e-4, 1000.0
    spec = NetlistBC.rcr(3, Rp=Rp, C=C, Rd=Rd, Pd=Pd)
    g, o = Netlist(spec), OracleNetlist(spec)
    Pn = Qn = 0.0
    rng = np.random.default_rng(3)
    for _ in range(12):
        ref = po.rcr_coeffs(Rp, C, Rd, Pd, Pd, Pn, Qn, ALFI * DT)
        assert _close(g.implicit_coefficients(ALFI * DT), ref, 1e-12)
        assert _close(o.implicit_coefficients(ALFI * DT), ref, 1e-12)
        q = 20.0 * rng.standard_normal()
        g.update(DT, q)
        g.finalize_step()
        o.update(DT, q)
        o.finalize_step()
        d1, h1 = po.rcr_coeffs(Rp, C, Rd, Pd, Pd, Pn, Qn, DT)
        Pn, Qn = d1 * q + h1, q
        assert _close(g.get()[0][0], Pn, 1e-12) and _close(o.interface_pressure(), Pn, 1e-12)
    g.close()


def _random_circuit(rng, nextra=6, with_inductor=True, with_diode=True, fixed_flow=True):
    """A random tree from the interface node 1 plus a few cycles; leaves get
    fixed pressures (or, for one leaf, a fixed flow on its component);
    pressure chambers end at a fixed-pressure leaf of their own."""
    comps = [("r", 1, 2, float(rng.uniform(50, 150)))]
    nodes = [2]
    nxt = 3
    kinds = ["r", "c", "v"] + (["l"] if with_inductor else []) + (["d"] if with_diode else [])
    volumes, chamber_leaves = {}, set()
    for _ in range(nextra):
        a = int(rng.choice(nodes))
        k = str(rng.choice(kinds))
        val = {"r": rng.uniform(100, 2000), "c": rng.uniform(1e-5, 1e-3), "l": rng.uniform(1.0, 10.0),
               "d": rng.uniform(1.0, 20.0), "v": rng.uniform(500.0, 5000.0)}[k]
        if k == "v":
            comps.append((k, a, nxt, float(val)))
            volumes[len(comps)] = (float(rng.uniform(20.0, 60.0)), float(rng.uniform(0.0, 10.0)))
            chamber_leaves.add(nxt)
            nxt += 1
            continue
        comps.append((k, a, nxt, float(val)) if rng.random() < 0.7 else (k, nxt, a, float(val)))
        nodes.append(nxt)
        nxt += 1
    # one cycle between two existing non-interface nodes
    a, b = rng.choice(nodes, size=2, replace=False)
    comps.append(("r", int(a), int(b), float(rng.uniform(100, 1000))))
    # a resistor from node 2 to a fixed-pressure leaf: flow can always leave
    comps.append(("r", 2, nxt, float(rng.uniform(500, 3000))))
    nxt += 1
    deg = np.zeros(nxt, dtype=int)
    for _, s, e, _ in comps:
        deg[s] += 1
        deg[e] += 1
    leaves = [i for i in range(2, nxt) if deg[i] == 1]
    pres, flows = {}, {}
    for i, leaf in enumerate(leaves):
        j = next(j for j, c in enumerate(comps) if leaf in (c[1], c[2]))
        if fixed_flow and i == 0 and len(leaves) > 1 and comps[j][0] in ("r", "c") and leaf not in chamber_leaves:
            flows[j + 1] = float(rng.uniform(-2, 2))
        else:
            pres[leaf] = float(rng.uniform(0, 50)) if rng.random() < 0.5 else 0.0
    init = {i: float(rng.uniform(0, 100)) for i in range(1, nxt)}
    return NetlistBC(srfid=3, components=comps, prescribed_pressures=pres, prescribed_flows=flows,
                     interface_component=1, initial_pressures=init, volumes=volumes)


@pytest.mark.parametrize("seed", range(16))
def test_random_circuits_match_oracle(seed):
    """Coefficients, nodal pressures, component flows and diode states over
    ten steps of random interface flows, library vs oracle."""
    rng = np.random.default_rng(100 + seed)
    spec = _random_circuit(rng)
    o = OracleNetlist(spec)
    try:
        g = Netlist(spec)
    except RuntimeError as e:  # the generator may build a blocked or singular circuit
        pytest.skip(str(e))
    if not g.flow_permitted():
        g.close()
        pytest.skip("closed diodes block the interface in this draw")
    for step in range(10):
        if not g.flow_permitted():
            break
        try:
            a = g.implicit_coefficients(ALFI * DT)
        except RuntimeError as e:
            # a draw whose closed diodes cut off a fixed-flow leaf: the system
            # is singular for the oracle too
            assert "SINGULAR" in str(e)
            A, _, _ = o._system(ALFI * DT)
            assert np.linalg.cond(A) > 1e12
            break
        b = o.implicit_coefficients(ALFI * DT)
        assert _close(a, b, 1e-10), (step, a, b)
        q = float(30.0 * rng.standard_normal())
        g.update(DT, q)
        o.update(DT, q)
        p, f, op, vol = g.get()
        assert _close(p, [o.pressure(i + 1) for i in range(len(p))], 1e-10)
        assert _close(f, o.q, 1e-10)
        assert _close([vol[j] for j in o.vol_comps], [o.vol[j] for j in o.vol_comps], 1e-10)
        g.finalize_step()
        o.finalize_step()
        assert list(g.get()[2]) == list(o.open)
    g.close()


def test_diode_opens_and_closes_like_oracle():
    """A diode branch in parallel with a resistor to ground: closed at the
    start, open after a positive pressure drop, closed again under backflow."""
    spec = NetlistBC(srfid=3, components=[("r", 1, 2, 100.0), ("d", 2, 3, 5.0), ("c", 3, 4, 1e-4),
                                          ("r", 2, 5, 800.0)],
                     prescribed_pressures={4: 0.0, 5: 0.0}, interface_component=1)
    g, o = Netlist(spec), OracleNetlist(spec)
    states = []
    for q in [10.0, 10.0, 10.0, -40.0, -40.0, -40.0]:
        assert _close(g.implicit_coefficients(ALFI * DT), o.implicit_coefficients(ALFI * DT), 1e-12)
        g.update(DT, q)
        o.update(DT, q)
        g.finalize_step()
        o.finalize_step()
        states.append(bool(g.get()[2][1]))
        assert states[-1] == o.open[1]
    assert states[0] and not states[-1], states
    g.close()


def test_series_diode_blocks_interface():
    """Closed diodes on every path from the interface: the circuit takes the
    Dirichlet design (CircuitData.cxx:482-540).  No implicit coefficients
    (CRIMSON_ERR_STATE); the update takes the 3D surface pressure, and the
    diode opens under a positive pressure drop, returning the circuit to the
    Neumann design -- library vs oracle throughout."""
    spec = NetlistBC(srfid=3, components=[("r", 1, 2, 100.0), ("d", 2, 3, 5.0), ("c", 3, 4, 1e-4)],
                     prescribed_pressures={4: 0.0}, interface_component=1)
    g, o = Netlist(spec), OracleNetlist(spec)
    assert not g.flow_permitted() and not o.permitted
    a, b = ctypes.c_double(), ctypes.c_double()
    rc = N.lib().crimson_netlist_implicit_coefficients(g.h, ALFI * DT, ctypes.byref(a), ctypes.byref(b))
    assert rc == 8  # CRIMSON_ERR_STATE
    with pytest.raises(RuntimeError):
        g.update(DT, 1.0)
    g.update_pressure(DT, 500.0)
    o.update_pressure(DT, 500.0)
    p, q, _, _ = g.get()
    assert _close(p, [o.pressure(i + 1) for i in range(len(p))], 1e-12) and _close(q, o.q, 1e-12)
    assert p[0] == 500.0 and q[0] == 0.0
    g.finalize_step()
    o.finalize_step()
    assert g.flow_permitted() and o.permitted      # the diode opened
    with pytest.raises(RuntimeError):
        g.update_pressure(DT, 500.0)
    assert _close(g.implicit_coefficients(ALFI * DT), o.implicit_coefficients(ALFI * DT), 1e-12)
    g.close()


@pytest.mark.parametrize("case", ["two_3d_flows", "interface_not_node1", "missing_node", "not_square",
                                  "interface_shared"])
def test_malformed_circuits_rejected(case):
    comps = [("r", 1, 2, 100.0), ("c", 2, 3, 1e-4), ("r", 2, 4, 1000.0)]
    pres = {3: 0.0, 4: 0.0}
    kw = {}
    if case == "two_3d_flows":
        kw = dict(prescribed_flows={})
        spec = NetlistBC(srfid=3, components=comps, prescribed_pressures=pres, interface_component=1)
        nl = Netlist(spec)  # valid; then a raw call with two 3D flows
        nl.close()
        kind = np.array([0, 1, 0], np.int32)
        st = np.array([1, 2, 2], np.int32)
        en = np.array([2, 3, 4], np.int32)
        val = np.array([100.0, 1e-4, 1000.0])
        p0 = np.zeros(4)
        pn = np.array([3, 4], np.int32)
        pv = np.zeros(2)
        fc = np.array([1, 3], np.int32)
        fk = np.array([1, 1], np.int32)
        fv = np.zeros(2)
        h = ctypes.c_void_p()
        rc = N.lib().crimson_netlist_create(ctypes.byref(h), 3, N.ip(kind), N.ip(st), N.ip(en), N.dp(val), None,
                                            None, 4, N.dp(p0), 2, N.ip(pn), N.dp(pv), 2, N.ip(fc), N.ip(fk),
                                            N.dp(fv), 1)
        assert rc == 1 and not h.value
        return
    if case == "interface_not_node1":
        comps = [("r", 2, 1, 100.0), ("c", 1, 3, 1e-4), ("r", 1, 4, 1000.0)]
    elif case == "missing_node":
        comps = [("r", 1, 2, 100.0), ("c", 2, 3, 1e-4), ("r", 2, 5, 1000.0)]
        pres = {3: 0.0, 5: 0.0}
    elif case == "not_square":
        pres = {3: 0.0}
    elif case == "interface_shared":
        comps = comps + [("r", 1, 4, 50.0)]
    with pytest.raises(RuntimeError):
        Netlist(NetlistBC(srfid=3, components=comps, prescribed_pressures=pres, interface_component=1, **kw))


def test_state_checkpoint_round_trip():
    """Restoring a checkpointed circuit state reproduces the steps after it
    bit for bit."""
    rng = np.random.default_rng(9)
    spec = NetlistBC(srfid=3, components=[("r", 1, 2, 100.0), ("l", 2, 3, 4.0), ("c", 3, 4, 2e-4),
                                          ("d", 3, 5, 3.0), ("r", 5, 6, 500.0)],
                     prescribed_pressures={4: 0.0, 6: 10.0}, interface_component=1,
                     initial_pressures={2: 20.0, 3: 20.0, 5: 15.0})
    g = Netlist(spec)
    qs = 25.0 * rng.standard_normal(8)
    for q in qs[:3]:
        g.implicit_coefficients(ALFI * DT)
        g.update(DT, q)
        g.finalize_step()
    ck = g.state()

    def run():
        out = []
        for q in qs[3:]:
            out.append(g.implicit_coefficients(ALFI * DT))
            g.update(DT, q)
            g.finalize_step()
            out.append(tuple(g.get()[0]))
        return out

    a = run()
    g.set_state(ck)
    b = run()
    assert a == b
    g.close()


def test_volume_tracking_component_with_fixed_flow():
    """A volume-tracking component whose flow is prescribed integrates its
    volume (V = V_hist + Delt q), beside a pressure chamber on the outlet."""
    spec = NetlistBC(srfid=3, components=[("r", 1, 2, 100.0), ("v", 2, 3, 2000.0), ("t", 2, 4, 0.0),
                                          ("r", 2, 5, 700.0)],
                     prescribed_pressures={3: 0.0, 4: 0.0, 5: 0.0}, prescribed_flows={3: 0.5},
                     interface_component=1, initial_pressures={2: 40.0},
                     volumes={2: (30.0, 10.0), 3: (5.0, 0.0)})
    g, o = Netlist(spec), OracleNetlist(spec)
    for step in range(6):
        assert _close(g.implicit_coefficients(ALFI * DT), o.implicit_coefficients(ALFI * DT), 1e-12)
        g.update(DT, 12.0)
        o.update(DT, 12.0)
        p, f, _, vol = g.get()
        assert _close(vol[2], 5.0 + (step + 1) * DT * 0.5, 1e-12)
        assert _close(p[1], (vol[1] - 10.0) * 2000.0, 1e-12)
        assert _close(p, [o.pressure(i + 1) for i in range(len(p))], 1e-12)
        g.finalize_step()
        o.finalize_step()
    g.close()
