"""Readers of the reference's netlist input files into :class:`NetlistBC`.

Two formats, as the reference reads them:

* ``netlist_surfaces.dat`` (NetlistReader, flowsolver/src/fileReaders.cxx:
  443-760): '#' lines and blank lines are skipped; per circuit the number of
  components, then per component its type letter (r, c, i, d, t, v), start
  node, end node and parameter (volume-tracking types add their initial
  volume on the same line); the prescribed pressures (count, nodes, values,
  types f/l), the prescribed flows (count, components, values, types f/t),
  the initial pressures (count, then "node pressure" lines), the 3D
  interface node, and the component and node control lists ("index type
  script" lines).
* ``netlist_surfaces.xml`` (NetlistXmlReader, flowsolver/src/
  NetlistXmlReader.cxx:30-460): ``netlistCircuits/circuit`` elements with
  ``components/component`` (index, type, startNodeIndex, endNodeIndex,
  parameterValue, initialVolume, initialUnstressedVolume,
  prescribedFlowType, prescribedFlowValue) and ``nodes/node`` (index,
  initialPressure, isAt3DInterface, prescribedPressureType; a fixed
  pressure takes the node's initialPressure); ``control`` elements (type,
  source) on components and nodes.

* ``netlist_closed_loop_downstream.xml`` (NetlistDownstreamXmlReader,
  NetlistXmlReader.cxx:470-640): loop-closing circuits in the same XML form,
  whose nodes carry ``upstreamConnectivity/connection`` elements
  (upstreamCircuitSurfaceIndex, connectsToUpstreamNode).

Each circuit comes back as a dict; :func:`to_netlistbc` turns one into a
:class:`NetlistBC` for a coupled surface, binding its customPython controls
to the controllers the caller supplies, and raises for what the library
does not model (left-ventricular pressures, built-in controllers, an
interface node other than 1).
"""
from __future__ import annotations

import os
import xml.etree.ElementTree as ET
from typing import Dict, List, Optional

from .problem import NetlistBC, NetlistLoopBC

_DAT_KINDS = {"r": "r", "c": "c", "i": "l", "d": "d", "t": "t", "v": "v"}
_XML_KINDS = {"resistor": "r", "capacitor": "c", "inductor": "l", "diode": "d", "volumetracking": "t",
              "volumetrackingpressurechamber": "v"}


def _dat_lines(text: str):
    """The non-comment, non-blank lines split on whitespace."""
    for line in text.splitlines():
        s = line.strip()
        if s and not s.startswith("#"):
            yield s.split()


def parse_netlist_dat(text: str) -> List[Dict]:
    lines = _dat_lines(text)
    out = []
    for first in lines:
        c: Dict = {"components": [], "volumes": {}, "prescribed_pressures": {}, "pressure_types": {},
                   "prescribed_flows": {}, "flow_types": {}, "initial_pressures": {}, "controls": 0}
        ncomp = int(first[0])
        for j in range(ncomp):
            kind = next(lines)[0]
            if kind not in _DAT_KINDS:
                raise ValueError(f"unknown netlist component type {kind!r}")
            st = int(next(lines)[0])
            en = int(next(lines)[0])
            par = next(lines)
            c["components"].append((_DAT_KINDS[kind], st, en, float(par[0])))
            if kind in ("t", "v"):
                if len(par) < 2:
                    raise ValueError("a volume-tracking component needs its initial volume")
                c["volumes"][j + 1] = (float(par[1]), 0.0)
        npp = int(next(lines)[0])
        nodes = [int(next(lines)[0]) for _ in range(npp)]
        vals = [float(next(lines)[0]) for _ in range(npp)]
        types = [next(lines)[0] for _ in range(npp)]
        for nd, v, t in zip(nodes, vals, types):
            c["prescribed_pressures"][nd] = v
            c["pressure_types"][nd] = t
        npf = int(next(lines)[0])
        comps = [int(next(lines)[0]) for _ in range(npf)]
        vals = [float(next(lines)[0]) for _ in range(npf)]
        types = [next(lines)[0] for _ in range(npf)]
        for j, v, t in zip(comps, vals, types):
            c["prescribed_flows"][j] = v
            c["flow_types"][j] = t
        nn = int(next(lines)[0])
        for _ in range(nn):
            t = next(lines)
            c["initial_pressures"][int(t[0])] = float(t[1])
        # older files end here: interface node 1, no controls
        t = next(lines, None)
        c["interface_node"] = int(t[0]) if t is not None else 1
        c["control_specs"] = []
        for item in (("component", "node") if t is not None else ()):  # component controls, then node controls
            k = int(next(lines)[0])
            for _ in range(k):
                f = next(lines)
                c["control_specs"].append((item, int(f[0]), f[1], f[2] if len(f) > 2 else ""))
            c["controls"] += k
        out.append(c)
    return out


def _text(el, tag, default=None):
    e = el.find(tag)
    return e.text.strip() if e is not None and e.text is not None else default


def parse_netlist_xml(text: str) -> List[Dict]:
    root = ET.fromstring(text)
    out = []
    for circ in root.findall("circuit"):
        c: Dict = {"components": [], "volumes": {}, "prescribed_pressures": {}, "pressure_types": {},
                   "prescribed_flows": {}, "flow_types": {}, "initial_pressures": {}, "controls": 0,
                   "interface_node": None, "control_specs": [], "connections": []}
        for j, comp in enumerate(circ.find("components").findall("component")):
            kind = _text(comp, "type").lower()
            if kind not in _XML_KINDS:
                raise ValueError(f"unknown netlist component type {kind!r}")
            k = _XML_KINDS[kind]
            c["components"].append((k, int(_text(comp, "startNodeIndex")), int(_text(comp, "endNodeIndex")),
                                    float(_text(comp, "parameterValue"))))
            if k in ("t", "v"):
                v0 = _text(comp, "initialVolume")
                if v0 is None:
                    raise ValueError("a volume-tracking component needs its initial volume")
                c["volumes"][j + 1] = (float(v0), float(_text(comp, "initialUnstressedVolume", "0")))
            ft = _text(comp, "prescribedFlowType")
            if ft is not None:
                t = {"fixed": "f", "threedinterface": "t"}[ft.lower()]
                c["prescribed_flows"][j + 1] = float(_text(comp, "prescribedFlowValue", "-1")) if t == "f" else -1.0
                c["flow_types"][j + 1] = t
            for ctl in comp.findall("control"):
                c["control_specs"].append(("component", j + 1, _text(ctl, "type", ""), _text(ctl, "source", "")))
                c["controls"] += 1
        for node in circ.find("nodes").findall("node"):
            idx = int(_text(node, "index"))
            p0 = float(_text(node, "initialPressure"))
            c["initial_pressures"][idx] = p0
            if (_text(node, "isAt3DInterface") or "").lower() == "true":
                c["interface_node"] = idx
            pt = _text(node, "prescribedPressureType")
            if pt is not None:
                t = {"fixed": "f", "leftventricular": "l"}[pt.lower()]
                c["prescribed_pressures"][idx] = p0 if t == "f" else 1.0
                c["pressure_types"][idx] = t
            for ctl in node.findall("control"):
                c["control_specs"].append(("node", idx, _text(ctl, "type", ""), _text(ctl, "source", "")))
                c["controls"] += 1
            for conn in node.findall("upstreamConnectivity/connection"):
                c["connections"].append((idx, int(_text(conn, "upstreamCircuitSurfaceIndex")),
                                         int(_text(conn, "connectsToUpstreamNode"))))
        out.append(c)
    return out


# control types of the inputs (fileReaders.cxx:680-760, NetlistXmlReader.cxx:60-130)
# that act through a user controller, and the parameter each one drives
_CONTROL_TARGETS = {("component", "custompython"): "component",
                    ("component", "custompythonunstressedvolume"): "unstressed_volume",
                    ("node", "custompython"): "pressure",
                    ("component", "prescribedperiodicflow"): "flow",
                    ("node", "prescribedperiodicpressure"): "pressure",
                    ("component", "bleed"): "component",
                    ("component", "bleedresistance"): "component",
                    ("component", "bleedcompliance"): "component",
                    ("component", "l"): "component",
                    ("component", "leftventricularelastance"): "component"}
_PERIODIC = ("prescribedperiodicflow", "prescribedperiodicpressure")
_BLEED = ("bleed", "bleedresistance", "bleedcompliance")
_LV = ("l", "leftventricularelastance")


def to_netlistbc(circuit: Dict, srfid: int, ignore_controls: bool = False, controllers=None,
                 data_dir: Optional[str] = None, shared_nodes=(), loop_closing: bool = False) -> NetlistBC:
    """One parsed circuit as the outlet of surface ``srfid``.  A circuit's
    customPython controls (component parameter, unstressed volume, node
    pressure) take their controller from ``controllers``, a mapping from the
    script name of the input to a
    :class:`~crimsonflowsolver_b200.controllers.ParameterController`; its
    prescribedPeriodicFlow / prescribedPeriodicPressure controls read the
    table ``<source>.dat`` from ``data_dir`` (unless ``controllers`` names
    them); with ``ignore_controls`` the parameters stay at their input
    values; bleed and left-ventricular elastance controls take the built-in
    :class:`~crimsonflowsolver_b200.controllers.BleedController` and
    :class:`~crimsonflowsolver_b200.controllers.LeftVentricularElastanceController`
    (the latter sets its chamber's elastance to the starting value).
    ``shared_nodes`` and ``loop_closing`` describe a member of a closed loop:
    the nodes it shares with the loop, and whether it is the loop-closing
    circuit (no 3D interface)."""
    from .controllers import BleedController, LeftVentricularElastanceController, PeriodicTableController

    bound = []
    components = list(circuit["components"])
    if circuit["controls"] and not ignore_controls:
        for item, index, ctype, source in circuit.get("control_specs", []):
            target = _CONTROL_TARGETS.get((item, ctype.lower()))
            if target is None:
                raise NotImplementedError(f"netlist control type {ctype!r} on {item} {index} is not supported")
            if ctype.lower() in _BLEED:
                bound.append((target, index, BleedController(f"bleed{index}")))
            elif ctype.lower() in _LV:
                k, st, en, _ = components[index - 1]
                if k not in ("t", "v"):
                    raise ValueError(f"an LV elastance control needs a volume-tracking component, not {k!r}")
                ctl = LeftVentricularElastanceController(f"lvElastance{index}")
                components[index - 1] = (k, st, en, ctl.elastance())   # the set-up value
                bound.append((target, index, ctl))
            elif controllers is not None and source in controllers:
                bound.append((target, index, controllers[source]))
            elif ctype.lower() in _PERIODIC and data_dir is not None:
                path = os.path.join(data_dir, source + ".dat")
                bound.append((target, index, PeriodicTableController.from_file(source, path)))
            else:
                raise NotImplementedError(f"no controller given for the control script {source!r}")
    if any(t != "f" for t in circuit["pressure_types"].values()):
        raise NotImplementedError("only fixed nodal pressures are supported")
    if circuit.get("interface_node") not in (None, 1):
        raise NotImplementedError("the 3D interface node must be node 1")
    iface = [j for j, t in circuit["flow_types"].items() if t == "t"]
    if loop_closing:
        if iface:
            raise ValueError("a loop-closing circuit has no 3D interface flow")
        iface = [0]
    elif len(iface) != 1:
        raise ValueError("exactly one component must carry the 3D interface flow")
    fixed_flows = {j: v for j, v in circuit["prescribed_flows"].items() if circuit["flow_types"][j] == "f"}
    return NetlistBC(srfid=srfid, components=components,
                     prescribed_pressures=dict(circuit["prescribed_pressures"]), prescribed_flows=fixed_flows,
                     interface_component=iface[0], initial_pressures=dict(circuit["initial_pressures"]),
                     volumes=dict(circuit["volumes"]), controllers=bound,
                     shared_nodes=tuple(sorted(set(int(d) for d in shared_nodes))))


def closed_loops(circuits: List[Dict], srfids: List[int], downstream: List[Dict], ignore_controls: bool = False,
                 controllers=None, data_dir: Optional[str] = None):
    """The netlist boundary circuits of surfaces ``srfids`` (parsed
    ``circuits`` in the same order) and the parsed loop-closing circuits
    ``downstream``: returns (the circuits that connect to no loop-closing
    circuit, as :class:`NetlistBC`; one :class:`NetlistLoopBC` per
    loop-closing circuit, its upstream circuits in input order).  A circuit
    connected to more than one loop-closing circuit is rejected, as the
    reference asserts (NetlistBoundaryCircuitWhenDownstreamCircuitsExist.cxx:
    33)."""
    if len(circuits) != len(srfids):
        raise ValueError(f"{len(circuits)} circuits, {len(srfids)} surfaces given")
    owner: Dict[int, int] = {}
    for li, d in enumerate(downstream):
        if not d["connections"]:
            raise ValueError("a loop-closing circuit without connections")
        for _, srf, _ in d["connections"]:
            if srf not in srfids:
                raise ValueError(f"a loop-closing circuit connects to surface {srf}, which has no netlist circuit")
            if owner.setdefault(srf, li) != li:
                raise NotImplementedError(f"surface {srf} connects to more than one loop-closing circuit")
    kw = dict(ignore_controls=ignore_controls, controllers=controllers, data_dir=data_dir)
    standalone, members = [], {}
    for c, srf in zip(circuits, srfids):
        if srf not in owner:
            standalone.append(to_netlistbc(c, srf, **kw))
            continue
        conns = downstream[owner[srf]]["connections"]
        members[srf] = to_netlistbc(c, srf, shared_nodes=[u for _, s2, u in conns if s2 == srf], **kw)
    loops = []
    for d in downstream:
        ups = [members[s] for s in srfids if s in members and any(s == s2 for _, s2, _ in d["connections"])]
        down = to_netlistbc(d, 0, shared_nodes=[n for n, _, _ in d["connections"]], loop_closing=True, **kw)
        loops.append(NetlistLoopBC(upstream=ups, downstream=down, connections=list(d["connections"])))
    return standalone, loops


def read_netlists(path: str, srfids: List[int], controllers=None) -> List[NetlistBC]:
    """Read a netlist_surfaces.dat or .xml; circuit k couples surface
    srfids[k]; ``controllers`` maps control script names to controllers."""
    with open(path) as f:
        text = f.read()
    circuits = parse_netlist_xml(text) if path.endswith(".xml") else parse_netlist_dat(text)
    if len(circuits) != len(srfids):
        raise ValueError(f"{len(circuits)} circuits in {path}, {len(srfids)} surfaces given")
    return [to_netlistbc(c, s, controllers=controllers, data_dir=os.path.dirname(os.path.abspath(path)))
            for c, s in zip(circuits, srfids)]


def netlist_surfaces_of_solver_inp(text: str) -> List[int]:
    """The "List of Netlist LPN Surfaces" of a solver.inp: the surface each
    netlist circuit couples, in input order."""
    for line in text.splitlines():
        key, _, val = line.partition(":")
        if key.strip().lower() == "list of netlist lpn surfaces":
            return [int(t) for t in val.split("#")[0].split()]
    return []


def read_closed_loops(surfaces_path: str, downstream_path: str, srfids: List[int], controllers=None):
    """Read a netlist_surfaces file and a netlist_closed_loop_downstream.xml:
    (standalone circuits, loops) as :func:`closed_loops` returns them."""
    with open(surfaces_path) as f:
        text = f.read()
    circuits = parse_netlist_xml(text) if surfaces_path.endswith(".xml") else parse_netlist_dat(text)
    with open(downstream_path) as f:
        downstream = parse_netlist_xml(f.read())
    return closed_loops(circuits, srfids, downstream, controllers=controllers,
                        data_dir=os.path.dirname(os.path.abspath(surfaces_path)))