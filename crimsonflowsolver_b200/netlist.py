"""Netlist outlet circuits on the library's C ABI (crimson_netlist_*).

:class:`Netlist` owns one circuit handle built from a :class:`NetlistBC`
description; the calls mirror NetlistCircuit (flowsolver/src/
NetlistCircuit.cxx): implicit coefficients at the start of a step, update
with the end-of-step interface flow -- or, while closed diodes block the
interface (the Dirichlet design), with the 3D surface pressure --
finalisation (histories and diode switching).  :class:`NetlistLoop` solves
a closed loop -- upstream circuits coupled to 3D surfaces joined through a
loop-closing circuit (ClosedLoopDownstreamSubsection.cxx) -- as one system.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from .problem import NetlistBC, NetlistLoopBC

KINDS = {"r": 0, "c": 1, "l": 2, "i": 2, "d": 3, "t": 4, "v": 5}
# controllable parameters (crimson_netlist_set_parameter)
TARGETS = {"component": 0, "unstressed_volume": 1, "pressure": 2, "flow": 3}


class Netlist:
    def __init__(self, spec: NetlistBC):
        self.spec = spec
        comps = spec.components
        nn = spec.nnodes
        kind = np.array([KINDS[c[0]] for c in comps], dtype=np.int32)
        st = np.array([c[1] for c in comps], dtype=np.int32)
        en = np.array([c[2] for c in comps], dtype=np.int32)
        val = np.array([c[3] for c in comps], dtype=np.float64)
        p0 = np.array([spec.initial_pressures.get(i + 1, 0.0) for i in range(nn)], dtype=np.float64)
        v0 = np.array([spec.volumes.get(j + 1, (0.0, 0.0))[0] for j in range(len(comps))], dtype=np.float64)
        vu = np.array([spec.volumes.get(j + 1, (0.0, 0.0))[1] for j in range(len(comps))], dtype=np.float64)
        pn = np.array(sorted(spec.prescribed_pressures), dtype=np.int32)
        pv = np.array([spec.prescribed_pressures[k] for k in pn], dtype=np.float64)
        iface = int(spec.interface_component)
        fixed = sorted(spec.prescribed_flows)
        fc = ([iface] if iface else []) + fixed
        fk = ([1] if iface else []) + [0] * len(fixed)
        fv = ([0.0] if iface else []) + [spec.prescribed_flows[k] for k in fixed]
        fc, fk, fv = (np.array(fc, dtype=np.int32), np.array(fk, dtype=np.int32), np.array(fv, dtype=np.float64))
        self.ncomp, self.nnodes = len(comps), nn
        h = ctypes.c_void_p()
        if spec.shared_nodes or not iface:
            sh = np.array(sorted(spec.shared_nodes), dtype=np.int32)
            N.check(N.lib().crimson_netlist_create_member(
                ctypes.byref(h), len(comps), N.ip(kind), N.ip(st), N.ip(en), N.dp(val), N.dp(v0), N.dp(vu), nn,
                N.dp(p0), len(pn), N.ip(pn), N.dp(pv), len(fc), N.ip(fc), N.ip(fk), N.dp(fv), 1 if iface else 0,
                len(sh), N.ip(sh)), "crimson_netlist_create_member")
        else:
            N.check(N.lib().crimson_netlist_create(ctypes.byref(h), len(comps), N.ip(kind), N.ip(st), N.ip(en),
                                                   N.dp(val), N.dp(v0), N.dp(vu), nn, N.dp(p0), len(pn), N.ip(pn),
                                                   N.dp(pv), len(fc), N.ip(fc), N.ip(fk), N.dp(fv), 1),
                    "crimson_netlist_create")
        self.h = h

    def flow_permitted(self) -> bool:
        v = ctypes.c_int()
        N.check(N.lib().crimson_netlist_flow_permitted(self.h, ctypes.byref(v)), "crimson_netlist_flow_permitted")
        return bool(v.value)

    def implicit_coefficients(self, alfi_delt: float):
        a, b = ctypes.c_double(), ctypes.c_double()
        N.check(N.lib().crimson_netlist_implicit_coefficients(self.h, alfi_delt, ctypes.byref(a), ctypes.byref(b)),
                "crimson_netlist_implicit_coefficients")
        return a.value, b.value

    def update(self, delt: float, q: float) -> None:
        """updateLPN with the end-of-step interface flow (Neumann design)."""
        N.check(N.lib().crimson_netlist_update(self.h, delt, q), "crimson_netlist_update")

    def update_pressure(self, delt: float, p: float) -> None:
        """updateLPN with the 3D surface's mean pressure (Dirichlet design:
        closed diodes block the interface)."""
        N.check(N.lib().crimson_netlist_update_pressure(self.h, delt, p), "crimson_netlist_update_pressure")

    def finalize_step(self) -> None:
        N.check(N.lib().crimson_netlist_finalize_step(self.h), "crimson_netlist_finalize_step")

    def get(self):
        """(nodal pressures, component flows, diode open flags, volumes)."""
        p = np.zeros(self.nnodes)
        q = np.zeros(self.ncomp)
        o = np.zeros(self.ncomp, dtype=np.int32)
        v = np.zeros(self.ncomp)
        N.check(N.lib().crimson_netlist_get(self.h, N.dp(p), N.dp(q), N.ip(o), N.dp(v)), "crimson_netlist_get")
        return p, q, o.astype(bool), v

    def get_parameter(self, target: str, index: int) -> float:
        """A controllable parameter: target "component" (R, C, L, a diode's
        open resistance, a chamber's elastance), "unstressed_volume",
        "pressure" (node) or "flow" (fixed prescribed flow); index 1-based."""
        v = ctypes.c_double()
        N.check(N.lib().crimson_netlist_get_parameter(self.h, TARGETS[target], int(index), ctypes.byref(v)),
                "crimson_netlist_get_parameter")
        return v.value

    def set_parameter(self, target: str, index: int, value: float) -> None:
        N.check(N.lib().crimson_netlist_set_parameter(self.h, TARGETS[target], int(index), float(value)),
                "crimson_netlist_set_parameter")

    def observables(self):
        """(pressures by node, flows by component, volumes by volume-tracking
        component), 1-based dictionaries as control scripts receive them."""
        p, q, _, v = self.get()
        vols = {j + 1: float(v[j]) for j, c in enumerate(self.spec.components) if c[0] in ("t", "v")}
        return ({i + 1: float(x) for i, x in enumerate(p)}, {j + 1: float(x) for j, x in enumerate(q)}, vols)

    def state(self) -> np.ndarray:
        n = ctypes.c_int()
        N.check(N.lib().crimson_netlist_state_size(self.h, ctypes.byref(n)), "crimson_netlist_state_size")
        buf = np.zeros(n.value)
        N.check(N.lib().crimson_netlist_state(self.h, N.dp(buf), 0), "crimson_netlist_state")
        return buf

    def set_state(self, buf: np.ndarray) -> None:
        buf = np.ascontiguousarray(buf, dtype=np.float64)
        N.check(N.lib().crimson_netlist_state(self.h, N.dp(buf), 1), "crimson_netlist_state")

    def close(self) -> None:
        if getattr(self, "h", None):
            N.lib().crimson_netlist_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NetlistLoop:
    """A closed loop (:class:`NetlistLoopBC`) on crimson_netlist_loop_*: the
    member circuits (``upstream`` in input order, ``downstream``) are
    :class:`Netlist` objects the loop owns."""

    def __init__(self, spec: NetlistLoopBC):
        self.spec = spec
        self.upstream = [Netlist(c) for c in spec.upstream]
        self.downstream = Netlist(spec.downstream)
        cd = np.array([c[0] for c in spec.connections], dtype=np.int32)
        ck = np.array([spec.upstream_index(c[1]) for c in spec.connections], dtype=np.int32)
        cu = np.array([c[2] for c in spec.connections], dtype=np.int32)
        ups = (ctypes.c_void_p * len(self.upstream))(*[m.h.value for m in self.upstream])
        h = ctypes.c_void_p()
        N.check(N.lib().crimson_netlist_loop_create(ctypes.byref(h), len(self.upstream), ups, self.downstream.h,
                                                    len(cd), N.ip(cd), N.ip(ck), N.ip(cu)),
                "crimson_netlist_loop_create")
        self.h = h

    @property
    def members(self):
        return self.upstream + [self.downstream]

    def flow_permitted(self):
        """Per upstream circuit: whether flow can cross its 3D interface."""
        return [m.flow_permitted() for m in self.upstream]

    def implicit_coefficients(self, alfi_delt: float):
        """Per upstream circuit (dp_dq, hop); NaN in the Dirichlet design."""
        n = len(self.upstream)
        a, b = np.zeros(n), np.zeros(n)
        N.check(N.lib().crimson_netlist_loop_implicit_coefficients(self.h, alfi_delt, N.dp(a), N.dp(b)),
                "crimson_netlist_loop_implicit_coefficients")
        return list(zip(a.tolist(), b.tolist()))

    def update(self, delt: float, flows, pressures=None) -> None:
        """updateLPN of every member: upstream circuit k takes flows[k] (its
        end-of-step interface flow) or, in the Dirichlet design,
        pressures[k] (its 3D surface's mean pressure)."""
        n = len(self.upstream)
        q = np.ascontiguousarray(flows, dtype=np.float64).reshape(n)
        p = np.zeros(n) if pressures is None else np.ascontiguousarray(pressures, dtype=np.float64).reshape(n)
        N.check(N.lib().crimson_netlist_loop_update(self.h, delt, N.dp(q), N.dp(p)), "crimson_netlist_loop_update")

    def finalize_step(self) -> None:
        N.check(N.lib().crimson_netlist_loop_finalize_step(self.h), "crimson_netlist_loop_finalize_step")

    def close(self) -> None:
        if getattr(self, "h", None):
            N.lib().crimson_netlist_loop_free(self.h)
            self.h = None
        for m in getattr(self, "upstream", []) + ([self.downstream] if hasattr(self, "downstream") else []):
            m.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
