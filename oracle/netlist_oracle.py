"""CPU restatement of the reference's netlist outlet circuits (test infrastructure).

Only the tests, smoke() and bench.py's CPU legs use this module, as the
checker of the library's crimson_netlist_* calls.  It follows
flowsolver/src/NetlistCircuit.cxx, CircuitData.cxx and CircuitComponent.cxx:

* the linear system of generateLinearSystemWithoutFactorisation
  (NetlistCircuit.cxx:1057-1302): unknowns [nodal pressures | history
  pressures | component flows | history flows]; rows: one per component
  (resistor p_s - p_e - R q = 0; open diode the same with its resistance,
  closed diode q = 0; capacitor p_s - p_e - (alfi_delt / C) q - h_s + h_e = 0;
  inductor p_s - p_e - (L / alfi_delt)(q - q_hist) = 0), one Kirchhoff row
  per node with more than one incident component (876-917), then identity
  rows for fixed pressures, history pressures, prescribed flows and history
  flows (1262-1296), all in ascending index order;
* the right-hand side of assembleRHS (1370-1580), the 3D flow multiplied by
  the interface sign (CircuitData.cxx:186-207);
* the inverse and x = A^-1 b of solveLinearSystem (1723-1733), the
  coefficients of computeImplicitCoefficients (1764-1800);
* updateLPN (1582-1594), finalizeLPNAtEndOfTimestep (732-737) with the
  diode rule of CircuitComponent.cxx:4-17 and the closed-diode start of
  NetlistBoundaryCondition.cxx:10-35;
* volume-tracking components (V - V_hist - alfi_delt q = 0) and pressure
  chambers (the same plus p_start / E - V = -V_unstressed, the start node
  then taking E (V - V_unstressed), CircuitComponent.cxx:188-209), with the
  tracked and history volumes after the history flows (1147-1241, 1282-1287);
* the search for a path from the interface through flow-permitting
  components to a free end (CircuitData.cxx:388-470), and the Dirichlet
  design while none exists (CircuitData.cxx:482-540): the interface node
  joins the prescribed pressures with the 3D surface pressure
  (NetlistCircuit.cxx:1386-1410), the interface component leaves the
  prescribed flows.

* closed loops (ClosedLoopDownstreamSubsection.cxx:101-500, 609-940): each
  member circuit leaves out the Kirchhoff rows of the nodes it shares with
  the loop (NetlistCircuit.cxx:880-920), the blocks of the upstream circuits
  and then the loop-closing circuit sit on the diagonal, followed by one
  Kirchhoff row per shared node of the loop-closing circuit and one
  pressure-equality row per connection; the implicit coefficients of
  upstream circuit k come from the inverse at (its node 1, its 3D-flow row)
  (852-888).

numpy's LAPACK inverse stands in for PETSc's dense MatMatSolve.
"""
from __future__ import annotations

import numpy as np


class OracleNetlist:
    def __init__(self, spec):
        self.comps = [("l" if k == "i" else k, int(s), int(e), float(v)) for k, s, e, v in spec.components]
        self.np_ = max(max(s, e) for _, s, e, _ in self.comps)
        self.nc = len(self.comps)
        self.fixed = {int(k): float(v) for k, v in spec.prescribed_pressures.items()}
        self.fixed_flow = {int(k): float(v) for k, v in spec.prescribed_flows.items()}
        self.iface = int(spec.interface_component)   # 0: a loop-closing circuit
        self.shared = set(int(d) for d in getattr(spec, "shared_nodes", ()))
        self.p = np.array([spec.initial_pressures.get(i + 1, 0.0) for i in range(self.np_)], dtype=float)
        self.q = np.zeros(self.nc)
        self.sign = 1.0 if not self.iface or self.comps[self.iface - 1][1] == 1 else -1.0
        cap_nodes = set()
        for k, s, e, _ in self.comps:
            if k == "c":
                cap_nodes.update((s, e))
        self.hist_nodes = sorted(cap_nodes)
        self.hist_comps = [j for j, c in enumerate(self.comps) if c[0] == "l"]
        self.vol_comps = [j for j, c in enumerate(self.comps) if c[0] in ("t", "v")]
        self.vol = {j: float(spec.volumes[j + 1][0]) for j in self.vol_comps}
        self.v0 = {j: float(spec.volumes[j + 1][1]) for j in self.vol_comps}
        self.hist_v = dict(self.vol)
        self.nchamber = sum(1 for c in self.comps if c[0] == "v")
        count = np.zeros(self.np_ + 1, dtype=int)
        for _, s, e, _ in self.comps:
            count[s] += 1
            count[e] += 1
        self.kirch = [i for i in range(1, self.np_ + 1) if count[i] > 1 and i not in self.shared]
        self.pp = sorted(self.fixed)
        self.pf = sorted(set(self.fixed_flow) | ({self.iface} if self.iface else set()))
        self.open = [c[0] != "d" for c in self.comps]  # diodes start closed
        self.p3d = 0.0
        self.permitted = self.flow_permitted()
        self.hist_p = {i: self.pressure(i) for i in self.hist_nodes}
        self.hist_q = {j: self.q[j] for j in self.hist_comps}
        self.last_q = 0.0
        self.n = self.np_ + len(self.hist_nodes) + self.nc + len(self.hist_comps) + 2 * len(self.vol_comps)

    def flow_permitted(self):
        """Whether some flow-permitting path leads from the interface
        component to a component end no other component touches (other
        than the interface node)."""
        if not self.iface:
            return True
        touching = {}
        for j, (_, s, e, _) in enumerate(self.comps):
            touching.setdefault(s, set()).add(j)
            touching.setdefault(e, set()).add(j)
        todo, seen = [self.iface - 1], set()
        while todo:
            j = todo.pop()
            if j in seen:
                continue
            seen.add(j)
            if not self.open[j]:
                continue
            _, s, e, _ = self.comps[j]
            ends = [(s, touching[s] - {j}), (e, touching[e] - {j})]
            if any(not others and node != 1 for node, others in ends):
                return True
            for _, others in ends:
                todo.extend(others)
        return False

    def pressure(self, node):
        return self.fixed.get(node, self.p[node - 1])

    def _system(self, alfi_delt):
        n, np_, nc = self.n, self.np_, self.nc
        nhp = len(self.hist_nodes)
        fq = np_ + nhp          # first flow unknown
        fhq = fq + nc           # first history-flow unknown
        hp_col = {node: np_ + i for i, node in enumerate(self.hist_nodes)}
        hq_col = {j: fhq + i for i, j in enumerate(self.hist_comps)}
        fv = fhq + len(self.hist_comps)
        v_col = {j: fv + i for i, j in enumerate(self.vol_comps)}
        hv_col = {j: fv + len(self.vol_comps) + i for i, j in enumerate(self.vol_comps)}
        rows = n - len(self.shared)
        A = np.zeros((rows, n))
        b = np.zeros(rows)
        r = 0
        for j, (k, s, e, v) in enumerate(self.comps):
            if k in ("t", "v"):
                A[r, fq + j] = -alfi_delt
                A[r, v_col[j]] = 1.0
                A[r, hv_col[j]] = -1.0
                if k == "v":
                    r += 1
                    A[r, s - 1] = 1.0 / v
                    A[r, v_col[j]] = -1.0
                    b[r] = -self.v0[j]
            elif k == "d" and not self.open[j]:
                A[r, fq + j] = 1.0
            else:
                A[r, s - 1] = 1.0
                A[r, e - 1] = -1.0
                if k in ("r", "d"):
                    A[r, fq + j] = -v
                elif k == "c":
                    A[r, fq + j] = -alfi_delt / v
                    A[r, hp_col[s]] = -1.0
                    A[r, hp_col[e]] = 1.0
                else:
                    A[r, fq + j] = -v / alfi_delt
                    A[r, hq_col[j]] = v / alfi_delt
            r += 1
        for node in self.kirch:
            for j, (_, s, e, _) in enumerate(self.comps):
                if e == node:
                    A[r, fq + j] = 1.0
                if s == node:
                    A[r, fq + j] = -1.0
            r += 1
        dirichlet = not self.permitted
        for node in sorted(set(self.pp) | ({1} if dirichlet else set())):
            A[r, node - 1] = 1.0
            b[r] = self.fixed[node] if node in self.fixed else self.p3d
            r += 1
        for node in self.hist_nodes:
            A[r, hp_col[node]] = 1.0
            b[r] = self.hist_p[node]
            r += 1
        iface_row = None
        for comp in self.pf:
            if dirichlet and comp == self.iface:
                continue
            A[r, fq + comp - 1] = 1.0
            if comp == self.iface:
                b[r] = self.last_q * self.sign
                iface_row = r
            else:
                b[r] = self.fixed_flow[comp]
            r += 1
        for j in self.hist_comps:
            A[r, hq_col[j]] = 1.0
            b[r] = self.hist_q[j]
            r += 1
        for j in self.vol_comps:
            A[r, hv_col[j]] = 1.0
            b[r] = self.hist_v[j]
            r += 1
        assert r == rows
        return A, b, iface_row

    def implicit_coefficients(self, alfi_delt):
        assert self.permitted, "no implicit coefficients in the Dirichlet design"
        A, b, col = self._system(alfi_delt)
        Ainv = np.linalg.inv(A)
        x = Ainv @ b
        return self.sign * Ainv[0, col], x[0] - Ainv[0, col] * b[col]

    def update(self, delt, q):
        assert self.permitted
        self.last_q = q
        self._update(delt)

    def update_pressure(self, delt, p):
        assert not self.permitted
        self.p3d = p
        self._update(delt)

    def _update(self, delt):
        A, b, _ = self._system(delt)
        self.take(np.linalg.inv(A) @ b)

    def take(self, x):
        """Pressures, flows and volumes from this circuit's solution segment."""
        self.p = x[:self.np_].copy()
        fq = self.np_ + len(self.hist_nodes)
        self.q = x[fq:fq + self.nc].copy()
        fv = fq + self.nc + len(self.hist_comps)
        for i, j in enumerate(self.vol_comps):
            self.vol[j] = x[fv + i]
            k, s, _, v = self.comps[j]
            if k == "v":
                self.p[s - 1] = (self.vol[j] - self.v0[j]) * v

    def finalize_step(self):
        self.hist_p = {i: self.pressure(i) for i in self.hist_nodes}
        self.hist_q = {j: self.q[j] for j in self.hist_comps}
        self.hist_v = dict(self.vol)
        for j, (k, s, e, _) in enumerate(self.comps):
            if k == "d":
                self.open[j] = (self.pressure(s) - self.pressure(e) >= -1e-8) or (self.q[j] >= 1e-8)
        self.permitted = self.flow_permitted()

    def interface_pressure(self):
        return self.pressure(1)

    # ---- control systems (ControlSystemsManager.cxx:125-330) ----
    def get_parameter(self, target, index):
        j = index - 1
        if target == "component":
            return self.comps[j][3]
        if target == "unstressed_volume":
            assert self.comps[j][0] == "v"
            return self.v0[j]
        if target == "pressure":
            return self.fixed[index] if index in self.fixed else float(self.p[j])
        if target == "flow":
            return self.fixed_flow[index]
        raise KeyError(target)

    def set_parameter(self, target, index, value):
        j = index - 1
        if target == "component":
            k, s, e, _ = self.comps[j]
            self.comps[j] = (k, s, e, float(value))
        elif target == "unstressed_volume":
            assert self.comps[j][0] == "v"
            self.v0[j] = float(value)
        elif target == "pressure":
            if index in self.fixed:
                self.fixed[index] = float(value)
            else:
                self.p[j] = float(value)
        elif target == "flow":
            assert index in self.fixed_flow
            self.fixed_flow[index] = float(value)
        else:
            raise KeyError(target)

    def observables(self):
        p = {i + 1: float(self.pressure(i + 1)) for i in range(self.np_)}
        q = {j + 1: float(self.q[j]) for j in range(self.nc)}
        v = {j + 1: float(self.vol[j]) for j in self.vol_comps}
        return p, q, v


class OracleLoop:
    """A closed loop: upstream circuits (input order), the loop-closing
    circuit, and the connections (downstream node, upstream index 0-based,
    upstream node) in file order."""

    def __init__(self, upstream, downstream, connections):
        self.up = list(upstream)
        self.down = downstream
        self.conn = [(int(d), int(k), int(u)) for d, k, u in connections]
        self.members = self.up + [self.down]

    def _system(self, alfi_delt):
        blocks = [m._system(alfi_delt) for m in self.members]
        n = sum(m.n for m in self.members)
        A = np.zeros((n, n))
        b = np.zeros(n)
        r0, c0 = [], []
        r = c = 0
        for m, (Am, bm, _) in zip(self.members, blocks):
            A[r:r + Am.shape[0], c:c + m.n] = Am
            b[r:r + Am.shape[0]] = bm
            r0.append(r)
            c0.append(c)
            r += Am.shape[0]
            c += m.n

        def kirchhoff(row, mi, node):
            m = self.members[mi]
            fq = c0[mi] + m.np_ + len(m.hist_nodes)
            for j, (_, s, e, _) in enumerate(m.comps):
                if e == node:
                    A[row, fq + j] = 1.0
                if s == node:
                    A[row, fq + j] = -1.0

        for d in sorted({d for d, _, _ in self.conn}):
            for k in range(len(self.up)):
                for d2, k2, u in self.conn:
                    if d2 == d and k2 == k:
                        kirchhoff(r, k, u)
                        break
            kirchhoff(r, len(self.up), d)
            r += 1
        for d, k, u in self.conn:
            A[r, c0[k] + u - 1] = 1.0
            A[r, c0[-1] + d - 1] = -1.0
            r += 1
        assert r == n
        return A, b, r0, c0, [blk[2] for blk in blocks]

    def implicit_coefficients(self, alfi_delt):
        A, b, r0, c0, irow = self._system(alfi_delt)
        Ainv = np.linalg.inv(A)
        x = Ainv @ b
        out = []
        for k, m in enumerate(self.up):
            if not m.permitted:
                out.append((float("nan"), float("nan")))
                continue
            col = r0[k] + irow[k]
            g = Ainv[c0[k], col]
            out.append((m.sign * g, x[c0[k]] - g * b[col]))
        return out

    def update(self, delt, flows, pressures):
        for k, m in enumerate(self.up):
            if m.permitted:
                m.last_q = flows[k]
            else:
                m.p3d = pressures[k]
        A, b, _, c0, _ = self._system(delt)
        x = np.linalg.inv(A) @ b
        for m, c in zip(self.members, c0):
            m.take(x[c:c + m.n])

    def finalize_step(self):
        for m in self.members:
            m.finalize_step()


def run_controllers(bound, delt):
    """The control systems' update of one step: ascending priority, each
    controller given the values the earlier ones published (the first
    publication of a name kept), its return value set as the parameter."""
    order = sorted(range(len(bound)), key=lambda k: bound[k][3].getControllerPriority())
    gathered = {}
    for k in order:
        circuit, target, index, ctl = bound[k]
        ctl.receive_broadcast(gathered)
        p, q, v = circuit.observables()
        circuit.set_parameter(target, index, float(ctl.updateControl(circuit.get_parameter(target, index), delt,
                                                                     p, q, v)))
        for name, data in ctl.broadcast_data().items():
            if name not in gathered:
                gathered[name] = data
