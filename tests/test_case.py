"""CPU: the case driver's solver.inp reader (crimsonflowsolver_b200/case.py)
on the reference's own solver.inp files (tests/golden/
netlist_closed_loops.json) and on settings it must reject."""
import dataclasses
import json
import os

import pytest

from crimsonflowsolver_b200 import case
from tests.fixtures import closed_loop_heart_case, closed_loop_heart_mesh

HERE = os.path.dirname(os.path.abspath(__file__))


def _inp(name):
    with open(os.path.join(HERE, "golden", "netlist_closed_loops.json")) as f:
        return json.load(f)[name]["solver_inp"]


def test_closed_loop_heart_settings():
    """closedLoopHeart's solver.inp with input.config's defaults gives the
    parameters its test case is run with (tests/fixtures.py)."""
    s = case.parse_solver_inp(_inp("netlist/closedLoopHeart"))
    assert s["list of netlist lpn surfaces"] == "5 6 7" and s["solver type"] == "memLS"
    P = case.flow_params(s)
    _, _, _, ref = closed_loop_heart_case()
    fields = [f.name for f in dataclasses.fields(ref) if f.name not in ("netlists", "loops", "rcr")]
    assert {f: getattr(P, f) for f in fields} == {f: getattr(ref, f) for f in fields}


def test_every_reference_memls_case_reads():
    """The closed-loop cases' solver.inp files: the memLS one (closedLoopHeart)
    maps, the others (ACUSIM, purely zero-dimensional) are rejected by
    name."""
    with open(os.path.join(HERE, "golden", "netlist_closed_loops.json")) as f:
        cases = json.load(f)
    ok = 0
    for name, v in cases.items():
        s = case.parse_solver_inp(v["solver_inp"])
        if s.get("solver type", "").lower() != "memls" or s.get("simulate in purely zero dimensions") == "True":
            with pytest.raises(NotImplementedError):
                case.flow_params(s)
            continue
        P = case.flow_params(s)
        assert P.nitr * 2 == len(s["step construction"].split()) and P.Delt > 0
        ok += 1
    assert ok >= 1


def test_rejections_and_defaults():
    base = "Viscosity : 0.04\nTime Step Size : 0.001\n"
    P = case.flow_params(case.parse_solver_inp(base))
    assert (P.rho, P.rhoinf, P.nitr, P.kspace, P.epstol_ns, P.rescontrol) == (1.0, -1.0, 1, 50, 0.4, False)
    P = case.flow_params(case.parse_solver_inp(base + "Time Integration Rule: Second Order\n"
                                               "Time Integration Rho Infinity: 0.2\nStep Construction: 0 1 0 1 # x\n"))
    assert P.rhoinf == 0.2 and P.nitr == 2
    for bad in ("Solver Type: ACUSIM with P Projection", "Deformable Wall: True",
                "Time Varying Boundary Conditions From File: True", "Simulate in Purely Zero Dimensions: True",
                "Number of RCR Surfaces: 2", "Step Construction: 0 1 1 0"):
        with pytest.raises(NotImplementedError):
            case.flow_params(case.parse_solver_inp(base + bad + "\n"))
    with pytest.raises(ValueError):
        case.flow_params(case.parse_solver_inp(base + "Residual Control: True\n"))
    with pytest.raises(ValueError):
        case.flow_params(case.parse_solver_inp("Viscosity: 0.04\n"))


def test_case_from_parts():
    m, y, ac, ref = closed_loop_heart_case()
    c = case.Case(case.parse_solver_inp(_inp("netlist/closedLoopHeart")), m, y, ac, loops=ref.loops)
    assert c.nsteps == 5 and c.P.outlets()[0].srfid == 5 and len(c.P.loops) == 1
    m2, _, _ = closed_loop_heart_mesh()
    m2.dirichlet_values = m2.dirichlet_values.copy()
    m2.dirichlet_values[0, 0] = 1.0
    with pytest.raises(NotImplementedError):
        case.Case(c.settings, m2, y, ac)
