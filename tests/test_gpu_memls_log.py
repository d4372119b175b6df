"""The per-solve log in memLS's memLS_NS.log format: a header line
(gnNo, tasks, coupled faces) when the file is new, then one fixed-width line
per solve whose fields are the solve's own statistics."""
import numpy as np
import pytest

from crimsonflowsolver_b200 import FlowParams, RCR, mesh, solver
from tests.linsys import first_system

pytestmark = pytest.mark.gpu


def _fields(line):
    """Split one line by the Fortran format (I4.3,I3,I4,I5,3I4,3ES9.2E2,3I4)."""
    widths = [4, 3, 4, 5, 4, 4, 4, 9, 9, 9, 4, 4, 4]
    out, pos = [], 0
    for w in widths:
        out.append(line[pos:pos + w])
        pos += w
    return [int(out[i]) for i in range(7)] + [float(out[i]) for i in range(7, 10)] + [int(out[i]) for i in (10, 11, 12)]


def test_log_lines_match_stats(tmp_path):
    m = mesh.cylinder(ncross=8, naxial=10)
    m.set_inflow(10.0)
    P = FlowParams(rcr=[RCR(srfid=3)])
    elm = solver.ElmGMR(m, P)
    colm, rowp = elm.genadj()
    F, Res4, Val4, faceRes, out, state = first_system(m, P, colm, rowp)
    ms = solver.MemLS(P, 2, nshg=m.nshg, colm=colm, rowp=rowp)
    log = tmp_path / "memLS_NS.log"
    try:
        nodes, sv = solver.dirichlet_face(m)
        ms.bc_create(1, nodes, 3, 0, sv)
        nn, vv = solver.neumann_face(m, 3)
        ms.bc_create(2, nn, 3, 1, vv)
        ms.set_log(str(log))
        stats = [ms.solve(Res4, Val4.copy(), faceRes)[1] for _ in range(2)]
        ms.set_log(None)
        ms.solve(Res4, Val4.copy(), faceRes)
    finally:
        ms.close()
        elm.close()
    lines = log.read_text().splitlines()
    assert len(lines) == 3
    assert [int(v) for v in lines[0].split()] == [m.nshg, 1, 1]
    for line, st in zip(lines[1:], stats):
        f = _fields(line)
        assert f[0] == 100 * st.RI.suc + 10 * st.GM.suc + st.CG.suc
        assert f[1:4] == [st.RI.itr, st.GM.itr, st.CG.itr]
        assert abs(sum(f[4:7]) - 100) <= 2
        assert f[7] == pytest.approx(st.RI.iNorm, rel=1e-2)
        assert f[8] == pytest.approx(st.RI.fNorm / st.RI.iNorm, rel=1e-2)
        assert f[10:12] == [st.Resm, st.Resc]
