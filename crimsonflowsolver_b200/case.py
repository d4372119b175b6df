"""Run one of the reference's case directories on the device path.

A case directory of the reference (flowsolver's ``solver.inp``, the PHASTA
``geombc.dat.1`` and ``restart.<numstart>.1``, ``numstart.dat``, the netlist
inputs ``netlist_surfaces.xml`` / ``.dat`` and
``netlist_closed_loop_downstream.xml``) becomes a :class:`Case`:

* :func:`parse_solver_inp` reads ``Key : value  # comment`` lines the way
  the reference's input reader does (input_fform.cxx; keys compared without
  case), :func:`flow_params` maps the keys this path uses onto
  :class:`~crimsonflowsolver_b200.problem.FlowParams`, the unset ones taking
  configs/input.config's defaults (:data:`INPUT_CONFIG_DEFAULTS`);
* settings outside the path (another linear solver, deformable walls,
  prescribed inflow from bct.dat, RCR surfaces from rcrt.dat, the purely
  zero-dimensional mode) raise ``NotImplementedError``;
* :meth:`Case.run` steps the device solver (``FlowSolver``: ``crimson_step``
  with the netlist circuits and closed loops coupled) and keeps the
  reference's history files: ``FlowHist.dat`` and ``PressHist.dat``
  (bctcardio.f90:1021-1040: the flow and the NASC-weighted mean pressure of
  every output surface, one row per step after the initial row) and a
  ``restart.<step>.1`` per step (restar.f90).
"""
from __future__ import annotations

import os
from typing import Dict, List, Optional

import numpy as np

from .problem import FlowParams

# configs/input.config values of the keys :func:`flow_params` reads (the
# memLS column of its linear-solver section)
INPUT_CONFIG_DEFAULTS = {
    "solver type": "memLS",
    "time integration rule": "First Order",
    "time integration rho infinity": "0.5",
    "step construction": "0 1",
    "tau c scale factor": "1.0",
    "tau time constant": "1.",
    "include viscous correction in stabilization": "True",
    "influx coefficient": "0.5",
    "number of krylov vectors per gmres sweep": "50",
    "number of gmres sweeps per solve": "1",
    "tolerance on momentum equations": "0.01",
    "tolerance on continuity equations": "0.2",
    "tolerance on memls ns solver": "0.4",
    "maximum number of iterations per nonlinear iteration": "200",
    "number of velocity projection vectors": "10",
    "density": "1.0",
    "residual control": "False",
    "deformable wall": "False",
    "time varying boundary conditions from file": "False",
    "simulate in purely zero dimensions": "False",
    "number of rcr surfaces": "0",
    "number of experimental rcr surfaces": "0",
    "number of netlist lpn surfaces": "0",
    "number of loop closing netlist circuits": "0",
}


def _key(k: str) -> str:
    return " ".join(k.strip().lower().split())


def parse_solver_inp(text: str) -> Dict[str, str]:
    """``{normalised key: value}`` of a solver.inp: '#' starts a comment,
    blank and comment lines are skipped, ``{`` / ``}`` section lines too."""
    out: Dict[str, str] = {}
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        if not line or ":" not in line:
            continue
        k, v = line.split(":", 1)
        out[_key(k)] = v.strip()
    return out


def _get(s: Dict[str, str], key: str) -> str:
    return s.get(key, INPUT_CONFIG_DEFAULTS.get(key, ""))


def _true(v: str) -> bool:
    return v.strip().lower() == "true"


def flow_params(settings: Dict[str, str], **extra) -> FlowParams:
    """FlowParams from parsed solver.inp settings (:func:`parse_solver_inp`);
    ``extra`` sets further fields (netlists, loops, precision ...)."""
    s = settings
    if _get(s, "solver type").lower() != "memls":
        raise NotImplementedError(f"Solver Type {_get(s, 'solver type')!r}: only memLS is on this path")
    for key in ("deformable wall", "time varying boundary conditions from file", "simulate in purely zero dimensions"):
        if _true(_get(s, key)):
            raise NotImplementedError(f"{key} = True is not supported")
    nrcr = sum(int(_get(s, key) or 0) for key in ("number of rcr surfaces", "number of experimental rcr surfaces"))
    if nrcr != len(extra.get("rcr", [])):
        raise NotImplementedError("RCR surfaces: read rcrt.dat with parse_rcrt and pass them as rcr=")
    steps = _get(s, "step construction").split()
    if len(steps) % 2 or any(steps[i] != "0" or steps[i + 1] != "1" for i in range(0, len(steps), 2)):
        raise NotImplementedError(f"Step Construction {' '.join(steps)!r}: only solve/update pairs '0 1'")
    rule = _get(s, "time integration rule").lower()
    rhoinf = -1.0 if rule == "first order" else float(_get(s, "time integration rho infinity"))
    for key in ("viscosity", "time step size"):
        if key not in s:
            raise ValueError(f"solver.inp has no {key!r} (input.config gives no default)")
    rescontrol = _true(_get(s, "residual control"))
    if rescontrol and not ("residual criteria" in s and "minimum required iterations" in s):
        raise ValueError("Residual Control needs Residual Criteria and Minimum Required Iterations")
    kw = dict(rho=float(_get(s, "density")), mu=float(s["viscosity"]), Delt=float(s["time step size"]), rhoinf=rhoinf,
              nitr=len(steps) // 2, taucfct=float(_get(s, "tau c scale factor")),
              dtsfct=float(_get(s, "tau time constant")),
              idiff=1 if _true(_get(s, "include viscous correction in stabilization")) else 0,
              stabflux_coeff=float(_get(s, "influx coefficient")),
              kspace=int(_get(s, "number of krylov vectors per gmres sweep")),
              ngmres=int(_get(s, "number of gmres sweeps per solve")),
              epstol_mom=float(_get(s, "tolerance on momentum equations")),
              epstol_cont=float(_get(s, "tolerance on continuity equations")),
              epstol_ns=float(_get(s, "tolerance on memls ns solver")),
              maxiters=int(_get(s, "maximum number of iterations per nonlinear iteration")),
              nprjs=int(_get(s, "number of velocity projection vectors")),
              rescontrol=rescontrol, res_criteria=float(s["residual criteria"]) if rescontrol else 0.0,
              min_iters=int(s["minimum required iterations"]) if rescontrol else 0)
    kw.update(extra)
    return FlowParams(**kw)


def parse_rcrt(text: str, srfids: List[int]):
    """rcrt.dat (RcrtReader, fileReaders.cxx:273-380; general_rcrbc.f90:
    34-60): the largest number of distal-pressure points, then per RCR
    surface its number of points, Rp, C, Rd and the (time, Pd) points.
    Returns :class:`~crimsonflowsolver_b200.problem.RCR` outlets; a distal
    pressure that varies in time is not supported."""
    from .problem import RCR

    tok = text.split()
    pos = 1
    out = []
    for srf in srfids:
        npts = int(tok[pos])
        rp, c, rd = (float(t) for t in tok[pos + 1:pos + 4])
        pd = [float(tok[pos + 5 + 2 * i]) for i in range(npts)]
        pos += 4 + 2 * npts
        if any(v != pd[0] for v in pd):
            raise NotImplementedError(f"surface {srf}: a time-varying distal pressure is not supported")
        out.append(RCR(srfid=srf, Rp=rp, C=c, Rd=rd, Pd=pd[0]))
    return out


def _write_hist(path: str, rows: List[np.ndarray]) -> None:
    """OutputDataFile's layout (bctcardio.f90): the row count, then one row
    of values per line."""
    with open(path, "w") as f:
        f.write(f"{len(rows):12d}\n")
        for r in rows:
            f.write("".join(f"  {v:.15E}" for v in r) + "\n")


class Case:
    """A reference case on the device path.  ``settings`` are parsed
    solver.inp settings; ``mesh``, ``y``, ``ac`` the geometry and the state
    the case starts from (restart ``step0``); ``netlists`` / ``loops`` its
    netlist circuits (:func:`netlist_io.closed_loops`)."""

    def __init__(self, settings: Dict[str, str], mesh, y, ac, netlists=(), loops=(), step0: int = 0, **extra):
        dv = getattr(mesh, "dirichlet_values", None)
        if dv is not None and len(dv) and np.any(np.delete(np.asarray(dv), 3, axis=1) != 0.0):
            # only the no-slip / zero-velocity rows (their fourth column holds
            # the unit the reference's presolver writes) are read
            raise NotImplementedError("geombc prescribes non-zero Dirichlet values")
        self.settings = settings
        self.mesh, self.y0, self.ac0, self.step0 = mesh, np.asarray(y, float), np.asarray(ac, float), int(step0)
        self.P = flow_params(settings, netlists=list(netlists), loops=list(loops), **extra)
        self.nsteps = int(settings.get("number of timesteps", "0") or 0)

    @classmethod
    def from_directory(cls, path: str, controllers=None, **extra) -> "Case":
        """Read solver.inp, numstart.dat, geombc.dat.1, restart.<numstart>.1
        and the netlist inputs of a reference case directory.  ``controllers``
        maps control script names to controllers."""
        from . import netlist_io, phasta

        with open(os.path.join(path, "solver.inp")) as f:
            settings = parse_solver_inp(f.read())
        step0 = 0
        if os.path.exists(os.path.join(path, "numstart.dat")):
            with open(os.path.join(path, "numstart.dat")) as f:
                step0 = int(f.read().split()[0])
        mesh = phasta.read_geombc(os.path.join(path, "geombc.dat.1"))
        y, ac, _ = phasta.read_restart(os.path.join(path, f"restart.{step0}.1"))
        srfids = [int(t) for t in settings.get("list of netlist lpn surfaces", "").split()]
        standalone, loops = [], []
        if srfids:
            xml = os.path.join(path, "netlist_surfaces.xml")
            spath = xml if os.path.exists(xml) else os.path.join(path, "netlist_surfaces.dat")
            with open(spath) as f:
                text = f.read()
            circuits = netlist_io.parse_netlist_xml(text) if spath.endswith(".xml") else netlist_io.parse_netlist_dat(text)
            downstream = []
            if int(_get(settings, "number of loop closing netlist circuits") or 0) > 0:
                with open(os.path.join(path, "netlist_closed_loop_downstream.xml")) as f:
                    downstream = netlist_io.parse_netlist_xml(f.read())
            standalone, loops = netlist_io.closed_loops(circuits, srfids, downstream, controllers=controllers,
                                                        data_dir=path)
        rcr_srf = [int(t) for key in ("list of rcr surfaces", "list of experimental rcr surfaces")
                   for t in settings.get(key, "").split()]
        if rcr_srf and "rcr" not in extra:
            with open(os.path.join(path, "rcrt.dat")) as f:
                extra["rcr"] = parse_rcrt(f.read(), rcr_srf)
        return cls(settings, mesh, y, ac, standalone, loops, step0, **extra)

    def run(self, steps: Optional[int] = None, out_dir: Optional[str] = None, write_restarts: bool = False):
        """Step the device solver ``steps`` times (default: Number of
        Timesteps).  Returns {"flow": rows, "pressure": rows} over the
        coupled surfaces (srflist order), the first row for the initial
        state; with ``out_dir`` writes FlowHist.dat / PressHist.dat there (and
        restart.<step>.1 per step with ``write_restarts``)."""
        from . import phasta
        from .solver import FlowSolver

        steps = self.nsteps if steps is None else int(steps)
        G = FlowSolver(self.mesh, self.P, inflow=lambda t: 0.0)
        try:
            y0 = self.y0.copy()
            full = ((self.mesh.iBC >> 3) & 7) == 7   # itrBC on the restart state
            y0[full, 0:3] = self.mesh.BC[full, 2:5]
            G.set_state(y0, self.ac0)
            q, p = G.outlet_state()
            if self.P.rcr and self.step0 == 0:
                # the RCRs start from the surfaces' initial pressure and flow
                # (callCPPSetPressureFromFortran, itrdrv.f90:748-760;
                # AbstractBoundaryCondition.cxx:105-117)
                from . import _native as N

                pn, qn = np.ascontiguousarray(p), np.ascontiguousarray(q)
                N.check(N.lib().crimson_rcr_state(G.elm.h, len(pn), N.dp(pn), N.dp(qn), 1), "crimson_rcr_state")
            flows, pressures = [q], [p]
            for k in range(steps):
                G.step()
                q, p = G.outlet_state()
                flows.append(q)
                pressures.append(p)
                if out_dir is not None and write_restarts:
                    y, ac = G.state()
                    phasta.write_restart(os.path.join(out_dir, f"restart.{self.step0 + k + 1}.1"), y, ac,
                                         self.step0 + k + 1)
        finally:
            G.close()
        if out_dir is not None:
            _write_hist(os.path.join(out_dir, "FlowHist.dat"), flows)
            _write_hist(os.path.join(out_dir, "PressHist.dat"), pressures)
        return {"flow": np.array(flows), "pressure": np.array(pressures)}
