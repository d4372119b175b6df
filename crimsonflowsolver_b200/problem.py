"""Flow, time-integration and memLS solver settings shared by every driver.

The fields mirror the reference's ``solver.inp`` keys (defaults from
configs/input.config and the reference test cases):

* rho, mu                    ``Density`` / ``Viscosity`` (datmat)
* rhoinf                     ``Time Integration Rho Infinity`` (second order)
* Delt                       ``Time Step Size``
* dtsfct, taucfct            ``Tau Time Constant`` / ``Tau C Scale Factor``
* idiff                      ``Include Viscous Correction in Stabilization`` (1 for p=1)
* iconvflow                  ``Flow Advection Form`` (2 = Convective)
* stabflux_coeff             ``Influx Coefficient``
* ibksiz                     ``Number of Elements Per Block``
* nitr                       number of solve/update pairs in ``Step Construction``
* rescontrol, res_criteria,  ``Residual Control`` / ``Residual Criteria`` /
  min_iters                  ``Minimum Required Iterations``
* epstol_mom, epstol_cont,   memLS tolerances (epstol(1), epstol(7), epstol(8))
  epstol_ns
* kspace, ngmres, maxiters,  memLS sizes (Kspace, nGMRES, maxIters, nPrjs)
  nprjs

Tolerances: the outer NSSOLVER loop estimates its residual as
sqrt(|R0|^2 - xB.B) (flowsolver/src/memLS.f90:1545).  In FP64 that estimate
has a floor of a few 1e-7 relative: xB comes from a Gram system whose
condition number grows with the number of directions, so xB.B carries
~1e-13 relative error, and below the floor the argument of the square root
is roundoff that can go negative (NaN), turning the convergence branch into a
coin toss.  The defaults therefore use ``epstol_ns`` = 1e-5 with inner GMRES /
CG tolerances of 1e-4; each outer iteration then reduces the estimate about
7x and every solve on the test tubes converges by the estimate in ~7 outer
iterations, far from the floor.  A requested "solver tolerance 1e-8" maps
onto this setting (the tightest the reference's estimator can decide).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Tuple


def time_params(rhoinf: float):
    """(almi, alfi, gami) of flowsolver/src/itrPC.f90:16-37."""
    if rhoinf < 0.0 or rhoinf > 1.0:
        return 1.0, 1.0, 1.0
    almi = (3.0 - rhoinf) / (1.0 + rhoinf) / 2.0
    alfi = 1.0 / (1.0 + rhoinf)
    gami = 0.5 + almi - alfi
    return almi, alfi, gami


@dataclass
class RCR:
    """Three-element Windkessel outlet (flowsolver/src/RCR.cxx)."""
    srfid: int
    Rp: float = 100.0
    C: float = 1e-4
    Rd: float = 1000.0
    Pd: float = 0.0


@dataclass
class NetlistBC:
    """Netlist (0D lumped-parameter) outlet circuit (flowsolver/src/
    NetlistCircuit.cxx), the input a netlist XML description carries.

    components: (kind, start node, end node, value) with kind "r" (resistor),
    "c" (capacitor), "l" or "i" (inductor), "d" (diode; value = open
    resistance), "t" (volume tracking) or "v" (pressure chamber; value =
    elastance); nodes are numbered 1..N and node 1 is the 3D interface node.
    prescribed_pressures: node -> fixed pressure ('f').
    prescribed_flows: component (1-based) -> fixed flow ('f').
    interface_component: the component (1-based) carrying the 3D flow ('t').
    initial_pressures: node -> initial pressure (default 0).
    volumes: component (1-based) -> (initial volume, unstressed volume) for
    the "t" and "v" components.
    controllers: (target, index, controller) triples: a
    :class:`~crimsonflowsolver_b200.controllers.ParameterController` that
    sets, after every step, the component value ("component"), a chamber's
    unstressed volume ("unstressed_volume"), a node's pressure ("pressure")
    or a component's fixed flow ("flow") of item ``index`` (1-based).
    shared_nodes: for a member of a closed loop (:class:`NetlistLoopBC`), the
    nodes it shares with the loop's other circuits; interface_component 0
    marks the loop-closing circuit, which has no 3D interface.
    """
    srfid: int
    components: List[Tuple[str, int, int, float]]
    prescribed_pressures: Dict[int, float] = field(default_factory=dict)
    prescribed_flows: Dict[int, float] = field(default_factory=dict)
    interface_component: int = 1
    initial_pressures: Dict[int, float] = field(default_factory=dict)
    volumes: Dict[int, Tuple[float, float]] = field(default_factory=dict)
    controllers: List[Tuple[str, int, object]] = field(default_factory=list)
    shared_nodes: Tuple[int, ...] = ()

    @property
    def nnodes(self) -> int:
        return max(max(s, e) for _, s, e, _ in self.components)

    @staticmethod
    def rcr(srfid: int, Rp: float = 100.0, C: float = 1e-4, Rd: float = 1000.0, Pd: float = 0.0) -> "NetlistBC":
        """The three-element Windkessel as a circuit: 1 -Rp- 2, 2 -C- 3 (ground),
        2 -Rd- 4 (distal pressure Pd)."""
        return NetlistBC(srfid=srfid, components=[("r", 1, 2, Rp), ("c", 2, 3, C), ("r", 2, 4, Rd)],
                         prescribed_pressures={3: 0.0, 4: Pd}, interface_component=1)


@dataclass
class FlowParams:
    rho: float = 1.06
    mu: float = 0.04
    rhoinf: float = 0.0
    Delt: float = 1e-3
    dtsfct: float = 1.0
    taucfct: float = 1.0
    idiff: int = 1
    iconvflow: int = 2
    stabflux_coeff: float = 0.5
    ibksiz: int = 255
    nitr: int = 3
    rescontrol: bool = False
    res_criteria: float = 0.0
    min_iters: int = 0
    epstol_mom: float = 1e-4
    epstol_cont: float = 1e-4
    epstol_ns: float = 1e-5
    kspace: int = 50
    ngmres: int = 10
    maxiters: int = 500
    nprjs: int = 10
    rcr: List[RCR] = field(default_factory=list)
    # netlist outlet circuits, coupled after the RCR surfaces (not reference
    # settings names: the reference reads them from its netlist XML input)
    netlists: List[NetlistBC] = field(default_factory=list)
    # closed loops of netlist circuits (NetlistLoopBC)
    loops: list = field(default_factory=list)
    # NS solve arithmetic: "fp64" (memLS's), "mixed" (FP32 matrices in the
    # inner Krylov matvecs, FP64 outer vectors and iterative refinement of at
    # most max_refine sweeps, until the FP64 defect |R - A x| / |R| is at
    # most refine_tol, epstol_ns when refine_tol <= 0) or "mixed_f32_tangent"
    # (mixed, and FP32 element quadrature of the tangent in the time step).
    # Not reference settings.
    precision: str = "fp64"
    max_refine: int = 4
    refine_tol: float = 0.0
    # Mixed precision only: 1 runs the inner CG on the explicit FP32 Schur
    # operator S = L - Gt G formed once per NS solve, 0 (default: measured
    # faster on the 4M-tet cylinder, 0.0739 vs 0.0765 ms per CG iteration) on
    # the two FP32 products L P and Gt (G P) (crimson_memls_ls_set_schur).
    explicit_schur: int = 0

    def outlets(self) -> list:
        """Coupled outlet surfaces in srflist order: the RCRs, the netlists,
        then the upstream circuits of each closed loop."""
        return list(self.rcr) + list(self.netlists) + [c for lp in self.loops for c in lp.upstream]

    @property
    def almi(self) -> float:
        return time_params(self.rhoinf)[0]

    @property
    def alfi(self) -> float:
        return time_params(self.rhoinf)[1]

    @property
    def gami(self) -> float:
        return time_params(self.rhoinf)[2]

    @property
    def Dtgl(self) -> float:
        return 1.0 / self.Delt


@dataclass
class NetlistLoopBC:
    """A closed loop of netlist circuits (flowsolver/src/
    ClosedLoopDownstreamSubsection.cxx): the upstream circuits coupled to 3D
    surfaces (input order), one loop-closing circuit (interface_component 0)
    and the connections (downstream node, upstream surface id, upstream
    node) in the order of the downstream input."""
    upstream: List[NetlistBC]
    downstream: NetlistBC
    connections: List[Tuple[int, int, int]]

    def upstream_index(self, srfid: int) -> int:
        for k, c in enumerate(self.upstream):
            if c.srfid == srfid:
                return k
        raise ValueError(f"surface {srfid} is not an upstream circuit of the loop")
