"""Host-side mirror of the reference's ElmGMR / memLS / SolFlow / time-step
interfaces, over the C ABI of libcrimson_b200.so.

* :class:`ElmGMR`   - ``ElmGMR(u,y,ac,x,...,iBC,BC,...,res,...,rowp,colm,lhsK,lhsP,...)``
  (flowsolver/src/elmgmr.f90:1-8) and ``genadj`` (flowsolver/src/genadj.f90:1).
* :class:`MemLS`    - ``memLS_LS_CREATE`` / ``memLS_LHS_CREATE`` / ``memLS_BC_CREATE``
  / ``memLS_SOLVE`` (flowsolver/src/memLS.f90:1379, 1080, 272, 1947).
* :class:`FlowSolver` - ``itrdrv_iter_step`` (flowsolver/src/itrdrv.f90:1239)
  with the SolFlow assembly + solve (flowsolver/src/solfar.f90:120-280) kept on
  the device between calls.

Arrays are numpy in the reference layouts (column-major, 1-based indices) at
this boundary, exactly what a Fortran caller would pass; device tensors
(torch) are accepted by the ``*_device`` methods.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Optional, Sequence

import numpy as np

from . import _native as N
from .problem import FlowParams


PRECISIONS = {"fp64": 0, "mixed": 1, "mixed_f32_tangent": 2}


def make_params(P: FlowParams) -> N.Params:
    return N.Params(rho=P.rho, mu=P.mu, alfi=P.alfi, almi=P.almi, gami=P.gami, Delt=P.Delt, Dtgl=1.0 / P.Delt,
                    dtsfct=P.dtsfct, taucfct=P.taucfct, flmpl=0.0, flmpr=0.0, stabflux_coeff=P.stabflux_coeff,
                    idiff=P.idiff, iconvflow=P.iconvflow, itau=0, ibksiz=P.ibksiz, ndofBC=7, nthreads=1)


def _f(a, dtype):
    return np.asfortranarray(np.asarray(a, dtype=dtype))


class ElmGMR:
    """Assembly context: mesh, boundary data and the device CSR pattern."""

    def __init__(self, mesh, P: FlowParams, srflist: Optional[Sequence[int]] = None):
        L = N.lib()
        self.mesh = mesh
        self.P = P
        self.nshg = mesh.nshg
        self.nelem = mesh.nelem
        self._prm = make_params(P)
        h = ctypes.c_void_p()
        ien = _f(mesh.ien.astype(np.int64) + 1, np.int32)
        x = _f(mesh.x, np.float64)
        N.check(L.crimson_ctx_create(ctypes.byref(h), ctypes.byref(self._prm), self.nshg, self.nshg, self.nelem,
                                     N.ip(ien), N.dp(x)), "crimson_ctx_create")
        self.h = h
        self.set_bc(mesh.iBC, mesh.BC)
        if mesh.ienb is not None and len(mesh.ienb):
            ienb = _f(mesh.ienb.astype(np.int64) + 1, np.int32)
            iBCB = _f(mesh.iBCB, np.int32)
            BCB = _f(mesh.BCB, np.float64)
            N.check(L.crimson_set_boundary(self.h, ienb.shape[0], N.ip(ienb), N.ip(iBCB), N.dp(BCB)),
                    "crimson_set_boundary")
        if srflist is None:
            srflist = [r.srfid for r in P.outlets()]
        self.srflist = list(srflist)
        if self.srflist:
            sl = np.asarray(self.srflist, dtype=np.int32)
            nd = np.ascontiguousarray(mesh.ndsurf.astype(np.int32))
            nabi = _f(mesh.NABI, np.float64)
            N.check(L.crimson_set_outlets(self.h, len(sl), N.ip(sl), N.ip(nd), N.dp(nabi)), "crimson_set_outlets")
        self.nnz = None

    def set_bc(self, iBC, BC) -> None:
        ib = np.ascontiguousarray(np.asarray(iBC, dtype=np.int32))
        bc = _f(BC, np.float64)
        N.check(N.lib().crimson_set_bc(self.h, N.ip(ib), N.dp(bc)), "crimson_set_bc")

    def genadj(self):
        """(colm, rowp), 1-based, as genadj returns them."""
        L = N.lib()
        nnz = ctypes.c_longlong(0)
        N.check(L.crimson_genadj(self.h, None, None, 0, ctypes.byref(nnz)), "crimson_genadj")
        self.nnz = nnz.value
        colm = np.zeros(self.nshg + 1, dtype=np.int32)
        rowp = np.zeros(self.nnz, dtype=np.int32)
        N.check(L.crimson_genadj(self.h, N.ip(colm), N.ip(rowp), self.nnz, ctypes.byref(nnz)), "crimson_genadj")
        return colm, rowp

    def _nnz(self) -> int:
        if self.nnz is None:
            nnz = ctypes.c_longlong(0)
            N.check(N.lib().crimson_genadj(self.h, None, None, 0, ctypes.byref(nnz)), "crimson_genadj")
            self.nnz = nnz.value
        return self.nnz

    @staticmethod
    def _coefs(coef1, coef2, n):
        if n == 0:
            return None, None
        c1 = np.ascontiguousarray(np.asarray(coef1 if coef1 is not None else np.zeros(n), dtype=np.float64))
        c2 = np.ascontiguousarray(np.asarray(coef2 if coef2 is not None else np.zeros(n), dtype=np.float64))
        return c1, c2

    def __call__(self, y, ac, coef1=None, coef2=None, lhs: bool = True):
        """res (nshg, 4), lhsK (nnz, 9), lhsP (nnz, 4) from host y, ac (nshg, 4)."""
        nnz = self._nnz()
        yF = _f(y, np.float64)
        aF = _f(ac, np.float64)
        res = np.zeros((self.nshg, 4), order="F")
        lhsK = np.zeros((nnz, 9)) if lhs else None
        lhsP = np.zeros((nnz, 4)) if lhs else None
        c1, c2 = self._coefs(coef1, coef2, len(self.srflist))
        N.check(N.lib().crimson_elmgmr(self.h, N.dp(yF), N.dp(aF), N.dp(c1), N.dp(c2), N.dp(res), N.dp(lhsK),
                                       N.dp(lhsP), 1 if lhs else 0), "crimson_elmgmr")
        return {"res": np.ascontiguousarray(res), "lhsK": lhsK, "lhsP": lhsP}

    def device(self, d_y, d_ac, d_res, d_lhsK=None, d_lhsP=None, coef1=None, coef2=None, lhs: bool = True) -> None:
        """Device-resident ElmGMR on torch tensors: y, ac, res (nshg, 4); lhsK (nnz, 9); lhsP (nnz, 4)."""
        c1, c2 = self._coefs(coef1, coef2, len(self.srflist))
        N.check(N.lib().crimson_elmgmr_device(self.h, d_y.data_ptr(), d_ac.data_ptr(), N.dp(c1), N.dp(c2),
                                              d_res.data_ptr(), d_lhsK.data_ptr() if lhs else None,
                                              d_lhsP.data_ptr() if lhs else None, 1 if lhs else 0),
                "crimson_elmgmr_device")

    def sclr(self, y, s, sdot, isclr: int = 1, diffus: float = 0.0, bcbs=None, lhs: bool = True):
        """ElmGMRSclr (flowsolver/src/elmgmr.f90:599-822) from host arrays:
        y (nshg, 4) the flow state, s and sdot (nshg) the scalar and its
        rate, bcbs (nface, 3) the prescribed fluxes of faces whose iBCB bit
        4 + isclr is set.  Returns res (nshg) and lhsS (nnz)."""
        nnz = self._nnz()
        yF = _f(y, np.float64)
        sv = np.ascontiguousarray(np.asarray(s, dtype=np.float64).reshape(-1))
        sd = np.ascontiguousarray(np.asarray(sdot, dtype=np.float64).reshape(-1))
        if yF.shape != (self.nshg, 4) or sv.size != self.nshg or sd.size != self.nshg:
            raise ValueError("y must be (nshg, 4) and s, sdot (nshg)")
        bF = _f(bcbs, np.float64) if bcbs is not None else None
        res = np.zeros(self.nshg)
        lhsS = np.zeros(nnz) if lhs else None
        N.check(N.lib().crimson_elmgmr_sclr(self.h, int(isclr), float(diffus), N.dp(yF), N.dp(sv), N.dp(sd),
                                            N.dp(bF), N.dp(res), N.dp(lhsS), 1 if lhs else 0),
                "crimson_elmgmr_sclr")
        return {"res": res, "lhsS": lhsS}

    def sclr_device(self, d_y, d_s, d_sdot, d_res, d_lhsS=None, isclr: int = 1, diffus: float = 0.0, d_bcbs=None,
                    lhs: bool = True) -> None:
        """Device-resident ElmGMRSclr on torch tensors: y (nshg, 4), s, sdot,
        res (nshg), bcbs (nface, 3), lhsS (nnz); on the context's stream."""
        N.check(N.lib().crimson_elmgmr_sclr_device(self.h, int(isclr), float(diffus), d_y.data_ptr(),
                                                   d_s.data_ptr(), d_sdot.data_ptr(),
                                                   d_bcbs.data_ptr() if d_bcbs is not None else None,
                                                   d_res.data_ptr(), d_lhsS.data_ptr() if lhs else None,
                                                   1 if lhs else 0), "crimson_elmgmr_sclr_device")

    @property
    def stream_handle(self) -> int:
        return N.lib().crimson_ctx_stream(self.h)

    def close(self) -> None:
        if getattr(self, "h", None):
            N.lib().crimson_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MemLS:
    """memLS NS solver: an ls handle plus an lhs (pattern + faces)."""

    def __init__(self, P: FlowParams, nfaces: int, nshg: int = 0, colm=None, rowp=None, ctx: Optional[ElmGMR] = None):
        L = N.lib()
        ls = ctypes.c_void_p()
        rin = np.array([P.epstol_mom, P.epstol_cont])
        ain = np.array([1e-10, 1e-10])
        mit = np.array([P.ngmres, P.maxiters], dtype=np.int32)
        N.check(L.crimson_memls_ls_create(ctypes.byref(ls), 3, 1 | 4 | 8 | 16 | 64, P.epstol_ns, 0.0, P.nprjs,
                                          P.kspace, N.dp(rin), N.dp(ain), N.ip(mit)), "crimson_memls_ls_create")
        self.ls = ls
        if P.precision not in PRECISIONS:
            L.crimson_memls_ls_free(ls)
            self.ls = None
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, got {P.precision!r}")
        N.check(L.crimson_memls_ls_set_precision(ls, PRECISIONS[P.precision], P.max_refine, P.refine_tol),
                "crimson_memls_ls_set_precision")
        N.check(L.crimson_memls_ls_set_schur(ls, int(P.explicit_schur)), "crimson_memls_ls_set_schur")
        lhs = ctypes.c_void_p()
        self._ctx = ctx   # an lhs made from a context must be freed before it
        if ctx is not None:
            N.check(L.crimson_memls_lhs_create_from_ctx(ctypes.byref(lhs), ctx.h, nfaces),
                    "crimson_memls_lhs_create_from_ctx")
            self.nshg = ctx.nshg
        else:
            colm = np.ascontiguousarray(colm, dtype=np.int32)
            rowp = np.ascontiguousarray(rowp, dtype=np.int32)
            gn = np.arange(1, nshg + 1, dtype=np.int32)
            N.check(L.crimson_memls_lhs_create(ctypes.byref(lhs), nshg, nshg, rowp.size, N.ip(gn), N.ip(colm),
                                               N.ip(rowp), nfaces), "crimson_memls_lhs_create")
            self.nshg = nshg
        self.lhs = lhs
        self.nfaces = nfaces

    def bc_create(self, faIn: int, gnodes0, dof: int, bctype: int, val) -> None:
        g = np.ascontiguousarray(np.asarray(gnodes0, dtype=np.int64) + 1, dtype=np.int32)
        v = np.ascontiguousarray(np.asarray(val, dtype=np.float64).reshape(len(g), dof))
        N.check(N.lib().crimson_memls_bc_create(self.lhs, faIn, len(g), dof, bctype, N.ip(g), N.dp(v)),
                "crimson_memls_bc_create")

    def solve(self, Res4, Val4, faceRes, incL=None):
        """memLS_SOLVE with host Ri (nshg, 4) and Val (nnz, 16); Val is scaled in place."""
        Ri = np.ascontiguousarray(np.array(Res4, dtype=np.float64))
        assert Val4.dtype == np.float64 and Val4.flags.c_contiguous
        fr = np.ascontiguousarray(np.asarray(faceRes, dtype=np.float64))
        inc = np.ones(self.nfaces, dtype=np.int32) if incL is None else np.ascontiguousarray(incL, dtype=np.int32)
        st = N.LsStats()
        N.check(N.lib().crimson_memls_solve(self.lhs, self.ls, 4, N.dp(Ri), N.dp(Val4), N.ip(inc), N.dp(fr),
                                            ctypes.byref(st)), "crimson_memls_solve")
        return Ri, st

    def solflow_device(self, ctx: ElmGMR, d_res, d_lhsK, d_lhsP, faceRes, d_sol, incL=None):
        fr = np.ascontiguousarray(np.asarray(faceRes, dtype=np.float64))
        inc = np.ones(self.nfaces, dtype=np.int32) if incL is None else np.ascontiguousarray(incL, dtype=np.int32)
        st = N.LsStats()
        N.check(N.lib().crimson_solflow_device(ctx.h, self.lhs, self.ls, d_res.data_ptr(), d_lhsK.data_ptr(),
                                               d_lhsP.data_ptr(), N.ip(inc), N.dp(fr), d_sol.data_ptr(),
                                               ctypes.byref(st)), "crimson_solflow_device")
        return st

    def set_log(self, path) -> None:
        """Append one memLS_NS.log-format line per solve to path (None: off)."""
        N.check(N.lib().crimson_memls_ls_set_log(self.ls, path.encode() if path else None),
                "crimson_memls_ls_set_log")

    def schur_info(self):
        """(state, nnz, sliced positions, average formation ms) of the explicit
        FP32 Schur operator on this lhs (state 1: in use, 0: not built, -1:
        the pattern does not allow it)."""
        st, nnz, npad, fm = ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_double()
        N.check(N.lib().crimson_memls_schur_info(self.lhs, ctypes.byref(st), ctypes.byref(nnz), ctypes.byref(npad),
                                                 ctypes.byref(fm)), "crimson_memls_schur_info")
        return st.value, nnz.value, npad.value, fm.value

    def refine_info(self):
        """(sweeps, relative FP64 defect) of the last mixed-precision solve."""
        steps = ctypes.c_int()
        rel = ctypes.c_double()
        N.check(N.lib().crimson_memls_refine_info(self.lhs, ctypes.byref(steps), ctypes.byref(rel)),
                "crimson_memls_refine_info")
        return steps.value, rel.value

    def close(self) -> None:
        L = N.lib()
        if getattr(self, "lhs", None):
            L.crimson_memls_lhs_free(self.lhs)
            self.lhs = None
        if getattr(self, "ls", None):
            L.crimson_memls_ls_free(self.ls)
            self.ls = None
        self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dirichlet_face(mesh):
    """memLS face 1: nodes with a prescribed velocity, val = 1 on free components
    (flowsolver/src/itrdrv.f90:949-992)."""
    iBC = mesh.iBC
    nodes = np.nonzero(((iBC >> 3) & 7) != 0)[0]
    sv = np.zeros((len(nodes), 3))
    sv[:, 0] = ((iBC[nodes] >> 3) & 1) == 0
    sv[:, 1] = ((iBC[nodes] >> 4) & 1) == 0
    sv[:, 2] = ((iBC[nodes] >> 5) & 1) == 0
    return nodes, sv


def neumann_face(mesh, srfid: int):
    """Coupled outlet face: nodes with ndsurf == srfid, val = NABI (itrdrv.f90:812-879)."""
    nodes = np.nonzero(mesh.ndsurf == srfid)[0]
    return nodes, mesh.NABI[nodes]


def _with_codes(mesh, iBC):
    """A view of mesh with other nodal codes."""
    import copy

    m = copy.copy(mesh)
    m.iBC = iBC
    return m


class FlowSolver:
    """Device-resident time stepping (itrdrv_iter_step) with RCR and netlist outlets."""

    def __init__(self, mesh, P: FlowParams, inflow: Optional[Callable[[float], float]] = None):
        self.mesh = mesh
        self.P = P
        self.elm = ElmGMR(mesh, P)
        self.elm._nnz()
        nc = len(self.elm.srflist)
        self.memls = MemLS(P, 1 + nc, ctx=self.elm)
        outlets = P.outlets()
        # a netlist surface starts from zero-velocity Dirichlet codes, which
        # crimson_step releases while the circuit takes flow and keeps while
        # its closed diodes block the interface (itrdrv.f90:1114-1133)
        iBC0 = np.asarray(mesh.iBC, dtype=np.int32).copy()
        for r in outlets:
            if hasattr(r, "components"):
                iBC0[mesh.ndsurf == r.srfid] |= 7 << 3
        if not np.array_equal(iBC0, mesh.iBC):
            self.elm.set_bc(iBC0, mesh.BC)
        nodes, sv = dirichlet_face(_with_codes(mesh, iBC0))
        self.memls.bc_create(1, nodes, 3, 0, sv)
        for k, r in enumerate(outlets):
            nn, vv = neumann_face(mesh, r.srfid)
            self.memls.bc_create(2 + k, nn, 3, 1, vv)
        L = N.lib()
        self.netlists, self.loops = [], []
        if nc:
            # RCR parameters per surface (zeros on netlist surfaces, whose
            # coefficients come from the circuit)
            arr = lambda f: np.ascontiguousarray(np.array([getattr(r, f, 0.0) for r in outlets], dtype=np.float64))
            N.check(L.crimson_set_rcr(self.elm.h, nc, N.dp(arr("Rp")), N.dp(arr("C")), N.dp(arr("Rd")),
                                      N.dp(arr("Pd"))), "crimson_set_rcr")
            from .netlist import Netlist, NetlistLoop

            in_loop = {id(c) for lp in P.loops for c in lp.upstream}
            for k, r in enumerate(outlets):
                if hasattr(r, "components") and id(r) not in in_loop:
                    nl = Netlist(r)
                    N.check(L.crimson_set_outlet_netlist(self.elm.h, k, nl.h), "crimson_set_outlet_netlist")
                    self.netlists.append(nl)
            pos = {id(r): k for k, r in enumerate(outlets)}
            for spec in P.loops:
                lp = NetlistLoop(spec)
                sf = np.array([pos[id(c)] for c in spec.upstream], dtype=np.int32)
                N.check(L.crimson_set_outlet_netlist_loop(self.elm.h, lp.h, N.ip(sf)), "crimson_set_outlet_netlist_loop")
                self.loops.append(lp)
        self.inflow = inflow if inflow is not None else (lambda t: 10.0)
        if mesh.inlet_nodes is not None and len(mesh.inlet_nodes):
            nodes1 = np.ascontiguousarray(mesh.inlet_nodes.astype(np.int64) + 1, dtype=np.int32)
            prof = np.ascontiguousarray(mesh.inlet_profile, dtype=np.float64)
            N.check(L.crimson_set_inflow(self.elm.h, len(nodes1), N.ip(nodes1), N.dp(prof)), "crimson_set_inflow")
        self.istep = 0
        y0 = np.zeros((mesh.nshg, 4))
        mesh.set_inflow(self.inflow(0.0))
        full = ((mesh.iBC >> 3) & 7) == 7
        y0[full, 0:3] = mesh.BC[full, 2:5]
        self.set_state(y0, np.zeros_like(y0))

    def set_state(self, y, ac) -> None:
        N.check(N.lib().crimson_state_set(self.elm.h, N.dp(_f(y, np.float64)), N.dp(_f(ac, np.float64))),
                "crimson_state_set")

    def state(self):
        y = np.zeros((self.mesh.nshg, 4), order="F")
        ac = np.zeros((self.mesh.nshg, 4), order="F")
        N.check(N.lib().crimson_state_get(self.elm.h, N.dp(y), N.dp(ac)), "crimson_state_get")
        return np.ascontiguousarray(y), np.ascontiguousarray(ac)

    def outlet_state(self):
        """(flows, mean pressures) of the coupled surfaces for the current
        state (crimson_outlet_state: GetFlowQ, integrScalar(p) / area)."""
        n = len(self.elm.srflist)
        q, p = np.zeros(n), np.zeros(n)
        N.check(N.lib().crimson_outlet_state(self.elm.h, n, N.dp(q), N.dp(p)), "crimson_outlet_state")
        return q, p

    def close(self) -> None:
        """Free the memLS handles, then the context they borrow from."""
        if getattr(self, "memls", None) is not None:
            self.memls.close()
            self.memls = None
        if getattr(self, "elm", None) is not None:
            self.elm.close()
            self.elm = None
        for nl in getattr(self, "netlists", []) + getattr(self, "loops", []):
            nl.close()
        self.netlists, self.loops = [], []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self) -> N.StepStats:
        t1 = self.P.Delt * (self.istep + 1)
        args = N.StepArgs(nitr=self.P.nitr, inflow_scale=self.inflow(t1), rescontrol=int(bool(self.P.rescontrol)),
                          res_criteria=float(self.P.res_criteria), min_iters=int(self.P.min_iters))
        st = N.StepStats()
        N.check(N.lib().crimson_step(self.elm.h, self.memls.lhs, self.memls.ls, ctypes.byref(args),
                                     ctypes.byref(st)), "crimson_step")
        self.istep += 1
        # the netlists' control systems, after the step's finalisation (itrdrv.f90:2100)
        circuits = self.netlists + [m for lp in self.loops for m in lp.members]
        bound = [(nl, t, i, c) for nl in circuits for t, i, c in nl.spec.controllers]
        if bound:
            from .controllers import run_controllers

            run_controllers(bound, self.P.Delt)
        return st
