"""ctypes binding of the CPU FP64 oracle (test infrastructure only).

Used by tests/, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` as
the checker and the timed CPU baseline.  The product path never imports it.

``OracleFlow`` sequences the oracle routines the way the reference's
``itrdrv_iter_step`` (flowsolver/src/itrdrv.f90:1239-1613) and ``SolFlow``
(flowsolver/src/solfar.f90:120-280) do: predict, itrBC, then per nonlinear
iteration y_alpha -> ElmGMR -> pack Res4/Val4 -> memLS_SOLVE -> correct ->
itrBC, then the RCR history update (RCR.cxx:49-81,
AbstractBoundaryCondition.cxx:32-91).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)
_c_ll_p = ctypes.POINTER(ctypes.c_longlong)


class OrcParams(ctypes.Structure):
    _fields_ = [("rho", ctypes.c_double), ("mu", ctypes.c_double), ("alfi", ctypes.c_double),
                ("almi", ctypes.c_double), ("gami", ctypes.c_double), ("Delt", ctypes.c_double),
                ("Dtgl", ctypes.c_double), ("dtsfct", ctypes.c_double), ("taucfct", ctypes.c_double),
                ("flmpl", ctypes.c_double), ("flmpr", ctypes.c_double), ("stabflux_coeff", ctypes.c_double),
                ("idiff", ctypes.c_int), ("iconvflow", ctypes.c_int), ("itau", ctypes.c_int),
                ("ibksiz", ctypes.c_int), ("ndofBC", ctypes.c_int), ("nthreads", ctypes.c_int)]


class OrcSubLs(ctypes.Structure):
    _fields_ = [("absTol", ctypes.c_double), ("relTol", ctypes.c_double), ("iNorm", ctypes.c_double),
                ("fNorm", ctypes.c_double), ("dB", ctypes.c_double), ("callD", ctypes.c_double),
                ("suc", ctypes.c_int), ("mItr", ctypes.c_int), ("sD", ctypes.c_int), ("itr", ctypes.c_int),
                ("cM", ctypes.c_int), ("cN", ctypes.c_int), ("cD", ctypes.c_int), ("reserve", ctypes.c_int)]


class OrcLsStats(ctypes.Structure):
    _fields_ = [("GM", OrcSubLs), ("CG", OrcSubLs), ("RI", OrcSubLs), ("LS_type", ctypes.c_int),
                ("Resm", ctypes.c_int), ("Resc", ctypes.c_int)]


def build() -> str:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        L.orc_genadj.argtypes = [ctypes.c_int, ctypes.c_int, _c_int_p, _c_int_p, _c_int_p, ctypes.c_longlong, _c_ll_p]
        L.orc_elmgmr.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_int_p,
                                 _c_dbl_p, _c_dbl_p, _c_dbl_p, _c_int_p, _c_dbl_p, ctypes.c_int, _c_int_p, _c_int_p,
                                 _c_dbl_p, ctypes.c_int, _c_int_p, _c_dbl_p, _c_dbl_p, _c_int_p, _c_dbl_p, _c_int_p,
                                 _c_int_p, ctypes.c_longlong, _c_dbl_p, _c_dbl_p, _c_dbl_p, ctypes.c_int, _c_dbl_p,
                                 _c_dbl_p]
        L.orc_getflowq.argtypes = [ctypes.c_int, _c_dbl_p, ctypes.c_int, _c_int_p, _c_int_p, _c_dbl_p, _c_dbl_p]
        L.orc_elmgmr_sclr.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, _c_int_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, _c_dbl_p,
                                      _c_int_p, ctypes.c_int, _c_int_p, _c_int_p, _c_dbl_p, _c_int_p, _c_int_p,
                                      ctypes.c_longlong, _c_dbl_p, _c_dbl_p, ctypes.c_int, _c_dbl_p]
        L.orc_solflow_pack.argtypes = [ctypes.c_int, ctypes.c_longlong, _c_int_p, _c_int_p, _c_dbl_p, _c_dbl_p,
                                       _c_dbl_p, _c_dbl_p, _c_dbl_p]
        L.orc_memls_ls_create.restype = ctypes.c_void_p
        L.orc_memls_ls_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, _c_dbl_p, _c_dbl_p, _c_int_p]
        L.orc_memls_ls_free.argtypes = [ctypes.c_void_p]
        L.orc_memls_lhs_create.restype = ctypes.c_void_p
        L.orc_memls_lhs_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_longlong, _c_int_p, _c_int_p,
                                           _c_int_p, ctypes.c_int]
        L.orc_memls_lhs_free.argtypes = [ctypes.c_void_p]
        L.orc_memls_bc_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          _c_int_p, _c_dbl_p]
        L.orc_memls_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, _c_dbl_p, _c_dbl_p, _c_int_p,
                                      _c_dbl_p, ctypes.POINTER(OrcLsStats)]
        L.orc_memls_set_threads.argtypes = [ctypes.c_int]
        L.orc_rcr_coeffs.argtypes = [ctypes.c_double] * 8 + [_c_dbl_p, _c_dbl_p]
        L.orc_itr_bc.argtypes = [ctypes.c_int, _c_int_p, _c_dbl_p, _c_dbl_p]
        _lib = L
    return _lib


def _ip(a):
    return a.ctypes.data_as(_c_int_p) if a is not None else None


def _dp(a):
    return a.ctypes.data_as(_c_dbl_p) if a is not None else None


def make_params(P, nthreads: int = 1) -> OrcParams:
    return OrcParams(rho=P.rho, mu=P.mu, alfi=P.alfi, almi=P.almi, gami=P.gami, Delt=P.Delt, Dtgl=1.0 / P.Delt,
                     dtsfct=P.dtsfct, taucfct=P.taucfct, flmpl=0.0, flmpr=0.0, stabflux_coeff=P.stabflux_coeff,
                     idiff=P.idiff, iconvflow=P.iconvflow, itau=0, ibksiz=P.ibksiz, ndofBC=7, nthreads=nthreads)


def genadj(ien0: np.ndarray, nshg: int):
    """colm (nshg+1) and rowp (nnz), 1-based, from 0-based ien (nelem, 4)."""
    L = lib()
    ienF = np.asfortranarray(ien0.astype(np.int32) + 1)
    colm = np.zeros(nshg + 1, dtype=np.int32)
    nnz = ctypes.c_longlong(0)
    rc = L.orc_genadj(nshg, ien0.shape[0], _ip(ienF), _ip(colm), None, 0, ctypes.byref(nnz))
    assert rc == 0
    rowp = np.zeros(nnz.value, dtype=np.int32)
    rc = L.orc_genadj(nshg, ien0.shape[0], _ip(ienF), _ip(colm), _ip(rowp), nnz.value, ctypes.byref(nnz))
    assert rc == 0, rc
    return colm, rowp


class Elm:
    """Holds Fortran-ordered mesh arrays for repeated ElmGMR calls."""

    def __init__(self, mesh, P, colm, rowp, nthreads: int = 1):
        self.m = mesh
        self.P = P
        self.prm = make_params(P, nthreads)
        self.ienF = np.asfortranarray(mesh.ien.astype(np.int32) + 1)
        self.xF = np.asfortranarray(mesh.x)
        self.colm, self.rowp = colm, rowp
        self.nnz = int(rowp.size)
        if mesh.ienb is not None and len(mesh.ienb):
            self.nface = mesh.ienb.shape[0]
            self.ienbF = np.asfortranarray(mesh.ienb.astype(np.int32) + 1)
            self.iBCBF = np.asfortranarray(mesh.iBCB.astype(np.int32))
            self.BCBF = np.asfortranarray(mesh.BCB)
        else:
            self.nface = 0
            self.ienbF = np.zeros((1, 4), dtype=np.int32, order="F")
            self.iBCBF = np.zeros((1, 2), dtype=np.int32, order="F")
            self.BCBF = np.zeros((1, 3, 6), order="F")
        self.iBC = np.ascontiguousarray(mesh.iBC.astype(np.int32))
        self.BCF = np.asfortranarray(mesh.BC)
        self.ndsurf = np.ascontiguousarray(mesh.ndsurf.astype(np.int32))
        self.NABIF = np.asfortranarray(mesh.NABI)

    def __call__(self, y, ac, lhs=True, srflist=None, coef1=None, coef2=None, want_q=False):
        L = lib()
        m = self.m
        nshg = m.nshg
        yF = np.asfortranarray(y, dtype=np.float64)
        acF = np.asfortranarray(ac, dtype=np.float64)
        res = np.zeros((nshg, 4), order="F")
        lhsK = np.zeros((self.nnz, 9)) if lhs else None
        lhsP = np.zeros((self.nnz, 4)) if lhs else None
        qres = np.zeros((nshg, 9), order="F") if want_q else None
        rmass = np.zeros(nshg) if want_q else None
        nc = 0 if srflist is None else len(srflist)
        sl = np.ascontiguousarray(np.asarray(srflist if nc else [0], dtype=np.int32))
        c1 = np.ascontiguousarray(np.asarray(coef1 if nc else [0.0], dtype=np.float64))
        c2 = np.ascontiguousarray(np.asarray(coef2 if nc else [0.0], dtype=np.float64))
        self.BCF = np.asfortranarray(m.BC)
        rc = L.orc_elmgmr(ctypes.byref(self.prm), nshg, nshg, m.nelem, _ip(self.ienF), _dp(self.xF), _dp(yF),
                          _dp(acF), _ip(self.iBC), _dp(self.BCF), self.nface, _ip(self.ienbF), _ip(self.iBCBF),
                          _dp(self.BCBF), nc, _ip(sl), _dp(c1), _dp(c2), _ip(self.ndsurf), _dp(self.NABIF),
                          _ip(self.colm), _ip(self.rowp), self.nnz, _dp(res), _dp(lhsK), _dp(lhsP), 1 if lhs else 0,
                          _dp(qres), _dp(rmass))
        if rc != 0:
            raise RuntimeError(f"orc_elmgmr failed rc={rc}")
        out = {"res": np.ascontiguousarray(res), "lhsK": lhsK, "lhsP": lhsP}
        if want_q:
            out["qres"] = np.ascontiguousarray(qres)
            out["rmass"] = rmass
        return out


def elmgmr_sclr(elm, y, s, sdot, isclr=1, diffus=0.2, bcbs=None, lhs=True):
    """ElmGMRSclr (elmgmr.f90:599-822) on the oracle: res (nshg), lhsS (nnz),
    qres (nshg, 3).  elm is an :class:`Elm` (mesh arrays and pattern)."""
    L = lib()
    m = elm.m
    nshg = m.nshg
    yF = np.asfortranarray(y, dtype=np.float64)
    sv = np.ascontiguousarray(s, dtype=np.float64)
    sd = np.ascontiguousarray(sdot, dtype=np.float64)
    res = np.zeros(nshg)
    lhsS = np.zeros(elm.nnz) if lhs else None
    qres = np.zeros((nshg, 3), order="F")
    bF = np.asfortranarray(bcbs, dtype=np.float64) if bcbs is not None else None
    rc = L.orc_elmgmr_sclr(ctypes.byref(elm.prm), isclr, diffus, nshg, nshg, m.nelem, _ip(elm.ienF), _dp(elm.xF),
                           _dp(yF), _dp(sv), _dp(sd), _ip(elm.iBC), elm.nface, _ip(elm.ienbF), _ip(elm.iBCBF),
                           _dp(bF), _ip(elm.colm), _ip(elm.rowp), elm.nnz, _dp(res), _dp(lhsS), 1 if lhs else 0,
                           _dp(qres))
    if rc != 0:
        raise RuntimeError(f"orc_elmgmr_sclr failed rc={rc}")
    return {"res": res, "lhsS": lhsS, "qres": np.ascontiguousarray(qres)}


def getflowq(mesh, y, srflist):
    L = lib()
    q = np.zeros(len(srflist))
    sl = np.asarray(srflist, dtype=np.int32)
    L.orc_getflowq(mesh.nshg, _dp(np.asfortranarray(y)), len(srflist), _ip(sl),
                   _ip(np.ascontiguousarray(mesh.ndsurf.astype(np.int32))), _dp(np.asfortranarray(mesh.NABI)),
                   _dp(q))
    return q


def solflow_pack(nshg, colm, rowp, res, lhsK, lhsP):
    L = lib()
    nnz = rowp.size
    Res4 = np.zeros((nshg, 4))
    Val4 = np.zeros((nnz, 16))
    L.orc_solflow_pack(nshg, nnz, _ip(colm), _ip(rowp), _dp(np.asfortranarray(res)), _dp(np.ascontiguousarray(lhsK)),
                       _dp(np.ascontiguousarray(lhsP)), _dp(Res4), _dp(Val4))
    return Res4, Val4


def rcr_coeffs(Rp, C, Rd, Pdn, Pdn1, Pn, Qn, alfi_delt):
    s = ctypes.c_double()
    o = ctypes.c_double()
    lib().orc_rcr_coeffs(Rp, C, Rd, Pdn, Pdn1, Pn, Qn, alfi_delt, ctypes.byref(s), ctypes.byref(o))
    return s.value, o.value


class MemLS:
    """memLS lhs + ls handles (memLS_LHS_CREATE / memLS_LS_CREATE / memLS_BC_CREATE)."""

    def __init__(self, nshg, colm, rowp, nfaces, P, nthreads: int = 1):
        L = lib()
        self.nshg = nshg
        self.nnz = rowp.size
        gn = np.arange(1, nshg + 1, dtype=np.int32)
        self.lhs = L.orc_memls_lhs_create(nshg, nshg, self.nnz, _ip(gn), _ip(colm), _ip(rowp), nfaces)
        rin = np.array([P.epstol_mom, P.epstol_cont])
        ain = np.array([1e-10, 1e-10])
        min_ = np.array([P.ngmres, P.maxiters], dtype=np.int32)
        self.ls = L.orc_memls_ls_create(3, 1 | 4 | 8 | 16 | 64, P.epstol_ns, 0.0, P.nprjs, P.kspace, _dp(rin),
                                        _dp(ain), _ip(min_))
        self.nthreads = nthreads

    def bc_create(self, faIn, gnodes0, dof, bctype, val):
        g = np.ascontiguousarray(np.asarray(gnodes0, dtype=np.int32) + 1)
        v = np.ascontiguousarray(np.asarray(val, dtype=np.float64).reshape(len(g), dof))
        rc = lib().orc_memls_bc_create(self.lhs, faIn, len(g), dof, bctype, _ip(g), _dp(v))
        assert rc == 0

    def solve(self, Res4, Val4, faceRes):
        L = lib()
        L.orc_memls_set_threads(self.nthreads)
        Ri = np.ascontiguousarray(Res4.copy())
        inc = np.ones(len(faceRes), dtype=np.int32)
        fr = np.ascontiguousarray(np.asarray(faceRes, dtype=np.float64))
        st = OrcLsStats()
        rc = L.orc_memls_solve(self.lhs, self.ls, 4, _dp(Ri), _dp(Val4), _ip(inc), _dp(fr), ctypes.byref(st))
        if rc != 0:
            raise RuntimeError(f"orc_memls_solve failed rc={rc}")
        return Ri, st

    def __del__(self):
        try:
            L = lib()
            L.orc_memls_lhs_free(self.lhs)
            L.orc_memls_ls_free(self.ls)
        except Exception:
            pass


def itr_bc(mesh, y):
    """itrBC (flowsolver/src/itrbc.f90:33-101) in place on y (nshg, 4): the
    velocity components a node's iBC prescribes (all three, or one or two
    through the BC coefficients) and the prescribed pressure."""
    n = mesh.nshg
    yF = np.asfortranarray(y)
    iBC = np.ascontiguousarray(mesh.iBC.astype(np.int32))
    BCF = np.asfortranarray(mesh.BC)
    lib().orc_itr_bc(n, _ip(iBC), _dp(BCF), _dp(yF))
    y[:] = yF


def dirichlet_face(mesh):
    """Face 1: nodes with any prescribed velocity, val = 1 on free comps (itrdrv.f90:949-992)."""
    iBC = mesh.iBC
    nodes = np.nonzero(((iBC >> 3) & 7) != 0)[0]
    sv = np.zeros((len(nodes), 3))
    sv[:, 0] = ((iBC[nodes] >> 3) & 1) == 0
    sv[:, 1] = ((iBC[nodes] >> 4) & 1) == 0
    sv[:, 2] = ((iBC[nodes] >> 5) & 1) == 0
    return nodes, sv


def neumann_face(mesh, srfid):
    """Coupled outlet face: nodes with ndsurf == srfid, val = NABI (itrdrv.f90:812-879)."""
    nodes = np.nonzero(mesh.ndsurf == srfid)[0]
    return nodes, mesh.NABI[nodes]


def pressure_nodes(mesh, srfid):
    """The nodes integrScalar sums over for surface srfid
    (boundarydata.f90:1101-1140): ndsurf == srfid, and the edge nodes of the
    wall (ndsurf 1) whose edsurf is srfid (boundarydata.f90:186-253: the
    last face of a surface > 1 touching the node), ascending."""
    ed = np.zeros(mesh.nshg, dtype=np.int64)
    for f in range(mesh.ienb.shape[0]):
        s = int(mesh.iBCB[f, 1])
        if s > 1:
            for a in range(3):
                nd = mesh.ienb[f, a]
                if mesh.ndsurf[nd] == 1:
                    ed[nd] = s
    return np.nonzero((mesh.ndsurf == srfid) | ((mesh.ndsurf == 1) & (ed == srfid)))[0]


def surface_areas(mesh):
    """NASC (AsBNASC, asbnabi.f90:191-340): per node the integral of its
    shape function over the faces with the natural-pressure bit, the 3-point
    triangle rule, faces in order and each face's points summed first."""
    B3, C3, A3 = 0.666666666666667, 0.166666666666667, 0.3333333333333330
    r3 = ((B3, C3, C3), (C3, B3, C3), (C3, C3, B3))
    x = mesh.x
    nasc = np.zeros(mesh.nshg)
    for f in range(mesh.ienb.shape[0]):
        if not (int(mesh.iBCB[f, 0]) >> 1) & 1:
            continue
        nd = mesh.ienb[f, :3]
        v1 = x[nd[1]] - x[nd[0]]
        v2 = x[nd[2]] - x[nd[0]]
        t1 = v1[1] * v2[2] - v2[1] * v1[2]
        t2 = v2[0] * v1[2] - v1[0] * v2[2]
        t3 = v1[0] * v2[1] - v2[0] * v1[1]
        temp = 1.0 / np.sqrt(t1 * t1 + t2 * t2 + t3 * t3)
        rl = [0.0, 0.0, 0.0]
        for q in range(3):
            w = (2.0 * A3) / (4.0 * temp)
            for a in range(3):
                rl[a] = rl[a] + r3[q][a] * w
        for a in range(3):
            nasc[nd[a]] = nasc[nd[a]] + rl[a]
    return nasc


def netlist_surface_codes(mesh, outlets):
    """The codes a netlist surface starts from: zero-velocity Dirichlet codes
    on its nodes (ndsurf), released while the circuit takes flow
    (itrdrv.f90:1114-1133)."""
    iBC = mesh.iBC.copy()
    for r in outlets:
        if hasattr(r, "components"):
            nodes = np.nonzero(mesh.ndsurf == r.srfid)[0]
            iBC[nodes] = iBC[nodes] | (7 << 3)
    return iBC


class OracleFlow:
    """Time stepper over the oracle routines (itrdrv_iter_step + SolFlow).

    Netlist outlets: the surface nodes start from zero-velocity Dirichlet
    codes; each step the codes are iBC_original with zeros on every coupled
    surface that takes flow, and memLS's face 1 follows them; a netlist
    whose closed diodes block the interface is not coupled that step and is
    updated with the surface's mean pressure (NASC-weighted) at its end."""

    def __init__(self, mesh, P, nthreads: int = 1, inflow=None):
        import copy

        self.P = P
        self.nthreads = nthreads
        # coupled outlets: RCRs, then netlist circuits (netlist_oracle.py)
        self.rcr = P.outlets() if hasattr(P, "outlets") else list(P.rcr)
        self.srflist = [r.srfid for r in self.rcr]
        self.m = copy.copy(mesh)
        self.iBC_orig = netlist_surface_codes(mesh, self.rcr)
        self.m.iBC = self.iBC_orig.copy()
        self.colm, self.rowp = genadj(mesh.ien, mesh.nshg)
        self.elm = Elm(self.m, P, self.colm, self.rowp, nthreads)
        from oracle.netlist_oracle import OracleLoop, OracleNetlist

        self.netlists = [OracleNetlist(r) if hasattr(r, "components") else None for r in self.rcr]
        # closed loops: their upstream circuits are the outlets' circuits
        self.loops, self.loop_surfaces = [], []
        pos = {id(r): k for k, r in enumerate(self.rcr)}
        for spec in getattr(P, "loops", []):
            sf = [pos[id(c)] for c in spec.upstream]
            self.loops.append(OracleLoop([self.netlists[k] for k in sf], OracleNetlist(spec.downstream),
                                         [(d, spec.upstream_index(s), u) for d, s, u in spec.connections]))
            self.loop_surfaces.append(sf)
        self.in_loop = {k for sf in self.loop_surfaces for k in sf}
        self.onodes = [np.nonzero(mesh.ndsurf == s)[0] for s in self.srflist]
        self.nasc = surface_areas(mesh) if any(nl is not None for nl in self.netlists) else None
        self.pnodes = [pressure_nodes(mesh, s) for s in self.srflist]
        self.memls = MemLS(mesh.nshg, self.colm, self.rowp, 1 + len(self.rcr), P, nthreads)
        nodes, sv = dirichlet_face(self.m)
        self.memls.bc_create(1, nodes, 3, 0, sv)
        for k, r in enumerate(self.rcr):
            nn, vv = neumann_face(mesh, r.srfid)
            self.memls.bc_create(2 + k, nn, 3, 1, vv)
        self.inflow = inflow if inflow is not None else (lambda t: 10.0)
        n = mesh.nshg
        self.yold = np.zeros((n, 4))
        self.acold = np.zeros((n, 4))
        self.y = np.zeros((n, 4))
        self.ac = np.zeros((n, 4))
        self.istep = 0
        self.Pn = np.zeros(len(self.rcr))
        self.Qn = np.zeros(len(self.rcr))
        self.stats = []
        self.res_iter = 0      # residual control: iterations since the last early exit
        self.res_norms = []
        mesh.set_inflow(self.inflow(0.0))
        self._itr_bc(self.yold)

    def _itr_bc(self, y):
        """itrBC (itrbc.f90:33-101) in place on y (nshg, 4)."""
        itr_bc(self.m, y)

    def _blocked(self, k):
        return self.netlists[k] is not None and not self.netlists[k].permitted

    def _set_codes(self):
        """iBC = iBC_original, zero on the coupled surfaces that take flow;
        face 1 rebuilt when the codes change (rebuildMemLS_lhs)."""
        codes = self.iBC_orig.copy()
        for k in range(len(self.rcr)):
            if not self._blocked(k):
                codes[self.onodes[k]] = 0
        if not np.array_equal(codes, self.m.iBC):
            self.m.iBC = codes
            self.elm.iBC = np.ascontiguousarray(codes.astype(np.int32))
            nodes, sv = dirichlet_face(self.m)
            self.memls.bc_create(1, nodes, 3, 0, sv)

    def implicit_coeffs(self, n, alpha_form=True):
        P = self.P
        c1 = np.zeros(len(self.rcr))
        c2 = np.zeros(len(self.rcr))
        for lp, sf in zip(self.loops, self.loop_surfaces):
            for k, (a, b) in zip(sf, lp.implicit_coefficients(P.alfi * P.Delt if alpha_form else P.Delt)):
                c1[k], c2[k] = a, b
        for k, r in enumerate(self.rcr):
            if self._blocked(k):
                c1[k] = c2[k] = 0.0
                continue
            if k in self.in_loop:
                continue
            if self.netlists[k] is not None:
                c1[k], c2[k] = self.netlists[k].implicit_coefficients(P.alfi * P.Delt if alpha_form else P.Delt)
            elif alpha_form:
                c1[k], c2[k] = rcr_coeffs(r.Rp, r.C, r.Rd, r.Pd, r.Pd, self.Pn[k], self.Qn[k], P.alfi * P.Delt)
            else:
                c1[k], c2[k] = rcr_coeffs(r.Rp, r.C, r.Rd, r.Pd, r.Pd, self.Pn[k], self.Qn[k], P.Delt)
        return c1, c2

    def _res_control(self, res):
        """Residual control (itrdrv.f90:1516-1522): totres of rstatic.f90
        counted per assembled iteration; True ends the step early."""
        totres = float(np.sqrt(np.sum(np.asarray(res, dtype=float) ** 2) / self.m.nshg))
        self.res_norms.append(totres)
        self.res_iter += 1
        if totres < self.P.res_criteria and self.res_iter >= self.P.min_iters:
            self.res_iter = 0
            return True
        return False

    def solflow(self, c1, c2, stop=None):
        P = self.P
        yA = self.y.copy()
        acA = self.ac.copy()
        # itrYAlpha (itrPC.f90:326-336)
        yA[:, 0:3] = self.yold[:, 0:3] + P.alfi * (self.y[:, 0:3] - self.yold[:, 0:3])
        acA[:, 0:3] = self.acold[:, 0:3] + P.almi * (self.ac[:, 0:3] - self.acold[:, 0:3])
        acA[:, 3] = 0.0
        yA[:, 3] = self.y[:, 3]
        out = self.elm(yA, acA, lhs=True, srflist=self.srflist, coef1=c1, coef2=c2)
        if stop is not None and stop(out["res"]):
            return None
        Res4, Val4 = solflow_pack(self.m.nshg, self.colm, self.rowp, out["res"], out["lhsK"], out["lhsP"])
        faceRes = np.zeros(1 + len(self.rcr))
        faceRes[1:] = c1
        faceRes = faceRes * P.alfi * P.gami * P.Delt
        sol, st = self.memls.solve(Res4, Val4, faceRes)
        return sol, st, out

    def step(self):
        P = self.P
        n = self.istep
        t1 = P.Delt * (n + 1)
        self.m.set_inflow(self.inflow(t1))
        # itrPredict, ipred = 1
        fct = (P.gami - 1.0) / P.gami
        self.y = self.yold.copy()
        self.ac = self.acold * fct
        self._set_codes()
        self._itr_bc(self.y)
        c1, c2 = self.implicit_coeffs(n, True)
        for _ in range(P.nitr):
            r = self.solflow(c1, c2, stop=self._res_control if getattr(P, "rescontrol", False) else None)
            if r is None:
                break
            sol, st, _out = r
            self.stats.append((st.RI.itr, st.GM.itr, st.CG.itr, st.RI.iNorm, st.RI.fNorm))
            # itrCorrect (itrPC.f90:176-182)
            self.y[:, 0:3] = self.y[:, 0:3] + (P.gami * P.Delt) * sol[:, 0:3]
            self.y[:, 3] = self.y[:, 3] + (P.gami * P.alfi * P.Delt) * sol[:, 3]
            self.ac[:, 0:3] = self.ac[:, 0:3] + sol[:, 0:3]
            self._itr_bc(self.y)
        # RCR history update at n+1; netlists: updateLPN + finalizeLPNAtEndOfTimestep
        if self.rcr:
            q1 = getflowq(self.m, self.y, self.srflist)
            d1, h1 = self.implicit_coeffs(n, False)
            Pn = d1 * q1 + h1

            def p3d(k):
                # integrScalar(p) / area (elmgmr.f90:1733-1743), edge nodes included
                w = self.nasc[self.pnodes[k]]
                return float(np.sum(w * self.y[self.pnodes[k], 3]) / np.sum(w))

            for lp, sf in zip(self.loops, self.loop_surfaces):
                lp.update(P.Delt, [q1[k] for k in sf], [0.0 if lp.up[j].permitted else p3d(k)
                                                         for j, k in enumerate(sf)])
                lp.finalize_step()
            for k, nl in enumerate(self.netlists):
                if nl is not None:
                    if k not in self.in_loop:
                        if nl.permitted:
                            nl.update(P.Delt, q1[k])
                        else:
                            nl.update_pressure(P.Delt, p3d(k))
                        nl.finalize_step()
                    Pn[k] = nl.interface_pressure()
            self.Pn = Pn
            self.Qn = q1
        self.yold = self.y.copy()
        self.acold = self.ac.copy()
        self.istep += 1
        # control systems after the finalisation (itrdrv.f90:2100)
        bound = [(nl, t, i, c) for nl, r in zip(self.netlists, self.rcr) if nl is not None
                 for t, i, c in r.controllers]
        bound += [(lp.down, t, i, c) for lp, spec in zip(self.loops, getattr(P, "loops", []))
                  for t, i, c in spec.downstream.controllers]
        if bound:
            from oracle.netlist_oracle import run_controllers

            run_controllers(bound, self.P.Delt)
