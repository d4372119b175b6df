"""Seeded synthetic linear-tet meshes and boundary data for the assembly/solve path.

The reference reads meshes from PHASTA ``geombc`` files written by its
presolver.  The benchmark workloads here are synthetic stand-ins with the
shapes, sizes and boundary-condition layout of the reference's use case
(vascular tubes with a Dirichlet inflow, no-slip rigid wall and coupled
outlets):

* :func:`cylinder` - straight tube: a structured hex grid whose cross-section
  is masked to the disc (cells whose centre lies inside radius R), split into
  6 tets per hex, interior nodes jittered.
* :func:`lattice` - a jittered 3-D lattice of linear tets with random nodal
  states (the assembly / SpMV microbenchmark).
* :func:`bifurcation` - a Y-shaped tube swept from jittered structured rings
  along three centrelines.

All node and element numbering is 0-based here; the C-ABI boundary converts to
the reference's 1-based convention where it mirrors a Fortran interface.

Boundary data follow the reference's conventions:

* ``iBC`` bits 3,4,5 mark prescribed x1,x2,x3 velocity (flowsolver/src/
  bc3res.f90:46-113, ``ibits(iBC,3,3)``); ``BC[:,2:5]`` hold the prescribed
  velocity for the all-three-components case (flowsolver/src/itrbc.f90:83-87).
* boundary faces carry ``iBCB`` = (flag bits, surface id) and ``BCB`` values
  per face node (flowsolver/src/e3b.f90:19-33); outlet faces use the
  natural-pressure bit 1 with zero ``BCB`` pressure, as the reference's
  coupled and zero-pressure surfaces do (e3b.f90:281-300).
* ``NABI`` = integral of N_a n over the pressure-flagged faces and ``ndsurf``
  follow flowsolver/src/asbnabi.f90:108-140.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

# Surface ids: 1 = wall (sticky in ndsurf, asbnabi.f90:131-135), 2 = inlet, 3.. = outlets.
SRF_WALL = 1
SRF_INLET = 2
SRF_OUTLET0 = 3

NDOFBC = 7  # BC(nshg, ndofBC) columns used on this path (itrbc.f90, bc3res.f90)

# Kuhn split of a hex (vertex v = dx + 2*dy + 4*dz) into 6 tets sharing the
# main diagonal 0-7; conforming when every hex uses the same split.
_KUHN = np.array([
    [0, 1, 3, 7], [0, 1, 5, 7], [0, 2, 3, 7],
    [0, 2, 6, 7], [0, 4, 5, 7], [0, 4, 6, 7]], dtype=np.int64)

# 3-point triangle rule of the reference boundary quadrature (symtri.c rst3/wt3,
# weights doubled in genint.f90:86) evaluated with the tet shape functions as
# genshpb.f90:31-36 does: par = (B, C, C) and L4 = 1 - B - C - C.
_TRI_B = 0.666666666666667
_TRI_C = 0.166666666666667
_TRI_W = 0.3333333333333330000000000000000000


def _tri_shape_table() -> np.ndarray:
    pts = [(_TRI_B, _TRI_C, _TRI_C), (_TRI_C, _TRI_B, _TRI_C), (_TRI_C, _TRI_C, _TRI_B)]
    tab = np.zeros((3, 4))
    for q, (r, s, t) in enumerate(pts):
        tab[q] = (r, s, t, 1.0 - r - s - t)
    return tab


@dataclass
class Mesh:
    x: np.ndarray                      # (numnp, 3) float64
    ien: np.ndarray                    # (nelem, 4) int32, 0-based
    name: str = "mesh"
    ienb: Optional[np.ndarray] = None  # (nface, 4) int32, face nodes first, opposite node last
    iBCB: Optional[np.ndarray] = None  # (nface, 2) int32: flag bits, surface id
    BCB: Optional[np.ndarray] = None   # (nface, 3, 6) float64
    iBC: Optional[np.ndarray] = None   # (nshg,) int32
    BC: Optional[np.ndarray] = None    # (nshg, NDOFBC) float64
    ndsurf: Optional[np.ndarray] = None  # (nshg,) int32
    NABI: Optional[np.ndarray] = None  # (nshg, 3) float64
    inlet_nodes: Optional[np.ndarray] = None
    inlet_profile: Optional[np.ndarray] = None   # (n_inlet, 3) velocity for unit mean speed
    outlets: List[int] = field(default_factory=list)

    @property
    def nshg(self) -> int:
        return int(self.x.shape[0])

    @property
    def nelem(self) -> int:
        return int(self.ien.shape[0])

    def set_inflow(self, mean_speed: float) -> None:
        """Write the inflow profile scaled to ``mean_speed`` into BC[:, 2:5]."""
        if self.inlet_nodes is None or len(self.inlet_nodes) == 0:
            return
        self.BC[self.inlet_nodes, 2:5] = self.inlet_profile * mean_speed


def _orient(x: np.ndarray, ien: np.ndarray) -> np.ndarray:
    """Order tet nodes the reference's way: det[x1-x4, x2-x4, x3-x4] > 0.

    The reference Jacobian is dxdxi(:,j) = (x_j - x_4)/2 (e3metric.f90:26-38
    with the halved linear-tet shgl), so WdetJ > 0 needs the face (1,2,3)
    normal (x2-x1)x(x3-x1) to point away from node 4 - the opposite of the
    usual right-handed ordering.  Nodes 2,3 are swapped where needed.
    """
    a = x[ien[:, 1]] - x[ien[:, 0]]
    b = x[ien[:, 2]] - x[ien[:, 0]]
    c = x[ien[:, 3]] - x[ien[:, 0]]
    vol = np.einsum("ij,ij->i", a, np.cross(b, c))
    neg = vol > 0
    ien = ien.copy()
    ien[neg, 1], ien[neg, 2] = ien[neg, 2].copy(), ien[neg, 1].copy()
    return ien


def _hex_to_tets(hex_nodes: np.ndarray) -> np.ndarray:
    """hex_nodes (nhex, 8) in v = dx + 2dy + 4dz order -> (6*nhex, 4) tets."""
    tets = hex_nodes[:, _KUHN]            # (nhex, 6, 4)
    return tets.reshape(-1, 4)


def _boundary_faces(ien: np.ndarray) -> np.ndarray:
    """Faces that belong to exactly one tet: (nface, 4) = 3 face nodes + opposite node."""
    nel = ien.shape[0]
    loc = np.array([[1, 2, 3, 0], [0, 2, 3, 1], [0, 1, 3, 2], [0, 1, 2, 3]])
    allf = ien[:, loc].reshape(-1, 4)              # (4*nel, 4)
    key = np.sort(allf[:, :3], axis=1).astype(np.int64)
    nmax = int(ien.max()) + 1
    k = (key[:, 0] * nmax + key[:, 1]) * nmax + key[:, 2] if nmax < 2 ** 21 else None
    if k is None:
        view = np.ascontiguousarray(key).view(np.dtype((np.void, 24))).ravel()
        _, inv, cnt = np.unique(view, return_inverse=True, return_counts=True)
    else:
        _, inv, cnt = np.unique(k, return_inverse=True, return_counts=True)
    once = cnt[inv] == 1
    return allf[once]


def _orient_faces_outward(x: np.ndarray, fb: np.ndarray) -> np.ndarray:
    v1 = x[fb[:, 1]] - x[fb[:, 0]]
    v2 = x[fb[:, 2]] - x[fb[:, 0]]
    n = np.cross(v1, v2)
    inward = np.einsum("ij,ij->i", n, x[fb[:, 3]] - x[fb[:, 0]]) > 0
    fb = fb.copy()
    fb[inward, 1], fb[inward, 2] = fb[inward, 2].copy(), fb[inward, 1].copy()
    return fb


def compute_nabi(x: np.ndarray, ienb: np.ndarray, iBCB: np.ndarray, nshg: int):
    """NABI(i,:) = sum over pressure-flagged faces of N_i n dGamma, and ndsurf.

    Follows flowsolver/src/asbnabi.f90:39-140 for linear tets (lcsyst = 1):
    bnorm from (x2-x1) x (x3-x1), WdetJb = Qwtb/(4*temp) with temp = 1/|n|,
    boundary shape values of genshpb.f90, and the sticky surface 1 rule when
    pushing face ids to ``ndsurf``.
    """
    tab = _tri_shape_table()
    qwtb = 2.0 * _TRI_W
    v1 = x[ienb[:, 1]] - x[ienb[:, 0]]
    v2 = x[ienb[:, 2]] - x[ienb[:, 0]]
    t1 = v1[:, 1] * v2[:, 2] - v2[:, 1] * v1[:, 2]
    t2 = v2[:, 0] * v1[:, 2] - v1[:, 0] * v2[:, 2]
    t3 = v1[:, 0] * v2[:, 1] - v2[:, 0] * v1[:, 1]
    temp = 1.0 / np.sqrt(t1 ** 2 + t2 ** 2 + t3 ** 2)
    bnorm = np.stack([t1 * temp, t2 * temp, t3 * temp], axis=1)
    wdetjb = qwtb / (4.0 * temp)
    flag = (iBCB[:, 0] >> 1) & 1
    bw = bnorm * (wdetjb * flag)[:, None]
    nabi = np.zeros((nshg, 3))
    for q in range(3):
        for a in range(3):
            np.add.at(nabi, ienb[:, a], tab[q, a] * bw)
    ndsurf = np.zeros(nshg, dtype=np.int32)
    for f in range(ienb.shape[0]):
        s = int(iBCB[f, 1])
        if s != 0:
            for a in range(3):
                nd = ienb[f, a]
                if ndsurf[nd] != 1:
                    ndsurf[nd] = s
    return nabi, ndsurf


def _finish_tube(m: Mesh, fb: np.ndarray, srf: np.ndarray, inlet_axis_profile) -> Mesh:
    """Attach iBC/BC/iBCB/BCB/NABI/ndsurf for a tube with inlet, wall and outlets."""
    nshg = m.nshg
    order = np.argsort(srf, kind="stable")        # wall faces (id 1) first
    fb, srf = fb[order], srf[order]
    iBCB = np.zeros((fb.shape[0], 2), dtype=np.int32)
    iBCB[:, 1] = srf
    iBCB[srf >= SRF_OUTLET0, 0] = 2                # natural pressure bit, BCB p = 0
    BCB = np.zeros((fb.shape[0], 3, 6))
    wall_nodes = np.unique(fb[srf == SRF_WALL, :3])
    inlet_nodes = np.setdiff1d(np.unique(fb[srf == SRF_INLET, :3]), wall_nodes)
    iBC = np.zeros(nshg, dtype=np.int32)
    iBC[wall_nodes] = 8 + 16 + 32
    iBC[inlet_nodes] = 8 + 16 + 32
    BC = np.zeros((nshg, NDOFBC))
    m.ienb = fb.astype(np.int32)
    m.iBCB = iBCB
    m.BCB = BCB
    m.iBC = iBC
    m.BC = BC
    m.inlet_nodes = inlet_nodes.astype(np.int64)
    m.inlet_profile = inlet_axis_profile(inlet_nodes)
    m.NABI, m.ndsurf = compute_nabi(m.x, m.ienb, m.iBCB, nshg)
    m.outlets = sorted(int(s) for s in np.unique(srf) if s >= SRF_OUTLET0)
    return m


def cylinder(ncross: int = 24, naxial: int = 40, radius: float = 1.0, length: float = 10.0,
             jitter: float = 0.05, seed: int = 1, name: str = "cylinder", n_outlets: int = 1) -> Mesh:
    """Straight tube: ncross x ncross hex cross-section masked to the disc, naxial layers.

    Cells whose centre lies inside ``radius`` are kept; each hex is split into
    6 Kuhn tets.  Nodes not on the boundary are jittered uniformly by
    ``jitter`` x the local edge length in every coordinate (seeded).
    Inlet at z = 0 (parabolic profile, unit mean speed), outlet cap at
    z = length.  With ``n_outlets`` > 1 the cap is split into that many
    equal angular sectors (by face centroid), each its own outlet surface
    (ids 3, 4, ...): outlets branching from the distal cap.
    """
    h = 2.0 * radius / ncross
    hz = length / naxial
    cc = -radius + h * (np.arange(ncross) + 0.5)
    cx, cy = np.meshgrid(cc, cc, indexing="ij")
    keep = (cx ** 2 + cy ** 2) < radius ** 2
    # node (i, j) used if any adjacent kept cell
    used = np.zeros((ncross + 1, ncross + 1), dtype=bool)
    ki, kj = np.nonzero(keep)
    for di in (0, 1):
        for dj in (0, 1):
            used[ki + di, kj + dj] = True
    nid2 = -np.ones((ncross + 1, ncross + 1), dtype=np.int64)
    ui, uj = np.nonzero(used)
    nid2[ui, uj] = np.arange(len(ui))
    n2 = len(ui)
    gx = -radius + h * ui
    gy = -radius + h * uj
    nz = naxial + 1
    x = np.zeros((n2 * nz, 3))
    for k in range(nz):
        x[k * n2:(k + 1) * n2, 0] = gx
        x[k * n2:(k + 1) * n2, 1] = gy
        x[k * n2:(k + 1) * n2, 2] = hz * k
    # hexes, layer-major for locality
    hv = np.zeros((len(ki), 8), dtype=np.int64)
    for v in range(8):
        dx, dy, dz = v & 1, (v >> 1) & 1, (v >> 2) & 1
        hv[:, v] = nid2[ki + dx, kj + dy] + dz * n2
    hexes = np.concatenate([hv + k * n2 for k in range(naxial)], axis=0)
    ien = _hex_to_tets(hexes)
    fb = _boundary_faces(ien)
    bnodes = np.unique(fb[:, :3])
    rng = np.random.default_rng(seed)
    interior = np.ones(x.shape[0], dtype=bool)
    interior[bnodes] = False
    amp = jitter * min(h, hz)
    x[interior] += rng.uniform(-amp, amp, size=(int(interior.sum()), 3))
    ien = _orient(x, ien).astype(np.int32)
    fb = _boundary_faces(ien)
    fb = _orient_faces_outward(x, fb)
    zc = x[fb[:, :3], 2].mean(axis=1)
    srf = np.full(fb.shape[0], SRF_WALL, dtype=np.int32)
    srf[zc < 1e-9 * length] = SRF_INLET
    cap = zc > length * (1 - 1e-9)
    if n_outlets <= 1:
        srf[cap] = SRF_OUTLET0
    else:
        xc = x[fb[:, :3], 0].mean(axis=1)
        yc = x[fb[:, :3], 1].mean(axis=1)
        sector = np.floor((np.arctan2(yc, xc) + np.pi) / (2.0 * np.pi) * n_outlets).astype(np.int32)
        srf[cap] = SRF_OUTLET0 + np.clip(sector[cap], 0, n_outlets - 1)

    def profile(nodes):
        r2 = (x[nodes, 0] ** 2 + x[nodes, 1] ** 2) / radius ** 2
        p = np.zeros((len(nodes), 3))
        p[:, 2] = 2.0 * np.clip(1.0 - r2, 0.0, None)
        return p

    m = Mesh(x=x, ien=ien, name=name)
    return _finish_tube(m, fb, srf, profile)


def bifurcation(h: float = 0.036, parent_radius: float = 1.0, daughter_radius: float = 0.7,
                parent_length: float = 5.0, daughter_length: float = 5.0, angle_deg: float = 30.0,
                jitter: float = 0.05, seed: int = 3, name: str = "bifurcation") -> Mesh:
    """Y-bifurcation: a parent tube along +z (inlet at z = 0) splitting at
    B = (0, 0, parent_length) into two daughters along (+-sin a, 0, cos a).

    Built the way :func:`cylinder` is, on one structured grid of spacing h:
    hex cells whose centre lies inside the union of the three tubes (each a
    finite cylinder about its centreline; the parent reaches half a radius
    past B so the junction closes) are kept and split into 6 Kuhn tets; the
    walls are the grid's staircase approximation of the tubes.  Interior
    nodes are jittered by ``jitter`` x h (seeded).  A boundary face is an
    outlet of daughter k (ids 3, 4) when the cell beyond it lies inside
    daughter k's radius but past its end; the inlet is the z = 0 plane;
    everything else is wall.  h = 0.036 cm gives about 4M tets.
    """
    a = np.deg2rad(angle_deg)
    Bz = parent_length
    dirs = [np.array([np.sin(a), 0.0, np.cos(a)]), np.array([-np.sin(a), 0.0, np.cos(a)])]
    B = np.array([0.0, 0.0, Bz])
    ends = [B + daughter_length * d for d in dirs]
    rmax = max(parent_radius, daughter_radius)
    lo = np.array([min(e[0] for e in ends) - rmax - h, -rmax - h, 0.0])
    hi = np.array([max(e[0] for e in ends) + rmax + h, rmax + h, max(e[2] for e in ends) + rmax + h])
    nc = np.ceil((hi - lo) / h).astype(np.int64)
    # cell centres, z-major order (layer by layer, for locality)
    ck, cj, ci = np.meshgrid(np.arange(nc[2]), np.arange(nc[1]), np.arange(nc[0]), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    cen = lo + h * (np.stack([ci, cj, ck], axis=1) + 0.5)

    def inside(p):
        par = (p[:, 0] ** 2 + p[:, 1] ** 2 < parent_radius ** 2) & (p[:, 2] > 0.0) & \
              (p[:, 2] < Bz + 0.5 * parent_radius)
        inn = par.copy()
        for d in dirs:
            s = (p - B) @ d
            r2 = np.sum((p - B - s[:, None] * d) ** 2, axis=1)
            inn |= (s > 0.0) & (s < daughter_length) & (r2 < daughter_radius ** 2)
        return inn

    keep = inside(cen)
    ci, cj, ck = ci[keep], cj[keep], ck[keep]
    nn = nc + 1
    gid = lambda i, j, k: (k * nn[1] + j) * nn[0] + i
    hv = np.zeros((ci.size, 8), dtype=np.int64)
    for v in range(8):
        dx, dy, dz = v & 1, (v >> 1) & 1, (v >> 2) & 1
        hv[:, v] = gid(ci + dx, cj + dy, ck + dz)
    used, inv = np.unique(hv, return_inverse=True)
    hexes = inv.reshape(hv.shape)
    gk = used // (nn[0] * nn[1])
    gj = (used // nn[0]) % nn[1]
    gi = used % nn[0]
    x = lo + h * np.stack([gi, gj, gk], axis=1).astype(np.float64)
    ien = _hex_to_tets(hexes)
    fb = _boundary_faces(ien)
    bnodes = np.unique(fb[:, :3])
    rng = np.random.default_rng(seed)
    interior = np.ones(x.shape[0], dtype=bool)
    interior[bnodes] = False
    x[interior] += rng.uniform(-jitter * h, jitter * h, size=(int(interior.sum()), 3))
    ien = _orient(x, ien).astype(np.int32)
    fb = _boundary_faces(ien)
    fb = _orient_faces_outward(x, fb)
    v1 = x[fb[:, 1]] - x[fb[:, 0]]
    v2 = x[fb[:, 2]] - x[fb[:, 0]]
    nrm = np.cross(v1, v2)
    nrm /= np.linalg.norm(nrm, axis=1)[:, None]
    # centre of the grid cell across the face (faces lie on grid planes; the
    # jitter moves interior nodes only)
    beyond = x[fb[:, :3]].mean(axis=1) + 0.5 * h * nrm
    beyond = lo + h * (np.floor((beyond - lo) / h) + 0.5)
    srf = np.full(fb.shape[0], SRF_WALL, dtype=np.int32)
    srf[beyond[:, 2] < 0.0] = SRF_INLET
    for k, d in enumerate(dirs):
        s = (beyond - B) @ d
        r2 = np.sum((beyond - B - s[:, None] * d) ** 2, axis=1)
        srf[(s >= daughter_length) & (r2 < daughter_radius ** 2)] = SRF_OUTLET0 + k

    def profile(nodes):
        r2 = (x[nodes, 0] ** 2 + x[nodes, 1] ** 2) / parent_radius ** 2
        p = np.zeros((len(nodes), 3))
        p[:, 2] = 2.0 * np.clip(1.0 - r2, 0.0, None)
        return p

    m = Mesh(x=x, ien=ien, name=name)
    return _finish_tube(m, fb, srf, profile)


def bifurcation_rcr(seed: int = 3, Rp: float = 100.0, C: float = 1e-4, Rd: float = 1000.0, spread: float = 0.2):
    """RCR values of the two daughters: the nominal values scaled by
    independent factors uniform in [1 - spread, 1 + spread] (seeded)."""
    rng = np.random.default_rng(seed)
    f = rng.uniform(1.0 - spread, 1.0 + spread, size=(2, 3))
    return [dict(srfid=SRF_OUTLET0 + k, Rp=Rp * f[k, 0], C=C * f[k, 1], Rd=Rd * f[k, 2]) for k in range(2)]


def lattice(n: int, jitter: float = 0.05, seed: int = 5, name: str = "lattice") -> Mesh:
    """n^3 hexes on a unit-spaced jittered lattice split into 6n^3 tets (no boundary data)."""
    nn = n + 1
    i, j, k = np.meshgrid(np.arange(nn), np.arange(nn), np.arange(nn), indexing="ij")
    x = np.stack([i.ravel(order="F"), j.ravel(order="F"), k.ravel(order="F")], axis=1).astype(np.float64)
    rng = np.random.default_rng(seed)
    x += rng.uniform(-jitter, jitter, size=x.shape)
    c = np.arange(n)
    ci, cj, ck = np.meshgrid(c, c, c, indexing="ij")
    base = (ci + nn * cj + nn * nn * ck).ravel(order="F")
    hv = np.zeros((base.size, 8), dtype=np.int64)
    for v in range(8):
        dx, dy, dz = v & 1, (v >> 1) & 1, (v >> 2) & 1
        hv[:, v] = base + dx + nn * dy + nn * nn * dz
    ien = _orient(x, _hex_to_tets(hv)).astype(np.int32)
    m = Mesh(x=x, ien=ien, name=name)
    m.iBC = np.zeros(m.nshg, dtype=np.int32)
    m.BC = np.zeros((m.nshg, NDOFBC))
    m.ndsurf = np.zeros(m.nshg, dtype=np.int32)
    m.NABI = np.zeros((m.nshg, 3))
    return m


def random_state(nshg: int, seed: int = 5, dtype=np.float64):
    """Nodal y (u,v,w,p) and ac ~ N(0,1): the microbenchmark state."""
    rng = np.random.default_rng(seed)
    y = rng.standard_normal((nshg, 4)).astype(dtype)
    ac = rng.standard_normal((nshg, 4)).astype(dtype)
    return y, ac


def cylinder_for_tets(target_tets: int, **kw) -> Mesh:
    """Cylinder with the 60k-tet case's aspect (ncross:naxial = 24:40) sized to ~target_tets."""
    # tets ~= 6 * (pi/4) * ncross^2 * naxial with naxial = 5/3 ncross
    nc = int(round((target_tets / (6 * np.pi / 4 * 5.0 / 3.0)) ** (1.0 / 3.0)))
    return cylinder(ncross=nc, naxial=int(round(nc * 5.0 / 3.0)), **kw)
