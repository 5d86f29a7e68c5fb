"""Seeded generator for terrain-following prism-column meshes with median-dual metrics.

The reference solver (``lippsLFroude_implgwopks3D_unstr3.f``) ships no mesh and no
generator: it reads ``mesh3d.d`` in the list-directed layout of ``input``
(lippsLFroude_implgwopks3D_unstr3.f:2343-2641).  This module builds the meshes the
workloads are quoted on and writes/reads that layout.

Construction (all geometry is exact for the surfaces it defines, so every dual cell
closes to round-off):

* Horizontal: ``nx * ny`` nodes on a doubly periodic ``Lx * Ly`` square, each node
  at the centre of a regular cell jittered uniformly by ``+-jitter*h`` (seeded with
  ``numpy.random.default_rng(seed)``), Delaunay-triangulated on the torus.  The
  median-dual cell of a node is the union of the quads (node, edge midpoint,
  triangle centroid, edge midpoint) of its triangles.
* Vertical: ``L`` levels ``zeta_k`` over depth ``H`` with Gal-Chen terrain-following
  height ``z = h(x,y) + zeta * (1 - h/H)``.  Level ``k`` owns the slab between the
  half levels ``zeta_{k-1/2}`` and ``zeta_{k+1/2}`` (clamped to 0 and H).
* Terrain: a Witch-of-Agnesi hill ``h = h0 / (1 + r^2/a^2)^{3/2}`` on the minimum-image
  distance ``r`` from the domain centre (so the terrain is periodic).

The terrain surface of each cell is piecewise linear over the fan triangles
(node, polygon vertex, next polygon vertex) of the dual polygon, with ``h`` evaluated
at the node, the edge midpoints and the triangle centroids.  With that surface:

* lateral face of horizontal edge (a,b) at level k:  ``S = dzeta_k * (Tx_e, Ty_e, 0)``
  where ``T_e = sum_seg 0.5*(s_A + s_B) * rot(B - A)``, ``s = 1 - h/H``, over the two
  dual segments (midpoint -> centroid);
* face of vertical edge (c,k)->(c,k+1): ``S = ((1-zeta_{k+1/2}/H) Ax_c,
  (1-zeta_{k+1/2}/H) Ay_c, Az_c)`` with ``(Ax, Ay, Az)`` the vector area of the dual
  polygon lifted onto the terrain;
* dual volume: ``vol = dzeta_k * W_c`` with ``W_c = sum_fan A_tri (1 - hbar_tri/H)``.

The periodic square is represented as a torus: edges wrap around and there are no
duplicate nodes, so the reference's periodic duplicate lists (``icoin``, ``icoin2``,
``icoin4``) are empty and its ``cyclicr*`` routines are no-ops on this input.
``generate(..., duplicates=True)`` builds the reference's duplicate-node form of a periodic
domain instead, and ``merge_duplicates`` converts that form to the torus.
Semi-edges are not used (``nbface = 0``); the top and bottom of every column are
boundary points of type 11 (normal velocity removed by ``bcv``) with the outward
dual face as ``sbb`` and its unit normal as ``anp``.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Optional

import numpy as np


# ----------------------------------------------------------------------------------
# mesh containers
# ----------------------------------------------------------------------------------
@dataclasses.dataclass
class ColumnMesh:
    """Compact description of an extruded prism-column mesh (2D data x levels)."""

    nx: int
    ny: int
    L: int
    Lx: float
    Ly: float
    H: float
    h0: float
    half_width: float
    xy: np.ndarray          # (NC, 2) node positions in [0,Lx) x [0,Ly)
    hnode: np.ndarray       # (NC,) terrain height at the nodes
    tri: np.ndarray         # (2*NC, 3) triangles (CCW), column indices
    edges2d: np.ndarray     # (NE2, 2) int64, a < b
    T: np.ndarray           # (NE2, 2) lateral face vector per unit dzeta
    A: np.ndarray           # (NC, 3) lifted dual-polygon vector area
    W: np.ndarray           # (NC,) volume per unit dzeta
    zeta: np.ndarray        # (L,) computational levels
    zeta_half: np.ndarray   # (L+1,) half levels (0 ... H)
    periodic: bool = True
    # open (non-periodic) meshes only: one lateral boundary entry per boundary column and
    # side, (column, type, Tx, Ty) with T the outward face vector per unit dzeta
    bcol: Optional[np.ndarray] = None     # (nb,) int64
    btype: Optional[np.ndarray] = None    # (nb,) int32: 7 inflow x=0, 8 outflow x=Lx, 5 y=0, 6 y=Ly
    bT: Optional[np.ndarray] = None       # (nb, 2)
    # duplicate-node periodic form only: column pairs / quadruples of copies
    coin: Optional[np.ndarray] = None     # (n, 2) x = 0 ~ x = Lx
    coin2: Optional[np.ndarray] = None    # (n, 2) y = 0 ~ y = Ly
    coin4: Optional[np.ndarray] = None    # (1, 4) the corners

    @property
    def ncol(self) -> int:
        return self.xy.shape[0]

    @property
    def npoin(self) -> int:
        return self.ncol * self.L

    @property
    def dzeta(self) -> np.ndarray:
        return np.diff(self.zeta_half)

    def node(self, c, k):
        return np.asarray(c) * self.L + np.asarray(k)

    def max_degree(self) -> int:
        """Largest 3D node degree (2D degree + up to 2 vertical neighbours)."""
        deg = np.bincount(self.edges2d.ravel(), minlength=self.ncol)
        return int(deg.max()) + (2 if self.L > 2 else 1)

    def to_reference(self) -> "RefMesh":
        return expand_reference(self)


@dataclasses.dataclass
class RefMesh:
    """Mesh arrays in the layout of the reference COMMON blocks, 0-based indices.

    Component arrays are (n, 3) row-major here; the C boundary receives them as
    separate component pointers (the Fortran ``sn(nedgex,3)`` column slices).
    """

    npoin: int
    nedge: int
    nbface: int
    nboun: int
    coord: np.ndarray       # (npoin, 3)
    vol: np.ndarray         # (npoin,)
    iedge: np.ndarray       # (nedge, 2) int32, 0-based
    sn: np.ndarray          # (nedge, 3)
    kbface: np.ndarray      # (nbface, 2) int32
    sb: np.ndarray          # (nbface, 3)
    ibpoin: np.ndarray      # (nboun, 2) int32: node (0-based), type
    sbb: np.ndarray         # (nboun, 3)
    anp: np.ndarray         # (nboun, 3)
    icoin: np.ndarray       # (ncoin, 2) int32
    icoin2: np.ndarray      # (ncoin2, 2) int32
    icoin4: np.ndarray      # (ncoin4, 4) int32

    @property
    def nbpoin(self) -> int:
        return self.nboun


# ----------------------------------------------------------------------------------
# generator
# ----------------------------------------------------------------------------------
def agnesi(x, y, Lx, Ly, h0, a, periodic=True):
    """Witch-of-Agnesi hill centred in the domain, periodic via minimum image."""
    dx = np.asarray(x) - 0.5 * Lx
    dy = np.asarray(y) - 0.5 * Ly
    if periodic:
        dx = dx - Lx * np.round(dx / Lx)
        dy = dy - Ly * np.round(dy / Ly)
    return h0 / (1.0 + (dx * dx + dy * dy) / (a * a)) ** 1.5


def _open_delaunay(pts: np.ndarray, Lx: float, Ly: float):
    """Delaunay triangulation of a point set whose hull is the rectangle [0,Lx]x[0,Ly].

    Points on the sides are collinear, which Qhull may drop as coplanar.  The
    triangulation is therefore computed on a copy whose side points bulge outward by a
    tiny amount (a strictly convex hull, every point a vertex) and then used with the
    true positions; triangles are checked for positive area there.
    """
    from scipy.spatial import Delaunay

    q = pts.copy()
    u = q[:, 0] / Lx
    v = q[:, 1] / Ly
    eps = 1e-6
    q[:, 0] += np.where(u <= 0.0, -eps * Lx * np.sin(np.pi * v), 0.0)
    q[:, 0] += np.where(u >= 1.0, eps * Lx * np.sin(np.pi * v), 0.0)
    q[:, 1] += np.where(v <= 0.0, -eps * Ly * np.sin(np.pi * u), 0.0)
    q[:, 1] += np.where(v >= 1.0, eps * Ly * np.sin(np.pi * u), 0.0)
    simp = Delaunay(q).simplices.astype(np.int64)
    P = pts[simp]
    cr = ((P[:, 1, 0] - P[:, 0, 0]) * (P[:, 2, 1] - P[:, 0, 1])
          - (P[:, 1, 1] - P[:, 0, 1]) * (P[:, 2, 0] - P[:, 0, 0]))
    flip = cr < 0
    simp[flip] = simp[flip][:, [0, 2, 1]]
    P = pts[simp]
    cr = np.abs(cr)
    h2 = Lx * Ly / pts.shape[0]
    if cr.min() < 1e-3 * h2:
        raise RuntimeError("open Delaunay produced a degenerate triangle")
    if abs(0.5 * cr.sum() - Lx * Ly) > 1e-9 * Lx * Ly:
        raise RuntimeError("open Delaunay does not cover the rectangle")
    return simp, P


def _periodic_delaunay(pts: np.ndarray, Lx: float, Ly: float, margin: float):
    from scipy.spatial import Delaunay

    n = pts.shape[0]
    ext, idx = [], []
    for sx in (-1, 0, 1):
        for sy in (-1, 0, 1):
            q = pts + np.array([sx * Lx, sy * Ly])
            m = ((q[:, 0] > -margin) & (q[:, 0] < Lx + margin)
                 & (q[:, 1] > -margin) & (q[:, 1] < Ly + margin))
            ext.append(q[m])
            idx.append(np.nonzero(m)[0])
    ext = np.concatenate(ext)
    idx = np.concatenate(idx)
    simp = Delaunay(ext).simplices
    P = ext[simp]                                   # (nt, 3, 2)
    cen = P.mean(axis=1)
    keep = (cen[:, 0] >= 0) & (cen[:, 0] < Lx) & (cen[:, 1] >= 0) & (cen[:, 1] < Ly)
    simp, P = simp[keep], P[keep]
    cr = ((P[:, 1, 0] - P[:, 0, 0]) * (P[:, 2, 1] - P[:, 0, 1])
          - (P[:, 1, 1] - P[:, 0, 1]) * (P[:, 2, 0] - P[:, 0, 0]))
    flip = cr < 0
    simp[flip] = simp[flip][:, [0, 2, 1]]
    P[flip] = P[flip][:, [0, 2, 1]]
    tri = idx[simp]
    if tri.shape[0] != 2 * n:
        raise RuntimeError(f"periodic Delaunay produced {tri.shape[0]} triangles, expected {2 * n}")
    return tri.astype(np.int64), P


def level_set(L: int, H: float, stretch_dz0: Optional[float] = None) -> np.ndarray:
    """Computational levels.  Uniform, or geometric with first spacing ``stretch_dz0``."""
    if stretch_dz0 is None:
        return np.linspace(0.0, H, L)
    n = L - 1
    # find ratio q with dz0 * (q^n - 1)/(q - 1) = H
    lo, hi = 1.0 + 1e-12, 4.0
    for _ in range(200):
        q = 0.5 * (lo + hi)
        s = stretch_dz0 * (q ** n - 1.0) / (q - 1.0)
        if s > H:
            hi = q
        else:
            lo = q
    dz = stretch_dz0 * q ** np.arange(n)
    z = np.concatenate([[0.0], np.cumsum(dz)])
    z *= H / z[-1]
    return z


def generate(nx: int, ny: Optional[int] = None, L: int = 41, Lx: float = 120e3,
             Ly: Optional[float] = None, H: float = 20e3, h0: float = 400.0,
             half_width: float = 10e3, jitter: float = 0.3, seed: int = 0,
             stretch_dz0: Optional[float] = None, periodic: bool = True,
             duplicates: bool = False) -> ColumnMesh:
    """Build the jittered prism-column mesh (see module docstring).

    ``duplicates=True`` (periodic only) builds the reference's own periodic form instead of the
    torus: ``(nx+1) * (ny+1)`` nodes from corner to corner, the nodes of opposite sides
    duplicates of one another (same tangential jitter), listed in ``icoin`` (x sides),
    ``icoin2`` (y sides) and ``icoin4`` (the four corners) for the reference's ``cyclicr``
    routines (ref.f:4377-4446).  Each copy carries its part of the dual cell; the bottom
    boundary normal ``anp`` of every copy is the normal of the whole cell.

    ``periodic=False`` builds the open channel used with ``iper = 0``: ``nx * ny`` nodes
    from corner to corner of the rectangle, side nodes jittered along their side only,
    corners fixed, and lateral boundary points on the four sides: inflow (type 7) at
    ``x = 0``, outflow (type 8) at ``x = Lx``, walls (types 5 and 6) at ``y = 0`` and
    ``y = Ly``.  A side node's lateral face is the vertical strip over its two half side
    edges, ``dzeta_k * sum 0.5*(s_A + s_B) * rot(B - A)`` like the interior faces.
    """
    ny = nx if ny is None else ny
    Ly = Lx if Ly is None else Ly
    if duplicates and not periodic:
        raise ValueError("duplicates=True describes a periodic domain")
    torus = periodic and not duplicates
    rng = np.random.default_rng(seed)
    if torus:
        I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
        hx, hy = Lx / nx, Ly / ny
        base = np.stack([(I.ravel() + 0.5) * hx, (J.ravel() + 0.5) * hy], axis=1)
    elif duplicates:
        nxx, nyy = nx + 1, ny + 1
        I, J = np.meshgrid(np.arange(nxx), np.arange(nyy), indexing="xy")
        hx, hy = Lx / nx, Ly / ny
        base = np.stack([I.ravel() * hx, J.ravel() * hy], axis=1)
    else:
        nxx, nyy = nx, ny
        I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
        hx, hy = Lx / (nx - 1), Ly / (ny - 1)
        base = np.stack([I.ravel() * hx, J.ravel() * hy], axis=1)
    jit = rng.uniform(-jitter, jitter, size=base.shape) * np.array([hx, hy])
    if not torus:
        Ir, Jr = I.ravel(), J.ravel()
        iside = (Ir == 0) | (Ir == nxx - 1)
        jside = (Jr == 0) | (Jr == nyy - 1)
        jit[iside, 0] = 0.0
        jit[jside, 1] = 0.0
        if duplicates:       # a copy moves along its side exactly like its partner
            jit[Ir == nxx - 1, 1] = jit[(Ir == 0), 1]
            jit[Jr == nyy - 1, 0] = jit[(Jr == 0), 0]
    xy = base + jit
    return _build(xy, nx, ny, L, Lx, Ly, H, h0, half_width, stretch_dz0, periodic, torus, duplicates,
                  nxx if not torus else nx, nyy if not torus else ny)


def coarsen(cm: ColumnMesh) -> ColumnMesh:
    """The mesh on every other column of a torus mesh made by ``generate``: the nodes of even
    grid row and column (every node keeps its exact position, terrain height and levels), newly
    Delaunay-triangulated on the torus with their own median-dual metrics.  These are the coarser
    meshes of the multigrid V-cycle (the reference reads them as ``mesh3d_c.d`` and
    ``mesh3d_cc.d``, ref.f:2343-2641); every coarse node coincides with a fine node, as the
    reference's ``matching`` (ref.f:2684-2720) requires.  Levels are not coarsened."""
    if not cm.periodic or cm.coin is not None or cm.nx % 2 or cm.ny % 2:
        raise ValueError("coarsen takes a torus mesh with an even number of columns each way")
    xy = cm.xy.reshape(cm.ny, cm.nx, 2)[::2, ::2].reshape(-1, 2).copy()
    out = _build(xy, cm.nx // 2, cm.ny // 2, cm.L, cm.Lx, cm.Ly, cm.H, cm.h0, cm.half_width, None,
                 True, True, False, cm.nx // 2, cm.ny // 2)
    out.zeta = np.asarray(cm.zeta).copy()
    out.zeta_half = np.asarray(cm.zeta_half).copy()
    return out


def coarse_match(fine: ColumnMesh, coarse: ColumnMesh) -> np.ndarray:
    """For every node of a ``coarsen``-ed mesh, its node in the fine mesh (0-based, in the node
    numbering of ``to_reference``): the reference's ``match`` arrays (ref.f:2684-2720)."""
    cols = np.arange(fine.ncol).reshape(fine.ny, fine.nx)[::2, ::2].ravel()
    if not np.array_equal(fine.xy[cols], coarse.xy):
        raise ValueError("coarse columns are not the even-index columns of the fine mesh")
    return (cols[:, None] * fine.L + np.arange(fine.L)[None, :]).ravel()


def _build(xy, nx, ny, L, Lx, Ly, H, h0, half_width, stretch_dz0, periodic, torus, duplicates, nxx, nyy):
    """Mesh on the horizontal points ``xy`` (see ``generate``)."""
    hx, hy = Lx / nx, Ly / ny
    ncol = xy.shape[0]

    if torus:
        tri, P = _periodic_delaunay(xy, Lx, Ly, margin=4.0 * max(hx, hy))
    else:
        tri, P = _open_delaunay(xy, Lx, Ly)
    hnode = agnesi(xy[:, 0], xy[:, 1], Lx, Ly, h0, half_width, periodic)

    def hf(p):
        return agnesi(p[..., 0], p[..., 1], Lx, Ly, h0, half_width, periodic)

    nt = tri.shape[0]
    g = P.mean(axis=1)                                      # (nt, 2)
    hg = hf(g)
    # edges in CCW order: (v0,v1), (v1,v2), (v2,v0)
    ei = np.array([[0, 1], [1, 2], [2, 0]])
    p_idx = tri[:, ei[:, 0]]                                # (nt, 3)
    q_idx = tri[:, ei[:, 1]]
    Pp = P[:, ei[:, 0]]                                     # (nt, 3, 2)
    Pq = P[:, ei[:, 1]]
    M = 0.5 * (Pp + Pq)                                     # midpoints (nt, 3, 2)
    hm = hf(M)
    a = np.minimum(p_idx, q_idx)
    b = np.maximum(p_idx, q_idx)
    key = (a * ncol + b).ravel()
    ukey, inv, cnt = np.unique(key, return_inverse=True, return_counts=True)
    if torus and not np.all(cnt == 2):
        raise RuntimeError("torus triangulation has an edge not shared by two triangles")
    edges2d = np.stack([ukey // ncol, ukey % ncol], axis=1)
    ne2 = edges2d.shape[0]
    if torus and ne2 != 3 * ncol:
        raise RuntimeError(f"expected {3 * ncol} edges, got {ne2}")

    # lateral face vectors: segment midpoint -> centroid, oriented p -> q, flipped to a -> b
    v = g[:, None, :] - M                                   # (nt, 3, 2)
    nrm = np.stack([v[..., 1], -v[..., 0]], axis=-1)        # rot(g - m), oriented p -> q
    sgn = np.where(p_idx == a, 1.0, -1.0)                   # +1 when p is the canonical a
    smid = 1.0 - hm / H
    scen = 1.0 - hg / H
    contrib = (0.5 * (smid + scen[:, None]) * sgn)[..., None] * nrm
    contrib = contrib.reshape(-1, 2)
    T = np.stack([np.bincount(inv, weights=contrib[:, 0], minlength=ne2),
                  np.bincount(inv, weights=contrib[:, 1], minlength=ne2)], axis=1)

    # column quantities from the fan triangles (node, m_next, g) and (node, g, m_prev)
    A = np.zeros((ncol, 3))
    W = np.zeros(ncol)
    for i in range(3):
        node = tri[:, i]
        Pn = np.concatenate([P[:, i], hnode[node][:, None]], axis=1)           # (nt, 3)
        m_next = np.concatenate([M[:, i], hm[:, i][:, None]], axis=1)          # edge (i, i+1)
        m_prev = np.concatenate([M[:, (i + 2) % 3], hm[:, (i + 2) % 3][:, None]], axis=1)
        G3 = np.concatenate([g, hg[:, None]], axis=1)
        for (Q1, Q2) in ((m_next, G3), (G3, m_prev)):
            s = 0.5 * np.cross(Q1 - Pn, Q2 - Pn)
            hbar = (Pn[:, 2] + Q1[:, 2] + Q2[:, 2]) / 3.0
            for d in range(3):
                A[:, d] += np.bincount(node, weights=s[:, d], minlength=ncol)
            W += np.bincount(node, weights=s[:, 2] * (1.0 - hbar / H), minlength=ncol)

    bcol = btype = bT = None
    if not periodic:
        # side half-edges of the boundary edges (one triangle each), CCW so the domain is on
        # the left and rot(B - A) = (dy, -dx) is the outward normal
        bmask = (cnt[inv] == 1).reshape(-1, 3)
        t_i, e_i = np.nonzero(bmask)
        Pp_b, Pq_b, M_b = Pp[t_i, e_i], Pq[t_i, e_i], M[t_i, e_i]
        sp = 1.0 - hnode[p_idx[t_i, e_i]] / H
        sq = 1.0 - hnode[q_idx[t_i, e_i]] / H
        sm = smid[t_i, e_i]

        def rot(v):
            return np.stack([v[:, 1], -v[:, 0]], axis=1)

        tp = (0.5 * (sp + sm))[:, None] * rot(M_b - Pp_b)
        tq = (0.5 * (sm + sq))[:, None] * rot(Pq_b - M_b)
        tol = 1e-9 * max(Lx, Ly)
        side = np.full(t_i.shape[0], -1)
        side[np.abs(M_b[:, 0]) < tol] = 0                       # x = 0: inflow
        side[np.abs(M_b[:, 0] - Lx) < tol] = 1                  # x = Lx: outflow
        side[np.abs(M_b[:, 1]) < tol] = 2                       # y = 0: wall
        side[np.abs(M_b[:, 1] - Ly) < tol] = 3                  # y = Ly: wall
        if np.any(side < 0):
            raise RuntimeError("open mesh has a boundary edge off the rectangle's sides")
        cols = np.concatenate([p_idx[t_i, e_i], q_idx[t_i, e_i]])
        sides = np.concatenate([side, side])
        key2 = sides * ncol + cols
        uk, inv2 = np.unique(key2, return_inverse=True)
        tt = np.concatenate([tp, tq])
        bT = np.stack([np.bincount(inv2, weights=tt[:, 0], minlength=uk.shape[0]),
                       np.bincount(inv2, weights=tt[:, 1], minlength=uk.shape[0])], axis=1)
        bcol = (uk % ncol).astype(np.int64)
        btype = np.array([7, 8, 5, 6], dtype=np.int32)[uk // ncol]

    coin = coin2 = coin4 = None
    if duplicates:
        cidx = np.arange(ncol).reshape(nyy, nxx)
        coin = np.stack([cidx[1:-1, 0], cidx[1:-1, -1]], axis=1)          # x = 0 ~ x = Lx
        coin2 = np.stack([cidx[0, 1:-1], cidx[-1, 1:-1]], axis=1)         # y = 0 ~ y = Ly
        coin4 = np.array([[cidx[0, 0], cidx[0, -1], cidx[-1, 0], cidx[-1, -1]]])

    zeta = level_set(L, H, stretch_dz0)
    zh = np.empty(L + 1)
    zh[0] = 0.0
    zh[1:L] = 0.5 * (zeta[:-1] + zeta[1:])
    zh[L] = H
    return ColumnMesh(nx=nx, ny=ny, L=L, Lx=Lx, Ly=Ly, H=H, h0=h0, half_width=half_width,
                      xy=xy, hnode=hnode, tri=tri, edges2d=edges2d.astype(np.int64), T=T,
                      A=A, W=W, zeta=zeta, zeta_half=zh, periodic=periodic,
                      bcol=bcol, btype=btype, bT=bT, coin=coin, coin2=coin2, coin4=coin4)


def expand_reference(cm: ColumnMesh) -> RefMesh:
    """Expand a ColumnMesh into the reference's node/edge/boundary arrays.

    Node ``c*L + k`` is column ``c`` at level ``k``.  Horizontal edge ``e*L + k`` joins
    ``(a,k)`` and ``(b,k)``; vertical edge ``NE2*L + c*(L-1) + k`` joins ``(c,k)`` and
    ``(c,k+1)``.  Boundary points: bottoms of all columns, then tops, then (open meshes)
    the lateral side points.
    """
    L, NC, NE2, H = cm.L, cm.ncol, cm.edges2d.shape[0], cm.H
    dz = cm.dzeta
    zh = cm.zeta_half
    npoin = NC * L
    coord = np.empty((npoin, 3))
    coord[:, 0] = np.repeat(cm.xy[:, 0], L)
    coord[:, 1] = np.repeat(cm.xy[:, 1], L)
    coord[:, 2] = (cm.hnode[:, None] + cm.zeta[None, :] * (1.0 - cm.hnode[:, None] / H)).ravel()
    vol = (cm.W[:, None] * dz[None, :]).ravel()

    nh = NE2 * L
    nv = NC * (L - 1)
    nedge = nh + nv
    iedge = np.empty((nedge, 2), dtype=np.int32)
    sn = np.zeros((nedge, 3))
    ks = np.arange(L)
    iedge[:nh, 0] = (cm.edges2d[:, 0:1] * L + ks[None, :]).ravel()
    iedge[:nh, 1] = (cm.edges2d[:, 1:2] * L + ks[None, :]).ravel()
    sn[:nh, 0] = (cm.T[:, 0:1] * dz[None, :]).ravel()
    sn[:nh, 1] = (cm.T[:, 1:2] * dz[None, :]).ravel()
    kv = np.arange(L - 1)
    cs = np.arange(NC)
    iedge[nh:, 0] = (cs[:, None] * L + kv[None, :]).ravel()
    iedge[nh:, 1] = (cs[:, None] * L + kv[None, :] + 1).ravel()
    fac = 1.0 - zh[1:L] / H                                   # (L-1,)
    sn[nh:, 0] = (cm.A[:, 0:1] * fac[None, :]).ravel()
    sn[nh:, 1] = (cm.A[:, 1:2] * fac[None, :]).ravel()
    sn[nh:, 2] = np.repeat(cm.A[:, 2], L - 1)

    nlat = 0 if cm.periodic else cm.bcol.shape[0] * L
    nboun = 2 * NC + nlat
    ibpoin = np.empty((nboun, 2), dtype=np.int32)
    ibpoin[:NC, 0] = cs * L
    ibpoin[NC:2 * NC, 0] = cs * L + (L - 1)
    ibpoin[:2 * NC, 1] = 11
    sbb = np.zeros((nboun, 3))
    sbb[:NC] = -cm.A
    sbb[NC:2 * NC, 2] = cm.A[:, 2]
    anp = np.zeros((nboun, 3))
    anp[:2 * NC] = sbb[:2 * NC] / np.linalg.norm(sbb[:2 * NC], axis=1)[:, None]
    if nlat:
        # lateral side points, entry by entry over the levels of each (column, side)
        ibpoin[2 * NC:, 0] = (cm.bcol[:, None] * L + ks[None, :]).ravel()
        ibpoin[2 * NC:, 1] = np.repeat(cm.btype, L)
        sbb[2 * NC:, 0] = (cm.bT[:, 0:1] * dz[None, :]).ravel()
        sbb[2 * NC:, 1] = (cm.bT[:, 1:2] * dz[None, :]).ravel()
        unit = {7: (-1.0, 0.0), 8: (1.0, 0.0), 5: (0.0, -1.0), 6: (0.0, 1.0)}
        nrm = np.array([unit[int(t)] for t in cm.btype])
        anp[2 * NC:, 0] = np.repeat(nrm[:, 0], L)
        anp[2 * NC:, 1] = np.repeat(nrm[:, 1], L)
    z2 = np.zeros((0, 2), dtype=np.int32)
    lists = [z2.copy(), z2.copy(), np.zeros((0, 4), dtype=np.int32)]
    if cm.coin is not None:
        # the bottom normal of every copy is that of the whole cell (sum over its copies)
        Ab = cm.A.copy()
        for grp in (cm.coin, cm.coin2, cm.coin4):
            Ab[grp] = cm.A[grp].sum(axis=1, keepdims=True)
        anp[:NC] = -Ab / np.linalg.norm(Ab, axis=1)[:, None]
        lists = [(grp[:, None, :] * L + ks[None, :, None]).reshape(-1, grp.shape[1]).astype(np.int32)
                 for grp in (cm.coin, cm.coin2, cm.coin4)]
    return RefMesh(npoin=npoin, nedge=nedge, nbface=0, nboun=nboun, coord=coord, vol=vol,
                   iedge=iedge, sn=sn, kbface=z2.copy(), sb=np.zeros((0, 3)), ibpoin=ibpoin,
                   sbb=sbb, anp=anp, icoin=lists[0], icoin2=lists[1], icoin4=lists[2])


def merge_duplicates(rm: RefMesh):
    """Convert a periodic mesh in the reference's duplicate-node form to the torus form.

    The reference keeps the nodes of opposite periodic sides as separate copies, each with part
    of the dual cell, and sums their partial results with ``cyclicr``/``cyclicr2``/``cyclicr4``
    (ref.f:4377-4446) after every edge loop; ``vol`` is summed the same way at set-up
    (ref.f:99-103).  The library takes a periodic domain as a torus instead (wrap-around edges,
    one node per physical point, empty lists).  This merges every group of copies into its
    lowest-numbered node: volumes are summed in ``cyclicr`` order, faces joining the same pair
    of merged nodes (the two halves of a seam face) are summed, and boundary points of one merged
    node and type are combined (face vectors summed, unit normal of the sum).  Returns the torus
    mesh and, for every node of ``rm``, its node in the torus (for moving fields between the two).
    """
    n = rm.npoin
    parent = np.arange(n)

    def find(i):
        while parent[i] != i:
            parent[i] = parent[parent[i]]
            i = parent[i]
        return i

    for grp in (rm.icoin, rm.icoin2, rm.icoin4):
        for row in np.asarray(grp):
            r = [find(int(i)) for i in row]
            lo = min(r)
            for x in r:
                parent[x] = lo
    root = np.array([find(i) for i in range(n)])
    reps = np.unique(root)
    new = np.full(n, -1, dtype=np.int64)
    new[reps] = np.arange(reps.shape[0])
    node_of = new[root]

    vol = rm.vol.astype(np.float64).copy()
    for grp in (rm.icoin, rm.icoin2, rm.icoin4):        # cyclicr, cyclicr2, cyclicr4 in order
        grp = np.asarray(grp)
        if grp.shape[0]:
            tot = vol[grp[:, 0]].copy()
            for q in range(1, grp.shape[1]):
                tot = tot + vol[grp[:, q]]
            for q in range(grp.shape[1]):
                vol[grp[:, q]] = tot

    faces, S = {}, []
    for (i1, i2), sv in zip(np.concatenate([rm.iedge, rm.kbface]), np.concatenate([rm.sn, rm.sb])):
        a, b = int(node_of[i1]), int(node_of[i2])
        if a == b:
            raise ValueError("a face joins two copies of one node")
        key = (min(a, b), max(a, b))
        sgn = 1.0 if a == key[0] else -1.0
        if key in faces:
            S[faces[key]] = S[faces[key]] + sgn * sv
        else:
            faces[key] = len(S)
            S.append(sgn * sv)
    iedge = np.array(list(faces.keys()), dtype=np.int32).reshape(-1, 2)
    sn = np.array(S).reshape(-1, 3)

    bkey, sbb = {}, []
    btype = []
    for (i, t), sv in zip(rm.ibpoin, rm.sbb):
        key = (int(node_of[i]), int(t))
        if key in bkey:
            sbb[bkey[key]] = sbb[bkey[key]] + sv
        else:
            bkey[key] = len(sbb)
            sbb.append(sv.copy())
            btype.append(key)
    ibpoin = np.array(btype, dtype=np.int32).reshape(-1, 2)
    sbb = np.array(sbb).reshape(-1, 3)
    anp = sbb / np.linalg.norm(sbb, axis=1)[:, None]
    z2 = np.zeros((0, 2), dtype=np.int32)
    torus = RefMesh(npoin=reps.shape[0], nedge=iedge.shape[0], nbface=0, nboun=ibpoin.shape[0],
                    coord=rm.coord[reps].copy(), vol=vol[reps], iedge=iedge, sn=sn,
                    kbface=z2.copy(), sb=np.zeros((0, 3)), ibpoin=ibpoin, sbb=sbb, anp=anp,
                    icoin=z2.copy(), icoin2=z2.copy(), icoin4=np.zeros((0, 4), dtype=np.int32))
    return torus, node_of


# ----------------------------------------------------------------------------------
# checks
# ----------------------------------------------------------------------------------
def closure_residual(rm: RefMesh, include_boundary: bool = True) -> np.ndarray:
    """Per-node sum of outward dual-face vectors (zero for a closed dual cell)."""
    out = np.zeros((rm.npoin, 3))
    for d in range(3):
        out[:, d] += np.bincount(rm.iedge[:, 0], weights=rm.sn[:, d], minlength=rm.npoin)
        out[:, d] -= np.bincount(rm.iedge[:, 1], weights=rm.sn[:, d], minlength=rm.npoin)
        if rm.nbface:
            out[:, d] += np.bincount(rm.kbface[:, 0], weights=rm.sb[:, d], minlength=rm.npoin)
            out[:, d] -= np.bincount(rm.kbface[:, 1], weights=rm.sb[:, d], minlength=rm.npoin)
        if include_boundary:
            out[:, d] += np.bincount(rm.ibpoin[:, 0], weights=rm.sbb[:, d], minlength=rm.npoin)
    return out


# ----------------------------------------------------------------------------------
# reference text formats (list-directed, as read by `input`, ref.f:2172-2679)
# ----------------------------------------------------------------------------------
def write_mesh3d(path: str, rm: RefMesh, iper: int = 2) -> None:
    """Write ``mesh3d.d`` in the order ``input`` reads it (1-based indices)."""
    with open(path, "w") as f:
        f.write(f"{rm.npoin} {rm.nedge} {rm.nbface} {rm.nbpoin} {rm.nboun}\n")
        ids = np.arange(1, rm.npoin + 1)
        np.savetxt(f, np.column_stack([ids, rm.coord, rm.vol]), fmt="%d %.17e %.17e %.17e %.17e")
        eid = np.arange(1, rm.nedge + 1)
        np.savetxt(f, np.column_stack([eid, rm.iedge + 1]), fmt="%d %d %d")
        np.savetxt(f, np.column_stack([eid, rm.sn]), fmt="%d %.17e %.17e %.17e")
        bid = np.arange(1, rm.nbface + 1)
        if rm.nbface:
            np.savetxt(f, np.column_stack([bid, rm.kbface + 1]), fmt="%d %d %d")
            np.savetxt(f, np.column_stack([bid, rm.sb]), fmt="%d %.17e %.17e %.17e")
        pid = np.arange(1, rm.nboun + 1)
        ib = rm.ibpoin.copy()
        ib[:, 0] += 1
        np.savetxt(f, np.column_stack([pid, ib]), fmt="%d %d %d")
        np.savetxt(f, np.column_stack([pid, rm.sbb]), fmt="%d %.17e %.17e %.17e")
        np.savetxt(f, np.column_stack([pid, rm.anp]), fmt="%d %.17e %.17e %.17e")
        if iper == 2:
            for lst in (rm.icoin, rm.icoin2, rm.icoin4):
                f.write(f"{lst.shape[0]}\n")
                if lst.shape[0]:
                    np.savetxt(f, lst + 1, fmt="%d")


def read_mesh3d(path: str, iper: int = 2) -> RefMesh:
    """Read a ``mesh3d.d`` written in the reference layout (isfera=0)."""
    with open(path) as f:
        toks = f.read().split()
    pos = 0

    def take(n, cols, dtype=float):
        nonlocal pos
        a = np.array(toks[pos:pos + n * cols], dtype=float).reshape(n, cols) if n else np.zeros((0, cols))
        pos += n * cols
        return a.astype(dtype)

    npoin, nedge, nbface, nbpoin, nboun = (int(t) for t in toks[0:5])
    pos = 5
    a = take(npoin, 5)
    coord, vol = a[:, 1:4], a[:, 4]
    iedge = take(nedge, 3)[:, 1:3].astype(np.int32) - 1
    sn = take(nedge, 4)[:, 1:4]
    kbface = take(nbface, 3)[:, 1:3].astype(np.int32) - 1
    sb = take(nbface, 4)[:, 1:4]
    ib = take(nboun, 3)[:, 1:3].astype(np.int32)
    ib[:, 0] -= 1
    sbb = take(nboun, 4)[:, 1:4]
    anp = take(nboun, 4)[:, 1:4]
    lists = []
    if iper == 2:
        for w in (2, 2, 4):
            n = int(toks[pos]); pos += 1
            lists.append(take(n, w).astype(np.int32) - 1)
    else:
        lists = [np.zeros((0, 2), np.int32), np.zeros((0, 2), np.int32), np.zeros((0, 4), np.int32)]
    return RefMesh(npoin=npoin, nedge=nedge, nbface=nbface, nboun=nboun, coord=coord, vol=vol,
                   iedge=iedge, sn=sn, kbface=kbface, sb=sb, ibpoin=ib, sbb=sbb, anp=anp,
                   icoin=lists[0], icoin2=lists[1], icoin4=lists[2])


def write_reference_inputs(directory: str, rm: RefMesh, params) -> None:
    """Write every input file the reference program opens (ref.f:32-44).

    The multigrid meshes and match maps are written as copies of the fine mesh and the
    identity map: with ``mg_flag=0`` the reference reads but does not use them.
    """
    os.makedirs(directory, exist_ok=True)
    write_mesh3d(os.path.join(directory, "mesh3d.d"), rm, params.iper)
    for name in ("mesh3d_c.d", "mesh3d_cc.d"):
        write_mesh3d(os.path.join(directory, name), rm, params.iper)
    for name in ("match1.d", "match2.d"):
        np.savetxt(os.path.join(directory, name), np.arange(1, rm.npoin + 1), fmt="%d")
    params.write_input_files(directory)
