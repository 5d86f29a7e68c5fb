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
def agnesi(x, y, Lx, Ly, h0, a):
    """Witch-of-Agnesi hill centred in the domain, periodic via minimum image."""
    dx = np.asarray(x) - 0.5 * Lx
    dy = np.asarray(y) - 0.5 * Ly
    dx = dx - Lx * np.round(dx / Lx)
    dy = dy - Ly * np.round(dy / Ly)
    return h0 / (1.0 + (dx * dx + dy * dy) / (a * a)) ** 1.5


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
             stretch_dz0: Optional[float] = None) -> ColumnMesh:
    """Build the jittered periodic prism-column mesh (see module docstring)."""
    ny = nx if ny is None else ny
    Ly = Lx if Ly is None else Ly
    hx, hy = Lx / nx, Ly / ny
    rng = np.random.default_rng(seed)
    I, J = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    base = np.stack([(I.ravel() + 0.5) * hx, (J.ravel() + 0.5) * hy], axis=1)
    jit = rng.uniform(-jitter, jitter, size=base.shape) * np.array([hx, hy])
    xy = base + jit
    ncol = xy.shape[0]

    tri, P = _periodic_delaunay(xy, Lx, Ly, margin=4.0 * max(hx, hy))
    hnode = agnesi(xy[:, 0], xy[:, 1], Lx, Ly, h0, half_width)

    def hf(p):
        return agnesi(p[..., 0], p[..., 1], Lx, Ly, h0, half_width)

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
    if not np.all(cnt == 2):
        raise RuntimeError("torus triangulation has an edge not shared by two triangles")
    edges2d = np.stack([ukey // ncol, ukey % ncol], axis=1)
    ne2 = edges2d.shape[0]
    if ne2 != 3 * ncol:
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

    zeta = level_set(L, H, stretch_dz0)
    zh = np.empty(L + 1)
    zh[0] = 0.0
    zh[1:L] = 0.5 * (zeta[:-1] + zeta[1:])
    zh[L] = H
    return ColumnMesh(nx=nx, ny=ny, L=L, Lx=Lx, Ly=Ly, H=H, h0=h0, half_width=half_width,
                      xy=xy, hnode=hnode, tri=tri, edges2d=edges2d.astype(np.int64), T=T,
                      A=A, W=W, zeta=zeta, zeta_half=zh)


def expand_reference(cm: ColumnMesh) -> RefMesh:
    """Expand a ColumnMesh into the reference's node/edge/boundary arrays.

    Node ``c*L + k`` is column ``c`` at level ``k``.  Horizontal edge ``e*L + k`` joins
    ``(a,k)`` and ``(b,k)``; vertical edge ``NE2*L + c*(L-1) + k`` joins ``(c,k)`` and
    ``(c,k+1)``.  Boundary points: bottoms of all columns, then tops.
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

    nboun = 2 * NC
    ibpoin = np.empty((nboun, 2), dtype=np.int32)
    ibpoin[:NC, 0] = cs * L
    ibpoin[NC:, 0] = cs * L + (L - 1)
    ibpoin[:, 1] = 11
    sbb = np.zeros((nboun, 3))
    sbb[:NC] = -cm.A
    sbb[NC:, 2] = cm.A[:, 2]
    anp = sbb / np.linalg.norm(sbb, axis=1)[:, None]
    z2 = np.zeros((0, 2), dtype=np.int32)
    return RefMesh(npoin=npoin, nedge=nedge, nbface=0, nboun=nboun, coord=coord, vol=vol,
                   iedge=iedge, sn=sn, kbface=z2.copy(), sb=np.zeros((0, 3)), ibpoin=ibpoin,
                   sbb=sbb, anp=anp, icoin=z2.copy(), icoin2=z2.copy(),
                   icoin4=np.zeros((0, 4), dtype=np.int32))


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
