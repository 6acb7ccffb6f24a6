"""Host-side locally refined 2+1D space-time meshes and their DOF maps (P1).

In the reference the adaptive meshes come from its own refinement (src/mesh/refinement,
``refine_points_n_times`` in algorithm/support/space_time_1d.hpp:67) and the DOF maps from
its FE spaces (src/finite_element/fespace); both are host integer work.  The hot path
consumes only their flattened form (geometry rows, CellRestriction rows with weights,
Y -> X ancestors).  This module builds such inputs for benchmarks of the learned-
preconditioner configuration (about 4M space-time DOFs, several levels of local
refinement near a seeded interior point, a diffusivity with contrast 1e4) without the
reference:

* time is cut into intervals, uniformly at the base level and then halved again near t*;
* each time interval carries one conforming spatial triangulation from a nested hierarchy
  M^0 = the uniform union-jack mesh of the base level, M^{j+1} = newest-vertex bisection of
  M^j (each triangle whose centroid lies within r_j of x* bisected twice, conforming
  closure), the depth of an interval falling with its distance from t*;
* Y (broken in time): P1 x P1 on every interval's mesh, zero on the spatial boundary;
* X (continuous in time): at every time level the trace space is P1 on the coarser of the
  two adjacent interval meshes; the finer side's nodes that the coarser mesh lacks are
  hanging nodes, their restriction rows the barycentric weights of the coarse triangle
  that contains them (several weighted entries per row, as the reference's
  constrained_dofs.hpp:133-226 produces);
* Y cells coincide with X cells (the first pass of an inner loop), so y_to_x is the
  identity.

Local DOF order i_space * 2 + i_time, vertices of every triangle counter-clockwise with the
newest vertex first (its refinement edge is v1 v2).
"""
from __future__ import annotations

import math

import numpy as np

from .mesh import Restriction, SpaceTimeProblem, _triangles


class Bisection:
    """Conforming newest-vertex bisection of a triangulation of the unit square."""

    def __init__(self, level: int):
        n = 2 ** (level + 1)
        tris = _triangles(n)
        self.n = n
        grid_ids = tris[..., 1] * (n + 1) + tris[..., 0]
        ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="xy")
        self.xy = [tuple(p) for p in np.stack([ii.ravel() / n, jj.ravel() / n], -1)]
        self.tris = [tuple(int(v) for v in t) for t in grid_ids]   # (peak, b, c): refinement edge b c
        self.alive = [True] * len(self.tris)
        self.edge = {}                                             # edge key -> triangles
        for t, tri in enumerate(self.tris):
            self._add(t, tri)
        self.mid = {}                                              # edge key -> midpoint vertex

    @staticmethod
    def _key(a, b):
        return (a, b) if a < b else (b, a)

    def _add(self, t, tri):
        for e in ((tri[0], tri[1]), (tri[1], tri[2]), (tri[2], tri[0])):
            self.edge.setdefault(self._key(*e), []).append(t)

    def _remove(self, t, tri):
        for e in ((tri[0], tri[1]), (tri[1], tri[2]), (tri[2], tri[0])):
            lst = self.edge[self._key(*e)]
            lst.remove(t)
            if not lst:
                del self.edge[self._key(*e)]

    def _midpoint(self, b, c):
        k = self._key(b, c)
        m = self.mid.get(k)
        if m is None:
            pb, pc = self.xy[b], self.xy[c]
            m = len(self.xy)
            self.xy.append(((pb[0] + pc[0]) * 0.5, (pb[1] + pc[1]) * 0.5))
            self.mid[k] = m
        return m

    def _split(self, t):
        a, b, c = self.tris[t]
        m = self._midpoint(b, c)
        self._remove(t, self.tris[t])
        self.alive[t] = False
        kids = []
        for tri in ((m, a, b), (m, c, a)):   # newest vertex m first, orientation kept
            k = len(self.tris)
            self.tris.append(tri)
            self.alive.append(True)
            self._add(k, tri)
            kids.append(k)
        return kids

    def bisect(self, t):
        """Bisect triangle t and whatever closure needs; returns its two children."""
        a, b, c = self.tris[t]
        nb = [s for s in self.edge.get(self._key(b, c), []) if s != t]
        if nb:
            s = nb[0]
            sa, sb, sc = self.tris[s]
            if self._key(sb, sc) != self._key(b, c):
                # the neighbour's refinement edge differs: bisect it first; one of its
                # children then shares t's refinement edge as its own
                self.bisect(s)
                nb = [u for u in self.edge.get(self._key(b, c), []) if u != t]
                s = nb[0]
            self._split(s)
        return self._split(t)

    def active(self):
        return np.array([tri for tri, ok in zip(self.tris, self.alive) if ok], dtype=np.int64)

    def coords(self):
        return np.asarray(self.xy, dtype=np.float64)


def spatial_hierarchy(level: int, center, depth: int, radius0: float, shrink: float = 0.5):
    """[M^0, ..., M^depth]: M^{j+1} bisects twice every triangle of M^j whose centroid lies
    within radius0 * shrink^j of center (with conforming closure).  Returns (coords, meshes)."""
    bis = Bisection(level)
    meshes = [bis.active()]
    for j in range(depth):
        r = radius0 * shrink ** j
        xy = bis.coords()
        ids = [t for t, ok in enumerate(bis.alive) if ok]
        tri = np.array([bis.tris[t] for t in ids])
        cen = xy[tri].mean(axis=1)
        near = np.hypot(cen[:, 0] - center[0], cen[:, 1] - center[1]) <= r
        for t in np.asarray(ids)[near]:
            if not bis.alive[t]:
                continue   # already split by an earlier closure: its children are finer already
            for k in bis.bisect(int(t)):
                if bis.alive[k]:
                    bis.bisect(k)
        meshes.append(bis.active())
    return bis.coords(), meshes


def _locate(xy, tris, pts):
    """For every point: (triangle index, barycentric weights) in the triangulation."""
    P = xy[tris]                                              # [nt, 3, 2]
    lo, hi = P.min(axis=1), P.max(axis=1)
    nb = 256
    cell = lambda v: np.clip((v * nb).astype(np.int64), 0, nb - 1)  # noqa: E731
    buckets = {}
    bx0, by0 = cell(lo[:, 0] - 1e-12), cell(lo[:, 1] - 1e-12)
    bx1, by1 = cell(hi[:, 0] + 1e-12), cell(hi[:, 1] + 1e-12)
    for t in range(len(tris)):
        for i in range(bx0[t], bx1[t] + 1):
            for j in range(by0[t], by1[t] + 1):
                buckets.setdefault(i * nb + j, []).append(t)
    out_t = np.empty(len(pts), dtype=np.int64)
    out_w = np.empty((len(pts), 3))
    qx, qy = cell(pts[:, 0]), cell(pts[:, 1])
    for q, p in enumerate(pts):
        best = None
        for t in buckets.get(int(qx[q]) * nb + int(qy[q]), []):
            a, b, c = P[t]
            d = (b[0] - a[0]) * (c[1] - a[1]) - (c[0] - a[0]) * (b[1] - a[1])
            l1 = ((p[0] - a[0]) * (c[1] - a[1]) - (c[0] - a[0]) * (p[1] - a[1])) / d
            l2 = ((b[0] - a[0]) * (p[1] - a[1]) - (p[0] - a[0]) * (b[1] - a[1])) / d
            w = np.array([1.0 - l1 - l2, l1, l2])
            if w.min() >= -1e-12:
                best = (t, w)
                break
        if best is None:
            raise RuntimeError("point location failed")
        out_t[q], out_w[q] = best
    # snap rounding: weights of nested dyadic refinements are dyadic rationals
    out_w = np.round(out_w * 2 ** 20) / 2 ** 20
    return out_t, out_w


def time_intervals(level: int, t_star: float, extra: int, width0: float):
    """Base 2^level intervals, then `extra` rounds of halving every interval that lies
    within width0 * 2^-j of t_star (round j)."""
    t = np.linspace(0.0, 1.0, 2 ** level + 1)
    for j in range(extra):
        w = width0 * 0.5 ** j
        mids = 0.5 * (t[:-1] + t[1:])
        near = np.abs(mids - t_star) <= w + 0.5 * (t[1:] - t[:-1])
        t = np.sort(np.concatenate([t, mids[near]]))
    return t


def locally_refined_problem(level: int = 6, seed: int = 0, depth: int = 5, radius0: float = 0.25,
                            time_rounds: int = 3, kappa_range=(0.01, 100.0), kappa_blocks: int = 8,
                            u0_kind: int = 0, return_hierarchy: bool = False):
    """The learned-preconditioner benchmark's problem: outer level `level` uniform base, a
    seeded interior point (x*, t*) drawn uniformly from [0.25, 0.75]^3, `depth` levels of
    local spatial bisection around x* (interval depth falling by one per step of
    2^-(level+1) away from t*... see interval_depths) and `time_rounds` halvings of the
    intervals near t*; kappa log-uniform in kappa_range, constant on each of the
    kappa_blocks x kappa_blocks squares of the unit square (so constant on every cell)."""
    rng = np.random.default_rng(seed)
    cx, cy, ts = rng.uniform(0.25, 0.75, 3)
    xy, meshes = spatial_hierarchy(level, (cx, cy), depth, radius0)
    T = time_intervals(level, ts, time_rounds, 2.0 ** -(level - 1))
    nint = len(T) - 1
    mids = 0.5 * (T[:-1] + T[1:])
    # depth per interval: full depth at t*, one level less per base interval of distance
    dist = np.abs(mids - ts) * 2 ** level
    dk = np.clip(depth - np.floor(dist).astype(np.int64), 0, depth)
    nv = len(xy)
    on_bnd = (np.abs(xy[:, 0]) < 1e-14) | (np.abs(xy[:, 0] - 1) < 1e-14) | \
             (np.abs(xy[:, 1]) < 1e-14) | (np.abs(xy[:, 1] - 1) < 1e-14)
    # interior vertex numbering of every mesh of the hierarchy
    vnum = []
    for M in meshes:
        present = np.zeros(nv, dtype=bool)
        present[M.ravel()] = True
        inner = present & ~on_bnd
        idx = -np.ones(nv, dtype=np.int64)
        idx[inner] = np.arange(int(inner.sum()))
        vnum.append(idx)
    # X time levels: trace depth e_i = min of the adjacent intervals' depths
    e = np.empty(nint + 1, dtype=np.int64)
    e[0], e[-1] = dk[0], dk[-1]
    e[1:-1] = np.minimum(dk[:-1], dk[1:])
    x_base = np.zeros(nint + 2, dtype=np.int64)
    for i in range(nint + 1):
        x_base[i + 1] = x_base[i] + int((vnum[e[i]] >= 0).sum())
    n_u = int(x_base[-1])
    y_base = np.zeros(nint + 1, dtype=np.int64)
    for k in range(nint):
        y_base[k + 1] = y_base[k] + 2 * int((vnum[dk[k]] >= 0).sum())
    n_lambda = int(y_base[-1])
    # hanging-node weights: vertex of M^d not in M^e, located in M^e -> per vertex id the
    # coarse triangle's vertices and weights (index table over all vertex ids)
    hang = {}

    def hanging(d, ee):
        key = (d, ee)
        if key not in hang:
            fine = np.unique(meshes[d].ravel())
            in_coarse = np.zeros(nv, dtype=bool)
            in_coarse[meshes[ee].ravel()] = True
            q = fine[~in_coarse[fine]]
            t, w = _locate(xy, meshes[ee], xy[q])
            row = -np.ones(nv, dtype=np.int64)
            row[q] = np.arange(len(q))
            hang[key] = (row, meshes[ee][t], w)
        return hang[key]

    geo_parts, yd_parts, vid_parts, xd_parts, xw_parts = [], [], [], [], []
    for k in range(nint):
        M = meshes[dk[k]]
        nt_ = M.shape[0]
        g = np.empty((nt_, 8))
        g[:, :6] = xy[M].reshape(nt_, 6)
        g[:, 6], g[:, 7] = T[k], T[k + 1]
        geo_parts.append(g)
        vid_parts.append(M.astype(np.int32))
        # Y: interior vertex of this interval's mesh, two time levels
        yv = vnum[dk[k]][M]                                   # [nt, 3]
        yid = np.where(yv[:, :, None] >= 0, y_base[k] + 2 * yv[:, :, None] + np.arange(2)[None, None, :], -1)
        yd_parts.append(yid.reshape(nt_, 6))
        # X: bottom level k (a = 0), top level k + 1 (a = 1); up to 3 entries per row
        dofs = -np.ones((nt_, 3, 2, 3), dtype=np.int64)
        wts = np.zeros((nt_, 3, 2, 3))
        for lvl, a in ((k, 0), (k + 1, 1)):
            ee = e[lvl]
            num = vnum[ee]
            direct = num[M]                                    # [nt, 3]
            dofs[:, :, a, 0] = np.where(direct >= 0, x_base[lvl] + direct, -1)
            wts[:, :, a, 0] = np.where(direct >= 0, 1.0, 0.0)
            if ee < dk[k]:
                row, cverts, cw = hanging(dk[k], ee)
                hr = row[M]                                    # [nt, 3] row of the hanging table or -1
                hmask = hr >= 0
                hv = cverts[hr[hmask]]                         # [nh, 3] coarse vertices
                hwt = cw[hr[hmask]]
                hn = num[hv]
                ok = (hn >= 0) & (hwt != 0.0)
                dd = np.where(ok, x_base[lvl] + hn, -1)
                ww = np.where(ok, hwt, 0.0)
                sub_d = dofs[:, :, a, :]
                sub_w = wts[:, :, a, :]
                sub_d[hmask] = dd
                sub_w[hmask] = ww
                dofs[:, :, a, :] = sub_d
                wts[:, :, a, :] = sub_w
        xd_parts.append(dofs.reshape(nt_ * 6, 3))
        xw_parts.append(wts.reshape(nt_ * 6, 3))
    ncell = sum(g.shape[0] for g in geo_parts)
    geo = np.concatenate(geo_parts)
    ydof = np.concatenate(yd_parts).ravel()
    has = ydof >= 0
    y_off = np.zeros(ydof.size + 1, dtype=np.int32)
    y_off[1:] = np.cumsum(has)
    y_r = Restriction(y_off, ydof[has].astype(np.int32), np.ones(int(has.sum())), 6)
    xd = np.concatenate(xd_parts)
    xw = np.concatenate(xw_parts)
    # entries of a row in coarse-vertex order, the absent ones dropped
    keep = xd >= 0
    cnt = keep.sum(axis=1)
    x_off = np.zeros(cnt.size + 1, dtype=np.int32)
    x_off[1:] = np.cumsum(cnt)
    x_r = Restriction(x_off, xd[keep].astype(np.int32), xw[keep], 6)
    # kappa per cell from its block of the unit square
    lo, hi = kappa_range
    kb = np.exp(rng.uniform(math.log(lo), math.log(hi), (kappa_blocks, kappa_blocks)))
    cen = geo[:, :6].reshape(-1, 3, 2).mean(axis=1)
    bi = np.clip((cen * kappa_blocks).astype(np.int64), 0, kappa_blocks - 1)
    kap = kb[bi[:, 0], bi[:, 1]]
    m_cells = np.stack([kap, np.zeros_like(kap), kap], axis=1)
    prob = SpaceTimeProblem(
        p=1, y_geometry=geo, x_geometry=geo.copy(), y_to_x=np.arange(ncell, dtype=np.int32),
        y_restriction=y_r, x_restriction=x_r, n_lambda=n_lambda, n_u=n_u, m_cells=m_cells, u0_kind=u0_kind,
        y_vertex_ids=np.concatenate(vid_parts),
        meta=dict(level=level, seed=seed, depth=depth, point=(float(cx), float(cy), float(ts)),
                  intervals=nint, interval_depths=dk.tolist(), spatial_triangles=[int(M.shape[0]) for M in meshes],
                  kappa_range=list(kappa_range), kappa_blocks=kappa_blocks))
    if return_hierarchy:
        return prob, (xy, meshes, T, dk, e)
    return prob
