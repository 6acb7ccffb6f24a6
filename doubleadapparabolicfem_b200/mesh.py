"""Host-side uniform space-time prism meshes and DOF maps for the hot path.

In the reference the mesh, the FE spaces and their DOF maps are host integer work
done by ``mesh::Mesh`` / ``finite_element::FESpace`` (src/mesh, src/finite_element/fespace);
they stay on the host.  This module builds the same *uniform* meshes the
reference reaches with its uniform isotropic X refinement
(algorithm/adaptive_driver.hpp:1751-1830, the ``uniform_standard`` runs of the
paper data) so that benchmarks and tests can run without the reference:

* outer level L >= 1 of the unit square x (0,1): n = 2^(L+1) squares per side,
  every square split by one diagonal, '/' when (i+j) is even and '\\' when odd
  (the union-jack pattern newest-vertex bisection produces from the two-triangle
  root), and nt = 2^L time slabs;
* X = continuous-in-time P_p x P_p, Y = broken-in-time P_p x P_p, homogeneous
  Dirichlet data on the spatial boundary (boundary local DOFs have empty
  restriction rows, as in src/finite_element/assembly/constrained_dofs.hpp:133-226);
* local DOF order i_space*(p+1) + i_time with triangle nodes in the reference's
  equidistant order (vertices v0, v1, v2 of the cell; for p=2: v0, m01, v1, m02,
  m12, v2).

Cell geometry and DOF counts equal the reference's; the DOF *numbering* is this
module's own (time-level major, then lexicographic in space), so comparisons
against reference fixtures go through a coordinate-based permutation.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Restriction:
    """Flattened CellRestriction: row (cell c, local i) = entries offsets[c*ndof+i]:offsets[c*ndof+i+1]."""
    offsets: np.ndarray   # int32 [n_cells*ndof+1]
    dofs: np.ndarray      # int32
    weights: np.ndarray   # float64
    ndof: int


@dataclass
class SpaceTimeProblem:
    """Host inputs of the main-system assembly (see include/apf_b200.h, apf_problem_desc)."""
    p: int
    y_geometry: np.ndarray          # [n_y_cells, 8] x0 y0 x1 y1 x2 y2 t0 t1
    x_geometry: np.ndarray          # [n_x_cells, 8]
    y_to_x: np.ndarray              # int32 [n_y_cells]
    y_restriction: Restriction
    x_restriction: Restriction
    n_lambda: int
    n_u: int
    m_cells: np.ndarray | None = None     # [n_y_cells, 3] or None (identity)
    ell_cells: np.ndarray | None = None   # [n_y_cells] or None (zero load)
    u0_kind: int = 0                      # 0 sin(pi x) sin(pi y), 1 one, 2 zero
    y_vertex_ids: np.ndarray | None = None  # [n_y_cells, 3] spatial vertex ids (estimator patches)
    meta: dict = field(default_factory=dict)
    dim_space: int = 2                    # 1: 1+1D quads, geometry rows x0 x1 t0 t1, m_cells [n_y_cells]

    @property
    def ndof(self) -> int:
        if self.dim_space == 1:
            return (self.p + 1) * (self.p + 1)
        return (self.p + 1) * (self.p + 2) // 2 * (self.p + 1)

    @property
    def n_y_cells(self) -> int:
        return int(self.y_geometry.shape[0])

    @property
    def n_x_cells(self) -> int:
        return int(self.x_geometry.shape[0])


def _triangles(n: int):
    """Vertex grid indices (i, j) of the 2 n^2 triangles, counter-clockwise, right angle first."""
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    ii = ii.ravel()
    jj = jj.ravel()
    even = ((ii + jj) % 2) == 0
    tris = np.empty((2 * n * n, 3, 2), dtype=np.int64)
    # '/' diagonal (i,j)-(i+1,j+1): lower-right and upper-left triangles
    # '\' diagonal (i+1,j)-(i,j+1): lower-left and upper-right triangles
    a = np.stack([ii, jj], -1)
    b = np.stack([ii + 1, jj], -1)
    c = np.stack([ii + 1, jj + 1], -1)
    d = np.stack([ii, jj + 1], -1)
    t0 = np.where(even[:, None, None], np.stack([b, c, a], 1), np.stack([a, b, d], 1))
    t1 = np.where(even[:, None, None], np.stack([d, a, c], 1), np.stack([c, d, b], 1))
    tris[0::2] = t0
    tris[1::2] = t1
    return tris


def uniform_problem(level: int, p: int = 1, u0_kind: int = 0, m_cells=None) -> SpaceTimeProblem:
    """Uniform 2+1D space-time mesh of outer level ``level`` (>= 1) on (0,1)^2 x (0,1)."""
    if level < 1:
        raise ValueError("level must be >= 1")
    if p not in (1, 2):
        raise ValueError("p must be 1 or 2")
    n = 2 ** (level + 1)
    nt = 2 ** level
    tris = _triangles(n)                              # [ntri, 3, 2] integer grid coordinates
    ntri = tris.shape[0]
    ns = (p + 1) * (p + 2) // 2
    ntl = p + 1
    ndof = ns * ntl
    # spatial nodes on the p-refined grid (coordinates in units of h/p)
    G = p * n + 1
    v = tris * p                                     # vertex nodes on the refined grid
    if p == 1:
        snodes = v                                   # v0 v1 v2
    else:
        m01 = (v[:, 0] + v[:, 1]) // 2
        m02 = (v[:, 0] + v[:, 2]) // 2
        m12 = (v[:, 1] + v[:, 2]) // 2
        snodes = np.stack([v[:, 0], m01, v[:, 1], m02, m12, v[:, 2]], 1)
    si, sj = snodes[..., 0], snodes[..., 1]
    interior = (si > 0) & (si < G - 1) & (sj > 0) & (sj < G - 1)
    n_in = (G - 2)
    sp_id = np.where(interior, (sj - 1) * n_in + (si - 1), -1)   # interior spatial node id
    n_sp = n_in * n_in
    # time: slab k, local time node a -> X time level k*p + a ; Y local (k, a)
    h = 1.0 / n
    xy = tris.astype(np.float64) * h
    geo_tri = xy.reshape(ntri, 6)
    cells_k = np.repeat(np.arange(nt), ntri)                       # slab-major cell order
    geo = np.empty((nt * ntri, 8))
    geo[:, :6] = np.tile(geo_tri, (nt, 1))
    geo[:, 6] = cells_k / nt
    geo[:, 7] = (cells_k + 1) / nt
    # local DOF ids
    sp = np.tile(sp_id, (nt, 1))                                   # [ncell, ns]
    k = cells_k[:, None, None]
    a = np.arange(ntl)[None, None, :]
    spb = sp[:, :, None]
    x_ids = np.where(spb >= 0, (k * p + a) * n_sp + spb, -1).reshape(-1, ndof)
    y_ids = np.where(spb >= 0, (k * ntl + a) * n_sp + spb, -1).reshape(-1, ndof)
    n_u = (nt * p + 1) * n_sp
    n_lambda = nt * ntl * n_sp

    def restriction(ids):
        has = (ids.ravel() >= 0)
        offsets = np.zeros(ids.size + 1, dtype=np.int32)
        offsets[1:] = np.cumsum(has)
        dofs = ids.ravel()[has].astype(np.int32)
        return Restriction(offsets, dofs, np.ones(dofs.size), ndof)

    ncell = geo.shape[0]
    # spatial vertex ids (grid index of the P1 vertices), the same in every slab
    vids = (tris[..., 1] * (n + 1) + tris[..., 0]).astype(np.int32)
    return SpaceTimeProblem(
        p=p, y_geometry=geo, x_geometry=geo.copy(), y_to_x=np.arange(ncell, dtype=np.int32),
        y_restriction=restriction(y_ids), x_restriction=restriction(x_ids),
        n_lambda=int(n_lambda), n_u=int(n_u), m_cells=m_cells, u0_kind=u0_kind,
        y_vertex_ids=np.tile(vids, (nt, 1)),
        meta=dict(level=level, n=n, nt=nt, n_spatial_interior=n_sp))


def uniform_problem_1d(level: int, u0_kind: int = 0, m_cells=None) -> SpaceTimeProblem:
    """1+1D heat problem on (0,1) x (0,1), P1 x P1 quadrilaterals, after the example's
    initial refinement and `level` uniform outer refinements: n = 2^(level+1) intervals in
    space and in time (the reference's `uniform_standard` outer iteration `level`; X has
    (n-1)(n+1) true DOFs, Y (n-1) 2n).  Homogeneous Dirichlet data at x = 0, 1: the
    boundary nodes own no true DOF (empty restriction rows).  Cells are numbered time
    slab by time slab, left to right; DOFs by spatial node, then time."""
    n = 2 ** (level + 1)
    h = 1.0 / n
    m_idx, i_idx = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")  # time slab m, space cell i
    m_idx = m_idx.ravel()
    i_idx = i_idx.ravel()
    geo = np.stack([i_idx * h, (i_idx + 1) * h, m_idx * h, (m_idx + 1) * h], axis=1).astype(np.float64)
    n_cells = n * n

    def restriction(dof_of):
        offsets = np.zeros(n_cells * 4 + 1, dtype=np.int32)
        dofs = []
        k = 0
        for c in range(n_cells):
            for loc in range(4):
                s_node, a = loc >> 1, loc & 1
                node = i_idx[c] + s_node
                if 0 < node < n:
                    dofs.append(dof_of(node, m_idx[c], a))
                k += 1
                offsets[k] = len(dofs)
        d = np.asarray(dofs, dtype=np.int32)
        return Restriction(offsets, d, np.ones(len(d)), 4)

    x_r = restriction(lambda node, m, a: (node - 1) * (n + 1) + m + a)
    y_r = restriction(lambda node, m, a: (node - 1) * (2 * n) + 2 * m + a)
    return SpaceTimeProblem(p=1, y_geometry=geo, x_geometry=geo.copy(), y_to_x=np.arange(n_cells, dtype=np.int32),
                            y_restriction=y_r, x_restriction=x_r, n_lambda=(n - 1) * 2 * n, n_u=(n - 1) * (n + 1),
                            m_cells=m_cells, u0_kind=u0_kind, dim_space=1,
                            meta={"level": level, "intervals": n})


def dof_coordinates(problem: SpaceTimeProblem, space: str):
    """(x, y, t, slab_mid) of every true DOF of space 'x' or 'y' (slab_mid distinguishes the
    two Y DOFs at a slab interface; for X it is 0)."""
    geo = problem.y_geometry if space == "y" else problem.x_geometry
    R = problem.y_restriction if space == "y" else problem.x_restriction
    n = problem.n_lambda if space == "y" else problem.n_u
    p = problem.p
    ns = (p + 1) * (p + 2) // 2
    ntl = p + 1
    tn = np.array([(b / p, c / p) for c in range(p + 1) for b in range(p + 1 - c)])
    out = np.full((n, 4), np.nan)
    cnt = np.diff(R.offsets)
    rows = np.repeat(np.arange(cnt.size), cnt)
    cell = rows // R.ndof
    loc = rows % R.ndof
    s, a = loc // ntl, loc % ntl
    g = geo[cell]
    xi, eta = tn[s, 0], tn[s, 1]
    x = g[:, 0] + (g[:, 2] - g[:, 0]) * xi + (g[:, 4] - g[:, 0]) * eta
    y = g[:, 1] + (g[:, 3] - g[:, 1]) * xi + (g[:, 5] - g[:, 1]) * eta
    t = g[:, 6] + (g[:, 7] - g[:, 6]) * a / p
    mid = 0.5 * (g[:, 6] + g[:, 7]) if space == "y" else np.zeros_like(t)
    out[R.dofs] = np.stack([x, y, t, mid], -1)
    return out
