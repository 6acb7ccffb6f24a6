"""ORACLE — CPU restatement of the reference's hot-path arithmetic (test infrastructure).

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import this module, and only as the
checker or as the timed CPU baseline; the product path never calls it.

Parity status: PINNED.  Every function here is checked in ``tests/`` against
fixtures written by the reference's own C++ templates (``oracle/ref_dump.cpp``,
compiled from the reference sources with ``oracle/shim`` standing in for Eigen)
and, for DOF counts and estimator values, against the reference's published
``algorithm_data_plot`` CSV rows copied into ``tests/golden``.

Restated reference code (paths relative to the reference project root):

* quadrature — ``src/quadrature/reference_triangle_duffy.hpp`` (Duffy rule of
  order (D+3)/2 squared), ``src/quadrature/reference_quadrature.hpp:36``
  (prism = Duffy triangle x Gauss–Legendre time), Gauss–Legendre on [0,1];
* bases — ``src/finite_element/basis/functions/triangular_prism_lagrange.hpp:27-30``
  (local index ``i_space * N_time + i_time``), equidistant triangle nodes in
  ``src/finite_element/nodes/triangle_equidistant.hpp`` order, equidistant
  time nodes ``i/Q``;
* geometry — ``src/finite_element/geometry/cell_geometry.hpp:188-302``;
* main blocks — ``src/finite_element/assembly/main_system/dense_local_main_blocks_2d.hpp``
  (Y-cell loop ``:212-327`` for A_y, B, f; trace loop ``:760-800`` for C_signed, g),
  scatter with the per-local-entry ``zero_tol`` filter
  ``src/finite_element/assembly/scatter.hpp:66-115,227-254``;
* graph-norm preconditioner block — ``src/finite_element/assembly/main_system/parabolic_graph_norm.hpp:22-65``
  and ``src/linear_algebra/preconditioners/schur_approximations.hpp:79-287``;
* full saddle matrix of the direct-solver path — ``src/finite_element/assembly/main_system/two_pass_full_saddle_2d.hpp:468``
  (structural pattern, numeric fill, ``prune(1.0, zero_tol)``);
* time-slab space and slab reconstruction lambda~ on adaptive meshes —
  ``src/finite_element/time_slabs/time_slab_builder.hpp:53-215`` (slab times = distinct
  Y-cell endpoints, every Y cell cut into one slab cell per slab it spans),
  ``time_slab.hpp:185-242`` (a slab cell is its source cell over the slab interval),
  ``time_slab_reconstruction_operator.hpp:686-830`` (per slab, A_slab lambda~ = rhs with the
  main-system forms: the Y-norm stiffness and l - d_t u - M grad u tested against the slab
  space).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp


# ----------------------------------------------------------------------------
# quadrature
# ----------------------------------------------------------------------------
def gauss_legendre01(n: int):
    """n-point Gauss–Legendre rule mapped to [0,1] (src/quadrature/gauss_legendre_1d.hpp)."""
    x, w = np.polynomial.legendre.leggauss(n)
    return 0.5 * (x + 1.0), 0.5 * w


def duffy_triangle(degree: int):
    """Collapsed (Duffy) rule on conv{(0,0),(1,0),(0,1)} exact to ``degree``.

    reference_triangle_duffy.hpp: order = (degree+3)//2, points (u, (1-u) v),
    weights w_u w_v (1-u), u outer / v inner loop order.
    """
    order = (degree + 3) // 2
    u, wu = gauss_legendre01(order)
    pts, wts = [], []
    for i in range(order):
        for j in range(order):
            pts.append((u[i], (1.0 - u[i]) * u[j]))
            wts.append(wu[i] * wu[j] * (1.0 - u[i]))
    return np.array(pts), np.array(wts)


def prism_rule(q_space: int, q_time: int):
    """Tensor prism rule: Duffy(q_space) x GL(q_time) (tensor_product_quadrature.hpp order:
    triangle point outer, time point inner)."""
    tp, tw = duffy_triangle(q_space)
    t, w = gauss_legendre01(q_time)
    pts = np.array([(a[0], a[1], tt) for a in tp for tt in t])
    wts = np.array([aw * ww for aw in tw for ww in w])
    return pts, wts


# ----------------------------------------------------------------------------
# bases
# ----------------------------------------------------------------------------
def triangle_nodes(p: int):
    """Equidistant triangle nodes in reference order: c outer, b inner, (b/p, c/p)."""
    return np.array([(b / p, c / p) for c in range(p + 1) for b in range(p + 1 - c)])


def _bary(xi, eta):
    return np.stack([1.0 - xi - eta, xi, eta], axis=-1)


def tri_lagrange(p: int, xi, eta):
    """Values [..., N] and gradients [..., N, 2] of the nodal Lagrange basis on the
    reference triangle (same node order as triangle_nodes)."""
    xi = np.asarray(xi, dtype=np.float64)
    eta = np.asarray(eta, dtype=np.float64)
    L = _bary(xi, eta)
    dL = np.array([[-1.0, -1.0], [1.0, 0.0], [0.0, 1.0]])
    if p == 1:
        vals = L
        grads = np.broadcast_to(dL, xi.shape + (3, 2)).copy()
        return vals, grads
    if p == 2:
        # nodes: (0,0) (.5,0) (1,0) (0,.5) (.5,.5) (0,1)  == v0, e01, v1, e02, e12, v2
        l0, l1, l2 = L[..., 0], L[..., 1], L[..., 2]
        vals = np.stack([
            l0 * (2 * l0 - 1), 4 * l0 * l1, l1 * (2 * l1 - 1),
            4 * l0 * l2, 4 * l1 * l2, l2 * (2 * l2 - 1)], axis=-1)
        g0, g1, g2 = dL
        def gv(a):
            return a[..., None]
        grads = np.stack([
            gv(4 * l0 - 1) * g0,
            4 * (gv(l0) * g1 + gv(l1) * g0),
            gv(4 * l1 - 1) * g1,
            4 * (gv(l0) * g2 + gv(l2) * g0),
            4 * (gv(l1) * g2 + gv(l2) * g1),
            gv(4 * l2 - 1) * g2], axis=-2)
        return vals, grads
    raise NotImplementedError("p must be 1 or 2")


def seg_lagrange(q: int, tau):
    """Values [..., q+1] and derivatives of the equidistant Lagrange basis on [0,1]
    (nodes i/q in order)."""
    tau = np.asarray(tau, dtype=np.float64)
    nodes = np.arange(q + 1) / q
    vals, ders = [], []
    for i in range(q + 1):
        v = np.ones_like(tau)
        for k in range(q + 1):
            if k != i:
                v = v * (tau - nodes[k]) / (nodes[i] - nodes[k])
        d = np.zeros_like(tau)
        for m in range(q + 1):
            if m == i:
                continue
            term = np.ones_like(tau) / (nodes[i] - nodes[m])
            for k in range(q + 1):
                if k != i and k != m:
                    term = term * (tau - nodes[k]) / (nodes[i] - nodes[k])
            d = d + term
        vals.append(v)
        ders.append(d)
    return np.stack(vals, -1), np.stack(ders, -1)


def prism_basis(p: int, pts):
    """Prism values [nq, N] and reference gradients [nq, N, 3]; local index i_s*(p+1)+i_t."""
    tv, tg = tri_lagrange(p, pts[:, 0], pts[:, 1])
    sv, sd = seg_lagrange(p, pts[:, 2])
    nq = pts.shape[0]
    ns, nt = tv.shape[1], sv.shape[1]
    vals = (tv[:, :, None] * sv[:, None, :]).reshape(nq, ns * nt)
    g = np.empty((nq, ns, nt, 3))
    g[..., 0] = tg[:, :, None, 0] * sv[:, None, :]
    g[..., 1] = tg[:, :, None, 1] * sv[:, None, :]
    g[..., 2] = tv[:, :, None] * sd[:, None, :]
    return vals, g.reshape(nq, ns * nt, 3)


# ----------------------------------------------------------------------------
# mesh input
# ----------------------------------------------------------------------------
@dataclass
class Restriction:
    """Flattened CellRestriction (src/finite_element/assembly/constrained_dofs.hpp:37-58):
    row (cell c, local i) = entries offsets[c*ndof+i] : offsets[c*ndof+i+1]."""
    offsets: np.ndarray
    dofs: np.ndarray
    weights: np.ndarray
    ndof: int

    @property
    def n_cells(self):
        return (len(self.offsets) - 1) // self.ndof


@dataclass
class MainProblem:
    p: int
    y_geom: np.ndarray         # [ny, 8] x0 y0 x1 y1 x2 y2 t0 t1
    x_geom: np.ndarray         # [nx, 8]
    y_to_x: np.ndarray         # [ny] index into x cells
    y_restr: Restriction
    x_restr: Restriction
    n_lambda: int
    n_u: int
    m_cells: np.ndarray | None = None   # [ny, 3] (m00, m01, m11) per Y cell; None = identity
    dim_space: int = 2                  # 1: quads, geometry rows x0 x1 t0 t1, m_cells [ny]


def geometry_terms(geom):
    """J, inverse, |det J| per cell (cell_geometry.hpp:188-242)."""
    x0, y0 = geom[:, 0], geom[:, 1]
    J00 = geom[:, 2] - x0
    J01 = geom[:, 4] - x0
    J10 = geom[:, 3] - y0
    J11 = geom[:, 5] - y0
    det = J00 * J11 - J01 * J10
    inv = 1.0 / det
    invJT = np.stack([np.stack([J11 * inv, -J10 * inv], -1),
                      np.stack([-J01 * inv, J00 * inv], -1)], -2)   # [n,2,2] rows: invJT0*, invJT1*
    invJ = np.stack([np.stack([J11 * inv, -J01 * inv], -1),
                     np.stack([-J10 * inv, J00 * inv], -1)], -2)
    t0, t1 = geom[:, 6], geom[:, 7]
    return dict(x0=x0, y0=y0, J=np.stack([np.stack([J00, J01], -1), np.stack([J10, J11], -1)], -2),
                invJ=invJ, invJT=invJT, absdet=np.abs(det), t0=t0, ht=t1 - t0)


def _expand(restr: Restriction):
    """Per (cell, local) lists as padded arrays [n_cells, ndof, kmax] (dof=-1 for padding)."""
    cnt = np.diff(restr.offsets)
    kmax = max(1, int(cnt.max()) if cnt.size else 1)
    n = cnt.size
    dofs = -np.ones((n, kmax), dtype=np.int64)
    w = np.zeros((n, kmax))
    for k in range(kmax):
        has = cnt > k
        idx = restr.offsets[:-1][has] + k
        dofs[has, k] = restr.dofs[idx]
        w[has, k] = restr.weights[idx]
    return dofs.reshape(-1, restr.ndof, kmax), w.reshape(-1, restr.ndof, kmax)


def scatter_matrix(local, test_restr: Restriction, trial_restr: Restriction, shape, zero_tol,
                   test_cells=None, trial_cells=None):
    """A += C_test^T A_c C_trial with the per-entry |a_ij| <= zero_tol skip
    (scatter.hpp:66-115); duplicate summation as setFromTriplets."""
    td, tw = _expand(test_restr)
    rd, rw = _expand(trial_restr)
    if test_cells is not None:
        td, tw = td[test_cells], tw[test_cells]
    if trial_cells is not None:
        rd, rw = rd[trial_cells], rw[trial_cells]
    keep = np.abs(local) > zero_tol                              # [n, ni, nj]
    rows, cols, vals = [], [], []
    for a in range(td.shape[2]):
        for b in range(rd.shape[2]):
            I = td[:, :, a][:, :, None]
            J = rd[:, :, b][:, None, :]
            v = tw[:, :, a][:, :, None] * rw[:, :, b][:, None, :] * local
            m = keep & (I >= 0) & (J >= 0)
            I, J = np.broadcast_arrays(I, J)
            rows.append(I[m]); cols.append(J[m]); vals.append(v[m])
    rows = np.concatenate(rows); cols = np.concatenate(cols); vals = np.concatenate(vals)
    return sp.csc_matrix((vals, (rows, cols)), shape=shape)


def scatter_vector(local, restr: Restriction, n, zero_tol, cells=None):
    d, w = _expand(restr)
    if cells is not None:
        d, w = d[cells], w[cells]
    out = np.zeros(n)
    keep = np.abs(local) > zero_tol
    for a in range(d.shape[2]):
        m = keep & (d[:, :, a] >= 0)
        np.add.at(out, d[:, :, a][m], (w[:, :, a] * local)[m])
    return out


def sin_initial(x, y):
    return np.sin(math.pi * x) * np.sin(math.pi * y)


def one_initial(x, y):
    return np.ones_like(x)


def assemble_main_blocks(prob: MainProblem, u0=sin_initial, ell=None, zero_tol=1e-15, g_scale=-1.0):
    """Restatement of assemble_main_system_blocks for 2+1D (assemble_saddle_problem.hpp:131)."""
    p = prob.p
    qs, qt = 4 * p + 1, 2 * p + 1
    pts, wts = prism_rule(qs, qt)
    phi, dphi_ref = prism_basis(p, pts)            # [nq,N], [nq,N,3]
    gy = geometry_terms(prob.y_geom)
    gx = geometry_terms(prob.x_geom[prob.y_to_x])
    ny = prob.y_geom.shape[0]
    N = phi.shape[1]
    M = prob.m_cells if prob.m_cells is not None else np.tile([1.0, 0.0, 1.0], (ny, 1))
    Mt = np.stack([np.stack([M[:, 0], M[:, 1]], -1), np.stack([M[:, 1], M[:, 2]], -1)], -2)
    dmu = gy["absdet"][:, None] * gy["ht"][:, None] * wts[None, :]          # [n,nq]
    # physical qp (SpaceTimeTriPrismMap2P1D: x = v0 + J xi, t = t0 + ht tau)
    xq = gy["x0"][:, None] + gy["J"][:, 0, 0][:, None] * pts[None, :, 0] + gy["J"][:, 0, 1][:, None] * pts[None, :, 1]
    yq = gy["y0"][:, None] + gy["J"][:, 1, 0][:, None] * pts[None, :, 0] + gy["J"][:, 1, 1][:, None] * pts[None, :, 1]
    tq = gy["t0"][:, None] + gy["ht"][:, None] * pts[None, :, 2]
    grad_phi = np.einsum("nab,qjb->nqja", gy["invJT"], dphi_ref[:, :, :2])   # [n,nq,N,2]
    Mgrad_phi = np.einsum("nab,nqjb->nqja", Mt, grad_phi)
    # X basis at the Y quadrature points, mapped through X's reference coordinates
    dx = xq - gx["x0"][:, None]
    dy = yq - gx["y0"][:, None]
    xi_x = gx["invJ"][:, 0, 0][:, None] * dx + gx["invJ"][:, 0, 1][:, None] * dy
    eta_x = gx["invJ"][:, 1, 0][:, None] * dx + gx["invJ"][:, 1, 1][:, None] * dy
    tau_x = (tq - gx["t0"][:, None]) / gx["ht"][:, None]
    xpts = np.stack([xi_x.ravel(), eta_x.ravel(), tau_x.ravel()], -1)
    _, dpsi_ref = prism_basis(p, xpts)
    dpsi_ref = dpsi_ref.reshape(ny, -1, N, 3)
    grad_psi = np.einsum("nab,nqjb->nqja", gx["invJT"], dpsi_ref[..., :2])
    dt_psi = dpsi_ref[..., 2] / gx["ht"][:, None, None]
    A = np.einsum("nqia,nqja,nq->nij", grad_phi, Mgrad_phi, dmu)
    B = (np.einsum("nqi,qj,nq->nij", dt_psi, phi, dmu)
         + np.einsum("nqia,nqja,nq->nij", grad_psi, Mgrad_phi, dmu))
    if ell is None:
        f_loc = np.zeros((ny, N))
    else:
        f_loc = np.einsum("nq,qj,nq->nj", ell(xq, yq, tq), phi, dmu)
    A_y = scatter_matrix(A, prob.y_restr, prob.y_restr, (prob.n_lambda, prob.n_lambda), zero_tol)
    Bm = scatter_matrix(B, prob.x_restr, prob.y_restr, (prob.n_u, prob.n_lambda), zero_tol,
                        test_cells=prob.y_to_x)
    f = scatter_vector(f_loc, prob.y_restr, prob.n_lambda, zero_tol)
    C, g = assemble_trace_blocks(prob, u0, zero_tol, g_scale)
    return dict(A_y=A_y, B=Bm, C_signed=C, f=f, g=g)


def assemble_main_full_saddle_two_pass(prob: MainProblem, u0=sin_initial, ell=None, zero_tol=1e-15, g_scale=-1.0):
    """Restatement of assemble_main_full_saddle_two_pass_2d
    (src/finite_element/assembly/main_system/two_pass_full_saddle_2d.hpp:468): the full
    saddle matrix K = [A_y B^T; B C_signed] of the direct-solver path and rhs = [f; g].

    Pattern pass (:740-790): the union over Y cells of the restricted (Y x Y), (X ancestor
    x Y) and transposed couplings and over bottom X cells of (X x X), with no value filter.
    Numeric pass (scatter_matrix_by_slots, :431-459): the local entries with |a_ij| >
    zero_tol added into those slots in cell order, so every slot holds the block path's
    sum.  Then ``prune(1.0, zero_tol)`` (:1720) drops every entry with |value| <= zero_tol,
    structural slots no entry reached included.  The local vectors keep the per-entry
    filter (:93-122)."""
    blocks = assemble_main_blocks(prob, u0, ell, zero_tol, g_scale)
    K = sp.bmat([[blocks["A_y"], blocks["B"].T], [blocks["B"], blocks["C_signed"]]], format="csr")
    K.sum_duplicates()
    K.data[np.abs(K.data) <= zero_tol] = 0.0
    K.eliminate_zeros()
    K.sort_indices()
    return K, np.concatenate([blocks["f"], blocks["g"]])


def bottom_cells(x_geom):
    """X cells whose bottom face lies on t = 0 (mesh temporal_boundary[0])."""
    return np.nonzero(x_geom[:, 6] == 0.0)[0]


def assemble_trace_blocks(prob: MainProblem, u0, zero_tol=1e-15, g_scale=-1.0):
    """C_signed = -int_{t=0} psi_i psi_j, g = g_scale int u0 psi_i(.,0)
    (dense_local_main_blocks_2d.hpp:760-800; Duffy bottom rule of degree 4p+1)."""
    p = prob.p
    tp, tw = duffy_triangle(4 * p + 1)
    tv, _ = tri_lagrange(p, tp[:, 0], tp[:, 1])
    sv, _ = seg_lagrange(p, np.zeros(1))
    vals = (tv[:, :, None] * sv[0][None, None, :]).reshape(len(tw), -1)   # [nq,N]
    cells = bottom_cells(prob.x_geom)
    gx = geometry_terms(prob.x_geom[cells])
    dg = gx["absdet"][:, None] * tw[None, :]
    xq = gx["x0"][:, None] + gx["J"][:, 0, 0][:, None] * tp[None, :, 0] + gx["J"][:, 0, 1][:, None] * tp[None, :, 1]
    yq = gx["y0"][:, None] + gx["J"][:, 1, 0][:, None] * tp[None, :, 0] + gx["J"][:, 1, 1][:, None] * tp[None, :, 1]
    C_loc = -np.einsum("qi,qj,nq->nij", vals, vals, dg)
    g_loc = g_scale * np.einsum("nq,qi,nq->ni", u0(xq, yq), vals, dg)
    C = scatter_matrix(C_loc, prob.x_restr, prob.x_restr, (prob.n_u, prob.n_u), zero_tol,
                       test_cells=cells, trial_cells=cells)
    g = scatter_vector(g_loc, prob.x_restr, prob.n_u, zero_tol, cells=cells)
    return C, g


def assemble_graph_norm(prob: MainProblem, A_y, C_signed, zero_tol=1e-15, diag_tol=1e-14):
    """Hhat = -C_signed + B_dt diag(A_y)^-1 B_dt^T + A_x
    (parabolic_graph_norm.hpp:22-65; schur_approximations.hpp:79-287 with zero_tol 0)."""
    p = prob.p
    qs, qt = 4 * p + 1, 2 * p + 1
    pts, wts = prism_rule(qs, qt)
    phi, dphi_ref = prism_basis(p, pts)
    gy = geometry_terms(prob.y_geom)
    gx = geometry_terms(prob.x_geom[prob.y_to_x])
    ny = prob.y_geom.shape[0]
    N = phi.shape[1]
    dmu = gy["absdet"][:, None] * gy["ht"][:, None] * wts[None, :]
    xq = gy["x0"][:, None] + gy["J"][:, 0, 0][:, None] * pts[None, :, 0] + gy["J"][:, 0, 1][:, None] * pts[None, :, 1]
    yq = gy["y0"][:, None] + gy["J"][:, 1, 0][:, None] * pts[None, :, 0] + gy["J"][:, 1, 1][:, None] * pts[None, :, 1]
    tq = gy["t0"][:, None] + gy["ht"][:, None] * pts[None, :, 2]
    dx = xq - gx["x0"][:, None]
    dy = yq - gx["y0"][:, None]
    xpts = np.stack([(gx["invJ"][:, 0, 0][:, None] * dx + gx["invJ"][:, 0, 1][:, None] * dy).ravel(),
                     (gx["invJ"][:, 1, 0][:, None] * dx + gx["invJ"][:, 1, 1][:, None] * dy).ravel(),
                     ((tq - gx["t0"][:, None]) / gx["ht"][:, None]).ravel()], -1)
    _, dpsi_ref = prism_basis(p, xpts)
    dt_psi = dpsi_ref[..., 2].reshape(ny, -1, N) / gx["ht"][:, None, None]
    Bdt_loc = np.einsum("nqi,qj,nq->nij", dt_psi, phi, dmu)
    B_dt = scatter_matrix(Bdt_loc, prob.x_restr, prob.y_restr, (prob.n_u, prob.n_lambda), zero_tol,
                          test_cells=prob.y_to_x)
    # A_x on the X space itself (mat_A.hpp with the X space's own cells and M)
    gxx = geometry_terms(prob.x_geom)
    nx = prob.x_geom.shape[0]
    if prob.m_cells is None:
        Mx = np.tile([1.0, 0.0, 1.0], (nx, 1))
    else:
        # piecewise-constant M per cell: take it from any Y cell inside each X cell
        Mx = np.zeros((nx, 3))
        Mx[prob.y_to_x] = prob.m_cells
    Mxt = np.stack([np.stack([Mx[:, 0], Mx[:, 1]], -1), np.stack([Mx[:, 1], Mx[:, 2]], -1)], -2)
    dmux = gxx["absdet"][:, None] * gxx["ht"][:, None] * wts[None, :]
    gpsi = np.einsum("nab,qjb->nqja", gxx["invJT"], dphi_ref[:, :, :2])
    A_x_loc = np.einsum("nqia,nab,nqjb,nq->nij", gpsi, Mxt, gpsi, dmux)
    A_x = scatter_matrix(A_x_loc, prob.x_restr, prob.x_restr, (prob.n_u, prob.n_u), zero_tol)
    return _hhat_from_blocks(A_y, C_signed, A_x, B_dt, diag_tol, prob.n_u)


def _hhat_from_blocks(A_y, C_signed, A_x, B_dt, diag_tol, n_u):
    """Hhat in the reference's own summation order (schur_approximations.hpp:107-200 and
    sparse_matrix_ops.hpp:286-316, zero_tol 0): hpar = setFromTriplets of -C (C's stored
    entries, column-major) followed by (1/A_cc * B_ic) * B_jc for every lambda column c in
    ascending order (its rows in storage order, i outer, j inner), each stored entry of hpar
    the sum of its triplets in that order; then Hhat = hpar's nonzero entries plus A_x's.
    The order matters on adaptive meshes, where Schur terms cancel exactly."""
    d = A_y.diagonal()
    if np.any(~(d > diag_tol)):
        raise RuntimeError("diagonal_schur_approximation: A_y diagonal must be positive.")
    inv = 1.0 / d
    B_dt = B_dt.tocsc()
    B_dt.sort_indices()
    Cc = C_signed.tocsc()
    Cc.sort_indices()
    # triplets in generation order
    c_cols = np.repeat(np.arange(Cc.shape[1]), np.diff(Cc.indptr))
    keep = Cc.data != 0.0
    rows = [Cc.indices[keep]]
    cols = [c_cols[keep]]
    vals = [-Cc.data[keep]]
    bl = np.diff(B_dt.indptr)
    for c in np.nonzero(bl)[0]:
        r = B_dt.indices[B_dt.indptr[c]:B_dt.indptr[c + 1]]
        v = B_dt.data[B_dt.indptr[c]:B_dt.indptr[c + 1]]
        nz = v != 0.0
        r, v = r[nz], v[nz]
        contrib = (inv[c] * v)[:, None] * v[None, :]
        rr, cc = np.broadcast_arrays(r[:, None], r[None, :])
        k = np.abs(contrib) > 0.0
        rows.append(rr[k]); cols.append(cc[k]); vals.append(contrib[k])
    rows = np.concatenate(rows); cols = np.concatenate(cols); vals = np.concatenate(vals)
    # per entry, the triplets' sum in generation order (stable sort, sequential sums)
    order = np.lexsort((cols, rows)) if len(rows) else np.zeros(0, dtype=np.int64)
    key = rows[order].astype(np.int64) * n_u + cols[order]
    starts = np.concatenate([[0], np.nonzero(np.diff(key))[0] + 1]) if len(key) else np.zeros(0, dtype=np.int64)
    sums = np.empty(len(starts))
    sv = vals[order]
    bounds = np.append(starts, len(sv))
    for g in range(len(starts)):
        acc = 0.0
        for t in range(bounds[g], bounds[g + 1]):
            acc += sv[t]
        sums[g] = acc
    hk = key[starts] if len(key) else key
    hpar_keep = sums != 0.0
    Ax = A_x.tocoo()
    ax_keep = Ax.data != 0.0
    H = sp.csc_matrix((np.concatenate([sums[hpar_keep], Ax.data[ax_keep]]),
                       (np.concatenate([hk[hpar_keep] // n_u, Ax.row[ax_keep]]),
                        np.concatenate([hk[hpar_keep] % n_u, Ax.col[ax_keep]]))), shape=(n_u, n_u))
    return dict(Hhat=H, B_dt=B_dt, A_x=A_x)


# ---------------------------------------------------------------------------------------
# 1+1D (P1 x P1 quadrilaterals, QSpace = QTime = 3 Gauss points): the generic branch of
# assemble_main_system_blocks with local_bilinear_forms.hpp:24-81,
# local_mixed_bilinear_forms.hpp:15-153, local_trace_bilinear_forms.hpp:20-49; local index
# i = i_space * 2 + i_time (quadrilateral_basis_tables.hpp:33-35).
# ---------------------------------------------------------------------------------------
def sin_initial_1d(x):
    return np.sin(math.pi * x)


def one_initial_1d(x):
    return np.ones_like(x)


def _quad_basis(xi, tau):
    """P1 x P1 values, d/dxi, d/dtau at reference points -> three [nq, 4] arrays."""
    N = np.stack([1.0 - xi, xi], -1)
    dN = np.stack([-np.ones_like(xi), np.ones_like(xi)], -1)
    T = np.stack([1.0 - tau, tau], -1)
    dT = np.stack([-np.ones_like(tau), np.ones_like(tau)], -1)
    v = (N[:, :, None] * T[:, None, :]).reshape(len(xi), 4)
    vx = (dN[:, :, None] * T[:, None, :]).reshape(len(xi), 4)
    vt = (N[:, :, None] * dT[:, None, :]).reshape(len(xi), 4)
    return v, vx, vt


def _quad_rule():
    gx, gw = gauss_legendre01(3)
    xi, tau = np.meshgrid(gx, gx, indexing="ij")
    w = np.outer(gw, gw)
    return xi.ravel(), tau.ravel(), w.ravel()


def assemble_main_blocks_1d(prob: MainProblem, u0=sin_initial_1d, ell=None, zero_tol=1e-15, g_scale=-1.0):
    """Restatement of assemble_main_system_blocks for 1+1D P1 (assemble_saddle_problem.hpp:131)."""
    xi, tau, w = _quad_rule()
    gy, gx = prob.y_geom, prob.x_geom[prob.y_to_x]
    ny = gy.shape[0]
    m = prob.m_cells if prob.m_cells is not None else np.ones(ny)
    hy, ky = gy[:, 1] - gy[:, 0], gy[:, 3] - gy[:, 2]
    v, vx, vt = _quad_basis(xi, tau)
    dmu = (hy * ky)[:, None] * w[None, :]
    phi_x = vx[None, :, :] / hy[:, None, None]
    A = np.einsum("n,nqi,nqj,nq->nij", m, phi_x, phi_x, dmu)
    # X basis at the Y points through the X cell's reference coordinates
    xq = gy[:, 0:1] + hy[:, None] * xi[None, :]
    tq = gy[:, 2:3] + ky[:, None] * tau[None, :]
    hx, kx = gx[:, 1] - gx[:, 0], gx[:, 3] - gx[:, 2]
    pv, pvx, pvt = _quad_basis(((xq - gx[:, 0:1]) / hx[:, None]).ravel(), ((tq - gx[:, 2:3]) / kx[:, None]).ravel())
    psi_x = pvx.reshape(ny, -1, 4) / hx[:, None, None]
    psi_t = pvt.reshape(ny, -1, 4) / kx[:, None, None]
    B = np.einsum("nqi,qj,nq->nij", psi_t, v, dmu) + np.einsum("n,nqi,nqj,nq->nij", m, psi_x, phi_x, dmu)
    f_loc = np.zeros((ny, 4)) if ell is None else np.einsum("nq,qj,nq->nj", ell(xq, tq), v, dmu)
    A_y = scatter_matrix(A, prob.y_restr, prob.y_restr, (prob.n_lambda, prob.n_lambda), zero_tol)
    Bm = scatter_matrix(B, prob.x_restr, prob.y_restr, (prob.n_u, prob.n_lambda), zero_tol, test_cells=prob.y_to_x)
    f = scatter_vector(f_loc, prob.y_restr, prob.n_lambda, zero_tol)
    # trace blocks on the X cells at t = 0 (3-point Gauss bottom rule)
    cells = np.nonzero(prob.x_geom[:, 2] == 0.0)[0]
    bx, bw = gauss_legendre01(3)
    bv, _, _ = _quad_basis(bx, np.zeros_like(bx))
    gc = prob.x_geom[cells]
    hc = gc[:, 1] - gc[:, 0]
    dg = hc[:, None] * bw[None, :]
    C_loc = -np.einsum("qi,qj,nq->nij", bv, bv, dg)
    g_loc = g_scale * np.einsum("nq,qi,nq->ni", u0(gc[:, 0:1] + hc[:, None] * bx[None, :]), bv, dg)
    C = scatter_matrix(C_loc, prob.x_restr, prob.x_restr, (prob.n_u, prob.n_u), zero_tol,
                       test_cells=cells, trial_cells=cells)
    g = scatter_vector(g_loc, prob.x_restr, prob.n_u, zero_tol, cells=cells)
    Bdt_loc = np.einsum("nqi,qj,nq->nij", psi_t, v, dmu)
    return dict(A_y=A_y, B=Bm, C_signed=C, f=f, g=g, _Bdt_loc=Bdt_loc)


def assemble_graph_norm_1d(prob: MainProblem, A_y, C_signed, zero_tol=1e-15, diag_tol=1e-14):
    """Hhat = -C_signed + B_dt diag(A_y)^-1 B_dt^T + A_x for 1+1D P1 (parabolic_graph_norm.hpp:22-65)."""
    blocks = assemble_main_blocks_1d(prob, zero_tol=zero_tol)
    B_dt = scatter_matrix(blocks["_Bdt_loc"], prob.x_restr, prob.y_restr, (prob.n_u, prob.n_lambda), zero_tol,
                          test_cells=prob.y_to_x)
    xi, tau, w = _quad_rule()
    gxx = prob.x_geom
    nx = gxx.shape[0]
    mx = np.ones(nx)
    if prob.m_cells is not None:
        mx[prob.y_to_x] = prob.m_cells
    h, k = gxx[:, 1] - gxx[:, 0], gxx[:, 3] - gxx[:, 2]
    _, vx, _ = _quad_basis(xi, tau)
    px = vx[None, :, :] / h[:, None, None]
    A_x_loc = np.einsum("n,nqi,nqj,nq->nij", mx, px, px, (h * k)[:, None] * w[None, :])
    A_x = scatter_matrix(A_x_loc, prob.x_restr, prob.x_restr, (prob.n_u, prob.n_u), zero_tol)
    return _hhat_from_blocks(A_y, C_signed, A_x, B_dt, diag_tol, prob.n_u)


def load_csc(d, name):
    shape = tuple(np.load(f"{d}/{name}_shape.npy"))
    return sp.csc_matrix((np.load(f"{d}/{name}_values.npy"), np.load(f"{d}/{name}_inner.npy"),
                          np.load(f"{d}/{name}_outer.npy")), shape=shape)


def load_problem(d, p) -> MainProblem:
    def restr(prefix):
        return Restriction(np.load(f"{d}/{prefix}_offsets.npy"), np.load(f"{d}/{prefix}_dofs.npy"),
                           np.load(f"{d}/{prefix}_weights.npy"), (p + 1) * (p + 2) // 2 * (p + 1))
    n_lambda = int(np.load(f"{d}/A_y_shape.npy")[0])
    n_u = int(np.load(f"{d}/C_signed_shape.npy")[0])
    return MainProblem(p=p, y_geom=np.load(f"{d}/y_geometry.npy"), x_geom=np.load(f"{d}/x_geometry.npy"),
                       y_to_x=np.load(f"{d}/y_to_x_cell.npy"), y_restr=restr("y_restriction"),
                       x_restr=restr("x_restriction"), n_lambda=n_lambda, n_u=n_u)


# ----------------------------------------------------------------------------
# time-slab space and the slab reconstruction (adaptive meshes)
# ----------------------------------------------------------------------------
_NODE_VERTICES = {1: [(0, 0), (1, 1), (2, 2)],
                  2: [(0, 0), (0, 1), (1, 1), (0, 2), (1, 2), (2, 2)]}


def slab_space(p: int, y_geom, y_vertex_ids, y_restr: Restriction):
    """The reference's time-slab space of a Y space (time_slab_builder.hpp:53-215).

    Slab times: the sorted distinct time endpoints of the Y cells; slab cells: every Y cell
    once per slab it spans, slabs in time order and each slab's cells in Y order.  The slab
    space is P_p x P_p per slab, continuous in space inside a slab and broken between slabs;
    spatial nodes whose Y restriction rows are all empty are Dirichlet nodes.  Returns
    (source Y cell, slab id, slab geometry, Restriction, number of slab DOFs); the DOF
    numbering is this function's own (first appearance per slab)."""
    ns, nt = len(_NODE_VERTICES[p]), p + 1
    nd = ns * nt
    ny = y_geom.shape[0]
    times = np.unique(y_geom[:, 6:8].ravel())
    kb = np.searchsorted(times, y_geom[:, 6])
    ke = np.searchsorted(times, y_geom[:, 7])
    src, slab = [], []
    for k in range(len(times) - 1):
        cells = np.nonzero((kb <= k) & (k < ke))[0]
        src.extend(cells.tolist())
        slab.extend([k] * len(cells))
    src = np.asarray(src, dtype=np.int64)
    slab = np.asarray(slab, dtype=np.int64)
    off = y_restr.offsets
    empty = (off[1:] == off[:-1]).reshape(ny, ns, nt).all(axis=2)
    dof = -np.ones((len(src), nd), dtype=np.int64)
    base = 0
    for k in range(len(times) - 1):
        ids = {}
        for i in np.nonzero(slab == k)[0]:
            for s_, (va, vb) in enumerate(_NODE_VERTICES[p]):
                if empty[src[i], s_]:
                    continue
                a, b = int(y_vertex_ids[src[i], va]), int(y_vertex_ids[src[i], vb])
                key = (min(a, b), max(a, b))
                j = ids.setdefault(key, len(ids))
                dof[i, s_ * nt:(s_ + 1) * nt] = base + j * nt + np.arange(nt)
        base += len(ids) * nt
    flat = dof.ravel()
    counts = (flat >= 0).astype(np.int64)
    offsets = np.concatenate([[0], np.cumsum(counts)])
    restr = Restriction(offsets, flat[flat >= 0], np.ones(int(counts.sum())), nd)
    geom = y_geom[src].copy()
    geom[:, 6] = times[slab]
    geom[:, 7] = times[slab + 1]
    return src, slab, geom, restr, base


def slab_reconstruction(prob: MainProblem, y_vertex_ids, u, ell=None, zero_tol=1e-15):
    """lambda~ on the slab space (time_slab_reconstruction_operator.hpp:686-830): the slab
    forms are the main-system ones with the slab space as test space, so
    A_slab lambda~ = f_slab - B_slab^T u, solved directly.  Returns (source, slab, slab
    geometry, slab restriction, lambda~ as slab DOFs)."""
    import scipy.sparse.linalg as spl
    src, slab, geom, restr, n = slab_space(prob.p, prob.y_geom, y_vertex_ids, prob.y_restr)
    sprob = MainProblem(p=prob.p, y_geom=geom, x_geom=prob.x_geom, y_to_x=np.asarray(prob.y_to_x)[src],
                        y_restr=restr, x_restr=prob.x_restr, n_lambda=n, n_u=prob.n_u,
                        m_cells=None if prob.m_cells is None else np.asarray(prob.m_cells)[src])
    blocks = assemble_main_blocks(sprob, ell=ell, zero_tol=zero_tol)
    lt = spl.spsolve(blocks["A_y"].tocsc(), blocks["f"] - blocks["B"].T @ u)
    return src, slab, geom, restr, lt


def nodal_values(restr: Restriction, v):
    """[n_cells, ndof] local values of a true-DOF vector through a restriction."""
    n = (len(restr.offsets) - 1) // restr.ndof
    rows = np.repeat(np.arange(len(restr.offsets) - 1), np.diff(restr.offsets))
    out = np.zeros(len(restr.offsets) - 1)
    np.add.at(out, rows, restr.weights * v[restr.dofs])
    return out.reshape(n, restr.ndof)


# ----------------------------------------------------------------------------
# the driver's G^delta estimator (algorithm/adaptive_driver.hpp:2690-2900)
# ----------------------------------------------------------------------------
def prism_nodes(q: int):
    """Reference nodes of the degree-q prism in local order i_s*(q+1)+i_t."""
    tn = triangle_nodes(q)
    tt = np.arange(q + 1) / q
    return np.array([(a, b, t) for (a, b) in tn for t in tt])


def interpolate_nodal(p: int, src_nodal, src_geom, src_index, dst_geom, q: int):
    """[n_dst, nodes of degree q]: the degree-p prism function of each source cell (nodal
    values src_nodal[src_index[c]]) at the degree-q nodes of the destination cell c, which
    lies inside it (exact for nested cells: prolong_true_coefficients_nodal evaluates the
    same way)."""
    ref = prism_nodes(q)
    n = dst_geom.shape[0]
    si = np.arange(n) if src_index is None else np.asarray(src_index)
    out = np.empty((n, ref.shape[0]))
    for c in range(n):
        d, s = dst_geom[c], src_geom[si[c]]
        px = d[0] + (d[2] - d[0]) * ref[:, 0] + (d[4] - d[0]) * ref[:, 1]
        py = d[1] + (d[3] - d[1]) * ref[:, 0] + (d[5] - d[1]) * ref[:, 1]
        pt = d[6] + (d[7] - d[6]) * ref[:, 2]
        J = np.array([[s[2] - s[0], s[4] - s[0]], [s[3] - s[1], s[5] - s[1]]])
        rs = np.linalg.solve(J, np.stack([px - s[0], py - s[1]]))
        pts = np.stack([rs[0], rs[1], (pt - s[6]) / (s[7] - s[6])], axis=1)
        vals, _ = prism_basis(p, pts)
        out[c] = vals @ src_nodal[si[c]]
    return out


def true_from_nodal(restr: Restriction, local, n: int):
    """True-DOF vector from per-cell nodal values: each true DOF takes the value at its first
    unconstrained occurrence (a local row with the single entry (dof, 1))."""
    out = np.full(n, np.nan)
    off = restr.offsets
    flat = local.ravel()
    for row in range(len(off) - 1):
        a, b = off[row], off[row + 1]
        if b - a == 1 and restr.weights[a] == 1.0 and np.isnan(out[restr.dofs[a]]):
            out[restr.dofs[a]] = flat[row]
    return out


def g_delta(prob: MainProblem, g_restr: Restriction, n_g: int, lam, u, ell=None, zero_tol=1e-15):
    """||lambda_G - lambda_delta||^2_{A_G} on the Y cells with the degree-(p+1) space G
    (restriction g_restr): A_G lambda_G = f_G - B(X,G)^T u_delta.  B(X,G)^T u_delta is the
    mixed form with u_delta interpolated into G (exact: X restricted to a Y cell is a
    degree-p polynomial, G broken in time), so every block is a same-degree G form."""
    import scipy.sparse.linalg as spl
    ny = prob.y_geom.shape[0]
    q = prob.p + 1
    gprob = MainProblem(p=q, y_geom=prob.y_geom, x_geom=prob.y_geom, y_to_x=np.arange(ny), y_restr=g_restr,
                        x_restr=g_restr, n_lambda=n_g, n_u=n_g, m_cells=prob.m_cells)
    blocks = assemble_main_blocks(gprob, ell=ell, zero_tol=zero_tol)
    u_g = true_from_nodal(g_restr, interpolate_nodal(prob.p, nodal_values(prob.x_restr, u), prob.x_geom,
                                                     prob.y_to_x, prob.y_geom, q), n_g)
    l_g = true_from_nodal(g_restr, interpolate_nodal(prob.p, nodal_values(prob.y_restr, lam), prob.y_geom, None,
                                                     prob.y_geom, q), n_g)
    A = blocks["A_y"].tocsc()
    rhs = blocks["f"] - blocks["B"].T @ u_g
    lam_g = spl.spsolve(A, rhs)
    d = lam_g - l_g
    return float(d @ (A @ d)), {"A_g": A, "f_g": blocks["f"], "rhs_g": rhs, "lambda_g": lam_g,
                                "lambda_delta_in_g": l_g, "u_in_g": u_g}
