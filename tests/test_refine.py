"""The host generator of locally refined meshes (doubleadapparabolicfem_b200.refine), used by
the learned-preconditioner benchmark: its triangulations are conforming in space on every
time interval, its X space (with hanging nodes at the time levels where the interval meshes
differ) is continuous in time, and the GPU path assembles, solves and estimates on it the
same blocks as the oracle restatement.
"""
import numpy as np
import pytest

from conftest import HHAT_RESIDUE, assert_same_sparse


@pytest.fixture(scope="module")
def small():
    from doubleadapparabolicfem_b200.refine import locally_refined_problem
    return locally_refined_problem(level=3, seed=4, depth=4, radius0=0.3, time_rounds=2, return_hierarchy=True)


def test_interval_meshes_are_conforming(small):
    prob, (xy, meshes, T, dk, e) = small
    for M in meshes:
        edges = np.sort(np.concatenate([M[:, [0, 1]], M[:, [1, 2]], M[:, [2, 0]]]), axis=1)
        keys, counts = np.unique(edges, axis=0, return_counts=True)
        assert counts.max() == 2
        b = keys[counts == 1]
        # every edge with one triangle lies on the boundary of the unit square
        pa, pb = xy[b[:, 0]], xy[b[:, 1]]
        on_side = ((np.abs(pa[:, 0] - pb[:, 0]) < 1e-14) & np.isin(np.round(pa[:, 0], 14), [0.0, 1.0])) | \
                  ((np.abs(pa[:, 1] - pb[:, 1]) < 1e-14) & np.isin(np.round(pa[:, 1], 14), [0.0, 1.0]))
        assert on_side.all()
        # the triangles tile the square
        P = xy[M]
        area = 0.5 * np.abs((P[:, 1, 0] - P[:, 0, 0]) * (P[:, 2, 1] - P[:, 0, 1]) -
                            (P[:, 2, 0] - P[:, 0, 0]) * (P[:, 1, 1] - P[:, 0, 1]))
        assert abs(area.sum() - 1.0) < 1e-12
    # nested: every vertex of a coarser mesh is a vertex of the finer ones
    for a, b in zip(meshes[:-1], meshes[1:]):
        assert np.isin(np.unique(a), np.unique(b)).all()
    assert len(meshes[-1]) > len(meshes[0])


def test_x_space_is_continuous_in_time_and_has_hanging_nodes(small):
    """A random X DOF vector, evaluated from the cells below and above every time level at
    every vertex of both sides, agrees; restriction rows with several weighted entries exist."""
    prob, (xy, meshes, T, dk, e) = small
    import apf_oracle as O
    cnt = np.diff(prob.x_restriction.offsets)
    assert (cnt > 1).sum() > 50
    rng = np.random.default_rng(0)
    v = rng.standard_normal(prob.n_u)
    R = O.Restriction(prob.x_restriction.offsets, prob.x_restriction.dofs, prob.x_restriction.weights, 6)
    nodal = O.nodal_values(R, v)                                  # [cells, 6], index s * 2 + a
    geo = prob.x_geometry
    for lvl in range(1, len(T) - 1):
        below = np.nonzero(geo[:, 7] == T[lvl])[0]
        above = np.nonzero(geo[:, 6] == T[lvl])[0]

        def field(cells, a):
            # value of the P1 trace at points: locate each point in a triangle of `cells`
            P = geo[cells, :6].reshape(-1, 3, 2)
            vals = nodal[cells][:, [0 + a, 2 + a, 4 + a]]

            def at(pts):
                out = np.empty(len(pts))
                for q, p in enumerate(pts):
                    d = (P[:, 1, 0] - P[:, 0, 0]) * (P[:, 2, 1] - P[:, 0, 1]) - \
                        (P[:, 2, 0] - P[:, 0, 0]) * (P[:, 1, 1] - P[:, 0, 1])
                    l1 = ((p[0] - P[:, 0, 0]) * (P[:, 2, 1] - P[:, 0, 1]) - (P[:, 2, 0] - P[:, 0, 0]) * (p[1] - P[:, 0, 1])) / d
                    l2 = ((P[:, 1, 0] - P[:, 0, 0]) * (p[1] - P[:, 0, 1]) - (p[0] - P[:, 0, 0]) * (P[:, 1, 1] - P[:, 0, 1])) / d
                    w = np.stack([1 - l1 - l2, l1, l2], 1)
                    t = np.nonzero(w.min(1) >= -1e-12)[0][0]
                    out[q] = w[t] @ vals[t]
                return out
            return at

        pts = np.unique(np.concatenate([geo[below, :6], geo[above, :6]]).reshape(-1, 2), axis=0)
        top = field(below, 1)(pts)
        bottom = field(above, 0)(pts)
        assert np.abs(top - bottom).max() <= 1e-12 * max(1.0, np.abs(v).max()), lvl


def test_dof_counts_and_kappa(small):
    prob, _ = small
    for r, n in ((prob.x_restriction, prob.n_u), (prob.y_restriction, prob.n_lambda)):
        used = np.zeros(n, dtype=bool)
        used[r.dofs] = True
        assert used.all()
    k = prob.m_cells[:, 0]
    assert k.min() >= 0.01 and k.max() <= 100.0 and k.max() / k.min() > 100.0
    assert (prob.m_cells[:, 1] == 0).all() and (prob.m_cells[:, 2] == k).all()


@pytest.mark.gpu
def test_refined_problem_blocks_solve_and_estimate(gpu_ctx, small):
    """GPU blocks on the generated mesh equal the oracle restatement's (patterns bit-exact,
    values 1e-12); MINRES with the plain and the learned preconditioner reaches the FP64
    true residual 1e-10 (checked on the host); the estimator runs (every Y cell in one time
    slab: lambda~ = lambda_delta)."""
    import scipy.sparse as sp
    import apf_oracle as O
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.estimator import estimate
    from doubleadapparabolicfem_b200 import learned as LM
    from doubleadapparabolicfem_b200.solver import SolverOptions, solve_saddle_system_with_preconditioner
    prob, _ = small
    op = O.MainProblem(p=1, y_geom=prob.y_geometry, x_geom=prob.x_geometry, y_to_x=prob.y_to_x,
                       y_restr=O.Restriction(prob.y_restriction.offsets, prob.y_restriction.dofs,
                                             prob.y_restriction.weights, 6),
                       x_restr=O.Restriction(prob.x_restriction.offsets, prob.x_restriction.dofs,
                                             prob.x_restriction.weights, 6),
                       n_lambda=prob.n_lambda, n_u=prob.n_u, m_cells=prob.m_cells)
    want = O.assemble_main_blocks(op)
    gn = O.assemble_graph_norm(op, want["A_y"], want["C_signed"])
    blocks = assemble_main_system_blocks(prob, ctx=gpu_ctx)
    for nm, mine in (("A_y", blocks.A_y()), ("B", blocks.lower_left_B()), ("C_signed", blocks.C_signed())):
        assert_same_sparse(want[nm], mine, 1e-12, nm)
    assert_same_sparse(gn["Hhat"], blocks.assemble_parabolic_graph_norm_approximation(), 1e-12, "Hhat",
                       residue=HHAT_RESIDUE)
    K = sp.bmat([[want["A_y"], want["B"].T], [want["B"], want["C_signed"]]]).tocsr()
    b = np.concatenate([want["f"], want["g"]])
    for precond in ("amg_block", "learned"):
        if precond == "learned":
            LM.use_model(gpu_ctx, LM.LearnedModel.load())
        x, diag = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=1e-10, preconditioner=precond))
        assert np.linalg.norm(K @ x - b) / np.linalg.norm(b) <= 1e-10, precond
    cells, totals = estimate(blocks)
    assert np.isfinite(cells["eta"]).all() and totals["flux_squared"] > 0.0
    assert totals["reconstruction_squared"] <= 1e-12 * totals["flux_squared"]
