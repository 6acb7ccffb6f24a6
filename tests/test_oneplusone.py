"""1+1D path (P1 x P1 quadrilaterals, the reference's CPU-runnable configuration):
assembly, graph-norm block, MINRES, edge-patch estimator and X-marking indicators.

CPU tests pin the oracle's 1+1D restatement (oracle/apf_oracle.py) and the host mesh
generator against the reference's own outputs (fixtures written by the reference
templates through oracle/_ref, tests/golden/make_golden.py) and the published uniform
rows of the paper data.  GPU tests (marked gpu) compare the library, called through
its C ABI, with the same fixtures: patterns bit-exact, values within 1e-12 of the
block's largest entry; MINRES to a relative residual of 1e-10 (the configuration's
tolerance) and 1e-13 for the estimator comparisons, whose per-cell values then agree
to 1e-9 of the largest cell (1e-10 on the totals).
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES_1D, HHAT_RESIDUE, assert_same_sparse, load_golden, to_product_problem

# adaptive 1+1D meshes from the reference: X refined locally (hanging nodes in space and
# time), Y refined beyond X by one pass of the reference's inner loop
ADAPTIVE_CASES_1D = ["d1_adapt_smooth", "d1_adapt_nonmatching"]

import apf_oracle as O


def _fixture(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def _paper_rows_1d(example="smooth_initial"):
    with open(os.path.join(GOLDEN, "paper_uniform_rows.json")) as fh:
        return [r for r in json.load(fh) if r["dimension"] == "1d" and r["p"] == "p1" and r["example"] == example]


def _oracle_u0_ell(example, n_cells):
    if example == "smooth_initial":
        return O.sin_initial_1d, None
    return O.one_initial_1d, (lambda x, t: np.full_like(x, 2.0))


# ---------------------------------------------------------------------------------------
# CPU: oracle and mesh generator
# ---------------------------------------------------------------------------------------
@pytest.mark.parametrize("name", GOLDEN_CASES_1D + ADAPTIVE_CASES_1D)
def test_oracle_1d_blocks_match_reference(name):
    prob, ref, example = load_golden(name)
    u0, ell = _oracle_u0_ell(example, prob.y_geom.shape[0])
    out = O.assemble_main_blocks_1d(prob, u0=u0, ell=ell)
    for nm in ("A_y", "B", "C_signed"):
        assert_same_sparse(ref[nm], out[nm], 1e-12, nm)
    assert np.abs(out["f"] - ref["f"]).max() <= 1e-12 * max(1.0, np.abs(ref["f"]).max())
    assert np.abs(out["g"] - ref["g"]).max() <= 1e-12 * np.abs(ref["g"]).max()
    gn = O.assemble_graph_norm_1d(prob, ref["A_y"], ref["C_signed"])
    residue = HHAT_RESIDUE if name in ADAPTIVE_CASES_1D else 0.0
    assert_same_sparse(ref["Hhat"], gn["Hhat"], 1e-12, "Hhat", residue=residue)


def test_adaptive_1d_fixtures_have_hanging_nodes():
    for name in ADAPTIVE_CASES_1D:
        prob, ref, _ = load_golden(name)
        assert (np.diff(prob.x_restr.offsets) > 1).sum() > 10, name
        assert (np.diff(prob.y_restr.offsets) > 1).sum() > 10, name
        assert prob.y_geom.shape[0] > prob.x_geom.shape[0], name
        assert np.load(os.path.join(GOLDEN, f"{name}.npz"))["est_recon"].sum() > 0.0


def test_uniform_1d_dof_counts_match_paper_data():
    from doubleadapparabolicfem_b200.mesh import uniform_problem_1d
    checked = 0
    for r in _paper_rows_1d():
        level = int(r["outer_iteration"])
        if level > 7:
            continue
        prob = uniform_problem_1d(level)
        assert prob.n_u == int(r["x_true_dofs_before"]), r
        assert prob.n_lambda == int(r["y_true_dofs_after"]), r
        checked += 1
    assert checked >= 6


def test_reference_1d_fixtures_match_paper():
    """The reference's own 1+1D inner iteration (fixtures) reproduces the published
    y_flux_squared, lambda_y_squared and eta_squared of the uniform runs (6 digits)."""
    for name, example in (("d1_l2_smooth", "smooth_initial"), ("d1_l5_smooth", "smooth_initial"),
                          ("d1_l2_nonmatching", "non_matching_initial")):
        z = _fixture(name)
        level = int(z["meta_level"][0])
        row = [r for r in _paper_rows_1d(example) if int(r["outer_iteration"]) == level][0]
        for key, val in (("y_flux_squared", z["est_flux"].sum()), ("lambda_y_squared", z["xind_lambda_by_x"].sum()),
                         ("eta_squared", np.nansum(z["xind_eta_by_x"]))):
            want = float(row[key])
            assert abs(val - want) <= 1e-5 * want, (name, key, val, want)


def _dof_keys(geom, restr, space):
    """DOF -> (x, t, side) key from cell geometry x0 x1 t0 t1: X DOFs by their space-time
    node, Y DOFs (broken in time) by node and the time interval they belong to."""
    keys = {}
    for c in range(geom.shape[0]):
        x0, x1, t0, t1 = geom[c]
        for loc in range(4):
            s, a = loc >> 1, loc & 1
            b, e = restr.offsets[c * 4 + loc], restr.offsets[c * 4 + loc + 1]
            for k in range(b, e):
                x = x1 if s else x0
                if space == "x":
                    key = (round(x * 2 ** 20), round((t1 if a else t0) * 2 ** 20))
                else:
                    key = (round(x * 2 ** 20), round(t0 * 2 ** 20), a)
                keys[int(restr.dofs[k])] = key
    return keys


def _permutation(ref_prob, mine, space):
    rk = _dof_keys(ref_prob.y_geom if space == "y" else ref_prob.x_geom,
                   ref_prob.y_restr if space == "y" else ref_prob.x_restr, space)
    mk = _dof_keys(mine.y_geometry if space == "y" else mine.x_geometry,
                   mine.y_restriction if space == "y" else mine.x_restriction, space)
    inv = {v: k for k, v in mk.items()}
    return np.array([inv[rk[i]] for i in range(len(rk))])


def _oracle_problem(mine):
    return O.MainProblem(p=1, y_geom=mine.y_geometry, x_geom=mine.x_geometry, y_to_x=mine.y_to_x,
                         y_restr=O.Restriction(mine.y_restriction.offsets, mine.y_restriction.dofs,
                                               mine.y_restriction.weights, 4),
                         x_restr=O.Restriction(mine.x_restriction.offsets, mine.x_restriction.dofs,
                                               mine.x_restriction.weights, 4),
                         n_lambda=mine.n_lambda, n_u=mine.n_u, dim_space=1)


def test_generated_1d_mesh_assembles_to_reference_blocks():
    """The host generator's mesh and numbering, assembled by the oracle, equal the
    reference's blocks after the DOF permutation (pattern bit-exact, values 1e-12)."""
    import scipy.sparse as sp
    from doubleadapparabolicfem_b200.mesh import uniform_problem_1d
    prob, ref, _ = load_golden("d1_l2_smooth")
    mine = uniform_problem_1d(2)
    py, px = _permutation(prob, mine, "y"), _permutation(prob, mine, "x")
    out = O.assemble_main_blocks_1d(_oracle_problem(mine))
    Py = sp.csr_matrix((np.ones(len(py)), (np.arange(len(py)), py)), shape=(len(py), len(py)))
    Px = sp.csr_matrix((np.ones(len(px)), (np.arange(len(px)), px)), shape=(len(px), len(px)))
    assert_same_sparse(ref["A_y"], Py @ out["A_y"] @ Py.T, 1e-12, "A_y")
    assert_same_sparse(ref["B"], Px @ out["B"] @ Py.T, 1e-12, "B")
    assert_same_sparse(ref["C_signed"], Px @ out["C_signed"] @ Px.T, 1e-12, "C")
    assert np.abs(Px @ out["g"] - ref["g"]).max() <= 1e-12 * np.abs(ref["g"]).max()


# ---------------------------------------------------------------------------------------
# GPU: the library through its C ABI
# ---------------------------------------------------------------------------------------
def _assemble(ctx, prob):
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    blocks = assemble_main_system_blocks(prob, ctx=ctx)
    blocks.assemble_parabolic_graph_norm_approximation()
    return blocks


@pytest.mark.gpu
@pytest.mark.parametrize("name", GOLDEN_CASES_1D)
def test_1d_assembly_matches_reference(gpu_ctx, name):
    import scipy.sparse as sp
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    prob, ref, example = load_golden(name)
    blocks = assemble_main_system_blocks(to_product_problem(prob, example), ctx=gpu_ctx)
    assert_same_sparse(ref["A_y"], blocks.A_y(), 1e-12, "A_y")
    assert_same_sparse(ref["B"], blocks.lower_left_B(), 1e-12, "B")
    assert_same_sparse(ref["B"], blocks.block("BT").T, 1e-12, "B^T")
    assert_same_sparse(ref["C_signed"], blocks.C_signed(), 1e-12, "C_signed")
    f, g = blocks.f(), blocks.g()
    assert np.abs(f - ref["f"]).max() <= 1e-12 * max(1.0, np.abs(ref["f"]).max())
    assert np.abs(g - ref["g"]).max() <= 1e-12 * np.abs(ref["g"]).max()
    K_ref = sp.bmat([[ref["A_y"], ref["B"].T], [ref["B"], ref["C_signed"]]]).tocsr()
    assert_same_sparse(K_ref, blocks.K(), 1e-12, "K")
    assert_same_sparse(ref["Hhat"], blocks.assemble_parabolic_graph_norm_approximation(1e-14), 1e-12, "Hhat")


@pytest.mark.gpu
@pytest.mark.parametrize("name", GOLDEN_CASES_1D)
def test_1d_cycle_matches_reference(gpu_ctx, name):
    """Solve (MINRES, 1e-13), edge-patch estimator and X-marking indicators against the
    reference's direct solve and its own per-cell indicators."""
    from doubleadapparabolicfem_b200.estimator import estimate, x_marking_indicator_components
    from doubleadapparabolicfem_b200.solver import SolverOptions, solve_saddle_system_with_preconditioner
    prob, ref, example = load_golden(name)
    z = _fixture(name)
    blocks = _assemble(gpu_ctx, to_product_problem(prob, example))
    x, diag = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=1e-13))
    nl = prob.n_lambda
    for mine, theirs in ((x[:nl], z["lambda_delta"]), (x[nl:], z["u_delta"])):
        assert np.abs(mine - theirs).max() <= 1e-9 * np.abs(theirs).max()
    cells, totals = estimate(blocks)
    scale = np.abs(z["est_flux"]).max()
    assert np.abs(cells["flux"] - z["est_flux"]).max() <= 1e-9 * scale
    assert np.abs(cells["divergence"] - z["est_div"]).max() <= 1e-9 * scale
    assert np.abs(cells["eta"] - z["est_eta"]).max() <= 1e-9 * scale
    assert abs(totals["flux_squared"] - z["est_flux"].sum()) <= 1e-10 * z["est_flux"].sum()
    assert totals["reconstruction_squared"] <= 1e-12 * z["est_flux"].sum()
    assert totals["n_patches"] == totals["n_slabs"] * (int(np.sqrt(prob.y_geom.shape[0])) + 1)
    xc, xt = x_marking_indicator_components(blocks)
    pairs = [("lambda_y_squared_by_y_cell", "xind_lambda_by_y"), ("lambda_y_squared_by_x_cell", "xind_lambda_by_x"),
             ("initial_trace_squared_by_x_cell", "xind_trace_by_x"), ("eta_squared_by_x_cell", "xind_eta_by_x")]
    for mine, theirs in pairs:
        r = np.nan_to_num(z[theirs], nan=0.0)
        assert np.abs(xc[mine] - r).max() <= 1e-9 * max(np.abs(r).max(), 1e-300), mine
    assert abs(xt["eta_squared"] - np.nansum(z["xind_eta_by_x"])) <= 1e-10 * np.nansum(z["xind_eta_by_x"])


@pytest.mark.gpu
def test_1d_configuration_cycle_and_paper_values(gpu_ctx):
    """The CPU-runnable configuration: 64 x 64 = 4,096 elements (outer level 5) on the host
    generator's mesh, MINRES to the FP64 true relative residual 1e-10, then the estimator;
    y_flux_squared, lambda_y_squared and eta_squared of outer levels 0-6 against the
    published uniform rows (6 digits)."""
    from doubleadapparabolicfem_b200.estimator import estimate, x_marking_indicator_components
    from doubleadapparabolicfem_b200.mesh import uniform_problem_1d
    from doubleadapparabolicfem_b200.solver import SolverOptions, solve_saddle_system_with_preconditioner
    rows = {int(r["outer_iteration"]): r for r in _paper_rows_1d()}
    for level in range(0, 7):
        blocks = _assemble(gpu_ctx, uniform_problem_1d(level))
        _, diag = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=1e-10), copy_out=False)
        assert diag["final_true_residual"] <= 1e-10, (level, diag["final_true_residual"])
        _, totals = estimate(blocks)
        _, xt = x_marking_indicator_components(blocks)
        for key, val in (("y_flux_squared", totals["flux_squared"]), ("lambda_y_squared", xt["lambda_y_squared"]),
                         ("eta_squared", xt["eta_squared"])):
            want = float(rows[level][key])
            assert abs(val - want) <= 1e-5 * want, (level, key, val, want)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ADAPTIVE_CASES_1D)
def test_1d_adaptive_cycle_matches_reference(gpu_ctx, name):
    """Adaptive 1+1D meshes: blocks (patterns bit-exact, 1e-12; Hhat's significant pattern),
    MINRES (1e-13), then the slab reconstruction on the time-slab space (Y cells cut at every
    time endpoint), the edge-patch estimator and the X-marking indicators against the
    reference's own per-cell values: 1e-9 of the largest cell eta, totals 1e-10 (recon 1e-8)."""
    from doubleadapparabolicfem_b200.estimator import estimate, x_marking_indicator_components
    from doubleadapparabolicfem_b200.solver import SolverOptions, solve_saddle_system_with_preconditioner
    prob, ref, example = load_golden(name)
    z = _fixture(name)
    blocks = _assemble(gpu_ctx, to_product_problem(prob, example))
    assert_same_sparse(ref["A_y"], blocks.A_y(), 1e-12, "A_y")
    assert_same_sparse(ref["B"], blocks.lower_left_B(), 1e-12, "B")
    assert_same_sparse(ref["C_signed"], blocks.C_signed(), 1e-12, "C_signed")
    assert_same_sparse(ref["Hhat"], blocks.assemble_parabolic_graph_norm_approximation(1e-14), 1e-12, "Hhat",
                       residue=HHAT_RESIDUE)
    x, diag = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=1e-13))
    nl = prob.n_lambda
    for mine, theirs in ((x[:nl], z["lambda_delta"]), (x[nl:], z["u_delta"])):
        assert np.abs(mine - theirs).max() <= 1e-9 * np.abs(theirs).max()
    cells, totals = estimate(blocks)
    scale = np.abs(z["est_eta"]).max()
    for key, ref_key in (("flux", "est_flux"), ("divergence", "est_div"), ("reconstruction", "est_recon"),
                         ("eta", "est_eta")):
        assert np.abs(cells[key] - z[ref_key]).max() <= 1e-9 * scale, key
    assert abs(totals["flux_squared"] - z["est_flux"].sum()) <= 1e-10 * z["est_flux"].sum()
    assert abs(totals["reconstruction_squared"] - z["est_recon"].sum()) <= 1e-8 * z["est_recon"].sum()
    xc, xt = x_marking_indicator_components(blocks)
    xs = np.nanmax(np.abs(z["xind_eta_by_x"]))
    for mine, theirs in (("lambda_y_squared_by_y_cell", "xind_lambda_by_y"),
                         ("lambda_y_squared_by_x_cell", "xind_lambda_by_x"),
                         ("initial_trace_squared_by_x_cell", "xind_trace_by_x"),
                         ("eta_squared_by_x_cell", "xind_eta_by_x")):
        assert np.abs(xc[mine] - np.nan_to_num(z[theirs], nan=0.0)).max() <= 1e-9 * xs, mine
