"""CPU tests: the oracle restatement against the reference's own outputs, and the
host-side mesh generator against the reference's meshes and published DOF counts."""
import json
import os

import numpy as np
import pytest

from conftest import (ADAPTIVE_CASES, DRIVER_CASES, G_DELTA_CASES, GOLDEN, GOLDEN_CASES, HHAT_RESIDUE,
                      assert_same_sparse, load_g_space, load_golden)

import apf_oracle as O


ALL_2D = GOLDEN_CASES + ADAPTIVE_CASES + DRIVER_CASES + ["p1_kappa_uniform"]


@pytest.mark.parametrize("name", ALL_2D)
def test_oracle_main_blocks_match_reference(name):
    prob, ref, example = load_golden(name)
    u0 = O.sin_initial if example == "smooth_initial" else O.one_initial
    out = O.assemble_main_blocks(prob, u0=u0)
    for nm in ("A_y", "B", "C_signed"):
        assert_same_sparse(ref[nm], out[nm], 1e-12, nm)
    assert np.abs(out["f"] - ref["f"]).max() <= 1e-12 * max(1.0, np.abs(ref["f"]).max())
    assert np.abs(out["g"] - ref["g"]).max() <= 1e-12 * np.abs(ref["g"]).max()


@pytest.mark.parametrize("name", ALL_2D)
def test_oracle_graph_norm_matches_reference(name):
    prob, ref, example = load_golden(name)
    gn = O.assemble_graph_norm(prob, ref["A_y"], ref["C_signed"])
    residue = HHAT_RESIDUE if name in ADAPTIVE_CASES + DRIVER_CASES else 0.0
    assert_same_sparse(ref["Hhat"], gn["Hhat"], 1e-12, "Hhat", residue=residue)


M_ANISO = (2.0, 0.5, 1.0)  # (m00, m01, m11) of the fixtures' second two-pass call


@pytest.mark.parametrize("name", ALL_2D)
def test_oracle_two_pass_full_saddle_matches_reference(name):
    prob, ref, example = load_golden(name)
    u0 = O.sin_initial if example == "smooth_initial" else O.one_initial
    assert ref["K2p_pattern_reuse_count"] == 1
    m_example = prob.m_cells
    for key, m in (("K2p", None), ("K2p_aniso", M_ANISO)):
        prob.m_cells = m_example if m is None else np.tile(m, (prob.y_geom.shape[0], 1))
        K, rhs = O.assemble_main_full_saddle_two_pass(prob, u0=u0)
        assert_same_sparse(ref[key], K, 1e-12, key)
        assert np.abs(rhs - ref[key + "_rhs"]).max() <= 1e-12 * np.abs(ref[key + "_rhs"]).max()
    # the identity coefficient's right-angle couplings cancel to zero and are pruned; the
    # anisotropic one keeps them, so the two patterns differ
    assert ref["K2p"].nnz < ref["K2p_aniso"].nnz


def test_adaptive_fixtures_have_hanging_nodes_and_finer_y():
    """The adaptive fixtures exercise what uniform meshes cannot: restriction rows with several
    weighted entries (space-time hanging nodes of X, temporal ones of Y), Y cells finer than
    their X ancestors, and Y cells spanning several time slabs."""
    for name in ADAPTIVE_CASES:
        prob, ref, _ = load_golden(name)
        xo = np.diff(prob.x_restr.offsets)
        yo = np.diff(prob.y_restr.offsets)
        assert xo.max() >= 3 and (xo > 1).sum() > 10, name
        assert (yo > 1).sum() > 0, name
        assert prob.y_geom.shape[0] > prob.x_geom.shape[0], name
        z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
        assert len(z["slab_of_cell"]) > prob.y_geom.shape[0], name


@pytest.mark.parametrize("name", ADAPTIVE_CASES + DRIVER_CASES)
def test_oracle_slab_reconstruction_matches_reference(name):
    """lambda~ of the slab reconstruction on the reference's own time-slab space, from the
    reference's u_delta: the slab DOF count and lambda~ at every slab cell's vertices and
    slab end times (1e-12 of the largest value)."""
    prob, ref, example = load_golden(name)
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    src, slab, geom, restr, lt = O.slab_reconstruction(prob, z["y_vertex_ids"], z["u_delta"])
    assert len(lt) == int(z["slab_dof_base"][-1])
    nodal = O.nodal_values(restr, lt)
    p = prob.p
    vertex_nodes = [0, 1, 2] if p == 1 else [0, 2, 5]
    time_nodes = [0, 1] if p == 1 else [0, 2]
    mine = np.stack([nodal[:, s * (p + 1) + a] for s in vertex_nodes for a in time_nodes], axis=1)
    cell_index = {int(c): i for i, c in enumerate(z["y_cell_ids"])}
    order = {(int(k), cell_index[int(c)]): i for i, (k, c) in enumerate(zip(z["slab_of_cell"], z["slab_source_cell"]))}
    perm = [order[(int(k), int(c))] for k, c in zip(slab, src)]
    theirs = z["slab_lambda_tilde"][perm]
    assert np.abs(mine - theirs).max() <= 1e-12 * np.abs(theirs).max()


@pytest.mark.parametrize("name", G_DELTA_CASES)
def test_oracle_g_delta_matches_reference(name):
    """The driver's G^delta estimator restated with every block a same-degree G form
    (u_delta and lambda_delta interpolated into G) against the reference's own computation
    on the same solution: A_G pattern and values to 1e-12 (P2 stiffness entries that cancel
    exactly leave residues below 1e-13 of the largest entry that the reference keeps where
    kappa lifts them above its 1e-15 filter: the significant pattern is compared), f_G, rhs_G = f_G -
    B(X,G)^T u_delta and lambda_G to 1e-12 of their largest entries, and
    ||lambda_G - lambda_delta||^2_{A_G} to 1e-10."""
    import scipy.sparse as sp
    prob, ref, example = load_golden(name)
    n_g, g, z = load_g_space(name)
    e, info = O.g_delta(prob, g, n_g, z["lambda_delta"], z["u_delta"])
    A_ref = sp.csc_matrix((z["A_g_values"], z["A_g_inner"], z["A_g_outer"]),
                          shape=tuple(int(v) for v in z["A_g_shape"]))
    assert_same_sparse(A_ref, info["A_g"], 1e-12, "A_G", residue=HHAT_RESIDUE)
    for key in ("f_g", "rhs_g", "lambda_g", "lambda_delta_in_g"):
        scale = max(np.abs(z[key]).max(), 1e-300)
        assert np.abs(info[key] - z[key]).max() <= 1e-12 * scale, key
    want = float(z["g_lambda_difference_squared"][0])
    assert want > 0 and abs(e - want) <= 1e-10 * want, (e, want)


def _paper_rows():
    with open(os.path.join(GOLDEN, "paper_uniform_rows.json")) as fh:
        return json.load(fh)


@pytest.mark.parametrize("p", [1, 2])
def test_uniform_mesh_dof_counts_match_paper_data(p):
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    rows = [r for r in _paper_rows() if r["dimension"] == "2d" and r["p"] == f"p{p}"
            and r["example"] == "smooth_initial"]
    assert rows
    checked = 0
    for r in rows:
        level = int(r["outer_iteration"])
        if level < 1 or level > (5 if p == 1 else 4):
            continue
        prob = uniform_problem(level, p)
        assert prob.n_u == int(r["x_true_dofs_before"]), r
        assert prob.n_lambda == int(r["y_true_dofs_after"]), r
        checked += 1
    assert checked >= 3


def _cell_key(geom):
    tri = geom[:, :6].reshape(-1, 3, 2)
    order = np.lexsort((tri[:, :, 1], tri[:, :, 0]))
    tri_sorted = np.take_along_axis(tri, order[:, :, None], axis=1).reshape(-1, 6)
    return np.round(np.concatenate([tri_sorted, geom[:, 6:]], 1) * 2 ** 20).astype(np.int64)


@pytest.mark.parametrize("name", ["p1_l1_smooth", "p1_l2_smooth", "p2_l1_smooth"])
def test_uniform_mesh_geometry_equals_reference(name):
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    prob, ref, _ = load_golden(name)
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    mine = uniform_problem(int(z["meta_level"][0]), prob.p)
    a = _cell_key(prob.y_geom)
    b = _cell_key(mine.y_geometry)
    sa = a[np.lexsort(a.T[::-1])]
    sb = b[np.lexsort(b.T[::-1])]
    assert np.array_equal(sa, sb)
    assert mine.n_lambda == prob.n_lambda and mine.n_u == prob.n_u


def dof_permutation(prob_ref, prob_mine, space):
    """perm[i_ref] = i_mine by matching DOF coordinates."""
    from doubleadapparabolicfem_b200.mesh import dof_coordinates, SpaceTimeProblem, Restriction
    ref_as_product = SpaceTimeProblem(
        p=prob_ref.p, y_geometry=prob_ref.y_geom, x_geometry=prob_ref.x_geom, y_to_x=prob_ref.y_to_x,
        y_restriction=Restriction(prob_ref.y_restr.offsets, prob_ref.y_restr.dofs, prob_ref.y_restr.weights,
                                  prob_ref.y_restr.ndof),
        x_restriction=Restriction(prob_ref.x_restr.offsets, prob_ref.x_restr.dofs, prob_ref.x_restr.weights,
                                  prob_ref.x_restr.ndof),
        n_lambda=prob_ref.n_lambda, n_u=prob_ref.n_u)
    cr = np.round(dof_coordinates(ref_as_product, space) * 2 ** 20).astype(np.int64)
    cm = np.round(dof_coordinates(prob_mine, space) * 2 ** 20).astype(np.int64)
    kr = np.lexsort(cr.T[::-1])
    km = np.lexsort(cm.T[::-1])
    assert np.array_equal(cr[kr], cm[km])
    perm = np.empty(len(kr), dtype=np.int64)
    perm[kr] = km
    return perm


@pytest.mark.parametrize("name", ["p1_l2_smooth", "p2_l1_smooth"])
def test_generated_mesh_assembles_to_reference_blocks(name):
    """Our own uniform mesh + numbering, assembled by the oracle, equals the reference's
    blocks after the coordinate permutation (pattern bit-exact, values 1e-12)."""
    import scipy.sparse as sp
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    prob, ref, example = load_golden(name)
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    mine = uniform_problem(int(z["meta_level"][0]), prob.p)
    py = dof_permutation(prob, mine, "y")
    px = dof_permutation(prob, mine, "x")
    mp = O.MainProblem(p=mine.p, y_geom=mine.y_geometry, x_geom=mine.x_geometry, y_to_x=mine.y_to_x,
                       y_restr=O.Restriction(mine.y_restriction.offsets, mine.y_restriction.dofs,
                                             mine.y_restriction.weights, mine.ndof),
                       x_restr=O.Restriction(mine.x_restriction.offsets, mine.x_restriction.dofs,
                                             mine.x_restriction.weights, mine.ndof),
                       n_lambda=mine.n_lambda, n_u=mine.n_u)
    out = O.assemble_main_blocks(mp)
    Py = sp.csr_matrix((np.ones(len(py)), (np.arange(len(py)), py)), shape=(len(py), len(py)))
    Px = sp.csr_matrix((np.ones(len(px)), (np.arange(len(px)), px)), shape=(len(px), len(px)))
    assert_same_sparse(ref["A_y"], Py @ out["A_y"] @ Py.T, 1e-12, "A_y")
    assert_same_sparse(ref["B"], Px @ out["B"] @ Py.T, 1e-12, "B")
    assert_same_sparse(ref["C_signed"], Px @ out["C_signed"] @ Px.T, 1e-12, "C")
    assert np.abs(Px @ out["g"] - ref["g"]).max() <= 1e-12 * np.abs(ref["g"]).max()


def _paper_row(level, p="p1", example="smooth_initial"):
    rows = [r for r in _paper_rows() if r["dimension"] == "2d" and r["p"] == p and r["example"] == example
            and int(r["outer_iteration"]) == level]
    return rows[0]


@pytest.mark.parametrize("name", ["p1_l1_smooth", "p1_l2_smooth", "p1_l3_smooth"])
def test_reference_x_indicators_match_paper(name):
    """The reference's own X-marking indicators (written by the oracle driver) reproduce
    the published lambda_y_squared and eta_squared of the uniform runs (6 digits)."""
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    row = _paper_row(int(z["meta_level"][0]))
    lam = float(row["lambda_y_squared"])
    eta = float(row["eta_squared"])
    assert abs(z["xind_lambda_by_x"].sum() - lam) <= 1e-5 * lam
    assert abs(np.nansum(z["xind_eta_by_x"]) - eta) <= 1e-5 * eta
    assert abs(z["xind_lambda_by_y"].sum() - z["xind_lambda_by_x"].sum()) <= 1e-12 * lam


def test_y_estimator_threshold_matches_paper():
    """apf_y_estimator_threshold_squared (a host function of the library, no GPU needed)
    against the published thresholds, from the published lambda^2 and eta^2."""
    from doubleadapparabolicfem_b200 import build
    build.build()
    from doubleadapparabolicfem_b200.estimator import y_estimator_threshold_squared
    checked = 0
    for r in _paper_rows():
        if r["dimension"] != "2d" or not r.get("y_estimator_threshold_squared") or not r.get("configured_rho"):
            continue
        lam, eta = float(r["lambda_y_squared"]), float(r["eta_squared"])
        got = y_estimator_threshold_squared(float(r["configured_rho"]), lam, eta - lam)
        want = float(r["y_estimator_threshold_squared"])
        assert abs(got - want) <= 2e-5 * want + 1e-12, r
        checked += 1
    assert checked >= 10
    with pytest.raises(Exception):
        y_estimator_threshold_squared(0.0, 1.0, 1.0)
