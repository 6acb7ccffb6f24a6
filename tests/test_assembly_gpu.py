"""GPU parity tests of the main-system assembly (through the C ABI).

Bar: sparsity patterns bit-exact, values within 1e-12 relative to the block's
largest entry (the reference computes in FP64 with a different summation order).
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES, REPO, assert_same_sparse, load_golden, to_product_problem

import apf_oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _csc_of_B_from_BT(BT):
    # B^T in CSR has exactly the arrays of B in CSC
    return BT.T


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_assembly_matches_reference_fixtures(gpu_ctx, name):
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    prob, ref, example = load_golden(name)
    blocks = assemble_main_system_blocks(to_product_problem(prob, example), ctx=gpu_ctx)
    assert_same_sparse(ref["A_y"], blocks.A_y(), RTOL, "A_y")
    assert_same_sparse(ref["B"], blocks.lower_left_B(), RTOL, "B")
    assert_same_sparse(ref["B"], blocks.block("BT").T, RTOL, "B^T")
    assert_same_sparse(ref["C_signed"], blocks.C_signed(), RTOL, "C_signed")
    f, g = blocks.f(), blocks.g()
    assert np.abs(f - ref["f"]).max() <= RTOL * max(1.0, np.abs(ref["f"]).max())
    assert np.abs(g - ref["g"]).max() <= RTOL * np.abs(ref["g"]).max()
    # K = [A_y B^T; B C]
    import scipy.sparse as sp
    K_ref = sp.bmat([[ref["A_y"], ref["B"].T], [ref["B"], ref["C_signed"]]]).tocsr()
    assert_same_sparse(K_ref, blocks.K(), RTOL, "K")
    H = blocks.assemble_parabolic_graph_norm_approximation(1e-14)
    assert_same_sparse(ref["Hhat"], H, RTOL, "Hhat")


@pytest.mark.parametrize("level,p", [(2, 1), (3, 1), (1, 2), (2, 2)])
def test_assembly_on_generated_mesh_matches_oracle(gpu_ctx, level, p):
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    mine = uniform_problem(level, p)
    mp = O.MainProblem(p=p, y_geom=mine.y_geometry, x_geom=mine.x_geometry, y_to_x=mine.y_to_x,
                       y_restr=O.Restriction(mine.y_restriction.offsets, mine.y_restriction.dofs,
                                             mine.y_restriction.weights, mine.ndof),
                       x_restr=O.Restriction(mine.x_restriction.offsets, mine.x_restriction.dofs,
                                             mine.x_restriction.weights, mine.ndof),
                       n_lambda=mine.n_lambda, n_u=mine.n_u)
    ref = O.assemble_main_blocks(mp)
    blocks = assemble_main_system_blocks(mine, ctx=gpu_ctx)
    assert_same_sparse(ref["A_y"], blocks.A_y(), RTOL, "A_y")
    assert_same_sparse(ref["B"], blocks.lower_left_B(), RTOL, "B")
    assert_same_sparse(ref["C_signed"], blocks.C_signed(), RTOL, "C")
    gn = O.assemble_graph_norm(mp, ref["A_y"], ref["C_signed"])
    assert_same_sparse(gn["Hhat"], blocks.assemble_parabolic_graph_norm_approximation(), RTOL, "Hhat")


def _ref_bin():
    path = os.path.join(REPO, "oracle", "_ref", "apf_ref_dump")
    return path if os.path.exists(path) else None


@pytest.mark.slow
@pytest.mark.parametrize("level,p", [(3, 1), (4, 1), (2, 2)])
def test_assembly_matches_reference_binary_larger(gpu_ctx, level, p):
    """Larger meshes dumped on the spot by the compiled reference (oracle/_ref)."""
    exe = _ref_bin()
    if exe is None:
        pytest.skip("oracle/_ref/apf_ref_dump not built")
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    tmp = tempfile.mkdtemp()
    try:
        subprocess.run([exe, "2", str(p), str(level), "smooth_initial", tmp], check=True, capture_output=True)
        prob = O.load_problem(tmp, p)
        ref = {nm: O.load_csc(tmp, nm) for nm in ("A_y", "B", "C_signed", "Hhat")}
        g_ref = np.load(os.path.join(tmp, "g.npy"))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    blocks = assemble_main_system_blocks(to_product_problem(prob, "smooth_initial"), ctx=gpu_ctx)
    assert_same_sparse(ref["A_y"], blocks.A_y(), RTOL, "A_y")
    assert_same_sparse(ref["B"], blocks.lower_left_B(), RTOL, "B")
    assert_same_sparse(ref["C_signed"], blocks.C_signed(), RTOL, "C")
    assert np.abs(blocks.g() - g_ref).max() <= RTOL * np.abs(g_ref).max()
    assert_same_sparse(ref["Hhat"], blocks.assemble_parabolic_graph_norm_approximation(), RTOL, "Hhat")


def test_assembly_invariants_full_size(gpu_ctx):
    """Size-independent properties at the benchmark's P1 level-5 mesh (262,144 prisms):
    A_y and Hhat symmetric with positive diagonal; A_y 1 = 0 on rows away from the
    boundary (stiffness of a constant); B restricted to the time derivative part
    sums to zero over each column set (B_dt^T 1 = 0 for interior X rows)."""
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    mine = uniform_problem(5, 1)
    blocks = assemble_main_system_blocks(mine, ctx=gpu_ctx)
    A = blocks.A_y()
    assert A.shape == (254016, 254016)
    assert abs(A - A.T).max() <= 1e-13 * abs(A).max()
    assert (A.diagonal() > 0).all()
    H = blocks.assemble_parabolic_graph_norm_approximation()
    assert abs(H - H.T).max() <= 1e-13 * abs(H).max()
    assert (H.diagonal() > 0).all()
    C = blocks.C_signed()
    # -C_signed is the t=0 mass matrix: its entries sum to the integral of the
    # interior-node hat functions' products, a positive number below |Omega| = 1
    s = -C.sum()
    assert 0.9 < s < 1.0
