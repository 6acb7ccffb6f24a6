"""GPU tests of the block-preconditioned MINRES (through the C ABI).

Parity of MINRES iterates with the reference is not pinned (the reference uses
Eigen's MINRES with exact sparse Cholesky blocks); the acceptance test is the
reference's own: FP64 true relative residual ||K x - b|| / ||b|| <= tol, checked here
on the host in FP64 with the reference's K and rhs, plus agreement with a direct solve.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from conftest import GOLDEN_CASES, load_golden, to_product_problem

pytestmark = pytest.mark.gpu


def _ref_system(ref):
    K = sp.bmat([[ref["A_y"], ref["B"].T], [ref["B"], ref["C_signed"]]]).tocsc()
    b = np.concatenate([ref["f"], ref["g"]])
    return K, b


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_minres_reaches_true_residual_on_reference_system(gpu_ctx, name):
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.solver import SolverOptions, solve_saddle_system_with_preconditioner
    prob, ref, example = load_golden(name)
    blocks = assemble_main_system_blocks(to_product_problem(prob, example), ctx=gpu_ctx)
    blocks.assemble_parabolic_graph_norm_approximation()
    x, diag = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=1e-10, amg_coarse_size=64))
    K, b = _ref_system(ref)
    rel = np.linalg.norm(K @ x - b) / np.linalg.norm(b)
    assert rel <= 1e-10, (rel, diag)
    assert diag["converged"] == 1
    assert abs(diag["final_true_residual"] - rel) <= 1e-12
    x_direct = spla.spsolve(K, b)
    assert np.linalg.norm(x - x_direct) <= 1e-6 * np.linalg.norm(x_direct)


@pytest.mark.parametrize("level,p", [(3, 1), (4, 1), (2, 2)])
def test_minres_generated_mesh(gpu_ctx, level, p):
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    from doubleadapparabolicfem_b200.solver import SolverOptions, solve_saddle_system_with_preconditioner
    prob = uniform_problem(level, p)
    blocks = assemble_main_system_blocks(prob, ctx=gpu_ctx)
    blocks.assemble_parabolic_graph_norm_approximation()
    x, diag = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=1e-8))
    K = blocks.K()
    b = np.concatenate([blocks.f(), blocks.g()])
    rel = np.linalg.norm(K @ x - b) / np.linalg.norm(b)
    assert rel <= 1e-8, (rel, diag)
    assert diag["iterations"] < 1000


def test_minres_failure_raises_with_diagnostics(gpu_ctx):
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    from doubleadapparabolicfem_b200.solver import (PreconditionedSolveFailure, SolverOptions,
                                                    solve_saddle_system_with_preconditioner)
    blocks = assemble_main_system_blocks(uniform_problem(3, 1), ctx=gpu_ctx)
    blocks.assemble_parabolic_graph_norm_approximation()
    with pytest.raises(PreconditionedSolveFailure) as e:
        solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=1e-12, max_iterations=3,
                                                                      true_residual_check_interval=1))
    assert e.value.diagnostics["iterations"] <= 3
    assert e.value.diagnostics["converged"] == 0


@pytest.mark.parametrize("level,p", [(3, 1), (2, 2)])
def test_correction_equation_and_residual_norms(gpu_ctx, level, p):
    """The device correction equation (K d = b - K x0 from zero, x = x0 + d; the dispatcher's
    solve_correction_equation, solve_saddle_system.hpp:75-86) against the same equation with
    the residual formed on the host, and the device residual norms against numpy."""
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    from doubleadapparabolicfem_b200.solver import (SolverOptions, residual_norms,
                                                    solve_saddle_system_with_preconditioner)
    blocks = assemble_main_system_blocks(uniform_problem(level, p), ctx=gpu_ctx)
    blocks.assemble_parabolic_graph_norm_approximation()
    K = blocks.K()
    b = np.concatenate([blocks.f(), blocks.g()])
    x0 = np.random.default_rng(3).standard_normal(b.size) * 1e-2
    tol = 1e-10
    x, diag = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=tol), initial_guess=x0,
                                                      correction=True)
    r0 = b - K @ x0
    # the tolerance is relative to the correction equation's right-hand side
    assert np.linalg.norm(K @ x - b) <= 1.0001 * tol * np.linalg.norm(r0), diag
    assert diag["converged"] == 1
    d_host, diag_host = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=tol), rhs=r0)
    # the two right-hand sides differ by the SpMV's rounding only; on this rough r0 that
    # moves MINRES's stopping iteration by up to ~15 %, so the solutions are compared
    assert diag_host["converged"] == 1
    assert np.linalg.norm(x - (x0 + d_host)) <= 1e-6 * np.linalg.norm(x)
    # the system holds x0 + d after the correction solve
    res, bn = residual_norms(blocks)
    assert abs(bn - np.linalg.norm(b)) <= 1e-13 * np.linalg.norm(b)
    # (d_host's solve replaced the held solution: compare against it)
    assert abs(res - np.linalg.norm(K @ d_host - b)) <= 1e-10 * np.linalg.norm(b)
    res0, _ = residual_norms(blocks, x0)
    assert abs(res0 - np.linalg.norm(r0)) <= 1e-12 * np.linalg.norm(b)
