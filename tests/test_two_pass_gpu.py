"""GPU parity tests of the two-pass full saddle assembly (assemble_main_full_saddle_two_pass_2d,
two_pass_full_saddle_2d.hpp:468) through the C ABI.

Bar: against the reference's own two-pass output (fixtures ``K2p`` and, on the reference's
cached pattern with M = [[2, 0.5], [0.5, 1]], ``K2p_aniso``) patterns bit-exact and values
within 1e-12 of the largest entry; against the device's own block path (K pruned of
|value| <= zero_tol) and between cached and uncached calls, bit for bit.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN_CASES, assert_same_sparse, load_golden, to_product_problem

import apf_oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-12
M_ANISO = (2.0, 0.5, 1.0)


def _pruned(K, tol=1e-15):
    K = K.tocsr(copy=True)
    K.data[np.abs(K.data) <= tol] = 0.0
    K.eliminate_zeros()
    return K


def _assert_identical(a, b, what):
    a, b = a.tocsr(), b.tocsr()
    assert a.shape == b.shape, what
    assert np.array_equal(a.indptr, b.indptr), f"{what}: row pointers"
    assert np.array_equal(a.indices, b.indices), f"{what}: columns"
    assert np.array_equal(a.data, b.data), f"{what}: values differ bitwise"


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_two_pass_matches_reference_fixtures(gpu_ctx, name):
    from doubleadapparabolicfem_b200.assembly import (TwoPassFullSaddleAssemblyCache,
                                                      assemble_main_full_saddle_two_pass)
    prob, ref, example = load_golden(name)
    problem = to_product_problem(prob, example)
    cache = TwoPassFullSaddleAssemblyCache(gpu_ctx)
    try:
        first = assemble_main_full_saddle_two_pass(problem, ctx=gpu_ctx, assembly_cache=cache)
        assert_same_sparse(ref["K2p"], first.matrix, RTOL, "K")
        rhs = first.rhs
        assert np.abs(rhs - ref["K2p_rhs"]).max() <= RTOL * np.abs(ref["K2p_rhs"]).max()
        first.close()
        problem.m_cells = np.tile(M_ANISO, (problem.y_geometry.shape[0], 1))
        second = assemble_main_full_saddle_two_pass(problem, ctx=gpu_ctx, assembly_cache=cache)
        assert_same_sparse(ref["K2p_aniso"], second.matrix, RTOL, "K (anisotropic M, cached pattern)")
        assert np.abs(second.rhs - ref["K2p_aniso_rhs"]).max() <= RTOL * np.abs(ref["K2p_aniso_rhs"]).max()
        second.close()
        st = cache.stats()
        assert st["pattern_builds"] == 1
        assert st["pattern_reuse_count"] == ref["K2p_pattern_reuse_count"] == 1
    finally:
        cache.close()


@pytest.mark.parametrize("level,p", [(3, 1), (2, 2)])
def test_two_pass_equals_pruned_block_path_bitwise(gpu_ctx, level, p):
    from doubleadapparabolicfem_b200.assembly import assemble_main_full_saddle_two_pass, assemble_main_system_blocks
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    rng = np.random.default_rng(7 + level)
    prob = uniform_problem(level, p)
    ny = prob.y_geometry.shape[0]
    # SPD per-cell tensors with a spread of scales
    k = np.exp(rng.uniform(np.log(0.1), np.log(10.0), ny))
    prob.m_cells = np.stack([k, 0.3 * k * rng.uniform(-1, 1, ny), k * rng.uniform(0.5, 2.0, ny)], 1)
    blocks = assemble_main_system_blocks(prob, ctx=gpu_ctx)
    K_block = blocks.K()
    f, g = blocks.f(), blocks.g()
    blocks.close()
    two = assemble_main_full_saddle_two_pass(prob, ctx=gpu_ctx)
    _assert_identical(_pruned(K_block), two.matrix, "two-pass K vs pruned block-path K")
    assert np.array_equal(two.rhs, np.concatenate([f, g]))
    two.close()


def test_two_pass_cache_reuse_is_bitwise_and_rebuilds_on_a_new_mesh(gpu_ctx):
    from doubleadapparabolicfem_b200.assembly import (TwoPassFullSaddleAssemblyCache,
                                                      assemble_main_full_saddle_two_pass)
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    rng = np.random.default_rng(11)
    cache = TwoPassFullSaddleAssemblyCache(gpu_ctx)
    try:
        prob = uniform_problem(4, 1)
        ny = prob.y_geometry.shape[0]
        assemble_main_full_saddle_two_pass(prob, ctx=gpu_ctx, assembly_cache=cache).close()
        for trial in range(3):
            k = np.exp(rng.uniform(np.log(0.01), np.log(100.0), ny))
            prob.m_cells = np.stack([k, np.zeros(ny), k], 1)
            prob.ell_cells = rng.uniform(-1.0, 1.0, ny)
            cached = assemble_main_full_saddle_two_pass(prob, ctx=gpu_ctx, assembly_cache=cache)
            fresh = assemble_main_full_saddle_two_pass(prob, ctx=gpu_ctx)
            _assert_identical(fresh.matrix, cached.matrix, f"cached vs fresh, trial {trial}")
            assert np.array_equal(fresh.rhs, cached.rhs)
            cached.close()
            fresh.close()
        st = cache.stats()
        assert st["pattern_builds"] == 1 and st["pattern_reuse_count"] == 3
        # another mesh: the key differs, the pattern is rebuilt and the result is right
        other = uniform_problem(3, 1)
        two = assemble_main_full_saddle_two_pass(other, ctx=gpu_ctx, assembly_cache=cache)
        K_ref, rhs_ref = O.assemble_main_full_saddle_two_pass(
            O.MainProblem(p=1, y_geom=other.y_geometry, x_geom=other.x_geometry, y_to_x=other.y_to_x,
                          y_restr=O.Restriction(other.y_restriction.offsets, other.y_restriction.dofs,
                                                other.y_restriction.weights, other.ndof),
                          x_restr=O.Restriction(other.x_restriction.offsets, other.x_restriction.dofs,
                                                other.x_restriction.weights, other.ndof),
                          n_lambda=other.n_lambda, n_u=other.n_u))
        assert_same_sparse(K_ref, two.matrix, RTOL, "K after a mesh change")
        assert np.abs(two.rhs - rhs_ref).max() <= RTOL * np.abs(rhs_ref).max()
        two.close()
        assert cache.stats()["pattern_builds"] == 2
    finally:
        cache.close()


def test_two_pass_rejects_one_plus_one_d(gpu_ctx):
    from doubleadapparabolicfem_b200._lib import ApfError
    from doubleadapparabolicfem_b200.assembly import assemble_main_full_saddle_two_pass
    from doubleadapparabolicfem_b200.mesh import uniform_problem_1d
    with pytest.raises(ApfError):
        assemble_main_full_saddle_two_pass(uniform_problem_1d(2), ctx=gpu_ctx)
