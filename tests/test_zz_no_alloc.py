"""GPU test of apf_true_residual_noalloc, the allocation-free residual check.

Some callers cannot allocate device memory at the point where they need the FP64 true
residual of a solve (their device memory is owned by their own pool, or the GPU is so full
that a late allocation could fail).  This entry point computes ||b - K x|| / ||b|| from
device arrays the caller already holds, with its scratch in a fixed device array.  The test
checks it through the C ABI against the residual the MINRES entry point reports for the
same K, x and b, on two calls in a row, and that the second call leaves the device's free
memory unchanged.  It lives in its own file named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(ctx, rows, rp, ci, va, x, b):
    from doubleadapparabolicfem_b200 import _lib
    a, r = C.c_double(), C.c_double()
    rc = ctx.lib.apf_true_residual_noalloc(ctx.handle, rows, C.c_void_p(rp), C.c_void_p(ci), C.c_void_p(va),
                                           C.c_void_p(x), C.c_void_p(b), C.byref(a), C.byref(r))
    return rc, a.value, r.value


def test_noalloc_residual_matches_minres_report(gpu_ctx):
    import torch
    from doubleadapparabolicfem_b200 import _lib
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    from doubleadapparabolicfem_b200.solver import SolverOptions, solve_saddle_system_with_preconditioner

    blocks = assemble_main_system_blocks(uniform_problem(3, 1), ctx=gpu_ctx)
    blocks.assemble_parabolic_graph_norm_approximation()
    _, diag = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=1e-10), copy_out=False)
    rp, ci, va = blocks.block_device_ptrs("K")
    sol = C.c_void_p()
    gpu_ctx.check(gpu_ctx.lib.apf_system_solution_device_ptr(blocks.handle, C.byref(sol)))
    n = blocks.n_lambda() + blocks.n_u()
    b = torch.from_numpy(np.concatenate([blocks.f(), blocks.g()])).to(f"cuda:{gpu_ctx.device}")
    torch.cuda.synchronize()

    results = []
    free_before_second = None
    for call in range(2):
        if call == 1:
            torch.cuda.synchronize()
            free_before_second = torch.cuda.mem_get_info(gpu_ctx.device)[0]
        rc, absolute, relative = _noalloc(gpu_ctx, n, rp, ci, va, sol.value, b.data_ptr())
        assert rc == _lib.APF_OK, gpu_ctx.lib.apf_ctx_last_error(gpu_ctx.handle)
        results.append((absolute, relative))
    free_after_second = torch.cuda.mem_get_info(gpu_ctx.device)[0]

    # The solver evaluates the same FP64 residual with its own SpMV (another summation
    # order): b - K x carries rounding of order eps * ||b||, so near convergence the two
    # relative residuals agree to an absolute 1e-14, not to a fraction of their size.
    reported = diag["final_true_residual"]
    for absolute, relative in results:
        assert abs(relative - reported) <= 1e-12 * reported + 1e-14, (relative, reported)
        assert abs(absolute - relative * float(torch.linalg.norm(b))) <= 1e-12 * absolute
    assert results[0] == results[1]
    assert free_after_second == free_before_second


def test_noalloc_rejects_rows_beyond_scratch_limit(gpu_ctx):
    from doubleadapparabolicfem_b200 import _lib
    # the row count is checked on the host before anything else, so nothing is launched
    rc, _, _ = _noalloc(gpu_ctx, 20_000_000, 0, 0, 0, 0, 0)
    assert rc == _lib.APF_ERR_CAPACITY
    assert "scratch limit" in gpu_ctx.lib.apf_ctx_last_error(gpu_ctx.handle).decode()
