"""GPU test of apf_true_residual_noalloc, the allocation-free residual check.

Some callers cannot allocate device memory at the point where they need the FP64 true
residual of a solve (their device memory is owned by their own pool, or the GPU is so full
that a late allocation could fail).  This entry point computes ||b - K x|| / ||b|| from
device arrays the caller already holds, with its scratch in a fixed device array; only its
first call on a device (the set-up: the scratch address and the kernels' code) may take
device memory.  The test checks it through the C ABI against the residual computed on the
host in FP64 (scipy) and against the one the MINRES entry point reports, on calls in a row,
one of them with a matrix of another row length (another kernel variant), and that no call
after the set-up changes the device's free memory.  It lives in its own file named to be
collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(ctx, rows, rp, ci, va, x, b):
    a, r = C.c_double(), C.c_double()
    rc = ctx.lib.apf_true_residual_noalloc(ctx.handle, rows, C.c_void_p(rp), C.c_void_p(ci), C.c_void_p(va),
                                           C.c_void_p(x), C.c_void_p(b), C.byref(a), C.byref(r))
    return rc, a.value, r.value


def _host_residual(A, x, b):
    r = b - A @ x
    return float(np.linalg.norm(r)), float(np.linalg.norm(r) / np.linalg.norm(b))


def test_noalloc_residual_matches_host_and_minres(gpu_ctx):
    import torch
    from doubleadapparabolicfem_b200 import _lib
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    from doubleadapparabolicfem_b200.solver import SolverOptions, solve_saddle_system_with_preconditioner

    dev = f"cuda:{gpu_ctx.device}"
    blocks = assemble_main_system_blocks(uniform_problem(3, 1), ctx=gpu_ctx)
    blocks.assemble_parabolic_graph_norm_approximation()
    x_host, diag = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=1e-10))
    K = blocks.K().tocsr()
    A = blocks.A_y().tocsr()
    f, g = blocks.f(), blocks.g()
    b_host = np.concatenate([f, g])
    nl = blocks.n_lambda()
    n = nl + blocks.n_u()
    # K (about 23 entries per row) and A_y (about 9.5) select different lanes-per-row kernels
    assert K.nnz / K.shape[0] > 14 >= A.nnz / A.shape[0]
    krp, kci, kva = blocks.block_device_ptrs("K")
    arp, aci, ava = blocks.block_device_ptrs("A_y")
    x = torch.from_numpy(x_host).to(dev)
    b = torch.from_numpy(b_host).to(dev)
    rng = np.random.default_rng(5)
    xa_host, fa_host = rng.standard_normal(nl), rng.standard_normal(nl)
    xa = torch.from_numpy(xa_host).to(dev)
    fa = torch.from_numpy(fa_host).to(dev)
    torch.cuda.synchronize()

    # first call on this device: the set-up (may allocate)
    rc, _, _ = _noalloc(gpu_ctx, n, krp, kci, kva, x.data_ptr(), b.data_ptr())
    assert rc == _lib.APF_OK, gpu_ctx.lib.apf_ctx_last_error(gpu_ctx.handle)
    torch.cuda.synchronize()
    free_after_setup = torch.cuda.mem_get_info(gpu_ctx.device)[0]

    k_results = []
    for _ in range(2):
        rc, absolute, relative = _noalloc(gpu_ctx, n, krp, kci, kva, x.data_ptr(), b.data_ptr())
        assert rc == _lib.APF_OK, gpu_ctx.lib.apf_ctx_last_error(gpu_ctx.handle)
        k_results.append((absolute, relative))
    rc, a_abs, a_rel = _noalloc(gpu_ctx, nl, arp, aci, ava, xa.data_ptr(), fa.data_ptr())
    assert rc == _lib.APF_OK, gpu_ctx.lib.apf_ctx_last_error(gpu_ctx.handle)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(gpu_ctx.device)[0] == free_after_setup

    # against the host FP64 residual (another summation order: b - K x carries rounding of
    # order eps ||b||, so near convergence they agree to an absolute 1e-14 of ||b||)
    h_abs, h_rel = _host_residual(K, x_host, b_host)
    for absolute, relative in k_results:
        assert abs(relative - h_rel) <= 1e-10 * h_rel + 1e-14, (relative, h_rel)
        assert abs(absolute - h_abs) <= 1e-10 * h_abs + 1e-14 * np.linalg.norm(b_host)
    assert k_results[0] == k_results[1]
    # and the residual the solver reported for the same solve
    reported = diag["final_true_residual"]
    assert abs(k_results[0][1] - reported) <= 1e-12 * reported + 1e-14, (k_results[0][1], reported)
    # the A_y call: far from a solution, so the residual is large and agrees relatively
    ha_abs, ha_rel = _host_residual(A, xa_host, fa_host)
    assert abs(a_abs - ha_abs) <= 1e-12 * ha_abs and abs(a_rel - ha_rel) <= 1e-12 * ha_rel


def test_noalloc_rejects_rows_beyond_scratch_limit(gpu_ctx):
    from doubleadapparabolicfem_b200 import _lib
    # the row count is checked on the host before anything else, so nothing is launched
    rc, _, _ = _noalloc(gpu_ctx, 20_000_000, 0, 0, 0, 0, 0)
    assert rc == _lib.APF_ERR_CAPACITY
    assert "scratch limit" in gpu_ctx.lib.apf_ctx_last_error(gpu_ctx.handle).decode()
