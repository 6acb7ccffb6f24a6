"""Batches of independent problems stacked into one system (doubleadapparabolicfem_b200/batch.py).

CPU: the stacked problem assembles (oracle restatement) to the block-diagonal union of the
problems' own blocks.  GPU: a seeded batch with piecewise-constant kappa, solved and
estimated as one stacked system, against every problem solved on its own (FP64 path):
each problem's own true relative residual meets the tolerance, per-cell indicators agree
to 1e-9 of the problem's largest cell value; the FP32-refined patch solves agree with the
FP64 path to 1e-9 of the largest cell value.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import assert_same_sparse

import apf_oracle as O


def _oracle(prob):
    return O.MainProblem(p=prob.p, y_geom=prob.y_geometry, x_geom=prob.x_geometry, y_to_x=prob.y_to_x,
                         y_restr=O.Restriction(prob.y_restriction.offsets, prob.y_restriction.dofs,
                                               prob.y_restriction.weights, prob.ndof),
                         x_restr=O.Restriction(prob.x_restriction.offsets, prob.x_restriction.dofs,
                                               prob.x_restriction.weights, prob.ndof),
                         n_lambda=prob.n_lambda, n_u=prob.n_u, m_cells=prob.m_cells)


def test_stacked_problem_is_the_block_diagonal_union():
    from doubleadapparabolicfem_b200.batch import random_batch, stack
    problems = random_batch(3, seed=5, cells=(200, 5000))
    stacked, off = stack(problems)
    whole = O.assemble_main_blocks(_oracle(stacked))
    parts = [O.assemble_main_blocks(_oracle(q)) for q in problems]
    for nm in ("A_y", "B", "C_signed"):
        assert_same_sparse(sp.block_diag([p[nm] for p in parts]), whole[nm], 1e-14, nm)
    assert np.array_equal(np.concatenate([p["g"] for p in parts]), whole["g"])
    assert off["lambda"][-1] == stacked.n_lambda and off["u"][-1] == stacked.n_u


def _shard_rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from doubleadapparabolicfem_b200.batch import random_batch, shard, stack
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    problems = random_batch(12, seed=4, cells=(200, 5000))
    mine = shard(problems, rank, world)
    stacked, _ = stack(mine) if mine else (None, None)
    got = [None] * world
    dist.all_gather_object(got, [q.meta["index"] for q in mine])
    cells = torch.tensor([float(sum(q.n_y_cells for q in mine))], dtype=torch.float64)
    dist.all_reduce(cells)
    if rank == 0:
        out.put((got, float(cells[0]), [sum(problems[i].n_y_cells for i in g) for g in got],
                 max(q.n_y_cells for q in problems), sum(q.n_y_cells for q in problems),
                 stacked.n_y_cells if stacked is not None else 0, sum(q.n_y_cells for q in mine)))
    dist.destroy_process_group()


def test_batch_shards_over_two_ranks_without_overlap():
    """The multi-GPU form of a batch on two gloo ranks (CPU): every problem on exactly one
    rank, the cell loads within one problem of each other, each rank's stack holding its
    shard, and the scalar totals combined by one reduction."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, total, loads, biggest, all_cells, stacked_cells, mine_cells = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(got[0] + got[1]) == list(range(12)) and not set(got[0]) & set(got[1])
    assert total == all_cells
    assert abs(loads[0] - loads[1]) <= biggest
    assert stacked_cells == mine_cells


@pytest.mark.gpu
def test_batched_solve_and_estimate_match_single_problems(gpu_ctx):
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.batch import random_batch, solve_batch
    from doubleadapparabolicfem_b200.estimator import estimate
    from doubleadapparabolicfem_b200.solver import SolverOptions, solve_saddle_system_with_preconditioner
    problems = random_batch(5, seed=3, cells=(300, 40000))
    tol = 1e-11
    res, stats = solve_batch(problems, gpu_ctx, tol=tol, patch_precision="fp64", keep_cells=True)
    assert len(stats) == 1 and stats[0]["problems"] == 5
    res32, _ = solve_batch(problems, gpu_ctx, tol=tol, patch_precision="fp32_refined", keep_cells=True)
    for q, r, r32 in zip(problems, res, res32):
        assert r["residual"] <= tol
        blocks = assemble_main_system_blocks(q, ctx=gpu_ctx)
        blocks.assemble_parabolic_graph_norm_approximation()
        _, diag = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=tol), copy_out=False)
        cells, _ = estimate(blocks)
        blocks.close()
        scale = np.abs(cells["flux"]).max()
        for key in ("flux", "divergence", "eta"):
            assert np.abs(r[key] - cells[key]).max() <= 1e-9 * scale, (q.meta, key)
            assert np.abs(r32[key] - r[key]).max() <= 1e-9 * scale, (q.meta, key, "fp32")


@pytest.mark.gpu
def test_partitioned_solve_meets_every_problems_own_tolerance(gpu_ctx):
    """Two stacked problems, the second one's right-hand side scaled by 1e-3: the stacked
    MINRES is accepted only when each problem's own relative true residual meets the
    tolerance (checked here on the host with the stacked K), which needs the global residual
    well below it; the restarts keep tightening the backend tolerance until then (a restart
    that needs no iteration because the global residual already met the tightened tolerance
    no longer ends the solve)."""
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.batch import part_residuals, random_batch, set_partition, stack
    from doubleadapparabolicfem_b200.solver import SolverOptions, solve_saddle_system_with_preconditioner
    problems = random_batch(2, seed=7, cells=(2000, 20000))
    prob, off = stack(problems)
    blocks = assemble_main_system_blocks(prob, ctx=gpu_ctx)
    blocks.assemble_parabolic_graph_norm_approximation()
    set_partition(blocks, off)
    nl = blocks.n_lambda()
    rows = [np.r_[off["lambda"][p]:off["lambda"][p + 1], nl + off["u"][p]:nl + off["u"][p + 1]] for p in range(2)]
    rhs = np.concatenate([blocks.f(), blocks.g()])
    rhs[rows[1]] *= 1e-3
    tol = 1e-8
    x, diag = solve_saddle_system_with_preconditioner(blocks, SolverOptions(tolerance=tol), rhs=rhs)
    assert diag["converged"] == 1
    assert part_residuals(blocks, 2).max() <= tol
    K = blocks.K().tocsr()
    r = rhs - K @ x
    for rr in rows:
        assert np.linalg.norm(r[rr]) <= tol * np.linalg.norm(rhs[rr]) * (1 + 1e-6)
    blocks.close()
