"""Batches of independent 2+1D problems (the batching form of the method; the reference
solves one problem per call).

Problems are stacked into one system: cells, true DOFs and spatial vertex ids are
concatenated with offsets, so the assembly, the graph-norm block, the AMG set-up, every
MINRES iteration and the estimator each run over all problems of a wave in one launch per
kernel.  The stacked matrices are block diagonal (no entry couples two problems), the AMG
never aggregates across problems (aggregates follow matrix couplings), and the edge of each
vertex patch stays inside its problem (vertex ids are offset).  MINRES runs one Krylov
sequence over the stacked system and accepts only when every problem's own relative true
residual ||b_p - K_p x_p|| / ||b_p|| meets the tolerance (apf_system_set_partition).

``random_batch`` draws the problems of the batching configuration from a seed: element
counts log-uniform in [1e4, 5e5]; each mesh is the largest uniform outer level below its
count, locally refined by bisection around a seeded point until the count is reached;
diffusivity kappa piecewise constant per X cell, log-uniform in [0.1, 10] (M = kappa I).

    python -m doubleadapparabolicfem_b200.batch --problems 256 --seed 0

prints one JSON line with the batch throughput and the FP32-refined patch solves' error
against the FP64 path.  Under ``torchrun --nproc-per-node N`` each GPU solves its ``shard``
of the batch (no exchange between GPUs); rank 0 prints the totals (elements summed, wall
time of the slowest rank).
"""
from __future__ import annotations

import argparse
import ctypes as C
import dataclasses
import json
import math
import os
import time

import numpy as np

from . import _lib
from .mesh import Restriction, SpaceTimeProblem, uniform_problem


def cells_of_level(level: int) -> int:
    """Prisms of the uniform outer level (2 n^2 triangles x n/2 slabs, n = 2^(level+1))."""
    return 2 ** (3 * level + 3)


def level_for_cells(target: float, levels=range(1, 7)) -> int:
    return min(levels, key=lambda L: abs(math.log(cells_of_level(L)) - math.log(target)))


def level_below_cells(target: float, levels=range(1, 7)) -> int:
    """The largest uniform outer level with at most `target` prisms (at least the first)."""
    fit = [L for L in levels if cells_of_level(L) <= target]
    return max(fit) if fit else min(levels)


def refined_to_cells(target: float, level: int, point_seed: int, cache: dict, max_depth: int = 8):
    """The uniform outer level `level` locally refined around a seeded point
    (refine.locally_refined_problem: newest-vertex bisection near the point in the time
    intervals near it) with the smallest depth that reaches `target` prisms."""
    from .refine import locally_refined_problem
    for depth in range(1, max_depth + 1):
        key = (level, depth, point_seed)
        if key not in cache:
            cache[key] = locally_refined_problem(level=level, seed=point_seed, depth=depth, radius0=0.5,
                                                 time_rounds=2, kappa_blocks=1)
        if cache[key].n_y_cells >= target or depth == max_depth:
            return cache[key], depth


def random_batch(n_problems: int, seed: int = 0, cells=(1e4, 5e5), kappa=(0.1, 10.0), meshes: str = "refined",
                 point_seeds: int = 4) -> list[SpaceTimeProblem]:
    """The batching configuration's problems from a seed: a target element count log-uniform in
    `cells`; meshes = "refined": the largest uniform outer level below the target, then local
    bisection around one of `point_seeds` seeded points with the smallest depth that reaches
    the target (as the reference's refine_points_n_times is repeated until the count is
    met); meshes = "uniform": the nearest uniform outer level.  kappa per X cell log-uniform
    in `kappa` (M = kappa I on the cell's Y cells)."""
    rng = np.random.default_rng(seed)
    cache: dict = {}
    out = []
    for i in range(n_problems):
        target = math.exp(rng.uniform(math.log(cells[0]), math.log(cells[1])))
        if meshes == "refined":
            level = level_below_cells(target)
            base, depth = refined_to_cells(target, level, int(rng.integers(point_seeds)), cache)
        else:
            level, depth = level_for_cells(target), 0
            if level not in cache:
                cache[level] = uniform_problem(level, 1)
            base = cache[level]
        kap_x = np.exp(rng.uniform(math.log(kappa[0]), math.log(kappa[1]), size=base.n_x_cells))
        kap = kap_x[np.asarray(base.y_to_x)]
        m = np.zeros((base.n_y_cells, 3))
        m[:, 0] = kap
        m[:, 2] = kap
        out.append(dataclasses.replace(base, m_cells=m, meta={"level": level, "depth": depth, "target_cells": target,
                                                               "index": i}))
    return out


def shard(problems: list[SpaceTimeProblem], rank: int, world: int) -> list[SpaceTimeProblem]:
    """The problems one of ``world`` GPUs solves when a batch is spread over several: the
    problems are independent, so each GPU stacks and solves its own share with no exchange
    between GPUs.  Greedy by decreasing cell count onto the GPU with the fewest cells so far
    (ties: the lower problem index, the lower rank), so every rank computes the same split
    from the same batch and every problem lands on exactly one rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    loads = [0] * world
    owner = [0] * len(problems)
    for i in sorted(range(len(problems)), key=lambda k: (-problems[k].n_y_cells, k)):
        r = min(range(world), key=lambda k: (loads[k], k))
        owner[i] = r
        loads[r] += problems[i].n_y_cells
    return [q for q, r in zip(problems, owner) if r == rank]


def stack(problems: list[SpaceTimeProblem]):
    """One block-diagonal problem from independent ones -> (problem, offsets), offsets =
    {"y_cells", "x_cells", "lambda", "u"} arrays of len(problems) + 1."""
    if not problems:
        raise ValueError("empty batch")
    p = problems[0].p
    if any(q.p != p or q.u0_kind != problems[0].u0_kind or getattr(q, "dim_space", 2) != 2 for q in problems):
        raise ValueError("a batch needs one degree, one u0 and 2+1D problems")
    n = len(problems)
    oy = np.zeros(n + 1, dtype=np.int64)
    ox = np.zeros(n + 1, dtype=np.int64)
    ol = np.zeros(n + 1, dtype=np.int64)
    ou = np.zeros(n + 1, dtype=np.int64)
    for k, q in enumerate(problems):
        oy[k + 1] = oy[k] + q.n_y_cells
        ox[k + 1] = ox[k] + q.n_x_cells
        ol[k + 1] = ol[k] + q.n_lambda
        ou[k + 1] = ou[k] + q.n_u
    if ol[-1] >= 2 ** 31 or ou[-1] >= 2 ** 31:
        raise ValueError("stacked system exceeds int32 DOF indices")

    def restr(parts, dof_off):
        offs, dofs, ws = [np.zeros(1, dtype=np.int64)], [], []
        base = 0
        for r, d0 in zip(parts, dof_off):
            offs.append(r.offsets[1:].astype(np.int64) + base)
            dofs.append(r.dofs.astype(np.int64) + d0)
            ws.append(r.weights)
            base += int(r.offsets[-1])
        return Restriction(np.concatenate(offs).astype(np.int32), np.concatenate(dofs).astype(np.int32),
                           np.concatenate(ws), parts[0].ndof)

    m_rows = []
    for q in problems:
        if q.m_cells is None:
            m_rows.append(np.tile([1.0, 0.0, 1.0], (q.n_y_cells, 1)))
        else:
            m_rows.append(np.asarray(q.m_cells, dtype=np.float64).reshape(q.n_y_cells, 3))
    ell = None
    if any(q.ell_cells is not None for q in problems):
        ell = np.concatenate([np.zeros(q.n_y_cells) if q.ell_cells is None else q.ell_cells for q in problems])
    vids, voff = [], 0
    for q in problems:
        if q.y_vertex_ids is None:
            raise ValueError("stacked problems need their spatial vertex ids")
        vids.append(q.y_vertex_ids.astype(np.int64) + voff)
        voff += int(q.y_vertex_ids.max()) + 1
    stacked = SpaceTimeProblem(
        p=p, y_geometry=np.vstack([q.y_geometry for q in problems]),
        x_geometry=np.vstack([q.x_geometry for q in problems]),
        y_to_x=np.concatenate([q.y_to_x.astype(np.int64) + ox[k] for k, q in enumerate(problems)]).astype(np.int32),
        y_restriction=restr([q.y_restriction for q in problems], ol[:-1]),
        x_restriction=restr([q.x_restriction for q in problems], ou[:-1]),
        n_lambda=int(ol[-1]), n_u=int(ou[-1]), m_cells=np.vstack(m_rows), ell_cells=ell,
        u0_kind=problems[0].u0_kind, y_vertex_ids=np.vstack(vids).astype(np.int32))
    return stacked, {"y_cells": oy, "x_cells": ox, "lambda": ol, "u": ou}


def set_partition(blocks, offsets):
    lam = np.ascontiguousarray(offsets["lambda"], dtype=np.int32)
    u = np.ascontiguousarray(offsets["u"], dtype=np.int32)
    ctx = blocks.ctx
    ctx.check(ctx.lib.apf_system_set_partition(ctx.handle, blocks.handle, len(lam) - 1,
                                               C.c_void_p(lam.ctypes.data), C.c_void_p(u.ctypes.data)))


def part_residuals(blocks, n_parts):
    out = np.empty(n_parts)
    ctx = blocks.ctx
    ctx.check(ctx.lib.apf_system_part_residuals(ctx.handle, blocks.handle, C.c_void_p(out.ctypes.data)))
    return out


def waves(problems, max_cells):
    """Consecutive groups of problems with at most max_cells cells (at least one problem)."""
    cur, size = [], 0
    for q in problems:
        if cur and size + q.n_y_cells > max_cells:
            yield cur
            cur, size = [], 0
        cur.append(q)
        size += q.n_y_cells
    if cur:
        yield cur


def solve_batch(problems, ctx, tol=1e-8, patch_precision="fp64", max_cells_per_wave=6_000_000,
                estimate_too=True, keep_cells=False, compare_fp64=False, amg_strength=None):
    """Assemble, solve and estimate every problem, wave by wave.  Returns per-problem results
    (true relative residual, flux^2 / div^2 / eta^2 totals, optionally per-cell arrays) and
    per-wave statistics."""
    from .assembly import assemble_main_system_blocks
    from .estimator import estimate
    from .solver import SolverOptions, solve_saddle_system_with_preconditioner
    from concurrent.futures import ThreadPoolExecutor
    results, wave_stats = [], []
    groups = list(waves(problems, max_cells_per_wave))
    # the host stacks the next wave while the device works on the current one
    pool = ThreadPoolExecutor(max_workers=1)
    pending = pool.submit(stack, groups[0]) if groups else None
    for gi, wave in enumerate(groups):
        t0 = time.perf_counter()
        stacked, off = pending.result()
        pending = pool.submit(stack, groups[gi + 1]) if gi + 1 < len(groups) else None
        t1 = time.perf_counter()
        blocks = assemble_main_system_blocks(stacked, ctx=ctx)
        set_partition(blocks, off)
        blocks.assemble_parabolic_graph_norm_approximation()
        opts = SolverOptions(tolerance=tol)
        if amg_strength is not None:
            opts.amg_strength = amg_strength
        _, diag = solve_saddle_system_with_preconditioner(blocks, opts, copy_out=False)
        res = part_residuals(blocks, len(wave))
        cells = None
        cells64 = None
        if estimate_too:
            cells, _ = estimate(blocks, patch_precision=patch_precision)
            if compare_fp64 and patch_precision != "fp64":
                cells64, _ = estimate(blocks, patch_precision="fp64")
        ctx.synchronize()
        t2 = time.perf_counter()
        for k, q in enumerate(wave):
            r = {"residual": float(res[k]), "n_cells": q.n_y_cells, "n_dofs": q.n_lambda + q.n_u,
                 "level": q.meta.get("level")}
            if cells is not None:
                sl = slice(int(off["y_cells"][k]), int(off["y_cells"][k + 1]))
                for key in ("flux", "divergence", "eta"):
                    r[key + "_squared"] = float(cells[key][sl].sum())
                    if keep_cells:
                        r[key] = cells[key][sl].copy()
                if cells64 is not None:
                    scale = float(np.abs(cells64["flux"][sl]).max())
                    r["fp32_refined_max_cell_err"] = float(np.abs(cells["eta"][sl] - cells64["eta"][sl]).max() / scale)
                    r["fp32_refined_total_rel_err"] = float(abs(cells["flux"][sl].sum() - cells64["flux"][sl].sum()) /
                                                            cells64["flux"][sl].sum())
            results.append(r)
        wave_stats.append({"problems": len(wave), "cells": int(off["y_cells"][-1]),
                           "dofs": int(off["lambda"][-1] + off["u"][-1]), "minres_iterations": diag["iterations"],
                           "host_stack_wait_s": t1 - t0, "device_s": t2 - t1})
        blocks.close()
    pool.shutdown()
    return results, wave_stats


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--problems", type=int, default=256)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--max-cells-per-wave", type=int, default=6_000_000)
    ap.add_argument("--patch-precision", default="fp32_refined", choices=["fp64", "fp32_refined"])
    ap.add_argument("--meshes", default="refined", choices=["refined", "uniform"])
    ap.add_argument("--amg-strength", type=float, default=None,
                    help="AMG strength-of-connection threshold (default: 0.003 on refined meshes, where it cut the "
                         "batch from 70.5 to 59.2 s; the library's on uniform ones)")
    args = ap.parse_args()
    from .assembly import Context
    # one process per GPU (torchrun): each rank solves its shard of the batch; only the
    # scalar totals are combined (elements summed, wall time the slowest rank's)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("gloo", rank=rank, world_size=world)
    ctx = Context(local)
    t0 = time.perf_counter()
    problems = shard(random_batch(args.problems, args.seed, meshes=args.meshes), rank, world)
    t_gen = time.perf_counter() - t0
    # warm-up on the smallest problem (kernel loading, pool growth)
    if problems:
        solve_batch(sorted(problems, key=lambda q: q.n_y_cells)[:1], ctx, args.tol, args.patch_precision)
    t1 = time.perf_counter()
    if dist:
        dist.barrier()
        t1 = time.perf_counter()
    if args.amg_strength is None and args.meshes == "refined":
        args.amg_strength = 0.003
    res, stats = solve_batch(problems, ctx, args.tol, args.patch_precision, args.max_cells_per_wave,
                             amg_strength=args.amg_strength)
    wall = time.perf_counter() - t1
    # the FP32-refined patch solves against the FP64 path on the first wave (a rank with an
    # empty shard has none)
    cmp = []
    if problems:
        first = next(waves(problems, args.max_cells_per_wave))
        cmp, _ = solve_batch(first, ctx, args.tol, "fp32_refined", args.max_cells_per_wave, compare_fp64=True)
    level_ids = list(range(16))
    counts = [sum(1 for q in problems if int(q.meta["level"]) == lv) for lv in level_ids]
    summed = [float(sum(r["n_cells"] for r in res)), float(sum(r["n_dofs"] for r in res))] + [float(c) for c in counts]
    worst = [wall, sum(w["device_s"] for w in stats), max((r["residual"] for r in res), default=0.0),
             max((r["fp32_refined_max_cell_err"] for r in cmp), default=0.0),
             max((r["fp32_refined_total_rel_err"] for r in cmp), default=0.0)]
    if dist:
        # every rank's totals: elements, DOFs and problems per level summed; wall time, device
        # time, the largest per-problem residual and the FP32 errors the worst over the ranks
        ts = torch.tensor(summed, dtype=torch.float64)
        dist.all_reduce(ts)
        tw = torch.tensor(worst, dtype=torch.float64)
        dist.all_reduce(tw, op=dist.ReduceOp.MAX)
        summed, worst = ts.tolist(), tw.tolist()
        dist.destroy_process_group()
        if rank != 0:
            return
    cells, dofs = int(summed[0]), int(summed[1])
    levels = {lv: int(c) for lv, c in zip(level_ids, summed[2:]) if c > 0}
    wall, device_s = worst[0], worst[1]
    print(json.dumps({
        "workload": f"{args.problems} independent 2+1D P1 problems (seed {args.seed}, {args.meshes} meshes: element "
                    f"counts log-uniform in [1e4, 5e5]), kappa log-uniform [0.1, 10] per X cell, tol {args.tol}, "
                    f"patch solves {args.patch_precision}, AMG strength "
                    f"{args.amg_strength if args.amg_strength is not None else 'default'}",
        "n_gpus": world, "scaling": "strong (one batch split over the GPUs)",
        "problems_per_level": {str(k): v for k, v in sorted(levels.items())},
        "cells": cells, "dofs": dofs, "waves": len(stats),
        "elements_per_s": cells / wall, "dofs_per_s": dofs / wall,
        "device_elements_per_s": cells / device_s if device_s > 0 else None, "wall_s": wall,
        "device_s_slowest_rank": device_s,
        "host_stack_wait_s_rank0": sum(w["host_stack_wait_s"] for w in stats), "host_generate_s_rank0": t_gen,
        "max_part_residual": worst[2],
        "minres_iterations_per_wave_rank0": [w["minres_iterations"] for w in stats],
        "fp32_refined_vs_fp64_first_wave": {
            "max_cell_err_over_max_cell": worst[3],
            "max_total_rel_err": worst[4]},
    }))


if __name__ == "__main__":
    main()
