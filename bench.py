"""Benchmark: one inner iteration of the adaptive cycle of the 2+1D space-time heat problem on B200.

Workload (default, ``--workload refined``: the learned-preconditioner configuration the
metric is quoted on): 2+1D heat equation on (0,1)^2 x (0,1), u0 = sin(pi x) sin(pi y),
f = 0, P1, FP64, on a locally refined space-time mesh of about 4M DOFs
(doubleadapparabolicfem_b200.refine.locally_refined_problem: the uniform outer-level-6 base,
6 levels of newest-vertex bisection around a seeded interior point in the time intervals near
it, 2 halvings of those intervals; 2.84M prisms, 4.21M DOFs, 128k hanging-node rows in X) and
a diffusivity kappa log-uniform in [0.01, 100], constant on each square of a 4 x 4
partition (contrast up to 1e4).  The learned preconditioner is timed as the line's value,
the plain block preconditioner on the same steps beside it; both build their AMG
hierarchies with strength threshold 0.003 (REFINED_AMG_STRENGTH).  ``--workload uniform``: the
uniform outer level ``--level`` mesh (default 6: 2,097,152 prisms, 3,112,897 DOFs) with
M = I.  Synthetic inputs generated on the host.

A step = the hot path of one inner iteration over one mesh, as
compute_adaptive_test_space_iteration runs it: main-system assembly (A_y, B, B^T,
C_signed, K, f, g), the parabolic graph-norm block Hhat, the block preconditioner's
set-up, MINRES to FP64 true relative residual 1e-8, and the equilibrated-flux estimator
(slab reconstruction, vertex-patch flux solves, per-cell indicators) and the driver's
X-marking indicators, from inputs already in HBM.  ``e2e`` = the same through the C ABI
from pinned host buffers (H2D of the mesh inputs and D2H of the solution and the
per-cell Y and X indicators inside the timed region).

Multi-GPU: the path runs one problem per GPU (replicas; no collective in the data
path).  ``value`` = total DOFs processed by all ranks / max-over-ranks time.

``--impl reference`` times the reference's own CPU implementation of the same inner
iteration (oracle/_ref/apf_ref_dump: the reference templates compiled here) on the host
cores, on a bounded sample of the workload: the same mesh family two outer levels coarser
(its own local refinement at the same point, kappa of the same law), every stage of the
reference's own code (its two-pass saddle assembly, slab reconstruction, patch solves,
indicators) timed; its main saddle solve, which the reference runs with PARDISO (absent
here), is not factored (the oracle shim's stand-in direct solver would dominate and is not
the reference's code), so the reference's DOFs/s excludes the solve while ours includes it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "2+1D adaptive-cycle DOFs/s at 1e-8 residual; learned vs plain precond on B200"
UNIT = "DOFs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="refined", choices=["refined", "uniform"])
    ap.add_argument("--seed", type=int, default=0, help="seed of the refined workload's point and kappa")
    ap.add_argument("--level", type=int, default=6)
    ap.add_argument("--p", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-estimator", action="store_true")
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--profile-run", action="store_true",
                    help="one device-resident step and exit (a short program for ncu captures); no JSON line")
    ap.add_argument("--pool-reserve-gb", type=float, default=0.0,
                    help="grow the device memory pool to this size once before the warm-up")
    ap.add_argument("--amg-smooth-steps", type=int, default=None,
                    help="damped-Jacobi sweeps per side of the V-cycle (default: the library's)")
    ap.add_argument("--amg-strength", type=float, default=None,
                    help="AMG strength-of-connection threshold (default: the library's; the refined workload: 0.003)")
    ap.add_argument("--amg-aggressive-levels", type=int, default=None,
                    help="finest AMG levels aggregated from a distance-2 independent set (default: the library's)")
    ap.add_argument("--precond", default="learned", choices=["learned", "plain"],
                    help="learned: the shipped model (plain block preconditioner as fallback), timed beside plain")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region by an in-process NVML
    thread (every 0.5 s; an nvidia-smi process polling the driver every 200 ms was seen to
    stall the library's launches)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, device, period=0.5):
        self.device = device
        self.period = period
        self.samples = []
        self._stop = None
        self._t = None
        self._nvml = None

    def _run(self):
        nv = self._nvml
        h = nv.nvmlDeviceGetHandleByIndex(self.device)
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                get = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                    nv.nvmlDeviceGetCurrentClocksThrottleReasons
                reasons = get(h)
                self.samples.append((sm, mx, reasons))
            except Exception:
                pass
            self._stop.wait(self.period)

    def __enter__(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nvml = pynvml
        except Exception:
            return self
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        if self._t:
            self._stop.set()
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [s[0] for s in self.samples]
        reasons = sorted({name for s in self.samples for name, bit in self.REASONS.items() if s[2] & bit})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(s[1] for s in self.samples), "reasons": reasons,
                "samples": len(self.samples), "source": "nvml"}


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# the refined workload: generator settings (refine.locally_refined_problem)
REFINED = dict(depth=6, radius0=0.15, time_rounds=2, kappa_range=(0.01, 100.0), kappa_blocks=4)
# AMG strength-of-connection threshold for the refined workload (both preconditioners): with
# kappa jumps of 1e4 across block edges and cells graded over six bisection levels, the default
# 0.08 drops too many couplings; a sweep over {0.08, 0.02, 0.01, 0.005, 0.003, 0.002, 0} gave the
# fewest MINRES iterations for plain and learned at 0.003
REFINED_AMG_STRENGTH = 0.003
# steps of the plain-preconditioner comparison and of the e2e measurement (at most; a step of
# the refined workload takes seconds, the plain solver's many more)
PLAIN_STEPS, E2E_STEPS = 2, 3


def build_problem(args):
    if args.workload == "uniform":
        from doubleadapparabolicfem_b200.mesh import uniform_problem
        return uniform_problem(args.level, args.p)
    from doubleadapparabolicfem_b200.refine import locally_refined_problem
    if args.p != 1:
        raise SystemExit("the refined workload is P1")
    return locally_refined_problem(level=args.level, seed=args.seed, **REFINED)


def workload_text(args, prob=None):
    if args.workload == "uniform":
        return f"2+1D heat, u0=sin(pi x)sin(pi y), M=I, uniform outer level {args.level} P{args.p}"
    return (f"2+1D heat, u0=sin(pi x)sin(pi y), P1, outer level {args.level} base locally refined "
            f"({REFINED['depth']} levels of bisection near a seeded point, seed {args.seed}), kappa log-uniform "
            f"[{REFINED['kappa_range'][0]}, {REFINED['kappa_range'][1]}] on {REFINED['kappa_blocks']}x"
            f"{REFINED['kappa_blocks']} blocks, learned vs plain preconditioner")


def refined_point(args):
    import numpy as np
    return np.random.default_rng(args.seed).uniform(0.25, 0.75, 3)


def sample_level_for(level: int) -> int:
    """Outer level of the bounded CPU sample: two levels below the workload (the reference's
    own stages at outer level 4 take a few seconds per inner iteration on 8 cores)."""
    return max(1, level - 2)


def cpu_reference_sample(args, reps: int, threads: int | None = None):
    """Time the reference's own CPU inner iteration (oracle/_ref) on a bounded sample of the
    workload: its own mesh at the sample level (refined workload: its refine_points_n_times at
    the same point, depth rounds, kappa of the same law on the same blocks), every stage of its
    own code; the main solve (PARDISO in the reference) is not factored."""
    exe = os.path.join(REPO, "oracle", "_ref", "apf_ref_dump")
    if not os.path.exists(exe):
        return None
    env = dict(os.environ)
    env["APF_REF_CYCLE"] = "1"
    env["APF_SHIM_SKIP_PARDISO"] = "1"
    if args.workload == "refined":
        x, y, t = refined_point(args)
        env["APF_REF_X_POINTS"] = f"{x},{y},{t}"
        env["APF_REF_X_ROUNDS"] = str(REFINED["depth"])
        lo, hi = REFINED["kappa_range"]
        env["APF_REF_KAPPA"] = f"{args.seed}:{lo}:{hi}"
        env["APF_REF_KAPPA_BLOCKS"] = str(REFINED["kappa_blocks"])
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    out = subprocess.run([exe, "bench", str(args.p), str(sample_level_for(args.level)), "smooth_initial", str(reps)],
                         capture_output=True, text=True, env=env, timeout=1800)
    if out.returncode != 0:
        return None
    info = json.loads(out.stdout.strip().splitlines()[-1])
    info["stages_s"] = info["mean_s"] - info.get("main_solve_mean_s", 0.0)
    return info


def sample_text(info, sample_level):
    return (f"one inner iteration of the reference's own code at outer level {sample_level} of the same mesh family "
            f"({info['n_cells']} prisms, {info['n_dofs']} DOFs): two-pass saddle assembly, slab reconstruction, "
            f"patch flux solves, indicators; main solve (PARDISO in the reference) not factored and not timed; "
            f"compiled -O3 -DNDEBUG, as the reference's release presets")


def run_reference(args, world, rank):
    # rank 0 alone times the reference CPU path; other ranks do no work
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    sample_level = sample_level_for(args.level)
    exe = os.path.join(REPO, "oracle", "_ref", "apf_ref_dump")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/apf_ref_dump was not built (needs the reference sources)"}))
        return
    # one run of the reference's binary: its own mesh is built once (host refinement), then
    # warm-up + timed repetitions of the inner iteration; the warm-ups are dropped
    info = cpu_reference_sample(args, args.warmup + args.steps, threads)
    if info is None or len(info.get("stage_s", [])) != args.warmup + args.steps:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/apf_ref_dump bench failed"}))
        return
    times = info["stage_s"][args.warmup:]
    t = sum(times)
    value = args.steps * info["n_dofs"] / t
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_text(args),
                   "stages": ["assembly", "slab_reconstruction", "patch_fluxes", "indicators"],
                   "excluded": "the main saddle solve (the reference's PARDISO / Eigen solvers are absent; "
                               "the oracle shim's stand-in is not the reference's code)",
                   "flux_squared": info.get("flux_squared")},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": info["threads"], "kind": "reference",
                         "sample": sample_text(info, sample_level) + " per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_ours(args, world, rank, local):
    import ctypes as C

    import numpy as np
    import torch
    from doubleadapparabolicfem_b200 import build as b
    from doubleadapparabolicfem_b200 import _lib
    from doubleadapparabolicfem_b200.assembly import Context, MainSystemBlocks, make_desc, _Keep
    from doubleadapparabolicfem_b200.mesh import SpaceTimeProblem, Restriction

    b.build()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.Stream(device=dev)
    ctx = Context(local, stream=stream.cuda_stream)
    lib = ctx.lib

    host = build_problem(args)
    n_dofs = host.n_lambda + host.n_u
    ny = host.n_y_cells
    run_estimator = not args.no_estimator

    def to_dev(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).to(dev)

    def to_pinned(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).pin_memory()

    def clone_problem(conv):
        return SpaceTimeProblem(
            p=host.p, y_geometry=conv(host.y_geometry, np.float64), x_geometry=conv(host.x_geometry, np.float64),
            y_to_x=conv(host.y_to_x, np.int32),
            y_restriction=Restriction(conv(host.y_restriction.offsets, np.int32), conv(host.y_restriction.dofs, np.int32),
                                      conv(host.y_restriction.weights, np.float64), host.ndof),
            x_restriction=Restriction(conv(host.x_restriction.offsets, np.int32), conv(host.x_restriction.dofs, np.int32),
                                      conv(host.x_restriction.weights, np.float64), host.ndof),
            n_lambda=host.n_lambda, n_u=host.n_u, u0_kind=host.u0_kind,
            m_cells=None if host.m_cells is None else conv(host.m_cells, np.float64),
            y_vertex_ids=conv(host.y_vertex_ids, np.int32))

    dprob = clone_problem(to_dev)
    hprob = clone_problem(to_pinned)
    h2d_tensors = [hprob.y_geometry, hprob.x_geometry, hprob.y_to_x, hprob.y_restriction.offsets,
                   hprob.y_restriction.dofs, hprob.y_restriction.weights, hprob.x_restriction.offsets,
                   hprob.x_restriction.dofs, hprob.x_restriction.weights]
    if hprob.m_cells is not None:
        h2d_tensors.append(hprob.m_cells)
    if run_estimator:
        h2d_tensors.append(hprob.y_vertex_ids)
    h2d_bytes = sum(int(t.numel() * t.element_size()) for t in h2d_tensors)
    x_host = torch.empty(n_dofs, dtype=torch.float64).pin_memory()
    eta_host = torch.empty(ny, dtype=torch.float64).pin_memory()
    eta_dev = torch.empty(ny, dtype=torch.float64, device=dev)
    nx = host.n_x_cells
    etax_host = torch.empty(nx, dtype=torch.float64).pin_memory()
    etax_dev = torch.empty(nx, dtype=torch.float64, device=dev)
    d2h_bytes = n_dofs * 8 + ((ny + nx) * 8 if run_estimator else 0)
    sopt = _lib.SolverOptions()
    lib.apf_solver_options_default(C.byref(sopt))
    sopt.tolerance = args.tol
    if args.amg_aggressive_levels is not None:
        sopt.amg_aggressive_levels = args.amg_aggressive_levels
    if args.amg_smooth_steps is not None:
        sopt.amg_smooth_steps = args.amg_smooth_steps
    if args.amg_strength is not None:
        sopt.amg_strength = args.amg_strength
    elif args.workload == "refined":
        sopt.amg_strength = REFINED_AMG_STRENGTH
    from doubleadapparabolicfem_b200 import learned as LM
    learned_model = None
    if args.precond == "learned" and os.path.exists(LM.DEFAULT_WEIGHTS):
        learned_model = LM.LearnedModel.load()
        LM.use_model(ctx, learned_model)
        sopt.preconditioner = _lib.APF_PRECOND_LEARNED
    solve_diags = []
    est_results = []

    def step(prob, on_device, allow_unconverged=False):
        keep = _Keep()
        desc = make_desc(prob, 1e-15, -1.0, keep)
        h = C.c_void_p()
        ctx.check(lib.apf_assemble_main_system(ctx.handle, C.byref(desc), 1 if on_device else 0, C.byref(h)))
        try:
            ctx.check(lib.apf_assemble_graph_norm(ctx.handle, h, 1e-14))
            d = _lib.SolverDiagnostics()
            out = None if on_device else C.c_void_p(x_host.data_ptr())
            rc = lib.apf_solve_minres(ctx.handle, h, C.byref(sopt), None, out, 0, C.byref(d))
            if not (allow_unconverged and rc == _lib.APF_ERR_NOT_CONVERGED):
                ctx.check(rc)
            solve_diags.append({k: getattr(d, k) for k, _ in d._fields_})
            if run_estimator:
                res = _lib.EstimatorResult()
                eta = eta_dev if on_device else eta_host
                ctx.check(lib.apf_estimate(ctx.handle, h, C.c_void_p(prob.y_vertex_ids.data_ptr()),
                                           1 if on_device else 0, None, None, None, C.c_void_p(eta.data_ptr()),
                                           C.byref(res)))
                xt = _lib.XIndicatorTotals()
                etax = etax_dev if on_device else etax_host
                ctx.check(lib.apf_x_indicators(ctx.handle, h, 1 if on_device else 0, None, None, None,
                                               C.c_void_p(etax.data_ptr()), C.byref(xt)))
                r = {k: getattr(res, k) for k, _ in res._fields_}
                r.update({"x_" + k: getattr(xt, k) for k, _ in xt._fields_})
                est_results.append(r)
        except Exception:
            lib.apf_system_destroy(h)
            raise
        return h

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def pool_stats():
        v = [C.c_int64() for _ in range(4)]
        ctx.check(lib.apf_ctx_pool_stats(ctx.handle, *[C.byref(x) for x in v]))
        return [round(x.value / 2 ** 30, 2) for x in v]

    if args.pool_reserve_gb > 0:
        ctx.check(lib.apf_ctx_reserve_pool(ctx.handle, int(args.pool_reserve_gb * 2 ** 30)))
    if args.profile_run:
        h = step(dprob, True)
        ctx.synchronize()
        sizes = []
        for block, name in ((0, "A_y"), (1, "Hhat_F")):
            r, na, npp, om, al = C.c_int(), C.c_int64(), C.c_int64(), C.c_double(), C.c_double()
            ctx.check(lib.apf_amg_level_info(ctx.handle, h, block, 0, C.byref(r), C.byref(na), C.byref(npp),
                                             C.byref(om), C.byref(al)))
            sizes.append(f"{name} level 0: {r.value} rows, {na.value} nonzeros")
        kr, kc, knnz = C.c_int32(), C.c_int32(), C.c_int64()
        ctx.check(lib.apf_system_block_info(h, _lib.BLOCKS["K"], C.byref(kr), C.byref(kc), C.byref(knnz)))
        sizes.append(f"K: {kr.value} rows, {knnz.value} nonzeros")
        lib.apf_system_destroy(h)
        print(f"profile run: {solve_diags[-1]['iterations']} MINRES iterations, {ctx.kernel_launches()} launches; "
              + "; ".join(sizes))
        return
    # warm-up
    for _ in range(args.warmup):
        lib.apf_system_destroy(step(dprob, True))
    ctx.synchronize()

    # timed device-resident steps
    launches0 = ctx.kernel_launches()
    barrier()
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    step_events = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        stage_ms = []
        for k in range(args.steps):
            ctx.check(lib.apf_ctx_set_timing(ctx.handle, 2))
            lib.apf_system_destroy(step(dprob, True))
            step_events[k].record(stream)
            rep = json.loads(lib.apf_ctx_timing_report(ctx.handle).decode())
            st = {k2[5:]: round(v[1], 1) for k2, v in rep.items() if k2.startswith("host:")}
            st["pool_gib_reserved_high_used_high"] = pool_stats()
            stage_ms.append(st)
        ctx.check(lib.apf_ctx_set_timing(ctx.handle, 0))
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    step_ms = [round(ev0.elapsed_time(step_events[0]), 2)] + [
        round(step_events[k - 1].elapsed_time(step_events[k]), 2) for k in range(1, args.steps)]
    barrier()
    launches = ctx.kernel_launches() - launches0
    elapsed = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    timed_diags = solve_diags[-args.steps:]
    timed_est = est_results[-args.steps:]

    # the plain block preconditioner on the same steps, for the learned-vs-plain comparison
    plain = None
    if sopt.preconditioner == _lib.APF_PRECOND_LEARNED:
        # the plain block preconditioner on the same mesh (up to PLAIN_STEPS steps; a plain
        # solve that misses the tolerance within max_iterations is recorded as such, its time
        # then a lower bound)
        n_plain = min(args.steps, PLAIN_STEPS)
        sopt.preconditioner = _lib.APF_PRECOND_AMG_BLOCK
        barrier()
        torch.cuda.synchronize(dev)
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p_events = [torch.cuda.Event(enable_timing=True) for _ in range(n_plain)]
        p0.record(stream)
        for k in range(n_plain):
            lib.apf_system_destroy(step(dprob, True, allow_unconverged=True))
            p_events[k].record(stream)
        p1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        plain_elapsed = max_over_ranks(p0.elapsed_time(p1) / 1e3)
        pd = solve_diags[-n_plain:]
        plain = {"value": n_plain * n_dofs * world / plain_elapsed, "ms_per_step": 1e3 * plain_elapsed / n_plain,
                 "steps": n_plain, "converged": [d["converged"] for d in pd],
                 "max_iterations": sopt.max_iterations,
                 "minres_iterations": [d["iterations"] for d in pd],
                 "final_true_residual_max": max(d["final_true_residual"] for d in pd),
                 "minres_solve_s_mean": sum(d["solve_seconds"] for d in pd) / len(pd),
                 "step_ms": [round(p0.elapsed_time(p_events[0]), 2)] + [
                     round(p_events[k - 1].elapsed_time(p_events[k]), 2) for k in range(1, n_plain)]}
        sopt.preconditioner = _lib.APF_PRECOND_LEARNED

    # e2e through the C ABI from pinned host buffers (up to E2E_STEPS steps)
    n_e2e = min(args.steps, E2E_STEPS)
    barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e_events = [torch.cuda.Event(enable_timing=True) for _ in range(n_e2e)]
    e0.record(stream)
    e2e_stage_ms = []
    for k in range(n_e2e):
        ctx.check(lib.apf_ctx_set_timing(ctx.handle, 2))
        lib.apf_system_destroy(step(hprob, False))
        e_events[k].record(stream)
        rep = json.loads(lib.apf_ctx_timing_report(ctx.handle).decode())
        e2e_stage_ms.append({k2[5:]: round(v[1], 1) for k2, v in rep.items() if k2.startswith("host:")})
    ctx.check(lib.apf_ctx_set_timing(ctx.handle, 0))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    e2e_elapsed = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    e2e_step_ms = [round(e0.elapsed_time(e_events[0]), 2)] + [
        round(e_events[k - 1].elapsed_time(e_events[k]), 2) for k in range(1, n_e2e)]
    e2e_diags = solve_diags[-n_e2e:]

    # one more device-resident step with per-kernel CUDA-event timing on the library's stream
    # (kernel breakdown and the roofline's launch durations; not part of the timed steps)
    ctx.check(lib.apf_ctx_set_timing(ctx.handle, 1))
    h = step(dprob, True)
    ctx.synchronize()
    report = json.loads(lib.apf_ctx_timing_report(ctx.handle).decode())
    ctx.check(lib.apf_ctx_set_timing(ctx.handle, 0))
    kernels = {k: v for k, v in report.items() if not k.startswith("host:")}
    host_ranges = {k[5:]: round(v[1], 3) for k, v in report.items() if k.startswith("host:")}
    amg_levels = {}
    for block, name in ((0, "A_y"), (1, "Hhat_F")):
        L, dc, sw, sm = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        ctx.check(lib.apf_amg_info(ctx.handle, h, block, C.byref(L), C.byref(dc), C.byref(sw), C.byref(sm)))
        rows = []
        for lv in range(L.value):
            r, na, npp, om, al = C.c_int(), C.c_int64(), C.c_int64(), C.c_double(), C.c_double()
            ctx.check(lib.apf_amg_level_info(ctx.handle, h, block, lv, C.byref(r), C.byref(na), C.byref(npp),
                                             C.byref(om), C.byref(al)))
            rows.append([r.value, na.value, npp.value])
        amg_levels[name] = {"rows_nnz_nnzP": rows, "dense_coarsest": bool(dc.value)}
    # the precision form of the patch solves on the same solution: FP64 (the bench line's
    # path) against FP32 factorisation + one FP64 refinement step
    patch_precision = None
    if run_estimator and args.p == 1:
        cells = {}
        for prec_name, prec in (("fp64", _lib.APF_PATCH_FP64), ("fp32_refined", _lib.APF_PATCH_FP32_REFINED)):
            ctx.check(lib.apf_ctx_set_patch_precision(ctx.handle, prec))
            fl = torch.empty(ny, dtype=torch.float64, device=dev)
            et = torch.empty(ny, dtype=torch.float64, device=dev)
            res = _lib.EstimatorResult()
            # one untimed call first: the launch-shape autotuner tunes a precision's buckets
            # on their first use
            ctx.check(lib.apf_estimate(ctx.handle, h, C.c_void_p(dprob.y_vertex_ids.data_ptr()), 1,
                                       C.c_void_p(fl.data_ptr()), None, None, C.c_void_p(et.data_ptr()),
                                       C.byref(res)))
            ctx.check(lib.apf_ctx_set_timing(ctx.handle, 1))
            ctx.check(lib.apf_estimate(ctx.handle, h, C.c_void_p(dprob.y_vertex_ids.data_ptr()), 1,
                                       C.c_void_p(fl.data_ptr()), None, None, C.c_void_p(et.data_ptr()),
                                       C.byref(res)))
            rep = json.loads(lib.apf_ctx_timing_report(ctx.handle).decode())
            ctx.check(lib.apf_ctx_set_timing(ctx.handle, 0))
            cells[prec_name] = (fl.cpu().numpy(), et.cpu().numpy(), res.flux_squared,
                                rep.get("est_patch_solve", [0, float("nan")])[1],
                                rep.get("host:call_estimate", [0, float("nan")])[1])
        ctx.check(lib.apf_ctx_set_patch_precision(ctx.handle, _lib.APF_PATCH_FP64))
        f64, f32 = cells["fp64"], cells["fp32_refined"]
        scale = float(np.abs(f64[0]).max())
        patch_precision = {
            "patch_solve_ms_fp64": round(f64[3], 3), "patch_solve_ms_fp32_refined": round(f32[3], 3),
            "estimate_ms_fp64": round(f64[4], 3), "estimate_ms_fp32_refined": round(f32[4], 3),
            "max_cell_flux_err_over_max_cell": float(np.abs(f32[0] - f64[0]).max() / scale),
            "max_cell_eta_err_over_max_cell": float(np.abs(f32[1] - f64[1]).max() / scale),
            "flux_total_rel_err": float(abs(f32[2] - f64[2]) / f64[2])}
    # the direct-solver path's two-pass full saddle assembly on the same mesh (not part of
    # the step): pattern + numeric pass, then the numeric pass alone on the cached pattern
    two_pass = None
    if args.p in (1, 2):
        keep = _Keep()
        desc = make_desc(dprob, 1e-15, -1.0, keep)
        cache = C.c_void_p()
        ctx.check(lib.apf_two_pass_cache_create(ctx.handle, C.byref(cache)))
        times = []
        for _ in range(3):
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            h2 = C.c_void_p()
            ctx.check(lib.apf_assemble_full_saddle_two_pass(ctx.handle, C.byref(desc), 1, cache, C.byref(h2)))
            t1.record(stream)
            torch.cuda.synchronize(dev)
            times.append(t0.elapsed_time(t1))
            r2, c2, n2 = C.c_int32(), C.c_int32(), C.c_int64()
            ctx.check(lib.apf_system_block_info(h2, _lib.BLOCKS["K"], C.byref(r2), C.byref(c2), C.byref(n2)))
            lib.apf_system_destroy(h2)
        nb, nr, ne = C.c_int64(), C.c_int64(), C.c_int64()
        ctx.check(lib.apf_two_pass_cache_stats(cache, C.byref(nb), C.byref(nr), C.byref(ne)))
        lib.apf_two_pass_cache_destroy(cache)
        two_pass = {"pattern_and_numeric_ms": round(times[0], 3),
                    "numeric_on_cached_pattern_ms": round(min(times[1:]), 3),
                    "pattern_entries": ne.value, "K_nnz_after_prune": n2.value,
                    "pattern_builds": nb.value, "pattern_reuse_count": nr.value}
    m = MainSystemBlocks(ctx, h, host)
    nnz_k = m.block_info("K")[2]
    nnz_h = m.block_info("Hhat")[2]
    m.close()
    peak, peak_kind = measured_peaks()
    # K SpMV inside MINRES: CSR values + column indices + row pointers once, x read once,
    # y written once
    spmv_bytes = 12.0 * nnz_k + 4.0 * (n_dofs + 1) + 16.0 * n_dofs
    spmv_launches, spmv_ms = kernels.get("minres_spmv_K", [1, float("nan")])
    spmv_achieved = spmv_bytes / (spmv_ms / 1e3 / spmv_launches) / 1e9
    # finest-level damped-Jacobi sweep of the two V-cycles (f32 values + int32 columns per
    # nonzero; x gathered once, b, the smoother weights and the new iterate per row); both
    # hierarchies run the same number of sweeps, so a launch averages the two operators
    sweep_bytes = None
    if amg_levels.get("A_y") and amg_levels.get("Hhat_F"):
        (ra, na, _), (rh, nh, _) = amg_levels["A_y"]["rows_nnz_nnzP"][0], amg_levels["Hhat_F"]["rows_nnz_nnzP"][0]
        sweep_bytes = 0.5 * ((8.0 * na + 32.0 * ra) + (8.0 * nh + 32.0 * rh))
    sweep_launches, sweep_ms = kernels.get("amg_sweep_l0", [1, float("nan")])
    sweep_achieved = sweep_bytes / (sweep_ms / 1e3 / sweep_launches) / 1e9 if sweep_bytes else None
    dominant = max(kernels.items(), key=lambda kv: kv[1][1])
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        info_cpu = cpu_reference_sample(args, 1, threads)
        if info_cpu:
            cpu = {"value": info_cpu["n_dofs"] / info_cpu["stages_s"], "unit": UNIT, "cores": info_cpu["threads"],
                   "kind": "reference", "sample": sample_text(info_cpu, sample_level_for(args.level))}
    total_ms = sum(v[1] for v in kernels.values())
    spmv_roof = {"kernel": "minres_spmv_K", "bound": "hbm", "achieved": spmv_achieved, "peak": peak, "unit": "GB/s",
                 "frac": spmv_achieved / peak, "peak_kind": peak_kind,
                 "algorithmic_bytes_per_launch": spmv_bytes, "launches_per_step": spmv_launches,
                 "share": spmv_ms / total_ms if total_ms else None,
                 "traffic": K_SPMV_TRAFFIC_RATIO * spmv_bytes,
                 "traffic_source": "DRAM bytes per launch of the K SpMV measured by ncu on the locally refined workload at "
                                   "outer level 5 (1.030 x its algorithmic bytes) times this launch's "
                                   "algorithmic bytes"}
    rooflines = [spmv_roof]
    if sweep_achieved:
        rooflines.insert(0, {
            "kernel": "amg_sweep_l0", "bound": "hbm", "achieved": sweep_achieved, "peak": peak, "unit": "GB/s",
            "frac": sweep_achieved / peak, "peak_kind": peak_kind,
            "algorithmic_bytes_per_launch": sweep_bytes, "launches_per_step": sweep_launches,
            "share": sweep_ms / total_ms if total_ms else None,
            "traffic": (SWEEP_L0_TRAFFIC_RATIO * sweep_bytes) if SWEEP_L0_TRAFFIC_RATIO else None,
            "traffic_source": ("DRAM bytes per launch of the finest-level sweeps measured by ncu on the locally refined "
                               "workload at outer level 5 (0.987 x their algorithmic bytes), times this "
                               "launch's algorithmic bytes")
            if SWEEP_L0_TRAFFIC_RATIO else "not captured"})
    # the line's roofline is the dominant kernel's when its byte model is known
    by_name = {r["kernel"]: r for r in rooflines}
    roofline_main = dict(by_name.get(dominant[0], spmv_roof))
    roofline_main["dominant_kernel"] = dominant[0]
    roofline_main["dominant_share"] = dominant[1][1] / total_ms if total_ms else None
    roofline_main["timing"] = ("per-launch CUDA events on the launching stream in one extra step with the two "
                               "V-cycles serialised (no overlap between their launches)")
    line = {
        "metric": METRIC,
        "value": args.steps * n_dofs * world / elapsed,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": workload_text(args),
                   "mesh": {"prisms": ny, "dofs": n_dofs, "n_lambda": host.n_lambda, "n_u": host.n_u,
                            "hanging_x_rows": int((np.diff(host.x_restriction.offsets) > 1).sum()),
                            **({k: host.meta[k] for k in ("point", "intervals", "spatial_triangles")}
                               if args.workload == "refined" else {})},
                   "stages": ["assembly", "graph_norm", "amg_setup", "minres"] +
                             (["slab_reconstruction", "patch_fluxes", "indicators", "x_indicators"]
                              if run_estimator else []),
                   "tolerance": args.tol,
                   "amg_aggressive_levels": sopt.amg_aggressive_levels,
                   "amg_smooth_steps": sopt.amg_smooth_steps, "amg_strength": sopt.amg_strength,
                   "preconditioner": ("learned smoother weights in the blkdiag(A_y, Hhat) SA-AMG V-cycles "
                                      "(plain fallback)" if plain else
                                      "plain: blkdiag(A_y, Hhat) by SA-AMG V-cycles"),
                   "learned_fallbacks": sum(d["learned_fallback"] for d in timed_diags),
                   "minres_solve_s_mean": sum(d["solve_seconds"] for d in timed_diags) / len(timed_diags),
                   "plain_preconditioner": plain,
                   "patch_precision_fp32_refined_vs_fp64": patch_precision,
                   "two_pass_full_saddle_assembly": two_pass,
                   "patch_launch_autotune": json.loads(lib.apf_ctx_autotune_report(ctx.handle).decode() or "{}"),
                   "minres_iterations": [d["iterations"] for d in timed_diags],
                   "step_ms": step_ms,
                   "step_stage_wall_ms": stage_ms,
                   "e2e_step_ms": e2e_step_ms,
                   "e2e_step_stage_wall_ms": e2e_stage_ms[-1] if e2e_stage_ms else None,
                   "final_true_residual_max": max(d["final_true_residual"] for d in timed_diags),
                   "e2e_final_true_residual_max": max(d["final_true_residual"] for d in e2e_diags),
                   "flux_squared": timed_est[-1]["flux_squared"] if timed_est else None,
                   "x_eta_squared": timed_est[-1]["x_eta_squared"] if timed_est else None,
                   "n_patches": timed_est[-1]["n_patches"] if timed_est else None,
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (mesh inputs %.0f MB; K %d nnz, Hhat %d nnz)" % (h2d_bytes / 1e6, nnz_k,
                                                                                               nnz_h)},
        "learned_vs_plain": None if plain is None else {
            "learned_ms_per_step": 1e3 * elapsed / args.steps, "plain_ms_per_step": plain["ms_per_step"],
            "step_speedup": plain["ms_per_step"] / (1e3 * elapsed / args.steps),
            "plain_converged": plain["converged"], "plain_max_iterations": plain["max_iterations"],
            "minres_iterations_learned": [d["iterations"] for d in timed_diags],
            "minres_iterations_plain": plain["minres_iterations"],
            "minres_solve_s_learned": sum(d["solve_seconds"] for d in timed_diags) / len(timed_diags),
            "minres_solve_s_plain": plain["minres_solve_s_mean"]},
        "e2e": {"value": n_e2e * n_dofs * world / e2e_elapsed, "unit": UNIT, "steps": n_e2e,
                "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes},
        "gpu_launches": launches,
        "roofline": roofline_main,
        "rooflines": rooflines,
        "kernel_times_ms_per_step": {k: round(v[1], 3) for k, v in
                                     sorted(kernels.items(), key=lambda kv: -kv[1][1])[:45]},
        "kernel_launches_per_step": {k: v[0] for k, v in sorted(kernels.items(), key=lambda kv: -kv[1][1])[:45]},
        "amg_levels": amg_levels,
        "kernel_ms_sum_per_step": round(total_ms, 3),
        "host_wall_ms_per_step": host_ranges,
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))


# dram__bytes_read.sum + dram__bytes_write.sum of the MINRES K SpMV per launch divided by its
# algorithmic bytes (12 nnz + 4 (n+1) + 16 n), from one ncu capture of the locally refined
# workload at outer level 5 (K: 661,835 rows, 16,645,725 nonzeros, 212.99 MB algorithmic;
# two launches moved 219.54 and 219.39 MB)
K_SPMV_TRAFFIC_RATIO = 1.030
# the same for the finest-level V-cycle sweeps (paired f32 SELL layout), on the locally
# refined workload at outer level 5 (kappa on 4 x 4 blocks, strength 0.003): six launches on
# A_y's finest operator (440,678 rows / 4,523,756 nonzeros, 50.29 MB algorithmic) moved
# 49.18 MB each, nine on Hhat_F's (221,157 rows / 3,493,345 nonzeros, 35.02 MB) 36.24 MB
# each: 1.001 of the algorithmic bytes (8 nnz + 32 rows) for one launch of each (the even
# slice widths add the padding; the new iterates mostly stay in L2)
SWEEP_L0_TRAFFIC_RATIO = 1.001


def main():
    args = parse()
    world, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    run_ours(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
