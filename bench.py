"""Benchmark: one adaptive-cycle hot path of the 2+1D space-time heat problem on B200.

Workload (default): 2+1D heat equation on (0,1)^2 x (0,1), u0 = sin(pi x) sin(pi y),
f = 0, M = I, uniform space-time prism mesh of outer level 6 (2,097,152 prisms,
n_lambda = 2,064,512, n_u = 1,048,385: 3,112,897 space-time DOFs), P1, FP64.
Synthetic input: the mesh and DOF maps are generated on the host
(doubleadapparabolicfem_b200.mesh.uniform_problem), with the reference's cell
geometry and DOF counts.

A step = the hot path over one mesh: main-system assembly (A_y, B, B^T, C_signed,
K, f, g) and the parabolic graph-norm preconditioner block Hhat, from inputs already
in HBM.  ``e2e`` = the same through the C ABI from pinned host buffers (H2D of the
mesh inputs and D2H of the right-hand sides inside the timed region).

Multi-GPU: the path runs one problem per GPU (replicas; no collective in the data
path).  ``value`` = total DOFs processed by all ranks / max-over-ranks time.

``--impl reference`` times the reference's own CPU implementation of the path
(oracle/_ref/apf_ref_dump: the reference templates compiled here) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "2+1D adaptive-cycle DOFs/s at 1e-8 residual; learned vs plain precond on B200"
UNIT = "DOFs/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--level", type=int, default=6)
    ap.add_argument("--p", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tol", type=float, default=1e-8)
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if len(s) > 5 + k and s[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_reference_sample(level: int, p: int, reps: int, threads: int | None = None):
    """Time the reference's own CPU path (oracle/_ref) on a bounded sample."""
    exe = os.path.join(REPO, "oracle", "_ref", "apf_ref_dump")
    if not os.path.exists(exe):
        return None
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    out = subprocess.run([exe, "bench", str(p), str(level), "smooth_initial", str(reps)], capture_output=True, text=True,
                         env=env, timeout=900)
    if out.returncode != 0:
        return None
    return json.loads(out.stdout.strip().splitlines()[-1])


def run_reference(args, world, rank):
    # rank 0 alone times the reference CPU path; other ranks do no work
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    # bounded sample of the workload: the same mesh family one outer level coarser
    # (1/8 of the cells), which keeps each step to a few seconds of CPU time
    sample_level = max(1, args.level - 1)
    exe = os.path.join(REPO, "oracle", "_ref", "apf_ref_dump")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/apf_ref_dump was not built (needs the reference sources)"}))
        return
    for _ in range(args.warmup):
        cpu_reference_sample(sample_level, args.p, 1, threads)
    times = []
    info = None
    for _ in range(args.steps):
        info = cpu_reference_sample(sample_level, args.p, 1, threads)
        times.append(info["mean_s"])
    t = sum(times)
    value = args.steps * info["n_dofs"] / t
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"2+1D heat, uniform outer level {args.level} P{args.p} mesh (sampled at level {sample_level})",
                   "stages": ["assembly", "graph_norm"]},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"outer level {sample_level} ({info['n_cells']} prisms, {info['n_dofs']} DOFs) per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def fill_kernel_bytes(problem, blocks_info):
    """Algorithmic bytes of the gather_rows_fill launches of one step: each launch reads
    its incidence list and the geometry / restriction rows of the incident cells once
    and writes its CSR block once."""
    ndof = problem.ndof
    ny, nx = problem.n_y_cells, problem.n_x_cells
    geo = 64
    restr = ndof * (4 + 4 + 8)          # offsets + dofs + weights per cell
    total = 0
    for name, (rows, cols, nnz, cells) in blocks_info.items():
        total += nnz * 12 + (rows + 1) * 4          # CSR written
        total += (rows + 1) * 4 + cells * ndof * 8  # incidence lists read
        total += cells * (geo + restr)              # cell data read
    return total


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    from doubleadapparabolicfem_b200 import build as b
    from doubleadapparabolicfem_b200 import _lib
    from doubleadapparabolicfem_b200.assembly import Context, MainSystemBlocks, make_desc, _Keep
    from doubleadapparabolicfem_b200.mesh import uniform_problem, SpaceTimeProblem, Restriction
    import ctypes as C

    b.build()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.Stream(device=dev)
    ctx = Context(local, stream=stream.cuda_stream)
    lib = ctx.lib

    host = uniform_problem(args.level, args.p)
    n_dofs = host.n_lambda + host.n_u

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
            n_lambda=host.n_lambda, n_u=host.n_u, u0_kind=host.u0_kind)

    dprob = clone_problem(to_dev)
    hprob = clone_problem(to_pinned)
    h2d_bytes = sum(int(t.numel() * t.element_size()) for t in (
        hprob.y_geometry, hprob.x_geometry, hprob.y_to_x, hprob.y_restriction.offsets, hprob.y_restriction.dofs,
        hprob.y_restriction.weights, hprob.x_restriction.offsets, hprob.x_restriction.dofs, hprob.x_restriction.weights))
    x_out = torch.empty(n_dofs, dtype=torch.float64).pin_memory()
    d2h_bytes = n_dofs * 8
    sopt = _lib.SolverOptions()
    lib.apf_solver_options_default(C.byref(sopt))
    sopt.tolerance = args.tol
    solve_diags = []

    def step(prob, on_device, read_back):
        keep = _Keep()
        desc = make_desc(prob, 1e-15, -1.0, keep)
        h = C.c_void_p()
        ctx.check(lib.apf_assemble_main_system(ctx.handle, C.byref(desc), 1 if on_device else 0, C.byref(h)))
        ctx.check(lib.apf_assemble_graph_norm(ctx.handle, h, 1e-14))
        d = _lib.SolverDiagnostics()
        out = C.c_void_p(x_out.data_ptr()) if read_back else None
        ctx.check(lib.apf_solve_minres(ctx.handle, h, C.byref(sopt), None, out, 0, C.byref(d)))
        solve_diags.append({k: getattr(d, k) for k, _ in d._fields_})
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

    # warm-up
    for _ in range(args.warmup):
        lib.apf_system_destroy(step(dprob, True, False))
    ctx.synchronize()

    # timed device-resident steps, with per-kernel CUDA-event timing on the library's stream
    launches0 = ctx.kernel_launches()
    ctx.check(lib.apf_ctx_set_timing(ctx.handle, 1))
    barrier()
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            lib.apf_system_destroy(step(dprob, True, False))
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    barrier()
    launches = ctx.kernel_launches() - launches0
    report = json.loads(lib.apf_ctx_timing_report(ctx.handle).decode())
    ctx.check(lib.apf_ctx_set_timing(ctx.handle, 0))
    elapsed = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)

    # e2e through the C ABI from pinned host buffers
    barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        lib.apf_system_destroy(step(hprob, False, True))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    e2e_elapsed = max_over_ranks(e0.elapsed_time(e1) / 1e3)

    # roofline of the dominant kernel (algorithmic bytes per launch / event-timed duration)
    dominant = max(report.items(), key=lambda kv: kv[1][1])
    h = step(dprob, True, False)
    m = MainSystemBlocks(ctx, h, host)
    info = {}
    cells = {"A_y": host.n_y_cells, "BT": host.n_y_cells, "B": host.n_y_cells, "C_signed": host.n_x_cells // (2 ** args.level),
             "A_x": host.n_x_cells, "B_dt": host.n_y_cells}
    for name in ("A_y", "BT", "B", "C_signed", "A_x", "B_dt"):
        r, c, nnz = m.block_info(name)
        info[name] = (r, c, nnz, cells[name])
    info["B_dtT"] = (host.n_lambda, host.n_u, info["B_dt"][2], host.n_y_cells)
    nnz_k = m.block_info("K")[2]
    nnz_h = m.block_info("Hhat")[2]
    m.close()
    peak, peak_kind = measured_peaks()
    fill_bytes = fill_kernel_bytes(host, info)
    fill_launches, fill_ms = report.get("gather_rows_fill", [1, float("nan")])
    fill_achieved = (fill_bytes / 7.0) / (fill_ms / 1e3 / fill_launches) / 1e9
    # K SpMV inside MINRES: CSR values + column indices + row pointers once, x read once, y written once
    spmv_bytes = 12.0 * nnz_k + 4.0 * (n_dofs + 1) + 16.0 * n_dofs
    spmv_launches, spmv_ms = report.get("minres_spmv_K", [1, float("nan")])
    spmv_achieved = spmv_bytes / (spmv_ms / 1e3 / spmv_launches) / 1e9
    its = [d["iterations"] for d in solve_diags[-args.steps:]]
    res = [d["final_true_residual"] for d in solve_diags[-args.steps:]]
    rank0 = rank == 0
    if not rank0:
        return
    cpu = None
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample_level = max(1, args.level - 2)
        info_cpu = cpu_reference_sample(sample_level, args.p, 2, threads)
        if info_cpu:
            cpu = {"value": info_cpu["n_dofs"] / info_cpu["mean_s"], "unit": UNIT, "cores": info_cpu["threads"],
                   "kind": "reference",
                   "sample": f"reference CPU assembly + graph norm on outer level {sample_level} "
                             f"({info_cpu['n_cells']} prisms, {info_cpu['n_dofs']} DOFs), mean of 2 reps"}
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
        "config": {"workload": f"2+1D heat, u0=sin(pi x)sin(pi y), uniform outer level {args.level} P{args.p} "
                               f"({host.n_y_cells} prisms, {n_dofs} DOFs)",
                   "stages": ["assembly", "graph_norm", "amg_setup", "minres"],
                   "tolerance": args.tol,
                   "preconditioner": "blkdiag(A_y, Hhat) by SA-AMG V-cycles",
                   "minres_iterations": its, "final_true_residual_max": max(res),
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (mesh inputs %.0f MB, outputs K %d nnz, Hhat %d nnz)" % (h2d_bytes / 1e6, nnz_k, nnz_h)},
        "e2e": {"value": args.steps * n_dofs * world / e2e_elapsed, "unit": UNIT,
                "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes},
        "gpu_launches": launches,
        "roofline": {"kernel": "minres_spmv_K", "bound": "hbm", "achieved": spmv_achieved, "peak": peak, "unit": "GB/s",
                     "frac": spmv_achieved / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": spmv_bytes, "traffic": None,
                     "dominant_kernel": dominant[0],
                     "assembly_gather_rows_fill": {"achieved": fill_achieved, "frac": fill_achieved / peak,
                                                   "algorithmic_bytes_per_launch": fill_bytes / 7.0}},
        "kernel_times_ms": {k: round(v[1] / args.steps, 4) for k, v in sorted(report.items(), key=lambda kv: -kv[1][1])},
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))


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
