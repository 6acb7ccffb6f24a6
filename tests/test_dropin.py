"""The compiled C++ drop-in (include/apf_b200_backend.hpp) inside the reference's own callers.

tests/dropin/_build/apf_dropin_test is built by __graft_entry__.build() (tests/dropin/Makefile)
from the reference's templates where the reference source tree is present, and travels with the
repository.  It runs, with la::b200::Backend and with the reference's Eigen backend side by side:
assemble_main_system_blocks + assemble_parabolic_graph_norm_approximation ("blocks"),
assemble_and_solve_into_functions with MINRES + ParabolicGraphNorm ("solve"), and the reference's
inner loop compute_adaptive_test_space_iteration + refine_test_space_from_marked_source_cells
("cycle": device assembly, graph-norm block and MINRES under the reference's host estimator,
marking and refinement).  Bars: block patterns bit-exact, values 1e-12 (Hhat on adaptive meshes:
the significant pattern, cancellation residues below 1e-13 may differ); the solve's FP64 true
residual (on the host, with the Eigen backend's K) within its tolerance and its solution within
1e-6 of the direct solution; per adaptive pass the same estimator total to 1e-8 and the same
marked cells as the Eigen backend with its direct solver.
"""
import json
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
PROGRAM = os.path.join(HERE, "dropin", "_build", "apf_dropin_test")

# X refined at two space-time points (hanging nodes) and kappa per X cell, as in the
# adaptive fixtures
ADAPTIVE_ENV = {"APF_REF_X_POINTS": "0.3,0.6,0.4;0.7,0.25,0.8", "APF_REF_X_ROUNDS": "2",
                "APF_REF_KAPPA": "7:0.01:100"}

needs_program = pytest.mark.skipif(not os.path.exists(PROGRAM),
                                   reason="drop-in test program not built (needs the reference source tree)")


def _run(args, env=None, timeout=900):
    e = dict(os.environ)
    for k in ADAPTIVE_ENV:
        e.pop(k, None)
    # the reference's host code single-threaded: its multi-threaded reductions round
    # differently from run to run, and a Doerfler tie broken the other way refines another
    # mesh with the same DOF counts (seen in the adaptive-driver comparison)
    e["OMP_NUM_THREADS"] = "1"
    e.update(env or {})
    r = subprocess.run([PROGRAM, *map(str, args)], capture_output=True, text=True, env=e, timeout=timeout)
    return r


def _json(r):
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@needs_program
def test_program_fails_loudly_without_a_device():
    """On a machine without a CUDA device the drop-in reports the context error; nothing falls
    back to the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    r = _run(["blocks", 1, 1, "smooth_initial"])
    assert r.returncode == 1
    assert "apf_ctx_create failed" in r.stderr


def _assert_blocks(d, hhat_residue):
    for name in ("A_y", "B", "C_signed"):
        assert d[name]["pattern_mismatches"] == 0 and d[name]["nnz_ref"] == d[name]["nnz_b200"], (name, d[name])
        assert d[name]["max_abs_diff_over_max"] <= 1e-12, (name, d[name])
    hh = d["Hhat_residue_1e-13"] if hhat_residue else d["Hhat"]
    assert hh["pattern_mismatches"] == 0, hh
    assert d["Hhat"]["max_abs_diff_over_max"] <= 1e-12, d["Hhat"]
    assert d["f"] <= 1e-12 and d["g"] <= 1e-12, d


@needs_program
@pytest.mark.gpu
@pytest.mark.parametrize("p,levels,example", [(1, 2, "smooth_initial"), (2, 1, "smooth_initial"),
                                              (1, 2, "non_matching_initial")])
def test_dropin_blocks_match_eigen_backend(p, levels, example):
    d = _json(_run(["blocks", p, levels, example]))
    assert d["n_lambda"] > 0 and d["n_u"] > 0
    _assert_blocks(d, hhat_residue=False)


@needs_program
@pytest.mark.gpu
def test_dropin_blocks_on_adaptive_mesh_with_kappa():
    d = _json(_run(["blocks", 1, 2, "smooth_initial"], env=ADAPTIVE_ENV))
    _assert_blocks(d, hhat_residue=True)


@needs_program
@pytest.mark.gpu
@pytest.mark.parametrize("env", [None, ADAPTIVE_ENV], ids=["uniform", "adaptive_kappa"])
def test_dropin_solve_through_reference_caller(env):
    d = _json(_run(["solve", 1, 3, "smooth_initial", 1e-10], env=env))
    assert d["effective_solver_minres"] == 1 and d["iterative"] == 1 and d["converged"] == 1
    assert d["iterations"] > 0 and d["iterations"] == d["device_iterations"]
    assert d["host_true_residual"] <= 1e-10, d
    assert abs(d["reported_true_residual"] - d["host_true_residual"]) <= 1e-12 + 1e-6 * d["host_true_residual"], d
    assert d["max_diff_to_direct_over_max"] <= 1e-6, d


@needs_program
@pytest.mark.gpu
def test_dropin_adaptive_inner_loop_matches_eigen_backend():
    """Three passes of the reference's inner loop compute_adaptive_test_space_iteration (solve,
    estimate, Doerfler marking) + Y refinement on an adaptive X with kappa per cell: with
    la::b200::Backend the call resolves to the drop-in's overload (device assembly, MINRES to
    1e-12 and device estimate, the reference's own combination and marking), which gives the
    same totals (1e-8) and the same marked cells (up to ties at the threshold, at most 2% of
    them) as the reference's host path on the Eigen backend with its direct solve; both test
    spaces are refined by the direct run's marks, so every pass compares the same mesh."""
    d = _json(_run(["cycle", 1, 2, "smooth_initial", 3, 1e-12], env=ADAPTIVE_ENV))
    assert len(d["passes"]) == 3
    for pas in d["passes"]:
        assert pas["y_cells"][0] == pas["y_cells"][1], pas
        assert abs(pas["flux_b200"] - pas["flux_direct"]) <= 1e-8 * pas["flux_direct"], pas
        # the same marking, up to cells whose indicators tie at the Doerfler threshold
        assert pas["marked"][1] > 0 and pas["marked_symmetric_difference"] <= max(2, pas["marked"][1] // 50), pas
        assert pas["minres_iterations"] > 0 and pas["minres_true_residual"] <= 1e-12, pas
    # the later passes run on the refined (Y finer than X) test space
    assert d["passes"][2]["y_cells"][0] > d["passes"][1]["y_cells"][0] > d["passes"][0]["y_cells"][0]
    # every b200 pass estimated on the device (the drop-in's inner-iteration overload)
    assert d["device_estimates"] == 3


@needs_program
@pytest.mark.gpu
@pytest.mark.parametrize("guess", [0, 1, 2], ids=["cold", "initial_guess", "correction_equation"])
def test_dropin_reference_adaptive_driver_matches_eigen_backend(guess):
    """The reference's whole adaptive algorithm (run_adaptive_driver: inner Y loops, X marking
    and refinement) for three outer cycles with kappa per block (no ties in the marking): the
    b200 backend (device assembly, graph-norm block, MINRES to 1e-12) follows the same
    trajectory as the Eigen backend with its direct solver -- the same X and Y DOF counts and
    inner iteration counts every cycle, and the same estimator totals to 1e-8 -- with a cold
    start, with the previous solution as MINRES's initial guess, and with the correction
    equation K d = b - K x0 (the dispatcher's right-hand-side path)."""
    # kappa per square of a 4 x 4 partition (by position: the driver refines X, so a table
    # per initial X cell would not cover the new cells)
    d = _json(_run(["adaptive", 1, 1, "smooth_initial", 3, 1e-12, 1, guess],
                   env={"APF_REF_KAPPA": "11:0.1:10", "APF_REF_KAPPA_BLOCKS": "4"}))
    a, b = d["b200"], d["direct"]
    assert len(a) == len(b) == 3
    for ra, rb in zip(a, b):
        assert (ra["x_dofs"], ra["y_dofs"], ra["inner"]) == (rb["x_dofs"], rb["y_dofs"], rb["inner"]), (ra, rb)
        for key in ("eta_squared", "lambda_y_squared", "y_estimator_squared"):
            assert abs(ra[key] - rb[key]) <= 1e-8 * abs(rb[key]), (key, ra, rb)
    assert a[-1]["x_dofs"] > a[0]["x_dofs"]
    # every inner iteration of the b200 run estimated on the device
    assert d["device_estimates"] >= sum(r["inner"] for r in a)


@needs_program
@pytest.mark.gpu
def test_dropin_adaptive_driver_with_learned_preconditioner():
    """The same three-cycle driver comparison with the learned preconditioner loaded from the
    shipped raw parameters (la::b200::Session::use_learned_model; the plain block
    preconditioner as its fallback): the same trajectory as the Eigen backend's direct solves,
    totals to 1e-8, every solve on the device."""
    params = os.path.join(os.path.dirname(HERE), "doubleadapparabolicfem_b200", "data", "learned_precond.params.f32")
    d = _json(_run(["adaptive", 1, 1, "smooth_initial", 3, 1e-12, 1, 0],
                   env={"APF_REF_KAPPA": "11:0.1:10", "APF_REF_KAPPA_BLOCKS": "4",
                        "APF_DROPIN_LEARNED_PARAMS": params}))
    a, b = d["b200"], d["direct"]
    assert len(a) == len(b) == 3
    for ra, rb in zip(a, b):
        assert (ra["x_dofs"], ra["y_dofs"], ra["inner"]) == (rb["x_dofs"], rb["y_dofs"], rb["inner"]), (ra, rb)
        for key in ("eta_squared", "lambda_y_squared", "y_estimator_squared"):
            assert abs(ra[key] - rb[key]) <= 1e-8 * abs(rb[key]), (key, ra, rb)
    assert d["device_solves"] >= sum(r["inner"] for r in a)


@needs_program
@pytest.mark.gpu
@pytest.mark.parametrize("p,levels,env", [
    (1, 2, ADAPTIVE_ENV),
    (2, 1, {"APF_REF_X_POINTS": "0.3,0.6,0.4", "APF_REF_X_ROUNDS": "1", "APF_REF_KAPPA": "5:0.1:10"})],
    ids=["p1", "p2"])
def test_dropin_device_estimate_matches_reference_estimator(p, levels, env):
    """la::b200::estimate (apf_estimate on the drop-in's solve, returned in the reference's
    cellwise error types and combined by its own combination function) after one pass of the
    reference's inner loop, so Y is finer than X and Y cells span several slabs, against the
    reference's host estimator on its direct solve: per-cell flux^2, recon^2, eta^2 within
    1e-9 of the largest eta^2, totals 1e-10 (recon 1e-8), the same slab count, and the
    reference's Doerfler marking of the device estimate equal to its marking of its own (up
    to ties at the threshold)."""
    d = _json(_run(["estimate", p, levels, "smooth_initial", 1e-12], env=env))
    assert d["y_cells"] > d["x_cells"] and d["cells_compared"] == d["y_cells"], d
    assert d["n_slabs"][0] == d["n_slabs"][1], d
    for key in ("flux", "recon", "eta"):
        assert d["max_cell_diff_over_max_eta"][key] <= 1e-9, (key, d)
    (ea, eb), (fa, fb), (ra, rb) = d["eta_total"], d["flux_total"], d["recon_total"]
    assert abs(ea - eb) <= 1e-10 * eb and abs(fa - fb) <= 1e-10 * fb, d
    assert rb > 0 and abs(ra - rb) <= 1e-8 * rb, d
    assert d["marked"][1] > 0 and d["marked_symmetric_difference"] <= max(2, d["marked"][1] // 50), d


def _flux_samples(path):
    """flux_reconstruction_samples.bin (write_time_slab_flux_reconstruction_samples_binary.hpp:
    int32 header of 11, int32 slab / slab-cell / source ids, reference lattice, time samples,
    then [cell][sample][sigma_x, sigma_y, div sigma])."""
    raw = open(path, "rb").read()
    h = np.frombuffer(raw[:44], dtype=np.int32)
    n_cells, nt, nsp, per_cell = int(h[2]), int(h[6]), int(h[7]), int(h[8])
    off = 44
    ids = np.frombuffer(raw[off:off + 12 * n_cells], dtype=np.int32).reshape(3, n_cells)
    off += 12 * n_cells
    lattice = np.frombuffer(raw[off:off + 16 * nsp], dtype=np.float64)
    off += 16 * nsp
    times = np.frombuffer(raw[off:off + 8 * nt], dtype=np.float64)
    off += 8 * nt
    values = np.frombuffer(raw[off:], dtype=np.float64)
    assert values.size == n_cells * per_cell * 3
    return h, ids, lattice, times, values.reshape(n_cells, per_cell, 3)


@needs_program
@pytest.mark.gpu
@pytest.mark.parametrize("p,levels,env", [
    (1, 2, ADAPTIVE_ENV),
    (2, 1, {"APF_REF_X_POINTS": "0.3,0.6,0.4", "APF_REF_X_ROUNDS": "1", "APF_REF_KAPPA": "5:0.1:10"})],
    ids=["p1", "p2"])
def test_dropin_snapshot_flux_samples_match_reference_writer(p, levels, env, tmp_path):
    """The driver's time-slab estimator snapshot for a b200 iteration state (the overload of
    write_time_slab_estimator_diagnostics_snapshot: vertex patches by the reference's writer,
    flux samples from the device flux through apf_flux_sample) against the reference's own
    writer on the Eigen backend's state (host patch solves on its direct solve), after one
    pass of the inner loop so that Y cells span several slabs: the same header, slab / slab-cell
    / source ids and lattice, sigma_x, sigma_y and div sigma within 1e-8 of each component's
    largest magnitude, and byte-identical vertex-patch files."""
    d = _json(_run(["snapshot", p, levels, "smooth_initial", 1e-12, str(tmp_path)], env=env))
    assert d["y_cells"] > d["x_cells"] and d["n_slabs"][0] == d["n_slabs"][1] > 1, d
    ha, ia, la, ta, va = _flux_samples(tmp_path / "b200" / "flux_reconstruction_samples.bin")
    hb, ib, lb, tb, vb = _flux_samples(tmp_path / "eigen" / "flux_reconstruction_samples.bin")
    assert np.array_equal(ha, hb) and np.array_equal(ia, ib), (ha, hb)
    assert np.array_equal(la, lb) and np.array_equal(ta, tb)
    assert ha[2] > d["y_cells"]  # slab cells: Y cells cut at the slab times
    for comp in range(3):
        scale = np.abs(vb[..., comp]).max()
        assert scale > 0
        err = np.abs(va[..., comp] - vb[..., comp]).max() / scale
        assert err <= 1e-8, (comp, err)
    pa = (tmp_path / "b200" / "time_slab_vertex_patches.bin").read_bytes()
    pb = (tmp_path / "eigen" / "time_slab_vertex_patches.bin").read_bytes()
    assert len(pa) > 0 and pa == pb


@needs_program
@pytest.mark.gpu
@pytest.mark.parametrize("example", ["smooth_initial", "non_matching_initial"])
def test_dropin_1d_blocks_match_eigen_backend(example):
    """1+1D P1 (the CPU-runnable configuration's element): the reference's 1D example on its
    unit space-time mesh, two uniform levels; the drop-in's blocks equal the Eigen backend's."""
    d = _json(_run(["blocks", "1d", 2, example]))
    _assert_blocks(d, hhat_residue=False)


@needs_program
@pytest.mark.gpu
def test_dropin_1d_solve_and_inner_loop():
    """1+1D through the reference's callers: assemble_and_solve_into_functions (true residual
    1e-10 on the host, 1e-6 of the direct solution) and two passes of its inner loop (device
    estimate and the reference's marking against its host path, the same marks)."""
    d = _json(_run(["solve", "1d", 3, "smooth_initial", 1e-10]))
    assert d["converged"] == 1 and d["host_true_residual"] <= 1e-10 and d["max_diff_to_direct_over_max"] <= 1e-6, d
    c = _json(_run(["cycle", "1d", 2, "smooth_initial", 2, 1e-12]))
    for pas in c["passes"]:
        assert pas["y_cells"][0] == pas["y_cells"][1], pas
        assert abs(pas["flux_b200"] - pas["flux_direct"]) <= 1e-8 * pas["flux_direct"], pas
        assert pas["marked_symmetric_difference"] <= max(2, pas["marked"][1] // 50), pas
    assert c["device_estimates"] == 2
    e = _json(_run(["estimate", "1d", 3, "smooth_initial", 1e-12]))
    assert e["y_cells"] > e["x_cells"] and e["n_slabs"][0] == e["n_slabs"][1], e
    for key in ("flux", "recon", "eta"):
        assert e["max_cell_diff_over_max_eta"][key] <= 1e-9, (key, e)
