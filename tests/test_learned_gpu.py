"""GPU tests of the learned MINRES preconditioner (no counterpart in the reference).

* the BF16 tensor-core forward pass against the FP32 pass and the FP64 oracle
  (bar: FP32 within 1e-4 of the oracle; BF16 within 3e-2 of the largest |y|: BF16 operands
  carry 8 mantissa bits);
* the row features against the oracle (FP32 storage: 1e-6 relative);
* the training loss (1e-6 relative) and its reverse-mode gradient on every parameter (the
  FP64 oracle's exact reverse-mode gradient, 1e-5 of the largest component) on an exported
  hierarchy;
* the trained model shipped with the package against the plain block preconditioner on
  held-out systems: fewer MINRES iterations to the same FP64 true residual;
* the fallback: a deliberately poor model that misses the tolerance is rerun plain.
"""
import os

import numpy as np
import pytest

import learned_oracle as O

pytestmark = pytest.mark.gpu


def _system(ctx, prob, coarse=64):
    from doubleadapparabolicfem_b200.assembly import assemble_main_system_blocks
    from doubleadapparabolicfem_b200.solver import SolverOptions, setup_preconditioner
    b = assemble_main_system_blocks(prob, ctx=ctx)
    b.assemble_parabolic_graph_norm_approximation()
    setup_preconditioner(b, SolverOptions(amg_coarse_size=coarse))
    return b


def _solve(ctx, blocks, prec, model=None, tol=1e-8, max_iterations=20000, coarse=64):
    from doubleadapparabolicfem_b200 import learned as LM
    from doubleadapparabolicfem_b200.solver import SolverOptions, solve_saddle_system_with_preconditioner
    if model is not None:
        LM.use_model(ctx, model)
    x, d = solve_saddle_system_with_preconditioner(
        blocks, SolverOptions(tolerance=tol, preconditioner=prec, max_iterations=max_iterations,
                              amg_coarse_size=coarse))
    return x, d


def _random_model(seed):
    from doubleadapparabolicfem_b200 import learned as LM
    m = LM.LearnedModel.initial(seed, scale=0.5)
    p = m.params.copy()
    rng = np.random.default_rng(seed + 1)
    p[LM.W3:LM.B3] = rng.normal(0, 0.3, LM.OUTPUTS * LM.HIDDEN)
    p[LM.B3:LM.ALPHA] = (0.1, -0.2)
    p[LM.ALPHA:] = rng.normal(0, 0.3, 2 * LM.MAX_LEVELS)
    m.set_params(p)
    return m


def test_forward_bf16_tensor_cores_vs_fp32_and_oracle(gpu_ctx):
    from doubleadapparabolicfem_b200 import learned as LM
    m = _random_model(3)
    F = np.random.default_rng(0).normal(0, 1, (1037, 8)).astype(np.float32)  # ragged tile count
    y32 = LM.forward(gpu_ctx, m, F, precision=0)
    y16 = LM.forward(gpu_ctx, m, F, precision=1)
    yo = O.mlp(m.params, F.astype(np.float64))
    scale = np.abs(yo).max()
    assert np.abs(y32 - yo).max() <= 1e-4 * max(1.0, scale)
    assert np.abs(y16 - yo).max() <= 3e-2 * max(1.0, scale)
    assert y16.shape == (1037, 2)
    assert LM.forward(gpu_ctx, m, F[:0], precision=1).size == 0


def test_row_features_match_oracle(gpu_ctx):
    from doubleadapparabolicfem_b200 import learned as LM
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    b = _system(gpu_ctx, uniform_problem(3, 1))
    for block in (0, 1):
        levels, info = LM.amg_hierarchy(b, block)
        assert info["levels"] >= 2
        for l in range(min(2, info["levels"])):
            ref = O.features(levels[l].A, l, block)
            got = levels[l].features.astype(np.float64)
            assert np.abs(got - ref).max() <= 1e-6 * max(1.0, np.abs(ref).max())


def test_loss_and_gradient_match_oracle(gpu_ctx):
    from doubleadapparabolicfem_b200 import learned as LM
    b = _system(gpu_ctx, LM.random_kappa_problem(2, seed=3, blocks_per_side=4), coarse=16)
    nl, nu = b.n_lambda(), b.n_u()
    model = _random_model(5)
    rng = np.random.default_rng(11)
    starts = rng.normal(0, 1, (2, nl + nu))
    steps = 2
    L_gpu, g_gpu = LM.loss_and_grad(b, model, samples=2, steps=steps, start_vectors=starts)
    hier = []
    for block in (0, 1):
        levels, info = LM.amg_hierarchy(b, block)
        assert info["levels"] >= 2 and info["smooth_steps"] == 2
        hier.append(O.Hierarchy([(lv.A, lv.P, lv.omega) for lv in levels], info["dense_coarse"],
                                info["coarse_sweeps"], block,
                                features_per_level=[lv.features.astype(np.float64) for lv in levels],
                                smooth_steps=info["smooth_steps"]))
    targets = [b.A_y(), b.block("Hhat")]
    S = [starts[:, :nl], starts[:, nl:]]
    params = model.params.astype(np.float64)
    L_or = O.loss(params, hier, targets, S, steps)
    assert abs(L_gpu - L_or) <= 1e-6 * max(1.0, abs(L_or)), (L_gpu, L_or)
    # every parameter against the exact FP64 reverse-mode gradient of the oracle's loss (with
    # the Gershgorin rescale factor held constant, as the device's backward pass treats it);
    # the device's MLP backward runs in FP32
    L64, g64 = O.loss_and_grad_fp64(params, hier, targets, S, steps)
    assert abs(L64 - L_or) <= 1e-12 * max(1.0, abs(L_or))
    g = g_gpu.astype(np.float64)
    err = np.abs(g - g64).max() / np.abs(g64).max()
    assert err <= 1e-5, err
    assert np.abs(g64).max() > 0


def test_shipped_model_beats_plain_on_held_out_systems(gpu_ctx):
    """What the trained model (data/learned_precond.npz, trained on outer levels 3-4) gains
    over the plain block preconditioner on systems it was not trained on, at the same FP64
    true residual: fewer MINRES iterations in total (geometric-mean gain > 1), and no system
    more than 5% worse."""
    from doubleadapparabolicfem_b200 import learned as LM
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    assert os.path.exists(LM.DEFAULT_WEIGHTS)
    model = LM.LearnedModel.load()
    gains = []
    for prob in (LM.random_kappa_problem(4, seed=90001), uniform_problem(4, 1), uniform_problem(5, 1),
                 LM.random_kappa_problem(5, seed=90002)):
        b = _system(gpu_ctx, prob, coarse=256)
        _, dp = _solve(gpu_ctx, b, "amg_block", coarse=256)
        _, dl = _solve(gpu_ctx, b, "learned", model, coarse=256)
        assert dp["converged"] == 1 and dl["converged"] == 1 and dl["learned_fallback"] == 0
        assert dl["final_true_residual"] <= 1e-8
        gains.append(dp["iterations"] / dl["iterations"])
        b.close()
    assert np.exp(np.mean(np.log(gains))) > 1.0 and min(gains) >= 0.95, gains


def test_shipped_model_is_faster_in_wall_time_on_a_high_contrast_system(gpu_ctx):
    """Wall time, not only iterations: on a held-out level-5 system with kappa contrast up to
    1e4 (the learned model saves ~20% of the iterations there) the learned solve, after a
    warm-up solve of each kind, is faster than the plain one (bar: 0.97x its time) at the
    same FP64 true residual."""
    from doubleadapparabolicfem_b200 import learned as LM
    model = LM.LearnedModel.load()
    b = _system(gpu_ctx, LM.random_kappa_problem(5, seed=90002), coarse=256)
    times = {}
    for prec in ("amg_block", "learned", "amg_block", "learned"):
        _, d = _solve(gpu_ctx, b, prec, model if prec == "learned" else None, coarse=256)
        assert d["converged"] == 1 and d["final_true_residual"] <= 1e-8
        times[prec] = (d["solve_seconds"], d["iterations"])   # the second solve of each kind stays
    b.close()
    (tp, ip), (tl, il) = times["amg_block"], times["learned"]
    assert il < ip, times
    assert tl < 0.97 * tp, times


def test_learned_solve_falls_back_to_plain(gpu_ctx):
    from doubleadapparabolicfem_b200 import learned as LM
    from doubleadapparabolicfem_b200.mesh import uniform_problem
    b = _system(gpu_ctx, uniform_problem(3, 1))
    _, dp = _solve(gpu_ctx, b, "amg_block")
    poor = np.zeros(LM.N_PARAMS, np.float32)
    poor[LM.ALPHA:] = -12.0  # alpha ~ 1e-5: the coarse corrections vanish
    _, dl = _solve(gpu_ctx, b, "learned", LM.LearnedModel(poor), max_iterations=dp["iterations"] + 20)
    assert dl["learned_fallback"] == 1 and dl["preconditioner_used"] == 0
    assert dl["converged"] == 1 and dl["final_true_residual"] <= 1e-8


def test_training_reduces_the_loss(gpu_ctx):
    from doubleadapparabolicfem_b200 import learned as LM
    systems = [_system(gpu_ctx, LM.random_kappa_problem(3, seed=s, blocks_per_side=4)) for s in (1, 2)]
    model = LM.LearnedModel.initial(0)
    hist = LM.train(gpu_ctx, systems, model, epochs=6, lr=1e-2, samples=2, steps=3)
    assert hist[-1] < hist[0]
