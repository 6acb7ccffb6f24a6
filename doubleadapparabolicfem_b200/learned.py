"""Learned MINRES preconditioner (no counterpart in the reference).

The reference preconditions MINRES with blkdiag(A_y, Hhat)^-1 by sparse Cholesky
(src/linear_algebra/eigen_backend/preconditioners/parabolic_graph_norm_minres.hpp:46-181);
this package applies one smoothed-aggregation V-cycle per block.  The learned variant
keeps the V-cycles and lets a small network choose their smoothing:

* per matrix row i of every non-coarsest AMG level, an MLP (8 -> 32 -> 32 -> 2, tanh) maps
  8 scale-free row features to y_i, and the damped-Jacobi weights become
  w_i^(o) = omega_l / a_ii * exp(0.5 tanh(y_i^(o))), o = 0 for the first pre-smoothing
  sweep and 1 for the later ones (post-smoothing runs them in reverse order);
* per block and level, alpha_l = 2 sigmoid(theta_l) scales the coarse correction.

Inference runs once per preconditioner set-up, in BF16 with FP32 accumulation on the
tensor cores.  Training minimises the energy-norm contraction of a few stationary V-cycle
iterations (after a burn-in that leaves the slowly contracting modes) on systems the method
itself assembles (seeded meshes with random piecewise-constant diffusivity), with the loss
gradient computed on the GPU by reverse mode through the V-cycles and the MLP (hand-written
FP32 forward / backward kernels); the optimiser step (Adam) runs on the host over the
1,442 parameters.  The plain block
preconditioner is the fallback (``apf_solve_minres`` reruns plain from the learned run's
iterate when the learned run misses the tolerance) and the judge (the FP64 true residual).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from .assembly import Context, MainSystemBlocks, _ptr
from .mesh import SpaceTimeProblem, uniform_problem

N_PARAMS = _lib.APF_LEARNED_NUM_PARAMS
N_FEATURES = 8
HIDDEN = 32
OUTPUTS = 2
MAX_LEVELS = 16
# flat parameter layout (apf_learned.cuh)
W1, B1 = 0, HIDDEN * N_FEATURES
W2 = B1 + HIDDEN
B2 = W2 + HIDDEN * HIDDEN
W3 = B2 + HIDDEN
B3 = W3 + OUTPUTS * HIDDEN
ALPHA = B3 + OUTPUTS

DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "learned_precond.npz")


def raw_params_path(npz_path: str):
    """The raw float32 copy of a saved model's parameters."""
    import pathlib
    p = pathlib.Path(npz_path)
    return p.with_name(p.name[:-4] + ".params.f32" if p.name.endswith(".npz") else p.name + ".params.f32")


class LearnedModel:
    """Parameters of the learned smoother model (host copy + library handle)."""

    def __init__(self, params: np.ndarray | None = None):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.apf_learned_model_create(C.byref(h))
        if rc != _lib.APF_OK:
            raise _lib.ApfError(rc, "apf_learned_model_create failed")
        self.handle = h
        self.set_params(np.zeros(N_PARAMS, np.float32) if params is None else params)

    def set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != N_PARAMS:
            raise ValueError(f"expected {N_PARAMS} parameters")
        rc = self.lib.apf_learned_model_set_params(self.handle, _ptr(p), N_PARAMS)
        if rc != _lib.APF_OK:
            raise _lib.ApfError(rc, "apf_learned_model_set_params failed")
        self.params = p.copy()

    @staticmethod
    def initial(seed: int = 0, scale: float = 0.3) -> "LearnedModel":
        """Small random hidden weights, zero output layer and alpha logits: starts at the plain
        preconditioner (w = omega / a_ii, alpha = 1) with non-zero gradients."""
        rng = np.random.default_rng(seed)
        p = np.zeros(N_PARAMS, np.float32)
        p[W1:B1] = rng.normal(0, scale, HIDDEN * N_FEATURES)
        p[W2:B2] = rng.normal(0, scale / np.sqrt(HIDDEN / N_FEATURES), HIDDEN * HIDDEN)
        p[W3:B3] = rng.normal(0, 1e-3, OUTPUTS * HIDDEN)
        return LearnedModel(p)

    def save(self, path: str, **meta):
        """The model as an npz (parameters and training metadata) and, beside it, the
        parameters alone as raw little-endian float32 (<path without .npz>.params.f32) for
        C and C++ callers (la::b200::Session::use_learned_model)."""
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.params, **{k: np.asarray(v) for k, v in meta.items()})
        raw_params_path(path).write_bytes(np.asarray(self.params, dtype="<f4").tobytes())

    @staticmethod
    def load(path: str = DEFAULT_WEIGHTS) -> "LearnedModel":
        with np.load(path) as z:
            return LearnedModel(z["params"])

    def close(self):
        if getattr(self, "handle", None):
            self.lib.apf_learned_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def use_model(ctx: Context, model: LearnedModel | None):
    """Make ``model`` the one APF_PRECOND_LEARNED set-ups of ``ctx`` use (None clears)."""
    ctx.check(ctx.lib.apf_ctx_set_learned_model(ctx.handle, model.handle if model is not None else None))


def loss_and_grad(blocks: MainSystemBlocks, model: LearnedModel, samples: int = 4, steps: int = 3, seed: int = 0,
                  start_vectors: np.ndarray | None = None, with_grad: bool = True, burn_in: int = 0):
    """Training objective and its gradient on an assembled system with a set-up preconditioner."""
    ctx = blocks.ctx
    loss = C.c_double()
    grad = np.zeros(N_PARAMS, np.float32) if with_grad else None
    sv = None if start_vectors is None else np.ascontiguousarray(start_vectors, dtype=np.float64)
    ctx.check(ctx.lib.apf_learned_loss_and_grad(ctx.handle, blocks.handle, model.handle, samples, steps, burn_in,
                                                seed, _ptr(sv), 0, C.byref(loss), _ptr(grad)))
    return loss.value, grad


def forward(ctx: Context, model: LearnedModel, features: np.ndarray, precision: int = 1) -> np.ndarray:
    """MLP outputs [rows, 2] (precision 0: FP32 CUDA cores, 1: BF16 tensor cores)."""
    f = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, N_FEATURES)
    y = np.empty((f.shape[0], OUTPUTS), np.float32)
    ctx.check(ctx.lib.apf_learned_forward(ctx.handle, model.handle, f.shape[0], _ptr(f), _ptr(y), precision, 0))
    return y


@dataclass
class AmgLevelData:
    A: object            # scipy CSR
    P: object | None     # scipy CSR (None on the coarsest level)
    omega: float
    alpha: float
    weights: np.ndarray  # smoother weights in use [2, rows] (first sweep, later sweeps)
    features: np.ndarray # [rows, 8]


def amg_hierarchy(blocks: MainSystemBlocks, block: int):
    """The set-up V-cycle hierarchy of block 0 (A_y) or 1 (Hhat) as host arrays."""
    import scipy.sparse as sp
    ctx = blocks.ctx
    lib = ctx.lib
    levels, dense, sweeps, smooth = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    ctx.check(lib.apf_amg_info(ctx.handle, blocks.handle, block, C.byref(levels), C.byref(dense), C.byref(sweeps),
                               C.byref(smooth)))
    out = []
    for l in range(levels.value):
        rows, nnz_a, nnz_p = C.c_int(), C.c_int64(), C.c_int64()
        omega, alpha = C.c_double(), C.c_double()
        ctx.check(lib.apf_amg_level_info(ctx.handle, blocks.handle, block, l, C.byref(rows), C.byref(nnz_a),
                                         C.byref(nnz_p), C.byref(omega), C.byref(alpha)))
        n = rows.value

        def fetch(which, nnz, ncols):
            rp = np.empty(n + 1, np.int32)
            ci = np.empty(nnz, np.int32)
            va = np.empty(nnz, np.float64)
            ctx.check(lib.apf_amg_level_copy(ctx.handle, blocks.handle, block, l, which, _ptr(rp), _ptr(ci), _ptr(va)))
            return sp.csr_matrix((va, ci, rp), shape=(n, ncols))

        A = fetch(0, nnz_a.value, n)
        w = np.empty((2, n))
        for o in range(2):
            ctx.check(lib.apf_amg_level_weights(ctx.handle, blocks.handle, block, l, o, _ptr(w[o])))
        f = np.empty((n, N_FEATURES), np.float32)
        ctx.check(lib.apf_amg_level_features(ctx.handle, blocks.handle, block, l, _ptr(f)))
        out.append(AmgLevelData(A=A, P=None, omega=omega.value, alpha=alpha.value, weights=w, features=f))
        out[-1]._nnz_p = nnz_p.value
    for l in range(levels.value - 1):
        nc = out[l + 1].A.shape[0]
        n = out[l].A.shape[0]
        rp = np.empty(n + 1, np.int32)
        ci = np.empty(out[l]._nnz_p, np.int32)
        va = np.empty(out[l]._nnz_p, np.float64)
        ctx.check(lib.apf_amg_level_copy(ctx.handle, blocks.handle, block, l, 1, _ptr(rp), _ptr(ci), _ptr(va)))
        out[l].P = sp.csr_matrix((va, ci, rp), shape=(n, nc))
    info = {"levels": levels.value, "dense_coarse": bool(dense.value), "coarse_sweeps": sweeps.value,
            "smooth_steps": smooth.value}
    return out, info


# ---------------------------------------------------------------------------------------
# method-generated training systems
# ---------------------------------------------------------------------------------------

def random_kappa_problem(level: int, seed: int, blocks_per_side: int = 8, kappa_range=(0.01, 100.0),
                         p: int = 1) -> SpaceTimeProblem:
    """Uniform outer-level ``level`` mesh with diffusivity kappa piecewise constant on a
    blocks_per_side^2 spatial partition of (0,1)^2 (constant in time), log-uniform in
    kappa_range; M = kappa I per cell."""
    rng = np.random.default_rng(seed)
    base = uniform_problem(level, p)
    geo = base.y_geometry
    cx = (geo[:, 0] + geo[:, 2] + geo[:, 4]) / 3.0
    cy = (geo[:, 1] + geo[:, 3] + geo[:, 5]) / 3.0
    ib = np.minimum((cx * blocks_per_side).astype(int), blocks_per_side - 1)
    jb = np.minimum((cy * blocks_per_side).astype(int), blocks_per_side - 1)
    lo, hi = np.log(kappa_range[0]), np.log(kappa_range[1])
    kap = np.exp(rng.uniform(lo, hi, (blocks_per_side, blocks_per_side)))[jb, ib]
    m = np.zeros((geo.shape[0], 3))
    m[:, 0] = kap
    m[:, 2] = kap
    return uniform_problem(level, p, m_cells=m)


class Adam:
    def __init__(self, n: int, lr: float = 3e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        self.m = np.zeros(n)
        self.v = np.zeros(n)
        self.t = 0
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps

    def step(self, params: np.ndarray, grad: np.ndarray) -> np.ndarray:
        self.t += 1
        g = grad.astype(np.float64)
        self.m = self.b1 * self.m + (1 - self.b1) * g
        self.v = self.b2 * self.v + (1 - self.b2) * g * g
        mh = self.m / (1 - self.b1 ** self.t)
        vh = self.v / (1 - self.b2 ** self.t)
        return (params - self.lr * mh / (np.sqrt(vh) + self.eps)).astype(np.float32)


def train(ctx: Context, systems, model: LearnedModel, epochs: int = 10, lr: float = 3e-3, samples: int = 4,
          steps: int = 3, seed: int = 0, log=None, train_alpha: bool = False, burn_in: int = 0):
    """Adam on the mean loss over ``systems`` (assembled MainSystemBlocks with set-up
    preconditioners).  Returns the per-epoch mean losses.

    The coarse-correction scales stay frozen unless ``train_alpha``: the stationary
    contraction rewards over-correction (alpha > 1), which lowers the contraction of the
    slow modes but stretches the spectrum MINRES sees and costs iterations."""
    opt = Adam(N_PARAMS, lr=lr)
    history = []
    params = model.params.copy()
    for ep in range(epochs):
        losses = []
        for k, blocks in enumerate(systems):
            loss, grad = loss_and_grad(blocks, model, samples=samples, steps=steps, seed=seed + 1000 * ep + k,
                                       burn_in=burn_in)
            if not train_alpha:
                grad[ALPHA:] = 0.0
            losses.append(loss)
            params = opt.step(params, grad)
            model.set_params(params)
        history.append(float(np.mean(losses)))
        if log:
            log(f"epoch {ep}: mean loss {history[-1]:.5f}")
    return history


def refined_training_problem(k: int, levels=(3, 4)):
    """The k-th locally refined training system: outer level from `levels`, 3 to 5 levels of
    bisection near a seeded point, diffusivity log-uniform in [0.01, 100] on 4x4 or 8x8 blocks
    (refine.locally_refined_problem; 30k-250k DOFs)."""
    from .refine import locally_refined_problem
    level = levels[k % len(levels)]
    return locally_refined_problem(level=level, seed=20_000 + k, depth=3 + k % 3, radius0=0.2,
                                   time_rounds=1 + k % 2, kappa_blocks=4 if (k // 2) % 2 else 8)


def train_default_model(out_path: str = DEFAULT_WEIGHTS, n_train: int = 24, levels=(3, 4), epochs: int = 40,
                        lr: float = 1e-2, seed: int = 0, device: int = 0, log=print, steps: int = 4,
                        burn_in: int = 8, n_refined: int = 0, refined_strength: float | None = None):
    """Train the shipped model on method-generated systems: uniform meshes of the given outer
    levels with seeded random piecewise-constant diffusivity (log-uniform in [0.01, 100] on
    4x4 or 8x8 blocks), the constant-diffusivity mesh of each level, and n_refined locally
    refined systems with such a diffusivity (refined_training_problem).  The AMG hierarchies
    the model is trained on are built with the library's default options, those of the
    refined systems with strength threshold ``refined_strength`` when given."""
    from .assembly import assemble_main_system_blocks
    from .solver import SolverOptions, setup_preconditioner
    ctx = Context(device)
    systems = []
    for k in range(n_train):
        level = levels[k % len(levels)]
        prob = random_kappa_problem(level, seed=10_000 + k, blocks_per_side=4 if k % 2 else 8)
        systems.append(prob)
    systems += [uniform_problem(level, 1) for level in levels]
    systems += [refined_training_problem(k, levels) for k in range(n_refined)]
    blocks = []
    n_plain = len(systems) - n_refined
    for k, prob in enumerate(systems):
        b = assemble_main_system_blocks(prob, ctx=ctx)
        b.assemble_parabolic_graph_norm_approximation()
        opts = SolverOptions()
        if k >= n_plain and refined_strength is not None:
            opts.amg_strength = refined_strength
        setup_preconditioner(b, opts)
        blocks.append(b)
    model = LearnedModel.initial(seed)
    hist = train(ctx, blocks, model, epochs=epochs, lr=lr, samples=2, steps=steps, seed=seed, log=log,
                 burn_in=burn_in)
    model.save(out_path, history=np.asarray(hist), levels=np.asarray(levels), n_train=n_train, epochs=epochs,
               steps=steps, burn_in=burn_in, n_refined=n_refined,
               refined_strength=-1.0 if refined_strength is None else refined_strength)
    return model, hist


def evaluate(level: int = 6, seeds=(1, 2), tol: float = 1e-8, device: int = 0, blocks_per_side: int = 8):
    """Learned vs plain block preconditioner on held-out systems of the learned-preconditioner
    configuration: uniform outer level ``level`` with seeded piecewise-constant diffusivity
    log-uniform in [0.01, 100] on blocks_per_side^2 blocks, MINRES to the FP64 true residual
    ``tol``.  Returns one record per system (iterations, solve seconds, true residuals)."""
    from .assembly import assemble_main_system_blocks
    from .solver import SolverOptions, solve_saddle_system_with_preconditioner
    ctx = Context(device)
    model = LearnedModel.load()
    use_model(ctx, model)
    out = []
    for seed in seeds:
        prob = random_kappa_problem(level, seed=seed, blocks_per_side=blocks_per_side)
        rec = {"level": level, "seed": seed, "dofs": prob.n_lambda + prob.n_u}
        for name, prec in (("plain", "amg_block"), ("learned", "learned")):
            b = assemble_main_system_blocks(prob, ctx=ctx)
            b.assemble_parabolic_graph_norm_approximation()
            solve_saddle_system_with_preconditioner(b, SolverOptions(tolerance=tol, preconditioner=prec),
                                                    copy_out=False)  # warm-up (set-up, graphs)
            _, d = solve_saddle_system_with_preconditioner(b, SolverOptions(tolerance=tol, preconditioner=prec),
                                                           copy_out=False)
            rec[name] = {"iterations": d["iterations"], "solve_s": d["solve_seconds"],
                         "true_residual": d["final_true_residual"], "fallback": d["learned_fallback"]}
            b.close()
        rec["iteration_gain"] = rec["plain"]["iterations"] / max(1, rec["learned"]["iterations"])
        rec["time_gain"] = rec["plain"]["solve_s"] / rec["learned"]["solve_s"]
        out.append(rec)
    return out


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="train the learned MINRES preconditioner on method-generated systems")
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--n-train", type=int, default=24)
    ap.add_argument("--levels", default="3,4")
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--lr", type=float, default=1e-2)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--burn-in", type=int, default=8)
    ap.add_argument("--refined", type=int, default=0, help="locally refined high-contrast systems added to the set")
    ap.add_argument("--refined-strength", type=float, default=None,
                    help="AMG strength threshold of the refined systems' hierarchies (default: the library's)")
    ap.add_argument("--evaluate", type=int, default=None, metavar="LEVEL",
                    help="instead of training: learned vs plain on seeded random-kappa systems of this level")
    a = ap.parse_args()
    if a.evaluate is not None:
        import json
        print(json.dumps(evaluate(a.evaluate)))
        raise SystemExit(0)
    train_default_model(a.out, a.n_train, tuple(int(x) for x in a.levels.split(",")), a.epochs, a.lr, a.seed,
                        steps=a.steps, burn_in=a.burn_in, n_refined=a.refined, refined_strength=a.refined_strength)
