"""Host-side mirror of the reference's preconditioned saddle solve.

``solve_saddle_system_with_preconditioner(blocks, options)`` mirrors
``la::preconditioners::solve_saddle_system_with_preconditioner``
(src/linear_algebra/preconditioners/solve_saddle_system.hpp:94-111) as dispatched to
``solve_minres_with_parabolic_graph_norm`` for MINRES + ParabolicGraphNorm
(src/linear_algebra/eigen_backend/preconditioners/parabolic_graph_norm_minres.hpp:232-369):
it returns the solution [lambda; u] and the iterative diagnostics, and raises
``PreconditionedSolveFailure`` (carrying the diagnostics) when the FP64 true residual
misses the tolerance, as the reference throws at parabolic_graph_norm_minres.hpp:357-366.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .assembly import MainSystemBlocks, _ptr


@dataclass
class SolverOptions:
    """The SolverOptions fields the MINRES path reads (src/linear_algebra/concepts/solver.hpp:212-255)."""
    tolerance: float = 1e-8
    max_iterations: int = 20000
    use_true_residual_batching: bool = True
    true_residual_check_interval: int = 100
    preconditioner: str = "amg_block"        # "amg_block" | "learned"
    amg_smooth_steps: int = 2
    amg_strength: float = 0.08
    amg_coarse_size: int = 256
    amg_aggressive_levels: int = 1
    amg_vcycles: int = 1

    def to_c(self) -> _lib.SolverOptions:
        o = _lib.SolverOptions()
        o.tolerance = self.tolerance
        o.max_iterations = self.max_iterations
        o.use_true_residual_batching = 1 if self.use_true_residual_batching else 0
        o.true_residual_check_interval = self.true_residual_check_interval
        o.preconditioner = {"amg_block": _lib.APF_PRECOND_AMG_BLOCK, "learned": _lib.APF_PRECOND_LEARNED}[self.preconditioner]
        o.amg_smooth_steps = self.amg_smooth_steps
        o.amg_strength = self.amg_strength
        o.amg_coarse_size = self.amg_coarse_size
        o.amg_aggressive_levels = self.amg_aggressive_levels
        o.amg_vcycles = self.amg_vcycles
        return o


class PreconditionedSolveFailure(RuntimeError):
    def __init__(self, message: str, diagnostics: dict):
        super().__init__(message)
        self.diagnostics = diagnostics


def _diag_dict(d: _lib.SolverDiagnostics) -> dict:
    return {name: getattr(d, name) for name, _ in d._fields_}


def setup_preconditioner(blocks: MainSystemBlocks, options: SolverOptions | None = None):
    options = options or SolverOptions()
    o = options.to_c()
    blocks.ctx.check(blocks.ctx.lib.apf_setup_preconditioner(blocks.ctx.handle, blocks.handle, C.byref(o)))


def solve_saddle_system_with_preconditioner(blocks: MainSystemBlocks, options: SolverOptions | None = None,
                                            initial_guess: np.ndarray | None = None, copy_out: bool = True,
                                            rhs: np.ndarray | None = None, correction: bool = False):
    """Solve K [lambda; u] = [f; g] (or K x = rhs).  correction=True with an initial guess
    x0 solves the correction equation K d = [f; g] - K x0 from zero on the device and
    returns x0 + d, as the reference's dispatcher does with
    MainSystemInitialGuess::solve_correction_equation (solve_saddle_system.hpp:75-86).
    Returns (solution or None, diagnostics dict)."""
    options = options or SolverOptions()
    ctx = blocks.ctx
    o = options.to_c()
    n = blocks.n_lambda() + blocks.n_u()
    out = np.empty(n) if copy_out else None
    guess = None
    if initial_guess is not None:
        guess = np.ascontiguousarray(initial_guess, dtype=np.float64)
        if guess.size != n:
            raise ValueError("initial guess size does not match the full saddle system")
    if correction and (guess is None or rhs is not None):
        raise ValueError("the correction equation needs an initial guess and the assembled right-hand side")
    d = _lib.SolverDiagnostics()
    if correction:
        rc = ctx.lib.apf_solve_minres_correction(ctx.handle, blocks.handle, C.byref(o), _ptr(guess), _ptr(out), 0,
                                                 C.byref(d))
    elif rhs is None:
        rc = ctx.lib.apf_solve_minres(ctx.handle, blocks.handle, C.byref(o), _ptr(guess), _ptr(out), 0, C.byref(d))
    else:
        b = np.ascontiguousarray(rhs, dtype=np.float64)
        if b.size != n:
            raise ValueError("right-hand side size does not match the full saddle system")
        rc = ctx.lib.apf_solve_minres_with_rhs(ctx.handle, blocks.handle, C.byref(o), _ptr(b), _ptr(guess), _ptr(out),
                                               0, C.byref(d))
    diag = _diag_dict(d)
    if rc == _lib.APF_ERR_NOT_CONVERGED:
        raise PreconditionedSolveFailure(ctx.lib.apf_ctx_last_error(ctx.handle).decode(), diag)
    ctx.check(rc)
    return out, diag


def residual_norms(blocks: MainSystemBlocks, x: np.ndarray | None = None) -> tuple[float, float]:
    """(||[f; g] - K x||, ||[f; g]||) on the device; x None = the solution the system holds
    (solve_main_system.hpp:540-572: the post-solve and initial-guess residual diagnostics)."""
    xp = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
    if xp is not None and xp.size != blocks.n_lambda() + blocks.n_u():
        raise ValueError("x size does not match the full saddle system")
    r, b = C.c_double(), C.c_double()
    blocks.ctx.check(blocks.ctx.lib.apf_system_residual_norms(blocks.ctx.handle, blocks.handle, _ptr(xp), 0,
                                                              C.byref(r), C.byref(b)))
    return r.value, b.value


def split_solution(blocks: MainSystemBlocks, x: np.ndarray):
    """[lambda; u] -> (lambda, u) (solve_main_system.hpp: update_from_true_solution)."""
    nl = blocks.n_lambda()
    return x[:nl], x[nl:]


def preconditioner_apply(blocks: MainSystemBlocks, r: np.ndarray, block: int = 2) -> np.ndarray:
    """z = P^{-1} r with the set-up preconditioner (block 0: A_y part, 1: Hhat part, 2: full)."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    z = np.empty_like(r)
    blocks.ctx.check(blocks.ctx.lib.apf_preconditioner_apply(blocks.ctx.handle, blocks.handle, block, _ptr(r), _ptr(z), 0))
    return z
