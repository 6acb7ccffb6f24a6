"""ORACLE (test infrastructure only): FP64 numpy restatement of the learned preconditioner's
training objective, used by tests/ to check the GPU loss and its reverse-mode gradient
(the learned preconditioner has no counterpart in the reference; the V-cycle restated here
is the package's own, read from its exported hierarchy).

Objects:
* ``features(A, level, block)``: the 8 scale-free row features;
* ``mlp(params, F)``: 8 -> 32 -> 32 -> 2 with tanh, FP64;
* ``weights(...)``: w_i^(o) = omega / a_ii * exp(0.5 tanh(y_i^(o))), each rescaled so that the
  symmetric Gershgorin bound of W^1/2 A W^1/2 stays <= 1.9;
* ``vcycle(...)``: ``smooth_steps`` damped-Jacobi sweeps before the coarse correction (the
  first with w^(0), the later ones with w^(1)), the same sweeps in reverse order after it,
  coarse correction scaled by alpha, coarsest level solved densely (or by the plain Jacobi
  sweeps);
* ``loss(...)``: sum over the two blocks of mean_e (1/k) log(||E^k e||_T^2 / ||e||_T^2),
  E = I - V T;
* ``fd_gradient(...)``: central finite differences of ``loss``.
"""
from __future__ import annotations

import numpy as np

N_FEATURES, HIDDEN, OUTPUTS, MAX_LEVELS = 8, 32, 2, 16
W1, B1 = 0, HIDDEN * N_FEATURES
W2 = B1 + HIDDEN
B2 = W2 + HIDDEN * HIDDEN
W3 = B2 + HIDDEN
B3 = W3 + OUTPUTS * HIDDEN
ALPHA = B3 + OUTPUTS
N_PARAMS = ALPHA + 2 * MAX_LEVELS
WEIGHT_RANGE = 0.5
SMOOTHER_BOUND = 1.9


def features(A, level: int, block: int) -> np.ndarray:
    A = A.tocsr()
    n = A.shape[0]
    d = A.diagonal()
    dinv = 1.0 / d
    F = np.zeros((n, N_FEATURES))
    for i in range(n):
        cols = A.indices[A.indptr[i]:A.indptr[i + 1]]
        vals = A.data[A.indptr[i]:A.indptr[i + 1]]
        off = cols != i
        c, v = cols[off], vals[off]
        nnz = len(cols)
        F[i, 0] = np.abs(v).sum() * dinv[i]
        F[i, 1] = (np.abs(v).max() if len(v) else 0.0) * dinv[i]
        F[i, 2] = v.sum() * dinv[i]
        F[i, 3] = (v * v * dinv[c]).sum() * dinv[i]
        F[i, 4] = nnz / 32.0
        F[i, 5] = (v > 0).sum() / (nnz - 1) if nnz > 1 else 0.0
        F[i, 6] = level / 8.0
        F[i, 7] = block
    return F


def mlp(params: np.ndarray, F: np.ndarray) -> np.ndarray:
    p = np.asarray(params, dtype=np.float64)
    h1 = np.tanh(F @ p[W1:B1].reshape(HIDDEN, N_FEATURES).T + p[B1:W2])
    h2 = np.tanh(h1 @ p[W2:B2].reshape(HIDDEN, HIDDEN).T + p[B2:W3])
    return h2 @ p[W3:B3].reshape(OUTPUTS, HIDDEN).T + p[B3:ALPHA]


def alpha(params, block: int, level: int) -> float:
    th = float(params[ALPHA + block * MAX_LEVELS + min(level, MAX_LEVELS - 1)])
    return 2.0 / (1.0 + np.exp(-th))


def weights(params, A, F, omega: float):
    """[w^(0), w^(1)] of one level."""
    A = A.tocsr()
    y = mlp(params, F)
    absA = abs(A)
    out = []
    for o in range(OUTPUTS):
        w = omega / A.diagonal() * np.exp(WEIGHT_RANGE * np.tanh(y[:, o]))
        sw = np.sqrt(w)
        g = (sw * (absA @ sw)).max()
        if g > SMOOTHER_BOUND:
            w = w * (SMOOTHER_BOUND / g)
        out.append(w)
    return out


class Hierarchy:
    """levels: list of (A_l, P_l or None, omega_l); features: per level [n_l, 8] (None = compute)."""

    def __init__(self, levels, dense_coarse: bool, coarse_sweeps: int, block: int, features_per_level=None,
                 smooth_steps: int = 1):
        self.smooth_steps = smooth_steps
        self.A = [l[0].tocsr() for l in levels]
        self.P = [l[1].tocsr() if l[1] is not None else None for l in levels]
        self.omega = [l[2] for l in levels]
        self.dense = dense_coarse
        self.sweeps = coarse_sweeps
        self.block = block
        self.F = features_per_level or [features(self.A[l], l, block) for l in range(len(self.A))]
        self.Cinv = np.linalg.inv(self.A[-1].toarray()) if dense_coarse else None

    def set_params(self, params):
        L = len(self.A)
        self.w = [weights(params, self.A[l], self.F[l], self.omega[l]) for l in range(L - 1)]
        self.alpha = [alpha(params, self.block, l) for l in range(L - 1)]

    def coarse(self, b):
        if self.dense:
            return self.Cinv @ b
        A = self.A[-1]
        w = self.omega[-1] / A.diagonal()
        x = w * b
        for _ in range(self.sweeps - 1):
            x = x + w * (b - A @ x)
        return x

    def vcycle(self, b, l=0):
        if l == len(self.A) - 1:
            return self.coarse(b)
        A, P, w = self.A[l], self.P[l], self.w[l]
        s = self.smooth_steps
        cls = [0] + [1] * (s - 1)
        x = w[0] * b
        for k in range(1, s):
            x = x + w[cls[k]] * (b - A @ x)
        xc = self.vcycle(P.T @ (b - A @ x), l + 1)
        x = x + self.alpha[l] * (P @ xc)
        for k in range(s):
            x = x + w[cls[s - 1 - k]] * (b - A @ x)
        return x


def block_loss(H: Hierarchy, T, starts, steps: int) -> float:
    total = 0.0
    for e in starts:
        q0 = e @ (T @ e)
        for _ in range(steps):
            e = e - H.vcycle(T @ e)
        qk = e @ (T @ e)
        total += (np.log(qk) - np.log(q0)) / steps
    return total / len(starts)


def loss(params, hierarchies, targets, starts_per_block, steps: int) -> float:
    L = 0.0
    for H, T, S in zip(hierarchies, targets, starts_per_block):
        H.set_params(params)
        L += block_loss(H, T, S, steps)
    return L


def fd_gradient(params, indices, hierarchies, targets, starts_per_block, steps: int, h: float = 1e-3):
    p = np.asarray(params, dtype=np.float64).copy()
    g = np.zeros(len(indices))
    for k, i in enumerate(indices):
        old = p[i]
        p[i] = old + h
        lp = loss(p, hierarchies, targets, starts_per_block, steps)
        p[i] = old - h
        lm = loss(p, hierarchies, targets, starts_per_block, steps)
        p[i] = old
        g[k] = (lp - lm) / (2 * h)
    return g
