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
* ``fd_gradient(...)``: central finite differences of ``loss``;
* ``loss_and_grad_fp64(...)``: the same loss and its exact gradient, in FP64 by reverse mode
  (torch autograd on the CPU) through the MLP, the weights and every V-cycle, with the
  Gershgorin rescale factor held constant, as the device's backward pass treats it.
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


# ----------------------------------------------------------------------------------------
# exact FP64 gradient (reverse mode)
# ----------------------------------------------------------------------------------------
def _torch_sparse(A):
    import torch
    A = A.tocoo()
    idx = torch.tensor(np.vstack([A.row, A.col]), dtype=torch.int64)
    return torch.sparse_coo_tensor(idx, torch.tensor(A.data, dtype=torch.float64), A.shape,
                                   check_invariants=False).coalesce()


def _torch_ops(H):
    """Sparse operators of a hierarchy as torch tensors (built once per hierarchy)."""
    if getattr(H, "_torch", None) is None:
        import torch
        H._torch = {
            "A": [_torch_sparse(A) for A in H.A],
            "absA": [_torch_sparse(abs(A)) for A in H.A],
            "P": [None if P is None else _torch_sparse(P) for P in H.P],
            "PT": [None if P is None else _torch_sparse(P.T.tocsr()) for P in H.P],
            "d": [torch.tensor(A.diagonal(), dtype=torch.float64) for A in H.A],
            "F": [torch.tensor(F, dtype=torch.float64) for F in H.F],
            "Cinv": None if H.Cinv is None else torch.tensor(H.Cinv, dtype=torch.float64),
        }
    return H._torch


def _mv(A, x):
    import torch
    return torch.sparse.mm(A, x.unsqueeze(1)).squeeze(1)


def loss_and_grad_fp64(params, hierarchies, targets, starts_per_block, steps: int):
    """(loss, d loss / d params) in FP64, the gradient exact up to rounding."""
    import torch
    p = torch.tensor(np.asarray(params, dtype=np.float64), requires_grad=True)
    w1 = p[W1:B1].reshape(HIDDEN, N_FEATURES)
    b1 = p[B1:W2]
    w2 = p[W2:B2].reshape(HIDDEN, HIDDEN)
    b2 = p[B2:W3]
    w3 = p[W3:B3].reshape(OUTPUTS, HIDDEN)
    b3 = p[B3:ALPHA]
    total = torch.zeros((), dtype=torch.float64)
    for H, T, S in zip(hierarchies, targets, starts_per_block):
        ops = _torch_ops(H)
        L = len(H.A)
        W, AL = [], []
        for l in range(L - 1):
            y = torch.tanh(torch.tanh(ops["F"][l] @ w1.T + b1) @ w2.T + b2) @ w3.T + b3
            ws = []
            for o in range(OUTPUTS):
                w = H.omega[l] / ops["d"][l] * torch.exp(WEIGHT_RANGE * torch.tanh(y[:, o]))
                with torch.no_grad():
                    sw = torch.sqrt(w)
                    g = float((sw * _mv(ops["absA"][l], sw)).max())
                if g > SMOOTHER_BOUND:
                    w = w * (SMOOTHER_BOUND / g)     # a constant factor: no gradient through the bound
                ws.append(w)
            W.append(ws)
            th = p[ALPHA + H.block * MAX_LEVELS + min(l, MAX_LEVELS - 1)]
            AL.append(2.0 / (1.0 + torch.exp(-th)))

        def coarse(b):
            if H.dense:
                return ops["Cinv"] @ b
            w = H.omega[-1] / ops["d"][-1]
            x = w * b
            for _ in range(H.sweeps - 1):
                x = x + w * (b - _mv(ops["A"][-1], x))
            return x

        def vcycle(b, l=0):
            if l == L - 1:
                return coarse(b)
            A, w, s_ = ops["A"][l], W[l], H.smooth_steps
            cls = [0] + [1] * (s_ - 1)
            x = w[0] * b
            for k in range(1, s_):
                x = x + w[cls[k]] * (b - _mv(A, x))
            xc = vcycle(_mv(ops["PT"][l], b - _mv(A, x)), l + 1)
            x = x + AL[l] * _mv(ops["P"][l], xc)
            for k in range(s_):
                x = x + w[cls[s_ - 1 - k]] * (b - _mv(A, x))
            return x

        Tt = _torch_sparse(T)
        acc = torch.zeros((), dtype=torch.float64)
        for e0 in S:
            e = torch.tensor(e0, dtype=torch.float64)
            q0 = e @ _mv(Tt, e)
            for _ in range(steps):
                e = e - vcycle(_mv(Tt, e))
            qk = e @ _mv(Tt, e)
            acc = acc + (torch.log(qk) - torch.log(q0)) / steps
        total = total + acc / len(S)
    total.backward()
    return float(total.detach()), p.grad.detach().numpy().copy()
