"""CPU tests of the learned-preconditioner oracle (FP64 restatement used by the GPU gradient
check): the restated V-cycle is a symmetric operator, zero parameters give the plain
damped-Jacobi weights with alpha = 1, the Gershgorin rescale keeps the smoother convergent,
and the finite-difference gradient is stable in the step size."""
import numpy as np
import scipy.sparse as sp

import learned_oracle as O


def _toy(block=0, n=48):
    A = sp.diags([-np.ones(n - 1), 2.2 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1]).tocsr()
    P = sp.kron(sp.eye(n // 2), np.ones((2, 1))).tocsr()
    A1 = (P.T @ A @ P).tocsr()
    P1 = sp.kron(sp.eye(n // 4), np.ones((2, 1))).tocsr()
    A2 = (P1.T @ A1 @ P1).tocsr()
    om = lambda M: 4.0 / (3.0 * (abs(M).sum(1).A1 / M.diagonal()).max())
    levels = [(A, P, om(A)), (A1, P1, om(A1)), (A2, None, om(A2))]
    return O.Hierarchy(levels, True, 8, block), A


def _params(seed):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.3, O.N_PARAMS)
    return p


def test_vcycle_is_symmetric():
    for steps in (1, 2, 3):
        H, A = _toy()
        H.smooth_steps = steps
        H.set_params(_params(1))
        rng = np.random.default_rng(2)
        a, b = rng.normal(size=A.shape[0]), rng.normal(size=A.shape[0])
        assert abs(H.vcycle(a) @ b - a @ H.vcycle(b)) <= 1e-12 * np.linalg.norm(a) * np.linalg.norm(b)


def test_zero_parameters_give_plain_smoother():
    H, A = _toy()
    H.set_params(np.zeros(O.N_PARAMS))
    for l in range(len(H.A) - 1):
        for o in range(O.OUTPUTS):
            assert np.allclose(H.w[l][o], H.omega[l] / H.A[l].diagonal(), rtol=1e-15)
        assert H.alpha[l] == 1.0


def test_gershgorin_rescale_bounds_the_smoother():
    H, A = _toy()
    p = np.zeros(O.N_PARAMS)
    p[O.B3:O.ALPHA] = 20.0  # weights exp(0.5) times the plain ones
    H.set_params(p)
    w = H.w[0][0]
    M = sp.diags(np.sqrt(w)) @ A @ sp.diags(np.sqrt(w))
    assert np.linalg.eigvalsh(M.toarray()).max() < 2.0


def test_fd_gradient_is_stable():
    H0, A = _toy(0)
    H1, _ = _toy(1)
    rng = np.random.default_rng(3)
    S = [rng.normal(size=(2, A.shape[0])), rng.normal(size=(2, A.shape[0]))]
    p = _params(4)
    idx = [O.ALPHA, O.ALPHA + O.MAX_LEVELS + 1, O.B3, O.W1 + 3]
    g1 = O.fd_gradient(p, idx, [H0, H1], [A, A], S, 2, h=1e-3)
    g2 = O.fd_gradient(p, idx, [H0, H1], [A, A], S, 2, h=5e-4)
    assert np.abs(g1 - g2).max() <= 1e-5 * max(1.0, np.abs(g1).max())
