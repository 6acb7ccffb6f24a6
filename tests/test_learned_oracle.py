"""CPU check of the learned preconditioner's FP64 oracle: the reverse-mode gradient of the
training loss (oracle/learned_oracle.py, loss_and_grad_fp64) equals central differences of
the loss to 1e-7 on a small synthetic two-level hierarchy whose weights stay below the
Gershgorin bound (there the rescale factor, held constant by the gradient, is inactive)."""
import numpy as np
import scipy.sparse as sp

import learned_oracle as O


def test_fp64_gradient_matches_central_differences():
    rng = np.random.default_rng(0)
    n = 60
    A = sp.diags([-1.0, 2.5, -1.0], [-1, 0, 1], shape=(n, n)).tocsr()
    P = sp.csr_matrix((np.ones(n), (np.arange(n), np.arange(n) // 3)), shape=(n, n // 3))
    Ac = (P.T @ A @ P).tocsr()
    H = O.Hierarchy([(A, P, 0.6), (Ac, None, 0.6)], True, 4, 0, smooth_steps=2)
    params = rng.normal(0.0, 0.3, O.N_PARAMS)
    starts = [rng.normal(0.0, 1.0, n) for _ in range(2)]
    loss, grad = O.loss_and_grad_fp64(params, [H], [A], [starts], 2)
    assert abs(loss - O.loss(params, [H], [A], [starts], 2)) <= 1e-12 * abs(loss)
    idx = [O.W1 + 3, O.B1 + 1, O.W2 + 40, O.W3 + 5, O.B3, O.ALPHA]
    fd = O.fd_gradient(params, idx, [H], [A], [starts], 2, h=1e-5)
    assert np.abs(grad[idx] - fd).max() <= 1e-7 * np.abs(fd).max()
    # parameters the loss does not see (the second block's coarse scales) get zero
    assert np.all(grad[O.ALPHA + O.MAX_LEVELS:] == 0.0)


def test_shipped_raw_parameters_match_the_npz():
    """The raw float32 copy of the shipped model (read by the C++ drop-in's
    Session::use_learned_model) holds exactly the npz's parameters."""
    from doubleadapparabolicfem_b200.learned import DEFAULT_WEIGHTS, raw_params_path
    with np.load(DEFAULT_WEIGHTS) as z:
        params = np.asarray(z["params"], dtype="<f4")
    raw = np.frombuffer(raw_params_path(DEFAULT_WEIGHTS).read_bytes(), dtype="<f4")
    assert raw.size == 1442 and np.array_equal(raw, params)
