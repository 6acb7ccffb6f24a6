import os
import sys

import numpy as np
import pytest

REPO = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
GOLDEN = os.path.join(REPO, "tests", "golden")
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libapf_b200.so")
    config.addinivalue_line("markers", "slow: larger cases")


GOLDEN_CASES = ["p1_l1_smooth", "p1_l2_smooth", "p2_l1_smooth", "p1_l1_nonmatching"]
# adaptive meshes (X refined locally with hanging nodes, Y refined beyond X by the
# reference's own marking) and a diffusivity per X cell (p1_adapt_kappa, p1_kappa_uniform)
ADAPTIVE_CASES = ["p1_adapt_smooth", "p1_adapt_kappa", "p1_adapt_nonmatching", "p2_adapt_smooth"]
KAPPA_CASES = ["p1_adapt_kappa", "p1_kappa_uniform"]
# the mesh of the reference's adaptive driver after three outer cycles (Y cells = X cells,
# several time slabs, hanging nodes from the driver's own refinement), kappa per block
DRIVER_CASES = ["p1_driver_kappa"]
# fixtures with the driver's G^delta estimator (APF_REF_G): P1 uniform, adaptive, adaptive + kappa
G_DELTA_CASES = ["p1_l2_smooth", "p1_adapt_smooth", "p1_adapt_kappa"]
GOLDEN_CASES_1D = ["d1_l2_smooth", "d1_l2_nonmatching", "d1_l5_smooth"]


def load_golden(name):
    """Golden fixture -> (oracle MainProblem, dict of reference outputs as scipy CSC / arrays)."""
    import apf_oracle as O
    import scipy.sparse as sp
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    p = int(z["meta_p"][0])
    dim = int(z["meta_dim"][0]) if "meta_dim" in z else 2
    ndof = (p + 1) * (p + 1) if dim == 1 else (p + 1) * (p + 2) // 2 * (p + 1)

    def restr(prefix):
        return O.Restriction(z[f"{prefix}_offsets"], z[f"{prefix}_dofs"], z[f"{prefix}_weights"], ndof)

    def csc(nm):
        sh = tuple(int(v) for v in z[f"{nm}_shape"])
        return sp.csc_matrix((z[f"{nm}_values"], z[f"{nm}_inner"], z[f"{nm}_outer"]), shape=sh)

    out = {nm: csc(nm) for nm in ("A_y", "B", "C_signed", "Hhat")}
    out["f"] = z["f"]
    out["g"] = z["g"]
    if "K2p_values" in z:
        # the reference's two-pass full saddle matrix: example coefficients, then the
        # constant anisotropic M = [[2, 0.5], [0.5, 1]] on the cached pattern
        for nm in ("K2p", "K2p_aniso"):
            out[nm] = csc(nm)
            out[nm + "_rhs"] = z[nm + "_rhs"]
        out["K2p_pattern_reuse_count"] = int(z["K2p_pattern_reuse_count"][0])
    m_cells = None
    if "kappa_y" in z and "kappa_x" not in z:
        # M = kappa I with kappa given per Y cell (a law by position, constant on each cell)
        kappa = z["kappa_y"]
        m_cells = np.stack([kappa, np.zeros_like(kappa), kappa], axis=1)
    if "kappa_x" in z:
        # M = kappa I with kappa constant per X cell: every Y cell takes its X ancestor's
        kappa = z["kappa_x"][z["y_to_x_cell"]]
        m_cells = np.stack([kappa, np.zeros_like(kappa), kappa], axis=1)
    prob = O.MainProblem(p=p, y_geom=z["y_geometry"], x_geom=z["x_geometry"], y_to_x=z["y_to_x_cell"],
                         y_restr=restr("y_restriction"), x_restr=restr("x_restriction"),
                         n_lambda=out["A_y"].shape[0], n_u=out["C_signed"].shape[0], m_cells=m_cells,
                         dim_space=dim)
    example = str(z["meta_example"][0])
    return prob, out, example


def load_g_space(name):
    """The reference's G space (degree p+1 on the Y cells) of a G^delta fixture: (n_g,
    Restriction with 18 local rows per Y cell) and the fixture arrays."""
    import apf_oracle as O
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    restr = O.Restriction(z["g_restriction_offsets"], z["g_restriction_dofs"], z["g_restriction_weights"], 18)
    return int(z["g_n_dofs"][0]), restr, z


def to_product_problem(prob, example):
    """Oracle MainProblem -> product SpaceTimeProblem (same arrays)."""
    from doubleadapparabolicfem_b200.mesh import Restriction, SpaceTimeProblem
    u0 = 0 if example == "smooth_initial" else 1
    ell = None
    if prob.dim_space == 1 and example == "non_matching_initial":
        ell = np.full(prob.y_geom.shape[0], 2.0)  # the 1+1D example's constant load
    return SpaceTimeProblem(
        p=prob.p, y_geometry=prob.y_geom, x_geometry=prob.x_geom, y_to_x=prob.y_to_x.astype(np.int32),
        y_restriction=Restriction(prob.y_restr.offsets.astype(np.int32), prob.y_restr.dofs.astype(np.int32),
                                  prob.y_restr.weights, prob.y_restr.ndof),
        x_restriction=Restriction(prob.x_restr.offsets.astype(np.int32), prob.x_restr.dofs.astype(np.int32),
                                  prob.x_restr.weights, prob.x_restr.ndof),
        n_lambda=prob.n_lambda, n_u=prob.n_u, m_cells=prob.m_cells, u0_kind=u0, ell_cells=ell,
        dim_space=prob.dim_space)


def assert_same_sparse(ref, mine, rtol, what="", residue=0.0):
    """Bit-exact pattern, values within rtol relative to max |ref|.

    residue > 0: stored entries with |value| <= residue * max |ref| on either side may be
    absent from the other.  On adaptive meshes Schur terms of the graph-norm block cancel
    exactly for some entries: whether such an entry is dropped (sum exactly 0) or kept as a
    rounding residue (~1e-22) depends on the last bit of its terms, so only the significant
    entries' pattern is compared there; every entry's value still is."""
    r = ref.tocsr()
    r.sort_indices()
    m = mine.tocsr()
    m.sort_indices()
    assert r.shape == m.shape, f"{what}: shape {r.shape} vs {m.shape}"
    scale = max(np.abs(r.data).max(initial=0.0), 1e-300)
    if residue > 0.0:
        cut = residue * scale
        rs = r.copy(); rs.data[np.abs(rs.data) <= cut] = 0.0; rs.eliminate_zeros()
        ms = m.copy(); ms.data[np.abs(ms.data) <= cut] = 0.0; ms.eliminate_zeros()
        assert np.array_equal(rs.indptr, ms.indptr) and np.array_equal(rs.indices, ms.indices), \
            f"{what}: significant patterns differ"
        err = np.abs((r - m).data).max(initial=0.0) / scale
        assert err <= rtol, f"{what}: max relative error {err:.3e} > {rtol:.1e}"
        return err
    assert np.array_equal(r.indptr, m.indptr), f"{what}: row pointers differ"
    assert np.array_equal(r.indices, m.indices), f"{what}: column indices differ"
    err = np.abs(r.data - m.data).max(initial=0.0) / scale
    assert err <= rtol, f"{what}: max relative error {err:.3e} > {rtol:.1e}"
    return err


# below this fraction of the largest |Hhat| entry, Schur-sum cancellation residues
HHAT_RESIDUE = 1e-13


@pytest.fixture(scope="session")
def gpu_ctx():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from doubleadapparabolicfem_b200 import build
    build.build()
    from doubleadapparabolicfem_b200.assembly import Context
    return Context(0)
