"""Host-side mirror of the reference's estimator entry points (2+1D: p = 1, 2; 1+1D: p = 1).

``estimate(blocks)`` runs, on the solution of the last
``solver.solve_saddle_system_with_preconditioner`` call, what one inner iteration of
``finite_element::time_slabs::compute_adaptive_test_space_iteration``
(src/finite_element/time_slabs/time_slab_adaptive_loop.hpp:727) computes after the
main solve:

* the slab reconstruction lambda~ (``TimeSlabReconstruction::solve_all_slabs``,
  time_slab_reconstruction.hpp:584);
* the vertex-patch equilibrated fluxes (``solve_all_patches``,
  time_slab_equilibrated_flux_reconstruction.hpp:2515);
* the per-source-cell maps ``by_source_cell_flux`` / ``by_source_cell_residual``
  (time_slab_equilibrated_flux_indicators.hpp:203), the reconstruction term
  (time_slab_error_norms.hpp:946) and eta^2 = flux^2 + reconstruction^2
  (time_slab_estimator_combination.hpp).

For 1+1D problems (``dim_space == 1``) the patches are the reference's edge patches
(``TimeSlabEquilibratedFluxReconstruction1plus1d``,
time_slab_equilibrated_flux_reconstruction.hpp:773) and the indicators those of
``compute_equilibrated_flux_error_squared_by_source_cell_1plus1d``
(time_slab_equilibrated_flux_indicators.hpp:23); no vertex ids are needed.

Per-cell results are numpy arrays over the Y cells in input order.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .assembly import MainSystemBlocks, _ptr


def estimate(blocks: MainSystemBlocks, y_vertex_ids: np.ndarray | None = None, patch_precision: str = "fp64"):
    """patch_precision: "fp64" (the reference's arithmetic) or "fp32_refined" (2+1D P1:
    FP32 patch factorisation plus one FP64 iterative-refinement step)."""
    prec = {"fp64": _lib.APF_PATCH_FP64, "fp32_refined": _lib.APF_PATCH_FP32_REFINED}[patch_precision]
    blocks.ctx.check(blocks.ctx.lib.apf_ctx_set_patch_precision(blocks.ctx.handle, prec))
    if getattr(blocks.problem, "dim_space", 2) == 1:
        vids = None  # 1+1D edge patches come from the cell intervals
    else:
        vids = y_vertex_ids if y_vertex_ids is not None else blocks.problem.y_vertex_ids
        if vids is None:
            raise ValueError("the estimator needs the spatial vertex ids of the Y cells")
        vids = np.ascontiguousarray(vids, dtype=np.int32)
    n = blocks.problem.n_y_cells
    out = {k: np.empty(n) for k in ("flux", "divergence", "reconstruction", "eta")}
    res = _lib.EstimatorResult()
    ctx = blocks.ctx
    ctx.check(ctx.lib.apf_estimate(ctx.handle, blocks.handle, _ptr(vids) if vids is not None else None, 0,
                                   _ptr(out["flux"]),
                                   _ptr(out["divergence"]), _ptr(out["reconstruction"]), _ptr(out["eta"]),
                                   C.byref(res)))
    totals = {name: getattr(res, name) for name, _ in res._fields_}
    return out, totals


def keep_flux(blocks: MainSystemBlocks, keep: bool = True):
    """Keep the equilibrated flux of the next 2+1D estimates on the device for flux_samples
    (the reference's flux reconstruction keeps its patch fluxes for
    sigma_and_div_sigma_on_slab_cell, time_slab_equilibrated_flux_reconstruction.hpp:1317-1341)."""
    blocks.ctx.check(blocks.ctx.lib.apf_system_keep_flux(blocks.ctx.handle, blocks.handle, 1 if keep else 0))


def flux_cells(blocks: MainSystemBlocks) -> tuple[np.ndarray, np.ndarray]:
    """(slab, source Y cell index) of every cell the kept flux lives on."""
    ctx = blocks.ctx
    n = C.c_int32()
    ctx.check(ctx.lib.apf_flux_cells(ctx.handle, blocks.handle, C.byref(n), None, None))
    slab = np.empty(n.value, dtype=np.int32)
    src = np.empty(n.value, dtype=np.int32)
    ctx.check(ctx.lib.apf_flux_cells(ctx.handle, blocks.handle, C.byref(n), _ptr(slab), _ptr(src)))
    return slab, src


def flux_samples(blocks: MainSystemBlocks, cells: np.ndarray, points: np.ndarray) -> np.ndarray:
    """[n, 3] = (sigma_x, sigma_y, div sigma) of the kept flux at physical points [n, 3] (x, y, t),
    point i on kept cell cells[i] (sigma_and_div_sigma_on_slab_cell)."""
    c = np.ascontiguousarray(cells, dtype=np.int32)
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    if pts.shape[0] != c.size:
        raise ValueError("one cell per point")
    out = np.empty((c.size, 3))
    blocks.ctx.check(blocks.ctx.lib.apf_flux_sample(blocks.ctx.handle, blocks.handle, c.size, _ptr(c), _ptr(pts),
                                                    _ptr(out), 0))
    return out


def x_marking_indicator_components(blocks: MainSystemBlocks):
    """The adaptive driver's X-marking indicators on the last solve, mirroring
    ``adaptive_algorithm::detail::compute_x_marking_indicator_components``
    (algorithm/detail/indicator_utilities.hpp:443-473).  Returns per-cell arrays
    ``lambda_y_squared_by_y_cell`` (Y cells), ``lambda_y_squared_by_x_cell``,
    ``initial_trace_squared_by_x_cell`` (0 off the t = 0 layer), ``eta_squared_by_x_cell``
    (X cells, input order) and the totals."""
    ny, nx = blocks.problem.n_y_cells, blocks.problem.n_x_cells
    out = {"lambda_y_squared_by_y_cell": np.empty(ny), "lambda_y_squared_by_x_cell": np.empty(nx),
           "initial_trace_squared_by_x_cell": np.empty(nx), "eta_squared_by_x_cell": np.empty(nx)}
    tot = _lib.XIndicatorTotals()
    ctx = blocks.ctx
    ctx.check(ctx.lib.apf_x_indicators(ctx.handle, blocks.handle, 0, _ptr(out["lambda_y_squared_by_y_cell"]),
                                       _ptr(out["lambda_y_squared_by_x_cell"]),
                                       _ptr(out["initial_trace_squared_by_x_cell"]),
                                       _ptr(out["eta_squared_by_x_cell"]), C.byref(tot)))
    return out, {name: getattr(tot, name) for name, _ in tot._fields_}


def g_estimator(blocks: MainSystemBlocks, n_g: int, g_offsets: np.ndarray, g_dofs: np.ndarray,
                g_weights: np.ndarray, tolerance: float = 1e-14):
    """The adaptive driver's G^delta estimator on the last solve, mirroring
    ``AdaptiveDriver::compute_g_estimator_for_accepted_inner_iteration_``
    (algorithm/adaptive_driver.hpp:2690-2900): the degree-(p+1) space G on the Y cells given
    by its flattened CellRestriction (offsets [n_y_cells * 18 + 1] for p = 1, the Y cells in
    input order), A_G lambda_G = f_G - B(X, G)^T u_delta, and ||lambda_G - lambda_delta||^2 in
    the A_G energy.  Returns a dict (``lambda_difference_squared``, ``solve_relative_residual``,
    ``solve_iterations``, ``n_g``)."""
    off = np.ascontiguousarray(g_offsets, dtype=np.int32)
    dofs = np.ascontiguousarray(g_dofs, dtype=np.int32)
    w = np.ascontiguousarray(g_weights, dtype=np.float64)
    if dofs.size != w.size or off.size != blocks.problem.n_y_cells * 18 + 1:
        raise ValueError("the G restriction does not match the Y cells (p = 1: 18 local rows per cell)")
    res = _lib.GEstimatorResult()
    ctx = blocks.ctx
    ctx.check(ctx.lib.apf_g_estimator(ctx.handle, blocks.handle, int(n_g), _ptr(off), _ptr(dofs), _ptr(w), dofs.size,
                                      float(tolerance), C.byref(res)))
    return {name: getattr(res, name) for name, _ in res._fields_}


def y_estimator_threshold_squared(rho: float, lambda_y_squared: float, initial_trace_squared: float) -> float:
    """rho^2 (lambda^2 + (1 + 1/(rho + 1/2)^2) trace^2)
    (algorithm/detail/indicator_utilities.hpp:475-491); raises for rho <= 0."""
    lib = _lib.load()
    out = C.c_double()
    rc = lib.apf_y_estimator_threshold_squared(rho, lambda_y_squared, initial_trace_squared, C.byref(out))
    if rc != _lib.APF_OK:
        raise _lib.ApfError(rc, "compute_y_estimator_threshold_squared: rho must be positive.")
    return out.value


def write_cellwise_error_binary(path: str, cell_ids: np.ndarray, values: np.ndarray, sort_descending: bool = True):
    """The reference's cellwise_error.bin (write_cellwise_error_binary,
    src/finite_element/io/write_cellwise_error_binary.hpp:24-79) from host arrays: int32
    [1, n], int32 cell ids, float64 values, entries by decreasing value (ties by cell id)."""
    lib = _lib.load()
    ids = np.ascontiguousarray(cell_ids, dtype=np.int32)
    v = np.ascontiguousarray(values, dtype=np.float64)
    if ids.size != v.size:
        raise ValueError("one value per cell id")
    rc = lib.apf_write_cellwise_error_binary(None, str(path).encode(), ids.size, _ptr(ids), _ptr(v), 0,
                                             1 if sort_descending else 0)
    if rc != _lib.APF_OK:
        raise _lib.ApfError(rc, f"write_cellwise_error_binary: cannot write {path}")


def write_cellwise_error_components_binary(path: str, cell_ids: np.ndarray, cells: dict,
                                           sort_descending: bool = True):
    """The reference's cellwise_error_components.bin
    (write_cellwise_error_components_binary,
    src/finite_element/io/write_cellwise_error_components_binary.hpp:12-88) from the per-cell
    arrays ``estimate`` returns (flux, reconstruction, divergence, eta): int32 [1, n, 4],
    int32 cell ids, then the four float64 columns, entries by decreasing eta."""
    lib = _lib.load()
    ids = np.ascontiguousarray(cell_ids, dtype=np.int32)
    cols = [np.ascontiguousarray(cells[k], dtype=np.float64) for k in ("flux", "reconstruction", "divergence", "eta")]
    if any(c.size != ids.size for c in cols):
        raise ValueError("one value per cell id in every column")
    rc = lib.apf_write_cellwise_error_components_binary(None, str(path).encode(), ids.size, _ptr(ids),
                                                        *[_ptr(c) for c in cols], 0, 1 if sort_descending else 0)
    if rc != _lib.APF_OK:
        raise _lib.ApfError(rc, f"write_cellwise_error_components_binary: cannot write {path}")


def write_x_indicator_components_binary(path: str, x_cell_ids: np.ndarray, lambda_by_x: np.ndarray,
                                        trace_by_x: np.ndarray, eta_by_x: np.ndarray):
    """The driver's x_indicator_components.bin (write_x_indicator_components_binary,
    algorithm/output/iteration_snapshot_writer.hpp:173-233) from host arrays: int32
    [1, n, 3], int32 X cell ids, float64 lambda_y, initial_trace, eta, by decreasing eta."""
    lib = _lib.load()
    ids = np.ascontiguousarray(x_cell_ids, dtype=np.int32)
    cols = [np.ascontiguousarray(c, dtype=np.float64) for c in (lambda_by_x, trace_by_x, eta_by_x)]
    if any(c.size != ids.size for c in cols):
        raise ValueError("one value per X cell id in every column")
    rc = lib.apf_write_x_indicator_components_binary(None, str(path).encode(), ids.size, _ptr(ids),
                                                     *[_ptr(c) for c in cols], 0)
    if rc != _lib.APF_OK:
        raise _lib.ApfError(rc, f"write_x_indicator_components_binary: cannot write {path}")
