"""Host-side mirror of the reference's main-system assembly interface.

``assemble_main_system_blocks(problem, ...)`` mirrors
``finite_element::system::assemble_main_system_blocks<QSpace, QTime, Backend>``
(src/finite_element/system/assemble_saddle_problem.hpp:131) and returns a
``MainSystemBlocks`` with the reference's accessors ``A_y()``, ``lower_left_B()``,
``C_signed()``, ``f()``, ``g()``, ``n_lambda()``, ``n_u()`` (:41-110).  The blocks
live on the GPU inside libapf_b200; accessors copy them to the host as
``scipy.sparse.csr_matrix`` on demand.

``MainSystemBlocks.assemble_parabolic_graph_norm_approximation`` mirrors
``finite_element::assembly::assemble_parabolic_graph_norm_approximation``
(src/finite_element/assembly/main_system/parabolic_graph_norm.hpp:22-65).

Errors raise ``ApfError`` with the library's message (the reference throws
``std::runtime_error``).  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np

from . import _lib
from .mesh import SpaceTimeProblem


class Context:
    """A libapf_b200 context bound to one CUDA device and stream."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.apf_ctx_create(device, C.c_void_p(stream) if stream else None, C.byref(h))
        if rc != _lib.APF_OK:
            raise _lib.ApfError(rc, "apf_ctx_create failed (no CUDA device?)")
        self.handle = h
        self.device = device

    def check(self, rc):
        _lib.check(self.handle, rc)

    def synchronize(self):
        self.check(self.lib.apf_ctx_synchronize(self.handle))

    def kernel_launches(self) -> int:
        return int(self.lib.apf_ctx_kernel_launches(self.handle))

    def close(self):
        if self.handle:
            self.lib.apf_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        # at interpreter shutdown the process exit releases the device resources
        if sys.is_finalizing():
            return
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Context | None = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _ptr(a):
    """Raw data pointer of a contiguous numpy array or a torch tensor (None passes through)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)


class _Keep:
    """Holds converted host arrays alive for the duration of a call."""

    def __init__(self):
        self.items = []

    def arr(self, a, dtype):
        if a is None:
            return None
        if hasattr(a, "data_ptr"):
            self.items.append(a)
            return a
        b = np.ascontiguousarray(a, dtype=dtype)
        self.items.append(b)
        return b


def make_desc(problem: SpaceTimeProblem, zero_tol: float, g_scale: float, keep: _Keep) -> _lib.ProblemDesc:
    d = _lib.ProblemDesc()
    d.p = problem.p
    d.n_y_cells = problem.n_y_cells
    d.n_x_cells = problem.n_x_cells
    d.n_lambda = problem.n_lambda
    d.n_u = problem.n_u
    d.y_geometry = _ptr(keep.arr(problem.y_geometry, np.float64))
    d.x_geometry = _ptr(keep.arr(problem.x_geometry, np.float64))
    d.y_to_x = _ptr(keep.arr(problem.y_to_x, np.int32))
    yr, xr = problem.y_restriction, problem.x_restriction
    d.y_restr_offsets = _ptr(keep.arr(yr.offsets, np.int32))
    d.y_restr_dofs = _ptr(keep.arr(yr.dofs, np.int32))
    d.y_restr_weights = _ptr(keep.arr(yr.weights, np.float64))
    d.y_restr_nnz = int(len(yr.dofs))
    d.x_restr_offsets = _ptr(keep.arr(xr.offsets, np.int32))
    d.x_restr_dofs = _ptr(keep.arr(xr.dofs, np.int32))
    d.x_restr_weights = _ptr(keep.arr(xr.weights, np.float64))
    d.x_restr_nnz = int(len(xr.dofs))
    d.m_cells = _ptr(keep.arr(problem.m_cells, np.float64))
    d.ell_cells = _ptr(keep.arr(problem.ell_cells, np.float64))
    d.u0_kind = int(problem.u0_kind)
    d.zero_tol = float(zero_tol)
    d.g_scale = float(g_scale)
    d.dim_space = int(getattr(problem, "dim_space", 2))
    return d


class MainSystemBlocks:
    """Device-resident saddle blocks [A_y B^T; B C_signed] [lambda; u] = [f; g]."""

    def __init__(self, ctx: Context, handle, problem: SpaceTimeProblem):
        self.ctx = ctx
        self.handle = handle
        self.problem = problem

    # -- reference accessors -------------------------------------------------
    def n_lambda(self) -> int:
        return self.problem.n_lambda

    def n_u(self) -> int:
        return self.problem.n_u

    def A_y(self):
        return self.block("A_y")

    def lower_left_B(self):
        return self.block("B")

    def C_signed(self):
        return self.block("C_signed")

    def f(self) -> np.ndarray:
        return self._vector(_lib.APF_VEC_F, self.problem.n_lambda)

    def g(self) -> np.ndarray:
        return self._vector(_lib.APF_VEC_G, self.problem.n_u)

    def K(self):
        """Full saddle matrix (saddle_point_system.hpp:105-137, make_full_system)."""
        return self.block("K")

    # -- graph norm ------------------------------------------------------------
    def assemble_parabolic_graph_norm_approximation(self, diagonal_tolerance: float = 1e-14):
        self.ctx.check(self.ctx.lib.apf_assemble_graph_norm(self.ctx.handle, self.handle, float(diagonal_tolerance)))
        return self.block("Hhat")

    # -- generic access ----------------------------------------------------------
    def block_info(self, name: str):
        r, c, n = C.c_int32(), C.c_int32(), C.c_int64()
        self.ctx.check(self.ctx.lib.apf_system_block_info(self.handle, _lib.BLOCKS[name], C.byref(r), C.byref(c),
                                                           C.byref(n)))
        return r.value, c.value, n.value

    def block(self, name: str):
        import scipy.sparse as sp
        rows, cols, nnz = self.block_info(name)
        rp = np.empty(rows + 1, dtype=np.int32)
        ci = np.empty(nnz, dtype=np.int32)
        va = np.empty(nnz, dtype=np.float64)
        self.ctx.check(self.ctx.lib.apf_system_block_copy(self.ctx.handle, self.handle, _lib.BLOCKS[name], _ptr(rp),
                                                           _ptr(ci), _ptr(va), 0))
        return sp.csr_matrix((va, ci, rp), shape=(rows, cols))

    def block_device_ptrs(self, name: str):
        a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
        self.ctx.check(self.ctx.lib.apf_system_block_device_ptrs(self.handle, _lib.BLOCKS[name], C.byref(a), C.byref(b),
                                                                  C.byref(c)))
        return a.value, b.value, c.value

    def _vector(self, which, n):
        out = np.empty(n, dtype=np.float64)
        self.ctx.check(self.ctx.lib.apf_system_vector_copy(self.ctx.handle, self.handle, which, _ptr(out), 0))
        return out

    def close(self):
        if self.handle:
            self.ctx.lib.apf_system_destroy(self.handle)
            self.handle = None

    def __del__(self):
        if sys.is_finalizing():
            return
        try:
            self.close()
        except Exception:
            pass


def assemble_main_system_blocks(problem: SpaceTimeProblem, zero_tol: float = 1e-15, g_scale: float = -1.0,
                                ctx: Context | None = None, inputs_on_device: bool = False) -> MainSystemBlocks:
    """GPU assembly of A_y, B, C_signed, f, g (and K) for a 2+1D space-time problem.

    ``inputs_on_device``: the problem's arrays are CUDA tensors (device pointers are
    passed straight through); otherwise they are host arrays copied by the library.
    """
    ctx = ctx or default_context()
    keep = _Keep()
    desc = make_desc(problem, zero_tol, g_scale, keep)
    h = C.c_void_p()
    ctx.check(ctx.lib.apf_assemble_main_system(ctx.handle, C.byref(desc), 1 if inputs_on_device else 0, C.byref(h)))
    return MainSystemBlocks(ctx, h, problem)


class TwoPassFullSaddleAssemblyCache:
    """Pattern cache of the two-pass full saddle assembly
    (TwoPassFullSaddleAssemblyCache2D, two_pass_full_saddle_2d.hpp:325-373): the pattern
    is kept on the device while the mesh and its DOF maps are unchanged."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.apf_two_pass_cache_create(self.ctx.handle, C.byref(h)))
        self.handle = h

    def stats(self) -> dict:
        b, r, e = C.c_int64(), C.c_int64(), C.c_int64()
        self.ctx.check(self.ctx.lib.apf_two_pass_cache_stats(self.handle, C.byref(b), C.byref(r), C.byref(e)))
        return {"pattern_builds": b.value, "pattern_reuse_count": r.value, "pattern_entries": e.value}

    @property
    def pattern_reuse_count(self) -> int:
        return self.stats()["pattern_reuse_count"]

    def close(self):
        if self.handle:
            self.ctx.lib.apf_two_pass_cache_destroy(self.handle)
            self.handle = None

    def __del__(self):
        if sys.is_finalizing():
            return
        try:
            self.close()
        except Exception:
            pass


class LinearSystem:
    """The direct-solver path's system (la::linear::LinearSystem,
    src/linear_algebra/system/linear_system.hpp:6-14): the full saddle matrix and
    rhs = [f; g], device-resident."""

    def __init__(self, blocks: MainSystemBlocks):
        self.blocks = blocks

    @property
    def matrix(self):
        return self.blocks.block("K")

    @property
    def rhs(self) -> np.ndarray:
        return np.concatenate([self.blocks.f(), self.blocks.g()])

    def matrix_device_ptrs(self):
        return self.blocks.block_device_ptrs("K")

    def close(self):
        self.blocks.close()


def assemble_main_full_saddle_two_pass(problem: SpaceTimeProblem, zero_tol: float = 1e-15, g_scale: float = -1.0,
                                       ctx: Context | None = None,
                                       assembly_cache: TwoPassFullSaddleAssemblyCache | None = None,
                                       inputs_on_device: bool = False) -> LinearSystem:
    """GPU two-pass full saddle assembly (assemble_main_full_saddle_two_pass_2d,
    two_pass_full_saddle_2d.hpp:468): structural pattern (kept in ``assembly_cache``
    while the mesh is unchanged), numeric pass, prune of |value| <= zero_tol.  2+1D."""
    ctx = ctx or (assembly_cache.ctx if assembly_cache is not None else default_context())
    keep = _Keep()
    desc = make_desc(problem, zero_tol, g_scale, keep)
    h = C.c_void_p()
    ctx.check(ctx.lib.apf_assemble_full_saddle_two_pass(ctx.handle, C.byref(desc), 1 if inputs_on_device else 0,
                                                        assembly_cache.handle if assembly_cache is not None else None,
                                                        C.byref(h)))
    return LinearSystem(MainSystemBlocks(ctx, h, problem))
