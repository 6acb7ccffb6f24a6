#pragma once
// ORACLE SHIM (test infrastructure only): the reference's Eigen-specific
// la::ops overloads (src/linear_algebra/eigen_backend/operations.hpp) reduce to
// the generic templates in linear_algebra/operations for these std-only types.
#include "shim_dense.hpp"
#include "shim_sparse.hpp"
#include "linear_algebra/operations/scalar_ops.hpp"
#include "linear_algebra/operations/dense_matrix_ops.hpp"
#include "linear_algebra/operations/sparse_matrix_ops.hpp"
#include "linear_algebra/operations/vector_ops.hpp"
#include "linear_algebra/preconditioners/schur_approximations.hpp"
