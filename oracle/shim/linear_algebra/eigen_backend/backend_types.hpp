#pragma once
// ORACLE SHIM (test infrastructure only): std-only stand-in for the reference's
// la::eigen::Backend type bundle (reference: src/linear_algebra/eigen_backend/backend_types.hpp).
#include "shim_dense.hpp"
#include "shim_sparse.hpp"

namespace la::eigen
{
    struct Backend
    {
        using scalar_type = double;
        using index_type = int;
        using SparseBuilder = la::eigen::SparseBuilder;
        using SparsePatternBuilder = la::eigen::SparsePatternBuilder;
        using Vector = la::eigen::Vector;
        using DenseMatrix = la::eigen::DenseMatrix;
        using DenseSolver = la::eigen::DenseDirectSolver;
        using SparseMatrix = la::eigen::SparseMatrix;
        using Solver = la::eigen::Solver;
    };
}
