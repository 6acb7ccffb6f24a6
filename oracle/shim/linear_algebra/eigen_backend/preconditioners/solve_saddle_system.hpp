#pragma once
// ORACLE SHIM (test infrastructure only).  Dispatcher specialisation mirroring
// src/linear_algebra/eigen_backend/preconditioners/solve_saddle_system.hpp:32-121:
// returns nullopt unless MINRES + ParabolicGraphNorm is requested, optionally
// solves the correction equation, and throws PreconditionedSolveFailure on
// non-convergence.

#include <optional>
#include <stdexcept>

#include "parabolic_graph_norm_minres.hpp"
#include "linear_algebra/eigen_backend/backend_types.hpp"
#include "linear_algebra/operations/linalg_ops.hpp"
#include "linear_algebra/preconditioners/solve_saddle_system.hpp"
#include "linear_algebra/system/saddle_point_system.hpp"

namespace la::preconditioners
{
    template<>
    struct SaddlePreconditionedSolveDispatcher<la::eigen::Backend>
    {
        template<class InitialGuess>
        [[nodiscard]] static std::optional<SaddlePreconditionedSolveResult<la::eigen::Backend>> solve(
            la::eigen::Solver&, const la::eigen::SparseMatrix& K, const la::eigen::Vector& rhs,
            const la::saddle::SaddlePointBlocks<la::eigen::Backend>& blocks,
            const la::concepts::SolverOptions& options, const InitialGuess& initial_guess,
            const SaddlePreconditionerContext<la::eigen::Backend>& context)
        {
            const auto validation = la::concepts::validate_solver_preconditioner(options.solver, options.preconditioner);
            if (!validation.accepted)
                throw std::invalid_argument(validation.rejection_reason);
            if (!is_saddle_preconditioned_solve_requested(options))
                return std::nullopt;
            blocks.validate();
            if (K.rows() != K.cols() || K.rows() != rhs.size())
                throw std::runtime_error("solve_saddle_system_with_preconditioner: system dimensions are inconsistent.");
            const la::eigen::Vector* guess = initial_guess.has_value() ? initial_guess.full_vector : nullptr;
            la::eigen::Vector residual;
            const la::eigen::Vector* b = &rhs;
            if (initial_guess.has_value() && initial_guess.solve_correction_equation)
            {
                residual = la::ops::subtract(rhs, la::ops::matvec(K, *initial_guess.full_vector));
                b = &residual;
                guess = nullptr;
            }
            if (context.graph_norm == nullptr)
                throw std::runtime_error("solve_saddle_system_with_preconditioner: ParabolicGraphNorm requires graph-norm block context from assembly.");
            auto m = la::eigen::preconditioners::solve_minres_with_parabolic_graph_norm(
                K, blocks, *context.graph_norm, *b, options, guess);
            SaddlePreconditionedSolveResult<la::eigen::Backend> result;
            result.solution = std::move(m.solution);
            result.diagnostics = std::move(m.diagnostics);
            result.setup_seconds = m.setup_seconds;
            result.solve_seconds = m.solve_seconds;
            if (initial_guess.has_value() && initial_guess.solve_correction_equation)
                result.solution = la::ops::add(*initial_guess.full_vector, result.solution);
            return result;
        }
    };
}
