#pragma once
// ORACLE SHIM (test infrastructure only).  Restates the reference's true-residual
// batch acceptance (src/linear_algebra/eigen_backend/preconditioners/
// iterative_residual_acceptance.hpp:32-216) for the std-only shim types:
//   * ||K x - b||_2 / ||b||_2 (denominator 1 when b = 0) is the acceptance test;
//   * iterations run in batches of `true_residual_check_interval`;
//   * after a batch whose backend test passed but whose true residual failed,
//     the backend tolerance is multiplied by 0.1 (floor max(eps, tol*sqrt(eps)));
//   * a batch that made no progress or produced non-finite numbers stops.

#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <vector>

#include "linear_algebra/concepts/solver.hpp"
#include "linear_algebra/eigen_backend/backend_types.hpp"

namespace la::eigen::preconditioners
{
    struct MonolithicResidualDiagnostics
    {
        double absolute = 0.0;
        double relative = 0.0;
    };

    struct ResidualCheckedIterativeSolveSummary
    {
        int iterations = 0;
        int batches = 0;
        double backend_reported_error = std::numeric_limits<double>::infinity();
        bool backend_converged = false;
        bool true_residual_stopping_used = false;
        MonolithicResidualDiagnostics residual{};
    };

    [[nodiscard]] inline MonolithicResidualDiagnostics compute_monolithic_residual_diagnostics(
        const la::eigen::SparseMatrix& K, const la::eigen::Vector& rhs, const la::eigen::Vector& solution)
    {
        if (K.rows() != K.cols() || K.rows() != rhs.size() || solution.size() != rhs.size())
            throw std::runtime_error("compute_monolithic_residual_diagnostics: inconsistent system dimensions.");
        std::vector<double> r(static_cast<std::size_t>(rhs.size()));
        K.multiply(solution.data(), r.data());
        double rr = 0.0, bb = 0.0;
        for (int i = 0; i < rhs.size(); ++i)
        {
            const double d = r[static_cast<std::size_t>(i)] - rhs[i];
            rr += d * d;
            bb += rhs[i] * rhs[i];
        }
        const double rn = std::sqrt(rr);
        const double bn = std::sqrt(bb);
        return {rn, rn / (bn > 0.0 ? bn : 1.0)};
    }

    inline void record_iterative_backend_status(
        la::concepts::SolverDiagnostics& d, int iterations, double err, bool conv)
    {
        d.iterative_stats.iterations = iterations;
        d.iterative_stats.final_error = err;
        d.iterative_stats.converged = conv;
        d.iterative_stats.backend_converged = conv;
        d.iterative_stats.backend_reported_error = err;
        d.iterative_stats.convergence_accepted_by_true_residual = false;
    }

    [[nodiscard]] inline bool record_true_residual_acceptance(
        la::concepts::SolverDiagnostics& d, const la::eigen::SparseMatrix& K,
        const la::eigen::Vector& rhs, const la::eigen::Vector& solution, double tol)
    {
        const auto res = compute_monolithic_residual_diagnostics(K, rhs, solution);
        d.linear_residual_absolute = res.absolute;
        d.linear_residual_relative = res.relative;
        d.iterative_stats.final_true_residual = res.relative;
        const bool ok = std::isfinite(res.relative) && res.relative <= tol;
        d.iterative_stats.convergence_accepted_by_true_residual = ok;
        d.iterative_stats.true_residual_stopping_used = true;
        d.iterative_stats.converged = ok;
        d.iterative_stats.final_error = res.relative;
        return ok;
    }

    inline void record_initial_guess_convergence(la::concepts::SolverDiagnostics& d, double rel)
    {
        d.iterative_stats.iterations = 0;
        d.iterative_stats.final_error = rel;
        d.iterative_stats.converged = true;
        d.iterative_stats.backend_converged = true;
        d.iterative_stats.backend_reported_error = rel;
        d.iterative_stats.convergence_accepted_by_true_residual = true;
        d.iterative_stats.residual_check_batches = 0;
        d.iterative_stats.final_true_residual = rel;
        d.iterative_stats.true_residual_stopping_used = true;
        d.linear_residual_relative = rel;
    }

    // IterativeSolver: set_max_iterations(int), set_tolerance(double),
    // solve_with_guess(b, x0, x) -> void, iterations(), error(), converged().
    template<class IterativeSolver>
    [[nodiscard]] inline ResidualCheckedIterativeSolveSummary solve_with_true_residual_batches(
        IterativeSolver& solver, const la::eigen::SparseMatrix& K, const la::eigen::Vector& rhs,
        const la::eigen::Vector& initial_guess, int max_iterations, int requested_batch_size,
        double tolerance, la::eigen::Vector& solution, la::concepts::SolverDiagnostics& diagnostics)
    {
        if (initial_guess.size() != rhs.size())
            throw std::runtime_error("solve_with_true_residual_batches: initial guess size mismatch.");
        const int limit = std::max(1, max_iterations);
        const int batch = std::min(limit, std::max(1, requested_batch_size));
        const double target = std::max(0.0, tolerance);
        const double min_backend = std::max(
            std::numeric_limits<double>::epsilon(), target * std::sqrt(std::numeric_limits<double>::epsilon()));
        la::eigen::Vector current = initial_guess;
        ResidualCheckedIterativeSolveSummary s;
        double backend_tol = target;
        while (s.iterations < limit)
        {
            solver.set_max_iterations(std::min(batch, limit - s.iterations));
            solver.set_tolerance(backend_tol);
            solver.solve_with_guess(rhs, current, solution);
            ++s.batches;
            s.iterations += std::max(0, solver.iterations());
            s.backend_reported_error = solver.error();
            s.backend_converged = solver.converged();
            record_iterative_backend_status(diagnostics, s.iterations, s.backend_reported_error, s.backend_converged);
            const bool ok = record_true_residual_acceptance(diagnostics, K, rhs, solution, target);
            s.residual.absolute = diagnostics.linear_residual_absolute.value_or(std::numeric_limits<double>::infinity());
            s.residual.relative = diagnostics.linear_residual_relative.value_or(std::numeric_limits<double>::infinity());
            s.true_residual_stopping_used = true;
            diagnostics.iterative_stats.residual_check_batches = s.batches;
            diagnostics.iterative_stats.final_true_residual = s.residual.relative;
            diagnostics.iterative_stats.true_residual_stopping_used = true;
            if (ok)
                return s;
            if (!std::isfinite(s.residual.relative) || !std::isfinite(s.backend_reported_error) || solver.iterations() <= 0)
                return s;
            current = solution;
            if (s.backend_converged)
                backend_tol = std::max(min_backend, backend_tol * 0.1);
        }
        return s;
    }
}
