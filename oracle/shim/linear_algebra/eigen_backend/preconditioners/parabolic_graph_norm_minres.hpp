#pragma once
// ORACLE SHIM (test infrastructure only).  Restates the reference's
// block-preconditioned MINRES (src/linear_algebra/eigen_backend/preconditioners/
// parabolic_graph_norm_minres.hpp:46-369) with std-only numerics:
//   * P = blkdiag(A_y, Hhat) applied exactly (the reference factors both blocks
//     with a sparse Cholesky; here the shim's exact sparse direct solver);
//   * MINRES: Paige & Saunders (1975), preconditioned Lanczos form, on the full
//     symmetric K (the reference reads K's lower triangle of a symmetric matrix);
//   * backend stopping test: ||r_0||_2 * (phibar_k / beta_1) < tol * ||b||_2,
//     i.e. the MINRES residual-norm estimate scaled to the unpreconditioned start
//     residual (the residual-norm recurrence used by Eigen's MINRES);
//   * true-residual batches as in iterative_residual_acceptance.hpp:118-216.
// Iterates and iteration counts are NOT pinned to Eigen's: the FP64 true
// relative residual is the acceptance test.

#include <chrono>
#include <cmath>
#include <iomanip>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "linear_algebra/concepts/solver.hpp"
#include "linear_algebra/eigen_backend/backend_types.hpp"
#include "linear_algebra/eigen_backend/operations.hpp"
#include "linear_algebra/eigen_backend/preconditioners/iterative_residual_acceptance.hpp"
#include "linear_algebra/preconditioners/schur_approximations.hpp"
#include "linear_algebra/preconditioners/solve_failure.hpp"
#include "linear_algebra/system/saddle_point_system.hpp"

namespace la::eigen::preconditioners
{
    using ParabolicGraphNormApproximation = la::preconditioners::ParabolicGraphNormApproximation<la::eigen::Backend>;
    using ParabolicGraphNormPreconditionerDiagnostics = la::preconditioners::ParabolicGraphNormPreconditionerDiagnostics;

    [[nodiscard]] inline ParabolicGraphNormApproximation parabolic_graph_norm_approximation(
        const la::eigen::SparseMatrix& A_y, const la::eigen::SparseMatrix& B_dt,
        const la::eigen::SparseMatrix& C_signed, const la::eigen::SparseMatrix& A_x,
        double diagonal_tolerance = 1.0e-14)
    {
        return la::preconditioners::parabolic_graph_norm_approximation<la::eigen::Backend>(
            A_y, B_dt, C_signed, A_x, diagonal_tolerance);
    }

    class ParabolicGraphNormBlockPreconditioner
    {
    public:
        void compute_from_graph_norm(const la::eigen::SparseMatrix& A_y, const ParabolicGraphNormApproximation& gn)
        {
            const auto t0 = std::chrono::steady_clock::now();
            if (A_y.rows() != A_y.cols())
                throw std::runtime_error("ParabolicGraphNormBlockPreconditioner: A_y must be square.");
            if (gn.hhat.rows() != gn.hhat.cols())
                throw std::runtime_error("ParabolicGraphNormBlockPreconditioner: Hhat must be square.");
            n_lambda_ = A_y.rows();
            n_u_ = gn.hhat.rows();
            a_.compute(A_y);
            if (!a_.ok())
                throw std::runtime_error("ParabolicGraphNormBlockPreconditioner: A_y is not SPD for the internal block factorization.");
            h_.compute(gn.hhat);
            if (!h_.ok())
                throw std::runtime_error("ParabolicGraphNormBlockPreconditioner: Hhat is not SPD for the internal block factorization.");
            const auto t1 = std::chrono::steady_clock::now();
            diag_ = {};
            diag_.is_spd = true;
            diag_.n_lambda = n_lambda_;
            diag_.n_u = n_u_;
            diag_.hhat_rows = gn.hhat.rows();
            diag_.hhat_cols = gn.hhat.cols();
            diag_.nnz_hhat = static_cast<int>(gn.hhat.nonzeros());
            diag_.setup_seconds = std::chrono::duration<double>(t1 - t0).count() + gn.diagnostics.setup_seconds;
            diag_.approximation = gn.diagnostics;
            ready_ = true;
        }
        void apply(const double* r, double* z) const
        {
            if (!ready_)
                throw std::runtime_error("ParabolicGraphNormBlockPreconditioner::solve called before successful setup.");
            a_.solve(r, z);
            h_.solve(r + n_lambda_, z + n_lambda_);
        }
        [[nodiscard]] const ParabolicGraphNormPreconditionerDiagnostics& diagnostics() const noexcept { return diag_; }

    private:
        int n_lambda_ = 0, n_u_ = 0;
        bool ready_ = false;
        la::eigen::shim_detail::SparseDirect a_{}, h_{};
        ParabolicGraphNormPreconditionerDiagnostics diag_{};
    };

    // Preconditioned MINRES (Paige & Saunders 1975) restated for the shim.
    class ShimMinres
    {
    public:
        ShimMinres(const la::eigen::SparseMatrix& K, const ParabolicGraphNormBlockPreconditioner& P) : K_(K), P_(P) {}
        void set_max_iterations(int n) { max_it_ = n; }
        void set_tolerance(double t) { tol_ = t; }
        [[nodiscard]] int iterations() const noexcept { return its_; }
        [[nodiscard]] double error() const noexcept { return err_; }
        [[nodiscard]] bool converged() const noexcept { return conv_; }

        void solve_with_guess(const la::eigen::Vector& b, const la::eigen::Vector& x0, la::eigen::Vector& x)
        {
            const int n = b.size();
            x = x0;
            its_ = 0;
            conv_ = false;
            double bn = 0.0;
            for (int i = 0; i < n; ++i) bn += b[i] * b[i];
            bn = std::sqrt(bn);
            if (bn == 0.0) { x.set_zero(); err_ = 0.0; conv_ = true; return; }
            std::vector<double> r1(n), r2(n), y(n), v(n), w(n, 0.0), w1(n, 0.0), w2(n, 0.0), ax(n);
            K_.multiply(x.data(), ax.data());
            double r0n = 0.0;
            for (int i = 0; i < n; ++i) { r1[i] = b[i] - ax[i]; r0n += r1[i] * r1[i]; }
            r0n = std::sqrt(r0n);
            P_.apply(r1.data(), y.data());
            double beta1 = 0.0;
            for (int i = 0; i < n; ++i) beta1 += r1[i] * y[i];
            if (!(beta1 >= 0.0)) throw std::runtime_error("MINRES: preconditioner is not positive definite.");
            beta1 = std::sqrt(beta1);
            if (beta1 == 0.0 || r0n <= tol_ * bn) { err_ = r0n / bn; conv_ = true; return; }
            r2 = r1;
            double oldb = 0.0, beta = beta1, dbar = 0.0, epsln = 0.0, phibar = beta1, cs = -1.0, sn = 0.0;
            while (its_ < max_it_)
            {
                ++its_;
                const double s = 1.0 / beta;
                for (int i = 0; i < n; ++i) v[i] = s * y[i];
                K_.multiply(v.data(), y.data());
                if (its_ >= 2)
                    for (int i = 0; i < n; ++i) y[i] -= (beta / oldb) * r1[i];
                double alfa = 0.0;
                for (int i = 0; i < n; ++i) alfa += v[i] * y[i];
                for (int i = 0; i < n; ++i) y[i] -= (alfa / beta) * r2[i];
                r1.swap(r2);
                r2 = y;
                P_.apply(r2.data(), y.data());
                oldb = beta;
                double bb = 0.0;
                for (int i = 0; i < n; ++i) bb += r2[i] * y[i];
                if (!(bb >= 0.0)) throw std::runtime_error("MINRES: preconditioner is not positive definite.");
                beta = std::sqrt(bb);
                const double oldeps = epsln;
                const double delta = cs * dbar + sn * alfa;
                const double gbar = sn * dbar - cs * alfa;
                epsln = sn * beta;
                dbar = -cs * beta;
                const double gamma = std::max(std::hypot(gbar, beta), 1e-300);
                cs = gbar / gamma;
                sn = beta / gamma;
                const double phi = cs * phibar;
                phibar = sn * phibar;
                for (int i = 0; i < n; ++i)
                {
                    const double wn = (v[i] - oldeps * w1[i] - delta * w2[i]) / gamma;
                    w1[i] = w2[i];
                    w2[i] = wn;
                    x[i] += phi * wn;
                }
                err_ = r0n * (phibar / beta1) / bn;
                if (err_ < tol_) { conv_ = true; break; }
                if (beta == 0.0) break;
            }
        }

    private:
        const la::eigen::SparseMatrix& K_;
        const ParabolicGraphNormBlockPreconditioner& P_;
        int max_it_ = 1000;
        double tol_ = 1e-10;
        int its_ = 0;
        double err_ = 0.0;
        bool conv_ = false;
    };

    struct ParabolicGraphNormMinresResult
    {
        la::eigen::Vector solution;
        la::concepts::SolverDiagnostics diagnostics{};
        double setup_seconds = 0.0;
        double solve_seconds = 0.0;
        ParabolicGraphNormPreconditionerDiagnostics preconditioner_diagnostics{};
    };

    [[nodiscard]] inline std::string format_parabolic_graph_norm_minres_failure(int it, double err, double rel)
    {
        std::ostringstream m;
        m << std::scientific << std::setprecision(12) << "MINRES(ParabolicGraphNorm) solve failed. iterations=" << it
          << ", error=" << err << ", true_relative_residual=" << rel;
        return m.str();
    }

    [[nodiscard]] inline ParabolicGraphNormMinresResult solve_minres_with_parabolic_graph_norm(
        const la::eigen::SparseMatrix& K, const la::saddle::SaddlePointBlocks<la::eigen::Backend>& blocks,
        const ParabolicGraphNormApproximation& graph_norm, const la::eigen::Vector& rhs,
        const la::concepts::SolverOptions& options, const la::eigen::Vector* initial_guess = nullptr)
    {
        if (options.solver != la::concepts::SolverType::MINRES ||
            options.preconditioner != la::concepts::PreconditionerType::ParabolicGraphNorm)
            throw std::runtime_error("solve_minres_with_parabolic_graph_norm requires MINRES with ParabolicGraphNorm preconditioner.");
        if (K.rows() != K.cols() || K.rows() != rhs.size())
            throw std::runtime_error("solve_minres_with_parabolic_graph_norm: system dimensions are inconsistent.");
        ParabolicGraphNormMinresResult result;
        result.solution.resize(rhs.size());
        result.solution.set_zero();
        result.diagnostics.requested_solver = options.solver;
        result.diagnostics.effective_solver = options.solver;
        result.diagnostics.preconditioner = options.preconditioner;
        result.diagnostics.rows = K.rows();
        result.diagnostics.cols = K.cols();
        result.diagnostics.nnz_matrix = K.nonzeros();
        result.diagnostics.direct = false;
        result.diagnostics.iterative = true;
        const auto t0 = std::chrono::steady_clock::now();
        ParabolicGraphNormBlockPreconditioner P;
        P.compute_from_graph_norm(blocks.A, graph_norm);
        const auto t1 = std::chrono::steady_clock::now();
        result.preconditioner_diagnostics = P.diagnostics();
        result.setup_seconds = std::chrono::duration<double>(t1 - t0).count() + graph_norm.diagnostics.setup_seconds;
        la::eigen::Vector start(rhs.size());
        if (initial_guess != nullptr)
        {
            const auto res = compute_monolithic_residual_diagnostics(K, rhs, *initial_guess);
            if (res.relative <= options.tolerance)
            {
                result.solution = *initial_guess;
                result.diagnostics.linear_residual_absolute = res.absolute;
                record_initial_guess_convergence(result.diagnostics, res.relative);
                return result;
            }
            start = *initial_guess;
        }
        ShimMinres minres(K, P);
        const int batch = options.use_true_residual_batching ? options.true_residual_check_interval : options.max_iterations;
        const auto summary = solve_with_true_residual_batches(
            minres, K, rhs, start, options.max_iterations, batch, options.tolerance, result.solution, result.diagnostics);
        const auto t2 = std::chrono::steady_clock::now();
        result.solve_seconds = std::chrono::duration<double>(t2 - t1).count();
        if (!result.diagnostics.iterative_stats.converged.value_or(false))
            throw la::preconditioners::PreconditionedSolveFailure(
                format_parabolic_graph_norm_minres_failure(
                    summary.iterations, summary.backend_reported_error,
                    result.diagnostics.linear_residual_relative.value_or(-1.0)),
                result.diagnostics);
        return result;
    }
}
