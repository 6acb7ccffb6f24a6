#pragma once
// ORACLE SHIM (test infrastructure only; never linked into the product library).
//
// std-only stand-ins for the dense part of the reference's Eigen wrapper API
// (reference: src/linear_algebra/eigen_backend/{vector,dense_matrix,dense_solver}.hpp).
// The reference's own assembly / estimator templates are compiled against these
// classes so that they run here without Eigen 3.4 (absent in this image).  Only
// the wrapper API is mirrored; the numerics are textbook methods:
//   * dense LU with partial (row) pivoting, Golub & Van Loan, Alg. 3.4.1;
//   * dense LU with complete pivoting (rank revealing), Golub & Van Loan, Alg. 3.4.2.

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <memory>
#include <stdexcept>
#include <utility>
#include <vector>

#include "linear_algebra/concepts/solver.hpp"

namespace la::eigen
{
    class Vector
    {
    public:
        using scalar_type = double;
        using index_type = int;

        Vector() = default;
        explicit Vector(index_type n) : data_(static_cast<std::size_t>(n), 0.0) {}

        void resize(index_type n) { data_.resize(static_cast<std::size_t>(n), 0.0); }
        void set_zero() { std::fill(data_.begin(), data_.end(), 0.0); }
        void add(index_type i, scalar_type v) { data_[static_cast<std::size_t>(i)] += v; }
        [[nodiscard]] index_type size() const noexcept { return static_cast<index_type>(data_.size()); }
        [[nodiscard]] scalar_type& operator[](index_type i) { return data_[static_cast<std::size_t>(i)]; }
        [[nodiscard]] scalar_type operator[](index_type i) const { return data_[static_cast<std::size_t>(i)]; }

        [[nodiscard]] double* data() noexcept { return data_.data(); }
        [[nodiscard]] const double* data() const noexcept { return data_.data(); }
        [[nodiscard]] std::vector<double>& storage() noexcept { return data_; }
        [[nodiscard]] const std::vector<double>& storage() const noexcept { return data_; }

    private:
        std::vector<double> data_{};
    };

    // Column-major dense matrix (Eigen::MatrixXd default storage order).
    class DenseMatrix
    {
    public:
        using scalar_type = double;
        using index_type = int;
        using Vector = la::eigen::Vector;

        DenseMatrix() = default;
        DenseMatrix(index_type rows, index_type cols) { set_zero(rows, cols); }

        void resize(index_type rows, index_type cols)
        {
            rows_ = rows;
            cols_ = cols;
            data_.resize(static_cast<std::size_t>(rows) * static_cast<std::size_t>(cols));
        }
        void set_zero() { std::fill(data_.begin(), data_.end(), 0.0); }
        void set_zero(index_type rows, index_type cols)
        {
            resize(rows, cols);
            set_zero();
        }
        void set_identity(index_type rows, index_type cols)
        {
            set_zero(rows, cols);
            for (int i = 0; i < std::min(rows, cols); ++i)
                (*this)(i, i) = 1.0;
        }
        void set(index_type i, index_type j, scalar_type v) { (*this)(i, j) = v; }
        void add(index_type i, index_type j, scalar_type v) { (*this)(i, j) += v; }

        void add_block(index_type r0, index_type c0, const DenseMatrix& b, scalar_type s = 1.0)
        {
            if (r0 < 0 || c0 < 0 || r0 + b.rows() > rows() || c0 + b.cols() > cols())
                throw std::runtime_error("DenseMatrix::add_block block does not fit.");
            for (int j = 0; j < b.cols(); ++j)
                for (int i = 0; i < b.rows(); ++i)
                    (*this)(r0 + i, c0 + j) += s * b(i, j);
        }
        void set_block(index_type r0, index_type c0, const DenseMatrix& b, scalar_type s = 1.0)
        {
            if (r0 < 0 || c0 < 0 || r0 + b.rows() > rows() || c0 + b.cols() > cols())
                throw std::runtime_error("DenseMatrix::set_block block does not fit.");
            for (int j = 0; j < b.cols(); ++j)
                for (int i = 0; i < b.rows(); ++i)
                    (*this)(r0 + i, c0 + j) = s * b(i, j);
        }
        void set_transpose_block(index_type r0, index_type c0, const DenseMatrix& b, scalar_type s = 1.0)
        {
            if (r0 < 0 || c0 < 0 || r0 + b.cols() > rows() || c0 + b.rows() > cols())
                throw std::runtime_error("DenseMatrix::set_transpose_block block does not fit.");
            for (int j = 0; j < b.cols(); ++j)
                for (int i = 0; i < b.rows(); ++i)
                    (*this)(r0 + j, c0 + i) = s * b(i, j);
        }

        [[nodiscard]] index_type rows() const noexcept { return rows_; }
        [[nodiscard]] index_type cols() const noexcept { return cols_; }
        [[nodiscard]] scalar_type coeff(index_type i, index_type j) const { return (*this)(i, j); }
        [[nodiscard]] scalar_type& operator()(index_type i, index_type j)
        {
            return data_[static_cast<std::size_t>(j) * static_cast<std::size_t>(rows_) + static_cast<std::size_t>(i)];
        }
        [[nodiscard]] scalar_type operator()(index_type i, index_type j) const
        {
            return data_[static_cast<std::size_t>(j) * static_cast<std::size_t>(rows_) + static_cast<std::size_t>(i)];
        }

        [[nodiscard]] Vector matvec(const Vector& x) const
        {
            if (cols() != x.size())
                throw std::runtime_error("DenseMatrix::matvec dimension mismatch.");
            Vector y(rows());
            for (int j = 0; j < cols_; ++j)
                for (int i = 0; i < rows_; ++i)
                    y[i] += (*this)(i, j) * x[j];
            return y;
        }
        [[nodiscard]] Vector transpose_matvec(const Vector& x) const
        {
            if (rows() != x.size())
                throw std::runtime_error("DenseMatrix::transpose_matvec dimension mismatch.");
            Vector y(cols());
            for (int j = 0; j < cols_; ++j)
            {
                double s = 0.0;
                for (int i = 0; i < rows_; ++i)
                    s += (*this)(i, j) * x[i];
                y[j] = s;
            }
            return y;
        }
        [[nodiscard]] scalar_type max_abs_coeff() const noexcept
        {
            double m = 0.0;
            for (double v : data_)
                m = std::max(m, std::abs(v));
            return m;
        }
        [[nodiscard]] double frobenius_norm() const noexcept
        {
            double s = 0.0;
            for (double v : data_)
                s += v * v;
            return std::sqrt(s);
        }
        [[nodiscard]] std::size_t estimated_memory_bytes() const noexcept
        {
            return static_cast<std::size_t>(rows()) * static_cast<std::size_t>(cols()) * sizeof(scalar_type);
        }
        [[nodiscard]] const std::vector<double>& storage() const noexcept { return data_; }

    private:
        int rows_ = 0;
        int cols_ = 0;
        std::vector<double> data_{};
    };

    namespace shim_detail
    {
        // In-place LU with row pivoting of a column-major n x n array.
        // Returns false when a pivot column is exactly zero.
        inline bool lu_partial_pivot(std::vector<double>& a, std::vector<int>& piv, int n)
        {
            piv.resize(static_cast<std::size_t>(n));
            bool ok = true;
            auto at = [&](int i, int j) -> double& { return a[static_cast<std::size_t>(j) * n + i]; };
            for (int k = 0; k < n; ++k)
            {
                int p = k;
                double best = std::abs(at(k, k));
                for (int i = k + 1; i < n; ++i)
                    if (std::abs(at(i, k)) > best) { best = std::abs(at(i, k)); p = i; }
                piv[static_cast<std::size_t>(k)] = p;
                if (p != k)
                    for (int j = 0; j < n; ++j) std::swap(at(k, j), at(p, j));
                const double d = at(k, k);
                if (d == 0.0) { ok = false; continue; }
                for (int i = k + 1; i < n; ++i) at(i, k) /= d;
                for (int j = k + 1; j < n; ++j)
                {
                    const double akj = at(k, j);
                    if (akj == 0.0) continue;
                    for (int i = k + 1; i < n; ++i) at(i, j) -= at(i, k) * akj;
                }
            }
            return ok;
        }

        inline void lu_partial_pivot_solve(const std::vector<double>& a, const std::vector<int>& piv, int n, double* x)
        {
            auto at = [&](int i, int j) { return a[static_cast<std::size_t>(j) * n + i]; };
            for (int k = 0; k < n; ++k)
            {
                const int p = piv[static_cast<std::size_t>(k)];
                if (p != k) std::swap(x[k], x[p]);
            }
            for (int j = 0; j < n; ++j)
            {
                const double xj = x[j];
                if (xj != 0.0)
                    for (int i = j + 1; i < n; ++i) x[i] -= at(i, j) * xj;
            }
            for (int j = n - 1; j >= 0; --j)
            {
                x[j] /= at(j, j);
                const double xj = x[j];
                if (xj != 0.0)
                    for (int i = 0; i < j; ++i) x[i] -= at(i, j) * xj;
            }
        }

        // Complete-pivoting LU: P A Q = L U.  Rank decided against threshold * max|pivot|.
        struct FullPivLU
        {
            int n = 0;
            std::vector<double> a{};
            std::vector<int> row_perm{};
            std::vector<int> col_perm{};
            double max_pivot = 0.0;
            int rank = 0;

            void compute(const DenseMatrix& A, double threshold)
            {
                n = A.rows();
                a = A.storage();
                row_perm.resize(static_cast<std::size_t>(n));
                col_perm.resize(static_cast<std::size_t>(n));
                for (int i = 0; i < n; ++i) { row_perm[static_cast<std::size_t>(i)] = i; col_perm[static_cast<std::size_t>(i)] = i; }
                auto at = [&](int i, int j) -> double& { return a[static_cast<std::size_t>(j) * n + i]; };
                max_pivot = 0.0;
                std::vector<double> pivots;
                for (int k = 0; k < n; ++k)
                {
                    int pi = k, pj = k;
                    double best = -1.0;
                    for (int j = k; j < n; ++j)
                        for (int i = k; i < n; ++i)
                            if (std::abs(at(i, j)) > best) { best = std::abs(at(i, j)); pi = i; pj = j; }
                    if (pi != k)
                    {
                        for (int j = 0; j < n; ++j) std::swap(at(k, j), at(pi, j));
                        std::swap(row_perm[static_cast<std::size_t>(k)], row_perm[static_cast<std::size_t>(pi)]);
                    }
                    if (pj != k)
                    {
                        for (int i = 0; i < n; ++i) std::swap(at(i, k), at(i, pj));
                        std::swap(col_perm[static_cast<std::size_t>(k)], col_perm[static_cast<std::size_t>(pj)]);
                    }
                    const double d = at(k, k);
                    pivots.push_back(std::abs(d));
                    max_pivot = std::max(max_pivot, std::abs(d));
                    if (d == 0.0) continue;
                    for (int i = k + 1; i < n; ++i) at(i, k) /= d;
                    for (int j = k + 1; j < n; ++j)
                    {
                        const double akj = at(k, j);
                        if (akj == 0.0) continue;
                        for (int i = k + 1; i < n; ++i) at(i, j) -= at(i, k) * akj;
                    }
                }
                rank = 0;
                for (double p : pivots)
                    if (p > threshold * max_pivot) ++rank;
            }

            [[nodiscard]] bool invertible() const noexcept { return rank == n; }

            void solve(const double* b, double* x) const
            {
                auto at = [&](int i, int j) { return a[static_cast<std::size_t>(j) * n + i]; };
                std::vector<double> y(static_cast<std::size_t>(n));
                for (int i = 0; i < n; ++i) y[static_cast<std::size_t>(i)] = b[row_perm[static_cast<std::size_t>(i)]];
                for (int j = 0; j < n; ++j)
                {
                    const double yj = y[static_cast<std::size_t>(j)];
                    for (int i = j + 1; i < n; ++i) y[static_cast<std::size_t>(i)] -= at(i, j) * yj;
                }
                for (int j = n - 1; j >= 0; --j)
                {
                    y[static_cast<std::size_t>(j)] /= at(j, j);
                    const double yj = y[static_cast<std::size_t>(j)];
                    for (int i = 0; i < j; ++i) y[static_cast<std::size_t>(i)] -= at(i, j) * yj;
                }
                for (int i = 0; i < n; ++i) x[col_perm[static_cast<std::size_t>(i)]] = y[static_cast<std::size_t>(i)];
            }
        };
    }

    class DenseDirectSolver
    {
    public:
        using Matrix = la::eigen::DenseMatrix;
        using Vector = la::eigen::Vector;
        using Options = la::concepts::SolverOptions;
        using Diagnostics = la::concepts::SolverDiagnostics;

        void compute(const Matrix& A) { compute(A, Options{}); }

        void compute(const Matrix& A, const Options& options)
        {
            if (A.rows() != A.cols())
                throw std::runtime_error("DenseDirectSolver::compute requires a square matrix.");
            if (A.rows() == 0)
                throw std::runtime_error("DenseDirectSolver::compute refuses an empty system.");
            computed_ = false;
            n_ = A.rows();
            diagnostics_ = Diagnostics{};
            diagnostics_.rows = A.rows();
            diagnostics_.cols = A.cols();
            diagnostics_.requested_solver = options.solver;
            diagnostics_.effective_solver = options.solver;
            diagnostics_.preconditioner = options.preconditioner;
            diagnostics_.nnz_matrix = static_cast<std::size_t>(A.rows()) * static_cast<std::size_t>(A.cols());
            diagnostics_.direct = true;
            diagnostics_.iterative = false;
            diagnostics_.direct_stats.n = A.rows();
            diagnostics_.direct_stats.nnz_matrix = diagnostics_.nnz_matrix;
            diagnostics_.matrix_norm = A.frobenius_norm();
            full_.reset();
            partial_ = false;
            switch (options.dense_factorization)
            {
            case la::concepts::DenseFactorizationType::PartialPivotDenseLU:
                lu_ = A.storage();
                shim_detail::lu_partial_pivot(lu_, piv_, n_);
                partial_ = true;
                computed_ = true;
                break;
            case la::concepts::DenseFactorizationType::RankRevealingDenseLU:
                full_ = std::make_unique<shim_detail::FullPivLU>();
                full_->compute(A, options.dense_rank_revealing_threshold);
                if (!full_->invertible())
                {
                    full_.reset();
                    throw std::runtime_error("DenseDirectSolver::compute found a singular matrix.");
                }
                computed_ = true;
                break;
            }
        }

        [[nodiscard]] Vector solve(const Vector& b) const
        {
            Vector x;
            solve(b, x);
            return x;
        }

        void solve(const Vector& b, Vector& x) const
        {
            if (!computed_)
                throw std::runtime_error("DenseDirectSolver::solve called before compute.");
            if (b.size() != n_)
                throw std::runtime_error("DenseDirectSolver::solve RHS dimension mismatch.");
            x.resize(n_);
            if (partial_)
            {
                for (int i = 0; i < n_; ++i) x[i] = b[i];
                shim_detail::lu_partial_pivot_solve(lu_, piv_, n_, x.data());
                return;
            }
            if (full_)
            {
                full_->solve(b.data(), x.data());
                return;
            }
            throw std::runtime_error("DenseDirectSolver::solve has no active factorization.");
        }

        [[nodiscard]] const Diagnostics& last_diagnostics() const noexcept { return diagnostics_; }

    private:
        int n_ = 0;
        bool computed_ = false;
        bool partial_ = false;
        std::vector<double> lu_{};
        std::vector<int> piv_{};
        std::unique_ptr<shim_detail::FullPivLU> full_{};
        mutable Diagnostics diagnostics_{};
    };
}
