#pragma once
#include <cstdlib>
// ORACLE SHIM (test infrastructure only; never linked into the product library).
//
// std-only stand-ins for the sparse part of the reference's Eigen wrapper API
// (reference: src/linear_algebra/eigen_backend/{sparse_builder,sparse_matrix,
// sparse_pattern_builder,solver}.hpp).  Semantics mirrored:
//   * SparseMatrix is compressed column storage with int32 indices and sorted
//     row indices per column (Eigen::SparseMatrix<double, ColMajor, int>);
//   * set_from_builder sums duplicate triplets in triplet order and keeps
//     explicit zeros produced by the summation (Eigen setFromTriplets +
//     makeCompressed; reference sparse_matrix.hpp:29-37);
//   * prune(ref, eps) keeps |v| > |ref| * eps.
// Solver replaces Eigen::SparseLU with a direct LU: dense partial-pivot LU for
// small systems, otherwise reverse Cuthill-McKee ordering + banded LU with
// partial pivoting (the LAPACK dgbtrf scheme).  Any exact direct solver gives
// the same solution to rounding, which is all the reference's call sites use.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <deque>
#include <numeric>
#include <stdexcept>
#include <utility>
#include <vector>

#include "shim_dense.hpp"
#include "linear_algebra/concepts/solver.hpp"

namespace la::eigen
{
    struct ShimTriplet
    {
        int r;
        int c;
        double v;
        [[nodiscard]] int row() const noexcept { return r; }
        [[nodiscard]] int col() const noexcept { return c; }
        [[nodiscard]] double value() const noexcept { return v; }
    };

    class SparseBuilder
    {
    public:
        using scalar_type = double;
        using index_type = int;
        using triplet_type = ShimTriplet;

        SparseBuilder() = default;
        void reserve(std::size_t n) { triplets_.reserve(n); }
        void add(index_type row, index_type col, scalar_type value) { triplets_.push_back({row, col, value}); }
        void clear() { triplets_.clear(); }
        void merge_from(const SparseBuilder& other)
        {
            triplets_.insert(triplets_.end(), other.triplets_.begin(), other.triplets_.end());
        }
        void merge_from(SparseBuilder&& other)
        {
            triplets_.insert(triplets_.end(), other.triplets_.begin(), other.triplets_.end());
            std::vector<triplet_type>().swap(other.triplets_);
        }
        [[nodiscard]] const std::vector<triplet_type>& triplets() const noexcept { return triplets_; }
        [[nodiscard]] std::vector<triplet_type>& triplets() noexcept { return triplets_; }
        [[nodiscard]] std::size_t size() const noexcept { return triplets_.size(); }
        [[nodiscard]] std::size_t capacity() const noexcept { return triplets_.capacity(); }
        [[nodiscard]] std::size_t estimated_memory_bytes() const noexcept
        {
            return triplets_.capacity() * sizeof(triplet_type);
        }

    private:
        std::vector<triplet_type> triplets_{};
    };

    class SparseMatrix
    {
    public:
        using scalar_type = double;
        using index_type = int;

        SparseMatrix() = default;
        SparseMatrix(index_type rows, index_type cols) { resize(rows, cols); }

        void resize(index_type rows, index_type cols)
        {
            rows_ = rows;
            cols_ = cols;
            outer_.assign(static_cast<std::size_t>(cols) + 1u, 0);
            inner_.clear();
            values_.clear();
        }

        void set_from_builder(const SparseBuilder& builder)
        {
            const auto& t = builder.triplets();
            std::vector<int> count(static_cast<std::size_t>(cols_) + 1u, 0);
            for (const auto& e : t)
            {
                if (e.r < 0 || e.r >= rows_ || e.c < 0 || e.c >= cols_)
                    throw std::runtime_error("SparseMatrix::set_from_builder: triplet out of range.");
                ++count[static_cast<std::size_t>(e.c) + 1u];
            }
            for (int c = 0; c < cols_; ++c)
                count[static_cast<std::size_t>(c) + 1u] += count[static_cast<std::size_t>(c)];
            std::vector<int> rows_tmp(t.size());
            std::vector<double> vals_tmp(t.size());
            std::vector<int> fill(count.begin(), count.end() - 1);
            for (const auto& e : t)
            {
                const int p = fill[static_cast<std::size_t>(e.c)]++;
                rows_tmp[static_cast<std::size_t>(p)] = e.r;
                vals_tmp[static_cast<std::size_t>(p)] = e.v;
            }
            outer_.assign(static_cast<std::size_t>(cols_) + 1u, 0);
            inner_.clear();
            values_.clear();
            inner_.reserve(t.size());
            values_.reserve(t.size());
            std::vector<int> order;
            for (int c = 0; c < cols_; ++c)
            {
                const int b = count[static_cast<std::size_t>(c)];
                const int e = count[static_cast<std::size_t>(c) + 1u];
                order.resize(static_cast<std::size_t>(e - b));
                std::iota(order.begin(), order.end(), b);
                // stable: duplicates are summed in triplet order
                std::stable_sort(order.begin(), order.end(), [&](int x, int y)
                                 { return rows_tmp[static_cast<std::size_t>(x)] < rows_tmp[static_cast<std::size_t>(y)]; });
                int last_row = -1;
                for (const int p : order)
                {
                    const int r = rows_tmp[static_cast<std::size_t>(p)];
                    if (r == last_row)
                        values_.back() += vals_tmp[static_cast<std::size_t>(p)];
                    else
                    {
                        inner_.push_back(r);
                        values_.push_back(vals_tmp[static_cast<std::size_t>(p)]);
                        last_row = r;
                    }
                }
                outer_[static_cast<std::size_t>(c) + 1u] = static_cast<int>(inner_.size());
            }
        }

        void set(index_type i, index_type j, scalar_type value) { ref_(i, j) = value; }
        void add(index_type i, index_type j, scalar_type value) { ref_(i, j) += value; }
        void compress() {}

        void prune(scalar_type reference, scalar_type epsilon)
        {
            const double cut = std::abs(reference) * epsilon;
            std::vector<int> no(static_cast<std::size_t>(cols_) + 1u, 0);
            std::size_t w = 0;
            for (int c = 0; c < cols_; ++c)
            {
                for (int p = outer_[static_cast<std::size_t>(c)]; p < outer_[static_cast<std::size_t>(c) + 1u]; ++p)
                {
                    if (std::abs(values_[static_cast<std::size_t>(p)]) > cut)
                    {
                        inner_[w] = inner_[static_cast<std::size_t>(p)];
                        values_[w] = values_[static_cast<std::size_t>(p)];
                        ++w;
                    }
                }
                no[static_cast<std::size_t>(c) + 1u] = static_cast<int>(w);
            }
            inner_.resize(w);
            values_.resize(w);
            outer_ = std::move(no);
        }

        [[nodiscard]] index_type rows() const noexcept { return rows_; }
        [[nodiscard]] index_type cols() const noexcept { return cols_; }
        [[nodiscard]] std::size_t nonzeros() const noexcept { return values_.size(); }

        [[nodiscard]] scalar_type coeff(index_type i, index_type j) const
        {
            const int p = find_(i, j);
            return p < 0 ? 0.0 : values_[static_cast<std::size_t>(p)];
        }

        template<class Func>
        void for_each_nonzero(Func&& f) const
        {
            for (int c = 0; c < cols_; ++c)
                for (int p = outer_[static_cast<std::size_t>(c)]; p < outer_[static_cast<std::size_t>(c) + 1u]; ++p)
                    f(inner_[static_cast<std::size_t>(p)], c, values_[static_cast<std::size_t>(p)]);
        }

        // y = A x
        void multiply(const double* x, double* y) const
        {
            std::fill(y, y + rows_, 0.0);
            for (int c = 0; c < cols_; ++c)
            {
                const double xc = x[c];
                for (int p = outer_[static_cast<std::size_t>(c)]; p < outer_[static_cast<std::size_t>(c) + 1u]; ++p)
                    y[inner_[static_cast<std::size_t>(p)]] += values_[static_cast<std::size_t>(p)] * xc;
            }
        }
        // y = A^T x
        void multiply_transpose(const double* x, double* y) const
        {
            for (int c = 0; c < cols_; ++c)
            {
                double s = 0.0;
                for (int p = outer_[static_cast<std::size_t>(c)]; p < outer_[static_cast<std::size_t>(c) + 1u]; ++p)
                    s += values_[static_cast<std::size_t>(p)] * x[inner_[static_cast<std::size_t>(p)]];
                y[c] = s;
            }
        }

        [[nodiscard]] double frobenius_norm() const noexcept
        {
            double s = 0.0;
            for (double v : values_)
                s += v * v;
            return std::sqrt(s);
        }

        [[nodiscard]] const std::vector<int>& outer() const noexcept { return outer_; }
        [[nodiscard]] const std::vector<int>& inner() const noexcept { return inner_; }
        [[nodiscard]] const std::vector<double>& values() const noexcept { return values_; }
        [[nodiscard]] std::vector<double>& values() noexcept { return values_; }

        void assign_compressed(int rows, int cols, std::vector<int> outer, std::vector<int> inner, std::vector<double> values)
        {
            rows_ = rows;
            cols_ = cols;
            outer_ = std::move(outer);
            inner_ = std::move(inner);
            values_ = std::move(values);
        }

    private:
        [[nodiscard]] int find_(int i, int j) const
        {
            if (j < 0 || j >= cols_ || outer_.empty())
                return -1;
            const auto b = inner_.begin() + outer_[static_cast<std::size_t>(j)];
            const auto e = inner_.begin() + outer_[static_cast<std::size_t>(j) + 1u];
            const auto it = std::lower_bound(b, e, i);
            if (it == e || *it != i)
                return -1;
            return static_cast<int>(it - inner_.begin());
        }

        double& ref_(int i, int j)
        {
            if (i < 0 || i >= rows_ || j < 0 || j >= cols_)
                throw std::runtime_error("SparseMatrix: index out of range.");
            const int p = find_(i, j);
            if (p >= 0)
                return values_[static_cast<std::size_t>(p)];
            const auto b = inner_.begin() + outer_[static_cast<std::size_t>(j)];
            const auto e = inner_.begin() + outer_[static_cast<std::size_t>(j) + 1u];
            const auto pos = static_cast<std::size_t>(std::lower_bound(b, e, i) - inner_.begin());
            inner_.insert(inner_.begin() + static_cast<std::ptrdiff_t>(pos), i);
            values_.insert(values_.begin() + static_cast<std::ptrdiff_t>(pos), 0.0);
            for (int c = j + 1; c <= cols_; ++c)
                ++outer_[static_cast<std::size_t>(c)];
            return values_[pos];
        }

        int rows_ = 0;
        int cols_ = 0;
        std::vector<int> outer_{0};
        std::vector<int> inner_{};
        std::vector<double> values_{};
    };

    class SparsePatternBuilder
    {
    public:
        using scalar_type = double;
        using index_type = int;
        using SparseMatrix = la::eigen::SparseMatrix;

        SparsePatternBuilder() = default;

        void resize(index_type rows, index_type cols)
        {
            rows_ = rows;
            cols_ = cols;
            rows_by_col_.assign(static_cast<std::size_t>(cols), {});
            matrix_ = SparseMatrix(rows, cols);
            finalized_ = false;
            entries_ = 0;
        }
        void reserve_pattern(std::size_t) {}
        void add_pattern(index_type row, index_type col)
        {
            check_(row, col);
            auto& r = rows_by_col_[static_cast<std::size_t>(col)];
            const auto it = std::lower_bound(r.begin(), r.end(), row);
            if (it == r.end() || *it != row)
                r.insert(it, row);
        }
        void finalize_pattern()
        {
            std::vector<int> outer(static_cast<std::size_t>(cols_) + 1u, 0);
            std::vector<int> inner;
            for (int c = 0; c < cols_; ++c)
            {
                const auto& r = rows_by_col_[static_cast<std::size_t>(c)];
                inner.insert(inner.end(), r.begin(), r.end());
                outer[static_cast<std::size_t>(c) + 1u] = static_cast<int>(inner.size());
            }
            entries_ = inner.size();
            std::vector<double> values(inner.size(), 0.0);
            matrix_.assign_compressed(rows_, cols_, std::move(outer), std::move(inner), std::move(values));
            std::vector<std::vector<int>>().swap(rows_by_col_);
            finalized_ = true;
        }
        void zero_values()
        {
            ensure_();
            std::fill(matrix_.values().begin(), matrix_.values().end(), 0.0);
        }
        void add(index_type row, index_type col, scalar_type value) { add_to_slot(slot(row, col), value); }
        [[nodiscard]] std::size_t slot(index_type row, index_type col) const
        {
            ensure_();
            check_(row, col);
            const auto& o = matrix_.outer();
            const auto& in = matrix_.inner();
            const auto b = in.begin() + o[static_cast<std::size_t>(col)];
            const auto e = in.begin() + o[static_cast<std::size_t>(col) + 1u];
            const auto it = std::lower_bound(b, e, row);
            if (it == e || *it != row)
                throw std::runtime_error("SparsePatternBuilder::add: entry is not in the finalized sparse pattern.");
            return static_cast<std::size_t>(it - in.begin());
        }
        void add_to_slot(std::size_t s, scalar_type value)
        {
            ensure_();
            if (s >= numeric_nonzeros())
                throw std::runtime_error("SparsePatternBuilder::add_to_slot: slot is out of bounds.");
            matrix_.values()[s] += value;
        }
        [[nodiscard]] index_type rows() const noexcept { return rows_; }
        [[nodiscard]] index_type cols() const noexcept { return cols_; }
        [[nodiscard]] std::size_t pattern_entries() const noexcept { return entries_; }
        [[nodiscard]] std::size_t pattern_candidate_count() const noexcept { return entries_; }
        [[nodiscard]] std::size_t pattern_duplicate_count() const noexcept { return 0; }
        [[nodiscard]] std::size_t pattern_candidate_bytes() const noexcept { return 0; }
        [[nodiscard]] std::size_t compact_pattern_bytes() const noexcept { return 0; }
        [[nodiscard]] std::size_t pattern_bytes_saved() const noexcept { return 0; }
        [[nodiscard]] std::size_t numeric_nonzeros() const noexcept { return matrix_.nonzeros(); }
        [[nodiscard]] std::size_t pattern_bytes() const noexcept { return entries_ * sizeof(int); }
        [[nodiscard]] std::size_t numeric_matrix_bytes() const noexcept
        {
            return numeric_nonzeros() * (sizeof(double) + sizeof(int)) + static_cast<std::size_t>(cols_ + 1) * sizeof(int);
        }
        [[nodiscard]] std::size_t slot_map_bytes() const noexcept { return 0; }
        [[nodiscard]] const SparseMatrix& matrix() const noexcept { return matrix_; }
        [[nodiscard]] SparseMatrix release_matrix()
        {
            ensure_();
            SparseMatrix out = std::move(matrix_);
            rows_ = cols_ = 0;
            finalized_ = false;
            entries_ = 0;
            return out;
        }

    private:
        void check_(int row, int col) const
        {
            if (row < 0 || col < 0 || row >= rows_ || col >= cols_)
                throw std::runtime_error("SparsePatternBuilder: sparse index is out of bounds.");
        }
        void ensure_() const
        {
            if (!finalized_)
                throw std::runtime_error("SparsePatternBuilder: pattern has not been finalized.");
        }
        int rows_ = 0;
        int cols_ = 0;
        std::vector<std::vector<int>> rows_by_col_{};
        SparseMatrix matrix_{};
        bool finalized_ = false;
        std::size_t entries_ = 0;
    };

    namespace shim_detail
    {
        // Reverse Cuthill-McKee ordering of the symmetrised pattern of A.
        inline std::vector<int> rcm_order(const SparseMatrix& A)
        {
            const int n = A.rows();
            std::vector<std::vector<int>> adj(static_cast<std::size_t>(n));
            A.for_each_nonzero([&](int i, int j, double)
                               {
                                   if (i != j)
                                   {
                                       adj[static_cast<std::size_t>(i)].push_back(j);
                                       adj[static_cast<std::size_t>(j)].push_back(i);
                                   } });
            for (auto& a : adj)
            {
                std::sort(a.begin(), a.end());
                a.erase(std::unique(a.begin(), a.end()), a.end());
            }
            std::vector<int> order;
            order.reserve(static_cast<std::size_t>(n));
            std::vector<char> seen(static_cast<std::size_t>(n), 0);
            std::vector<int> by_degree(static_cast<std::size_t>(n));
            std::iota(by_degree.begin(), by_degree.end(), 0);
            std::stable_sort(by_degree.begin(), by_degree.end(), [&](int a, int b)
                             { return adj[static_cast<std::size_t>(a)].size() < adj[static_cast<std::size_t>(b)].size(); });
            for (const int start : by_degree)
            {
                if (seen[static_cast<std::size_t>(start)])
                    continue;
                std::deque<int> q{start};
                seen[static_cast<std::size_t>(start)] = 1;
                while (!q.empty())
                {
                    const int v = q.front();
                    q.pop_front();
                    order.push_back(v);
                    std::vector<int> nb;
                    for (const int w : adj[static_cast<std::size_t>(v)])
                        if (!seen[static_cast<std::size_t>(w)])
                        {
                            seen[static_cast<std::size_t>(w)] = 1;
                            nb.push_back(w);
                        }
                    std::stable_sort(nb.begin(), nb.end(), [&](int a, int b)
                                     { return adj[static_cast<std::size_t>(a)].size() < adj[static_cast<std::size_t>(b)].size(); });
                    for (const int w : nb)
                        q.push_back(w);
                }
            }
            std::reverse(order.begin(), order.end());
            return order;
        }

        // Banded LU with partial pivoting (row interchanges), LAPACK dgbtrf layout:
        // band stored column-wise with kl extra rows for fill from pivoting.
        struct BandLU
        {
            int n = 0, kl = 0, ku = 0, ld = 0;
            std::vector<double> ab{};
            std::vector<int> piv{};
            bool ok = true;

            double& at(int i, int j) { return ab[static_cast<std::size_t>(j) * ld + (kl + ku + i - j)]; }
            [[nodiscard]] double at(int i, int j) const { return ab[static_cast<std::size_t>(j) * ld + (kl + ku + i - j)]; }

            void factor(int n_, int kl_, int ku_, const std::vector<int>& perm_new_to_old_inv, const SparseMatrix& A)
            {
                n = n_;
                kl = kl_;
                ku = ku_;
                ld = 2 * kl + ku + 1;
                ab.assign(static_cast<std::size_t>(n) * ld, 0.0);
                A.for_each_nonzero([&](int i, int j, double v)
                                   { at(perm_new_to_old_inv[static_cast<std::size_t>(i)], perm_new_to_old_inv[static_cast<std::size_t>(j)]) += v; });
                piv.assign(static_cast<std::size_t>(n), 0);
                ok = true;
                const int kv = ku + kl;
                for (int j = 0; j < n; ++j)
                {
                    const int km = std::min(kl, n - 1 - j);
                    int p = j;
                    double best = std::abs(at(j, j));
                    for (int i = j + 1; i <= j + km; ++i)
                        if (std::abs(at(i, j)) > best) { best = std::abs(at(i, j)); p = i; }
                    piv[static_cast<std::size_t>(j)] = p;
                    const int jend = std::min(n - 1, j + kv);
                    if (p != j)
                        for (int c = j; c <= jend; ++c) std::swap(at(j, c), at(p, c));
                    const double d = at(j, j);
                    if (d == 0.0) { ok = false; continue; }
                    for (int i = j + 1; i <= j + km; ++i) at(i, j) /= d;
                    for (int c = j + 1; c <= jend; ++c)
                    {
                        const double ajc = at(j, c);
                        if (ajc == 0.0) continue;
                        for (int i = j + 1; i <= j + km; ++i) at(i, c) -= at(i, j) * ajc;
                    }
                }
            }

            void solve(double* x) const
            {
                const int kv = ku + kl;
                for (int j = 0; j < n; ++j)
                {
                    const int p = piv[static_cast<std::size_t>(j)];
                    if (p != j) std::swap(x[j], x[p]);
                    const int km = std::min(kl, n - 1 - j);
                    const double xj = x[j];
                    if (xj != 0.0)
                        for (int i = j + 1; i <= j + km; ++i) x[i] -= at(i, j) * xj;
                }
                for (int j = n - 1; j >= 0; --j)
                {
                    x[j] /= at(j, j);
                    const double xj = x[j];
                    const int i0 = std::max(0, j - kv);
                    if (xj != 0.0)
                        for (int i = i0; i < j; ++i) x[i] -= at(i, j) * xj;
                }
            }
        };

        // Exact direct solver for a square sparse matrix.
        class SparseDirect
        {
        public:
            void compute(const SparseMatrix& A)
            {
                if (A.rows() != A.cols())
                    throw std::runtime_error("SparseDirect: matrix must be square.");
                n_ = A.rows();
                if (n_ <= 1500)
                {
                    dense_ = true;
                    lu_.assign(static_cast<std::size_t>(n_) * n_, 0.0);
                    A.for_each_nonzero([&](int i, int j, double v)
                                       { lu_[static_cast<std::size_t>(j) * n_ + i] += v; });
                    ok_ = lu_partial_pivot(lu_, piv_, n_);
                    return;
                }
                dense_ = false;
                const auto order = rcm_order(A);
                inv_.assign(static_cast<std::size_t>(n_), 0);
                for (int k = 0; k < n_; ++k)
                    inv_[static_cast<std::size_t>(order[static_cast<std::size_t>(k)])] = k;
                int kl = 0, ku = 0;
                A.for_each_nonzero([&](int i, int j, double)
                                   {
                                       const int pi = inv_[static_cast<std::size_t>(i)];
                                       const int pj = inv_[static_cast<std::size_t>(j)];
                                       kl = std::max(kl, pi - pj);
                                       ku = std::max(ku, pj - pi); });
                band_.factor(n_, kl, ku, inv_, A);
                ok_ = band_.ok;
            }
            [[nodiscard]] bool ok() const noexcept { return ok_; }
            void solve(const double* b, double* x) const
            {
                if (dense_)
                {
                    std::copy(b, b + n_, x);
                    lu_partial_pivot_solve(lu_, piv_, n_, x);
                    return;
                }
                std::vector<double> y(static_cast<std::size_t>(n_));
                for (int i = 0; i < n_; ++i)
                    y[static_cast<std::size_t>(inv_[static_cast<std::size_t>(i)])] = b[i];
                band_.solve(y.data());
                for (int i = 0; i < n_; ++i)
                    x[i] = y[static_cast<std::size_t>(inv_[static_cast<std::size_t>(i)])];
            }
            [[nodiscard]] int size() const noexcept { return n_; }

        private:
            int n_ = 0;
            bool dense_ = true;
            bool ok_ = false;
            std::vector<double> lu_{};
            std::vector<int> piv_{};
            std::vector<int> inv_{};
            BandLU band_{};
        };
    }

    class Solver
    {
    public:
        using Matrix = SparseMatrix;
        using VectorType = Vector;
        using Options = la::concepts::SolverOptions;
        using Diagnostics = la::concepts::SolverDiagnostics;

        void compute(const Matrix& A, const Options& options)
        {
            diagnostics_ = Diagnostics{};
            diagnostics_.rows = A.rows();
            diagnostics_.cols = A.cols();
            diagnostics_.requested_solver = options.solver;
            diagnostics_.effective_solver = la::concepts::SolverType::SparseLU;
            diagnostics_.preconditioner = options.preconditioner;
            diagnostics_.nnz_matrix = A.nonzeros();
            diagnostics_.direct = true;
            diagnostics_.iterative = false;
            const auto validation = la::concepts::validate_solver_preconditioner(options.solver, options.preconditioner);
            la::concepts::apply_solver_preconditioner_validation_to_diagnostics(diagnostics_, validation);
            if (!validation.accepted)
                throw std::invalid_argument(validation.rejection_reason);
            if (A.rows() == 0 || A.cols() == 0)
                throw std::invalid_argument("Solver::compute refuses to factor a linear system with zero rows or zero columns.");
            if (options.solver == la::concepts::SolverType::MINRES)
                throw std::invalid_argument("The generic solver wrapper does not construct MINRES.");
            // Stage timing of the reference's own code (bench.py --impl reference): with
            // APF_SHIM_SKIP_PARDISO=1 the shim does not factor systems whose options request
            // PARDISO (the production runs' main saddle solver, absent here, as is Eigen's);
            // solve() then returns its right-hand side as a placeholder.  The SparseLU
            // requests of the reference's own stages (slab reconstruction, local solves) are
            // factored as always.  Off unless set.
            static const bool skip_pardiso = std::getenv("APF_SHIM_SKIP_PARDISO") != nullptr;
            skipped_ = skip_pardiso && options.solver != la::concepts::SolverType::SparseLU;
            if (skipped_)
            {
                computed_ = true;
                return;
            }
            // PARDISO variants and SparseLU all map to the shim's exact direct solver.
            const auto t0 = std::chrono::steady_clock::now();
            direct_.compute(A);
            const auto t1 = std::chrono::steady_clock::now();
            diagnostics_.direct_stats.numeric_factorization_seconds = std::chrono::duration<double>(t1 - t0).count();
            if (!direct_.ok())
                throw std::runtime_error("SparseLU factorization failed.");
            computed_ = true;
        }
        [[nodiscard]] const Diagnostics& last_diagnostics() const noexcept { return diagnostics_; }
        void solve(const VectorType& b, VectorType& x) const
        {
            if (!computed_)
                throw std::runtime_error("Solver::solve called before compute.");
            x.resize(b.size());
            if (skipped_)
            {
                for (int i = 0; i < b.size(); ++i)
                    x[i] = b[i];
                return;
            }
            direct_.solve(b.data(), x.data());
        }
        void solve_with_initial_guess(const VectorType& b, const VectorType& guess, VectorType& x) const
        {
            if (guess.size() != b.size())
                throw std::runtime_error("Solver::solve_with_initial_guess initial guess size mismatch.");
            solve(b, x);
        }

    private:
        bool computed_ = false;
        bool skipped_ = false;
        shim_detail::SparseDirect direct_{};
        mutable Diagnostics diagnostics_{};
    };
}
