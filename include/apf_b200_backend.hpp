/*
 * apf_b200_backend.hpp — the C++20 drop-in of libapf_b200 for the reference's templates
 * (Rsmeets99/DoubleAdapParabolicFEM).
 *
 * It adds one linear-algebra backend, la::b200::Backend, whose host containers are the
 * reference's Eigen-backend types (so every host-side algorithm of the reference --
 * marking, refinement, the estimator, the direct solvers, the diagnostics -- runs on them
 * unchanged) and whose hot path runs on the B200 through the C ABI of apf_b200.h:
 *
 *   finite_element::system::assemble_main_system_blocks<QS, QT, la::b200::Backend>
 *       (src/finite_element/system/assemble_saddle_problem.hpp:131) -> apf_assemble_main_system;
 *       the blocks come back as the reference's host matrices, and the device system
 *       stays resident in the calling thread's session;
 *   la::preconditioners::parabolic_graph_norm_approximation<la::b200::Backend>, the Schur step of
 *       finite_element::assembly::assemble_parabolic_graph_norm_approximation
 *       (src/finite_element/assembly/main_system/parabolic_graph_norm.hpp:13-64;
 *       src/linear_algebra/preconditioners/schur_approximations.hpp:231-287) ->
 *       apf_assemble_graph_norm on that device system (the caller still assembles its host
 *       B_dt and A_x, which the device path does not need);
 *   la::preconditioners::SaddlePreconditionedSolveDispatcher<la::b200::Backend>::solve
 *       (src/linear_algebra/preconditioners/solve_saddle_system.hpp:43-111, the seam the Eigen
 *       backend specialises in src/linear_algebra/eigen_backend/preconditioners/
 *       solve_saddle_system.hpp:32-121) -> apf_solve_minres_with_rhs (block-preconditioned
 *       MINRES with the reference's true-residual batches) on the device system;
 *   finite_element::time_slabs::compute_adaptive_test_space_iteration<QS, QT, la::b200::Backend>
 *       (src/finite_element/time_slabs/time_slab_adaptive_loop.hpp:727) -> for MINRES +
 *       ParabolicGraphNorm a device-resident main solve (apf_assemble_main_system,
 *       apf_assemble_graph_norm, apf_solve_minres or apf_solve_minres_correction,
 *       apf_system_residual_norms: no host copies of the blocks, no host K, no host B_dt / A_x;
 *       only the solution comes back), other solvers through the seams above; then
 *       apf_estimate (la::b200::estimate) in place of the reference's host slab
 *       reconstruction, patch flux solves and indicators, then its own combination and
 *       marking (the reference's adaptive driver calls this);
 *   adaptive_algorithm::output::detail::write_time_slab_estimator_diagnostics_snapshot for a
 *       b200 iteration state (algorithm/output/iteration_snapshot_writer.hpp:143-170) -> the
 *       vertex patches by the reference's writer and flux_reconstruction_samples.bin from the
 *       flux the device estimate kept (apf_flux_sample).
 *
 * la::b200::session() holds the device context, the last system and the solve options;
 * use_learned_model(path) switches its solves to the learned preconditioner (plain fallback
 * armed), set_keep_flux(false) drops the kept flux when no snapshots are written.
 *
 * The assembly function is a constrained overload of the reference's own template, and the
 * Schur step and the dispatcher are full specialisations; qualified calls bind to the
 * overloads visible where the calling template is defined, so this header must be included
 * BEFORE the reference's solver and driver headers
 * (finite_element/system/solve_main_system.hpp, time_slabs/time_slab_adaptive_loop.hpp,
 * algorithm/...).  A solve whose blocks were not assembled through this backend in the
 * same thread throws instead of solving on the host.
 *
 * la::b200::estimate(y_space) returns the device estimate of the session's solved system in
 * the reference's cellwise error types (for its marking), in place of the host stages of
 * compute_adaptive_test_space_iteration after the main solve.
 *
 * Coefficients: M and ell are evaluated at each Y cell's centroid (the device assembly takes
 * them constant per cell, exact for the reference's piecewise-constant coefficients); u0
 * must be one of the examples' initial data sin(pi x) sin(pi y) (sin(pi x) in 1+1D), 1 or 0,
 * recognised by sampling.  Quadrature orders: the device blocks are the exact integrals,
 * equal to the reference's at its own orders (QSpace = 4p + 1, QTime = 2p + 1 in 2+1D;
 * 3 and 3 in 1+1D).
 *
 * Link with -lapf_b200.  Not thread-safe across threads sharing a session (each host thread
 * has its own).
 */
#pragma once

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <concepts>
#include <cstdint>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <limits>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>

#include "apf_b200.h"

#include "linear_algebra/eigen_backend/backend.hpp"
#include "linear_algebra/operations/linalg_ops.hpp"
#include "linear_algebra/preconditioners/solve_failure.hpp"
#include "linear_algebra/preconditioners/schur_approximations.hpp"
#include "linear_algebra/preconditioners/solve_saddle_system.hpp"
#include "finite_element/assembly/constrained_dofs.hpp"
#include "finite_element/assembly/detail/active_cell_locator.hpp"
#include "finite_element/system/assemble_saddle_problem.hpp"
#include "finite_element/system/main_preconditioner_context.hpp"
#include "finite_element/time_slabs/time_slab_cellwise_errors.hpp"
#include "finite_element/time_slabs/time_slab_estimator_combination.hpp"

namespace la::b200
{
    // Host containers of the reference's Eigen backend; a distinct type, so that the
    // overloads and the dispatcher specialisation below take over the hot path.
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

    // A failed C-ABI call: the status code and the context's message.
    class Error : public std::runtime_error
    {
    public:
        Error(int status, const std::string& message)
            : std::runtime_error(message), status_(status)
        {}

        [[nodiscard]] int status() const noexcept { return status_; }

    private:
        int status_;
    };

    inline void check(apf_ctx* ctx, int rc, const char* what)
    {
        if (rc == APF_OK)
            return;
        std::string msg = std::string("b200 backend: ") + what + " failed (status " + std::to_string(rc) + ")";
        if (ctx != nullptr)
        {
            const char* e = apf_ctx_last_error(ctx);
            if (e != nullptr && *e != '\0')
                msg += ": " + std::string(e);
        }
        throw Error(rc, msg);
    }

    // Per host thread: the device context and the device system of the last assembly, with
    // a few of its blocks' entries kept to recognise the host copies handed back to the
    // reference.
    class Session
    {
    public:
        struct Probe
        {
            int block, row, col;
            double value;
        };

        Session()
        {
            apf_solver_options_default(&options_);
        }
        Session(const Session&) = delete;
        Session& operator=(const Session&) = delete;

        ~Session()
        {
            release();
            if (ctx_ != nullptr)
                apf_ctx_destroy(ctx_);
            if (model_ != nullptr)
                apf_learned_model_destroy(model_);
        }

        // CUDA device of the context (before its first use; default: APF_B200_DEVICE or 0)
        void set_device(int device)
        {
            if (ctx_ != nullptr)
                throw std::logic_error("b200 backend: the session's context already exists");
            device_ = device;
        }

        [[nodiscard]] apf_ctx* context()
        {
            if (ctx_ == nullptr)
            {
                int device = device_;
                if (device < 0)
                {
                    const char* env = std::getenv("APF_B200_DEVICE");
                    device = env != nullptr ? std::atoi(env) : 0;
                }
                check(nullptr, apf_ctx_create(device, nullptr, &ctx_), "apf_ctx_create");
            }
            return ctx_;
        }

        // preconditioner kind and AMG parameters of the solves (tolerance, iteration limit
        // and batching come from the reference's SolverOptions of each solve)
        [[nodiscard]] apf_solver_options& solver_options() noexcept { return options_; }

        // the learned preconditioner for the following solves, with the plain block
        // preconditioner as its fallback (a learned run that misses the tolerance is rerun from
        // its iterate): the model's APF_LEARNED_NUM_PARAMS float32 parameters, raw
        // little-endian, as the Python package ships them
        // (doubleadapparabolicfem_b200/data/learned_precond.params.f32)
        void use_learned_model(const std::string& params_path)
        {
            std::ifstream f(params_path, std::ios::binary);
            std::vector<float> p(APF_LEARNED_NUM_PARAMS);
            if (!f.read(reinterpret_cast<char*>(p.data()), static_cast<std::streamsize>(p.size() * sizeof(float))) ||
                f.peek() != std::ifstream::traits_type::eof())
                throw std::runtime_error("b200 backend: " + params_path + " is not " +
                                         std::to_string(APF_LEARNED_NUM_PARAMS) + " float32 parameters");
            apf_ctx* ctx = context();
            if (model_ == nullptr)
                check(ctx, apf_learned_model_create(&model_), "apf_learned_model_create");
            check(ctx, apf_learned_model_set_params(model_, p.data(), APF_LEARNED_NUM_PARAMS),
                  "apf_learned_model_set_params");
            check(ctx, apf_ctx_set_learned_model(ctx, model_), "apf_ctx_set_learned_model");
            options_.preconditioner = APF_PRECOND_LEARNED;
        }

        [[nodiscard]] apf_system* system() const noexcept { return sys_; }
        [[nodiscard]] double zero_tol() const noexcept { return zero_tol_; }
        [[nodiscard]] const apf_solver_diagnostics& last_diagnostics() const noexcept { return last_diag_; }

        void adopt(apf_system* sys, double zero_tol)
        {
            release();
            sys_ = sys;
            zero_tol_ = zero_tol;
        }

        void release()
        {
            if (sys_ != nullptr)
                apf_system_destroy(sys_);
            sys_ = nullptr;
            probes_.clear();
        }

        void add_probe(const Probe& p) { probes_.push_back(p); }

        // the device system whose blocks the host matrices are (by their recorded entries)
        template<class SparseMatrix>
        [[nodiscard]] apf_system* system_for(int block, const SparseMatrix& M) const
        {
            if (sys_ == nullptr)
                return nullptr;
            int32_t rows = 0, cols = 0;
            int64_t nnz = 0;
            if (apf_system_block_info(sys_, block, &rows, &cols, &nnz) != APF_OK || M.rows() != rows ||
                M.cols() != cols)
                return nullptr;
            bool any = false;
            for (const Probe& p : probes_)
                if (p.block == block)
                {
                    any = true;
                    if (M.coeff(p.row, p.col) != p.value)
                        return nullptr;
                }
            return any ? sys_ : nullptr;
        }

        void set_last_diagnostics(const apf_solver_diagnostics& d) noexcept
        {
            last_diag_ = d;
            ++solves_;
            learned_fallbacks_ += d.learned_fallback != 0;
        }
        // device MINRES solves in this thread, and those whose learned run fell back to plain
        [[nodiscard]] long long device_solves() const noexcept { return solves_; }
        [[nodiscard]] long long learned_fallbacks() const noexcept { return learned_fallbacks_; }

        // estimates run through la::b200::estimate in this thread
        [[nodiscard]] long long device_estimates() const noexcept { return estimates_; }
        void count_estimate() noexcept { ++estimates_; }

        // whether la::b200::estimate keeps the flux on the device (default on) for the
        // snapshot writer (flux_reconstruction_samples.bin); the Y cell ids of that estimate in
        // the system's order
        void set_keep_flux(bool keep) noexcept { keep_flux_ = keep; }
        [[nodiscard]] bool keep_flux() const noexcept { return keep_flux_; }
        [[nodiscard]] std::vector<int>& flux_y_cells() noexcept { return flux_y_cells_; }

    private:
        int device_ = -1;
        apf_ctx* ctx_ = nullptr;
        apf_learned_model* model_ = nullptr;
        apf_system* sys_ = nullptr;
        double zero_tol_ = 1e-15;
        apf_solver_options options_{};
        apf_solver_diagnostics last_diag_{};
        long long estimates_ = 0, solves_ = 0, learned_fallbacks_ = 0;
        bool keep_flux_ = true;
        std::vector<int> flux_y_cells_;
        std::vector<Probe> probes_;
    };

    [[nodiscard]] inline Session& session()
    {
        thread_local Session s;
        return s;
    }

    namespace detail
    {
        constexpr int kProbesPerBlock = 16;

        // a block of the device system as the reference's host matrix (explicit zeros kept);
        // records probes of it in the session
        template<class B>
        [[nodiscard]] typename B::SparseMatrix download_block(Session& s, int block)
        {
            apf_ctx* ctx = s.context();
            apf_system* sys = s.system();
            int32_t rows = 0, cols = 0;
            int64_t nnz = 0;
            check(ctx, apf_system_block_info(sys, block, &rows, &cols, &nnz), "apf_system_block_info");
            std::vector<int32_t> rp(static_cast<std::size_t>(rows) + 1), ci(static_cast<std::size_t>(nnz));
            std::vector<double> va(static_cast<std::size_t>(nnz));
            check(ctx, apf_system_block_copy(ctx, sys, block, rp.data(), ci.data(), va.data(), 0),
                  "apf_system_block_copy");
            typename B::SparseBuilder builder;
            builder.reserve(static_cast<std::size_t>(nnz));
            for (int32_t i = 0; i < rows; ++i)
                for (int32_t k = rp[static_cast<std::size_t>(i)]; k < rp[static_cast<std::size_t>(i) + 1]; ++k)
                    builder.add(i, ci[static_cast<std::size_t>(k)], va[static_cast<std::size_t>(k)]);
            typename B::SparseMatrix M(rows, cols);
            M.set_from_builder(builder);
            if (nnz > 0)
            {
                // entries spread over the rows (binary search of the row of entry k)
                for (int q = 0; q < kProbesPerBlock; ++q)
                {
                    const int64_t k = (nnz - 1) * q / std::max(1, kProbesPerBlock - 1);
                    const auto it = std::upper_bound(rp.begin(), rp.end(), static_cast<int32_t>(k));
                    const int row = static_cast<int>(it - rp.begin()) - 1;
                    s.add_probe({block, row, ci[static_cast<std::size_t>(k)], va[static_cast<std::size_t>(k)]});
                }
            }
            return M;
        }

        template<class B>
        [[nodiscard]] typename B::Vector download_vector(Session& s, int which, int n)
        {
            std::vector<double> h(static_cast<std::size_t>(n));
            check(s.context(), apf_system_vector_copy(s.context(), s.system(), which, h.data(), 0),
                  "apf_system_vector_copy");
            typename B::Vector v(n);
            for (int i = 0; i < n; ++i)
                v[i] = h[static_cast<std::size_t>(i)];
            return v;
        }

        // host arrays of an apf_problem_desc built from the reference's spaces and problem data
        struct ProblemArrays
        {
            std::vector<double> y_geo, x_geo, m, ell, y_w, x_w;
            std::vector<int32_t> y_to_x, y_off, y_dofs, x_off, x_dofs;
            apf_problem_desc desc{};
        };

        template<class Space>
        void append_geometry(const Space& space, int c, std::vector<double>& out)
        {
            constexpr int dim = Space::GT::dim_space_v;
            const auto& mesh = space.mesh_ref();
            const auto& cell = mesh.cell(c);
            const auto& sv = mesh.spatial_vertices();
            const auto& tv = mesh.temporal_vertices();
            for (int k = 0; k < dim + 1; ++k)
                for (int d = 0; d < dim; ++d)
                    out.push_back(sv[cell.spatial_vertex_ids[k]][d]);
            out.push_back(tv[cell.temporal_vertex_ids[0]][0]);
            out.push_back(tv[cell.temporal_vertex_ids[1]][0]);
        }

        template<class Space>
        void append_restrictions(const Space& space, const std::vector<int>& cells, std::vector<int32_t>& off,
                                 std::vector<int32_t>& dofs, std::vector<double>& w)
        {
            off.assign(1, 0);
            for (const int c : cells)
            {
                const auto r = finite_element::assembly::build_cell_restriction(space, c);
                for (int i = 0; i < r.size(); ++i)
                {
                    for (const auto& e : r[i])
                    {
                        dofs.push_back(e.true_dof);
                        w.push_back(e.weight);
                    }
                    off.push_back(static_cast<int32_t>(dofs.size()));
                }
            }
        }

        // which of the examples' initial data u0 is (by values at interior sample points)
        template<int Dim, class U0>
        [[nodiscard]] int initial_kind(const U0& u0)
        {
            constexpr double pi = 3.14159265358979323846;
            const double samples[5][2] = {{0.13, 0.71}, {0.37, 0.29}, {0.5, 0.5}, {0.83, 0.17}, {0.61, 0.93}};
            bool sin_sin = true, one = true, zero = true;
            for (const auto& q : samples)
            {
                double v = 0.0;
                if constexpr (Dim == 1 && std::is_invocable_v<const U0&, double>)
                    v = static_cast<double>(u0(q[0]));
                else
                {
                    std::array<double, Dim> p{};
                    for (int d = 0; d < Dim; ++d)
                        p[static_cast<std::size_t>(d)] = q[d];
                    v = static_cast<double>(u0(p));
                }
                double s = std::sin(pi * q[0]);
                if constexpr (Dim == 2)
                    s *= std::sin(pi * q[1]);
                sin_sin = sin_sin && std::abs(v - s) <= 1e-12;
                one = one && std::abs(v - 1.0) <= 1e-12;
                zero = zero && std::abs(v) <= 1e-14;
            }
            if (sin_sin)
                return APF_U0_SIN_SIN;
            if (one)
                return APF_U0_ONE;
            if (zero)
                return APF_U0_ZERO;
            throw std::invalid_argument(
                "b200 backend: the initial datum is not one of the examples' u0 (sin(pi x) sin(pi y), 1, 0)");
        }

        // M(p) as the three entries m00, m01, m11 (2+1D) or one scalar (1+1D)
        template<int Dim, class Value>
        void append_m(const Value& v, std::vector<double>& out)
        {
            if constexpr (std::is_arithmetic_v<Value>)
            {
                out.push_back(static_cast<double>(v));
                if constexpr (Dim == 2)
                {
                    out.push_back(0.0);
                    out.push_back(static_cast<double>(v));
                }
            }
            else if constexpr (Dim == 1)
                out.push_back(v[0][0]);
            else
            {
                out.push_back(v[0][0]);
                out.push_back(v[0][1]);
                out.push_back(v[1][1]);
            }
        }

        template<class YSpace, class XSpace, class Problem>
        [[nodiscard]] ProblemArrays describe(const YSpace& y_space, const XSpace& x_space, const Problem& problem,
                                             double zero_tol, double g_scale)
        {
            constexpr int dim = YSpace::GT::dim_space_v;
            static_assert(dim == 1 || dim == 2, "b200 backend: 1+1D and 2+1D only");
            constexpr int p_space = YSpace::FETraitsType::p_space_v;
            static_assert(p_space == YSpace::FETraitsType::p_time_v, "b200 backend: equal space and time degrees");
            static_assert(dim == 2 ? (p_space == 1 || p_space == 2) : p_space == 1,
                          "b200 backend: P1 and P2 prisms (2+1D), P1 quadrilaterals (1+1D)");
            ProblemArrays a;
            const std::vector<int> y_cells(y_space.active_cells().begin(), y_space.active_cells().end());
            const std::vector<int> x_cells(x_space.active_cells().begin(), x_space.active_cells().end());
            const auto& mesh = x_space.mesh_ref();
            for (const int c : y_cells)
                append_geometry(y_space, c, a.y_geo);
            for (const int c : x_cells)
                append_geometry(x_space, c, a.x_geo);
            append_restrictions(y_space, y_cells, a.y_off, a.y_dofs, a.y_w);
            append_restrictions(x_space, x_cells, a.x_off, a.x_dofs, a.x_w);
            {
                finite_element::assembly::detail::ActiveAncestorCache<XSpace> ancestors(x_space);
                std::vector<int32_t> x_pos(static_cast<std::size_t>(mesh.n_cells()), -1);
                for (std::size_t k = 0; k < x_cells.size(); ++k)
                    x_pos[static_cast<std::size_t>(x_cells[k])] = static_cast<int32_t>(k);
                for (const int c : y_cells)
                {
                    const int32_t pos = x_pos[static_cast<std::size_t>(ancestors.find(c))];
                    if (pos < 0)
                        throw std::runtime_error("b200 backend: a Y cell has no active X ancestor");
                    a.y_to_x.push_back(pos);
                }
            }
            // coefficients at each Y cell's centroid
            const std::size_t row = dim == 2 ? 8u : 4u;
            for (std::size_t k = 0; k < y_cells.size(); ++k)
            {
                const double* g = a.y_geo.data() + k * row;
                std::array<double, dim + 1> p{};
                for (int d = 0; d < dim; ++d)
                {
                    double s = 0.0;
                    for (int v = 0; v < dim + 1; ++v)
                        s += g[v * dim + d];
                    p[static_cast<std::size_t>(d)] = s / (dim + 1);
                }
                p[dim] = 0.5 * (g[row - 2] + g[row - 1]);
                append_m<dim>(problem.M(p), a.m);
                a.ell.push_back(static_cast<double>(problem.ell(p)));
            }
            apf_problem_desc& d = a.desc;
            d.p = p_space;
            d.dim_space = dim;
            d.n_y_cells = static_cast<int>(y_cells.size());
            d.n_x_cells = static_cast<int>(x_cells.size());
            d.n_lambda = y_space.dof_handler_ref().n_true_dofs();
            d.n_u = x_space.dof_handler_ref().n_true_dofs();
            d.y_geometry = a.y_geo.data();
            d.x_geometry = a.x_geo.data();
            d.y_to_x = a.y_to_x.data();
            d.y_restr_offsets = a.y_off.data();
            d.y_restr_dofs = a.y_dofs.data();
            d.y_restr_weights = a.y_w.data();
            d.y_restr_nnz = static_cast<int32_t>(a.y_dofs.size());
            d.x_restr_offsets = a.x_off.data();
            d.x_restr_dofs = a.x_dofs.data();
            d.x_restr_weights = a.x_w.data();
            d.x_restr_nnz = static_cast<int32_t>(a.x_dofs.size());
            d.m_cells = a.m.data();
            d.ell_cells = a.ell.data();
            d.u0_kind = initial_kind<dim>(problem.u0);
            d.zero_tol = zero_tol;
            d.g_scale = g_scale;
            return a;
        }
    }
}

namespace la::b200
{
    // The equilibrated-flux estimate of the session's solved system in the reference's own
    // types: per source Y cell flux^2 and div^2 (CellwiseEquilibratedFluxError), the Y
    // reconstruction error (CellwiseSquaredError) and their combination by the reference's
    // combine_time_slab_estimator_squared_errors_deterministic
    // (time_slab_estimator_combination.hpp:90), ready for its marking
    // (estimator.doerfler_marking_deterministic).  Replaces the host stages of
    // compute_adaptive_test_space_iteration after the main solve (time_slab_adaptive_loop.hpp:
    // slab reconstruction, vertex-patch flux solves, indicators) with apf_estimate.
    struct DeviceEstimate
    {
        finite_element::time_slabs::CellwiseEquilibratedFluxError<int> flux{};
        finite_element::time_slabs::CellwiseSquaredError<int> reconstruction_y_squared{};
        finite_element::time_slabs::CellwiseTimeSlabEstimatorError<int> estimator{};
        int n_slabs = 0;
        int n_patches = 0;
    };

    // y_space: the Y space of the session's last assembly (its active cells in the same order)
    template<class YSpace>
    [[nodiscard]] DeviceEstimate estimate(const YSpace& y_space)
    {
        Session& s = session();
        apf_ctx* ctx = s.context();
        apf_system* sys = s.system();
        if (sys == nullptr)
            throw std::logic_error("b200 backend: estimate needs a system assembled and solved in this thread");
        const std::vector<int> cells(y_space.active_cells().begin(), y_space.active_cells().end());
        const std::size_t ny = cells.size();
        std::vector<int32_t> vids;
        constexpr int dim = YSpace::GT::dim_space_v;
        if constexpr (dim == 2)
        {
            const auto& mesh = y_space.mesh_ref();
            vids.reserve(3 * ny);
            for (const int c : cells)
                for (int k = 0; k < 3; ++k)
                    vids.push_back(mesh.cell(c).spatial_vertex_ids[k]);
        }
        std::vector<double> flux(ny), div(ny), recon(ny), eta(ny);
        apf_estimator_result res{};
        if constexpr (dim == 2)
            check(ctx, apf_system_keep_flux(ctx, sys, s.keep_flux() ? 1 : 0), "apf_system_keep_flux");
        check(ctx, apf_estimate(ctx, sys, dim == 2 ? vids.data() : nullptr, 0, flux.data(), div.data(), recon.data(),
                                eta.data(), &res),
              "apf_estimate");
        s.flux_y_cells() = dim == 2 && s.keep_flux() ? cells : std::vector<int>{};
        DeviceEstimate out;
        for (std::size_t k = 0; k < ny; ++k)
        {
            out.flux.by_source_cell_flux[cells[k]] = flux[k];
            out.flux.by_source_cell_residual[cells[k]] = div[k];
            out.reconstruction_y_squared.by_source_cell[cells[k]] = recon[k];
        }
        out.estimator = finite_element::time_slabs::combine_time_slab_estimator_squared_errors_deterministic(
            out.flux, out.reconstruction_y_squared);
        out.n_slabs = res.n_slabs;
        out.n_patches = res.n_patches;
        s.count_estimate();
        return out;
    }
}

namespace finite_element::system
{
    // assemble_main_system_blocks (assemble_saddle_problem.hpp:131) on the B200: the blocks
    // A_y, B, C_signed, f, g come back as host matrices; the device system stays in the
    // thread's session for the graph-norm block and the solve.
    template<int QSpace, int QTime, class Backend, class YSpaceType, class XSpaceType, class ExampleType>
        requires std::same_as<Backend, la::b200::Backend>
    [[nodiscard]] MainSystemBlocks<Backend> assemble_main_system_blocks(
        const YSpaceType& y_space, const XSpaceType& x_space, const ExampleType& example, double zero_tol = 1e-15,
        double g_scale = -1.0, const finite_element::detail::TimingRecorder& timing = {})
    {
        auto timer = timing.scoped("assembly.total_seconds");
        auto& s = la::b200::session();
        apf_ctx* ctx = s.context();
        const auto arrays = la::b200::detail::describe(y_space, x_space, example, zero_tol, g_scale);
        apf_system* sys = nullptr;
        la::b200::check(ctx, apf_assemble_main_system(ctx, &arrays.desc, 0, &sys), "apf_assemble_main_system");
        s.adopt(sys, zero_tol);
        const int nl = arrays.desc.n_lambda, nu = arrays.desc.n_u;
        auto A = la::b200::detail::download_block<Backend>(s, APF_BLOCK_A_Y);
        auto B = la::b200::detail::download_block<Backend>(s, APF_BLOCK_B);
        auto C = la::b200::detail::download_block<Backend>(s, APF_BLOCK_C);
        auto f = la::b200::detail::download_vector<Backend>(s, APF_VEC_F, nl);
        auto g = la::b200::detail::download_vector<Backend>(s, APF_VEC_G, nu);
        return MainSystemBlocks<Backend>(la::saddle::make_saddle_point_blocks<Backend>(
            std::move(A), std::move(B), std::move(C), std::move(f), std::move(g)));
    }
}

namespace la::b200::detail
{
    // the device MINRES options of a solve: the session's preconditioner and AMG parameters
    // with the tolerance, iteration limit and batching of the reference's SolverOptions
    [[nodiscard]] inline apf_solver_options minres_options(Session& s, const la::concepts::SolverOptions& options)
    {
        apf_solver_options o = s.solver_options();
        o.tolerance = options.tolerance;
        o.max_iterations = options.max_iterations;
        o.use_true_residual_batching = options.use_true_residual_batching ? 1 : 0;
        o.true_residual_check_interval = options.true_residual_check_interval;
        return o;
    }

    // the reference's SolverDiagnostics of a MINRES + ParabolicGraphNorm solve
    // (parabolic_graph_norm_minres.hpp:267-307, iterative_residual_acceptance.hpp:62-92) from
    // the device solve's diagnostics
    [[nodiscard]] inline la::concepts::SolverDiagnostics solver_diagnostics(Session& s,
                                                                            const la::concepts::SolverOptions& options,
                                                                            const apf_solver_diagnostics& d)
    {
        la::concepts::SolverDiagnostics diag;
        diag.requested_solver = options.solver;
        diag.effective_solver = la::concepts::SolverType::MINRES;
        diag.preconditioner = options.preconditioner;
        int32_t kr = 0, kc = 0;
        int64_t knnz = 0;
        check(s.context(), apf_system_block_info(s.system(), APF_BLOCK_K, &kr, &kc, &knnz), "apf_system_block_info");
        diag.rows = kr;
        diag.cols = kc;
        diag.nnz_matrix = static_cast<std::size_t>(knnz);
        diag.direct = false;
        diag.iterative = true;
        diag.linear_residual_relative = d.final_true_residual;
        diag.preconditioner_setup_seconds = d.setup_seconds;
        diag.preconditioner_stats.setup_seconds = d.setup_seconds;
        diag.preconditioner_stats.assumes_spd = true;
        diag.preconditioner_stats.assumes_symmetric = true;
        diag.preconditioner_stats.is_spd = true;
        diag.preconditioner_stats.is_symmetric = true;
        auto& it = diag.iterative_stats;
        it.iterations = d.iterations;
        it.final_error = d.backend_reported_error;
        it.converged = d.converged != 0;
        it.backend_converged = d.backend_converged != 0;
        it.backend_reported_error = d.backend_reported_error;
        it.convergence_accepted_by_true_residual = d.converged != 0;
        it.residual_check_batches = d.residual_check_batches;
        it.final_true_residual = d.final_true_residual;
        it.true_residual_stopping_used = options.use_true_residual_batching;
        return diag;
    }
}

namespace la::preconditioners
{
    // parabolic_graph_norm_approximation (src/linear_algebra/preconditioners/
    // schur_approximations.hpp:231-287), the Schur step of assemble_parabolic_graph_norm_approximation
    // (parabolic_graph_norm.hpp:13-64), on the B200 for the system of the thread's last b200
    // assembly: A_y and C_signed must be its blocks; Hhat is built on the device from the
    // device system (its own B_dt and A_x, with the assembly's zero_tol filter), so the host
    // B_dt and A_x the reference's caller assembled are only checked for their sizes.  A full
    // specialisation (the overload set of the caller's template cannot be extended without
    // an ambiguity, since Backend appears there only in non-deduced contexts).
    template<>
    [[nodiscard]] inline ParabolicGraphNormApproximation<la::b200::Backend>
    parabolic_graph_norm_approximation<la::b200::Backend>(const la::eigen::SparseMatrix& A_y,
                                                          const la::eigen::SparseMatrix& B_dt,
                                                          const la::eigen::SparseMatrix& C_signed,
                                                          const la::eigen::SparseMatrix& A_x,
                                                          double diagonal_tolerance, double zero_tol)
    {
        static_cast<void>(zero_tol);
        auto& s = la::b200::session();
        apf_system* sys = s.system_for(APF_BLOCK_A_Y, A_y);
        if (sys == nullptr || s.system_for(APF_BLOCK_C, C_signed) != sys)
            throw std::invalid_argument(
                "b200 backend: A_y and C_signed are not the blocks of this thread's last b200 assembly");
        if (B_dt.rows() != C_signed.rows() || B_dt.cols() != A_y.rows() || A_x.rows() != C_signed.rows() ||
            A_x.cols() != C_signed.cols())
            throw std::runtime_error("parabolic_graph_norm_approximation: block dimensions are inconsistent.");
        const auto t0 = std::chrono::steady_clock::now();
        apf_ctx* ctx = s.context();
        la::b200::check(ctx, apf_assemble_graph_norm(ctx, sys, diagonal_tolerance), "apf_assemble_graph_norm");
        ParabolicGraphNormApproximation<la::b200::Backend> out;
        out.hhat = la::b200::detail::download_block<la::b200::Backend>(s, APF_BLOCK_HHAT);
        auto& d = out.diagnostics;
        int32_t rows = 0, cols = 0;
        int64_t nnz = 0;
        la::b200::check(ctx, apf_system_block_info(sys, APF_BLOCK_HHAT, &rows, &cols, &nnz), "apf_system_block_info");
        d.hhat_rows = rows;
        d.hhat_cols = cols;
        d.hhat_nnz = static_cast<std::size_t>(nnz);
        la::b200::check(ctx, apf_system_block_info(sys, APF_BLOCK_C, &rows, &cols, &nnz), "apf_system_block_info");
        d.c_signed_nnz = static_cast<std::size_t>(nnz);
        la::b200::check(ctx, apf_system_block_info(sys, APF_BLOCK_BDT, &rows, &cols, &nnz), "apf_system_block_info");
        d.b_or_bdt_nnz_used = static_cast<std::size_t>(nnz);
        d.setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return out;
    }

    // The preconditioned saddle solve on the B200 (the seam of solve_saddle_system.hpp:43-111):
    // MINRES + ParabolicGraphNorm runs on the thread's device system; every other solver
    // request returns nullopt so that the reference's own direct path takes it, as for the
    // Eigen backend.
    template<>
    struct SaddlePreconditionedSolveDispatcher<la::b200::Backend>
    {
        template<class Solver, class Matrix, class Vector, class InitialGuess>
        [[nodiscard]] static std::optional<SaddlePreconditionedSolveResult<la::b200::Backend>> solve(
            Solver& solver, const Matrix& K, const Vector& rhs,
            const la::saddle::SaddlePointBlocks<la::b200::Backend>& blocks,
            const la::concepts::SolverOptions& options, const InitialGuess& initial_guess,
            const SaddlePreconditionerContext<la::b200::Backend>& context)
        {
            static_cast<void>(solver);
            const auto validation = la::concepts::validate_solver_preconditioner(options.solver, options.preconditioner);
            if (!validation.accepted)
                throw std::invalid_argument(validation.rejection_reason);
            if (!is_saddle_preconditioned_solve_requested(options))
                return std::nullopt;
            blocks.validate();
            if (K.rows() != K.cols() || K.rows() != rhs.size())
                throw std::runtime_error(
                    "solve_saddle_system_with_preconditioner: system dimensions are inconsistent.");
            if (initial_guess.has_value() && initial_guess.full_vector->size() != rhs.size())
                throw std::runtime_error("solve_saddle_system_with_preconditioner: initial guess size does not match "
                                         "the full saddle system.");
            if (context.graph_norm == nullptr)
                throw std::runtime_error("solve_saddle_system_with_preconditioner: ParabolicGraphNorm requires "
                                         "graph-norm block context from assembly.");
            auto& s = la::b200::session();
            apf_system* sys = s.system_for(APF_BLOCK_A_Y, blocks.A);
            if (sys == nullptr || s.system_for(APF_BLOCK_B, blocks.B) != sys ||
                s.system_for(APF_BLOCK_C, blocks.C) != sys ||
                s.system_for(APF_BLOCK_HHAT, context.graph_norm->hhat) != sys)
                throw std::invalid_argument(
                    "b200 backend: the saddle blocks and the graph-norm block were not assembled by the b200 backend "
                    "in this thread (include apf_b200_backend.hpp before the reference's solver headers)");
            apf_ctx* ctx = s.context();
            const int n = rhs.size();

            // the right-hand side solved for: b, or b - K x0 for the correction equation
            std::vector<double> b(static_cast<std::size_t>(n)), x0;
            const bool correction = initial_guess.has_value() && initial_guess.solve_correction_equation;
            if (correction)
            {
                const auto r = la::ops::subtract(rhs, la::ops::matvec(K, *initial_guess.full_vector));
                for (int i = 0; i < n; ++i)
                    b[static_cast<std::size_t>(i)] = r[i];
            }
            else
                for (int i = 0; i < n; ++i)
                    b[static_cast<std::size_t>(i)] = rhs[i];
            if (initial_guess.has_value() && !correction)
            {
                x0.resize(static_cast<std::size_t>(n));
                for (int i = 0; i < n; ++i)
                    x0[static_cast<std::size_t>(i)] = (*initial_guess.full_vector)[i];
            }

            const apf_solver_options o = la::b200::detail::minres_options(s, options);
            std::vector<double> x(static_cast<std::size_t>(n));
            apf_solver_diagnostics d{};
            const int rc = apf_solve_minres_with_rhs(ctx, sys, &o, b.data(), x0.empty() ? nullptr : x0.data(),
                                                     x.data(), 0, &d);
            s.set_last_diagnostics(d);
            if (rc != APF_OK && rc != APF_ERR_NOT_CONVERGED)
                la::b200::check(ctx, rc, "apf_solve_minres_with_rhs");

            auto diag = la::b200::detail::solver_diagnostics(s, options, d);
            if (rc == APF_ERR_NOT_CONVERGED)
                throw PreconditionedSolveFailure(apf_ctx_last_error(ctx), diag);

            SaddlePreconditionedSolveResult<la::b200::Backend> result;
            result.solution = typename la::b200::Backend::Vector(n);
            if (correction)
            {
                // the solution is x0 + d; the device system keeps it too (the estimate reads it)
                for (int i = 0; i < n; ++i)
                    x[static_cast<std::size_t>(i)] += (*initial_guess.full_vector)[i];
                la::b200::check(ctx, apf_system_set_solution(ctx, sys, x.data(), 0), "apf_system_set_solution");
            }
            for (int i = 0; i < n; ++i)
                result.solution[i] = x[static_cast<std::size_t>(i)];
            result.diagnostics = std::move(diag);
            result.setup_seconds = d.setup_seconds;
            result.solve_seconds = d.solve_seconds;
            return result;
        }
    };
}

// ---- the inner iteration with the device estimate --------------------------------------
// Declared after the seams above, so that the reference's solver headers included here bind
// to them; the reference's adaptive driver (algorithm/adaptive_driver.hpp), included after
// this header, binds to the overload below.
#include "finite_element/time_slabs/time_slab_adaptive_loop.hpp"
#include "finite_element/geometry/cell_geometry.hpp"
#include "finite_element/io/write_time_slab_flux_reconstruction_samples_binary.hpp"
#include "finite_element/io/write_time_slab_vertex_patches_binary.hpp"

namespace la::b200::detail
{
    // Whether the main solve of an inner iteration can stay on the device: MINRES with the
    // parabolic graph-norm preconditioner and no full-matrix symmetry scan (the reference's
    // Detailed diagnostics mode reads every entry of K on the host).
    [[nodiscard]] inline bool device_main_solve_applies(const la::concepts::SolverOptions& options)
    {
        return la::preconditioners::is_saddle_preconditioned_solve_requested(options) &&
               finite_element::system::detail::diagnostics_mode_with_required_residual(options) !=
                   la::concepts::SolverDiagnosticsMode::Detailed;
    }

    // assemble_and_solve_into_functions (solve_main_system.hpp:1815-2016) for MINRES +
    // ParabolicGraphNorm with every block kept on the device: assembly, the graph-norm block
    // Hhat (from the device's own B_dt and A_x, so the host assembly of both that
    // assemble_parabolic_graph_norm_approximation runs is skipped), the MINRES solve (with
    // the initial guess or the correction equation), and the Summary diagnostics' residuals;
    // only the solution comes back, into lambda_h and u_h.  The blocks are not copied to host
    // matrices and K is not composed on the host.
    template<class Backend, class YSpaceType, class XSpaceType, class ExampleType>
    [[nodiscard]] finite_element::system::SaddleProblemSolveResult<Backend, YSpaceType, XSpaceType>
    device_main_solve(finite_element::Function<YSpaceType, typename Backend::Vector>& lambda_h,
                      finite_element::Function<XSpaceType, typename Backend::Vector>& u_h,
                      const YSpaceType& y_space, const XSpaceType& x_space, const ExampleType& example,
                      const la::concepts::SolverOptions& options, double zero_tol,
                      const finite_element::system::MainSystemInitialGuess<Backend>& initial_guess,
                      const finite_element::detail::TimingRecorder& timing)
    {
        using Clock = std::chrono::steady_clock;
        const int nl = y_space.dof_handler_ref().n_true_dofs();
        const int nu = x_space.dof_handler_ref().n_true_dofs();
        if (nl == 0 || nu == 0)
            throw std::runtime_error("solve_main_system_blocks: refusing to solve main system with zero true DoFs. "
                                     "Y/lambda true DoFs=" + std::to_string(nl) + ", X/u true DoFs=" +
                                     std::to_string(nu) +
                                     ". Refine the mesh or use a space with interior true DoFs.");
        const int n = nl + nu;
        if (initial_guess.has_value() && initial_guess.full_vector->size() != n)
            throw std::runtime_error(
                "solve_main_system_blocks: initial guess size does not match the full saddle system.");
        Session& s = session();
        apf_ctx* ctx = s.context();
        {
            auto total = timing.scoped("main_system.assembly_total_wall");
            auto timer = timing.scoped("assembly.total_seconds");
            const ProblemArrays arrays = [&] {
                auto t = timing.scoped("b200.describe_spaces_wall");
                return describe(y_space, x_space, example, zero_tol, -1.0);
            }();
            auto t = timing.scoped("b200.upload_and_assembly_wall");
            apf_system* sys = nullptr;
            check(ctx, apf_assemble_main_system(ctx, &arrays.desc, 0, &sys), "apf_assemble_main_system");
            s.adopt(sys, zero_tol);
        }
        apf_system* sys = s.system();
        {
            // assemble_parabolic_graph_norm_approximation's default diagonal tolerance
            // (parabolic_graph_norm.hpp:29)
            auto timer = timing.scoped("main_system.construct_graph_norm_context");
            check(ctx, apf_assemble_graph_norm(ctx, sys, 1.0e-14), "apf_assemble_graph_norm");
        }
        std::vector<double> x0;
        if (initial_guess.has_value())
        {
            const auto& g = *initial_guess.full_vector;
            x0.resize(static_cast<std::size_t>(n));
            for (int i = 0; i < n; ++i)
                x0[static_cast<std::size_t>(i)] = g[i];
        }
        const apf_solver_options o = minres_options(s, options);
        std::vector<double> x(static_cast<std::size_t>(n));
        apf_solver_diagnostics d{};
        const auto solve_start = Clock::now();
        const int rc = initial_guess.has_value() && initial_guess.solve_correction_equation
                           ? apf_solve_minres_correction(ctx, sys, &o, x0.data(), x.data(), 0, &d)
                           : apf_solve_minres(ctx, sys, &o, x0.empty() ? nullptr : x0.data(), x.data(), 0, &d);
        timing.add("main_system.solver_total_wall", std::chrono::duration<double>(Clock::now() - solve_start).count());
        s.set_last_diagnostics(d);
        if (rc != APF_OK && rc != APF_ERR_NOT_CONVERGED)
            check(ctx, rc, "apf_solve_minres");
        auto diag = solver_diagnostics(s, options, d);
        if (rc == APF_ERR_NOT_CONVERGED)
            throw la::preconditioners::PreconditionedSolveFailure(apf_ctx_last_error(ctx), diag);

        const auto postprocess_start = Clock::now();
        // the residual diagnostics of solve_main_system_blocks (solve_main_system.hpp:1450-1470)
        auto relative = [](double r, double b) {
            return std::isfinite(r) ? r / (std::isfinite(b) && b > 0.0 ? b : 1.0)
                                    : std::numeric_limits<double>::quiet_NaN();
        };
        if (initial_guess.has_value())
        {
            auto timer = timing.scoped("main_system.correction_or_initial_guess_wall");
            double r0 = 0.0, b = 0.0, g2 = 0.0;
            check(ctx, apf_system_residual_norms(ctx, sys, x0.data(), 0, &r0, &b), "apf_system_residual_norms");
            for (const double v : x0)
                g2 += v * v;
            diag.initial_guess_norm = std::sqrt(g2);
            diag.initial_residual_absolute = r0;
            diag.initial_residual_relative = relative(r0, b);
        }
        if (finite_element::system::detail::diagnostics_mode_with_required_residual(options) !=
            la::concepts::SolverDiagnosticsMode::Off)
        {
            auto timer = timing.scoped("main_system.solver_residual_check_wall");
            double r = 0.0, b = 0.0;
            check(ctx, apf_system_residual_norms(ctx, sys, nullptr, 0, &r, &b), "apf_system_residual_norms");
            diag.linear_residual_absolute = r;
            diag.linear_residual_relative = relative(r, b);
        }
        finite_element::system::SaddleProblemSolveResult<Backend, YSpaceType, XSpaceType> result;
        result.lambda_true = typename Backend::Vector(nl);
        result.u_true = typename Backend::Vector(nu);
        for (int i = 0; i < nl; ++i)
            result.lambda_true[i] = x[static_cast<std::size_t>(i)];
        for (int i = 0; i < nu; ++i)
            result.u_true[i] = x[static_cast<std::size_t>(nl + i)];
        result.solver_diagnostics = std::move(diag);
        result.solver_setup_seconds = d.setup_seconds;
        result.solver_solve_seconds = d.solve_seconds;
        timing.add("main_system.solver_setup", result.solver_setup_seconds);
        timing.add("main_system.solver_solve", result.solver_solve_seconds);
        timing.add("solve.setup_seconds", result.solver_setup_seconds);
        timing.add("solve.factorization_seconds", result.solver_setup_seconds);
        timing.add("solve.backsolve_seconds", result.solver_solve_seconds);
        timing.add("main_system.postprocess_wall",
                   std::chrono::duration<double>(Clock::now() - postprocess_start).count());
        {
            auto timer = timing.scoped("main_system.solution_update_wall");
            auto function_timer = timing.scoped("main_system.function_update_wall");
            lambda_h.update_from_true_solution(result.lambda_true);
            u_h.update_from_true_solution(result.u_true);
        }
        return result;
    }
}

namespace la::b200
{
    // write_time_slab_flux_reconstruction_samples_binary
    // (src/finite_element/io/write_time_slab_flux_reconstruction_samples_binary.hpp:17-174) from
    // the device flux of this thread's last estimate: the reference's file layout and sample
    // lattice, slab cells in the order of the reference's slab space (the host reconstruction's
    // slab_space_ref(), which the driver builds), sample points mapped by the reference's
    // CellGeometry, and sigma_x, sigma_y, div sigma evaluated on the device (apf_flux_sample)
    // on the device cell with the same (slab, source Y cell).
    template<class FluxReconstructionType>
    void write_flux_reconstruction_samples_binary(const FluxReconstructionType& reconstruction,
                                                  const std::filesystem::path& output_dir,
                                                  const std::string& filename = "flux_reconstruction_samples.bin",
                                                  int samples_x_per_cell = 4, int samples_t_per_cell = 4)
    {
        using SlabSpaceType = typename FluxReconstructionType::SlabSpaceType;
        using GT = typename SlabSpaceType::GT;
        using int_t = finite_element::io::detail::binary_int_t;
        namespace iod = finite_element::io::detail;
        static_assert(GT::dim_space_v == 2 && GT::dim_time_v == 1, "flux samples: 2+1D reconstructions");
        if (samples_x_per_cell < 2 || samples_t_per_cell < 2)
            throw std::runtime_error(
                "write_time_slab_flux_reconstruction_samples_binary: need at least 2 samples per direction.");
        Session& s = session();
        apf_ctx* ctx = s.context();
        apf_system* sys = s.system();
        const std::vector<int>& y_cells = s.flux_y_cells();
        int32_t n_kept = 0;
        if (sys != nullptr)
            check(ctx, apf_flux_cells(ctx, sys, &n_kept, nullptr, nullptr), "apf_flux_cells");
        if (sys == nullptr || n_kept == 0 || y_cells.empty())
            throw std::runtime_error("b200 backend: no device flux for the flux samples (the session's last estimate "
                                     "did not keep one: la::b200::session().keep_flux())");
        std::vector<int32_t> kept_slab(static_cast<std::size_t>(n_kept)), kept_source(static_cast<std::size_t>(n_kept));
        check(ctx, apf_flux_cells(ctx, sys, &n_kept, kept_slab.data(), kept_source.data()), "apf_flux_cells");
        auto key = [](long long slab, long long y_cell) { return (slab << 32) | (y_cell & 0xffffffffll); };
        std::unordered_map<long long, int32_t> device_cell;
        device_cell.reserve(static_cast<std::size_t>(n_kept));
        for (int32_t c = 0; c < n_kept; ++c)
            device_cell.emplace(key(kept_slab[static_cast<std::size_t>(c)],
                                    y_cells.at(static_cast<std::size_t>(kept_source[static_cast<std::size_t>(c)]))),
                                c);

        const auto& slab_space = reconstruction.slab_space_ref();
        const int nx = samples_x_per_cell, nt = samples_t_per_cell;
        const int n_spatial = nx * (nx + 1) / 2;
        const auto ref_space = iod::make_triangle_barycentric_lattice_samples(nx);
        const auto ref_time = iod::make_interval_reference_samples(nt);
        std::vector<int_t> slab_ids, slab_cell_ids, source_ids;
        std::vector<int32_t> point_cell;
        std::vector<double> points;
        for (int slab_id = 0; slab_id < slab_space.n_slabs(); ++slab_id)
        {
            const auto& slab = slab_space.slab(slab_id);
            const auto& fes = slab.fespace_ref();
            using Geometry = finite_element::geometry::CellGeometry<std::remove_cvref_t<decltype(fes)>, 2>;
            for (const int slab_cell : slab.active_cells())
            {
                const int source = slab_space.source_cell_id(slab_id, slab_cell);
                const auto it = device_cell.find(key(slab_id, source));
                if (it == device_cell.end())
                    throw std::runtime_error("b200 backend: slab " + std::to_string(slab_id) + " cell of source Y cell " +
                                             std::to_string(source) + " has no device flux (the estimate's slabs "
                                             "differ from the reconstruction's)");
                slab_ids.push_back(static_cast<int_t>(slab_id));
                slab_cell_ids.push_back(static_cast<int_t>(slab_cell));
                source_ids.push_back(static_cast<int_t>(source));
                const auto geom = Geometry::make(fes, slab_cell);
                for (int jt = 0; jt < nt; ++jt)
                    for (int is = 0; is < n_spatial; ++is)
                    {
                        const auto p = Geometry::map_to_physical(
                            geom, {ref_space[2 * static_cast<std::size_t>(is)],
                                   ref_space[2 * static_cast<std::size_t>(is) + 1], ref_time[static_cast<std::size_t>(jt)]});
                        points.insert(points.end(), {p[0], p[1], p[2]});
                        point_cell.push_back(it->second);
                    }
            }
        }
        if (point_cell.size() > static_cast<std::size_t>(std::numeric_limits<int32_t>::max()))
            throw std::runtime_error("b200 backend: too many flux sample points for one apf_flux_sample call");
        std::vector<double> values(points.size());
        check(ctx, apf_flux_sample(ctx, sys, static_cast<int32_t>(point_cell.size()), point_cell.data(), points.data(),
                                   values.data(), 0),
              "apf_flux_sample");

        auto file = iod::open_binary_output(output_dir, filename, "write_time_slab_flux_reconstruction_samples_binary");
        const auto header = iod::make_versioned_header(
            iod::time_slab_flux_reconstruction_samples_binary_format_version, static_cast<int_t>(slab_space.n_slabs()),
            static_cast<int_t>(slab_ids.size()), static_cast<int_t>(GT::dim_space_v),
            static_cast<int_t>(GT::dim_time_v), static_cast<int_t>(nx), static_cast<int_t>(nt),
            static_cast<int_t>(n_spatial), static_cast<int_t>(n_spatial * nt), static_cast<int_t>(3),
            iod::function_sample_layout_triangle_barycentric_time);
        const char* what = "write_time_slab_flux_reconstruction_samples_binary";
        iod::write_binary_block(file, header, what);
        iod::write_binary_block(file, slab_ids, what);
        iod::write_binary_block(file, slab_cell_ids, what);
        iod::write_binary_block(file, source_ids, what);
        iod::write_binary_block(file, ref_space, what);
        iod::write_binary_block(file, ref_time, what);
        iod::write_binary_block(file, values, what);
    }
}

namespace adaptive_algorithm::output::detail
{
    // The driver's time-slab estimator snapshot (algorithm/output/iteration_snapshot_writer.hpp:
    // 143-170) for a b200 iteration state: the vertex patches by the reference's writer (host
    // topology, which the drop-in's inner iteration builds), the flux samples from the device
    // flux (its host reconstruction holds no patch solutions).  More specialised than the
    // reference's template, so the driver's call binds here for la::b200::Backend only.
    template<class XSpaceType, class YSpaceType>
    void write_time_slab_estimator_diagnostics_snapshot(
        const finite_element::time_slabs::AdaptiveTestSpaceIterationState<la::b200::Backend, XSpaceType, YSpaceType>&
            state,
        const std::filesystem::path& output_dir)
    {
        using GT = typename YSpaceType::GT;
        if constexpr (GT::dim_space_v == 2 && GT::dim_time_v == 1)
        {
            if (!state.flux_reconstruction.has_value())
                return;
            std::filesystem::create_directories(output_dir);
            finite_element::io::write_time_slab_vertex_patches_binary(state.flux_reconstruction->patch_set(), output_dir,
                                                                     "time_slab_vertex_patches.bin");
            la::b200::write_flux_reconstruction_samples_binary(*state.flux_reconstruction, output_dir,
                                                               "flux_reconstruction_samples.bin", 4, 4);
        }
    }
}

namespace finite_element::time_slabs
{
    // compute_adaptive_test_space_iteration (time_slab_adaptive_loop.hpp:727) on the B200: the
    // main solve through the b200 seams above, the estimate by apf_estimate in place of the
    // reference's host slab reconstruction, patch flux solves and indicators
    // (la::b200::estimate), then the reference's own combination, divergence check and
    // Doerfler marking.  The state's slab space and vertex-patch set are still built on the
    // host (their initialize() without any solve) because the driver reads n_slabs(),
    // n_patches() and copied_slab_cells() from them; lambda_tilde() is not reconstructed on
    // the host (the device estimate holds it).
    template<int QSpace, int QTime, class Backend, class XSpaceType, class YSpaceType, class ExampleType>
        requires std::same_as<Backend, la::b200::Backend>
    [[nodiscard]] AdaptiveTestSpaceIterationState<Backend, XSpaceType, YSpaceType> compute_adaptive_test_space_iteration(
        const YSpaceType& y_space, const XSpaceType& x_space, const ExampleType& example,
        typename Backend::Solver& solver, const la::concepts::SolverOptions& main_solver_options = {},
        const AdaptiveTestSpaceIterationParameters<Backend, XSpaceType, YSpaceType>& parameters = {},
        const la::concepts::SolverOptions& local_solver_options = la::concepts::make_sparse_lu_solver_options(),
        const AdaptiveTestSpaceSolutionSnapshot<Backend, XSpaceType, YSpaceType>* initial_guess_snapshot = nullptr)
    {
        static_cast<void>(local_solver_options);
        AdaptiveTestSpaceIterationState<Backend, XSpaceType, YSpaceType> state(y_space, x_space);
        {
            std::optional<typename Backend::Vector> guess_vector;
            finite_element::system::MainSystemInitialGuess<Backend> guess;
            if (initial_guess_snapshot != nullptr &&
                (parameters.use_adaptive_initial_guess || parameters.solve_main_system_correction))
            {
                guess_vector = finite_element::system::make_saddle_initial_guess_vector<Backend>(
                    initial_guess_snapshot->lambda_delta, initial_guess_snapshot->u_delta, y_space, x_space);
                guess.full_vector = &*guess_vector;
                guess.solve_correction_equation = parameters.solve_main_system_correction;
            }
            const auto main_solve =
                la::b200::detail::device_main_solve_applies(main_solver_options)
                    ? la::b200::detail::device_main_solve<Backend>(state.lambda_delta, state.u_delta, y_space,
                                                                   x_space, example, main_solver_options,
                                                                   parameters.zero_tol, guess, parameters.timing)
                    : finite_element::system::assemble_and_solve_into_functions<QSpace, QTime, Backend>(
                          state.lambda_delta, state.u_delta, y_space, x_space, example, solver,
                          main_solver_options, parameters.zero_tol, -1.0, guess,
                          static_cast<const finite_element::system::MainSystemTwoLevelHierarchy<YSpaceType,
                                                                                                XSpaceType>*>(nullptr),
                          parameters.timing);
            state.main_solve_diagnostics = main_solve.solver_diagnostics;
            state.main_solve_setup_seconds = main_solve.solver_setup_seconds;
            state.main_solve_solve_seconds = main_solve.solver_solve_seconds;
        }
        // host structures the driver reads (no solves)
        state.slab_reconstruction.emplace(y_space, x_space);
        state.slab_reconstruction->initialize(0.0, parameters.timing);
        state.flux_reconstruction.emplace(state.slab_reconstruction->slab_space_ref(), x_space);
        state.flux_reconstruction->initialize();
        // the estimate on the device, in the reference's types
        auto est = la::b200::estimate(y_space);
        state.flux_diagnostics = std::move(est.flux);
        state.reconstruction_y_squared = std::move(est.reconstruction_y_squared);
        state.estimator = std::move(est.estimator);
        const double div2 = state.estimator.divergence_residual_total();
        state.divergence_residual_l2 = std::sqrt(div2 > 0.0 ? div2 : 0.0);
        if (parameters.check_divergence_residual &&
            state.divergence_residual_l2 > parameters.divergence_residual_l2_tolerance)
            throw std::runtime_error("compute_adaptive_test_space_iteration: divergence residual L2 norm " +
                                     std::to_string(state.divergence_residual_l2) + " exceeds tolerance " +
                                     std::to_string(parameters.divergence_residual_l2_tolerance) + ".");
        DoerflerMarkingDiagnostics diagnostics;
        state.marked_source_cells = state.estimator.doerfler_marking_deterministic(
            parameters.doerfler_theta, parameters.doerfler_near_tie_tolerance, &diagnostics, parameters.timing);
        return state;
    }
}
