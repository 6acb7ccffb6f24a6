// Test program of the C++ drop-in (include/apf_b200_backend.hpp), built against the
// reference's own templates (with oracle/shim standing in for the Eigen wrapper layer, as for
// the oracle driver) and linked with libapf_b200.  It runs the reference's OWN callers with
// la::b200::Backend and compares them with the same callers on the reference's Eigen backend:
//
//   blocks <p> <levels> <example>
//       finite_element::system::assemble_main_system_blocks and
//       finite_element::assembly::assemble_parabolic_graph_norm_approximation with both backends
//       (src/finite_element/system/assemble_saddle_problem.hpp:131,
//        src/finite_element/assembly/main_system/parabolic_graph_norm.hpp:13): pattern and
//       value differences of A_y, B, C_signed, f, g and Hhat;
//   solve <p> <levels> <example> <tol>
//       finite_element::system::assemble_and_solve_into_functions
//       (src/finite_element/system/solve_main_system.hpp:1816) with MINRES + ParabolicGraphNorm on
//       la::b200::Backend; the FP64 true residual of its solution against the Eigen backend's K,
//       and its distance to the Eigen backend's direct solution;
//   cycle <p> <levels> <example> <passes> <tol>
//       the reference's inner loop, `passes` times: compute_adaptive_test_space_iteration
//       (src/finite_element/time_slabs/time_slab_adaptive_loop.hpp:727) and
//       refine_test_space_from_marked_source_cells (:2147-2186), once with la::b200::Backend
//       (device assembly, graph-norm block, MINRES and estimate; the reference's marking and
//       refinement) and once with the Eigen backend and its direct solver, each on its own
//       copy of the spaces; per pass the estimator totals, the marked cells of each run and the
//       Y meshes (both refined by the direct-solve run's marks);
//   estimate <p> <levels> <example> <tol>
//       after one pass of the reference's inner loop (Y finer than X): the device estimate in
//       the reference's types (la::b200::estimate) on the b200 solve against the reference's
//       host estimate on its direct solve -- per-cell flux^2 / recon^2 / eta^2, totals, slab
//       count and the Doerfler marking of each;
//   snapshot <p> <levels> <example> <tol> <outdir>
//       after one pass of the reference's inner loop (Y finer than X): the driver's time-slab
//       estimator snapshot (algorithm/output/iteration_snapshot_writer.hpp:143-170) of the
//       Eigen backend's iteration state into <outdir>/eigen and of the b200 state (flux
//       samples from the device flux) into <outdir>/b200;
//   adaptive <p> <levels> <example> <outer_cycles> <tol> [compare:1|0] [guess:0|1|2]
//       the reference's whole adaptive algorithm (adaptive_algorithm::run_adaptive_driver,
//       algorithm/adaptive_driver.hpp:3508) with each backend, each on its own spaces: per outer
//       cycle the X and Y DOF counts, the number of inner Y iterations and the estimator totals
//       (compare = 0: the b200 backend only; guess = 1: the previous solution as initial guess,
//       2: the correction equation).
//
// <p> = 1d runs the blocks / solve / cycle / estimate modes on the reference's 1+1D P1
// configuration (its 1D example on the unit space-time mesh).
// The adaptive-mesh options of the oracle driver (APF_REF_X_POINTS, APF_REF_X_ROUNDS,
// APF_REF_KAPPA, APF_REF_KAPPA_BLOCKS, APF_REF_DRIVER_OUTER) apply to all modes.  Each mode prints one JSON line.
#include "apf_b200_backend.hpp" // before the reference's solver headers (see its header comment)

#include <algorithm>
#include <chrono>
#include <cmath>
#include <iterator>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "algorithm/adaptive_driver.hpp"
#include "algorithm/example_registry.hpp"
#include "algorithm/examples/space_time_2d/initial_data_2d_examples.hpp"
#include "algorithm/examples/space_time_2d/space_time_2d_example.hpp"
#include "finite_element/assembly/main_system/parabolic_graph_norm.hpp"
#include "finite_element/fespace/fe_traits.hpp"
#include "finite_element/fespace/fespace.hpp"
#include "finite_element/fespace/policies.hpp"
#include "finite_element/system/solve_main_system.hpp"
#include "finite_element/time_slabs/time_slab_adaptive_loop.hpp"
#include "mesh/mesh_traits.hpp"

#include "ref_meshes.hpp"

namespace
{
    using EigenB = la::eigen::Backend;
    using B200 = la::b200::Backend;

    // CSR triplets of a host matrix, sorted by (row, col)
    struct Entries
    {
        std::vector<long long> key;
        std::vector<double> val;
    };

    template<class M>
    Entries entries(const M& A)
    {
        std::vector<std::pair<long long, double>> t;
        A.for_each_nonzero([&](int i, int j, double v) {
            t.emplace_back(static_cast<long long>(i) * A.cols() + j, v);
        });
        std::sort(t.begin(), t.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        Entries e;
        for (const auto& [k, v] : t)
        {
            e.key.push_back(k);
            e.val.push_back(v);
        }
        return e;
    }

    // {"pattern_equal": ..., "max_abs_diff_over_max": ..., "nnz": ...}; with residue > 0, entries
    // below residue * max|A| on one side only are not counted as pattern differences
    template<class M>
    std::string compare(const M& ref, const M& mine, double residue = 0.0)
    {
        const Entries a = entries(ref), b = entries(mine);
        double scale = 0.0;
        for (const double v : a.val)
            scale = std::max(scale, std::abs(v));
        std::size_t i = 0, j = 0, only = 0;
        double diff = 0.0;
        while (i < a.key.size() || j < b.key.size())
        {
            if (j == b.key.size() || (i < a.key.size() && a.key[i] < b.key[j]))
            {
                if (std::abs(a.val[i]) > residue * scale)
                    ++only;
                diff = std::max(diff, std::abs(a.val[i]));
                ++i;
            }
            else if (i == a.key.size() || b.key[j] < a.key[i])
            {
                if (std::abs(b.val[j]) > residue * scale)
                    ++only;
                diff = std::max(diff, std::abs(b.val[j]));
                ++j;
            }
            else
            {
                diff = std::max(diff, std::abs(a.val[i] - b.val[j]));
                ++i;
                ++j;
            }
        }
        char buf[256];
        std::snprintf(buf, sizeof(buf),
                      "{\"rows\": %d, \"nnz_ref\": %zu, \"nnz_b200\": %zu, \"pattern_mismatches\": %zu, "
                      "\"max_abs_diff_over_max\": %.3e}",
                      ref.rows(), a.key.size(), b.key.size(), only, scale > 0.0 ? diff / scale : diff);
        return buf;
    }

    template<class V>
    double vec_diff(const V& a, const V& b)
    {
        double d = 0.0, s = 0.0;
        for (int i = 0; i < a.size(); ++i)
        {
            d = std::max(d, std::abs(a[i] - b[i]));
            s = std::max(s, std::abs(a[i]));
        }
        return s > 0.0 ? d / s : d;
    }

    template<int P>
    struct Spaces
    {
        using GT = mesh::MeshTraits<2>;
        using FET = finite_element::FiniteElementTraits<GT, P, P>;
        using XSpace = finite_element::FESpace<GT, FET, finite_element::SpaceTimePolicy>;
        using YSpace = finite_element::FESpace<GT, FET, finite_element::SpaceOnlyPolicy>;
        static constexpr int QSpace = 4 * P + 1;
        static constexpr int QTime = 2 * P + 1;
        static constexpr int P_ = P;

        decltype(adaptive_algorithm::examples::make_2d_example(std::string{})) example;
        decltype(adaptive_algorithm::examples::make_initial_mesh_from_example(example)) mesh;
        XSpace x_space;
        YSpace y_space;

        Spaces(const std::string& name, int levels)
            : example(adaptive_algorithm::examples::make_2d_example(name)),
              mesh(adaptive_algorithm::examples::make_initial_mesh_from_example(example)),
              x_space(mesh),
              y_space(mesh)
        {
            adaptive_algorithm::examples::initialize_spaces_from_example(x_space, y_space, example);
            for (int k = 0; k < levels; ++k)
                apf_oracle::uniform_isotropic_refine(x_space);
            (void)apf_oracle::apply_adaptive_options_2d(x_space, example);
            y_space.initialize(x_space.active_cells());
            if (const int outer = apf_oracle::env_int("APF_REF_DRIVER_OUTER", 0); outer > 0)
            {
                // the mesh of the reference's adaptive driver after `outer` cycles (Eigen backend)
                typename la::eigen::Backend::Solver solver;
                la::concepts::SolverOptions opts;
                adaptive_algorithm::AdaptiveParameters par;
                par.max_outer_iterations = outer;
                par.polynomial_degree = P;
                par.output.print_iteration_tables = false;
                par.output.save_mesh_statistics = false;
                par.output.stream = &std::cerr;
                (void)adaptive_algorithm::run_adaptive_driver<QSpace, QTime, la::eigen::Backend>(
                    x_space, y_space, example.problem, solver, opts, par);
            }
        }
    };

    // 1+1D P1: the reference's 1D example on its unit space-time mesh, `levels` uniform outer
    // refinements, Gauss orders QSpace = QTime = 3 (the runner's 1+1D configuration)
    struct Spaces1D
    {
        using GT = mesh::MeshTraits<1>;
        using FET = finite_element::FiniteElementTraits<GT, 1, 1>;
        using XSpace = finite_element::FESpace<GT, FET, finite_element::SpaceTimePolicy>;
        using YSpace = finite_element::FESpace<GT, FET, finite_element::SpaceOnlyPolicy>;
        static constexpr int QSpace = 3;
        static constexpr int QTime = 3;
        static constexpr int P_ = 1;

        decltype(adaptive_algorithm::examples::make_1d_example(std::string{})) example;
        decltype(adaptive_algorithm::support::make_unit_mesh<GT>()) mesh;
        XSpace x_space;
        YSpace y_space;

        Spaces1D(const std::string& name, int levels)
            : example(adaptive_algorithm::examples::make_1d_example(name)),
              mesh(adaptive_algorithm::support::make_unit_mesh<GT>()),
              x_space(mesh),
              y_space(mesh)
        {
            adaptive_algorithm::examples::initialize_spaces_from_example(x_space, y_space, example);
            for (int k = 0; k < levels; ++k)
                apf_oracle::uniform_isotropic_refine(x_space);
            y_space.initialize(x_space.active_cells());
        }
    };

    la::concepts::SolverOptions minres_options(double tol)
    {
        la::concepts::SolverOptions o;
        o.solver = la::concepts::SolverType::MINRES;
        o.preconditioner = la::concepts::PreconditionerType::ParabolicGraphNorm;
        o.tolerance = tol;
        o.max_iterations = 20000;
        return o;
    }

    template<class S>
    int run_blocks(int levels, const std::string& name)
    {
        S s(name, levels);
        constexpr int P = S::P_;
        const auto ref = finite_element::system::assemble_main_system_blocks<S::QSpace, S::QTime, EigenB>(
            s.y_space, s.x_space, s.example.problem, 1e-15, -1.0);
        const auto mine = finite_element::system::assemble_main_system_blocks<S::QSpace, S::QTime, B200>(
            s.y_space, s.x_space, s.example.problem, 1e-15, -1.0);
        const auto gn_ref = finite_element::assembly::assemble_parabolic_graph_norm_approximation<S::QSpace, S::QTime,
                                                                                                  EigenB>(
            s.y_space, s.x_space, s.example.problem.M, ref.A_y(), ref.C_signed(), 1e-15, 1e-14);
        const auto gn_mine = finite_element::assembly::assemble_parabolic_graph_norm_approximation<S::QSpace, S::QTime,
                                                                                                   B200>(
            s.y_space, s.x_space, s.example.problem.M, mine.A_y(), mine.C_signed(), 1e-15, 1e-14);
        std::printf("{\"mode\": \"blocks\", \"p\": %d, \"levels\": %d, \"n_lambda\": %d, \"n_u\": %d, \"A_y\": %s, "
                    "\"B\": %s, \"C_signed\": %s, \"Hhat\": %s, \"Hhat_residue_1e-13\": %s, \"f\": %.3e, "
                    "\"g\": %.3e}\n",
                    P, levels, ref.n_lambda(), ref.n_u(), compare(ref.A_y(), mine.A_y()).c_str(),
                    compare(ref.lower_left_B(), mine.lower_left_B()).c_str(),
                    compare(ref.C_signed(), mine.C_signed()).c_str(),
                    compare(gn_ref.approximation.hhat, gn_mine.approximation.hhat).c_str(),
                    compare(gn_ref.approximation.hhat, gn_mine.approximation.hhat, 1e-13).c_str(),
                    vec_diff(ref.f(), mine.f()), vec_diff(ref.g(), mine.g()));
        return 0;
    }

    template<class S>
    int run_solve(int levels, const std::string& name, double tol)
    {
        S s(name, levels);
        constexpr int P = S::P_;
        using XSpace = typename S::XSpace;
        using YSpace = typename S::YSpace;
        // the Eigen backend's K, rhs and direct solution
        const auto ref = finite_element::system::assemble_main_system_blocks<S::QSpace, S::QTime, EigenB>(
            s.y_space, s.x_space, s.example.problem, 1e-15, -1.0);
        const auto full = ref.make_full_system(false);
        typename EigenB::Solver direct;
        la::concepts::SolverOptions lu;
        lu.solver = la::concepts::SolverType::SparseLU;
        direct.compute(full.matrix, lu);
        typename EigenB::Vector x_direct;
        direct.solve(full.rhs, x_direct);

        finite_element::Function<YSpace, typename B200::Vector> lambda_h(s.y_space);
        finite_element::Function<XSpace, typename B200::Vector> u_h(s.x_space);
        typename B200::Solver solver;
        const auto result = finite_element::system::assemble_and_solve_into_functions<S::QSpace, S::QTime, B200>(
            lambda_h, u_h, s.y_space, s.x_space, s.example.problem, solver, minres_options(tol));
        const int nl = result.lambda_true.size(), nu = result.u_true.size();
        typename EigenB::Vector x(nl + nu);
        for (int i = 0; i < nl; ++i)
            x[i] = result.lambda_true[i];
        for (int i = 0; i < nu; ++i)
            x[nl + i] = result.u_true[i];
        const auto Kx = la::ops::matvec(full.matrix, x);
        double rr = 0.0, bb = 0.0, dd = 0.0, xs = 0.0;
        for (int i = 0; i < nl + nu; ++i)
        {
            rr += (full.rhs[i] - Kx[i]) * (full.rhs[i] - Kx[i]);
            bb += full.rhs[i] * full.rhs[i];
            dd = std::max(dd, std::abs(x[i] - x_direct[i]));
            xs = std::max(xs, std::abs(x_direct[i]));
        }
        const auto& d = result.solver_diagnostics;
        const auto& last = la::b200::session().last_diagnostics();
        std::printf("{\"mode\": \"solve\", \"p\": %d, \"levels\": %d, \"n\": %d, \"tol\": %.1e, "
                    "\"effective_solver_minres\": %d, \"iterative\": %d, \"iterations\": %d, \"converged\": %d, "
                    "\"reported_true_residual\": %.6e, \"host_true_residual\": %.6e, "
                    "\"max_diff_to_direct_over_max\": %.3e, \"device_iterations\": %d}\n",
                    P, levels, nl + nu, tol,
                    d.effective_solver == la::concepts::SolverType::MINRES ? 1 : 0, d.iterative ? 1 : 0,
                    d.iterative_stats.iterations.value_or(-1), d.iterative_stats.converged.value_or(false) ? 1 : 0,
                    d.iterative_stats.final_true_residual.value_or(-1.0), std::sqrt(rr / bb), dd / xs,
                    last.iterations);
        return 0;
    }

    template<class S>
    int run_cycle(int levels, const std::string& name, int passes, double tol)
    {
        constexpr int P = S::P_;
        using XSpace = typename S::XSpace;
        using YSpace = typename S::YSpace;
        S a(name, levels), b(name, levels); // a: b200 backend, b: Eigen backend with its direct solver
        std::printf("{\"mode\": \"cycle\", \"p\": %d, \"levels\": %d, \"tol\": %.1e, \"passes\": [", P, levels, tol);
        for (int pass = 0; pass < passes; ++pass)
        {
            typename B200::Solver sa;
            finite_element::time_slabs::AdaptiveTestSpaceIterationParameters<B200, XSpace, YSpace> pa;
            const auto st_a = finite_element::time_slabs::compute_adaptive_test_space_iteration<S::QSpace, S::QTime,
                                                                                                B200>(
                a.y_space, a.x_space, a.example.problem, sa, minres_options(tol), pa);
            typename EigenB::Solver sb;
            la::concepts::SolverOptions lu;
            lu.solver = la::concepts::SolverType::SparseLU;
            finite_element::time_slabs::AdaptiveTestSpaceIterationParameters<EigenB, XSpace, YSpace> pb;
            const auto st_b = finite_element::time_slabs::compute_adaptive_test_space_iteration<S::QSpace, S::QTime,
                                                                                                EigenB>(
                b.y_space, b.x_space, b.example.problem, sb, lu, pb);
            const double fa = st_a.flux_diagnostics.total_flux(), fb = st_b.flux_diagnostics.total_flux();
            // marked cells of the two runs (Doerfler marking: cells whose indicators tie at the
            // threshold may fall either way under rounding differences)
            std::vector<int> ma(st_a.marked_source_cells.begin(), st_a.marked_source_cells.end());
            std::vector<int> mb(st_b.marked_source_cells.begin(), st_b.marked_source_cells.end());
            std::sort(ma.begin(), ma.end());
            std::sort(mb.begin(), mb.end());
            std::vector<int> sym;
            std::set_symmetric_difference(ma.begin(), ma.end(), mb.begin(), mb.end(), std::back_inserter(sym));
            const auto ny_a = a.y_space.active_cells().size(), ny_b = b.y_space.active_cells().size();
            const auto& d = st_a.main_solve_diagnostics;
            std::printf("%s{\"pass\": %d, \"y_cells\": [%zu, %zu], \"flux_b200\": %.15e, \"flux_direct\": %.15e, "
                        "\"marked\": [%zu, %zu], \"marked_symmetric_difference\": %zu, \"minres_iterations\": %d, "
                        "\"minres_true_residual\": %.3e}",
                        pass ? ", " : "", pass, ny_a, ny_b, fa, fb, ma.size(), mb.size(), sym.size(),
                        d.iterative_stats.iterations.value_or(-1),
                        d.iterative_stats.final_true_residual.value_or(-1.0));
            // both test spaces refined by the direct-solve run's marks, so that the next pass
            // compares the two backends on the same meshes
            finite_element::time_slabs::refine_test_space_from_marked_source_cells(a.y_space, a.x_space,
                                                                                   st_b.marked_source_cells);
            finite_element::time_slabs::refine_test_space_from_marked_source_cells(b.y_space, b.x_space,
                                                                                   st_b.marked_source_cells);
        }
        std::printf("], \"device_estimates\": %lld}\n", la::b200::session().device_estimates());
        return 0;
    }

    // the device estimate in the reference's types (la::b200::estimate) against the reference's
    // host estimate, after one pass of the reference's inner loop (Y finer than X, Y cells
    // across several slabs): per source Y cell flux^2, recon^2 and eta^2, totals, the slab
    // count and the Doerfler marking of the two estimates
    template<class S>
    int run_estimate(int levels, const std::string& name, double tol)
    {
        constexpr int P = S::P_;
        using XSpace = typename S::XSpace;
        using YSpace = typename S::YSpace;
        S a(name, levels), b(name, levels);
        la::concepts::SolverOptions lu;
        lu.solver = la::concepts::SolverType::SparseLU;
        finite_element::time_slabs::AdaptiveTestSpaceIterationParameters<EigenB, XSpace, YSpace> pb;
        {
            typename EigenB::Solver s0;
            const auto st0 = finite_element::time_slabs::compute_adaptive_test_space_iteration<S::QSpace, S::QTime,
                                                                                               EigenB>(
                b.y_space, b.x_space, b.example.problem, s0, lu, pb);
            finite_element::time_slabs::refine_test_space_from_marked_source_cells(a.y_space, a.x_space,
                                                                                   st0.marked_source_cells);
            finite_element::time_slabs::refine_test_space_from_marked_source_cells(b.y_space, b.x_space,
                                                                                   st0.marked_source_cells);
        }
        typename EigenB::Solver sb;
        const auto ref = finite_element::time_slabs::compute_adaptive_test_space_iteration<S::QSpace, S::QTime, EigenB>(
            b.y_space, b.x_space, b.example.problem, sb, lu, pb);
        finite_element::Function<YSpace, typename B200::Vector> lambda_h(a.y_space);
        finite_element::Function<XSpace, typename B200::Vector> u_h(a.x_space);
        typename B200::Solver sa;
        (void)finite_element::system::assemble_and_solve_into_functions<S::QSpace, S::QTime, B200>(
            lambda_h, u_h, a.y_space, a.x_space, a.example.problem, sa, minres_options(tol));
        const auto dev = la::b200::estimate(a.y_space);
        double scale = 0.0, d_flux = 0.0, d_recon = 0.0, d_eta = 0.0;
        for (const auto& [c, v] : ref.estimator.estimator_squared.by_source_cell)
            scale = std::max(scale, std::abs(v));
        for (const auto& [c, v] : ref.estimator.estimator_squared.by_source_cell)
        {
            d_eta = std::max(d_eta, std::abs(v - dev.estimator.estimator_squared.by_source_cell.at(c)));
            d_flux = std::max(d_flux, std::abs(ref.flux_diagnostics.by_source_cell_flux.at(c) -
                                               dev.flux.by_source_cell_flux.at(c)));
            d_recon = std::max(d_recon, std::abs(ref.reconstruction_y_squared.by_source_cell.at(c) -
                                                 dev.reconstruction_y_squared.by_source_cell.at(c)));
        }
        std::vector<int> ma = dev.estimator.doerfler_marking_deterministic(pb.doerfler_theta, pb.doerfler_near_tie_tolerance);
        std::vector<int> mb(ref.marked_source_cells.begin(), ref.marked_source_cells.end());
        std::sort(ma.begin(), ma.end());
        std::sort(mb.begin(), mb.end());
        std::vector<int> sym;
        std::set_symmetric_difference(ma.begin(), ma.end(), mb.begin(), mb.end(), std::back_inserter(sym));
        std::printf("{\"mode\": \"estimate\", \"p\": %d, \"levels\": %d, \"y_cells\": %zu, \"x_cells\": %zu, "
                    "\"cells_compared\": %zu, \"n_slabs\": [%d, %d], \"eta_total\": [%.15e, %.15e], "
                    "\"flux_total\": [%.15e, %.15e], \"recon_total\": [%.15e, %.15e], "
                    "\"max_cell_diff_over_max_eta\": {\"flux\": %.3e, \"recon\": %.3e, \"eta\": %.3e}, "
                    "\"marked\": [%zu, %zu], \"marked_symmetric_difference\": %zu}\n",
                    P, levels, a.y_space.active_cells().size(), a.x_space.active_cells().size(),
                    ref.estimator.estimator_squared.by_source_cell.size(), dev.n_slabs, ref.n_slabs(),
                    dev.estimator.total(), ref.estimator.total(), dev.flux.total_flux(), ref.flux_diagnostics.total_flux(),
                    dev.reconstruction_y_squared.total(), ref.reconstruction_y_squared.total(), d_flux / scale,
                    d_recon / scale, d_eta / scale, ma.size(), mb.size(), sym.size());
        return 0;
    }

    // the driver's time-slab estimator snapshot after one pass of the inner loop (Y finer than
    // X): the reference's writer on the Eigen backend's state (host patch solves) into
    // <outdir>/eigen, the b200 overload (device flux) into <outdir>/b200, each on its own copy
    // of the same spaces
    template<class S>
    int run_snapshot(int levels, const std::string& name, double tol, const std::string& outdir)
    {
        using XSpace = typename S::XSpace;
        using YSpace = typename S::YSpace;
        S a(name, levels), b(name, levels);
        la::concepts::SolverOptions lu;
        lu.solver = la::concepts::SolverType::SparseLU;
        finite_element::time_slabs::AdaptiveTestSpaceIterationParameters<EigenB, XSpace, YSpace> pb;
        {
            typename EigenB::Solver s0;
            const auto st0 = finite_element::time_slabs::compute_adaptive_test_space_iteration<S::QSpace, S::QTime,
                                                                                               EigenB>(
                b.y_space, b.x_space, b.example.problem, s0, lu, pb);
            finite_element::time_slabs::refine_test_space_from_marked_source_cells(a.y_space, a.x_space,
                                                                                   st0.marked_source_cells);
            finite_element::time_slabs::refine_test_space_from_marked_source_cells(b.y_space, b.x_space,
                                                                                   st0.marked_source_cells);
        }
        typename EigenB::Solver sb;
        const auto ref = finite_element::time_slabs::compute_adaptive_test_space_iteration<S::QSpace, S::QTime, EigenB>(
            b.y_space, b.x_space, b.example.problem, sb, lu, pb);
        finite_element::time_slabs::AdaptiveTestSpaceIterationParameters<B200, XSpace, YSpace> pa;
        typename B200::Solver sa;
        const auto dev = finite_element::time_slabs::compute_adaptive_test_space_iteration<S::QSpace, S::QTime, B200>(
            a.y_space, a.x_space, a.example.problem, sa, minres_options(tol), pa);
        adaptive_algorithm::output::detail::write_time_slab_estimator_diagnostics_snapshot(ref, outdir + "/eigen");
        adaptive_algorithm::output::detail::write_time_slab_estimator_diagnostics_snapshot(dev, outdir + "/b200");
        std::printf("{\"mode\": \"snapshot\", \"p\": %d, \"levels\": %d, \"y_cells\": %zu, \"x_cells\": %zu, "
                    "\"n_slabs\": [%d, %d], \"device_estimates\": %lld}\n",
                    S::P_, levels, a.y_space.active_cells().size(), a.x_space.active_cells().size(), dev.n_slabs(),
                    ref.n_slabs(), la::b200::session().device_estimates());
        return 0;
    }

    // the reference's whole adaptive algorithm (run_adaptive_driver, algorithm/adaptive_driver.hpp:3508)
    // with each backend: outer cycles of inner Y loops (solve, estimate, Doerfler marking, Y
    // refinement) and X marking + refinement
    template<int P>
    int run_adaptive(int levels, const std::string& name, int outer, double tol, bool compare, int guess)
    {
        using S = Spaces<P>;
        S a(name, levels), b(name, levels);
        adaptive_algorithm::AdaptiveParameters par;
        par.max_outer_iterations = outer;
        par.polynomial_degree = P;
        par.output.print_iteration_tables = !compare; // progress on stderr for long runs
        par.output.save_mesh_statistics = false;
        par.output.stream = &std::cerr;
        // guess 1: the previous inner iteration's solution as MINRES's initial guess;
        // 2: the correction equation K d = b - K x0 (MainSystemInitialGuess)
        par.use_adaptive_initial_guess = guess >= 1;
        par.solve_main_system_correction = guess == 2;
        par.timing.enabled = !compare; // the driver's own phase timing for the b200-only run
        if (const char* e = std::getenv("APF_DROPIN_AMG_STRENGTH"))
            la::b200::session().solver_options().amg_strength = std::atof(e);
        // the learned preconditioner (plain fallback) from the shipped raw parameters
        if (const char* e = std::getenv("APF_DROPIN_LEARNED_PARAMS"))
            la::b200::session().use_learned_model(e);
        const auto t0 = std::chrono::steady_clock::now();
        typename B200::Solver sa;
        const auto ra = adaptive_algorithm::run_adaptive_driver<S::QSpace, S::QTime, B200>(
            a.x_space, a.y_space, a.example.problem, sa, minres_options(tol), par);
        const auto t1 = std::chrono::steady_clock::now();
        typename EigenB::Solver sb;
        la::concepts::SolverOptions lu;
        lu.solver = la::concepts::SolverType::SparseLU;
        par.max_outer_iterations = compare ? outer : 0;
        const auto rb = adaptive_algorithm::run_adaptive_driver<S::QSpace, S::QTime, EigenB>(
            b.x_space, b.y_space, b.example.problem, sb, lu, par);
        const auto t2 = std::chrono::steady_clock::now();
        auto dump = [](const auto& r) {
            std::string out = "[";
            for (std::size_t k = 0; k < r.outer_iterations.size(); ++k)
            {
                const auto& o = r.outer_iterations[k];
                char buf[512];
                std::snprintf(buf, sizeof(buf),
                              "%s{\"outer\": %d, \"x_dofs\": %d, \"y_dofs\": %d, \"inner\": %zu, "
                              "\"eta_squared\": %.15e, \"lambda_y_squared\": %.15e, "
                              "\"initial_trace_squared\": %.15e, \"y_estimator_squared\": %.15e, "
                              "\"last_solve_iterations\": %d, \"last_solve_seconds\": %.4f}",
                              k ? ", " : "", o.outer_iteration, o.n_x_true_dofs_before, o.n_y_true_dofs_after,
                              o.inner_iterations.size(), o.eta_squared, o.lambda_y_squared,
                              o.initial_trace_squared, o.y_estimator_squared,
                              o.inner_iterations.empty() ? -1 : o.inner_iterations.back().main_solve.iteration_count,
                              o.inner_iterations.empty() ? 0.0 : o.inner_iterations.back().main_solve.backsolve_seconds);
                out += buf;
            }
            return out + "]";
        };
        // the driver's slowest phases (b200-only runs)
        std::string phases = "[";
        {
            std::vector<std::pair<double, std::string>> rec;
            for (const auto& r : ra.timing_records)
                if (r.metric_kind == adaptive_algorithm::MetricKind::duration_seconds)
                    rec.emplace_back(r.total_seconds, r.phase);
            std::sort(rec.rbegin(), rec.rend());
            // the 25 slowest, and every phase of the b200 main solve
            bool first = true;
            for (std::size_t k = 0; k < rec.size(); ++k)
            {
                const std::string& name = rec[k].second;
                if (k >= 25 && name.rfind("b200.", 0) != 0 && name.rfind("main_system.", 0) != 0)
                    continue;
                char buf[256];
                std::snprintf(buf, sizeof(buf), "%s[\"%s\", %.3f]", first ? "" : ", ", name.c_str(), rec[k].first);
                phases += buf;
                first = false;
            }
        }
        phases += "]";
        std::fprintf(stderr, "driver phases (total s): %s\n", phases.c_str());
        std::printf("{\"mode\": \"adaptive\", \"p\": %d, \"levels\": %d, \"tol\": %.1e, \"b200_s\": %.3f, "
                    "\"direct_s\": %.3f, \"device_estimates\": %lld, \"device_solves\": %lld, "
                    "\"learned_fallbacks\": %lld, \"b200\": %s, \"direct\": %s}\n",
                    P, levels, tol, std::chrono::duration<double>(t1 - t0).count(),
                    std::chrono::duration<double>(t2 - t1).count(), la::b200::session().device_estimates(), la::b200::session().device_solves(),
                    la::b200::session().learned_fallbacks(),
                    dump(ra).c_str(), dump(rb).c_str());
        return 0;
    }

    template<class S>
    int dispatch_common(const std::string& mode, int argc, char** argv)
    {
        const int levels = std::atoi(argv[3]);
        const std::string example = argv[4];
        if (mode == "blocks")
            return run_blocks<S>(levels, example);
        if (mode == "solve" && argc >= 6)
            return run_solve<S>(levels, example, std::atof(argv[5]));
        if (mode == "cycle" && argc >= 7)
            return run_cycle<S>(levels, example, std::atoi(argv[5]), std::atof(argv[6]));
        if (mode == "estimate" && argc >= 6)
            return run_estimate<S>(levels, example, std::atof(argv[5]));
        if constexpr (S::GT::dim_space_v == 2)
            if (mode == "snapshot" && argc >= 7)
                return run_snapshot<S>(levels, example, std::atof(argv[5]), argv[6]);
        return 2;
    }

    template<int P>
    int dispatch(const std::string& mode, int argc, char** argv)
    {
        const int levels = std::atoi(argv[3]);
        const std::string example = argv[4];
        if (mode != "adaptive")
            return dispatch_common<Spaces<P>>(mode, argc, argv);
        if (mode == "adaptive" && argc >= 7)
            return run_adaptive<P>(levels, example, std::atoi(argv[5]), std::atof(argv[6]),
                                   argc < 8 || std::atoi(argv[7]) != 0, argc < 9 ? 0 : std::atoi(argv[8]));
        return 2;
    }
}

int main(int argc, char** argv)
{
    if (argc < 5)
    {
        std::fprintf(stderr, "usage: apf_dropin_test blocks|solve|cycle|estimate|adaptive <p:1|2|1d> <levels> <example> [...]\n");
        return 2;
    }
    const std::string mode = argv[1];
    try
    {
        // <p>: 1 or 2 (2+1D prisms), or "1d" (1+1D P1 quadrilaterals)
        const std::string pa = argv[2];
        const int rc = pa == "1d" ? dispatch_common<Spaces1D>(mode, argc, argv)
                       : std::atoi(argv[2]) == 2 ? dispatch<2>(mode, argc, argv)
                                                 : dispatch<1>(mode, argc, argv);
        if (rc == 2)
            std::fprintf(stderr, "apf_dropin_test: bad arguments\n");
        return rc;
    }
    catch (const std::exception& e)
    {
        std::fprintf(stderr, "apf_dropin_test: %s\n", e.what());
        return 1;
    }
}
