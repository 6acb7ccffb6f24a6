// ORACLE (test infrastructure only; never linked into the product library).
//
// Runs the reference's OWN templates (compiled from the reference's source tree,
// with oracle/shim ahead of it on the include path in place of Eigen) on the
// benchmark problems and writes .npy fixtures:
//   * the mesh and DOF maps the reference builds (host inputs of the hot path),
//   * the assembled saddle blocks A_y, B, C_signed, f, g
//     (finite_element::system::assemble_main_system_blocks,
//      src/finite_element/system/assemble_saddle_problem.hpp:131),
//   * the parabolic graph-norm Schur approximation Hhat
//     (src/finite_element/assembly/main_system/parabolic_graph_norm.hpp:22),
//   * 2+1D: the direct-solver path's full saddle matrix and right-hand side by the
//     two-pass pattern + numeric assembly
//     (src/finite_element/assembly/main_system/two_pass_full_saddle_2d.hpp:468), twice
//     through one pattern cache: the example's coefficients, then a constant anisotropic
//     M = [[2, 0.5], [0.5, 1]] on the reused pattern,
//   * with APF_REF_ESTIMATE (2+1D and 1+1D): the reference's binary artifacts of the estimate,
//     cellwise_error.bin, cellwise_error_components.bin and x_indicator_components.bin
//     (src/finite_element/io/write_cellwise_error_binary.hpp,
//      src/finite_element/io/write_cellwise_error_components_binary.hpp,
//      algorithm/output/iteration_snapshot_writer.hpp:173-233),
//   * with APF_REF_ESTIMATE and APF_REF_G (2+1D P1): the driver's G^delta estimator, its
//     space's restriction, A_G, f_G, rhs_G = f_G - B(X,G)^T u_delta, lambda_G and
//     ||lambda_G - lambda_delta||^2_{A_G} (algorithm/adaptive_driver.hpp:2690-2900).
//
// usage: apf_ref_dump <dim:1|2> <p:1|2> <uniform_levels> <example> <outdir>
//        apf_ref_dump bench <p:1|2> <uniform_levels> <example> <reps>

#include <array>
#include <cmath>
#include <cstdio>
#include <memory>
#include <random>
#include <cstdlib>
#include <filesystem>
#include <limits>
#include <unordered_map>
#include <unordered_set>
#include <algorithm>
#include <chrono>
#include <omp.h>
#include <iostream>
#include <string>
#include <vector>

#include "linear_algebra/eigen_backend/backend.hpp"

#include "algorithm/adaptive_driver.hpp"
#include "algorithm/example_registry.hpp"
#include "algorithm/examples/space_time_2d/initial_data_2d_examples.hpp"
#include "algorithm/examples/space_time_2d/space_time_2d_example.hpp"
#include "algorithm/examples/space_time_1d/space_time_1d_example.hpp"
#include "algorithm/support/space_time_1d.hpp"
#include "algorithm/support/space_time_2d.hpp"
#include "finite_element/fespace/fe_traits.hpp"
#include "finite_element/fespace/fespace.hpp"
#include "finite_element/fespace/policies.hpp"
#include "finite_element/system/assemble_saddle_problem.hpp"
#include "finite_element/assembly/main_system/parabolic_graph_norm.hpp"
#include "finite_element/assembly/main_system/two_pass_full_saddle_2d.hpp"
#include "finite_element/io/write_cellwise_error_binary.hpp"
#include "finite_element/io/write_cellwise_error_components_binary.hpp"
#include "algorithm/output/iteration_snapshot_writer.hpp"
#include "finite_element/assembly/constrained_dofs.hpp"
#include "finite_element/fespace/prolongation.hpp"
#include "linear_algebra/operations/linalg_ops.hpp"
#include "finite_element/time_slabs/time_slab_adaptive_loop.hpp"
#include "algorithm/detail/indicator_utilities.hpp"
#include "mesh/mesh_traits.hpp"

#include "npy.hpp"
#include "ref_meshes.hpp"

namespace
{
    using Backend = la::eigen::Backend;

    void dump_csc(const std::string& dir, const std::string& name, const la::eigen::SparseMatrix& A)
    {
        apf_oracle::write_npy(dir + "/" + name + "_outer.npy", A.outer());
        apf_oracle::write_npy(dir + "/" + name + "_inner.npy", A.inner());
        apf_oracle::write_npy(dir + "/" + name + "_values.npy", A.values());
        const std::vector<int> shape{A.rows(), A.cols()};
        apf_oracle::write_npy(dir + "/" + name + "_shape.npy", shape);
    }

    void dump_vec(const std::string& dir, const std::string& name, const la::eigen::Vector& v)
    {
        apf_oracle::write_npy(dir + "/" + name + ".npy", v.storage());
    }

    // Flattened CellRestriction for a list of cells:
    // offsets[c*ndof + i] .. offsets[c*ndof+i+1] index (true_dof, weight) pairs.
    template<class Space>
    void dump_restrictions(const std::string& dir, const std::string& name, const Space& space, const std::vector<int>& cells)
    {
        std::vector<int> offsets{0};
        std::vector<int> dofs;
        std::vector<double> weights;
        for (const int c : cells)
        {
            const auto r = finite_element::assembly::build_cell_restriction(space, c);
            for (int i = 0; i < r.size(); ++i)
            {
                for (const auto& e : r[i])
                {
                    dofs.push_back(e.true_dof);
                    weights.push_back(e.weight);
                }
                offsets.push_back(static_cast<int>(dofs.size()));
            }
        }
        apf_oracle::write_npy(dir + "/" + name + "_offsets.npy", offsets);
        apf_oracle::write_npy(dir + "/" + name + "_dofs.npy", dofs);
        apf_oracle::write_npy(dir + "/" + name + "_weights.npy", weights);
    }

    // Per cell: x0 y0 x1 y1 x2 y2 t0 t1 (vertex order of the reference cell).
    template<class Space>
    void dump_geometry_2d(const std::string& dir, const std::string& name, const Space& space, const std::vector<int>& cells)
    {
        const auto& mesh = space.mesh_ref();
        std::vector<double> g;
        g.reserve(cells.size() * 8u);
        for (const int c : cells)
        {
            const auto& cell = mesh.cell(c);
            for (int k = 0; k < 3; ++k)
            {
                const auto& v = mesh.spatial_vertices()[cell.spatial_vertex_ids[k]];
                g.push_back(v[0]);
                g.push_back(v[1]);
            }
            g.push_back(mesh.temporal_vertices()[cell.temporal_vertex_ids[0]][0]);
            g.push_back(mesh.temporal_vertices()[cell.temporal_vertex_ids[1]][0]);
        }
        apf_oracle::write_npy(dir + "/" + name + ".npy", g.data(), {cells.size(), 8u});
    }


    using apf_oracle::apply_adaptive_options_2d;
    using apf_oracle::env_int;
    using apf_oracle::uniform_isotropic_refine;

    // The driver's G^delta estimator on the accepted Y mesh, step by step as
    // AdaptiveDriver::compute_g_estimator_for_accepted_inner_iteration_ runs it
    // (algorithm/adaptive_driver.hpp:2690-2900): the space G of degree p+1 on the Y cells
    // (broken in time), A_G, f_G, B(X,G), rhs = f_G - B^T u_delta, lambda_G (direct solve),
    // lambda_delta prolonged nodally into G, and ||lambda_G - lambda_delta||^2_{A_G}.
    template<int QSpace, int QTime, class XSpace, class YSpace, class Problem, class YFunction, class XFunction>
    void dump_g_delta(const std::string& dir, const XSpace& x_space, YSpace& y_space, const std::vector<int>& y_cells,
                      const Problem& problem, const YFunction& lambda_delta, const XFunction& u_delta)
    {
        using GT = typename YSpace::GT;
        using YFET = typename YSpace::FETraitsType;
        using GFET = finite_element::FiniteElementTraits<GT, YFET::p_space_v + 1, YFET::p_time_v + 1>;
        using GSpace = finite_element::FESpace<GT, GFET, finite_element::SpaceOnlyPolicy>;
        finite_element::FESpaceInitializationOptions options;
        options.search_index = finite_element::SearchIndexBuildMode::Disabled;
        options.build_refinement_indices = false;
        options.build_edge_interval_index = false;
        GSpace g_space(y_space.unsafe_mesh_ref());
        g_space.initialize(y_space.active_cells(), options);
        typename Backend::SparseMatrix A_g, B_xg;
        typename Backend::Vector f_g;
        finite_element::assembly::detail::AssemblySpaceCache<GSpace> g_cache(g_space);
        finite_element::assembly::detail::AssemblySpaceCache<XSpace> x_cache(x_space);
        finite_element::assembly::detail::ActiveAncestorCache<XSpace> ancestors(x_space);
        finite_element::assembly::assemble_mat_A<QSpace + 1, QTime + 1, Backend>(A_g, g_space, problem.M, g_cache,
                                                                                1e-15);
        finite_element::assembly::assemble_vec_f<QSpace + 1, QTime + 1>(f_g, g_space, problem.ell, g_cache, 1e-15);
        finite_element::assembly::assemble_mat_B<QSpace + 1, QTime + 1, Backend>(B_xg, x_space, g_space, x_cache,
                                                                                g_cache, ancestors, problem.M, 1e-15);
        const auto rhs_g = la::ops::subtract(f_g, la::ops::transpose_matvec(B_xg, u_delta.true_coefficients()));
        typename Backend::Solver solver;
        la::concepts::SolverOptions lu;
        lu.solver = la::concepts::SolverType::SparseLU;
        solver.compute(A_g, lu);
        typename Backend::Vector lambda_g;
        solver.solve(rhs_g, lambda_g);
        const auto lambda_delta_in_g = finite_element::fespace::prolong_true_coefficients_nodal(lambda_delta, g_space);
        const auto diff = la::ops::subtract(lambda_g, lambda_delta_in_g);
        const double energy =
            la::ops::quadratic_form<typename Backend::SparseMatrix, typename Backend::SparseBuilder>(A_g, diff);
        dump_restrictions(dir, "g_restriction", g_space, y_cells);
        dump_csc(dir, "A_g", A_g);
        dump_vec(dir, "f_g", f_g);
        dump_vec(dir, "rhs_g", rhs_g);
        dump_vec(dir, "lambda_g", lambda_g);
        dump_vec(dir, "lambda_delta_in_g", lambda_delta_in_g);
        const std::vector<double> e{energy};
        apf_oracle::write_npy(dir + "/g_lambda_difference_squared.npy", e);
        const std::vector<int> ng{g_space.dof_handler_ref().n_true_dofs()};
        apf_oracle::write_npy(dir + "/g_n_dofs.npy", ng);
        std::fprintf(stderr, "g_delta: n_g=%d ||lambda_G - lambda_delta||^2_A=%.12e\n", ng[0], energy);
    }

    // Times the reference's own CPU assembly path (main blocks + graph-norm block)
    // on the uniform mesh of outer level `levels`; prints one JSON line.
    template<int P>
    int bench_2d(int levels, const std::string& example_name, int reps)
    {
        constexpr int QSpace = 4 * P + 1;
        constexpr int QTime = 2 * P + 1;
        using GT = mesh::MeshTraits<2>;
        using FET = finite_element::FiniteElementTraits<GT, P, P>;
        using XSpace = finite_element::FESpace<GT, FET, finite_element::SpaceTimePolicy>;
        using YSpace = finite_element::FESpace<GT, FET, finite_element::SpaceOnlyPolicy>;
        auto example = adaptive_algorithm::examples::make_2d_example(example_name);
        auto mesh = adaptive_algorithm::examples::make_initial_mesh_from_example(example);
        XSpace x_space(mesh);
        YSpace y_space(mesh);
        adaptive_algorithm::examples::initialize_spaces_from_example(x_space, y_space, example);
        for (int k = 0; k < levels; ++k)
            uniform_isotropic_refine(x_space);
        (void)apply_adaptive_options_2d(x_space, example);
        y_space.initialize(x_space.active_cells());
        const int n_cells = static_cast<int>(y_space.active_cells().size());
        const int n_dofs = x_space.dof_handler_ref().n_true_dofs() + y_space.dof_handler_ref().n_true_dofs();
        double best = 1e300, total = 0.0;
        if (std::getenv("APF_REF_CYCLE") != nullptr)
        {
            // the reference's whole inner iteration (time_slab_adaptive_loop.hpp:727):
            // assembly, graph norm, main solve, slab reconstruction, patch flux solves,
            // indicators
            // the main solve inside it runs the oracle shim's direct solver (the reference's
            // own sparse solvers are Eigen / PARDISO, absent here): its time is reported
            // separately, and the reference's own stages are the rest
            double flux = 0.0, solve_total = 0.0;
            std::string stage_list; // per repetition: wall time less the main solve
            for (int r = 0; r < reps; ++r)
            {
                const auto t0 = std::chrono::steady_clock::now();
                typename Backend::Solver solver;
                la::concepts::SolverOptions opts;
                // the production runs' main solver (main_solver: pardiso_ldlt in the example
                // configurations); the shim factors it unless APF_SHIM_SKIP_PARDISO is set
                opts.solver = la::concepts::SolverType::PardisoLDLT;
                finite_element::time_slabs::AdaptiveTestSpaceIterationParameters<Backend, XSpace, YSpace> params;
                const auto state = finite_element::time_slabs::compute_adaptive_test_space_iteration<QSpace, QTime, Backend>(
                    y_space, x_space, example.problem, solver, opts, params);
                const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                best = std::min(best, dt);
                total += dt;
                solve_total += state.main_solve_setup_seconds + state.main_solve_solve_seconds;
                flux = state.flux_diagnostics.total_flux();
                char buf[64];
                std::snprintf(buf, sizeof(buf), "%s%.6f", r ? ", " : "",
                              dt - state.main_solve_setup_seconds - state.main_solve_solve_seconds);
                stage_list += buf;
            }
            std::printf("{\"stage\": \"inner_iteration\", \"p\": %d, \"level\": %d, \"n_cells\": %d, \"n_dofs\": %d, "
                        "\"reps\": %d, \"mean_s\": %.6f, \"best_s\": %.6f, \"main_solve_mean_s\": %.6f, "
                        "\"threads\": %d, \"flux_squared\": %.12e, \"stage_s\": [%s]}\n",
                        P, levels, n_cells, n_dofs, reps, total / reps, best, solve_total / reps, omp_get_max_threads(),
                        flux, stage_list.c_str());
            return 0;
        }
        for (int r = 0; r < reps; ++r)
        {
            const auto t0 = std::chrono::steady_clock::now();
            const auto blocks = finite_element::system::assemble_main_system_blocks<QSpace, QTime, Backend>(
                y_space, x_space, example.problem, 1e-15, -1.0);
            const auto gn = finite_element::assembly::assemble_parabolic_graph_norm_approximation<QSpace, QTime, Backend>(
                y_space, x_space, example.problem.M, blocks.A_y(), blocks.C_signed(), 1e-15, 1e-14);
            const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            best = std::min(best, dt);
            total += dt;
            if (gn.approximation.hhat.rows() < 0) return 3;
        }
        std::printf("{\"stage\": \"assembly+graph_norm\", \"p\": %d, \"level\": %d, \"n_cells\": %d, \"n_dofs\": %d, "
                    "\"reps\": %d, \"mean_s\": %.6f, \"best_s\": %.6f, \"threads\": %d}\n",
                    P, levels, n_cells, n_dofs, reps, total / reps, best, omp_get_max_threads());
        return 0;
    }

    template<int P>
    int run_2d(int levels, const std::string& example_name, const std::string& dir)
    {
        constexpr int QSpace = 4 * P + 1;
        constexpr int QTime = 2 * P + 1;
        using GT = mesh::MeshTraits<2>;
        using FET = finite_element::FiniteElementTraits<GT, P, P>;
        using XSpace = finite_element::FESpace<GT, FET, finite_element::SpaceTimePolicy>;
        using YSpace = finite_element::FESpace<GT, FET, finite_element::SpaceOnlyPolicy>;

        auto example = adaptive_algorithm::examples::make_2d_example(example_name);
        auto mesh = adaptive_algorithm::examples::make_initial_mesh_from_example(example);
        XSpace x_space(mesh);
        YSpace y_space(mesh);
        adaptive_algorithm::examples::initialize_spaces_from_example(x_space, y_space, example);
        for (int k = 0; k < levels; ++k)
            uniform_isotropic_refine(x_space);
        const std::vector<double> kx = apply_adaptive_options_2d(x_space, example);
        y_space.initialize(x_space.active_cells());
        const int driver_outer = env_int("APF_REF_DRIVER_OUTER", 0);
        if (driver_outer > 0)
        {
            // the reference's adaptive driver (algorithm/adaptive_driver.hpp:3508) for
            // `driver_outer` outer cycles: its own inner Y loops, X marking and refinement
            typename Backend::Solver solver;
            la::concepts::SolverOptions opts;
            adaptive_algorithm::AdaptiveParameters par;
            par.max_outer_iterations = driver_outer;
            par.polynomial_degree = P;
            par.output.print_iteration_tables = false;
            par.output.save_mesh_statistics = false;
            par.output.stream = &std::cerr;
            (void)adaptive_algorithm::run_adaptive_driver<QSpace, QTime, Backend>(x_space, y_space, example.problem,
                                                                                 solver, opts, par);
        }

        std::filesystem::create_directories(dir);
        if (!kx.empty() && driver_outer == 0 && env_int("APF_REF_KAPPA_BLOCKS", 0) == 0)
            apf_oracle::write_npy(dir + "/kappa_x.npy", kx);
        if (std::getenv("APF_REF_KAPPA") != nullptr)
        {
            // M = kappa I at each Y cell (the kappa law's value at the cell's centroid)
            std::vector<double> ky;
            for (const int c : y_space.active_cells())
            {
                const auto& cell = mesh.cell(c);
                const auto& sv = mesh.spatial_vertices();
                const auto& tv = mesh.temporal_vertices();
                adaptive_algorithm::examples::SpaceTime2DPoint q{};
                for (int k = 0; k < 3; ++k)
                {
                    q[0] += sv[cell.spatial_vertex_ids[k]][0] / 3.0;
                    q[1] += sv[cell.spatial_vertex_ids[k]][1] / 3.0;
                }
                q[2] = 0.5 * (tv[cell.temporal_vertex_ids[0]][0] + tv[cell.temporal_vertex_ids[1]][0]);
                ky.push_back(example.problem.M(q)[0][0]);
            }
            apf_oracle::write_npy(dir + "/kappa_y.npy", ky);
        }
        for (int pass = 0; pass < env_int("APF_REF_Y_PASSES", 0); ++pass)
        {
            typename Backend::Solver solver;
            la::concepts::SolverOptions opts;
            finite_element::time_slabs::AdaptiveTestSpaceIterationParameters<Backend, XSpace, YSpace> params;
            const auto state = finite_element::time_slabs::compute_adaptive_test_space_iteration<QSpace, QTime, Backend>(
                y_space, x_space, example.problem, solver, opts, params);
            std::cerr << "y pass " << pass << ": marked " << state.marked_source_cells.size() << " of "
                      << y_space.active_cells().size() << " Y cells\n";
            finite_element::time_slabs::refine_test_space_from_marked_source_cells(y_space, x_space,
                                                                                   state.marked_source_cells);
        }

        const auto& y_cells = y_space.active_cells();
        const auto& x_cells = x_space.active_cells();
        std::cerr << "2d p=" << P << " levels=" << levels << " x_cells=" << x_cells.size()
                  << " y_cells=" << y_cells.size()
                  << " n_x=" << x_space.dof_handler_ref().n_true_dofs()
                  << " n_y=" << y_space.dof_handler_ref().n_true_dofs() << "\n";

        std::filesystem::create_directories(dir);
        dump_geometry_2d(dir, "y_geometry", y_space, y_cells);
        {
            std::vector<int> vids;
            for (const int c : y_cells)
                for (int k = 0; k < 3; ++k)
                    vids.push_back(mesh.cell(c).spatial_vertex_ids[k]);
            apf_oracle::write_npy(dir + "/y_vertex_ids.npy", vids.data(), {y_cells.size(), 3u});
        }
        dump_geometry_2d(dir, "x_geometry", x_space, x_cells);
        dump_restrictions(dir, "y_restriction", y_space, y_cells);
        dump_restrictions(dir, "x_restriction", x_space, x_cells);
        {
            finite_element::assembly::detail::ActiveAncestorCache<XSpace> cache(x_space);
            std::vector<int> x_pos(static_cast<std::size_t>(mesh.n_cells()), -1);
            for (std::size_t k = 0; k < x_cells.size(); ++k)
                x_pos[static_cast<std::size_t>(x_cells[k])] = static_cast<int>(k);
            std::vector<int> anc;
            for (const int c : y_cells)
                anc.push_back(x_pos[static_cast<std::size_t>(cache.find(c))]);
            apf_oracle::write_npy(dir + "/y_to_x_cell.npy", anc);
            apf_oracle::write_npy(dir + "/y_cell_ids.npy", y_cells);
            apf_oracle::write_npy(dir + "/x_cell_ids.npy", x_cells);
        }

        const auto blocks = finite_element::system::assemble_main_system_blocks<QSpace, QTime, Backend>(
            y_space, x_space, example.problem, 1e-15, -1.0);
        dump_csc(dir, "A_y", blocks.A_y());
        dump_csc(dir, "B", blocks.lower_left_B());
        dump_csc(dir, "C_signed", blocks.C_signed());
        dump_vec(dir, "f", blocks.f());
        dump_vec(dir, "g", blocks.g());

        const auto gn = finite_element::assembly::assemble_parabolic_graph_norm_approximation<QSpace, QTime, Backend>(
            y_space, x_space, example.problem.M, blocks.A_y(), blocks.C_signed(), 1e-15, 1e-14);
        dump_csc(dir, "Hhat", gn.approximation.hhat);

        {
            namespace fa = finite_element::assembly;
            fa::detail::AssemblySpaceCache<YSpace> y_cache(y_space);
            fa::detail::AssemblySpaceCache<XSpace> x_cache(x_space);
            fa::detail::ActiveAncestorCache<XSpace> ancestors(x_space);
            fa::TwoPassFullSaddleAssemblyCache2D<Backend, XSpace, YSpace> cache;
            const finite_element::detail::TimingRecorder timing{};
            const auto full = fa::assemble_main_full_saddle_two_pass_2d<QSpace, QTime, Backend>(
                x_space, y_space, x_cache, y_cache, ancestors, example.problem.M, example.problem.ell,
                example.problem.u0, 1e-15, -1.0, timing, nullptr, 1, 0.0, &cache);
            dump_csc(dir, "K2p", full.matrix);
            dump_vec(dir, "K2p_rhs", full.rhs);
            const adaptive_algorithm::examples::SpaceTime2DDiffusionFunctionM m_aniso =
                [](const adaptive_algorithm::examples::SpaceTime2DPoint&) {
                    return finite_element::coefficients::DiffusionTensor<2>{{{2.0, 0.5}, {0.5, 1.0}}};
                };
            const auto aniso = fa::assemble_main_full_saddle_two_pass_2d<QSpace, QTime, Backend>(
                x_space, y_space, x_cache, y_cache, ancestors, m_aniso, example.problem.ell, example.problem.u0,
                1e-15, -1.0, timing, nullptr, 1, 0.0, &cache);
            dump_csc(dir, "K2p_aniso", aniso.matrix);
            dump_vec(dir, "K2p_aniso_rhs", aniso.rhs);
            const std::vector<int> reuse{static_cast<int>(cache.pattern_reuse_count)};
            apf_oracle::write_npy(dir + "/K2p_pattern_reuse_count.npy", reuse);
        }

        if (std::getenv("APF_REF_ESTIMATE") != nullptr)
        {
            // the reference's whole inner iteration (time_slab_adaptive_loop.hpp:727):
            // main solve (direct), slab reconstruction, vertex-patch flux solves, indicators
            typename Backend::Solver solver;
            la::concepts::SolverOptions opts;
            finite_element::time_slabs::AdaptiveTestSpaceIterationParameters<Backend, XSpace, YSpace> params;
            const auto state = finite_element::time_slabs::compute_adaptive_test_space_iteration<QSpace, QTime, Backend>(
                y_space, x_space, example.problem, solver, opts, params);
            dump_vec(dir, "lambda_delta", state.lambda_delta.true_coefficients());
            dump_vec(dir, "u_delta", state.u_delta.true_coefficients());
            if (state.slab_reconstruction.has_value())
            {
                // the reference's time-slab space (time_slab_builder.hpp:53-215) and its
                // reconstruction lambda~: per slab cell (slabs in time order, cells in each
                // slab's order) the slab, the source Y cell, the slab cell's geometry and
                // spatial vertex ids of the slab mesh, its restriction in the slab space (true
                // DOFs numbered slab after slab) and lambda~ at the 3 vertices x {t0, t1}
                const auto& ss = state.slab_reconstruction->slab_space_ref();
                const auto& lt = state.slab_reconstruction->reconstructed_function();
                std::vector<int> s_slab, s_source, s_vids, r_off{0}, r_dofs, s_dof_base{0};
                std::vector<double> s_geo, s_lt, r_w;
                for (int k = 0; k < ss.n_slabs(); ++k)
                {
                    const auto& slab = ss.slab(k);
                    const auto& smesh = slab.mesh_ref();
                    const int base = s_dof_base.back();
                    for (const int c : slab.active_cells())
                    {
                        s_slab.push_back(k);
                        s_source.push_back(slab.source_cell_id(c));
                        const auto& cell = smesh.cell(c);
                        for (int v = 0; v < 3; ++v)
                        {
                            const auto& xy = smesh.spatial_vertices()[cell.spatial_vertex_ids[v]];
                            s_geo.push_back(xy[0]);
                            s_geo.push_back(xy[1]);
                            s_vids.push_back(cell.spatial_vertex_ids[v]);
                        }
                        s_geo.push_back(slab.t_begin());
                        s_geo.push_back(slab.t_end());
                        for (int v = 0; v < 3; ++v)
                        {
                            const auto& xy = smesh.spatial_vertices()[cell.spatial_vertex_ids[v]];
                            for (const double t : {slab.t_begin(), slab.t_end()})
                                s_lt.push_back(lt.value_on_cell(k, c, typename XSpace::SpaceTimePoint{xy[0], xy[1], t}));
                        }
                        const auto r = finite_element::assembly::build_cell_restriction(slab.fespace_ref(), c);
                        for (int i = 0; i < r.size(); ++i)
                        {
                            for (const auto& e : r[i])
                            {
                                r_dofs.push_back(base + e.true_dof);
                                r_w.push_back(e.weight);
                            }
                            r_off.push_back(static_cast<int>(r_dofs.size()));
                        }
                    }
                    s_dof_base.push_back(base + slab.fespace_ref().dof_handler_ref().n_true_dofs());
                }
                apf_oracle::write_npy(dir + "/slab_of_cell.npy", s_slab);
                apf_oracle::write_npy(dir + "/slab_source_cell.npy", s_source);
                apf_oracle::write_npy(dir + "/slab_vertex_ids.npy", s_vids.data(), {s_slab.size(), 3u});
                apf_oracle::write_npy(dir + "/slab_geometry.npy", s_geo.data(), {s_slab.size(), 8u});
                apf_oracle::write_npy(dir + "/slab_lambda_tilde.npy", s_lt.data(), {s_slab.size(), 6u});
                apf_oracle::write_npy(dir + "/slab_restriction_offsets.npy", r_off);
                apf_oracle::write_npy(dir + "/slab_restriction_dofs.npy", r_dofs);
                apf_oracle::write_npy(dir + "/slab_restriction_weights.npy", r_w);
                apf_oracle::write_npy(dir + "/slab_dof_base.npy", s_dof_base);
            }
            auto dump_map = [&](const std::string& name, const auto& m) {
                std::vector<int> ids;
                std::vector<double> vals;
                for (const int c : y_cells)
                {
                    const auto it = m.find(c);
                    vals.push_back(it == m.end() ? std::numeric_limits<double>::quiet_NaN() : it->second);
                }
                apf_oracle::write_npy(dir + "/" + name + ".npy", vals);
            };
            // the driver's X-marking indicators (adaptive_driver.hpp:355-367)
            const auto xi = adaptive_algorithm::detail::compute_x_marking_indicator_components<QSpace, QTime>(
                x_space, state.lambda_delta, state.u_delta, example.problem.u0, example.problem.M);
            auto dump_over = [&](const std::string& name, const std::vector<int>& cells, const auto& m) {
                std::vector<double> vals;
                for (const int c : cells)
                {
                    const auto it = m.find(c);
                    vals.push_back(it == m.end() ? std::numeric_limits<double>::quiet_NaN() : it->second);
                }
                apf_oracle::write_npy(dir + "/" + name + ".npy", vals);
            };
            const std::vector<int> xcv(x_cells.begin(), x_cells.end());
            dump_map("xind_lambda_by_y", xi.lambda_y_squared_by_y_cell.by_source_cell);
            dump_over("xind_lambda_by_x", xcv, xi.lambda_y_squared_by_x_cell.by_source_cell);
            dump_over("xind_trace_by_x", xcv, xi.initial_trace_squared_by_x_cell.by_source_cell);
            dump_over("xind_eta_by_x", xcv, xi.eta_squared_by_x_cell.by_source_cell);
            dump_map("est_flux", state.flux_diagnostics.by_source_cell_flux);
            dump_map("est_div", state.flux_diagnostics.by_source_cell_residual);
            dump_map("est_recon", state.reconstruction_y_squared.by_source_cell);
            dump_map("est_eta", state.estimator.estimator_squared.by_source_cell);
            // the reference's binary artifacts of the estimate (sorted by decreasing value)
            finite_element::io::write_cellwise_error_binary(state.estimator.estimator_squared, dir,
                                                            "cellwise_error.bin");
            finite_element::io::write_cellwise_error_components_binary(state.estimator, dir,
                                                                       "cellwise_error_components.bin");
            adaptive_algorithm::output::detail::write_x_indicator_components_binary(xi, dir,
                                                                                    "x_indicator_components.bin");
            std::fprintf(stderr, "estimate: flux=%.6e div=%.6e recon=%.6e eta=%.6e\n",
                         state.flux_diagnostics.total_flux(), state.flux_diagnostics.total_residual(),
                         state.reconstruction_y_squared.total(), state.estimator.total());
            if constexpr (P == 1)
                if (std::getenv("APF_REF_G") != nullptr)
                    dump_g_delta<QSpace, QTime>(dir, x_space, y_space, y_cells, example.problem, state.lambda_delta,
                                                state.u_delta);
        }
        return 0;
    }

    // 1+1D: unit space-time square, the example's initial refinement, then `levels`
    // uniform outer refinements (space and time halved), P = 1 elements with the
    // runner's Gauss orders QSpace = QTime = 2P + 1
    // (algorithm/runners/detail/runner_case_execution.hpp:27-33).  Geometry rows are
    // x0 x1 t0 t1 (spatial vertices 0 and 1 of the cell, temporal vertices 0 and 1).
    template<int P>
    int run_1d(int levels, const std::string& example_name, const std::string& dir)
    {
        constexpr int QSpace = 2 * P + 1;
        constexpr int QTime = 2 * P + 1;
        using GT = mesh::MeshTraits<1>;
        using FET = finite_element::FiniteElementTraits<GT, P, P>;
        using XSpace = finite_element::FESpace<GT, FET, finite_element::SpaceTimePolicy>;
        using YSpace = finite_element::FESpace<GT, FET, finite_element::SpaceOnlyPolicy>;

        auto example = adaptive_algorithm::examples::make_1d_example(example_name);
        auto mesh = adaptive_algorithm::support::make_unit_mesh<GT>();
        XSpace x_space(mesh);
        YSpace y_space(mesh);
        adaptive_algorithm::examples::initialize_spaces_from_example(x_space, y_space, example);
        for (int k = 0; k < levels; ++k)
            uniform_isotropic_refine(x_space);
        if (const char* pts = std::getenv("APF_REF_X_POINTS"))
        {
            // 1+1D points "x,t;x,t"
            std::vector<typename XSpace::SpaceTimePoint> points;
            std::string str(pts);
            std::size_t pos = 0;
            while (pos < str.size())
            {
                std::size_t end = str.find(';', pos);
                if (end == std::string::npos) end = str.size();
                double a = 0.0, b = 0.0;
                if (std::sscanf(str.substr(pos, end - pos).c_str(), "%lf,%lf", &a, &b) == 2)
                    points.push_back(typename XSpace::SpaceTimePoint{a, b});
                pos = end + 1;
            }
            adaptive_algorithm::support::refine_points_n_times(x_space, points, env_int("APF_REF_X_ROUNDS", 1));
        }
        y_space.initialize(x_space.active_cells());
        for (int pass = 0; pass < env_int("APF_REF_Y_PASSES", 0); ++pass)
        {
            typename Backend::Solver solver;
            la::concepts::SolverOptions opts;
            finite_element::time_slabs::AdaptiveTestSpaceIterationParameters<Backend, XSpace, YSpace> params;
            const auto state = finite_element::time_slabs::compute_adaptive_test_space_iteration<QSpace, QTime, Backend>(
                y_space, x_space, example.problem, solver, opts, params);
            std::cerr << "y pass " << pass << ": marked " << state.marked_source_cells.size() << " of "
                      << y_space.active_cells().size() << " Y cells\n";
            finite_element::time_slabs::refine_test_space_from_marked_source_cells(y_space, x_space,
                                                                                   state.marked_source_cells);
        }

        const auto& y_cells = y_space.active_cells();
        const auto& x_cells = x_space.active_cells();
        std::cerr << "1d p=" << P << " levels=" << levels << " x_cells=" << x_cells.size()
                  << " y_cells=" << y_cells.size()
                  << " n_x=" << x_space.dof_handler_ref().n_true_dofs()
                  << " n_y=" << y_space.dof_handler_ref().n_true_dofs() << "\n";

        std::filesystem::create_directories(dir);
        auto dump_geometry_1d = [&](const std::string& name, const auto& cells) {
            std::vector<double> g;
            for (const int c : cells)
            {
                const auto& cell = mesh.cell(c);
                g.push_back(mesh.spatial_vertices()[cell.spatial_vertex_ids[0]][0]);
                g.push_back(mesh.spatial_vertices()[cell.spatial_vertex_ids[1]][0]);
                g.push_back(mesh.temporal_vertices()[cell.temporal_vertex_ids[0]][0]);
                g.push_back(mesh.temporal_vertices()[cell.temporal_vertex_ids[1]][0]);
            }
            apf_oracle::write_npy(dir + "/" + name + ".npy", g.data(), {cells.size(), 4u});
        };
        dump_geometry_1d("y_geometry", y_cells);
        dump_geometry_1d("x_geometry", x_cells);
        dump_restrictions(dir, "y_restriction", y_space, std::vector<int>(y_cells.begin(), y_cells.end()));
        dump_restrictions(dir, "x_restriction", x_space, std::vector<int>(x_cells.begin(), x_cells.end()));
        {
            finite_element::assembly::detail::ActiveAncestorCache<XSpace> cache(x_space);
            std::vector<int> x_pos(static_cast<std::size_t>(mesh.n_cells()), -1);
            for (std::size_t k = 0; k < x_cells.size(); ++k)
                x_pos[static_cast<std::size_t>(x_cells[k])] = static_cast<int>(k);
            std::vector<int> anc;
            for (const int c : y_cells)
                anc.push_back(x_pos[static_cast<std::size_t>(cache.find(c))]);
            apf_oracle::write_npy(dir + "/y_to_x_cell.npy", anc);
            apf_oracle::write_npy(dir + "/y_cell_ids.npy", std::vector<int>(y_cells.begin(), y_cells.end()));
            apf_oracle::write_npy(dir + "/x_cell_ids.npy", std::vector<int>(x_cells.begin(), x_cells.end()));
        }

        const auto blocks = finite_element::system::assemble_main_system_blocks<QSpace, QTime, Backend>(
            y_space, x_space, example.problem, 1e-15, -1.0);
        dump_csc(dir, "A_y", blocks.A_y());
        dump_csc(dir, "B", blocks.lower_left_B());
        dump_csc(dir, "C_signed", blocks.C_signed());
        dump_vec(dir, "f", blocks.f());
        dump_vec(dir, "g", blocks.g());
        const auto gn = finite_element::assembly::assemble_parabolic_graph_norm_approximation<QSpace, QTime, Backend>(
            y_space, x_space, example.problem.M, blocks.A_y(), blocks.C_signed(), 1e-15, 1e-14);
        dump_csc(dir, "Hhat", gn.approximation.hhat);

        if (std::getenv("APF_REF_ESTIMATE") != nullptr)
        {
            typename Backend::Solver solver;
            la::concepts::SolverOptions opts;
            finite_element::time_slabs::AdaptiveTestSpaceIterationParameters<Backend, XSpace, YSpace> params;
            const auto state = finite_element::time_slabs::compute_adaptive_test_space_iteration<QSpace, QTime, Backend>(
                y_space, x_space, example.problem, solver, opts, params);
            dump_vec(dir, "lambda_delta", state.lambda_delta.true_coefficients());
            dump_vec(dir, "u_delta", state.u_delta.true_coefficients());
            auto dump_over = [&](const std::string& name, const auto& cells, const auto& m) {
                std::vector<double> vals;
                for (const int c : cells)
                {
                    const auto it = m.find(c);
                    vals.push_back(it == m.end() ? std::numeric_limits<double>::quiet_NaN() : it->second);
                }
                apf_oracle::write_npy(dir + "/" + name + ".npy", vals);
            };
            const auto xi = adaptive_algorithm::detail::compute_x_marking_indicator_components<QSpace, QTime>(
                x_space, state.lambda_delta, state.u_delta, example.problem.u0, example.problem.M);
            dump_over("xind_lambda_by_y", y_cells, xi.lambda_y_squared_by_y_cell.by_source_cell);
            dump_over("xind_lambda_by_x", x_cells, xi.lambda_y_squared_by_x_cell.by_source_cell);
            dump_over("xind_trace_by_x", x_cells, xi.initial_trace_squared_by_x_cell.by_source_cell);
            dump_over("xind_eta_by_x", x_cells, xi.eta_squared_by_x_cell.by_source_cell);
            dump_over("est_flux", y_cells, state.flux_diagnostics.by_source_cell_flux);
            dump_over("est_div", y_cells, state.flux_diagnostics.by_source_cell_residual);
            finite_element::io::write_cellwise_error_binary(state.estimator.estimator_squared, dir,
                                                            "cellwise_error.bin");
            finite_element::io::write_cellwise_error_components_binary(state.estimator, dir,
                                                                       "cellwise_error_components.bin");
            adaptive_algorithm::output::detail::write_x_indicator_components_binary(xi, dir,
                                                                                    "x_indicator_components.bin");
            dump_over("est_recon", y_cells, state.reconstruction_y_squared.by_source_cell);
            dump_over("est_eta", y_cells, state.estimator.estimator_squared.by_source_cell);
            std::fprintf(stderr, "estimate: flux=%.6e div=%.6e recon=%.6e eta=%.6e\n",
                         state.flux_diagnostics.total_flux(), state.flux_diagnostics.total_residual(),
                         state.reconstruction_y_squared.total(), state.estimator.total());
        }
        return 0;
    }
}

int main(int argc, char** argv)
{
    if (argc == 6 && std::string(argv[1]) == "bench")
    {
        const int p = std::atoi(argv[2]);
        const int levels = std::atoi(argv[3]);
        const int reps = std::atoi(argv[5]);
        try
        {
            if (p == 1) return bench_2d<1>(levels, argv[4], reps);
            if (p == 2) return bench_2d<2>(levels, argv[4], reps);
        }
        catch (const std::exception& e)
        {
            std::fprintf(stderr, "apf_ref_dump: %s\n", e.what());
            return 1;
        }
        return 2;
    }
    if (argc != 6)
    {
        std::fprintf(stderr, "usage: %s <dim:2> <p:1|2> <uniform_levels> <example> <outdir>\n", argv[0]);
        return 2;
    }
    const int dim = std::atoi(argv[1]);
    const int p = std::atoi(argv[2]);
    const int levels = std::atoi(argv[3]);
    const std::string example = argv[4];
    const std::string dir = argv[5];
    try
    {
        if (dim == 1 && p == 1)
            return run_1d<1>(levels, example, dir);
        if (dim == 2 && p == 1)
            return run_2d<1>(levels, example, dir);
        if (dim == 2 && p == 2)
            return run_2d<2>(levels, example, dir);
    }
    catch (const std::exception& e)
    {
        std::fprintf(stderr, "apf_ref_dump: %s\n", e.what());
        return 1;
    }
    std::fprintf(stderr, "unsupported case\n");
    return 2;
}
