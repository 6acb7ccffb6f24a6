// ORACLE (test infrastructure only; never linked into the product library).
//
// Mesh helpers shared by the oracle driver (ref_dump.cpp) and the C++ drop-in test
// (tests/dropin/dropin_main.cpp): the reference driver's uniform isotropic refinement and
// the adaptive-mesh options, on the reference's own FE spaces.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "algorithm/examples/space_time_2d/space_time_2d_example.hpp"
#include "algorithm/support/space_time_2d.hpp"
#include "algorithm/support/space_time_1d.hpp"
#include "finite_element/coefficients/diffusion_coefficient.hpp"
#include "mesh/mesh_traits.hpp"

namespace apf_oracle
{
    // Mirror of the reference driver's uniform isotropic X refinement
    // (algorithm/adaptive_driver.hpp:1482-1830, refine_space_uniform_isotropically_):
    // spatial waves over all active descendants of the marked parents until every
    // descendant's x- and y-extent is strictly smaller than its parent's, then one
    // temporal split of every descendant.  One call = one `uniform_standard`
    // outer iteration of the paper runs.
    template<class Space>
    void uniform_isotropic_refine(Space& space)
    {
        auto& mesh = space.unsafe_mesh_ref();
        struct Ext { double sx, sy, t; };
        auto extents = [&](int c) {
            const auto& cell = mesh.cell(c);
            const auto& sv = mesh.spatial_vertices();
            const auto& tv = mesh.temporal_vertices();
            double mnx = 1e300, mxx = -1e300, mny = 1e300, mxy = -1e300, mnt = 1e300, mxt = -1e300;
            constexpr int dim = Space::GT::dim_space_v;
            for (const int v : cell.spatial_vertex_ids) {
                mnx = std::min(mnx, sv[v][0]); mxx = std::max(mxx, sv[v][0]);
                if constexpr (dim > 1) { mny = std::min(mny, sv[v][dim > 1 ? 1 : 0]); mxy = std::max(mxy, sv[v][dim > 1 ? 1 : 0]); }
            }
            if constexpr (dim == 1) { mny = 0.0; mxy = 1.0; }
            for (const int v : cell.temporal_vertex_ids) { mnt = std::min(mnt, tv[v][0]); mxt = std::max(mxt, tv[v][0]); }
            return Ext{mxx - mnx, mxy - mny, mxt - mnt};
        };
        auto smaller = [](double child, double parent) {
            const double tol = 64.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, parent);
            return child < parent - tol;
        };
        std::unordered_map<int, Ext> parents;
        for (const int c : space.active_cells()) parents.emplace(c, extents(c));
        auto ancestor = [&](int c) {
            while (c >= 0) { if (parents.count(c)) return c; c = mesh.cell(c).parent_id; }
            return -1;
        };
        auto refine_all = [&](const std::vector<int>& ids, mesh::RefinementType type) {
            std::unordered_set<int> add_ids, remove_ids;
            std::vector<int> changed;
            for (const int c : ids) {
                if (!space.is_active_cell(c)) continue;
                mesh.refine_storage_leaf_without_closure(c, type);
                remove_ids.insert(c);
                changed.push_back(c);
                for (const int ch : mesh.cell(c).children) { add_ids.insert(ch); changed.push_back(ch); }
            }
            space.unsafe_update_active_cells(add_ids, remove_ids);
            std::sort(changed.begin(), changed.end());
            changed.erase(std::unique(changed.begin(), changed.end()), changed.end());
            space.rebuild_incremental_after_refinement(changed);
        };
        for (int wave = 0; wave < 32; ++wave) {
            bool all_smaller = true;
            for (const int c : space.active_cells()) {
                const auto e = extents(c);
                const auto& pe = parents.at(ancestor(c));
                const bool sy_ok = Space::GT::dim_space_v == 1 || smaller(e.sy, pe.sy);
                if (!(smaller(e.sx, pe.sx) && sy_ok)) { all_smaller = false; break; }
            }
            const std::vector<int> targets(space.active_cells().begin(), space.active_cells().end());
            if (all_smaller) { refine_all(targets, mesh::RefinementType::temporal); return; }
            refine_all(targets, mesh::RefinementType::spatial);
        }
        throw std::runtime_error("uniform_isotropic_refine: no spatial shrink after 32 waves");
    }

    // Adaptive-mesh options (environment, all optional):
    //   APF_REF_X_POINTS="x,y,t;x,y,t"  X refined at these space-time points after the
    //                                    uniform levels, APF_REF_X_ROUNDS times (default 1),
    //                                    by the reference's refine_points_n_times
    //                                    (algorithm/support/space_time_1d.hpp:67): hanging
    //                                    nodes with weighted CellRestriction rows;
    //   APF_REF_KAPPA="seed:lo:hi"       M(p) = kappa[K] I with kappa log-uniform in [lo, hi]
    //                                    per active X cell K (the cell found by
    //                                    x_space.find_active_cell(p), fespace.hpp:616), or,
    //                                    with APF_REF_KAPPA_BLOCKS=n, per square of an n x n
    //                                    partition of the unit square;
    //   APF_REF_DRIVER_OUTER=n           (oracle driver) n outer cycles of the reference's
    //                                    adaptive driver (run_adaptive_driver) before the dump;
    //   APF_REF_Y_PASSES=n               n passes of the reference's inner loop before the
    //                                    dump: estimate, Doerfler marking, then
    //                                    refine_test_space_from_marked_source_cells
    //                                    (time_slab_adaptive_loop.hpp:2147-2186), so Y is
    //                                    finer than X.
    std::vector<std::array<double, 3>> parse_points(const char* s)
    {
        std::vector<std::array<double, 3>> out;
        std::string str(s);
        std::size_t pos = 0;
        while (pos < str.size())
        {
            std::size_t end = str.find(';', pos);
            if (end == std::string::npos) end = str.size();
            std::array<double, 3> p{};
            if (std::sscanf(str.substr(pos, end - pos).c_str(), "%lf,%lf,%lf", &p[0], &p[1], &p[2]) == 3)
                out.push_back(p);
            pos = end + 1;
        }
        return out;
    }

    int env_int(const char* name, int dflt)
    {
        const char* v = std::getenv(name);
        return v != nullptr ? std::atoi(v) : dflt;
    }

    // the adaptive-mesh options on a 2+1D X space after its uniform levels (see above);
    // returns the kappa of the active X cells (empty: M from the example)
    template<class XSpace, class Example>
    std::vector<double> apply_adaptive_options_2d(XSpace& x_space, Example& example)
    {
        if (const char* pts = std::getenv("APF_REF_X_POINTS"))
        {
            std::vector<typename XSpace::SpaceTimePoint> points;
            for (const auto& p : parse_points(pts))
                points.push_back(typename XSpace::SpaceTimePoint{p[0], p[1], p[2]});
            adaptive_algorithm::support::refine_points_n_times(x_space, points, env_int("APF_REF_X_ROUNDS", 1));
        }
        std::vector<double> kx;
        const char* ks = std::getenv("APF_REF_KAPPA");
        const int blocks = env_int("APF_REF_KAPPA_BLOCKS", 0);
        if (ks == nullptr)
            return kx;
        unsigned long long seed = 0;
        double lo = 1.0, hi = 1.0;
        std::sscanf(ks, "%llu:%lf:%lf", &seed, &lo, &hi);
        std::mt19937_64 rng(seed);
        std::uniform_real_distribution<double> uni(std::log(lo), std::log(hi));
        if (blocks > 0)
        {
            // kappa constant on each of blocks x blocks squares of the unit square
            auto table = std::make_shared<std::vector<double>>(static_cast<std::size_t>(blocks) * blocks);
            for (auto& v : *table)
                v = std::exp(uni(rng));
            example.problem.M = [table, blocks](const adaptive_algorithm::examples::SpaceTime2DPoint& p) {
                const int i = std::min(blocks - 1, std::max(0, static_cast<int>(p[0] * blocks)));
                const int j = std::min(blocks - 1, std::max(0, static_cast<int>(p[1] * blocks)));
                const double k = (*table)[static_cast<std::size_t>(i) * blocks + j];
                return finite_element::coefficients::DiffusionTensor<2>{{{k, 0.0}, {0.0, k}}};
            };
            return *table;
        }
        const auto& mesh = x_space.mesh_ref();
        auto kappa = std::make_shared<std::vector<double>>(static_cast<std::size_t>(mesh.n_cells()), 0.0);
        for (const int c : x_space.active_cells())
        {
            (*kappa)[static_cast<std::size_t>(c)] = std::exp(uni(rng));
            kx.push_back((*kappa)[static_cast<std::size_t>(c)]);
        }
        // the space's point-location index is built lazily on first use; build it here,
        // before the reference's OpenMP loops call M concurrently
        (void)x_space.find_active_cell(typename XSpace::SpaceTimePoint{0.5, 0.25, 0.5});
        const XSpace* xs = &x_space;
        example.problem.M = [xs, kappa](const adaptive_algorithm::examples::SpaceTime2DPoint& p) {
            const int c = xs->find_active_cell(p);
            const double k = (*kappa).at(static_cast<std::size_t>(c));
            return finite_element::coefficients::DiffusionTensor<2>{{{k, 0.0}, {0.0, k}}};
        };
        return kx;
    }
}
