// The adaptive driver's G^delta estimator on the device (p = 1 systems: G of degree 2).
//
// On the accepted Y mesh the reference builds the space G of degree p+1 on the Y cells
// (broken in time like Y), assembles A_G, f_G and the mixed block B(X, G), solves
//   A_G lambda_G = f_G - B(X, G)^T u_delta
// directly, prolongs lambda_delta nodally into G and reports ||lambda_G - lambda_delta||^2
// in the A_G energy (algorithm/adaptive_driver.hpp:2690-2900).
//
// Here B(X, G)^T u_delta is formed without the mixed-degree block: u_delta restricted to a Y
// cell is a degree-p polynomial, so it lies in G (which is broken in time) and
// B(X, G)^T u_delta = B(G, G)^T u_G with u_G its nodal interpolant in G; every block is then
// a same-degree G form gathered by the assembly kernels (G as both test and trial space on
// the Y cells).  lambda_G comes from AMG-preconditioned CG.
#include <cmath>
#include <numeric>
#include <vector>

#include "apf_gdelta.cuh"

namespace apf
{
    GDeltaResult g_delta(cudaStream_t s, System& S, int n_g, const std::vector<int>& off,
                         const std::vector<int>& dofs, const std::vector<double>& w, double tol)
    {
        const SystemInputs& in = S.in;
        require(in.dim == 2 && in.p == 1, APF_ERR_INVALID, "G^delta estimator: 2+1D systems of degree 1 (G of degree 2)");
        require(S.solution.size() == static_cast<std::size_t>(in.n_lambda + in.n_u), APF_ERR_INVALID,
                "G^delta estimator: solve the main system first");
        constexpr int q = 2, ndq = 18;
        const int ny = in.n_y_cells;
        require(n_g >= 0 && off.size() == static_cast<std::size_t>(ny) * ndq + 1 && off.front() == 0 &&
                    off.back() == static_cast<int>(dofs.size()) && dofs.size() == w.size(),
                APF_ERR_INVALID, "G^delta estimator: the G restriction does not match the Y cells");
        for (std::size_t r = 0; r + 1 < off.size(); ++r)
            require(off[r] <= off[r + 1], APF_ERR_INVALID, "G^delta estimator: restriction offsets");
        for (const int d : dofs)
            require(d >= 0 && d < n_g, APF_ERR_INVALID, "G^delta estimator: restriction DOF out of range");
        GDeltaResult res{};
        res.n_g = n_g;
        if (n_g == 0)
            return res;

        // G as both spaces on the Y cells (identity Y -> X map)
        SystemInputs g;
        g.p = q;
        g.ndof = ndq;
        g.dim = 2;
        g.n_y_cells = ny;
        g.n_x_cells = ny;
        g.n_lambda = n_g;
        g.n_u = n_g;
        g.u0_kind = in.u0_kind;
        g.zero_tol = in.zero_tol;
        g.g_scale = in.g_scale;
        auto clone = [&](const auto& src, auto& dst) {
            dst.allocate(src.size(), s);
            if (src.size())
                APF_CUDA(cudaMemcpyAsync(dst.get(), src.get(), src.size() * sizeof(*src.get()), cudaMemcpyDeviceToDevice,
                                         s));
        };
        clone(in.y_geo, g.y_geo);
        clone(in.y_geo, g.x_geo);
        if (in.m_y.size())
            clone(in.m_y, g.m_y);
        if (in.ell.size())
            clone(in.ell, g.ell);
        {
            std::vector<int> iota(static_cast<std::size_t>(ny));
            std::iota(iota.begin(), iota.end(), 0);
            g.y_to_x.upload(iota.data(), iota.size());
        }
        g.y_off.upload(off.data(), off.size());
        g.y_dofs.upload(dofs.data(), dofs.size());
        g.y_w.upload(w.data(), w.size());
        g.x_off.upload(off.data(), off.size());
        g.x_dofs.upload(dofs.data(), dofs.size());
        g.x_w.upload(w.data(), w.size());
        prepare_inputs(s, g);

        DeviceCsr A, Bt;
        DeviceBuffer<double> f;
        {
            APF_HOST_RANGE("g_delta_assembly");
            const Incidence inc = build_incidence(s, n_g, ny, nullptr, nullptr, g.y_off.get(), g.y_dofs.get(), ndq);
            const int offs[1] = {0};
            const Incidence* incs[1] = {&inc};
            const int ka[1] = {K_AY};
            gather_csr(s, g, g.zero_tol, n_g, n_g, 1, ka, incs, offs, g.kmax, A);
            const int kbt[1] = {K_BT};
            gather_csr(s, g, g.zero_tol, n_g, n_g, 1, kbt, incs, offs, g.kmax, Bt);
            gather_vector_host(s, g, g.zero_tol, 0, inc, n_g, g.ell.size() ? g.ell.get() : nullptr, g.u0_kind,
                               g.g_scale, f);
        }
        // u_delta and lambda_delta in G (nodal interpolation, exact)
        const int nl = in.n_lambda;
        DeviceBuffer<double> ug(n_g, s), lg(n_g, s);
        interpolate_to_space(s, q, in.p, ny, g.y_geo.get(), in.y_to_x.get(), in.x_geo.get(), in.x_off.get(),
                             in.x_dofs.get(), in.x_w.get(), S.solution.get() + nl, g.y_off.get(), g.y_dofs.get(),
                             g.y_w.get(), n_g, ug.get());
        interpolate_to_space(s, q, in.p, ny, g.y_geo.get(), nullptr, in.y_geo.get(), in.y_off.get(), in.y_dofs.get(),
                             in.y_w.get(), S.solution.get(), g.y_off.get(), g.y_dofs.get(), g.y_w.get(), n_g, lg.get());
        DeviceBuffer<double> rhs(n_g, s), lam(n_g, s), r(n_g, s), z(n_g, s), pv(n_g, s), qv(n_g, s);
        copy(s, n_g, f.get(), rhs.get());
        spmv(s, Bt, ug.get(), rhs.get(), -1.0, 1.0);
        lam.zero();
        // lambda_G by CG with an SA-AMG V-cycle (time levels aggregated separately)
        Amg amg;
        {
            APF_HOST_RANGE("g_delta_amg_setup");
            DeviceBuffer<int> comp;
            dof_time_components(s, g, true, comp);
            const AmgOptions o = S.precond ? S.precond_opts : AmgOptions{};
            amg.setup(s, A, o, S.ws, comp.get());
        }
        copy(s, n_g, rhs.get(), r.get());
        const double bn = std::sqrt(dot_host(s, S.ws, n_g, rhs.get(), rhs.get()));
        double rn = bn;
        int its = 0;
        if (bn > 0.0)
        {
            APF_HOST_RANGE("g_delta_pcg");
            amg.apply(s, r.get(), z.get());
            copy(s, n_g, z.get(), pv.get());
            double rz = dot_host(s, S.ws, n_g, r.get(), z.get());
            for (its = 1; its <= 1000; ++its)
            {
                spmv(s, A, pv.get(), qv.get());
                const double alpha = rz / dot_host(s, S.ws, n_g, pv.get(), qv.get());
                axpby(s, n_g, alpha, pv.get(), 1.0, lam.get());
                axpby(s, n_g, -alpha, qv.get(), 1.0, r.get());
                rn = std::sqrt(dot_host(s, S.ws, n_g, r.get(), r.get()));
                if (!(rn > tol * bn))
                    break;
                amg.apply(s, r.get(), z.get());
                const double rz2 = dot_host(s, S.ws, n_g, r.get(), z.get());
                axpby(s, n_g, 1.0, z.get(), rz2 / rz, pv.get());
                rz = rz2;
            }
        }
        require(!(rn > tol * bn), APF_ERR_NOT_CONVERGED, "G^delta estimator: CG missed its tolerance");
        // ||lambda_G - I_G lambda_delta||^2 in the A_G energy
        axpby(s, n_g, -1.0, lg.get(), 1.0, lam.get());
        spmv(s, A, lam.get(), qv.get());
        const double e = dot_host(s, S.ws, n_g, lam.get(), qv.get());
        require(std::isfinite(e), APF_ERR_NUMERIC, "G^delta estimator: non-finite energy");
        res.lambda_difference_squared = e > 0.0 ? e : 0.0;
        res.iterations = its;
        res.relative_residual = bn > 0.0 ? rn / bn : 0.0;
        return res;
    }
}
