// 1+1D element math: tensor P1 x P1 Lagrange quadrilaterals [x0, x1] x [t0, t1]
// (geometry row x0 x1 t0 t1), local index i = i_space * 2 + i_time with node 0 at the
// left / bottom end (src/finite_element/tables/quadrilateral_basis_tables.hpp:33-35).
// Polynomial integrands use their exact values (the reference's Gauss orders
// QSpace = QTime = 3 integrate them exactly); the initial datum u0 uses the reference's
// 3-point Gauss rule on the bottom edge (quadrilateral_basis_tables.hpp:19-23).
#pragma once

#include <cuda_runtime.h>

namespace apf
{
    namespace q1d
    {
        struct Quad
        {
            double x0, h, t0, k;
        };

        __device__ __forceinline__ Quad load(const double* __restrict__ g, int c)
        {
            const double2* q = reinterpret_cast<const double2*>(g + 4ll * c);
            const double2 a = q[0], b = q[1];
            return Quad{a.x, a.y - a.x, b.x, b.y - b.x};
        }

        __device__ __forceinline__ bool same(const double* __restrict__ gy, int cy, const double* __restrict__ gx, int cx)
        {
            const double4 a = reinterpret_cast<const double4*>(gy)[cy];
            const double4 b = reinterpret_cast<const double4*>(gx)[cx];
            return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w;
        }

        // 3-point Gauss-Legendre rule on [0, 1]
        __device__ __forceinline__ double gauss_x(int q)
        {
            const double r = 0.3872983346207416885; // sqrt(15) / 10
            return q == 0 ? 0.5 - r : (q == 1 ? 0.5 : 0.5 + r);
        }
        __device__ __forceinline__ double gauss_w(int q) { return q == 1 ? 8.0 / 18.0 : 5.0 / 18.0; }

        // linear nodal basis on [0, 1] and its derivative
        __device__ __forceinline__ double lin(int s, double x) { return s ? x : 1.0 - x; }
        __device__ __forceinline__ double dlin(int s) { return s ? 1.0 : -1.0; }

        // exact reference integrals: mass int N_s N_r, stiffness int N_s' N_r',
        // mixed int T_a' T_b
        __device__ __forceinline__ double mass(int s, int r) { return s == r ? 1.0 / 3.0 : 1.0 / 6.0; }
        __device__ __forceinline__ double stiff(int s, int r) { return s == r ? 1.0 : -1.0; }
        __device__ __forceinline__ double dmass(int a, int b) { return a ? 0.5 : -0.5; }

        // B(i in X, j in Y) = int (d_t psi_i phi_j + m d_x psi_i d_x phi_j) on Y cell gy with
        // the X basis of cell gx (any X cell containing gy; exact 3 x 3 Gauss otherwise)
        __device__ inline double mixed(const Quad& gy, const Quad& gx, bool same_cell, double m, int i, int j,
                                       bool dt_only)
        {
            const int si = i >> 1, ai = i & 1, sj = j >> 1, aj = j & 1;
            if (same_cell)
            {
                const double v = gy.h * mass(si, sj) * dmass(ai, aj);
                return dt_only ? v : v + m * (gy.k / gy.h) * stiff(si, sj) * mass(ai, aj);
            }
            double acc = 0.0;
            for (int qx = 0; qx < 3; ++qx)
                for (int qt = 0; qt < 3; ++qt)
                {
                    const double xi = gauss_x(qx), tau = gauss_x(qt);
                    const double x = gy.x0 + gy.h * xi, t = gy.t0 + gy.k * tau;
                    const double xx = (x - gx.x0) / gx.h, tx = (t - gx.t0) / gx.k;
                    const double psi_t = lin(si, xx) * dlin(ai) / gx.k;
                    const double psi_x = dlin(si) / gx.h * lin(ai, tx);
                    const double phi = lin(sj, xi) * lin(aj, tau);
                    const double phi_x = dlin(sj) / gy.h * lin(aj, tau);
                    double v = psi_t * phi;
                    if (!dt_only)
                        v += m * psi_x * phi_x;
                    acc += gauss_w(qx) * gauss_w(qt) * gy.h * gy.k * v;
                }
            return acc;
        }

        // g_i = g_scale int_{t0 = 0} u0 psi_i(x, 0) dx with the 3-point bottom rule
        template<class U0>
        __device__ inline double initial_load(const Quad& g, int i, double g_scale, U0 u0)
        {
            const int s = i >> 1, a = i & 1;
            if (a != 0)
                return 0.0;
            double acc = 0.0;
            for (int q = 0; q < 3; ++q)
            {
                const double xi = gauss_x(q);
                acc += g_scale * u0(g.x0 + g.h * xi) * lin(s, xi) * (g.h * gauss_w(q));
            }
            return acc;
        }
    }
}
