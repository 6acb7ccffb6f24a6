// Device-side element math shared by the assembly kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "apf_tables.hpp"

namespace apf
{
    // Affine prism: x = v0 + J xi, t = t0 + ht tau (cell_geometry.hpp:188-242).
    struct CellGeo
    {
        double x0, y0;
        double J00, J01, J10, J11;
        double iJ00, iJ01, iJ10, iJ11; // J^{-1}
        double det;                    // |det J|
        double t0, ht;
    };

    __device__ __forceinline__ CellGeo load_geo(const double* __restrict__ g, int c)
    {
        const double2* q = reinterpret_cast<const double2*>(g + 8ll * c);
        const double2 a = q[0], b = q[1], d = q[2], e = q[3];
        CellGeo o;
        o.x0 = a.x; o.y0 = a.y;
        o.J00 = b.x - a.x; o.J10 = b.y - a.y;
        o.J01 = d.x - a.x; o.J11 = d.y - a.y;
        const double dt = o.J00 * o.J11 - o.J01 * o.J10;
        const double inv = 1.0 / dt;
        o.iJ00 = o.J11 * inv; o.iJ01 = -o.J01 * inv;
        o.iJ10 = -o.J10 * inv; o.iJ11 = o.J00 * inv;
        o.det = fabs(dt);
        o.t0 = e.x;
        o.ht = e.y - e.x;
        return o;
    }

    __device__ __forceinline__ bool same_geometry(const double* __restrict__ gy, int cy,
                                                  const double* __restrict__ gx, int cx)
    {
        const double4* a = reinterpret_cast<const double4*>(gy + 8ll * cy);
        const double4* b = reinterpret_cast<const double4*>(gx + 8ll * cx);
        const double4 a0 = a[0], a1 = a[1], b0 = b[0], b1 = b[1];
        return a0.x == b0.x && a0.y == b0.y && a0.z == b0.z && a0.w == b0.w &&
               a1.x == b1.x && a1.y == b1.y && a1.z == b1.z && a1.w == b1.w;
    }

    // Q = G^T M G with G = J^{-T}: physical gradient g = G g_ref, so
    // (M g_r).g_s = g_s_ref^T Q g_r_ref.  Returned as (q00, q01, q11).
    __device__ __forceinline__ void q_form(const CellGeo& g, const double* __restrict__ m, int c,
                                           double& q00, double& q01, double& q11)
    {
        double m00 = 1.0, m01 = 0.0, m11 = 1.0;
        if (m)
        {
            m00 = m[3ll * c + 0];
            m01 = m[3ll * c + 1];
            m11 = m[3ll * c + 2];
        }
        // G = J^{-T}: G00 = iJ00, G01 = iJ10, G10 = iJ01, G11 = iJ11
        const double G00 = g.iJ00, G01 = g.iJ10, G10 = g.iJ01, G11 = g.iJ11;
        // MG columns
        const double MG00 = m00 * G00 + m01 * G10, MG01 = m00 * G01 + m01 * G11;
        const double MG10 = m01 * G00 + m11 * G10, MG11 = m01 * G01 + m11 * G11;
        q00 = G00 * MG00 + G10 * MG10;
        q01 = G00 * MG01 + G10 * MG11;
        q11 = G01 * MG01 + G11 * MG11;
    }

    __device__ __forceinline__ double ks(const RefTables& t, double q00, double q01, double q11, int s, int r)
    {
        return q00 * t.Sxx[0][s][r] + q01 * (t.Sxx[1][s][r] + t.Sxx[2][s][r]) + q11 * t.Sxx[3][s][r];
    }

    // Triangle and segment Lagrange bases (same node order as the tables).
    __device__ __forceinline__ double tri_basis(int p, int s, double x, double y)
    {
        const double l0 = 1.0 - x - y, l1 = x, l2 = y;
        if (p == 1)
            return s == 0 ? l0 : (s == 1 ? l1 : l2);
        switch (s)
        {
        case 0: return l0 * (2.0 * l0 - 1.0);
        case 1: return 4.0 * l0 * l1;
        case 2: return l1 * (2.0 * l1 - 1.0);
        case 3: return 4.0 * l0 * l2;
        case 4: return 4.0 * l1 * l2;
        default: return l2 * (2.0 * l2 - 1.0);
        }
    }
    __device__ __forceinline__ double seg_basis(int p, int a, double t)
    {
        if (p == 1)
            return a == 0 ? 1.0 - t : t;
        if (a == 0) return (2.0 * t - 1.0) * (t - 1.0);
        if (a == 1) return 4.0 * t * (1.0 - t);
        return t * (2.0 * t - 1.0);
    }

    // Same-cell mixed block B^{YY}((s,a),(r,b)) and its time-derivative part.
    __device__ __forceinline__ double b_same(const RefTables& t, const CellGeo& g, double q00, double q01,
                                             double q11, int i, int j, bool dt_only)
    {
        const int s = i / t.nt, a = i % t.nt, r = j / t.nt, b = j % t.nt;
        const double dtpart = g.det * t.Mx[s][r] * t.Dt[a][b];
        if (dt_only)
            return dtpart;
        return dtpart + g.det * g.ht * ks(t, q00, q01, q11, s, r) * t.Mt[a][b];
    }

    // Coefficient of X basis function i (on X cell gx) at Y node k (on Y cell gy):
    // psi_i restricted to the Y prism equals sum_k psi_i(node_k) phi_k exactly.
    __device__ __forceinline__ double transfer(const RefTables& t, const CellGeo& gy, const CellGeo& gx, int i, int k)
    {
        const int sk = k / t.nt, ak = k % t.nt;
        const double xi = t.tri_nodes[sk][0], eta = t.tri_nodes[sk][1], tau = t.time_nodes[ak];
        const double px = gy.x0 + gy.J00 * xi + gy.J01 * eta;
        const double py = gy.y0 + gy.J10 * xi + gy.J11 * eta;
        const double pt = gy.t0 + gy.ht * tau;
        const double dx = px - gx.x0, dy = py - gx.y0;
        const double rx = gx.iJ00 * dx + gx.iJ01 * dy;
        const double ry = gx.iJ10 * dx + gx.iJ11 * dy;
        const double rt = (pt - gx.t0) / gx.ht;
        const int si = i / t.nt, ai = i % t.nt;
        return tri_basis(t.p, si, rx, ry) * seg_basis(t.p, ai, rt);
    }

    // The same between degrees: basis function i of the degree-tb.p prism gx at node k of the
    // degree-tn.p prism gy (a degree-p function lies in the degree-(p+1) space exactly)
    __device__ __forceinline__ double transfer_between(const RefTables& tn, const RefTables& tb, const CellGeo& gy,
                                                       const CellGeo& gx, int i, int k)
    {
        const int sk = k / tn.nt, ak = k % tn.nt;
        const double xi = tn.tri_nodes[sk][0], eta = tn.tri_nodes[sk][1], tau = tn.time_nodes[ak];
        const double px = gy.x0 + gy.J00 * xi + gy.J01 * eta;
        const double py = gy.y0 + gy.J10 * xi + gy.J11 * eta;
        const double pt = gy.t0 + gy.ht * tau;
        const double dx = px - gx.x0, dy = py - gx.y0;
        const double rx = gx.iJ00 * dx + gx.iJ01 * dy;
        const double ry = gx.iJ10 * dx + gx.iJ11 * dy;
        const double rt = (pt - gx.t0) / gx.ht;
        const int si = i / tb.nt, ai = i % tb.nt;
        return tri_basis(tb.p, si, rx, ry) * seg_basis(tb.p, ai, rt);
    }
}
