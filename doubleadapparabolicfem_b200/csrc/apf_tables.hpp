// Reference-element tables for tensor P_p x P_p Lagrange prisms (p = 1, 2).
//
// The local blocks of an affine prism with a cell-constant diffusion tensor are
// Kronecker products of reference integrals (exact rationals, computed here with
// exact arithmetic) and per-cell geometric factors:
//   A  ((s,a),(r,b)) = |detJ| ht  Mt[a][b] * Ks[s][r],   Ks = sum_ab Q_ab Sxx[ab]
//   B  ((s,a),(r,b)) = |detJ| Mx[s][r] Dt[a][b] + |detJ| ht Ks[s][r] Mt[a][b]
//   C  ((s,a),(r,b)) = -|detJ| Mx[s][r] S0[a] S0[b]
// with Q = G^T M G, G = J^{-T}.  These are the integrals the reference evaluates
// with its (exact) quadrature in
// src/finite_element/assembly/main_system/dense_local_main_blocks_2d.hpp:212-327,760-800.
// Basis and node order follow
// src/finite_element/basis/functions/triangular_prism_lagrange.hpp:27-30 and
// src/finite_element/nodes/triangle_equidistant.hpp (c outer, b inner, (b/p, c/p)).
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <stdexcept>

namespace apf
{
    constexpr int kMaxNs = 6;
    constexpr int kMaxNt = 3;
    constexpr int kMaxNdof = 18;
    constexpr int kMaxBottomQ = 36;

    // Tables placed in __constant__ memory, one per degree.
    struct RefTables
    {
        int p, ns, nt, ndof;
        double Sxx[4][kMaxNs][kMaxNs]; // int d_a T_s d_b T_r, ab = 00,01,10,11
        double Mx[kMaxNs][kMaxNs];     // int T_s T_r
        double ix[kMaxNs];             // int T_s
        double Mt[kMaxNt][kMaxNt];     // int S_a S_b
        double Dt[kMaxNt][kMaxNt];     // int S_a' S_b
        double it[kMaxNt];             // int S_a
        double S0[kMaxNt];             // S_a(0)
        double tri_nodes[kMaxNs][2];
        double time_nodes[kMaxNt];
        int nbq;                       // bottom (t = 0) Duffy rule of degree 4p+1
        double bq_pts[kMaxBottomQ][2];
        double bq_w[kMaxBottomQ];
        double bq_T[kMaxBottomQ][kMaxNs];
    };

    namespace tables_detail
    {
        struct Rat
        {
            std::int64_t n = 0, d = 1;
            Rat() = default;
            Rat(std::int64_t a, std::int64_t b = 1) : n(a), d(b) { norm(); }
            void norm()
            {
                if (d < 0) { n = -n; d = -d; }
                const std::int64_t g = std::gcd(n < 0 ? -n : n, d);
                if (g > 1) { n /= g; d /= g; }
            }
            Rat operator+(const Rat& o) const { return Rat(n * o.d + o.n * d, d * o.d); }
            Rat operator*(const Rat& o) const { return Rat(n * o.n, d * o.d); }
            double value() const { return static_cast<double>(n) / static_cast<double>(d); }
        };

        // bivariate polynomial sum c[a][b] x^a y^b, total degree <= 4
        struct Poly2
        {
            Rat c[5][5];
        };
        struct Poly1
        {
            Rat c[5];
        };

        inline std::int64_t fact(int k)
        {
            std::int64_t f = 1;
            for (int i = 2; i <= k; ++i) f *= i;
            return f;
        }

        // int over the reference triangle of x^a y^b = a! b! / (a+b+2)!
        inline Rat tri_monomial(int a, int b) { return Rat(fact(a) * fact(b), fact(a + b + 2)); }

        inline Poly2 mul(const Poly2& p, const Poly2& q)
        {
            Poly2 r;
            for (int a = 0; a < 5; ++a)
                for (int b = 0; a + b < 5; ++b)
                    if (p.c[a][b].n)
                        for (int e = 0; a + e < 5; ++e)
                            for (int f = 0; a + b + e + f < 5; ++f)
                                if (q.c[e][f].n)
                                    r.c[a + e][b + f] = r.c[a + e][b + f] + p.c[a][b] * q.c[e][f];
            return r;
        }
        inline Rat integrate(const Poly2& p)
        {
            Rat s;
            for (int a = 0; a < 5; ++a)
                for (int b = 0; a + b < 5; ++b)
                    if (p.c[a][b].n) s = s + p.c[a][b] * tri_monomial(a, b);
            return s;
        }
        inline Poly2 dx(const Poly2& p)
        {
            Poly2 r;
            for (int a = 1; a < 5; ++a)
                for (int b = 0; a + b < 5; ++b) r.c[a - 1][b] = p.c[a][b] * Rat(a);
            return r;
        }
        inline Poly2 dy(const Poly2& p)
        {
            Poly2 r;
            for (int a = 0; a < 5; ++a)
                for (int b = 1; a + b < 5; ++b) r.c[a][b - 1] = p.c[a][b] * Rat(b);
            return r;
        }
        inline Poly1 mul1(const Poly1& p, const Poly1& q)
        {
            Poly1 r;
            for (int a = 0; a < 5; ++a)
                for (int b = 0; a + b < 5; ++b) r.c[a + b] = r.c[a + b] + p.c[a] * q.c[b];
            return r;
        }
        inline Poly1 d1(const Poly1& p)
        {
            Poly1 r;
            for (int a = 1; a < 5; ++a) r.c[a - 1] = p.c[a] * Rat(a);
            return r;
        }
        inline Rat integrate1(const Poly1& p)
        {
            Rat s;
            for (int a = 0; a < 5; ++a) s = s + p.c[a] * Rat(1, a + 1);
            return s;
        }

        // nodal Lagrange bases on the reference triangle
        inline void triangle_basis(int p, Poly2* T)
        {
            for (int i = 0; i < 6; ++i) T[i] = Poly2{};
            if (p == 1)
            {
                T[0].c[0][0] = 1; T[0].c[1][0] = -1; T[0].c[0][1] = -1;
                T[1].c[1][0] = 1;
                T[2].c[0][1] = 1;
                return;
            }
            // p == 2: nodes v0, e01, v1, e02, e12, v2
            T[0].c[0][0] = 1; T[0].c[1][0] = -3; T[0].c[0][1] = -3; T[0].c[2][0] = 2; T[0].c[1][1] = 4; T[0].c[0][2] = 2;
            T[1].c[1][0] = 4; T[1].c[2][0] = -4; T[1].c[1][1] = -4;
            T[2].c[1][0] = -1; T[2].c[2][0] = 2;
            T[3].c[0][1] = 4; T[3].c[1][1] = -4; T[3].c[0][2] = -4;
            T[4].c[1][1] = 4;
            T[5].c[0][1] = -1; T[5].c[0][2] = 2;
        }
        inline void segment_basis(int q, Poly1* S)
        {
            for (int i = 0; i < 3; ++i) S[i] = Poly1{};
            if (q == 1)
            {
                S[0].c[0] = 1; S[0].c[1] = -1;
                S[1].c[1] = 1;
                return;
            }
            // nodes 0, 1/2, 1
            S[0].c[0] = 1; S[0].c[1] = -3; S[0].c[2] = 2;
            S[1].c[1] = 4; S[1].c[2] = -4;
            S[2].c[1] = -1; S[2].c[2] = 2;
        }
        inline double eval2(const Poly2& p, double x, double y)
        {
            double s = 0.0;
            for (int a = 0; a < 5; ++a)
                for (int b = 0; a + b < 5; ++b)
                    if (p.c[a][b].n) s += p.c[a][b].value() * std::pow(x, a) * std::pow(y, b);
            return s;
        }

        // Gauss-Legendre nodes/weights on [0,1] by Newton iteration on P_n
        // (three-term recurrence for P_n and P_n'); standard textbook method.
        inline void gauss_legendre01(int n, double* x, double* w)
        {
            const double pi = 3.14159265358979323846;
            for (int i = 0; i < n; ++i)
            {
                double z = std::cos(pi * (i + 0.75) / (n + 0.5));
                double dp = 1.0;
                for (int it = 0; it < 100; ++it)
                {
                    double p0 = 1.0, p1 = z;
                    for (int k = 2; k <= n; ++k)
                    {
                        const double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                        p0 = p1;
                        p1 = pk;
                    }
                    if (n == 1) { p1 = z; p0 = 1.0; }
                    dp = n * (z * p1 - p0) / (z * z - 1.0);
                    const double dz = p1 / dp;
                    z -= dz;
                    if (std::abs(dz) < 1e-16) break;
                }
                double p0 = 1.0, p1 = z;
                for (int k = 2; k <= n; ++k)
                {
                    const double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                    p0 = p1;
                    p1 = pk;
                }
                dp = n * (z * p1 - p0) / (z * z - 1.0);
                // node z in (-1,1) ascending order after reversal
                x[n - 1 - i] = 0.5 * (z + 1.0);
                w[n - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp);
            }
        }
    }

    inline RefTables make_ref_tables(int p)
    {
        using namespace tables_detail;
        if (p != 1 && p != 2)
            throw std::invalid_argument("reference tables: p must be 1 or 2");
        RefTables t{};
        t.p = p;
        t.ns = (p + 1) * (p + 2) / 2;
        t.nt = p + 1;
        t.ndof = t.ns * t.nt;
        Poly2 T[6];
        Poly1 S[3];
        triangle_basis(p, T);
        segment_basis(p, S);
        for (int s = 0; s < t.ns; ++s)
        {
            const Poly2 gs[2] = {dx(T[s]), dy(T[s])};
            t.ix[s] = integrate(T[s]).value();
            for (int r = 0; r < t.ns; ++r)
            {
                const Poly2 gr[2] = {dx(T[r]), dy(T[r])};
                t.Mx[s][r] = integrate(mul(T[s], T[r])).value();
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b)
                        t.Sxx[a * 2 + b][s][r] = integrate(mul(gs[a], gr[b])).value();
            }
        }
        for (int a = 0; a < t.nt; ++a)
        {
            t.it[a] = integrate1(S[a]).value();
            t.S0[a] = S[a].c[0].value();
            for (int b = 0; b < t.nt; ++b)
            {
                t.Mt[a][b] = integrate1(mul1(S[a], S[b])).value();
                t.Dt[a][b] = integrate1(mul1(d1(S[a]), S[b])).value();
            }
        }
        int id = 0;
        for (int c = 0; c <= p; ++c)
            for (int b = 0; b <= p - c; ++b)
            {
                t.tri_nodes[id][0] = static_cast<double>(b) / p;
                t.tri_nodes[id][1] = static_cast<double>(c) / p;
                ++id;
            }
        for (int a = 0; a <= p; ++a)
            t.time_nodes[a] = static_cast<double>(a) / p;
        // Duffy rule of degree 4p+1: order (4p+4)/2 = 2p+2, points (u, (1-u) v)
        const int order = (4 * p + 1 + 3) / 2;
        double gx[16], gw[16];
        gauss_legendre01(order, gx, gw);
        t.nbq = order * order;
        int k = 0;
        for (int i = 0; i < order; ++i)
            for (int j = 0; j < order; ++j)
            {
                const double u = gx[i];
                t.bq_pts[k][0] = u;
                t.bq_pts[k][1] = (1.0 - u) * gx[j];
                t.bq_w[k] = gw[i] * gw[j] * (1.0 - u);
                for (int s = 0; s < t.ns; ++s)
                    t.bq_T[k][s] = eval2(T[s], t.bq_pts[k][0], t.bq_pts[k][1]);
                ++k;
            }
        return t;
    }
}
