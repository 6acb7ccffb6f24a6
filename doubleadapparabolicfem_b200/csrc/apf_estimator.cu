// Equilibrated-flux estimator of one inner iteration (p = 1) on the device.
//
// The reference computes, per time slab n and spatial vertex a, the mixed RT_1 x P_1
// problem on the vertex patch omega_a (time_slab_equilibrated_flux_reconstruction.hpp,
// dense_local_error_blocks_2d.hpp, vec_f_2d.hpp:27-80, vec_g_2d.hpp:30-95):
//   (M^-1 sigma, tau) + (div tau, r)      = -(psi_a grad theta~, tau)
//   (div sigma, q)          + (mu, E q)   =  (psi_a (l - d_t u) - grad psi_a . M grad theta~, q)
//   E r = 0   (one mean-zero row per time DOF, interior patches only)
// with theta~ = lambda~ + u, flux RT_1(omega_a) x P_1(slab) with zero normal flux on the
// patch boundary except on the physical boundary of boundary patches, and broken P_1 x P_1
// scalars; then sigma = sum_a sigma_a and per slab cell K
//   flux^2_K = ||M^-1/2 (sigma + M grad theta~)||^2_K,  div^2_K = ||l - d_t u - div sigma||^2_K.
//
// B200 design: the space-time patch operator is Mt (x) [A_x B_x^T 0; B_x 0 e^T; 0 e 0] for
// cell-constant M on a slab, so after multiplying the right-hand side by Mt^-1 the problem
// splits into one spatial system per time DOF sharing one matrix: one warp assembles that
// matrix (size ~ 7 x patch valence) in its slice of shared memory from reference-cell
// integral tables, factors it once (LU with partial pivoting) and solves both time
// components; patches are sorted into size buckets so each launch sizes shared memory to
// its largest patch.  Each patch writes its flux restricted
// to each of its cells into the cell's slot of that patch's vertex (3 slots per triangle),
// so the per-cell indicator kernel sums the slots in a fixed order: no atomics.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <future>
#include <numeric>
#include <thread>
#include <unordered_map>
#include <vector>

#include "apf_estimator.cuh"
#include "apf_quad1d.cuh"

namespace apf
{
    namespace
    {
        // reference RT_1 basis (8 functions) over the vector monomials
        // (1,0) (x,0) (y,0) (0,1) (0,x) (0,y) (x^2,xy) (xy,y^2); DOFs: edge k (opposite vertex
        // k, from v_{k+1} to v_{k+2}) moments with q = 1 and q = 2s-1 against the outward
        // normal, then the two interior moments int sigma_x, int sigma_y.
        struct EstTables
        {
            double rt[8][8];
            int nq;
            double qp[16][2];
            double qw[16];
            double tg[2];
            double tw[2];
        };
        __constant__ EstTables c_est;

        void mono(double x, double y, double v[8][2])
        {
            const double m[8][2] = {{1, 0}, {x, 0}, {y, 0}, {0, 1}, {0, x}, {0, y}, {x * x, x * y}, {x * y, y * y}};
            std::memcpy(v, m, sizeof(m));
        }

        void solve_dense_host(std::vector<double> a, int n, std::vector<double>& inv)
        {
            // Gauss-Jordan with partial pivoting: inv = a^-1 (row-major)
            inv.assign(static_cast<std::size_t>(n) * n, 0.0);
            for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
            for (int k = 0; k < n; ++k)
            {
                int p = k;
                for (int i = k + 1; i < n; ++i)
                    if (std::fabs(a[(size_t)i * n + k]) > std::fabs(a[(size_t)p * n + k])) p = i;
                for (int j = 0; j < n; ++j)
                {
                    std::swap(a[(size_t)k * n + j], a[(size_t)p * n + j]);
                    std::swap(inv[(size_t)k * n + j], inv[(size_t)p * n + j]);
                }
                const double d = a[(size_t)k * n + k];
                for (int j = 0; j < n; ++j)
                {
                    a[(size_t)k * n + j] /= d;
                    inv[(size_t)k * n + j] /= d;
                }
                for (int i = 0; i < n; ++i)
                {
                    if (i == k) continue;
                    const double f = a[(size_t)i * n + k];
                    if (f == 0.0) continue;
                    for (int j = 0; j < n; ++j)
                    {
                        a[(size_t)i * n + j] -= f * a[(size_t)k * n + j];
                        inv[(size_t)i * n + j] -= f * inv[(size_t)k * n + j];
                    }
                }
            }
        }

        EstTables make_est_tables()
        {
            EstTables t{};
            // Gauss-Legendre on [0,1], 4 points -> Duffy rule of degree 5 (16 points)
            const double g4x[4] = {0.06943184420297371, 0.33000947820757187, 0.6699905217924281, 0.9305681557970263};
            const double g4w[4] = {0.17392742256872692, 0.3260725774312731, 0.3260725774312731, 0.17392742256872692};
            t.nq = 16;
            int k = 0;
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; ++j)
                {
                    t.qp[k][0] = g4x[i];
                    t.qp[k][1] = (1.0 - g4x[i]) * g4x[j];
                    t.qw[k] = g4w[i] * g4w[j] * (1.0 - g4x[i]);
                    ++k;
                }
            t.tg[0] = 0.5 - 0.5 / std::sqrt(3.0);
            t.tg[1] = 0.5 + 0.5 / std::sqrt(3.0);
            t.tw[0] = t.tw[1] = 0.5;
            // DOF matrix D[dof][monomial]
            const double v[3][2] = {{0, 0}, {1, 0}, {0, 1}};
            std::vector<double> D(64, 0.0);
            for (int e = 0; e < 3; ++e)
            {
                const double* P = v[(e + 1) % 3];
                const double* Q = v[(e + 2) % 3];
                const double dx = Q[0] - P[0], dy = Q[1] - P[1];
                const double nrm[2] = {dy, -dx}; // outward (reference triangle is counter-clockwise) x edge length
                for (int g = 0; g < 4; ++g)
                {
                    const double s = g4x[g];
                    double m[8][2];
                    mono(P[0] + s * dx, P[1] + s * dy, m);
                    for (int mm = 0; mm < 8; ++mm)
                    {
                        const double fn = m[mm][0] * nrm[0] + m[mm][1] * nrm[1];
                        D[(2 * e + 0) * 8 + mm] += g4w[g] * fn;
                        D[(2 * e + 1) * 8 + mm] += g4w[g] * fn * (2.0 * s - 1.0);
                    }
                }
            }
            for (int q = 0; q < 16; ++q)
            {
                double m[8][2];
                mono(t.qp[q][0], t.qp[q][1], m);
                for (int mm = 0; mm < 8; ++mm)
                {
                    D[6 * 8 + mm] += t.qw[q] * m[mm][0];
                    D[7 * 8 + mm] += t.qw[q] * m[mm][1];
                }
            }
            // basis coefficients C with D C^T = I  ->  C^T = D^-1
            std::vector<double> Dinv;
            solve_dense_host(D, 8, Dinv);
            for (int j = 0; j < 8; ++j)
                for (int mm = 0; mm < 8; ++mm)
                    t.rt[j][mm] = Dinv[(size_t)mm * 8 + j];
            return t;
        }

        __device__ __forceinline__ void rt_ref(int j, double x, double y, double& vx, double& vy, double& dv)
        {
            const double* c = c_est.rt[j];
            vx = c[0] + c[1] * x + c[2] * y + c[6] * x * x + c[7] * x * y;
            vy = c[3] + c[4] * x + c[5] * y + c[6] * x * y + c[7] * y * y;
            dv = c[1] + c[5] + 3.0 * c[6] * x + 3.0 * c[7] * y;
        }

        struct Cell
        {
            double x0, y0, J00, J01, J10, J11, det, t0, ht;
            double g[3][2]; // gradients of the barycentric functions
            double m00, m01, m11, mi00, mi01, mi11;
            double ell;
        };

        __device__ Cell load_cell(const double* geo, const double* m, const double* ell, int c)
        {
            Cell k;
            const double* g = geo + 8ll * c;
            k.x0 = g[0]; k.y0 = g[1];
            k.J00 = g[2] - g[0]; k.J10 = g[3] - g[1];
            k.J01 = g[4] - g[0]; k.J11 = g[5] - g[1];
            k.det = k.J00 * k.J11 - k.J01 * k.J10;
            k.t0 = g[6]; k.ht = g[7] - g[6];
            const double id = 1.0 / k.det;
            // grad lambda_1 = first row of J^-1, grad lambda_2 = second row
            k.g[1][0] = k.J11 * id;  k.g[1][1] = -k.J01 * id;
            k.g[2][0] = -k.J10 * id; k.g[2][1] = k.J00 * id;
            k.g[0][0] = -k.g[1][0] - k.g[2][0];
            k.g[0][1] = -k.g[1][1] - k.g[2][1];
            k.m00 = 1.0; k.m01 = 0.0; k.m11 = 1.0;
            if (m)
            {
                k.m00 = m[3ll * c]; k.m01 = m[3ll * c + 1]; k.m11 = m[3ll * c + 2];
            }
            const double md = k.m00 * k.m11 - k.m01 * k.m01;
            k.mi00 = k.m11 / md; k.mi01 = -k.m01 / md; k.mi11 = k.m00 / md;
            k.ell = ell ? ell[c] : 0.0;
            return k;
        }

        // physical basis value / divergence at reference point; edge functions carry sign(detJ)
        __device__ __forceinline__ void rt_phys(const Cell& k, int j, double x, double y, double& vx, double& vy, double& dv)
        {
            double rx, ry, rd;
            rt_ref(j, x, y, rx, ry, rd);
            const double s = (j < 6 && k.det < 0.0) ? -1.0 : 1.0;
            const double f = s / k.det;
            vx = f * (k.J00 * rx + k.J01 * ry);
            vy = f * (k.J10 * rx + k.J11 * ry);
            dv = f * rd;
        }

        struct PatchArgs
        {
            int n_patches;
            const int* patch_slab;
            const int* patch_topo;
            const int* topo_ptr;       // patch cells of each topology patch
            const int* topo_cell;      // local cell index in the slab cell list
            const int* topo_center;    // local vertex index of the patch vertex in that cell
            const int* topo_edge;      // per patch cell x 3: free patch edge id (-1: constrained) | sign_p bit 30
            const int* topo_nfree;
            const int* topo_boundary;
            const int* slab_ptr;
            const int* slab_cells;
            const double* geo;
            const double* m;
            const double* ell;
            const double* theta;       // [cell][6] nodal lambda~ + u
            const double* u;           // [cell][6] nodal u
            double* sigma;             // [cell][3 slots][2 time][8]
            int nmax;
            int* status;
        };

        // Reference-cell integrals of the RT_1 basis against itself, its divergence and the
        // barycentric functions (exact with the 16-point rule: polynomial degree <= 4).
        struct PatchTables
        {
            double r00[8][8], r01[8][8], r11[8][8]; // int phi_j^a phi_l^b
            double rd[8][3];                       // int div phi_l lambda_r
            double rl[3][8][2];                    // int lambda_a phi_j^c
            double mm[3][3];                       // int lambda_a lambda_r
            double mmm[3][3][3];                   // int lambda_a lambda_s lambda_r
        };
        constexpr int kPatchTableDoubles = sizeof(PatchTables) / sizeof(double);
        // local entries of one patch cell (the index t of the patch kernels' entry loop)
        constexpr int kCellEntries = 113;

        PatchTables make_patch_tables(const EstTables& t)
        {
            PatchTables p{};
            for (int q = 0; q < t.nq; ++q)
            {
                const double x = t.qp[q][0], y = t.qp[q][1], w = t.qw[q];
                double v[8][2], d[8];
                for (int j = 0; j < 8; ++j)
                {
                    const double* c = t.rt[j];
                    v[j][0] = c[0] + c[1] * x + c[2] * y + c[6] * x * x + c[7] * x * y;
                    v[j][1] = c[3] + c[4] * x + c[5] * y + c[6] * x * y + c[7] * y * y;
                    d[j] = c[1] + c[5] + 3.0 * c[6] * x + 3.0 * c[7] * y;
                }
                const double l3[3] = {1.0 - x - y, x, y};
                for (int j = 0; j < 8; ++j)
                    for (int l = 0; l < 8; ++l)
                    {
                        p.r00[j][l] += w * v[j][0] * v[l][0];
                        p.r01[j][l] += w * v[j][0] * v[l][1];
                        p.r11[j][l] += w * v[j][1] * v[l][1];
                    }
                for (int l = 0; l < 8; ++l)
                    for (int r = 0; r < 3; ++r)
                        p.rd[l][r] += w * d[l] * l3[r];
                for (int a = 0; a < 3; ++a)
                    for (int j = 0; j < 8; ++j)
                        for (int c = 0; c < 2; ++c)
                            p.rl[a][j][c] += w * l3[a] * v[j][c];
                for (int a = 0; a < 3; ++a)
                    for (int r = 0; r < 3; ++r)
                    {
                        p.mm[a][r] += w * l3[a] * l3[r];
                        for (int s2 = 0; s2 < 3; ++s2)
                            p.mmm[a][s2][r] += w * l3[a] * l3[s2] * l3[r];
                    }
            }
            return p;
        }

        // block-wide barrier of a patch team (one warp: __syncwarp)
        template<int W>
        __device__ __forceinline__ void team_sync()
        {
            if (W == 1)
                __syncwarp();
            else
                __syncthreads();
        }

        // K[i][j] -= K[i][col] u for rows col < i < n (one thread per column j > col): four
        // rows per step, loads before stores, so four shared-memory round trips overlap (the
        // column col is read only, the column j belongs to this thread)
        template<class V>
        __device__ __forceinline__ void lu_column_update(V* K, int LD, int col, int j, int n, V u)
        {
            int i = col + 1;
            for (; i + 3 < n; i += 4)
            {
                const V l0 = K[i * LD + col], l1 = K[(i + 1) * LD + col];
                const V l2 = K[(i + 2) * LD + col], l3 = K[(i + 3) * LD + col];
                const V a0 = K[i * LD + j], a1 = K[(i + 1) * LD + j];
                const V a2 = K[(i + 2) * LD + j], a3 = K[(i + 3) * LD + j];
                K[i * LD + j] = a0 - l0 * u;
                K[(i + 1) * LD + j] = a1 - l1 * u;
                K[(i + 2) * LD + j] = a2 - l2 * u;
                K[(i + 3) * LD + j] = a3 - l3 * u;
            }
            for (; i < n; ++i)
                K[i * LD + j] -= K[i * LD + col] * u;
        }

        // arg-max over the team: (best, bi) of every thread -> the team's (largest value,
        // smallest index among ties), identical on every thread
        template<int W>
        __device__ __forceinline__ void team_argmax(double& best, int& bi)
        {
            for (int o = 16; o > 0; o >>= 1)
            {
                const double ov = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi))
                {
                    best = ov;
                    bi = oi;
                }
            }
            if (W == 1)
                return;
            __shared__ double s_v[W];
            __shared__ int s_i[W];
            const int warp = threadIdx.x >> 5;
            if ((threadIdx.x & 31) == 0)
            {
                s_v[warp] = best;
                s_i[warp] = bi;
            }
            __syncthreads();
            best = s_v[0];
            bi = s_i[0];
            for (int w = 1; w < W; ++w)
                if (s_v[w] > best || (s_v[w] == best && s_i[w] < bi))
                {
                    best = s_v[w];
                    bi = s_i[w];
                }
            __syncthreads();
        }

        // One warp per patch; the patch system (n rows, two right-hand-side columns at n and
        // n + 1) lives in this warp's slice of shared memory with an odd row stride, so
        // column walks (pivot search, back substitution) are free of bank conflicts.
        //   assembly : lanes over the 113 local entries of each patch cell, from the
        //              reference-cell tables (Piola map, cell-constant M);
        //   LU       : partial pivoting by a warp arg-max, right-looking update with lanes
        //              over columns, applied to both right-hand sides at once;
        //   solve    : column-oriented back substitution, lanes over rows.
        // Patches arrive sorted into size buckets; NMAX is the bucket's bound.
        //
        // F32 = true: the matrix is assembled and factored in FP32 (half the shared memory per
        // team, so twice the teams per SM), followed by one FP64 iterative-refinement step:
        // the FP64 residual Mt^-1 b - K x is formed matrix-free by a second pass over the
        // patch cells' local entries (row sums in a fixed order, so the result does not depend
        // on scheduling), solved with the FP32 factors and pivots, and added to x in FP64.
        template<int NMAX, int W, bool F32>
        __global__ void __launch_bounds__(32 * W) patch_solve(PatchArgs A, const PatchTables* __restrict__ tables,
                                                          const int* __restrict__ order, int count)
        {
            using V = typename std::conditional<F32, float, double>::type;
            constexpr int LD = NMAX + 3; // odd: NMAX is even
            extern __shared__ double sm[];
            PatchTables& T = *reinterpret_cast<PatchTables*>(sm);
            // F32: x [2][NMAX], b [2][NMAX], K x [2][NMAX] and one cell's entries [kCellEntries]
            // in FP64 ahead of the matrix
            double* xd = sm + kPatchTableDoubles + (kPatchTableDoubles & 1);
            double* bd = xd + 2 * NMAX;
            double* kx = bd + 2 * NMAX;
            double* ev = kx + 2 * NMAX;
            V* K = reinterpret_cast<V*>(xd + (F32 ? 6 * NMAX + kCellEntries : 0));
            int* piv = reinterpret_cast<int*>(K + NMAX * LD);
            const int lane = threadIdx.x;
            constexpr int NT = 32 * W; // threads of the patch team
            for (int i = lane; i < kPatchTableDoubles; i += NT)
                sm[i] = reinterpret_cast<const double*>(tables)[i];
            team_sync<W>();
            for (int idx = blockIdx.x; idx < count; idx += gridDim.x)
            {
                const int p = order[idx];
                const int slab = A.patch_slab[p], tp = A.patch_topo[p];
                const int cb = A.topo_ptr[tp], ce = A.topo_ptr[tp + 1], nc = ce - cb;
                const int nfree = A.topo_nfree[tp];
                const bool interior = A.topo_boundary[tp] == 0;
                const int nf = 2 * nfree + 2 * nc;
                const int n = nf + 3 * nc + (interior ? 1 : 0);
                if (n > NMAX)
                {
                    if (lane == 0)
                        atomicExch(A.status, APF_ERR_CAPACITY);
                    continue;
                }
                const int sb = A.slab_ptr[slab];
                for (int i = lane; i < n * LD; i += NT)
                    K[i] = 0.0;
                team_sync<W>();
                // every local entry (row, col, value) of the patch system, cell by cell, with its
                // entry index t < kCellEntries (the two entries of a symmetric pair share t);
                // cols n, n + 1 are the two right-hand sides.  after_cell(pd, sbase) runs once
                // per cell after the cell's entries (behind a team barrier).
                auto cell_entries = [&](auto&& sink, auto&& after_cell) {
                double ht = 0.0;
                for (int ic = 0; ic < nc; ++ic)
                {
                    const int c = A.slab_cells[sb + A.topo_cell[cb + ic]];
                    const int a = A.topo_center[cb + ic];
                    const Cell k = load_cell(A.geo, A.m, A.ell, c);
                    ht = k.ht;
                    const double adet = fabs(k.det);
                    // local dof -> patch dof and the coefficient of the physical basis:
                    // phi_j = e_j J phi^_j, e_j = orientation x Piola sign / det
                    int pd[8];
                    double e[8];
                    for (int ed = 0; ed < 3; ++ed)
                    {
                        const int code = A.topo_edge[3 * (cb + ic) + ed];
                        const int pe = code & 0xffff;
                        const double sp = (code >> 30) & 1 ? -1.0 : 1.0;
                        const bool free_edge = pe != 0xffff;
                        pd[2 * ed] = free_edge ? 2 * pe : -1;
                        pd[2 * ed + 1] = free_edge ? 2 * pe + 1 : -1;
                        e[2 * ed] = sp / k.det;     // (sdet sp) (sdet / det)
                        e[2 * ed + 1] = 1.0 / k.det; // (sdet sp sp) (sdet / det)
                    }
                    pd[6] = 2 * nfree + 2 * ic;
                    pd[7] = 2 * nfree + 2 * ic + 1;
                    e[6] = e[7] = 1.0 / k.det;
                    const int sbase = nf + 3 * ic;
                    // S = J^T M^-1 J
                    const double q00 = k.mi00 * k.J00 + k.mi01 * k.J10, q10 = k.mi01 * k.J00 + k.mi11 * k.J10;
                    const double q01 = k.mi00 * k.J01 + k.mi01 * k.J11, q11 = k.mi01 * k.J01 + k.mi11 * k.J11;
                    const double S00 = k.J00 * q00 + k.J10 * q10;
                    const double S01 = k.J00 * q01 + k.J10 * q11;
                    const double S11 = k.J01 * q01 + k.J11 * q11;
                    // time-weighted gradients of theta~: gth[kk] = grad theta~ tested with time basis kk
                    const double* th = A.theta + 6ll * c;
                    const double* uu = A.u + 6ll * c;
                    double gth[2][2];
                    for (int kk = 0; kk < 2; ++kk)
                    {
                        gth[kk][0] = gth[kk][1] = 0.0;
                        for (int s2 = 0; s2 < 3; ++s2)
                        {
                            const double wt = k.ht * ((kk == 0 ? 1.0 / 3.0 : 1.0 / 6.0) * th[2 * s2] +
                                                      (kk == 0 ? 1.0 / 6.0 : 1.0 / 3.0) * th[2 * s2 + 1]);
                            gth[kk][0] += k.g[s2][0] * wt;
                            gth[kk][1] += k.g[s2][1] * wt;
                        }
                    }
                    double du[3];
                    for (int s2 = 0; s2 < 3; ++s2)
                        du[s2] = (uu[2 * s2 + 1] - uu[2 * s2]) / k.ht;
                    for (int t = lane; t < kCellEntries; t += NT)
                    {
                        if (t < 64)
                        {
                            const int j = t >> 3, l = t & 7;
                            if (pd[j] < 0 || pd[l] < 0)
                                continue;
                            const double r = S00 * T.r00[j][l] + S01 * (T.r01[j][l] + T.r01[l][j]) + S11 * T.r11[j][l];
                            sink(t, pd[j], pd[l], e[j] * e[l] * adet * r);
                        }
                        else if (t < 88)
                        {
                            const int r = (t - 64) >> 3, l = (t - 64) & 7;
                            if (pd[l] < 0)
                                continue;
                            const double v = e[l] * adet * T.rd[l][r];
                            sink(t, sbase + r, pd[l], v);
                            sink(t, pd[l], sbase + r, v);
                        }
                        else if (t < 104)
                        {
                            const int j = (t - 88) >> 1, kk = (t - 88) & 1;
                            if (pd[j] < 0)
                                continue;
                            const double gJ0 = gth[kk][0] * k.J00 + gth[kk][1] * k.J10;
                            const double gJ1 = gth[kk][0] * k.J01 + gth[kk][1] * k.J11;
                            sink(t, pd[j], n + kk, -e[j] * adet * (gJ0 * T.rl[a][j][0] + gJ1 * T.rl[a][j][1]));
                        }
                        else if (t < 110)
                        {
                            const int r = (t - 104) >> 1, kk = (t - 104) & 1;
                            double acc = k.ell * T.mm[a][r];
                            for (int s2 = 0; s2 < 3; ++s2)
                                acc -= du[s2] * T.mmm[a][s2][r];
                            const double mg0 = k.m00 * gth[kk][0] + k.m01 * gth[kk][1];
                            const double mg1 = k.m01 * gth[kk][0] + k.m11 * gth[kk][1];
                            const double gpm = k.g[a][0] * mg0 + k.g[a][1] * mg1;
                            sink(t, sbase + r, n + kk, (0.5 * k.ht * acc - gpm / 6.0) * adet);
                        }
                        else if (interior)
                        {
                            // mean-zero row: int_K lambda_r = |K| / 6 on the reference scale
                            const int r = t - 110;
                            const double v = adet / 6.0;
                            sink(t, n - 1, sbase + r, v);
                            sink(t, sbase + r, n - 1, v);
                        }
                    }
                    team_sync<W>();
                    after_cell(pd, sbase);
                }
                return ht;
                };
                const double ht = cell_entries(
                    [&](int, int row, int col, double v) { K[row * LD + col] += static_cast<V>(v); },
                    [](const int*, int) {});
                // right-hand sides times Mt^-1 (Mt = ht [[1/3,1/6],[1/6,1/3]], inverse (1/ht) [[4,-2],[-2,4]])
                for (int i = lane; i < n; i += NT)
                {
                    const double b0 = K[i * LD + n], b1 = K[i * LD + n + 1];
                    K[i * LD + n] = static_cast<V>((4.0 * b0 - 2.0 * b1) / ht);
                    K[i * LD + n + 1] = static_cast<V>((-2.0 * b0 + 4.0 * b1) / ht);
                }
                team_sync<W>();
                // LU with partial pivoting on the augmented n x (n + 2) system
                bool singular = false;
                for (int col = 0; col < n; ++col)
                {
                    double best = -1.0;
                    int bi = n;
                    for (int i = col + lane; i < n; i += NT)
                    {
                        const double v = fabs(K[i * LD + col]);
                        if (v > best)
                        {
                            best = v;
                            bi = i;
                        }
                    }
                    team_argmax<W>(best, bi);
                    if (bi >= n || !(best > 0.0) || !isfinite(best))
                    {
                        singular = true;
                        break;
                    }
                    if (F32 && lane == 0)
                        piv[col] = bi;
                    if (bi != col)
                        for (int j = col + lane; j < n + 2; j += NT)
                        {
                            const V t0 = K[col * LD + j];
                            K[col * LD + j] = K[bi * LD + j];
                            K[bi * LD + j] = t0;
                        }
                    team_sync<W>();
                    const V inv = V(1) / K[col * LD + col];
                    for (int j = col + 1 + lane; j < n + 2; j += NT)
                    {
                        const V u = K[col * LD + j] * inv;
                        lu_column_update(K, LD, col, j, n, u);
                    }
                    team_sync<W>();
                }
                if (singular)
                {
                    if (lane == 0)
                        atomicExch(A.status, APF_ERR_NUMERIC);
                    team_sync<W>();
                    continue;
                }
                // back substitution, both right-hand sides, lanes over the rows above
                auto back_substitute = [&]() {
                    for (int i = n - 1; i >= 0; --i)
                    {
                        const V d = K[i * LD + i];
                        const V x0 = K[i * LD + n] / d, x1 = K[i * LD + n + 1] / d;
                        for (int r = lane; r < i; r += NT)
                        {
                            const V kri = K[r * LD + i];
                            K[r * LD + n] -= kri * x0;
                            K[r * LD + n + 1] -= kri * x1;
                        }
                        team_sync<W>();
                        if (lane == 0)
                        {
                            K[i * LD + n] = x0;
                            K[i * LD + n + 1] = x1;
                        }
                    }
                    team_sync<W>();
                };
                back_substitute();
                if (F32)
                {
                    // one FP64 refinement step
                    for (int i = lane; i < n; i += NT)
                    {
                        xd[i] = static_cast<double>(K[i * LD + n]);
                        xd[NMAX + i] = static_cast<double>(K[i * LD + n + 1]);
                        bd[i] = bd[NMAX + i] = kx[i] = kx[NMAX + i] = 0.0;
                    }
                    team_sync<W>();
                    // K x in a fixed order: the cell's matrix entries go to ev[t], then one lane
                    // per local row of the cell sums that row's entries in entry order (within a
                    // cell every (row, col) occurs once, and the cell's local rows are distinct
                    // patch rows); the right-hand-side entries are unique per cell as well
                    cell_entries(
                        [&](int t, int row, int col, double v) {
                            if (col >= n)
                                bd[(col - n) * NMAX + row] += v;
                            else
                                ev[t] = v;
                        },
                        [&](const int* pd, int sbase) {
                            const int q = lane;
                            double a0 = 0.0, a1 = 0.0;
                            int row = -1;
                            auto add = [&](double v, int col) {
                                a0 += v * xd[col];
                                a1 += v * xd[NMAX + col];
                            };
                            if (q < 8)
                            {
                                if (pd[q] >= 0)
                                {
                                    row = pd[q];
                                    for (int l = 0; l < 8; ++l)
                                        if (pd[l] >= 0)
                                            add(ev[8 * q + l], pd[l]);
                                    for (int r = 0; r < 3; ++r)
                                        add(ev[64 + 8 * r + q], sbase + r);
                                }
                            }
                            else if (q < 11)
                            {
                                const int r = q - 8;
                                row = sbase + r;
                                for (int l = 0; l < 8; ++l)
                                    if (pd[l] >= 0)
                                        add(ev[64 + 8 * r + l], pd[l]);
                                if (interior)
                                    add(ev[110 + r], n - 1);
                            }
                            else if (q == 11 && interior)
                            {
                                row = n - 1;
                                for (int r = 0; r < 3; ++r)
                                    add(ev[110 + r], sbase + r);
                            }
                            if (row >= 0)
                            {
                                kx[row] += a0;
                                kx[NMAX + row] += a1;
                            }
                            team_sync<W>();
                        });
                    for (int i = lane; i < n; i += NT)
                    {
                        const double b0 = bd[i], b1 = bd[NMAX + i];
                        K[i * LD + n] = static_cast<V>((4.0 * b0 - 2.0 * b1) / ht - kx[i]);
                        K[i * LD + n + 1] = static_cast<V>((-2.0 * b0 + 4.0 * b1) / ht - kx[NMAX + i]);
                    }
                    team_sync<W>();
                    // forward elimination of the residual with the recorded pivots and the
                    // multipliers K[i][col] / K[col][col] left below the diagonal
                    for (int col = 0; col < n; ++col)
                    {
                        const int pr = piv[col];
                        if (pr != col && lane < 2)
                        {
                            const V t0 = K[col * LD + n + lane];
                            K[col * LD + n + lane] = K[pr * LD + n + lane];
                            K[pr * LD + n + lane] = t0;
                        }
                        team_sync<W>();
                        const V inv = V(1) / K[col * LD + col];
                        const V r0 = K[col * LD + n] * inv, r1 = K[col * LD + n + 1] * inv;
                        for (int i = col + 1 + lane; i < n; i += NT)
                        {
                            const V l = K[i * LD + col];
                            K[i * LD + n] -= l * r0;
                            K[i * LD + n + 1] -= l * r1;
                        }
                        team_sync<W>();
                    }
                    back_substitute();
                    for (int i = lane; i < n; i += NT)
                    {
                        xd[i] += static_cast<double>(K[i * LD + n]);
                        xd[NMAX + i] += static_cast<double>(K[i * LD + n + 1]);
                    }
                    team_sync<W>();
                }
                auto solution = [&](int row, int kk) -> double {
                    return F32 ? xd[kk * NMAX + row] : static_cast<double>(K[row * LD + n + kk]);
                };
                // flux of this patch restricted to each of its cells -> slot of the patch vertex
                for (int t = lane; t < nc * 16; t += NT)
                {
                    const int ic = t >> 4, kk = (t >> 3) & 1, j = t & 7;
                    const int c = A.slab_cells[sb + A.topo_cell[cb + ic]];
                    const int a = A.topo_center[cb + ic];
                    double val = 0.0;
                    if (j < 6)
                    {
                        const int ed = j >> 1, m = j & 1;
                        const int code = A.topo_edge[3 * (cb + ic) + ed];
                        const int pe = code & 0xffff;
                        if (pe != 0xffff)
                        {
                            const double sp = (code >> 30) & 1 ? -1.0 : 1.0;
                            const double* g = A.geo + 8ll * c;
                            const double det = (g[2] - g[0]) * (g[5] - g[1]) - (g[4] - g[0]) * (g[3] - g[1]);
                            const double sn = (det < 0.0 ? -1.0 : 1.0) * sp;
                            const double cfj = m == 0 ? sn : sn * sp;
                            val = cfj * solution(2 * pe + m, kk);
                        }
                    }
                    else
                        val = solution(2 * nfree + 2 * ic + (j - 6), kk);
                    A.sigma[((3ll * c + a) * 2 + kk) * 8 + j] = val;
                }
                team_sync<W>();
            }
        }

        template<int NMAX, bool F32>
        constexpr std::size_t patch_smem_bytes()
        {
            return F32 ? sizeof(double) * (kPatchTableDoubles + (kPatchTableDoubles & 1) + 6 * NMAX + kCellEntries) +
                             sizeof(float) * NMAX * (NMAX + 3) + sizeof(int) * NMAX
                       : sizeof(double) * (kPatchTableDoubles + (kPatchTableDoubles & 1) + NMAX * (NMAX + 3));
        }

        struct IndicatorArgs
        {
            int n_cells;
            const double* geo;
            const double* m;
            const double* ell;
            const double* theta;
            const double* u;
            const double* lam_delta; // [cell][6]
            const double* lam_tilde; // [cell][6]
            const double* sigma;
            double* flux;
            double* div;
            double* recon;
            double* eta;
        };

        __global__ void cell_indicators(IndicatorArgs A)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.n_cells; c += gridDim.x * blockDim.x)
            {
                const Cell k = load_cell(A.geo, A.m, A.ell, c);
                double S[2][8];
                for (int kk = 0; kk < 2; ++kk)
                    for (int j = 0; j < 8; ++j)
                    {
                        double s = 0.0;
                        for (int slot = 0; slot < 3; ++slot)
                            s += A.sigma[((3ll * c + slot) * 2 + kk) * 8 + j];
                        S[kk][j] = s;
                    }
                const double* th = A.theta + 6ll * c;
                const double* uu = A.u + 6ll * c;
                double du[3];
                for (int s = 0; s < 3; ++s)
                    du[s] = (uu[2 * s + 1] - uu[2 * s]) / k.ht;
                const double adet = fabs(k.det);
                double flux = 0.0, div = 0.0;
                for (int gt = 0; gt < 2; ++gt)
                {
                    const double tau = c_est.tg[gt], wt = c_est.tw[gt] * k.ht;
                    const double tb[2] = {1.0 - tau, tau};
                    double gth0 = 0.0, gth1 = 0.0;
                    for (int s = 0; s < 3; ++s)
                    {
                        const double v = th[2 * s] * tb[0] + th[2 * s + 1] * tb[1];
                        gth0 += k.g[s][0] * v;
                        gth1 += k.g[s][1] * v;
                    }
                    const double mg0 = k.m00 * gth0 + k.m01 * gth1, mg1 = k.m01 * gth0 + k.m11 * gth1;
                    for (int q = 0; q < c_est.nq; ++q)
                    {
                        const double x = c_est.qp[q][0], y = c_est.qp[q][1];
                        double sx = 0.0, sy = 0.0, sd = 0.0;
                        for (int j = 0; j < 8; ++j)
                        {
                            double vx, vy, dv;
                            rt_phys(k, j, x, y, vx, vy, dv);
                            const double cj = S[0][j] * tb[0] + S[1][j] * tb[1];
                            sx += cj * vx;
                            sy += cj * vy;
                            sd += cj * dv;
                        }
                        const double ex = sx + mg0, ey = sy + mg1;
                        const double w = c_est.qw[q] * adet * wt;
                        flux += w * (ex * (k.mi00 * ex + k.mi01 * ey) + ey * (k.mi01 * ex + k.mi11 * ey));
                        const double l3[3] = {1.0 - x - y, x, y};
                        const double dtu = l3[0] * du[0] + l3[1] * du[1] + l3[2] * du[2];
                        const double r = k.ell - dtu - sd;
                        div += w * r * r;
                    }
                }
                // ||lambda_delta - lambda~||^2 in the local A_y energy: det ht Mt[a][b] Ks[s][r]
                double e[6];
                for (int i = 0; i < 6; ++i)
                    e[i] = A.lam_delta[6ll * c + i] - A.lam_tilde[6ll * c + i];
                double rec = 0.0;
                for (int i = 0; i < 6; ++i)
                    for (int j = 0; j < 6; ++j)
                    {
                        const int s = i / 2, a = i % 2, r = j / 2, b = j % 2;
                        const double mt = (a == b ? 1.0 / 3.0 : 1.0 / 6.0);
                        const double ks = k.g[s][0] * (k.m00 * k.g[r][0] + k.m01 * k.g[r][1]) +
                                          k.g[s][1] * (k.m01 * k.g[r][0] + k.m11 * k.g[r][1]);
                        rec += e[i] * (0.5 * adet * k.ht * mt * ks) * e[j];
                    }
                if (A.flux) A.flux[c] = flux;
                if (A.div) A.div[c] = div;
                if (A.recon) A.recon[c] = rec;
                if (A.eta) A.eta[c] = flux + rec;
            }
        }

        // nodal values of a true-DOF vector on every cell (restriction rows with weights)
        __global__ void gather_nodal(int n_cells, int ndof, const int* off, const int* dofs, const double* w,
                                     const double* vec, const double* vec2, double* out)
        {
            const long long total = (long long)n_cells * ndof;
            for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < total; r += (long long)gridDim.x * blockDim.x)
            {
                double s = 0.0;
                for (int e = off[r]; e < off[r + 1]; ++e)
                    s += w[e] * (vec[dofs[e]] + (vec2 ? vec2[dofs[e]] : 0.0));
                out[r] = s;
            }
        }

        __global__ void sum_partials_kernel(int n, const double* a, double* partials)
        {
            __shared__ double ws[8];
            double s = 0.0;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
                s += a[i];
            for (int o = 16; o > 0; o >>= 1)
                s += __shfl_down_sync(0xffffffffu, s, o);
            if ((threadIdx.x & 31) == 0)
                ws[threadIdx.x >> 5] = s;
            __syncthreads();
            if (threadIdx.x == 0)
            {
                double t = 0.0;
                for (int w = 0; w < 8; ++w)
                    t += ws[w];
                partials[blockIdx.x] = t;
            }
        }

        int nb(long long n, int threads = 256, int cap = 148 * 32)
        {
            return static_cast<int>(std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, cap)));
        }

        double device_sum(cudaStream_t s, int n, const double* a)
        {
            DeviceBuffer<double> parts(kRedBlocks, s);
            {
                APF_KERNEL("est_sum_partials", s);
                sum_partials_kernel<<<kRedBlocks, 256, 0, s>>>(n, a, parts.get());
            }
            std::vector<double> h(kRedBlocks);
            APF_CUDA(cudaMemcpyAsync(h.data(), parts.get(), kRedBlocks * sizeof(double), cudaMemcpyDeviceToHost, s));
            sync(s);
            double t = 0.0;
            for (double v : h)
                t += v;
            return t;
        }
    }

    // ---------------------------------------------------------------------------------------
    // p = 2: RT_2 x P_2 patches, broken P_2 x P_2 scalars, P_2 time basis (nodes 0, 1/2, 1)
    // ---------------------------------------------------------------------------------------
    namespace
    {
        // the 15 vector monomials spanning RT_2 on the reference triangle:
        // (P_2)^2 = {1, x, y, x^2, xy, y^2} e_1, same e_2, and x (x^2, xy, y^2)
        __host__ __device__ inline void mono15(double x, double y, double vx[15], double vy[15], double dv[15])
        {
            const double xx = x * x, xy = x * y, yy = y * y;
            const double ax[15] = {1, x, y, xx, xy, yy, 0, 0, 0, 0, 0, 0, xx * x, xx * y, xy * y};
            const double ay[15] = {0, 0, 0, 0, 0, 0, 1, x, y, xx, xy, yy, xx * y, xy * y, yy * y};
            const double ad[15] = {0, 1, 0, 2 * x, y, 0, 0, 0, 1, 0, x, 2 * y, 4 * xx, 4 * xy, 4 * yy};
            for (int m = 0; m < 15; ++m)
            {
                vx[m] = ax[m];
                vy[m] = ay[m];
                dv[m] = ad[m];
            }
        }

        // P_2 Lagrange basis on the reference triangle, node order v0, m01, v1, m02, m12, v2
        __host__ __device__ inline void p2_basis(double x, double y, double T[6], double Tx[6], double Ty[6])
        {
            const double l0 = 1.0 - x - y, l1 = x, l2 = y;
            T[0] = l0 * (2 * l0 - 1);  Tx[0] = -(4 * l0 - 1); Ty[0] = -(4 * l0 - 1);
            T[1] = 4 * l0 * l1;        Tx[1] = 4 * (l0 - l1); Ty[1] = -4 * l1;
            T[2] = l1 * (2 * l1 - 1);  Tx[2] = 4 * l1 - 1;    Ty[2] = 0;
            T[3] = 4 * l0 * l2;        Tx[3] = -4 * l2;       Ty[3] = 4 * (l0 - l2);
            T[4] = 4 * l1 * l2;        Tx[4] = 4 * l2;        Ty[4] = 4 * l1;
            T[5] = l2 * (2 * l2 - 1);  Tx[5] = 0;             Ty[5] = 4 * l2 - 1;
        }

        // P_2 time basis on [0, 1] with nodes 0, 1/2, 1 and its derivative
        __host__ __device__ inline void p2_time(double t, double S[3], double dS[3])
        {
            S[0] = (2 * t - 1) * (t - 1); dS[0] = 4 * t - 3;
            S[1] = 4 * t * (1 - t);       dS[1] = 4 - 8 * t;
            S[2] = t * (2 * t - 1);       dS[2] = 4 * t - 1;
        }

        // Reference-cell integrals for the p = 2 patch problems (16-point Duffy rule: exact up
        // to total degree 6, the highest here) and the time tables.
        struct Rt2Tables
        {
            double c[15][15];                     // phi_j = sum_m c[j][m] mono_m
            double r00[15][15], r01[15][15], r11[15][15]; // int phi_j^a phi_l^b
            double rd[15][6];                     // int div phi_l q_r
            double w[3][6][15];                   // int lambda_a grad T_s . phi_j
            double mq[3][6];                      // int lambda_a q_r
            double mqq[3][6][6];                  // int lambda_a T_s q_r
            double v[6][6][2];                    // int q_r d_c T_s
            double eq[6];                         // int q_r
            double mt[3][3], mtinv[3][3];         // int S_a S_b on [0, 1] and its inverse
            double dt[3][3];                      // int S_b' S_k  (index [b][k])
            double it[3];                         // int S_k
            double tg[3], tw[3];                  // 3-point Gauss on [0, 1]
        };
        constexpr int kRt2Doubles = sizeof(Rt2Tables) / sizeof(double);

        Rt2Tables make_rt2_tables(const EstTables& t)
        {
            Rt2Tables o{};
            const double g4x[4] = {0.06943184420297371, 0.33000947820757187, 0.6699905217924281, 0.9305681557970263};
            const double g4w[4] = {0.17392742256872692, 0.3260725774312731, 0.3260725774312731, 0.17392742256872692};
            // DOF functionals: 3 moments per edge (q = 1, 2s - 1, 6s^2 - 6s + 1 against the
            // outward normal times the edge length, edge k from v_{k+1} to v_{k+2}), then
            // int sigma . q for q = e_1, e_2, x e_1, x e_2, y e_1, y e_2
            std::vector<double> D(225, 0.0);
            const double vt[3][2] = {{0, 0}, {1, 0}, {0, 1}};
            for (int e = 0; e < 3; ++e)
            {
                const double* P = vt[(e + 1) % 3];
                const double* Q = vt[(e + 2) % 3];
                const double dx = Q[0] - P[0], dy = Q[1] - P[1];
                for (int g = 0; g < 4; ++g)
                {
                    const double sg = g4x[g];
                    double vx[15], vy[15], dv[15];
                    mono15(P[0] + sg * dx, P[1] + sg * dy, vx, vy, dv);
                    const double q[3] = {1.0, 2 * sg - 1, 6 * sg * sg - 6 * sg + 1};
                    for (int m = 0; m < 15; ++m)
                    {
                        const double fn = vx[m] * dy - vy[m] * dx;
                        for (int k = 0; k < 3; ++k)
                            D[(3 * e + k) * 15 + m] += g4w[g] * fn * q[k];
                    }
                }
            }
            for (int q = 0; q < t.nq; ++q)
            {
                const double x = t.qp[q][0], y = t.qp[q][1], w = t.qw[q];
                double vx[15], vy[15], dv[15];
                mono15(x, y, vx, vy, dv);
                for (int m = 0; m < 15; ++m)
                {
                    D[9 * 15 + m] += w * vx[m];
                    D[10 * 15 + m] += w * vy[m];
                    D[11 * 15 + m] += w * x * vx[m];
                    D[12 * 15 + m] += w * x * vy[m];
                    D[13 * 15 + m] += w * y * vx[m];
                    D[14 * 15 + m] += w * y * vy[m];
                }
            }
            std::vector<double> Dinv;
            solve_dense_host(D, 15, Dinv);
            for (int j = 0; j < 15; ++j)
                for (int m = 0; m < 15; ++m)
                    o.c[j][m] = Dinv[(size_t)m * 15 + j];
            for (int q = 0; q < t.nq; ++q)
            {
                const double x = t.qp[q][0], y = t.qp[q][1], w = t.qw[q];
                double vx[15], vy[15], dv[15];
                mono15(x, y, vx, vy, dv);
                double px[15], py[15], pd[15];
                for (int j = 0; j < 15; ++j)
                {
                    px[j] = py[j] = pd[j] = 0.0;
                    for (int m = 0; m < 15; ++m)
                    {
                        px[j] += o.c[j][m] * vx[m];
                        py[j] += o.c[j][m] * vy[m];
                        pd[j] += o.c[j][m] * dv[m];
                    }
                }
                double T[6], Tx[6], Ty[6];
                p2_basis(x, y, T, Tx, Ty);
                const double l3[3] = {1 - x - y, x, y};
                for (int j = 0; j < 15; ++j)
                    for (int l = 0; l < 15; ++l)
                    {
                        o.r00[j][l] += w * px[j] * px[l];
                        o.r01[j][l] += w * px[j] * py[l];
                        o.r11[j][l] += w * py[j] * py[l];
                    }
                for (int l = 0; l < 15; ++l)
                    for (int r = 0; r < 6; ++r)
                        o.rd[l][r] += w * pd[l] * T[r];
                for (int a = 0; a < 3; ++a)
                    for (int s2 = 0; s2 < 6; ++s2)
                    {
                        for (int j = 0; j < 15; ++j)
                            o.w[a][s2][j] += w * l3[a] * (Tx[s2] * px[j] + Ty[s2] * py[j]);
                        o.mq[a][s2] += w * l3[a] * T[s2];
                        for (int r = 0; r < 6; ++r)
                            o.mqq[a][s2][r] += w * l3[a] * T[s2] * T[r];
                    }
                for (int r = 0; r < 6; ++r)
                {
                    for (int s2 = 0; s2 < 6; ++s2)
                    {
                        o.v[r][s2][0] += w * T[r] * Tx[s2];
                        o.v[r][s2][1] += w * T[r] * Ty[s2];
                    }
                    o.eq[r] += w * T[r];
                }
            }
            // time: 3-point Gauss on [0, 1]
            const double h = 0.5 * std::sqrt(0.6);
            o.tg[0] = 0.5 - h; o.tg[1] = 0.5; o.tg[2] = 0.5 + h;
            o.tw[0] = 5.0 / 18.0; o.tw[1] = 8.0 / 18.0; o.tw[2] = 5.0 / 18.0;
            for (int g = 0; g < 3; ++g)
            {
                double S[3], dS[3];
                p2_time(o.tg[g], S, dS);
                for (int a = 0; a < 3; ++a)
                {
                    o.it[a] += o.tw[g] * S[a];
                    for (int b = 0; b < 3; ++b)
                    {
                        o.mt[a][b] += o.tw[g] * S[a] * S[b];
                        o.dt[a][b] += o.tw[g] * dS[a] * S[b];
                    }
                }
            }
            std::vector<double> M(9), Minv;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    M[a * 3 + b] = o.mt[a][b];
            solve_dense_host(M, 3, Minv);
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    o.mtinv[a][b] = Minv[a * 3 + b];
            return o;
        }

        // one warp per p = 2 patch (same structure as patch_solve): 3 edge moments per free
        // edge, 6 interior RT_2 moments and 6 scalars per patch cell, the mean-zero row, and
        // three right-hand-side columns (one per time DOF)
        template<int NMAX, int W>
        __global__ void __launch_bounds__(32 * W) patch_solve2(PatchArgs A, const Rt2Tables* __restrict__ tables,
                                                           const int* __restrict__ order, int count)
        {
            constexpr int LD = NMAX + 3; // odd: NMAX is even; columns n, n+1, n+2 hold the rhs
            extern __shared__ double sm[];
            Rt2Tables& T = *reinterpret_cast<Rt2Tables*>(sm);
            double* K = sm + kRt2Doubles + (kRt2Doubles & 1);
            const int lane = threadIdx.x;
            constexpr int NT = 32 * W; // threads of the patch team
            for (int i = lane; i < kRt2Doubles; i += NT)
                sm[i] = reinterpret_cast<const double*>(tables)[i];
            team_sync<W>();
            for (int idx = blockIdx.x; idx < count; idx += gridDim.x)
            {
                const int p = order[idx];
                const int slab = A.patch_slab[p], tp = A.patch_topo[p];
                const int cb = A.topo_ptr[tp], ce = A.topo_ptr[tp + 1], nc = ce - cb;
                const int nfree = A.topo_nfree[tp];
                const bool interior = A.topo_boundary[tp] == 0;
                const int nf = 3 * nfree + 6 * nc;
                const int n = nf + 6 * nc + (interior ? 1 : 0);
                if (n > NMAX)
                {
                    if (lane == 0)
                        atomicExch(A.status, APF_ERR_CAPACITY);
                    continue;
                }
                const int sb = A.slab_ptr[slab];
                for (int i = lane; i < n * LD; i += NT)
                    K[i] = 0.0;
                team_sync<W>();
                double ht = 0.0;
                for (int ic = 0; ic < nc; ++ic)
                {
                    const int c = A.slab_cells[sb + A.topo_cell[cb + ic]];
                    const int a = A.topo_center[cb + ic];
                    const Cell k = load_cell(A.geo, A.m, A.ell, c);
                    ht = k.ht;
                    const double adet = fabs(k.det);
                    int pd[15];
                    double e[15];
                    for (int ed = 0; ed < 3; ++ed)
                    {
                        const int code = A.topo_edge[3 * (cb + ic) + ed];
                        const int pe = code & 0xffff;
                        const double sp = (code >> 30) & 1 ? -1.0 : 1.0;
                        const bool free_edge = pe != 0xffff;
                        for (int m = 0; m < 3; ++m)
                        {
                            pd[3 * ed + m] = free_edge ? 3 * pe + m : -1;
                            // orientation sp^(m+1) times the Piola factor sign(det) / det
                            e[3 * ed + m] = (m == 1 ? 1.0 : sp) / k.det;
                        }
                    }
                    for (int m = 0; m < 6; ++m)
                    {
                        pd[9 + m] = 3 * nfree + 6 * ic + m;
                        e[9 + m] = 1.0 / k.det;
                    }
                    const int sbase = nf + 6 * ic;
                    const double q00 = k.mi00 * k.J00 + k.mi01 * k.J10, q10 = k.mi01 * k.J00 + k.mi11 * k.J10;
                    const double q01 = k.mi00 * k.J01 + k.mi01 * k.J11, q11 = k.mi01 * k.J01 + k.mi11 * k.J11;
                    const double S00 = k.J00 * q00 + k.J10 * q10;
                    const double S01 = k.J00 * q01 + k.J10 * q11;
                    const double S11 = k.J01 * q01 + k.J11 * q11;
                    // time-tested nodal data: th[s][kk] = ht sum_b Mt[kk][b] theta_{s,b},
                    // du[s][kk] = sum_b u_{s,b} int S_b' S_kk
                    const double* thc = A.theta + 18ll * c;
                    const double* uuc = A.u + 18ll * c;
                    double th[6][3], du[6][3];
                    for (int s2 = 0; s2 < 6; ++s2)
                        for (int kk = 0; kk < 3; ++kk)
                        {
                            double a1 = 0.0, a2 = 0.0;
                            for (int b = 0; b < 3; ++b)
                            {
                                a1 += T.mt[kk][b] * thc[3 * s2 + b];
                                a2 += uuc[3 * s2 + b] * T.dt[b][kk];
                            }
                            th[s2][kk] = k.ht * a1;
                            du[s2][kk] = a2;
                        }
                    // grad psi_a^T M G  (G = J^-T): row vector acting on reference gradients
                    const double mg0 = k.m00 * k.g[a][0] + k.m01 * k.g[a][1];
                    const double mg1 = k.m01 * k.g[a][0] + k.m11 * k.g[a][1];
                    // G = J^-T: (G v)_0 = (J11 v0 - J10 v1) / det, (G v)_1 = (-J01 v0 + J00 v1) / det
                    const double id = 1.0 / k.det;
                    const double h0 = (mg0 * k.J11 - mg1 * k.J01) * id; // (M grad psi)^T G e_0
                    const double h1 = (-mg0 * k.J10 + mg1 * k.J00) * id; // (M grad psi)^T G e_1
                    for (int t = lane; t < 384; t += NT)
                    {
                        if (t < 225)
                        {
                            const int j = t / 15, l = t % 15;
                            if (pd[j] < 0 || pd[l] < 0)
                                continue;
                            const double r = S00 * T.r00[j][l] + S01 * (T.r01[j][l] + T.r01[l][j]) + S11 * T.r11[j][l];
                            K[pd[j] * LD + pd[l]] += e[j] * e[l] * adet * r;
                        }
                        else if (t < 315)
                        {
                            const int r = (t - 225) / 15, l = (t - 225) % 15;
                            if (pd[l] < 0)
                                continue;
                            const double v = e[l] * adet * T.rd[l][r];
                            K[(sbase + r) * LD + pd[l]] += v;
                            K[pd[l] * LD + sbase + r] += v;
                        }
                        else if (t < 360)
                        {
                            const int j = (t - 315) / 3, kk = (t - 315) % 3;
                            if (pd[j] < 0)
                                continue;
                            double acc = 0.0;
                            for (int s2 = 0; s2 < 6; ++s2)
                                acc += th[s2][kk] * T.w[a][s2][j];
                            K[pd[j] * LD + n + kk] += -e[j] * adet * acc;
                        }
                        else if (t < 378)
                        {
                            const int r = (t - 360) / 3, kk = (t - 360) % 3;
                            double acc = k.ell * k.ht * T.it[kk] * T.mq[a][r];
                            double gx = 0.0, gy = 0.0;
                            for (int s2 = 0; s2 < 6; ++s2)
                            {
                                acc -= du[s2][kk] * T.mqq[a][s2][r];
                                gx += th[s2][kk] * T.v[r][s2][0];
                                gy += th[s2][kk] * T.v[r][s2][1];
                            }
                            K[(sbase + r) * LD + n + kk] += (acc - (h0 * gx + h1 * gy)) * adet;
                        }
                        else if (interior)
                        {
                            const int r = t - 378;
                            const double v = adet * T.eq[r];
                            K[(n - 1) * LD + sbase + r] += v;
                            K[(sbase + r) * LD + n - 1] += v;
                        }
                    }
                    team_sync<W>();
                }
                // right-hand sides times Mt^-1 = (1 / ht) mtinv
                for (int i = lane; i < n; i += NT)
                {
                    const double b0 = K[i * LD + n], b1 = K[i * LD + n + 1], b2 = K[i * LD + n + 2];
                    for (int kk = 0; kk < 3; ++kk)
                        K[i * LD + n + kk] = (T.mtinv[kk][0] * b0 + T.mtinv[kk][1] * b1 + T.mtinv[kk][2] * b2) / ht;
                }
                team_sync<W>();
                bool singular = false;
                for (int col = 0; col < n; ++col)
                {
                    double best = -1.0;
                    int bi = n;
                    for (int i = col + lane; i < n; i += NT)
                    {
                        const double v = fabs(K[i * LD + col]);
                        if (v > best)
                        {
                            best = v;
                            bi = i;
                        }
                    }
                    team_argmax<W>(best, bi);
                    if (bi >= n || !(best > 0.0) || !isfinite(best))
                    {
                        singular = true;
                        break;
                    }
                    if (bi != col)
                        for (int j = col + lane; j < n + 3; j += NT)
                        {
                            const double t0 = K[col * LD + j];
                            K[col * LD + j] = K[bi * LD + j];
                            K[bi * LD + j] = t0;
                        }
                    team_sync<W>();
                    const double inv = 1.0 / K[col * LD + col];
                    for (int j = col + 1 + lane; j < n + 3; j += NT)
                    {
                        const double u = K[col * LD + j] * inv;
                        lu_column_update(K, LD, col, j, n, u);
                    }
                    team_sync<W>();
                }
                if (singular)
                {
                    if (lane == 0)
                        atomicExch(A.status, APF_ERR_NUMERIC);
                    team_sync<W>();
                    continue;
                }
                for (int i = n - 1; i >= 0; --i)
                {
                    const double d = K[i * LD + i];
                    const double x0 = K[i * LD + n] / d, x1 = K[i * LD + n + 1] / d, x2 = K[i * LD + n + 2] / d;
                    for (int r = lane; r < i; r += NT)
                    {
                        const double kri = K[r * LD + i];
                        K[r * LD + n] -= kri * x0;
                        K[r * LD + n + 1] -= kri * x1;
                        K[r * LD + n + 2] -= kri * x2;
                    }
                    team_sync<W>();
                    if (lane == 0)
                    {
                        K[i * LD + n] = x0;
                        K[i * LD + n + 1] = x1;
                        K[i * LD + n + 2] = x2;
                    }
                }
                team_sync<W>();
                // flux of this patch on each of its cells -> slot of the patch vertex:
                // sigma slots [cell][3 vertices][3 time][15], coefficients of the cell's own
                // RT_2 basis with the orientation of its edges
                for (int t = lane; t < nc * 45; t += NT)
                {
                    const int ic = t / 45, kk = (t / 15) % 3, j = t % 15;
                    const int c = A.slab_cells[sb + A.topo_cell[cb + ic]];
                    const int a = A.topo_center[cb + ic];
                    double val = 0.0;
                    if (j < 9)
                    {
                        const int ed = j / 3, m = j % 3;
                        const int code = A.topo_edge[3 * (cb + ic) + ed];
                        const int pe = code & 0xffff;
                        if (pe != 0xffff)
                        {
                            const double sp = (code >> 30) & 1 ? -1.0 : 1.0;
                            const double* g = A.geo + 8ll * c;
                            const double det = (g[2] - g[0]) * (g[5] - g[1]) - (g[4] - g[0]) * (g[3] - g[1]);
                            const double cf = (det < 0.0 ? -1.0 : 1.0) * (m == 1 ? 1.0 : sp);
                            val = cf * K[(3 * pe + m) * LD + n + kk];
                        }
                    }
                    else
                        val = K[(3 * nfree + 6 * ic + (j - 9)) * LD + n + kk];
                    A.sigma[((3ll * c + a) * 3 + kk) * 15 + j] = val;
                }
                team_sync<W>();
            }
        }

        template<int NMAX>
        constexpr std::size_t patch2_smem_bytes()
        {
            return sizeof(double) * (kRt2Doubles + (kRt2Doubles & 1) + NMAX * (NMAX + 3));
        }

        // per slab cell (p = 2): flux^2 and div^2 with the 16-point Duffy rule x 3-point Gauss
        __global__ void cell_indicators2(IndicatorArgs A, const Rt2Tables* __restrict__ tables)
        {
            __shared__ double C[15][15];
            __shared__ double tg[3], tw[3];
            for (int i = threadIdx.x; i < 225; i += blockDim.x)
                C[i / 15][i % 15] = tables->c[i / 15][i % 15];
            if (threadIdx.x < 3)
            {
                tg[threadIdx.x] = tables->tg[threadIdx.x];
                tw[threadIdx.x] = tables->tw[threadIdx.x];
            }
            __syncthreads();
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.n_cells; c += gridDim.x * blockDim.x)
            {
                const Cell k = load_cell(A.geo, A.m, A.ell, c);
                const double sdet = k.det < 0.0 ? -1.0 : 1.0;
                const double adet = fabs(k.det);
                const double* th = A.theta + 18ll * c;
                const double* uu = A.u + 18ll * c;
                double Ssum[3][15];
                for (int kk = 0; kk < 3; ++kk)
                    for (int j = 0; j < 15; ++j)
                    {
                        double sj = 0.0;
                        for (int slot = 0; slot < 3; ++slot)
                            sj += A.sigma[((3ll * c + slot) * 3 + kk) * 15 + j];
                        Ssum[kk][j] = sj;
                    }
                double flux = 0.0, div = 0.0;
                for (int q = 0; q < c_est.nq; ++q)
                {
                    const double x = c_est.qp[q][0], y = c_est.qp[q][1];
                    double mvx[15], mvy[15], mdv[15];
                    mono15(x, y, mvx, mvy, mdv);
                    double T[6], Tx[6], Ty[6];
                    p2_basis(x, y, T, Tx, Ty);
                    // reference-basis values at this point (before the Piola map)
                    double bx[15], by[15], bd[15];
                    for (int j = 0; j < 15; ++j)
                    {
                        double vx = 0.0, vy = 0.0, dv = 0.0;
                        for (int m = 0; m < 15; ++m)
                        {
                            vx += C[j][m] * mvx[m];
                            vy += C[j][m] * mvy[m];
                            dv += C[j][m] * mdv[m];
                        }
                        const double f = (j < 9 ? sdet : 1.0) / k.det;
                        bx[j] = f * (k.J00 * vx + k.J01 * vy);
                        by[j] = f * (k.J10 * vx + k.J11 * vy);
                        bd[j] = f * dv;
                    }
                    for (int g = 0; g < 3; ++g)
                    {
                        double S[3], dS[3];
                        p2_time(tg[g], S, dS);
                        double sx = 0.0, sy = 0.0, sd = 0.0;
                        for (int kk = 0; kk < 3; ++kk)
                        {
                            double cx = 0.0, cy = 0.0, cd = 0.0;
                            for (int j = 0; j < 15; ++j)
                            {
                                cx += Ssum[kk][j] * bx[j];
                                cy += Ssum[kk][j] * by[j];
                                cd += Ssum[kk][j] * bd[j];
                            }
                            sx += S[kk] * cx;
                            sy += S[kk] * cy;
                            sd += S[kk] * cd;
                        }
                        // grad theta~ and d_t u at (x, t)
                        double gr0 = 0.0, gr1 = 0.0, dtu = 0.0;
                        for (int s2 = 0; s2 < 6; ++s2)
                        {
                            double v = 0.0, w = 0.0;
                            for (int b = 0; b < 3; ++b)
                            {
                                v += th[3 * s2 + b] * S[b];
                                w += uu[3 * s2 + b] * dS[b];
                            }
                            gr0 += v * Tx[s2];
                            gr1 += v * Ty[s2];
                            dtu += w * T[s2];
                        }
                        dtu /= k.ht;
                        // physical gradient G g_ref, G = J^-T
                        const double id = 1.0 / k.det;
                        const double p0 = (k.J11 * gr0 - k.J10 * gr1) * id;
                        const double p1 = (-k.J01 * gr0 + k.J00 * gr1) * id;
                        const double mg0 = k.m00 * p0 + k.m01 * p1, mg1 = k.m01 * p0 + k.m11 * p1;
                        const double ex = sx + mg0, ey = sy + mg1;
                        const double w = c_est.qw[q] * adet * tw[g] * k.ht;
                        flux += w * (ex * (k.mi00 * ex + k.mi01 * ey) + ey * (k.mi01 * ex + k.mi11 * ey));
                        const double r = k.ell - dtu - sd;
                        div += w * r * r;
                    }
                }
                if (A.flux) A.flux[c] = flux;
                if (A.div) A.div[c] = div;
            }
        }

        __global__ void cell_times_kernel(int n, const double* __restrict__ geo, double* __restrict__ times)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
            {
                times[2ll * c] = geo[8ll * c + 6];
                times[2ll * c + 1] = geo[8ll * c + 7];
            }
        }

        __global__ void add_kernel(int n, const double* __restrict__ a, const double* __restrict__ b,
                                   double* __restrict__ y)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                y[i] = a[i] + b[i];
        }
    }

    // ---------------------------------------------------------------------------
    // host-side patch topology (integer work; built once per distinct slab mesh)
    // ---------------------------------------------------------------------------
    void build_patches(const std::vector<double>& times, const std::vector<int>& vids, int n_cells, PatchSet& ps)
    {
        // slabs by the exact time interval of their cells (mesh times are dyadic; stacked
        // independent problems may share a start time with different steps): the distinct
        // intervals in time order, then a stable counting sort of the cells into them
        struct PairHash
        {
            std::size_t operator()(const std::pair<double, double>& p) const noexcept
            {
                std::uint64_t a, b;
                std::memcpy(&a, &p.first, 8);
                std::memcpy(&b, &p.second, 8);
                return static_cast<std::size_t>((a * 0x9E3779B97F4A7C15ull) ^ (b + 0x632BE59BD9B4E019ull + (a << 6)));
            }
        };
        std::vector<int> cell_slab(n_cells);
        {
            // open-addressing table of the distinct intervals (at most half full, grown by doubling)
            std::vector<std::pair<double, double>> intervals;
            std::vector<int> table(64, -1);
            const PairHash hasher;
            auto find_or_add = [&](const std::pair<double, double>& key) {
                std::size_t mask = table.size() - 1, h = hasher(key) & mask;
                while (table[h] >= 0 && intervals[table[h]] != key)
                    h = (h + 1) & mask;
                if (table[h] >= 0)
                    return table[h];
                const int id = static_cast<int>(intervals.size());
                intervals.push_back(key);
                table[h] = id;
                if (2 * intervals.size() > table.size())
                {
                    std::vector<int> bigger(table.size() * 2, -1);
                    const std::size_t m2 = bigger.size() - 1;
                    for (std::size_t q = 0; q < intervals.size(); ++q)
                    {
                        std::size_t g = hasher(intervals[q]) & m2;
                        while (bigger[g] >= 0)
                            g = (g + 1) & m2;
                        bigger[g] = static_cast<int>(q);
                    }
                    table.swap(bigger);
                }
                return id;
            };
            int last = -1;
            std::pair<double, double> last_key{0.0, 0.0};
            for (int c = 0; c < n_cells; ++c)
            {
                const std::pair<double, double> key{times[2ll * c], times[2ll * c + 1]};
                if (last < 0 || key != last_key)
                {
                    last = find_or_add(key);
                    last_key = key;
                }
                cell_slab[c] = last;
            }
            // renumber the intervals in time order
            std::vector<int> by_time(intervals.size());
            std::iota(by_time.begin(), by_time.end(), 0);
            std::sort(by_time.begin(), by_time.end(), [&](int a, int b) { return intervals[a] < intervals[b]; });
            std::vector<int> rank(intervals.size());
            for (std::size_t k = 0; k < by_time.size(); ++k)
                rank[by_time[k]] = static_cast<int>(k);
            for (int c = 0; c < n_cells; ++c)
                cell_slab[c] = rank[cell_slab[c]];
            ps.slab_ptr.assign(intervals.size() + 1, 0);
        }
        for (int c = 0; c < n_cells; ++c)
            ++ps.slab_ptr[cell_slab[c] + 1];
        for (std::size_t k = 1; k < ps.slab_ptr.size(); ++k)
            ps.slab_ptr[k] += ps.slab_ptr[k - 1];
        ps.slab_cells.assign(n_cells, 0);
        {
            std::vector<int> cursor(ps.slab_ptr.begin(), ps.slab_ptr.end() - 1);
            for (int c = 0; c < n_cells; ++c)
                ps.slab_cells[cursor[cell_slab[c]]++] = c;
        }
        const int n_slabs = static_cast<int>(ps.slab_ptr.size()) - 1;
        // group slabs with identical spatial meshes (same vertex-id sequence)
        std::vector<int> group_of(n_slabs, -1);
        std::vector<int> group_rep;
        // slab fingerprints on a few host threads, then groups by fingerprint with an exact
        // comparison against each group's first slab (also threaded)
        const int nthreads = std::max(1, std::min<int>(8, static_cast<int>(std::thread::hardware_concurrency())));
        auto parallel_slabs = [&](auto&& body) {
            std::vector<std::thread> pool;
            for (int t = 0; t < nthreads; ++t)
                pool.emplace_back([&, t]() {
                    for (int sl = t; sl < n_slabs; sl += nthreads)
                        body(sl);
                });
            for (auto& th : pool)
                th.join();
        };
        std::vector<std::uint64_t> fp(n_slabs);
        parallel_slabs([&](int sl) {
            std::uint64_t h = 1469598103934665603ull;
            for (int i = ps.slab_ptr[sl]; i < ps.slab_ptr[sl + 1]; ++i)
                for (int k = 0; k < 3; ++k)
                    h = (h ^ static_cast<std::uint64_t>(vids[3ll * ps.slab_cells[i] + k])) * 1099511628211ull;
            fp[sl] = h;
        });
        auto same_mesh = [&](int a, int r) {
            const int len = ps.slab_ptr[a + 1] - ps.slab_ptr[a];
            if (len != ps.slab_ptr[r + 1] - ps.slab_ptr[r])
                return false;
            for (int i = 0; i < len; ++i)
                for (int k = 0; k < 3; ++k)
                    if (vids[3ll * ps.slab_cells[ps.slab_ptr[a] + i] + k] != vids[3ll * ps.slab_cells[ps.slab_ptr[r] + i] + k])
                        return false;
            return true;
        };
        std::unordered_map<std::uint64_t, int> first_of;
        std::vector<int> tentative(n_slabs);
        for (int sl = 0; sl < n_slabs; ++sl)
            tentative[sl] = first_of.emplace(fp[sl], sl).first->second;
        std::vector<char> confirmed(n_slabs, 1);
        parallel_slabs([&](int sl) {
            if (tentative[sl] != sl)
                confirmed[sl] = same_mesh(sl, tentative[sl]) ? 1 : 0;
        });
        std::vector<int> group_of_rep(n_slabs, -1);
        for (int sl = 0; sl < n_slabs; ++sl)
        {
            int r = tentative[sl];
            if (r != sl && !confirmed[sl])
            {
                // equal fingerprints of different meshes: compare with every group so far
                r = sl;
                for (std::size_t g = 0; g < group_rep.size(); ++g)
                    if (same_mesh(sl, group_rep[g]))
                    {
                        r = group_rep[g];
                        break;
                    }
            }
            if (r == sl)
            {
                group_of_rep[sl] = static_cast<int>(group_rep.size());
                group_rep.push_back(sl);
            }
            group_of[sl] = group_of_rep[r];
        }
        // topology patches of every group
        ps.topo_ptr.assign(1, 0);
        ps.topo_cell.clear();
        ps.topo_center.clear();
        ps.topo_edge.clear();
        ps.topo_nfree.clear();
        ps.topo_boundary.clear();
        std::vector<int> group_first(group_rep.size()), group_count(group_rep.size());
        ps.max_cells = 0;
        ps.max_n = 0;
        for (std::size_t g = 0; g < group_rep.size(); ++g)
        {
            const int s = group_rep[g];
            const int b = ps.slab_ptr[s], len = ps.slab_ptr[s + 1] - b;
            auto vid = [&](int local, int k) { return vids[3ll * ps.slab_cells[b + local] + k]; };
            // edge multiplicity in the slab mesh: all edge keys sorted, counts by run length
            auto ekey = [](int p, int q) {
                const std::uint32_t lo = static_cast<std::uint32_t>(std::min(p, q)), hi = static_cast<std::uint32_t>(std::max(p, q));
                return (static_cast<std::uint64_t>(lo) << 32) | hi;
            };
            std::vector<std::uint64_t> ekeys(3ll * len);
            std::vector<int> eorder(3ll * len), ecount(3ll * len);
            for (int i = 0; i < len; ++i)
                for (int k = 0; k < 3; ++k)
                    ekeys[3ll * i + k] = ekey(vid(i, (k + 1) % 3), vid(i, (k + 2) % 3));
            std::iota(eorder.begin(), eorder.end(), 0);
            std::sort(eorder.begin(), eorder.end(), [&](int a, int b) { return ekeys[a] < ekeys[b]; });
            for (std::size_t e = 0; e < eorder.size();)
            {
                std::size_t f = e + 1;
                while (f < eorder.size() && ekeys[eorder[f]] == ekeys[eorder[e]])
                    ++f;
                for (std::size_t q = e; q < f; ++q)
                    ecount[eorder[q]] = static_cast<int>(f - e);
                e = f;
            }
            // vertex -> incident (local cell, local vertex), vertices in first-appearance order
            int vmax = -1;
            for (int i = 0; i < len; ++i)
                for (int k = 0; k < 3; ++k)
                    vmax = std::max(vmax, vid(i, k));
            std::vector<int> vindex(static_cast<std::size_t>(vmax) + 1, -1);
            std::vector<int> vfirst; // first incidence of each vertex, then counting sort
            std::vector<int> vcount;
            for (int i = 0; i < len; ++i)
                for (int k = 0; k < 3; ++k)
                {
                    int& vi = vindex[vid(i, k)];
                    if (vi < 0)
                    {
                        vi = static_cast<int>(vcount.size());
                        vcount.push_back(0);
                    }
                    ++vcount[vi];
                }
            const int nv = static_cast<int>(vcount.size());
            std::vector<int> vptr(nv + 1, 0);
            for (int v = 0; v < nv; ++v)
                vptr[v + 1] = vptr[v] + vcount[v];
            std::vector<std::pair<int, int>> incs(vptr[nv]);
            {
                std::vector<int> cur(vptr.begin(), vptr.end() - 1);
                for (int i = 0; i < len; ++i)
                    for (int k = 0; k < 3; ++k)
                        incs[cur[vindex[vid(i, k)]]++] = {i, k};
            }
            std::vector<char> vbound(nv, 0);
            for (std::size_t e = 0; e < ekeys.size(); ++e)
                if (ecount[e] == 1)
                {
                    vbound[vindex[static_cast<int>(ekeys[e] >> 32)]] = 1;
                    vbound[vindex[static_cast<int>(ekeys[e] & 0xffffffffu)]] = 1;
                }
            struct IncRange
            {
                const std::pair<int, int>* b;
                const std::pair<int, int>* e;
                const std::pair<int, int>* begin() const { return b; }
                const std::pair<int, int>* end() const { return e; }
                std::size_t size() const { return static_cast<std::size_t>(e - b); }
            };
            std::vector<IncRange> inc(nv);
            for (int v = 0; v < nv; ++v)
                inc[v] = IncRange{incs.data() + vptr[v], incs.data() + vptr[v + 1]};
            group_first[g] = static_cast<int>(ps.topo_nfree.size());
            group_count[g] = static_cast<int>(inc.size());
            for (std::size_t v = 0; v < inc.size(); ++v)
            {
                const bool boundary = vbound[v] != 0;
                std::vector<std::uint64_t> free_id; // free edges of the patch, in first-seen order
                free_id.reserve(16);
                int nfree = 0;
                for (const auto& [i, a] : inc[v])
                {
                    ps.topo_cell.push_back(i);
                    ps.topo_center.push_back(a);
                    const int va = vid(i, a);
                    for (int k = 0; k < 3; ++k)
                    {
                        const int P = vid(i, (k + 1) % 3), Q = vid(i, (k + 2) % 3);
                        const std::uint64_t ek = ekeys[3ll * i + k];
                        const int cnt = ecount[3ll * i + k];
                        const bool touches = P == va || Q == va;
                        const bool is_free = (touches && cnt == 2) || (boundary && cnt == 1);
                        int code = 0xffff;
                        if (is_free)
                        {
                            int id = 0;
                            while (id < nfree && free_id[id] != ek)
                                ++id;
                            if (id == nfree)
                            {
                                free_id.push_back(ek);
                                ++nfree;
                            }
                            code = id;
                        }
                        if (P > Q)
                            code |= 1 << 30; // local parameterisation runs from the higher to the lower id
                        ps.topo_edge.push_back(code);
                    }
                }
                ps.max_cells = std::max<int>(ps.max_cells, static_cast<int>(inc[v].size()));
                ps.max_n = std::max<int>(ps.max_n, 2 * nfree + 5 * static_cast<int>(inc[v].size()) + (boundary ? 0 : 1));
                ps.topo_ptr.push_back(static_cast<int>(ps.topo_cell.size()));
                ps.topo_nfree.push_back(nfree);
                ps.topo_boundary.push_back(boundary ? 1 : 0);
            }
        }
        ps.patch_slab.clear();
        ps.patch_topo.clear();
        {
            std::size_t total = 0;
            for (int s = 0; s < n_slabs; ++s)
                total += static_cast<std::size_t>(group_count[group_of[s]]);
            ps.patch_slab.reserve(total);
            ps.patch_topo.reserve(total);
        }
        for (int s = 0; s < n_slabs; ++s)
        {
            const int g = group_of[s];
            for (int v = 0; v < group_count[g]; ++v)
            {
                ps.patch_slab.push_back(s);
                ps.patch_topo.push_back(group_first[g] + v);
            }
        }
        ps.n_slabs = n_slabs;
    }

    void upload_est_tables_once()
    {
        static bool done = false;
        if (done)
            return;
        const EstTables t = make_est_tables();
        APF_CUDA(cudaMemcpyToSymbol(c_est, &t, sizeof(t)));
        done = true;
    }

    // ---------------------------------------------------------------------------
    // time-slab space of an adaptive Y (time_slab_builder.hpp:53-215): the slab times are
    // the distinct time endpoints of the active Y cells; every Y cell is cut into one slab
    // cell per slab it spans (slabs in time order, each slab's cells in Y order); the slab
    // space is P_p x P_p on each slab, continuous in space inside the slab (the reference's
    // refinement keeps each slab's spatial mesh conforming), broken between slabs, zero on
    // the Dirichlet boundary (the spatial nodes whose Y restriction rows are empty).
    // ---------------------------------------------------------------------------
    namespace
    {
        // per (Y cell, spatial node): 1 when the restriction rows of all its time nodes are empty
        __global__ void dirichlet_nodes_kernel(int n, int ns, int nt, const int* __restrict__ off,
                                               unsigned char* __restrict__ out)
        {
            for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < (long long)n * ns;
                 r += (long long)gridDim.x * blockDim.x)
            {
                bool empty = true;
                for (int a = 0; a < nt; ++a)
                    empty = empty && off[r * nt + a] == off[r * nt + a + 1];
                out[r] = empty ? 1 : 0;
            }
        }

        // flag = 1 when some restriction row has more than one entry or a weight other than 1
        __global__ void nontrivial_restriction_kernel(long long rows, const int* __restrict__ off,
                                                      const double* __restrict__ w, int* __restrict__ flag)
        {
            for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows;
                 r += (long long)gridDim.x * blockDim.x)
            {
                const int b = off[r], e = off[r + 1];
                if (e - b > 1 || (e - b == 1 && w[b] != 1.0))
                    *flag = 1;
            }
        }

        // per slab cell: the source Y cell's geometry row (gw values, the last two t0 t1) with
        // the slab's time interval, its M (mw values), load and X ancestor
        __global__ void slab_cells_kernel(int n, int gw, int mw, const int* __restrict__ source,
                                          const int* __restrict__ slab, const double* __restrict__ slab_times,
                                          const double* __restrict__ y_geo, const double* __restrict__ m_y,
                                          const double* __restrict__ ell_y, const int* __restrict__ y_to_x,
                                          double* __restrict__ geo, double* __restrict__ m, double* __restrict__ ell,
                                          int* __restrict__ to_x)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
            {
                const int y = source[c], k = slab[c];
                for (int j = 0; j < gw - 2; ++j)
                    geo[(long long)gw * c + j] = y_geo[(long long)gw * y + j];
                geo[(long long)gw * c + gw - 2] = slab_times[k];
                geo[(long long)gw * c + gw - 1] = slab_times[k + 1];
                if (m)
                    for (int j = 0; j < mw; ++j)
                        m[(long long)mw * c + j] = m_y[(long long)mw * y + j];
                if (ell)
                    ell[c] = ell_y[y];
                to_x[c] = y_to_x[y];
            }
        }

        // 1+1D: dst[c] (bilinear nodal values, index x_node * 2 + t_node) = the source quad's
        // bilinear function at the corners of quad c (inside it)
        __global__ void nodal_transfer_1d_kernel(int n, const double* __restrict__ dst_geo,
                                                 const int* __restrict__ src_index, const double* __restrict__ src_geo,
                                                 const double* __restrict__ src, double* __restrict__ dst)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
            {
                const int sc = src_index ? src_index[c] : c;
                const double* gd = dst_geo + 4ll * c;
                const double* gs = src_geo + 4ll * sc;
                const double* in = src + 4ll * sc;
                for (int k = 0; k < 4; ++k)
                {
                    const double x = gd[k >> 1], t = gd[2 + (k & 1)];
                    const double xi = (x - gs[0]) / (gs[1] - gs[0]), tau = (t - gs[2]) / (gs[3] - gs[2]);
                    const double bx[2] = {1.0 - xi, xi}, bt[2] = {1.0 - tau, tau};
                    double v = 0.0;
                    for (int i = 0; i < 2; ++i)
                        for (int b = 0; b < 2; ++b)
                            v += in[i * 2 + b] * bx[i] * bt[b];
                    dst[4ll * c + k] = v;
                }
            }
        }

        // 1+1D: out[c] = int_c m (d_x v)^2 of bilinear nodal values v on quad c
        __global__ void nodal_energy_1d_kernel(int n, const double* __restrict__ geo, const double* __restrict__ m,
                                               const double* __restrict__ v, double* __restrict__ out)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
            {
                const double* g = geo + 4ll * c;
                const double h = g[1] - g[0], ht = g[3] - g[2];
                const double d0 = v[4ll * c + 2] - v[4ll * c + 0], d1 = v[4ll * c + 3] - v[4ll * c + 1];
                const double mc = m ? m[c] : 1.0;
                out[c] = mc * (ht / h) * (d0 * d0 + d0 * d1 + d1 * d1) / 3.0;
            }
        }

        // out[y] = sum of a over the slab cells of Y cell y (in slab order)
        __global__ void reduce_to_source_kernel(int n, const int* __restrict__ ptr, const int* __restrict__ list,
                                                const double* __restrict__ a, double* __restrict__ out)
        {
            for (int y = blockIdx.x * blockDim.x + threadIdx.x; y < n; y += gridDim.x * blockDim.x)
            {
                double s = 0.0;
                for (int i = ptr[y]; i < ptr[y + 1]; ++i)
                    s += a[list[i]];
                out[y] = s;
            }
        }
    }

    struct SlabSpace
    {
        bool identity = true;        // slab space == Y (every Y cell in one slab, no hanging rows)
        int n_cells = 0;             // slab cells
        int n_slabs = 0;
        int n_dofs = 0;
        std::vector<double> slab_times;
        std::vector<int> source, slab; // per slab cell
        std::vector<double> times;     // per slab cell: t0 t1
        std::vector<int> vids;         // per slab cell: 3 spatial vertex ids
        std::vector<int> dof;          // per slab cell and local node: slab DOF or -1
        std::vector<int> src_ptr, src_list; // Y cell -> its slab cells
    };

    // host integer work: slabs, slab cells, slab DOFs.  keys: one 64-bit identity per (Y cell,
    // spatial node) shared by the nodes that coincide (ns per cell); bnode: Dirichlet flag per
    // (Y cell, spatial node); yvids (2+1D, may be empty): spatial vertex ids of the Y cells
    void build_slab_space(int ns, int nt, int ny, const std::vector<double>& ytimes, const std::vector<int>& yvids,
                          const std::vector<std::uint64_t>& keys, const std::vector<unsigned char>& bnode, SlabSpace& sp)
    {
        const int nd = ns * nt;
        std::vector<double>& T = sp.slab_times;
        T.assign(ytimes.begin(), ytimes.end());
        std::sort(T.begin(), T.end());
        T.erase(std::unique(T.begin(), T.end()), T.end());
        sp.n_slabs = std::max<int>(0, static_cast<int>(T.size()) - 1);
        auto index_of = [&](double t) {
            const auto it = std::lower_bound(T.begin(), T.end(), t);
            return static_cast<int>(it - T.begin());
        };
        std::vector<int> kb(ny), ke(ny), count(sp.n_slabs + 1, 0);
        for (int c = 0; c < ny; ++c)
        {
            kb[c] = index_of(ytimes[2ll * c]);
            ke[c] = index_of(ytimes[2ll * c + 1]);
            require(kb[c] < ke[c], APF_ERR_INVALID, "estimator: Y cell with an empty time interval");
            for (int k = kb[c]; k < ke[c]; ++k)
                ++count[k + 1];
        }
        for (int k = 0; k < sp.n_slabs; ++k)
            count[k + 1] += count[k];
        const int nsc = count[sp.n_slabs];
        sp.n_cells = nsc;
        sp.source.assign(nsc, 0);
        sp.slab.assign(nsc, 0);
        {
            std::vector<int> cur(count.begin(), count.end() - 1);
            for (int c = 0; c < ny; ++c)
                for (int k = kb[c]; k < ke[c]; ++k)
                {
                    const int i = cur[k]++;
                    sp.source[i] = c;
                    sp.slab[i] = k;
                }
        }
        sp.times.resize(2ll * nsc);
        for (int i = 0; i < nsc; ++i)
        {
            sp.times[2ll * i] = T[sp.slab[i]];
            sp.times[2ll * i + 1] = T[sp.slab[i] + 1];
        }
        if (!yvids.empty())
        {
            sp.vids.resize(3ll * nsc);
            for (int i = 0; i < nsc; ++i)
                for (int v = 0; v < 3; ++v)
                    sp.vids[3ll * i + v] = yvids[3ll * sp.source[i] + v];
        }
        auto node_key = [&](int i, int s) { return keys[static_cast<std::size_t>(sp.source[i]) * ns + s]; };
        // per slab (host threads): spatial node numbering in first-appearance order
        std::vector<int> local(static_cast<std::size_t>(nsc) * ns, -1), n_spatial(sp.n_slabs, 0);
        const int nthreads = std::max(1, std::min<int>(8, static_cast<int>(std::thread::hardware_concurrency())));
        {
            std::vector<std::thread> pool;
            for (int t = 0; t < nthreads; ++t)
                pool.emplace_back([&, t]() {
                    std::unordered_map<std::uint64_t, int> ids;
                    for (int k = t; k < sp.n_slabs; k += nthreads)
                    {
                        ids.clear();
                        for (int i = count[k]; i < count[k + 1]; ++i)
                            for (int s = 0; s < ns; ++s)
                            {
                                if (bnode[static_cast<std::size_t>(sp.source[i]) * ns + s])
                                    continue;
                                const auto it = ids.emplace(node_key(i, s), static_cast<int>(ids.size())).first;
                                local[static_cast<std::size_t>(i) * ns + s] = it->second;
                            }
                        n_spatial[k] = static_cast<int>(ids.size());
                    }
                });
            for (auto& th : pool)
                th.join();
        }
        std::vector<long long> base(sp.n_slabs + 1, 0);
        for (int k = 0; k < sp.n_slabs; ++k)
            base[k + 1] = base[k] + static_cast<long long>(n_spatial[k]) * nt;
        require(base[sp.n_slabs] < (1ll << 31), APF_ERR_CAPACITY, "estimator: slab space too large");
        sp.n_dofs = static_cast<int>(base[sp.n_slabs]);
        sp.dof.assign(static_cast<std::size_t>(nsc) * nd, -1);
        for (int i = 0; i < nsc; ++i)
            for (int s = 0; s < ns; ++s)
            {
                const int l = local[static_cast<std::size_t>(i) * ns + s];
                if (l < 0)
                    continue;
                for (int a = 0; a < nt; ++a)
                    sp.dof[static_cast<std::size_t>(i) * nd + s * nt + a] =
                        static_cast<int>(base[sp.slab[i]] + static_cast<long long>(l) * nt + a);
            }
        // Y cell -> slab cells
        sp.src_ptr.assign(ny + 1, 0);
        for (int i = 0; i < nsc; ++i)
            ++sp.src_ptr[sp.source[i] + 1];
        for (int c = 0; c < ny; ++c)
            sp.src_ptr[c + 1] += sp.src_ptr[c];
        sp.src_list.assign(nsc, 0);
        {
            std::vector<int> cur(sp.src_ptr.begin(), sp.src_ptr.end() - 1);
            for (int i = 0; i < nsc; ++i)
                sp.src_list[cur[sp.source[i]]++] = i;
        }
    }

    // the slab space's inputs as a main-system SystemInputs (Y := slab space, X borrowed
    // from the main system while the slab blocks are assembled)
    struct SlabSystem
    {
        SystemInputs in;
        DeviceBuffer<int> src_ptr, src_list;
    };

    void upload_slab_system(cudaStream_t s, const SystemInputs& yin, const SlabSpace& sp, SlabSystem& out)
    {
        SystemInputs& in = out.in;
        in.p = yin.p;
        in.ndof = yin.ndof;
        in.dim = yin.dim;
        in.n_y_cells = sp.n_cells;
        in.n_x_cells = yin.n_x_cells;
        in.n_lambda = sp.n_dofs;
        in.n_u = yin.n_u;
        in.u0_kind = yin.u0_kind;
        in.zero_tol = yin.zero_tol;
        in.g_scale = yin.g_scale;
        const int n = sp.n_cells, nd = yin.ndof;
        const int gw = yin.dim == 1 ? 4 : 8, mw = yin.dim == 1 ? 1 : 3;
        DeviceBuffer<int> d_source(0, s), d_slab(0, s);
        DeviceBuffer<double> d_times(0, s);
        d_source.upload(sp.source.data(), sp.source.size());
        d_slab.upload(sp.slab.data(), sp.slab.size());
        d_times.upload(sp.slab_times.data(), sp.slab_times.size());
        in.y_geo.allocate(static_cast<std::size_t>(gw) * n, s);
        in.y_to_x.allocate(n, s);
        if (yin.m_y.size())
            in.m_y.allocate(static_cast<std::size_t>(mw) * n, s);
        if (yin.ell.size())
            in.ell.allocate(n, s);
        if (n > 0)
        {
            APF_KERNEL("est_slab_cells", s);
            slab_cells_kernel<<<nb(n), 256, 0, s>>>(n, gw, mw, d_source.get(), d_slab.get(), d_times.get(),
                                                     yin.y_geo.get(), yin.m_y.size() ? yin.m_y.get() : nullptr,
                                                     yin.ell.size() ? yin.ell.get() : nullptr, yin.y_to_x.get(),
                                                     in.y_geo.get(), in.m_y.size() ? in.m_y.get() : nullptr,
                                                     in.ell.size() ? in.ell.get() : nullptr, in.y_to_x.get());
        }
        // restriction: one entry of weight 1 per non-Dirichlet node
        std::vector<int> off(static_cast<std::size_t>(n) * nd + 1, 0), dofs;
        dofs.reserve(sp.dof.size());
        for (std::size_t r = 0; r < sp.dof.size(); ++r)
        {
            if (sp.dof[r] >= 0)
                dofs.push_back(sp.dof[r]);
            off[r + 1] = static_cast<int>(dofs.size());
        }
        const std::vector<double> w(dofs.size(), 1.0);
        in.y_off.upload(off.data(), off.size());
        in.y_dofs.upload(dofs.data(), dofs.size());
        in.y_w.upload(w.data(), w.size());
        out.src_ptr.upload(sp.src_ptr.data(), sp.src_ptr.size());
        out.src_list.upload(sp.src_list.data(), sp.src_list.size());
        APF_CUDA(cudaGetLastError());
    }

    // swaps the main system's X inputs into a slab system for the lifetime of the guard
    struct BorrowX
    {
        SystemInputs& a;
        SystemInputs& b;
        BorrowX(SystemInputs& main, SystemInputs& slab) : a(main), b(slab) { swap_x(); }
        ~BorrowX() { swap_x(); }
        void swap_x()
        {
            std::swap(a.x_geo, b.x_geo);
            std::swap(a.x_off, b.x_off);
            std::swap(a.x_dofs, b.x_dofs);
            std::swap(a.x_w, b.x_w);
        }
    };

    // lambda~ on the slab space: A_slab lambda~ = f_slab - B_slab^T u, the slab Riesz
    // reconstruction of every slab at once (the slab blocks are the main-system A_y, B^T and
    // f with the slab space as test space: time_slab_reconstruction_operator.hpp:686-830
    // assembles the same forms), solved by CG with an SA-AMG V-cycle to 1e-14
    void reconstruct_lambda_slabs(cudaStream_t s, System& S, SlabSystem& sl, DeviceBuffer<double>& lt,
                                  EstimatorTotals& tot)
    {
        SystemInputs& in = sl.in;
        const int nl = in.n_lambda, nd = in.ndof;
        DeviceCsr A, Bt;
        DeviceBuffer<double> f;
        {
            APF_HOST_RANGE("est_slab_assembly");
            BorrowX borrow(S.in, in);
            prepare_inputs(s, in);
            const Incidence inc =
                build_incidence(s, nl, in.n_y_cells, nullptr, nullptr, in.y_off.get(), in.y_dofs.get(), nd);
            const int offs[1] = {0};
            const Incidence* incs[1] = {&inc};
            const int ka[1] = {K_AY};
            gather_csr(s, in, in.zero_tol, nl, nl, 1, ka, incs, offs, in.kmax, A);
            const int kbt[1] = {K_BT};
            gather_csr(s, in, in.zero_tol, nl, in.n_u, 1, kbt, incs, offs, in.kmax, Bt);
            gather_vector_host(s, in, in.zero_tol, 0, inc, nl, in.ell.size() ? in.ell.get() : nullptr, in.u0_kind,
                               in.g_scale, f);
            sync(s);
        }
        lt.allocate(static_cast<std::size_t>(nl), s);
        lt.zero();
        if (nl == 0)
            return;
        DeviceBuffer<double> rhs(nl, s), r(nl, s), z(nl, s), pv(nl, s), q(nl, s);
        copy(s, nl, f.get(), rhs.get());
        spmv(s, Bt, S.solution.get() + S.in.n_lambda, rhs.get(), -1.0, 1.0);
        Amg amg;
        {
            APF_HOST_RANGE("est_slab_amg_setup");
            DeviceBuffer<int> comp;
            dof_time_components(s, in, true, comp);
            AmgOptions o = S.precond_opts;
            amg.setup(s, A, o, S.ws, comp.get());
        }
        copy(s, nl, rhs.get(), r.get());
        const double bn = std::sqrt(dot_host(s, S.ws, nl, rhs.get(), rhs.get()));
        double rn = bn;
        int its = 0;
        if (bn > 0.0)
        {
            APF_HOST_RANGE("est_reconstruction_pcg");
            amg.apply(s, r.get(), z.get());
            copy(s, nl, z.get(), pv.get());
            double rz = dot_host(s, S.ws, nl, r.get(), z.get());
            for (its = 1; its <= 400; ++its)
            {
                spmv(s, A, pv.get(), q.get());
                const double alpha = rz / dot_host(s, S.ws, nl, pv.get(), q.get());
                axpby(s, nl, alpha, pv.get(), 1.0, lt.get());
                axpby(s, nl, -alpha, q.get(), 1.0, r.get());
                rn = std::sqrt(dot_host(s, S.ws, nl, r.get(), r.get()));
                if (!(rn > 1e-14 * bn))
                    break;
                amg.apply(s, r.get(), z.get());
                const double rz2 = dot_host(s, S.ws, nl, r.get(), z.get());
                axpby(s, nl, 1.0, z.get(), rz2 / rz, pv.get());
                rz = rz2;
            }
        }
        tot.recon_iterations = its;
        tot.recon_residual = bn > 0.0 ? rn / bn : 0.0;
    }

    void reconstruct_lambda(cudaStream_t s, System& S, DeviceBuffer<double>& lt, EstimatorTotals& tot)
    {
        const int nl = S.in.n_lambda;
        DeviceBuffer<double> rhs(nl, s), r(nl, s), z(nl, s), pv(nl, s), q(nl, s);
        copy(s, nl, S.f.get(), rhs.get());
        spmv(s, S.blocks[APF_BLOCK_BT], S.solution.get() + nl, rhs.get(), -1.0, 1.0);
        copy(s, nl, S.solution.get(), lt.get());
        const DeviceCsr& Ay = S.blocks[APF_BLOCK_A_Y];
        residual(s, Ay, lt.get(), rhs.get(), r.get());
        const double bn = std::sqrt(dot_host(s, S.ws, nl, rhs.get(), rhs.get()));
        double rn = std::sqrt(dot_host(s, S.ws, nl, r.get(), r.get()));
        int its = 0;
        if (bn > 0.0 && rn > 1e-14 * bn)
        {
            APF_HOST_RANGE("est_reconstruction_pcg");
            S.precond->amg_a.apply(s, r.get(), z.get());
            copy(s, nl, z.get(), pv.get());
            double rz = dot_host(s, S.ws, nl, r.get(), z.get());
            for (its = 1; its <= 400; ++its)
            {
                spmv(s, Ay, pv.get(), q.get());
                const double alpha = rz / dot_host(s, S.ws, nl, pv.get(), q.get());
                axpby(s, nl, alpha, pv.get(), 1.0, lt.get());
                axpby(s, nl, -alpha, q.get(), 1.0, r.get());
                rn = std::sqrt(dot_host(s, S.ws, nl, r.get(), r.get()));
                if (!(rn > 1e-14 * bn))
                    break;
                S.precond->amg_a.apply(s, r.get(), z.get());
                const double rz2 = dot_host(s, S.ws, nl, r.get(), z.get());
                axpby(s, nl, 1.0, z.get(), rz2 / rz, pv.get());
                rz = rz2;
            }
        }
        tot.recon_iterations = its;
        tot.recon_residual = bn > 0.0 ? rn / bn : 0.0;
    }

    namespace
    {
        // sigma_x, sigma_y and div sigma of the kept flux at physical points (x, y, t), point i
        // in estimator cell cell[i]: the cell's three vertex-patch slots summed in a fixed
        // order (as the indicator kernels do), in the cell's own RT_p basis (Piola map of the
        // affine cell) times the P_p time basis of its interval.  A cell index out of range
        // gives NaN values and sets *bad.
        __global__ void flux_sample_kernel(int n, const int* __restrict__ cell, const double* __restrict__ pts,
                                           int n_cells, const double* __restrict__ geo,
                                           const double* __restrict__ sigma, int p,
                                           const Rt2Tables* __restrict__ t2, double* __restrict__ out,
                                           int* __restrict__ bad)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                const int c = cell[i];
                if (c < 0 || c >= n_cells)
                {
                    out[3ll * i] = out[3ll * i + 1] = out[3ll * i + 2] = __longlong_as_double(0x7ff8000000000000ll);
                    *bad = 1;
                    continue;
                }
                const Cell k = load_cell(geo, nullptr, nullptr, c);
                const double dx = pts[3ll * i] - k.x0, dy = pts[3ll * i + 1] - k.y0;
                const double x = (k.J11 * dx - k.J01 * dy) / k.det;
                const double y = (-k.J10 * dx + k.J00 * dy) / k.det;
                const double tau = (pts[3ll * i + 2] - k.t0) / k.ht;
                double sx = 0.0, sy = 0.0, sd = 0.0;
                if (p == 1)
                {
                    const double tb[2] = {1.0 - tau, tau};
                    for (int j = 0; j < 8; ++j)
                    {
                        double cj = 0.0;
                        for (int a = 0; a < 2; ++a)
                        {
                            double sj = 0.0;
                            for (int slot = 0; slot < 3; ++slot)
                                sj += sigma[((3ll * c + slot) * 2 + a) * 8 + j];
                            cj += sj * tb[a];
                        }
                        double vx, vy, dv;
                        rt_phys(k, j, x, y, vx, vy, dv);
                        sx += cj * vx;
                        sy += cj * vy;
                        sd += cj * dv;
                    }
                }
                else
                {
                    double T[3], dT[3];
                    p2_time(tau, T, dT);
                    double mvx[15], mvy[15], mdv[15];
                    mono15(x, y, mvx, mvy, mdv);
                    const double sdet = k.det < 0.0 ? -1.0 : 1.0;
                    for (int j = 0; j < 15; ++j)
                    {
                        double vx = 0.0, vy = 0.0, dv = 0.0;
                        for (int m = 0; m < 15; ++m)
                        {
                            vx += t2->c[j][m] * mvx[m];
                            vy += t2->c[j][m] * mvy[m];
                            dv += t2->c[j][m] * mdv[m];
                        }
                        const double f = (j < 9 ? sdet : 1.0) / k.det;
                        double cj = 0.0;
                        for (int a = 0; a < 3; ++a)
                        {
                            double sj = 0.0;
                            for (int slot = 0; slot < 3; ++slot)
                                sj += sigma[((3ll * c + slot) * 3 + a) * 15 + j];
                            cj += T[a] * sj;
                        }
                        sx += cj * f * (k.J00 * vx + k.J01 * vy);
                        sy += cj * f * (k.J10 * vx + k.J11 * vy);
                        sd += cj * f * dv;
                    }
                }
                out[3ll * i] = sx;
                out[3ll * i + 1] = sy;
                out[3ll * i + 2] = sd;
            }
        }
    }

    void flux_sample(cudaStream_t s, const System& S, int n, const int* cell, const double* points, double* values,
                     bool on_device)
    {
        require(S.flux_cells > 0 && S.flux_sigma.size() > 0, APF_ERR_INVALID,
                "flux samples: no kept flux (set keep_flux and run a 2+1D estimate first)");
        require(n >= 0, APF_ERR_INVALID, "flux samples: negative point count");
        if (n == 0)
            return;
        if (!on_device)
            for (int i = 0; i < n; ++i)
                require(cell[i] >= 0 && cell[i] < S.flux_cells, APF_ERR_INVALID, "flux samples: cell index out of range");
        upload_est_tables_once();
        DeviceBuffer<double> d_t2(0, s);
        if (S.flux_p == 2)
        {
            const Rt2Tables t2 = make_rt2_tables(make_est_tables());
            d_t2.upload(reinterpret_cast<const double*>(&t2), kRt2Doubles);
        }
        DeviceBuffer<int> d_cell(0, s), bad(1, s);
        DeviceBuffer<double> d_pts(0, s), d_out(0, s);
        const int* pc = cell;
        const double* pp = points;
        double* po = values;
        if (!on_device)
        {
            d_cell.upload(cell, static_cast<std::size_t>(n));
            d_pts.upload(points, 3ull * n);
            d_out.allocate(3ull * n, s);
            pc = d_cell.get();
            pp = d_pts.get();
            po = d_out.get();
        }
        bad.zero();
        {
            APF_KERNEL("est_flux_sample", s);
            flux_sample_kernel<<<nb(n, 128), 128, 0, s>>>(n, pc, pp, S.flux_cells, S.flux_geo.get(), S.flux_sigma.get(),
                                                          S.flux_p,
                                                          reinterpret_cast<const Rt2Tables*>(d_t2.size() ? d_t2.get()
                                                                                                         : nullptr),
                                                          po, bad.get());
        }
        APF_CUDA(cudaGetLastError());
        int hbad = 0;
        APF_CUDA(cudaMemcpyAsync(&hbad, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        if (!on_device)
            APF_CUDA(cudaMemcpyAsync(values, d_out.get(), 3ull * n * sizeof(double), cudaMemcpyDeviceToHost, s));
        sync(s);
        require(hbad == 0, APF_ERR_INVALID, "flux samples: cell index out of range");
    }

    EstimatorTotals estimate(cudaStream_t s, System& S, const std::vector<int>& vids_host, double* flux, double* div,
                                double* recon, double* eta, bool out_on_device, int patch_precision,
                                PatchTuner* tuner)
    {
        SystemInputs& in = S.in;
        require(in.p == 1 || in.p == 2, APF_ERR_INVALID, "estimator: p must be 1 or 2");
        require(patch_precision == APF_PATCH_FP64 || (patch_precision == APF_PATCH_FP32_REFINED && in.p == 1),
                APF_ERR_INVALID, "estimator: FP32 patch solves are available for p = 1");
        require(S.solution.size() == static_cast<std::size_t>(in.n_lambda + in.n_u), APF_ERR_INVALID,
                "estimator: solve the main system first");
        require(S.precond != nullptr, APF_ERR_INVALID, "estimator: preconditioner missing");
        upload_est_tables_once();
        S.flux_cells = 0;
        S.flux_sigma = DeviceBuffer<double>();
        S.flux_geo = DeviceBuffer<double>();
        EstimatorTotals tot{};
        const int ny = in.n_y_cells, nl = in.n_lambda, nd = in.ndof;
        const int ns = in.p == 1 ? 3 : 6, nt = in.p + 1;
        // ---- Y cell time intervals (host) and whether the Y restriction is trivial
        std::vector<double> ytimes(2ll * ny);
        int nontrivial = 0;
        {
            DeviceBuffer<double> dt(2ll * ny, s);
            DeviceBuffer<int> flag(1, s);
            flag.zero();
            if (ny)
            {
                {
                    APF_KERNEL("est_cell_times", s);
                    cell_times_kernel<<<nb(ny), 256, 0, s>>>(ny, in.y_geo.get(), dt.get());
                }
                {
                    APF_KERNEL("est_restriction_check", s);
                    nontrivial_restriction_kernel<<<nb((long long)ny * nd), 256, 0, s>>>((long long)ny * nd,
                                                                                       in.y_off.get(), in.y_w.get(),
                                                                                       flag.get());
                }
                APF_CUDA(cudaMemcpyAsync(ytimes.data(), dt.get(), ytimes.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
                APF_CUDA(cudaMemcpyAsync(&nontrivial, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
            }
            sync(s);
        }
        // ---- time slabs: when every Y cell lies in one slab and Y has no hanging rows the
        // slab space is Y itself (uniform and space-only adaptive meshes); otherwise Y cells are
        // cut into slab cells and lambda~ lives on the slab space
        SlabSpace sp;
        {
            APF_HOST_RANGE("est_slab_space");
            std::vector<double> T(ytimes);
            std::sort(T.begin(), T.end());
            T.erase(std::unique(T.begin(), T.end()), T.end());
            bool one_slab_each = true;
            for (int c = 0; c < ny && one_slab_each; ++c)
            {
                const auto a = std::upper_bound(T.begin(), T.end(), ytimes[2ll * c]);
                one_slab_each = a != T.end() && *a == ytimes[2ll * c + 1];
            }
            sp.identity = one_slab_each && nontrivial == 0;
        }
        SlabSystem sl;
        if (!sp.identity)
        {
            APF_HOST_RANGE("est_slab_space");
            std::vector<unsigned char> bnode(static_cast<std::size_t>(ny) * ns);
            if (ny)
            {
                DeviceBuffer<unsigned char> d_bnode(bnode.size(), s);
                {
                    APF_KERNEL("est_dirichlet_nodes", s);
                    dirichlet_nodes_kernel<<<nb((long long)ny * ns), 256, 0, s>>>(ny, ns, nt, in.y_off.get(), d_bnode.get());
                }
                APF_CUDA(cudaMemcpyAsync(bnode.data(), d_bnode.get(), bnode.size(), cudaMemcpyDeviceToHost, s));
                sync(s);
            }
            // spatial nodes: vertex nodes keyed by their vertex id, P2 edge nodes by their two
            // vertex ids (node order v0 m01 v1 m02 m12 v2)
            static const int kNodeVerts[2][6][2] = {{{0, 0}, {1, 1}, {2, 2}, {0, 0}, {0, 0}, {0, 0}},
                                                    {{0, 0}, {0, 1}, {1, 1}, {0, 2}, {1, 2}, {2, 2}}};
            std::vector<std::uint64_t> keys(static_cast<std::size_t>(ny) * ns);
            for (int c = 0; c < ny; ++c)
                for (int q = 0; q < ns; ++q)
                {
                    const int a = vids_host[3ll * c + kNodeVerts[in.p - 1][q][0]];
                    const int b = vids_host[3ll * c + kNodeVerts[in.p - 1][q][1]];
                    const std::uint32_t lo = static_cast<std::uint32_t>(std::min(a, b));
                    const std::uint32_t hi = static_cast<std::uint32_t>(std::max(a, b));
                    keys[static_cast<std::size_t>(c) * ns + q] = (static_cast<std::uint64_t>(lo) << 32) | hi;
                }
            build_slab_space(ns, nt, ny, ytimes, vids_host, keys, bnode, sp);
            upload_slab_system(s, in, sp, sl);
        }
        // the cells the patches and indicators run on: Y cells, or slab cells
        const int nc = sp.identity ? ny : sp.n_cells;
        const double* cgeo = sp.identity ? in.y_geo.get() : sl.in.y_geo.get();
        const double* cm = sp.identity ? (in.m_y.size() ? in.m_y.get() : nullptr)
                                       : (sl.in.m_y.size() ? sl.in.m_y.get() : nullptr);
        const double* cell = sp.identity ? (in.ell.size() ? in.ell.get() : nullptr)
                                         : (sl.in.ell.size() ? sl.in.ell.get() : nullptr);
        const int* cx = sp.identity ? in.y_to_x.get() : sl.in.y_to_x.get();
        // ---- patch topology: host integer work on the cells' time intervals and vertex ids,
        // run on a host thread while the device solves the slab reconstruction
        std::future<PatchSet> patches = std::async(std::launch::async, [&sp, &ytimes, &vids_host, ny, nc]() {
            PatchSet ps;
            if (sp.identity)
                build_patches(ytimes, vids_host, ny, ps);
            else
                build_patches(sp.times, sp.vids, nc, ps);
            return ps;
        });
        // ---- lambda~
        DeviceBuffer<double> lt(sp.identity ? nl : 0, s);
        if (sp.identity)
            reconstruct_lambda(s, S, lt, tot);
        else
            reconstruct_lambda_slabs(s, S, sl, lt, tot);
        PatchSet ps;
        {
            APF_HOST_RANGE("est_patch_topology_wait");
            ps = patches.get();
        }
        // ---- nodal data per cell: lambda~ through the slab restriction; lambda_delta and u
        // as the local functions of the cell's Y cell and X ancestor at its nodes
        DeviceBuffer<double> theta((long long)nd * nc, s), ucell((long long)nd * nc, s), ldel((long long)nd * nc, s),
            ltil((long long)nd * nc, s);
        const double* u = S.solution.get() + nl;
        {
            const SystemInputs& li = sp.identity ? in : sl.in;
            APF_KERNEL("est_gather_nodal", s);
            gather_nodal<<<nb((long long)nc * nd), 256, 0, s>>>(nc, nd, li.y_off.get(), li.y_dofs.get(), li.y_w.get(),
                                                                lt.get(), nullptr, ltil.get());
        }
        {
            DeviceBuffer<double> ly((long long)nd * ny, s);
            {
                APF_KERNEL("est_gather_nodal", s);
                gather_nodal<<<nb((long long)ny * nd), 256, 0, s>>>(ny, nd, in.y_off.get(), in.y_dofs.get(),
                                                                    in.y_w.get(), S.solution.get(), nullptr, ly.get());
            }
            if (sp.identity)
                copy(s, nd * ny, ly.get(), ldel.get());
            else
            {
                DeviceBuffer<int> d_src(0, s);
                d_src.upload(sp.source.data(), sp.source.size());
                nodal_transfer(s, in.p, nc, cgeo, d_src.get(), in.y_geo.get(), ly.get(), ldel.get());
            }
        }
        {
            const int nx = in.n_x_cells;
            DeviceBuffer<double> ux((long long)nd * nx, s);
            {
                APF_KERNEL("est_gather_nodal", s);
                gather_nodal<<<nb((long long)nx * nd), 256, 0, s>>>(nx, nd, in.x_off.get(), in.x_dofs.get(),
                                                                    in.x_w.get(), u, nullptr, ux.get());
            }
            nodal_transfer(s, in.p, nc, cgeo, cx, in.x_geo.get(), ux.get(), ucell.get());
        }
        axpby(s, nd * nc, 1.0, ltil.get(), 0.0, theta.get());
        axpby(s, nd * nc, 1.0, ucell.get(), 1.0, theta.get());
        tot.n_slabs = ps.n_slabs;
        tot.n_patches = static_cast<int>(ps.patch_slab.size());
        tot.max_patch_cells = ps.max_cells;
        auto up = [&](DeviceBuffer<int>& d, const std::vector<int>& h) { d.upload(h.data(), h.size()); };
        DeviceBuffer<int> d_pslab(0, s), d_ptopo(0, s), d_tptr(0, s), d_tcell(0, s), d_tcen(0, s), d_tedge(0, s),
            d_tnf(0, s), d_tbd(0, s), d_sptr(0, s), d_scell(0, s), status(1, s);
        up(d_pslab, ps.patch_slab);
        up(d_ptopo, ps.patch_topo);
        up(d_tptr, ps.topo_ptr);
        up(d_tcell, ps.topo_cell);
        up(d_tcen, ps.topo_center);
        up(d_tedge, ps.topo_edge);
        up(d_tnf, ps.topo_nfree);
        up(d_tbd, ps.topo_boundary);
        up(d_sptr, ps.slab_ptr);
        up(d_scell, ps.slab_cells);
        status.zero();
        const bool p2 = in.p == 2;
        DeviceBuffer<double> sigma((p2 ? 135ll : 48ll) * nc, s);
        sigma.zero();
        PatchArgs pa{};
        pa.n_patches = tot.n_patches;
        pa.patch_slab = d_pslab.get();
        pa.patch_topo = d_ptopo.get();
        pa.topo_ptr = d_tptr.get();
        pa.topo_cell = d_tcell.get();
        pa.topo_center = d_tcen.get();
        pa.topo_edge = d_tedge.get();
        pa.topo_nfree = d_tnf.get();
        pa.topo_boundary = d_tbd.get();
        pa.slab_ptr = d_sptr.get();
        pa.slab_cells = d_scell.get();
        pa.geo = cgeo;
        pa.m = cm;
        pa.ell = cell;
        pa.theta = theta.get();
        pa.u = ucell.get();
        pa.sigma = sigma.get();
        pa.status = status.get();
        // patches sorted into size buckets (one warp each; shared memory sized per bucket)
        constexpr int kBuckets = kPatchBuckets;
        const int* kBucketMax = kPatchBucketMax;
        std::vector<int> bucket_count(kBuckets + 1, 0), order(tot.n_patches);
        {
            std::vector<signed char> bucket_of(tot.n_patches);
            for (int p = 0; p < tot.n_patches; ++p)
            {
                const int tp = ps.patch_topo[p];
                const int nc = ps.topo_ptr[tp + 1] - ps.topo_ptr[tp];
                const int n = (p2 ? 3 * ps.topo_nfree[tp] + 12 * nc : 2 * ps.topo_nfree[tp] + 5 * nc) +
                              (ps.topo_boundary[tp] ? 0 : 1);
                int b = 0;
                while (b < kBuckets && n > kBucketMax[b])
                    ++b;
                require(b < kBuckets, APF_ERR_CAPACITY, "estimator: patch too large (more than 144 unknowns)");
                bucket_of[p] = static_cast<signed char>(b);
                ++bucket_count[b + 1];
            }
            for (int b = 0; b < kBuckets; ++b)
                bucket_count[b + 1] += bucket_count[b];
            std::vector<int> fill(bucket_count.begin(), bucket_count.end() - 1);
            for (int p = 0; p < tot.n_patches; ++p)
                order[fill[bucket_of[p]]++] = p;
        }
        DeviceBuffer<int> d_order(0, s);
        up(d_order, order);
        const EstTables est = make_est_tables();
        const PatchTables ptab = make_patch_tables(est);
        DeviceBuffer<double> d_ptab(kPatchTableDoubles, s);
        d_ptab.upload(reinterpret_cast<const double*>(&ptab), kPatchTableDoubles);
        const PatchTables* tables = reinterpret_cast<const PatchTables*>(d_ptab.get());
        DeviceBuffer<double> d_rt2;
        const Rt2Tables* tables2 = nullptr;
        if (p2)
        {
            const Rt2Tables t2 = make_rt2_tables(est);
            d_rt2.allocate(kRt2Doubles, s);
            d_rt2.upload(reinterpret_cast<const double*>(&t2), kRt2Doubles);
            tables2 = reinterpret_cast<const Rt2Tables*>(d_rt2.get());
        }
        // one team of W warps per patch: larger patches get more warps (the LU's column
        // updates and the assembly spread over 32 W threads; shared memory bounds the teams
        // per SM).  W per (degree, precision, bucket) comes from the context's autotuner when
        // it is on (every candidate timed once on the bucket's own patches; all candidates
        // compute the same values in the same order), else from the size rule below.
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        const bool tuning = tuner && tuner->enabled;
        if (tuning)
        {
            APF_CUDA(cudaEventCreate(&ev0));
            APF_CUDA(cudaEventCreate(&ev1));
        }
        auto launch = [&](auto tag, int b) {
            constexpr int NMAX = decltype(tag)::value;
            constexpr int W_RULE = NMAX <= 48 ? 1 : (NMAX <= 64 ? 2 : 4);
            const int count = bucket_count[b + 1] - bucket_count[b];
            if (count == 0)
                return;
            pa.nmax = NMAX;
            const bool f32 = patch_precision == APF_PATCH_FP32_REFINED;
            auto run = [&](auto wtag, auto f32tag) {
                constexpr int W = decltype(wtag)::value;
                constexpr bool F32 = decltype(f32tag)::value;
                if (p2)
                {
                    constexpr std::size_t smem = patch2_smem_bytes<NMAX>();
                    APF_CUDA(cudaFuncSetAttribute(patch_solve2<NMAX, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)smem));
                    const int per_sm = std::max<int>(1, static_cast<int>((227u * 1024u) / (smem + 1024u)));
                    const int grid = std::max(1, std::min(count, 148 * std::min(per_sm, 32 / W)));
                    APF_KERNEL("est_patch_solve", s);
                    patch_solve2<NMAX, W><<<grid, 32 * W, smem, s>>>(pa, tables2, d_order.get() + bucket_count[b], count);
                    return;
                }
                constexpr std::size_t smem = patch_smem_bytes<NMAX, F32>();
                APF_CUDA(cudaFuncSetAttribute(patch_solve<NMAX, W, F32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem));
                const int per_sm = std::max<int>(1, static_cast<int>((227u * 1024u) / (smem + 1024u)));
                const int grid = std::max(1, std::min(count, 148 * std::min(per_sm, 32 / W)));
                APF_KERNEL("est_patch_solve", s);
                patch_solve<NMAX, W, F32><<<grid, 32 * W, smem, s>>>(pa, tables, d_order.get() + bucket_count[b], count);
            };
            auto run_w = [&](int w) {
                auto with_w = [&](auto wtag) {
                    if (f32 && !p2)
                        run(wtag, std::true_type{});
                    else
                        run(wtag, std::false_type{});
                };
                if (w == 1)
                    with_w(std::integral_constant<int, 1>{});
                else if (w == 2)
                    with_w(std::integral_constant<int, 2>{});
                else
                    with_w(std::integral_constant<int, 4>{});
                APF_CUDA(cudaGetLastError());
            };
            int* choice = tuner ? &tuner->width[p2 ? 1 : 0][f32 ? 1 : 0][b] : nullptr;
            if (tuning && *choice == 0)
            {
                static constexpr int kCand[3] = {1, 2, 4};
                float best = 0.0f;
                for (int k = 0; k < 3; ++k)
                {
                    APF_CUDA(cudaEventRecord(ev0, s));
                    run_w(kCand[k]);
                    APF_CUDA(cudaEventRecord(ev1, s));
                    APF_CUDA(cudaEventSynchronize(ev1));
                    float ms = 0.0f;
                    APF_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
                    tuner->ms[p2 ? 1 : 0][f32 ? 1 : 0][b][k] = ms;
                    tuner->patches[p2 ? 1 : 0][f32 ? 1 : 0][b] = count;
                    if (k == 0 || ms < best)
                    {
                        best = ms;
                        *choice = kCand[k];
                    }
                }
                return;
            }
            run_w(choice && *choice ? *choice : W_RULE);
        };
        APF_HOST_RANGE("est_patch_solves");
        if (tot.n_patches > 0)
        {
            static_assert(kPatchBuckets == 7 && kPatchBucketMax[0] == 30 && kPatchBucketMax[1] == 40 &&
                              kPatchBucketMax[2] == 48 && kPatchBucketMax[3] == 58 && kPatchBucketMax[4] == 64 &&
                              kPatchBucketMax[5] == 96 && kPatchBucketMax[6] == 144,
                          "bucket launches follow kPatchBucketMax");
            launch(std::integral_constant<int, 30>{}, 0);
            launch(std::integral_constant<int, 40>{}, 1);
            launch(std::integral_constant<int, 48>{}, 2);
            launch(std::integral_constant<int, 58>{}, 3);
            launch(std::integral_constant<int, 64>{}, 4);
            launch(std::integral_constant<int, 96>{}, 5);
            launch(std::integral_constant<int, 144>{}, 6);
            APF_CUDA(cudaGetLastError());
        }
        if (ev0)
            cudaEventDestroy(ev0);
        if (ev1)
            cudaEventDestroy(ev1);
        int hstat = 0;
        APF_CUDA(cudaMemcpyAsync(&hstat, status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        sync(s);
        if (hstat == APF_ERR_NUMERIC)
            throw Error(APF_ERR_NUMERIC, "estimator: singular patch system");
        if (hstat != 0)
            throw Error(APF_ERR_CAPACITY, "estimator: patch system larger than the kernel's buffer");
        // ---- indicators per cell, then (slab cells) summed onto their Y cells
        DeviceBuffer<double> f2(nc, s), d2(nc, s), r2(nc, s), e2(nc, s);
        IndicatorArgs ia{nc, cgeo, pa.m, pa.ell, theta.get(), ucell.get(), ldel.get(), ltil.get(), sigma.get(),
                         f2.get(), d2.get(), r2.get(), e2.get()};
        if (p2)
        {
            {
                APF_KERNEL("est_cell_indicators", s);
                cell_indicators2<<<nb(nc, 128), 128, 0, s>>>(ia, tables2);
            }
            // ||lambda_delta - lambda~||^2 in the local A_y energy, eta = flux + that
            if (sp.identity)
            {
                DeviceBuffer<double> dl(nl, s);
                copy(s, nl, S.solution.get(), dl.get());
                axpby(s, nl, -1.0, lt.get(), 1.0, dl.get());
                y_cell_energy(s, in, dl.get(), r2.get());
            }
            else
            {
                DeviceBuffer<double> dl((long long)nd * nc, s);
                copy(s, nd * nc, ldel.get(), dl.get());
                axpby(s, nd * nc, -1.0, ltil.get(), 1.0, dl.get());
                nodal_energy(s, in.p, nc, cgeo, cm, dl.get(), r2.get());
            }
            {
                APF_KERNEL("est_eta", s);
                add_kernel<<<nb(nc), 256, 0, s>>>(nc, f2.get(), r2.get(), e2.get());
            }
        }
        else
        {
            APF_KERNEL("est_cell_indicators", s);
            cell_indicators<<<nb(nc, 128), 128, 0, s>>>(ia);
        }
        APF_CUDA(cudaGetLastError());
        if (S.keep_flux)
        {
            // the flux stays on the device for flux_sample, keyed by (slab, source Y cell)
            S.flux_p = in.p;
            S.flux_cells = nc;
            S.flux_sigma = std::move(sigma);
            S.flux_geo.allocate(8ll * nc, s);
            copy(s, 8 * nc, cgeo, S.flux_geo.get());
            S.flux_slab.assign(static_cast<std::size_t>(nc), -1);
            for (int sb = 0; sb + 1 < static_cast<int>(ps.slab_ptr.size()); ++sb)
                for (int q = ps.slab_ptr[sb]; q < ps.slab_ptr[sb + 1]; ++q)
                    S.flux_slab[static_cast<std::size_t>(ps.slab_cells[q])] = sb;
            if (sp.identity)
            {
                S.flux_source.resize(static_cast<std::size_t>(nc));
                std::iota(S.flux_source.begin(), S.flux_source.end(), 0);
            }
            else
                S.flux_source = sp.source;
        }
        if (!sp.identity)
        {
            DeviceBuffer<double> tmp(nc, s);
            for (DeviceBuffer<double>* a : {&f2, &d2, &r2, &e2})
            {
                copy(s, nc, a->get(), tmp.get());
                a->allocate(ny, s);
                if (ny)
                {
                    APF_KERNEL("est_reduce_to_source", s);
                    reduce_to_source_kernel<<<nb(ny), 256, 0, s>>>(ny, sl.src_ptr.get(), sl.src_list.get(), tmp.get(),
                                                                   a->get());
                }
            }
            APF_CUDA(cudaGetLastError());
        }
        tot.flux = device_sum(s, ny, f2.get());
        tot.div = device_sum(s, ny, d2.get());
        tot.recon = device_sum(s, ny, r2.get());
        tot.eta = device_sum(s, ny, e2.get());
        const cudaMemcpyKind kind = out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        if (flux) APF_CUDA(cudaMemcpyAsync(flux, f2.get(), ny * sizeof(double), kind, s));
        if (div) APF_CUDA(cudaMemcpyAsync(div, d2.get(), ny * sizeof(double), kind, s));
        if (recon) APF_CUDA(cudaMemcpyAsync(recon, r2.get(), ny * sizeof(double), kind, s));
        if (eta) APF_CUDA(cudaMemcpyAsync(eta, e2.get(), ny * sizeof(double), kind, s));
        sync(s);
        return tot;
    }
}

// ---------------------------------------------------------------------------------------
// 1+1D (P1) edge-patch estimator.
//
// Restates TimeSlabEquilibratedFluxReconstruction1plus1d
// (src/finite_element/time_slabs/time_slab_equilibrated_flux_reconstruction.hpp:773-1880)
// and compute_equilibrated_flux_error_squared_by_source_cell_1plus1d
// (time_slab_equilibrated_flux_indicators.hpp:23-190):
//   * patches (time_slab_edge_patch_builder.hpp:353-537): per time slab, its cells sorted
//     by x; one boundary patch at each end (one cell) and one interior patch per shared
//     spatial vertex (left cell, right cell);
//   * flux space (patch_flux_space_1d.hpp): spatial functions {hat of the patch vertex,
//     x(1-x) bubble of every patch cell} x shifted Legendre {1, 2 tau - 1} in time, index
//     = i_space * 2 + i_time; scalar space (patch_scalar_space.hpp): boundary patch
//     {1, 2 x - 1}, interior patch {2 x - 1 on the left cell, 2 x - 1 on the right cell,
//     the weighted Haar function (h_R, -h_L) / (h_L + h_R)}, same time functions;
//   * local forms on 3 x 3 Gauss points of every patch cell (local_error_bilinear_forms.hpp,
//     local_error_linear_forms.hpp): A = (M^-1 sigma_j, sigma_i), B = (div sigma_j, q_i),
//     f = -(psi_a d_x theta~, sigma_i), g = (psi_a (l - d_t u) - d_x psi_a M d_x theta~, q_i),
//     entries of A and B with |a| <= zero_tol dropped (mat_A_1d.hpp, mat_B_1d.hpp), C = 0
//     (mat_C_1d.hpp); [A B^T; B 0] solved exactly (partial-pivot LU), one thread per patch;
//   * indicators per Y cell on 3 x 3 Gauss points: flux^2 = ((sigma + M d_x theta~)^2 / M),
//     div^2 = (l - d_t u - d_x sigma)^2, plus the reconstruction energy of lambda_delta -
//     lambda~ (time_slab_error_norms.hpp:946).
// ---------------------------------------------------------------------------------------
namespace apf
{
    namespace
    {
        constexpr int kEdgeMax = 12; // interior patch: 6 flux + 6 scalar unknowns

        struct EdgeArgs
        {
            int n_patches;
            const int* left;  // [patch] cell left of the patch vertex or -1
            const int* right; // [patch] cell right of the patch vertex or -1
            const double* geo;
            const double* m;
            const double* ell;
            const double* lt; // [cell][4] lambda~ nodal values
            const double* u;  // [cell][4] u_delta nodal values
            double zero_tol;
            double* sigma;    // [cell][2 slots][4]: hat L0, hat L1, bubble L0, bubble L1
            int* status;
        };

        // d_x and d_t of a P1 x P1 nodal function at (xi, tau) of cell g
        __device__ __forceinline__ void nodal_grad(const double* v, const q1d::Quad& g, double xi, double tau,
                                                   double& dx, double& dt)
        {
            dx = ((v[2] - v[0]) * (1.0 - tau) + (v[3] - v[1]) * tau) / g.h;
            dt = ((v[1] - v[0]) * (1.0 - xi) + (v[3] - v[2]) * xi) / g.k;
        }

        __global__ void edge_patch_solve(EdgeArgs A)
        {
            for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < A.n_patches; p += gridDim.x * blockDim.x)
            {
                const int cl = A.left[p], cr = A.right[p];
                const bool boundary = cl < 0 || cr < 0;
                const int nc = boundary ? 1 : 2;
                const int nfs = 1 + nc, nss = boundary ? 2 : 3;
                const int nf = 2 * nfs, ns = 2 * nss, n = nf + ns;
                double K[kEdgeMax][kEdgeMax + 1];
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j <= n; ++j)
                        K[i][j] = 0.0;
                double hl = 0.0, hr = 0.0;
                if (!boundary)
                {
                    hl = q1d::load(A.geo, cl).h;
                    hr = q1d::load(A.geo, cr).h;
                }
                double Aloc[6][6], Bloc[6][6];
                for (int i = 0; i < nf; ++i)
                    for (int j = 0; j < nf; ++j)
                        Aloc[i][j] = 0.0;
                for (int i = 0; i < ns; ++i)
                    for (int j = 0; j < nf; ++j)
                        Bloc[i][j] = 0.0;
                for (int pc = 0; pc < nc; ++pc)
                {
                    // patch cell pc: the left cell lies left of the vertex (hat = x), the
                    // right cell right of it (hat = 1 - x)
                    const int c = boundary ? (cl >= 0 ? cl : cr) : (pc == 0 ? cl : cr);
                    const bool left_of_vertex = boundary ? (cl >= 0) : (pc == 0);
                    const q1d::Quad g = q1d::load(A.geo, c);
                    const double m = A.m ? A.m[c] : 1.0;
                    const double ell = A.ell ? A.ell[c] : 0.0;
                    const int bub = boundary ? 1 : (left_of_vertex ? 1 : 2);
                    const double* lt = A.lt + 4ll * c;
                    const double* uu = A.u + 4ll * c;
                    const double jac = g.h * g.k;
                    for (int qx = 0; qx < 3; ++qx)
                    {
                        const double xi = q1d::gauss_x(qx), wx = q1d::gauss_w(qx);
                        const double psi = left_of_vertex ? xi : 1.0 - xi;
                        const double dpsi = (left_of_vertex ? 1.0 : -1.0) / g.h;
                        // spatial flux functions on this cell: hat (0) and the cell's bubble
                        const double sv[2] = {psi, xi * (1.0 - xi)};
                        const double sd[2] = {(left_of_vertex ? 1.0 : -1.0) / g.h, (1.0 - 2.0 * xi) / g.h};
                        const int sidx[2] = {0, bub};
                        // spatial scalar functions (value at xi, index)
                        double qv[3];
                        int qn = 0;
                        int qidx[3];
                        if (boundary)
                        {
                            qv[0] = 1.0; qidx[0] = 0;
                            qv[1] = 2.0 * xi - 1.0; qidx[1] = 1;
                            qn = 2;
                        }
                        else
                        {
                            qv[0] = 2.0 * xi - 1.0; qidx[0] = left_of_vertex ? 0 : 1;
                            qv[1] = left_of_vertex ? hr / (hl + hr) : -hl / (hl + hr); qidx[1] = 2;
                            qn = 2;
                        }
                        for (int qt = 0; qt < 3; ++qt)
                        {
                            const double tau = q1d::gauss_x(qt), w = wx * q1d::gauss_w(qt) * jac;
                            const double T[2] = {1.0, 2.0 * tau - 1.0};
                            double dlx, dlt, dux, dut;
                            nodal_grad(lt, g, xi, tau, dlx, dlt);
                            nodal_grad(uu, g, xi, tau, dux, dut);
                            const double gth = dlx + dux;
                            const double frhs = -psi * gth * w;
                            const double grhs = (psi * (ell - dut) - dpsi * m * gth) * w;
                            for (int a = 0; a < 2; ++a)
                                for (int ka = 0; ka < 2; ++ka)
                                {
                                    const int i = sidx[a] * 2 + ka;
                                    const double si = sv[a] * T[ka];
                                    K[i][n] += frhs * si;
                                    for (int b = 0; b < 2; ++b)
                                        for (int kb = 0; kb < 2; ++kb)
                                            Aloc[i][sidx[b] * 2 + kb] += si * sv[b] * T[kb] / m * w;
                                }
                            for (int a = 0; a < qn; ++a)
                                for (int ka = 0; ka < 2; ++ka)
                                {
                                    const int i = qidx[a] * 2 + ka;
                                    const double qi = qv[a] * T[ka];
                                    K[nf + i][n] += grhs * qi;
                                    for (int b = 0; b < 2; ++b)
                                        for (int kb = 0; kb < 2; ++kb)
                                            Bloc[i][sidx[b] * 2 + kb] += qi * sd[b] * T[kb] * w;
                                }
                        }
                    }
                }
                for (int i = 0; i < nf; ++i)
                    for (int j = 0; j < nf; ++j)
                        K[i][j] = fabs(Aloc[i][j]) > A.zero_tol ? Aloc[i][j] : 0.0;
                for (int i = 0; i < ns; ++i)
                    for (int j = 0; j < nf; ++j)
                    {
                        const double v = fabs(Bloc[i][j]) > A.zero_tol ? Bloc[i][j] : 0.0;
                        K[nf + i][j] = v;
                        K[j][nf + i] = v;
                    }
                // partial-pivot elimination on the augmented n x (n + 1) system
                bool singular = false;
                for (int col = 0; col < n; ++col)
                {
                    int piv = col;
                    double best = fabs(K[col][col]);
                    for (int i = col + 1; i < n; ++i)
                        if (fabs(K[i][col]) > best)
                        {
                            best = fabs(K[i][col]);
                            piv = i;
                        }
                    if (!(best > 0.0) || !isfinite(best))
                    {
                        singular = true;
                        break;
                    }
                    if (piv != col)
                        for (int j = col; j <= n; ++j)
                        {
                            const double t = K[col][j];
                            K[col][j] = K[piv][j];
                            K[piv][j] = t;
                        }
                    const double inv = 1.0 / K[col][col];
                    for (int i = col + 1; i < n; ++i)
                    {
                        const double l = K[i][col] * inv;
                        if (l != 0.0)
                            for (int j = col + 1; j <= n; ++j)
                                K[i][j] -= l * K[col][j];
                    }
                }
                if (singular)
                {
                    atomicExch(A.status, APF_ERR_NUMERIC);
                    continue;
                }
                double x[kEdgeMax];
                for (int i = n - 1; i >= 0; --i)
                {
                    double v = K[i][n];
                    for (int j = i + 1; j < n; ++j)
                        v -= K[i][j] * x[j];
                    x[i] = v / K[i][i];
                }
                // this patch's flux on each of its cells -> the cell's slot of the vertex
                for (int pc = 0; pc < nc; ++pc)
                {
                    const int c = boundary ? (cl >= 0 ? cl : cr) : (pc == 0 ? cl : cr);
                    const bool left_of_vertex = boundary ? (cl >= 0) : (pc == 0);
                    const int bub = boundary ? 1 : (left_of_vertex ? 1 : 2);
                    // slot 0: the patch at the cell's left vertex (cell right of it), 1: right
                    double* out = A.sigma + 8ll * c + (left_of_vertex ? 4 : 0);
                    out[0] = x[0];
                    out[1] = x[1];
                    out[2] = x[2 * bub];
                    out[3] = x[2 * bub + 1];
                }
            }
        }

        struct EdgeIndArgs
        {
            int n_cells;
            const double* geo;
            const double* m;
            const double* ell;
            const double* lt;
            const double* u;
            const double* sigma;
            double* flux;
            double* div;
        };

        __global__ void edge_cell_indicators(EdgeIndArgs A)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.n_cells; c += gridDim.x * blockDim.x)
            {
                const q1d::Quad g = q1d::load(A.geo, c);
                const double m = A.m ? A.m[c] : 1.0;
                const double ell = A.ell ? A.ell[c] : 0.0;
                const double* sg = A.sigma + 8ll * c;
                const double* lt = A.lt + 4ll * c;
                const double* uu = A.u + 4ll * c;
                double fl = 0.0, dv = 0.0;
                for (int qx = 0; qx < 3; ++qx)
                {
                    const double xi = q1d::gauss_x(qx);
                    for (int qt = 0; qt < 3; ++qt)
                    {
                        const double tau = q1d::gauss_x(qt);
                        const double w = q1d::gauss_w(qx) * q1d::gauss_w(qt) * g.h * g.k;
                        const double L1 = 2.0 * tau - 1.0, bub = xi * (1.0 - xi);
                        double sigma = 0.0, dsig = 0.0;
                        for (int slot = 0; slot < 2; ++slot)
                        {
                            const double* q = sg + 4 * slot;
                            const double hat = slot == 0 ? 1.0 - xi : xi;
                            const double dhat = (slot == 0 ? -1.0 : 1.0) / g.h;
                            const double th = q[0] + q[1] * L1, tb = q[2] + q[3] * L1;
                            sigma += th * hat + tb * bub;
                            dsig += th * dhat + tb * (1.0 - 2.0 * xi) / g.h;
                        }
                        double dlx, dlt, dux, dut;
                        nodal_grad(lt, g, xi, tau, dlx, dlt);
                        nodal_grad(uu, g, xi, tau, dux, dut);
                        const double e = sigma + m * (dlx + dux);
                        fl += e * e / m * w;
                        const double r = ell - dut - dsig;
                        dv += r * r * w;
                    }
                }
                A.flux[c] = fl;
                A.div[c] = dv;
            }
        }
    }

    EstimatorTotals estimate_1d(cudaStream_t s, System& S, double* flux, double* div, double* recon, double* eta,
                                bool out_on_device)
    {
        SystemInputs& in = S.in;
        require(in.dim == 1 && in.p == 1, APF_ERR_INVALID, "1+1D estimator: P1 only");
        require(S.solution.size() == static_cast<std::size_t>(in.n_lambda + in.n_u), APF_ERR_INVALID,
                "estimator: solve the main system first");
        require(S.precond != nullptr, APF_ERR_INVALID, "estimator: preconditioner missing");
        EstimatorTotals tot{};
        const int ny = in.n_y_cells, nl = in.n_lambda;
        // ---- Y cell intervals (host) and whether the Y restriction is trivial
        std::vector<double> ygeo(4ll * ny), ytimes(2ll * ny);
        int nontrivial = 0;
        if (ny)
        {
            DeviceBuffer<int> flag(1, s);
            flag.zero();
            {
                APF_KERNEL("est_restriction_check", s);
                nontrivial_restriction_kernel<<<nb(4ll * ny), 256, 0, s>>>(4ll * ny, in.y_off.get(), in.y_w.get(),
                                                                          flag.get());
            }
            APF_CUDA(cudaMemcpyAsync(ygeo.data(), in.y_geo.get(), ygeo.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
            APF_CUDA(cudaMemcpyAsync(&nontrivial, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
            sync(s);
        }
        for (int c = 0; c < ny; ++c)
        {
            ytimes[2ll * c] = ygeo[4ll * c + 2];
            ytimes[2ll * c + 1] = ygeo[4ll * c + 3];
        }
        // ---- time slabs (as in 2+1D): Y itself, or Y cells cut into slab cells
        SlabSpace sp;
        {
            std::vector<double> T(ytimes);
            std::sort(T.begin(), T.end());
            T.erase(std::unique(T.begin(), T.end()), T.end());
            bool one_slab_each = true;
            for (int c = 0; c < ny && one_slab_each; ++c)
            {
                const auto a = std::upper_bound(T.begin(), T.end(), ytimes[2ll * c]);
                one_slab_each = a != T.end() && *a == ytimes[2ll * c + 1];
            }
            sp.identity = one_slab_each && nontrivial == 0;
        }
        SlabSystem sl;
        std::vector<double> geo; // the cells' geometry on the host (Y cells or slab cells)
        if (!sp.identity)
        {
            APF_HOST_RANGE("est_slab_space");
            std::vector<unsigned char> bnode(2ll * ny);
            if (ny)
            {
                DeviceBuffer<unsigned char> d_bnode(bnode.size(), s);
                {
                    APF_KERNEL("est_dirichlet_nodes", s);
                    dirichlet_nodes_kernel<<<nb(2ll * ny), 256, 0, s>>>(ny, 2, 2, in.y_off.get(), d_bnode.get());
                }
                APF_CUDA(cudaMemcpyAsync(bnode.data(), d_bnode.get(), bnode.size(), cudaMemcpyDeviceToHost, s));
                sync(s);
            }
            // spatial nodes are points of the line: keyed by the bits of their coordinate
            std::vector<std::uint64_t> keys(2ll * ny);
            for (int c = 0; c < ny; ++c)
                for (int q = 0; q < 2; ++q)
                    std::memcpy(&keys[2ll * c + q], &ygeo[4ll * c + q], sizeof(double));
            build_slab_space(2, 2, ny, ytimes, {}, keys, bnode, sp);
            upload_slab_system(s, in, sp, sl);
            geo.resize(4ll * sp.n_cells);
            for (int i = 0; i < sp.n_cells; ++i)
            {
                geo[4ll * i] = ygeo[4ll * sp.source[i]];
                geo[4ll * i + 1] = ygeo[4ll * sp.source[i] + 1];
                geo[4ll * i + 2] = sp.times[2ll * i];
                geo[4ll * i + 3] = sp.times[2ll * i + 1];
            }
        }
        else
            geo.swap(ygeo);
        const int nc = sp.identity ? ny : sp.n_cells;
        const double* cgeo = sp.identity ? in.y_geo.get() : sl.in.y_geo.get();
        const double* cm = sp.identity ? (in.m_y.size() ? in.m_y.get() : nullptr)
                                       : (sl.in.m_y.size() ? sl.in.m_y.get() : nullptr);
        const double* cell = sp.identity ? (in.ell.size() ? in.ell.get() : nullptr)
                                         : (sl.in.ell.size() ? sl.in.ell.get() : nullptr);
        const int* cx = sp.identity ? in.y_to_x.get() : sl.in.y_to_x.get();
        // ---- edge patches: host integer work on the cells' intervals
        std::vector<int> order(nc);
        for (int c = 0; c < nc; ++c)
            order[c] = c;
        // slabs = distinct time intervals (in time order), cells of a slab by x
        std::sort(order.begin(), order.end(), [&](int a, int b) {
            const double* ga = &geo[4ll * a];
            const double* gb = &geo[4ll * b];
            if (ga[2] != gb[2]) return ga[2] < gb[2];
            if (ga[3] != gb[3]) return ga[3] < gb[3];
            if (ga[0] != gb[0]) return ga[0] < gb[0];
            if (ga[1] != gb[1]) return ga[1] < gb[1];
            return a < b;
        });
        std::vector<int> left, right;
        left.reserve(static_cast<std::size_t>(nc) + 64);
        right.reserve(static_cast<std::size_t>(nc) + 64);
        int n_slabs = 0;
        for (int b = 0; b < nc;)
        {
            int e = b + 1;
            while (e < nc && geo[4ll * order[e] + 2] == geo[4ll * order[b] + 2] &&
                   geo[4ll * order[e] + 3] == geo[4ll * order[b] + 3])
                ++e;
            ++n_slabs;
            left.push_back(-1);
            right.push_back(order[b]);
            for (int i = b; i + 1 < e; ++i)
            {
                require(std::fabs(geo[4ll * order[i] + 1] - geo[4ll * order[i + 1]]) <= 1e-12, APF_ERR_INVALID,
                        "1+1D estimator: adjacent slab cells are not spatially contiguous");
                left.push_back(order[i]);
                right.push_back(order[i + 1]);
            }
            left.push_back(order[e - 1]);
            right.push_back(-1);
            b = e;
        }
        const int np = static_cast<int>(left.size());
        tot.n_slabs = n_slabs;
        tot.n_patches = np;
        tot.max_patch_cells = nc > 1 ? 2 : 1;
        // ---- lambda~
        DeviceBuffer<double> lt(sp.identity ? nl : 0, s);
        if (sp.identity)
            reconstruct_lambda(s, S, lt, tot);
        else
            reconstruct_lambda_slabs(s, S, sl, lt, tot);
        // ---- nodal data per cell: lambda~ through the slab restriction, lambda_delta and u
        // as the bilinear functions of the cell's Y cell and X ancestor at its corners
        DeviceBuffer<double> ltil(4ll * nc, s), ucell(4ll * nc, s), ldel(4ll * nc, s);
        {
            const SystemInputs& li = sp.identity ? in : sl.in;
            APF_KERNEL("est_gather_nodal", s);
            gather_nodal<<<nb(4ll * nc), 256, 0, s>>>(nc, 4, li.y_off.get(), li.y_dofs.get(), li.y_w.get(), lt.get(),
                                                     nullptr, ltil.get());
        }
        {
            DeviceBuffer<double> ly(4ll * ny, s);
            {
                APF_KERNEL("est_gather_nodal", s);
                gather_nodal<<<nb(4ll * ny), 256, 0, s>>>(ny, 4, in.y_off.get(), in.y_dofs.get(), in.y_w.get(),
                                                         S.solution.get(), nullptr, ly.get());
            }
            if (sp.identity)
                copy(s, 4 * ny, ly.get(), ldel.get());
            else if (nc > 0)
            {
                DeviceBuffer<int> d_src(0, s);
                d_src.upload(sp.source.data(), sp.source.size());
                APF_KERNEL("nodal_transfer", s);
                nodal_transfer_1d_kernel<<<nb(nc), 256, 0, s>>>(nc, cgeo, d_src.get(), in.y_geo.get(), ly.get(),
                                                                ldel.get());
            }
        }
        {
            const int nx = in.n_x_cells;
            DeviceBuffer<double> ux(4ll * nx, s);
            if (nx > 0)
            {
                APF_KERNEL("est_gather_nodal", s);
                gather_nodal<<<nb(4ll * nx), 256, 0, s>>>(nx, 4, in.x_off.get(), in.x_dofs.get(), in.x_w.get(),
                                                         S.solution.get() + nl, nullptr, ux.get());
            }
            if (nc > 0)
            {
                APF_KERNEL("nodal_transfer", s);
                nodal_transfer_1d_kernel<<<nb(nc), 256, 0, s>>>(nc, cgeo, cx, in.x_geo.get(), ux.get(), ucell.get());
            }
        }
        APF_CUDA(cudaGetLastError());
        DeviceBuffer<int> d_left(0, s), d_right(0, s), status(1, s);
        d_left.upload(left.data(), left.size());
        d_right.upload(right.data(), right.size());
        status.zero();
        DeviceBuffer<double> sigma(8ll * nc, s);
        sigma.zero();
        EdgeArgs ea{};
        ea.n_patches = np;
        ea.left = d_left.get();
        ea.right = d_right.get();
        ea.geo = cgeo;
        ea.m = cm;
        ea.ell = cell;
        ea.lt = ltil.get();
        ea.u = ucell.get();
        ea.zero_tol = in.zero_tol;
        ea.sigma = sigma.get();
        ea.status = status.get();
        if (np > 0)
        {
            APF_KERNEL("est_edge_patch_solve", s);
            edge_patch_solve<<<nb(np, 64), 64, 0, s>>>(ea);
        }
        APF_CUDA(cudaGetLastError());
        int hstat = 0;
        APF_CUDA(cudaMemcpyAsync(&hstat, status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        sync(s);
        require(hstat == 0, APF_ERR_NUMERIC, "1+1D estimator: singular patch system");
        DeviceBuffer<double> f2(nc, s), d2(nc, s), r2(nc, s), e2(nc, s);
        EdgeIndArgs ia{};
        ia.n_cells = nc;
        ia.geo = cgeo;
        ia.m = ea.m;
        ia.ell = ea.ell;
        ia.lt = ltil.get();
        ia.u = ucell.get();
        ia.sigma = sigma.get();
        ia.flux = f2.get();
        ia.div = d2.get();
        if (nc > 0)
        {
            APF_KERNEL("est_cell_indicators", s);
            edge_cell_indicators<<<nb(nc, 128), 128, 0, s>>>(ia);
        }
        // ||lambda_delta - lambda~||^2 in the local A_y energy
        if (sp.identity)
        {
            DeviceBuffer<double> dl(nl, s);
            copy(s, nl, S.solution.get(), dl.get());
            axpby(s, nl, -1.0, lt.get(), 1.0, dl.get());
            y_cell_energy(s, in, dl.get(), r2.get());
        }
        else if (nc > 0)
        {
            DeviceBuffer<double> dl(4ll * nc, s);
            copy(s, 4 * nc, ldel.get(), dl.get());
            axpby(s, 4 * nc, -1.0, ltil.get(), 1.0, dl.get());
            APF_KERNEL("nodal_energy", s);
            nodal_energy_1d_kernel<<<nb(nc), 256, 0, s>>>(nc, cgeo, cm, dl.get(), r2.get());
        }
        if (nc > 0)
        {
            APF_KERNEL("est_eta", s);
            add_kernel<<<nb(nc), 256, 0, s>>>(nc, f2.get(), r2.get(), e2.get());
        }
        APF_CUDA(cudaGetLastError());
        if (!sp.identity)
        {
            DeviceBuffer<double> tmp(nc, s);
            for (DeviceBuffer<double>* a : {&f2, &d2, &r2, &e2})
            {
                copy(s, nc, a->get(), tmp.get());
                a->allocate(ny, s);
                if (ny)
                {
                    APF_KERNEL("est_reduce_to_source", s);
                    reduce_to_source_kernel<<<nb(ny), 256, 0, s>>>(ny, sl.src_ptr.get(), sl.src_list.get(), tmp.get(),
                                                                   a->get());
                }
            }
            APF_CUDA(cudaGetLastError());
        }
        tot.flux = device_sum(s, ny, f2.get());
        tot.div = device_sum(s, ny, d2.get());
        tot.recon = device_sum(s, ny, r2.get());
        tot.eta = device_sum(s, ny, e2.get());
        const cudaMemcpyKind kind = out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        if (flux) APF_CUDA(cudaMemcpyAsync(flux, f2.get(), ny * sizeof(double), kind, s));
        if (div) APF_CUDA(cudaMemcpyAsync(div, d2.get(), ny * sizeof(double), kind, s));
        if (recon) APF_CUDA(cudaMemcpyAsync(recon, r2.get(), ny * sizeof(double), kind, s));
        if (eta) APF_CUDA(cudaMemcpyAsync(eta, e2.get(), ny * sizeof(double), kind, s));
        sync(s);
        return tot;
    }
}
