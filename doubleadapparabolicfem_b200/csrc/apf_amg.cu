// Smoothed-aggregation AMG (see apf_amg.cuh).
//
// Setup per level: strength graph |a_ij| >= theta sqrt(a_ii a_jj) between unknowns of the
// same component (the time-local index of a Y DOF: the broken-in-time test space makes
// (1,-1) across the two time sides of a node a lower-energy mode than the constant, so the
// sides are aggregated separately and each keeps its own constant near-nullspace vector);
// aggregates from a distance-1 maximal independent set (hash priorities, deterministic; a
// level whose strong graph no longer coarsens -- coefficient jumps cut it into small pieces --
// is aggregated again with every coupling inside a component counted as strong);
// tentative prolongator T (one 1 per row); P = (I - omega D_F^-1 A_F) T with the filtered
// operator A_F (weak entries lumped onto the diagonal); A_c = P^T A P.  The coarsest
// operator is inverted densely on the device once per setup (Gauss-Jordan, one launch per
// pivot; or, when coarsening stalls above the dense size, smoothed with a fixed number of
// Jacobi sweeps).  The V-cycle uses
// the same damped-Jacobi sweeps before and after the coarse correction, so it is a
// symmetric positive definite linear operator.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "apf_amg.cuh"

namespace apf
{
    namespace
    {
        int nblocks(long long work, int threads, int cap = 148 * 32)
        {
            long long g = (work + threads - 1) / threads;
            return static_cast<int>(std::max<long long>(1, std::min<long long>(g, cap)));
        }

        __device__ __forceinline__ unsigned hash_u32(unsigned x)
        {
            x ^= x >> 16; x *= 0x7feb352dU;
            x ^= x >> 15; x *= 0x846ca68bU;
            x ^= x >> 16;
            return x;
        }
        __device__ __forceinline__ bool higher(int i, int j)
        {
            const unsigned hi = hash_u32(static_cast<unsigned>(i)), hj = hash_u32(static_cast<unsigned>(j));
            return hi > hj || (hi == hj && i > j);
        }

        struct Strength
        {
            const double* diag;
            double theta;
            const int* comp; // optional component of each unknown
            __device__ __forceinline__ bool operator()(int i, int j, double v) const
            {
                return j != i && (comp == nullptr || comp[i] == comp[j]) &&
                       fabs(v) >= theta * sqrt(fabs(diag[i] * diag[j]));
            }
        };

        __global__ void diag_kernel(int n, const int* rp, const int* ci, const double* va, double* d)
        {
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
            {
                double s = 0.0;
                for (int k = rp[r]; k < rp[r + 1]; ++k)
                    if (ci[k] == r)
                        s += va[k];
                d[r] = s;
            }
        }

        enum : int { UNDECIDED = 0, ROOT = 1, OUT = 2 };

        __global__ void mis_init(int n, const int* rp, const int* ci, const double* va, Strength st, int* state)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                bool any = false;
                for (int k = rp[i]; k < rp[i + 1] && !any; ++k)
                    any = st(i, ci[k], va[k]);
                state[i] = any ? UNDECIDED : ROOT;
            }
        }

        __global__ void mis_select(int n, const int* rp, const int* ci, const double* va, Strength st, const int* sin,
                                   int* sout, int* undecided)
        {
            int cnt = 0;
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                const int s0 = sin[i];
                if (s0 != UNDECIDED)
                {
                    sout[i] = s0;
                    continue;
                }
                bool is_max = true, has_root = false;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                {
                    const int j = ci[k];
                    if (!st(i, j, va[k]))
                        continue;
                    const int sj = sin[j];
                    if (sj == ROOT)
                        has_root = true;
                    else if (sj == UNDECIDED && higher(j, i))
                        is_max = false;
                }
                const int ns = has_root ? OUT : (is_max ? ROOT : UNDECIDED);
                sout[i] = ns;
                cnt += ns == UNDECIDED;
            }
            for (int o = 16; o > 0; o >>= 1)
                cnt += __shfl_down_sync(0xffffffffu, cnt, o);
            if ((threadIdx.x & 31) == 0 && cnt)
                atomicAdd(undecided, cnt);
        }

        // candidate (v, j) beats (bv, best): larger magnitude, values within a relative 1e-10
        // counting as equal (ties: smaller index), so that rounding-level differences between
        // couplings that are equal in exact arithmetic do not change the aggregates
        __device__ __forceinline__ bool stronger(double v, int j, double bv, int best)
        {
            if (best < 0)
                return true;
            const double tol = 1e-10 * fmax(v, bv);
            if (v > bv + tol)
                return true;
            return v >= bv - tol && j < best;
        }

        // distance-2 independent set (aggressive coarsening): a node is a root when its
        // priority key is the largest among the undecided nodes within two strong edges, out
        // when a root lies within two strong edges.  Pass A: per node, the largest undecided
        // key and whether a root is among itself and its strong neighbours; pass B: the same
        // over the strong neighbours' pass-A values.
        __device__ __forceinline__ unsigned long long mis_key(int i)
        {
            return (static_cast<unsigned long long>(hash_u32(static_cast<unsigned>(i))) << 32) | static_cast<unsigned>(i);
        }

        __global__ void mis2_pass_a(int n, const int* rp, const int* ci, const double* va, Strength st, const int* state,
                                    unsigned long long* m1, int* r1)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                unsigned long long m = state[i] == UNDECIDED ? mis_key(i) : 0ull;
                int r = state[i] == ROOT;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                {
                    const int j = ci[k];
                    if (!st(i, j, va[k]))
                        continue;
                    const int sj = state[j];
                    if (sj == UNDECIDED)
                        m = max(m, mis_key(j));
                    r |= sj == ROOT;
                }
                m1[i] = m;
                r1[i] = r;
            }
        }

        __global__ void mis2_pass_b(int n, const int* rp, const int* ci, const double* va, Strength st, const int* sin,
                                    const unsigned long long* m1, const int* r1, int* sout, int* undecided)
        {
            int cnt = 0;
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                const int s0 = sin[i];
                if (s0 != UNDECIDED)
                {
                    sout[i] = s0;
                    continue;
                }
                unsigned long long m = m1[i];
                int r = r1[i];
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                {
                    const int j = ci[k];
                    if (!st(i, j, va[k]))
                        continue;
                    m = max(m, m1[j]);
                    r |= r1[j];
                }
                const int ns = r ? OUT : (m == mis_key(i) ? ROOT : UNDECIDED);
                sout[i] = ns;
                cnt += ns == UNDECIDED;
            }
            for (int o = 16; o > 0; o >>= 1)
                cnt += __shfl_down_sync(0xffffffffu, cnt, o);
            if ((threadIdx.x & 31) == 0 && cnt)
                atomicAdd(undecided, cnt);
        }

        // second aggregation pass after distance-2 selection: a node without a strong root
        // neighbour joins the aggregate of its strongest assigned neighbour (ties: smallest
        // index); agg_in holds the first pass (-1: unassigned)
        __global__ void assign_aggregates2(int n, const int* rp, const int* ci, const double* va, Strength st,
                                           const int* agg_in, int* agg_out, int* status)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                if (agg_in[i] >= 0)
                {
                    agg_out[i] = agg_in[i];
                    continue;
                }
                int best = -1;
                double bv = -1.0;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                {
                    const int j = ci[k];
                    if (agg_in[j] < 0 || !st(i, j, va[k]))
                        continue;
                    const double v = fabs(va[k]);
                    if (stronger(v, j, bv, best))
                    {
                        bv = v;
                        best = j;
                    }
                }
                if (best < 0)
                {
                    atomicExch(status, APF_ERR_INTERNAL);
                    agg_out[i] = 0;
                }
                else
                    agg_out[i] = agg_in[best];
            }
        }

        __global__ void root_flags(int n, const int* state, int* flag)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                flag[i] = state[i] == ROOT;
        }

        // each non-root joins its strongest root neighbour (ties: smallest index)
        __global__ void assign_aggregates(int n, const int* rp, const int* ci, const double* va, Strength st,
                                          const int* state, const int* root_pos, int* agg, int* comp_coarse, int* status,
                                          bool allow_unassigned)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                if (state[i] == ROOT)
                {
                    agg[i] = root_pos[i];
                    if (comp_coarse)
                        comp_coarse[root_pos[i]] = st.comp ? st.comp[i] : 0;
                    continue;
                }
                int best = -1;
                double bv = -1.0;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                {
                    const int j = ci[k];
                    if (state[j] != ROOT || !st(i, j, va[k]))
                        continue;
                    const double v = fabs(va[k]);
                    if (stronger(v, j, bv, best))
                    {
                        bv = v;
                        best = j;
                    }
                }
                if (best < 0)
                {
                    if (!allow_unassigned)
                        atomicExch(status, APF_ERR_INTERNAL);
                    agg[i] = allow_unassigned ? -1 : 0;
                }
                else
                    agg[i] = root_pos[best];
            }
        }

        __global__ void tentative_fill(int n, const int* agg, int* rp, int* ci, double* va)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                rp[i] = i;
                ci[i] = agg[i];
                va[i] = 1.0;
                if (i == n - 1)
                    rp[n] = n;
            }
        }

        // M = I - omega D_F^-1 A_F on the strong pattern (+ diagonal)
        __global__ void filtered_count(int n, const int* rp, const int* ci, const double* va, Strength st, int* cnt)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                int c = 1;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                    c += st(i, ci[k], va[k]);
                cnt[i] = c;
            }
        }

        __global__ void filtered_fill(int n, const int* rp, const int* ci, const double* va, Strength st, double omega,
                                      const int* mp, int* mc, double* mv)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                double dF = 0.0;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                    if (!st(i, ci[k], va[k]))
                        dF += va[k]; // diagonal and lumped weak entries
                // lumping positive weak couplings can shrink the diagonal; keep it well away from 0
                const double dii = st.diag[i];
                if (!(dF >= 0.25 * dii))
                    dF = dii;
                const double s = dF != 0.0 ? omega / dF : 0.0;
                int o = mp[i];
                bool diag_done = false;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                {
                    const int j = ci[k];
                    if (!diag_done && j >= i)
                    {
                        mc[o] = i;
                        mv[o] = 1.0 - omega;
                        ++o;
                        diag_done = true;
                    }
                    if (st(i, j, va[k]))
                    {
                        mc[o] = j;
                        mv[o] = -s * va[k];
                        ++o;
                    }
                }
                if (!diag_done)
                {
                    mc[o] = i;
                    mv[o] = 1.0 - omega;
                }
            }
        }

        // kernel-timer names per operation and level (levels above 5 share one name)
        const char* level_name(int op, int l)
        {
            static const char* names[4][7] = {
                {"amg_sweep_l0", "amg_sweep_l1", "amg_sweep_l2", "amg_sweep_l3", "amg_sweep_l4", "amg_sweep_l5",
                 "amg_sweep_l6+"},
                {"amg_residual_l0", "amg_residual_l1", "amg_residual_l2", "amg_residual_l3", "amg_residual_l4",
                 "amg_residual_l5", "amg_residual_l6+"},
                {"amg_restrict_l0", "amg_restrict_l1", "amg_restrict_l2", "amg_restrict_l3", "amg_restrict_l4",
                 "amg_restrict_l5", "amg_restrict_l6+"},
                {"amg_prolong_l0", "amg_prolong_l1", "amg_prolong_l2", "amg_prolong_l3", "amg_prolong_l4",
                 "amg_prolong_l5", "amg_prolong_l6+"}};
            return names[op][l < 6 ? l : 6];
        }

        __global__ void jacobi_first(int n, const double* b, const double* dinv, double omega, double* x)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                x[i] = omega * dinv[i] * b[i];
        }

        // x = Cinv b, Cinv dense row-major n x n; one warp per row
        __global__ void dense_matvec(int n, const double* __restrict__ Cinv, const double* __restrict__ b, double* __restrict__ x)
        {
            const int lane = threadIdx.x & 31;
            const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            const int nw = (gridDim.x * blockDim.x) >> 5;
            for (int r = w; r < n; r += nw)
            {
                double s = 0.0;
                for (int k = lane; k < n; k += 32)
                    s += Cinv[(long long)r * n + k] * b[k];
                for (int o = 16; o > 0; o >>= 1)
                    s += __shfl_down_sync(0xffffffffu, s, o);
                if (lane == 0)
                    x[r] = s;
            }
        }

        // Gershgorin bound of rho(D^-1 A): max_i sum_j |a_ij| / a_ii (an upper bound, so the
        // damped-Jacobi factor 4 / (3 rho) keeps every sweep contractive and the V-cycle SPD)
        __global__ void gershgorin_kernel(int n, const int* rp, const int* ci, const double* va, unsigned long long* out)
        {
            double m = 0.0;
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
            {
                double d = 0.0, s = 0.0;
                for (int k = rp[r]; k < rp[r + 1]; ++k)
                {
                    s += fabs(va[k]);
                    if (ci[k] == r)
                        d += va[k];
                }
                if (d > 0.0)
                    m = fmax(m, s / d);
            }
            for (int o = 16; o > 0; o >>= 1)
                m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
            if ((threadIdx.x & 31) == 0)
                atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(m))); // non-negative doubles order like their bits
        }

        int read_int(cudaStream_t s, const int* d)
        {
            int h = 0;
            APF_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, s));
            sync(s);
            return h;
        }

        double spectral_radius(cudaStream_t s, const DeviceCsr& A)
        {
            DeviceBuffer<unsigned long long> out(1, s);
            out.zero();
            {
                APF_KERNEL("amg_gershgorin", s);
                gershgorin_kernel<<<nblocks(A.rows, 256, 1024), 256, 0, s>>>(A.rows, A.row_ptr.get(), A.col_idx.get(),
                                                                              A.values.get(), out.get());
            }
            unsigned long long h = 0;
            APF_CUDA(cudaMemcpyAsync(&h, out.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
            sync(s);
            double r;
            std::memcpy(&r, &h, sizeof(r));
            return r > 0.0 ? r : 1.0;
        }

        // coarsest operator scattered into a zeroed dense row-major n x n array (one thread per row)
        __global__ void csr_to_dense(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                     const double* __restrict__ va, double* __restrict__ D)
        {
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
                for (int k = rp[r]; k < rp[r + 1]; ++k)
                    D[(long long)r * n + ci[k]] += va[k];
        }

        // One Gauss-Jordan exchange step on pivot k (B from A, out of place): after the steps
        // k = 0..n-1 the array holds A^-1.  An SPD matrix needs no pivoting (every pivot is a
        // diagonal entry of a Schur complement, hence positive); a pivot that is not positive
        // and finite sets *status and the step leaves B = A.
        // C = (C + C^T) / 2 for a dense n x n row-major matrix: the inverse of a symmetric matrix
        // computed in finite precision is symmetric only up to cond(A) eps, and the coarse
        // solve must be exactly symmetric for the V-cycle to stay a symmetric operator
        __global__ void symmetrize_dense(int n, double* __restrict__ C)
        {
            const long long total = static_cast<long long>(n) * n;
            for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
                 e += (long long)gridDim.x * blockDim.x)
            {
                const int i = static_cast<int>(e / n), j = static_cast<int>(e % n);
                if (j <= i)
                    continue;
                const double v = 0.5 * (C[(long long)i * n + j] + C[(long long)j * n + i]);
                C[(long long)i * n + j] = v;
                C[(long long)j * n + i] = v;
            }
        }

        __global__ void gauss_jordan_step(int n, int k, const double* __restrict__ A, double* __restrict__ B,
                                          int* __restrict__ status)
        {
            const double p = A[(long long)k * n + k];
            const bool ok = p > 0.0 && isfinite(p);
            if (!ok && blockIdx.x == 0 && threadIdx.x == 0)
                *status = 1;
            const double ip = ok ? 1.0 / p : 0.0;
            const long long total = (long long)n * n;
            for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
                 t += (long long)gridDim.x * blockDim.x)
            {
                const int i = static_cast<int>(t / n), j = static_cast<int>(t % n);
                const double a = A[t];
                double v;
                if (!ok)
                    v = a;
                else if (i == k && j == k)
                    v = ip;
                else if (i == k)
                    v = -a * ip;
                else if (j == k)
                    v = a * ip;
                else
                    v = a - A[(long long)i * n + k] * A[(long long)k * n + j] * ip;
                B[t] = v;
            }
        }
    }

    void Amg::setup(cudaStream_t s, const DeviceCsr& A, const AmgOptions& opt, Workspace& w, const int* component)
    {
        opt_ = opt;
        levels_.clear();
        levels_.reserve(static_cast<std::size_t>(opt.max_levels));
        levels_.emplace_back();
        levels_[0].A = &A;
        if (component)
        {
            levels_[0].comp.allocate(static_cast<std::size_t>(A.rows), s);
            APF_CUDA(cudaMemcpyAsync(levels_[0].comp.get(), component, A.rows * sizeof(int), cudaMemcpyDeviceToDevice, s));
        }
        w.ensure(s);
        bool force_dense = false, force_jacobi = false;
        // a level whose strong graph no longer coarsens (coefficient jumps split it into many
        // small pieces) is aggregated once more with every coupling of its component strong
        bool weak_retry = false;
        jacobi_coarse_ = false;
        for (int l = 0;; ++l)
        {
            AmgLevel& L = levels_[static_cast<std::size_t>(l)];
            const DeviceCsr& Al = *L.A;
            const int n = Al.rows;
            L.x.allocate(n, s);
            L.b.allocate(n, s);
            L.r.allocate(n, s);
            L.t.allocate(n, s);
            if (!force_dense && n > opt.coarse_size && l + 1 >= opt.max_levels)
                force_jacobi = true;
            if (force_jacobi)
            {
                // coarsest level too large for a dense solve: a fixed number of damped-Jacobi
                // sweeps from zero (a symmetric positive definite polynomial in D^-1 A)
                inverse_diagonal(s, Al, L.dinv);
                L.omega = 4.0 / (3.0 * spectral_radius(s, Al));
                jacobi_coarse_ = true;
                n_coarse_ = n;
                break;
            }
            if (force_dense || n <= opt.coarse_size)
            {
                // the level's diagonal and damping too, so every level carries the same data
                // for inspection (the dense solve itself needs neither)
                if (L.dinv.size() != static_cast<std::size_t>(n))
                {
                    inverse_diagonal(s, Al, L.dinv);
                    L.omega = 4.0 / (3.0 * spectral_radius(s, Al));
                }
                // dense inverse on the device: scatter, then n Gauss-Jordan exchange steps
                const std::size_t nn = static_cast<std::size_t>(n) * n;
                coarse_inv_.allocate(nn, s);
                coarse_inv_.zero();
                DeviceBuffer<double> other(nn, s);
                DeviceBuffer<int> status(1, s);
                status.zero();
                {
                    APF_KERNEL("amg_coarse_dense", s);
                    csr_to_dense<<<nblocks(n, 128), 128, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(),
                                                                 coarse_inv_.get());
                }
                double* cur = coarse_inv_.get();
                double* nxt = other.get();
                const int gj_blocks = nblocks(static_cast<long long>(nn), 256, 148 * 8);
                for (int k = 0; k < n; ++k)
                {
                    {
                        APF_KERNEL("amg_coarse_gauss_jordan", s);
                        gauss_jordan_step<<<gj_blocks, 256, 0, s>>>(n, k, cur, nxt, status.get());
                    }
                    std::swap(cur, nxt);
                }
                if (cur != coarse_inv_.get())
                    APF_CUDA(cudaMemcpyAsync(coarse_inv_.get(), cur, nn * sizeof(double), cudaMemcpyDeviceToDevice, s));
                {
                    APF_KERNEL("amg_coarse_symmetrize", s);
                    symmetrize_dense<<<gj_blocks, 256, 0, s>>>(n, coarse_inv_.get());
                }
                APF_CUDA(cudaGetLastError());
                int bad = 0;
                APF_CUDA(cudaMemcpyAsync(&bad, status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
                sync(s);
                require(bad == 0, APF_ERR_NUMERIC, "AMG coarsest operator is not positive definite");
                n_coarse_ = n;
                break;
            }
            inverse_diagonal(s, Al, L.dinv);
            DeviceBuffer<double> diag(n, s);
            {
                APF_KERNEL("amg_diag", s);
                diag_kernel<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(), diag.get());
            }
            L.omega = 4.0 / (3.0 * spectral_radius(s, Al));
            const Strength st{diag.get(), weak_retry ? 0.0 : opt.strength, L.comp.size() ? L.comp.get() : nullptr};
            // aggregation
            DeviceBuffer<int> st0(n, s), st1(n, s), cnt(1, s);
            {
                APF_KERNEL("amg_mis_init", s);
                mis_init<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(), st, st0.get());
            }
            int* cur = st0.get();
            int* nxt = st1.get();
            const bool aggressive = l < opt.aggressive_levels;
            DeviceBuffer<unsigned long long> m1(aggressive ? n : 1, s);
            DeviceBuffer<int> r1(aggressive ? n : 1, s);
            for (int it = 0;; ++it)
            {
                require(it < 200, APF_ERR_INTERNAL, "AMG: independent-set selection did not finish");
                cnt.zero();
                if (aggressive)
                {
                    {
                        APF_KERNEL("amg_mis_select", s);
                        mis2_pass_a<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(),
                                                                    Al.values.get(), st, cur, m1.get(), r1.get());
                    }
                    APF_KERNEL("amg_mis_select", s);
                    mis2_pass_b<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(), st,
                                                                cur, m1.get(), r1.get(), nxt, cnt.get());
                }
                else
                {
                    APF_KERNEL("amg_mis_select", s);
                    mis_select<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(), st,
                                                               cur, nxt, cnt.get());
                }
                std::swap(cur, nxt);
                if (read_int(s, cnt.get()) == 0)
                    break;
            }
            DeviceBuffer<int> flag(n + 1, s), pos(n + 1, s), agg(n, s), status(1, s);
            status.zero();
            {
                APF_KERNEL("amg_root_flags", s);
                root_flags<<<nblocks(n, 256), 256, 0, s>>>(n, cur, flag.get());
            }
            const int nc = static_cast<int>(exclusive_scan(flag.get(), pos.get(), n, s));
            if (nc == 0 || nc > (4 * static_cast<long long>(n)) / 5)
            {
                if (!weak_retry && opt.strength > 0.0 && n > kMaxDense)
                {
                    weak_retry = true;
                    --l;
                    continue;
                }
                weak_retry = false;
                // coarsening stalls: this level becomes the coarsest one
                if (n <= kMaxDense)
                    force_dense = true;
                else
                    force_jacobi = true;
                --l;
                continue;
            }
            weak_retry = false; // the next level starts from the configured strength again
            DeviceBuffer<int> comp_c;
            if (st.comp)
                comp_c.allocate(nc, s);
            {
                APF_KERNEL("amg_assign", s);
                assign_aggregates<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(), st,
                                                                  cur, pos.get(), agg.get(),
                                                                  st.comp ? comp_c.get() : nullptr, status.get(), aggressive);
            }
            if (aggressive)
            {
                DeviceBuffer<int> agg2(n, s);
                {
                    APF_KERNEL("amg_assign", s);
                    assign_aggregates2<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(),
                                                                       Al.values.get(), st, agg.get(), agg2.get(),
                                                                       status.get());
                }
                agg = std::move(agg2);
            }
            require(read_int(s, status.get()) == 0, APF_ERR_INTERNAL, "AMG: a node has no aggregate");
            // tentative prolongator
            DeviceCsr T;
            T.rows = n;
            T.cols = nc;
            T.row_ptr.allocate(n + 1, s);
            T.col_idx.allocate(n, s);
            T.values.allocate(n, s);
            {
                APF_KERNEL("amg_tentative", s);
                tentative_fill<<<nblocks(n, 256), 256, 0, s>>>(n, agg.get(), T.row_ptr.get(), T.col_idx.get(), T.values.get());
            }
            // M = I - omega D_F^-1 A_F; P = M T
            DeviceCsr M;
            M.rows = M.cols = n;
            DeviceBuffer<int> mcnt(n + 1, s);
            {
                APF_KERNEL("amg_filtered_count", s);
                filtered_count<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(), st,
                                                               mcnt.get());
            }
            M.row_ptr.allocate(n + 1, s);
            const long long mnnz = exclusive_scan(mcnt.get(), M.row_ptr.get(), n, s);
            M.col_idx.allocate(mnnz, s);
            M.values.allocate(mnnz, s);
            {
                APF_KERNEL("amg_filtered_fill", s);
                filtered_fill<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(), st,
                                                              L.omega, M.row_ptr.get(), M.col_idx.get(), M.values.get());
            }
            DeviceCsr Ac;
            try
            {
                spgemm(s, M, T, L.P);
                transpose(s, L.P, L.R);
                DeviceCsr AP;
                spgemm(s, Al, L.P, AP);
                spgemm(s, L.R, AP, Ac);
            }
            catch (const Error& e)
            {
                if (e.code != APF_ERR_CAPACITY)
                    throw;
                // the Galerkin product got too dense: stop coarsening at this level
                L.P = DeviceCsr{};
                L.R = DeviceCsr{};
                if (n <= kMaxDense)
                    force_dense = true;
                else
                    force_jacobi = true;
                --l;
                continue;
            }
            levels_.emplace_back();
            AmgLevel& C = levels_.back();
            C.A_own = std::move(Ac);
            C.A = &C.A_own;
            if (comp_c.size())
                C.comp = std::move(comp_c);
            sync(s);
        }
        // f32 sliced-ELLPACK copies of the V-cycle operators: the V-cycle reads its matrices
        // 5 to 10 times per application, and f32 values (symmetric rounding, f64 products and
        // accumulation) cut those reads by a third while keeping the preconditioner a fixed
        // symmetric operator
        for (std::size_t l = 0; l < levels_.size(); ++l)
        {
            AmgLevel& L = levels_[l];
            if (!(l + 1 == levels_.size() && !jacobi_coarse_))
                L.A32 = make_sell32(s, *L.A);
            if (L.P.rows)
            {
                L.P32 = make_sell32(s, L.P);
                L.R32 = make_sell32(s, L.R);
            }
        }
        sync(s);
    }

    long long Amg::operator_nnz() const
    {
        long long t = 0;
        for (const auto& L : levels_)
            t += L.A ? L.A->nnz() : 0;
        return t;
    }

    std::vector<int> Amg::level_rows() const
    {
        std::vector<int> r;
        for (const auto& L : levels_)
            r.push_back(L.A ? L.A->rows : 0);
        return r;
    }

    // where level l's first smoothing iterate goes: x or the scratch t, chosen so that the
    // last of its pre + post sweeps writes x
    double* Amg::first_iterate(int l, double* x)
    {
        AmgLevel& L = levels_[static_cast<std::size_t>(l)];
        const bool coarsest = l == static_cast<int>(levels_.size()) - 1;
        const int pre = coarsest ? kCoarseSweeps : opt_.smooth_steps;
        const int post = coarsest ? 0 : opt_.smooth_steps;
        return (pre + post) % 2 == 1 ? x : L.t.get();
    }

    void Amg::vcycle(cudaStream_t s, int l, const double* b, double* x, bool first_done)
    {
        AmgLevel& L = levels_[static_cast<std::size_t>(l)];
        const DeviceCsr& A = *L.A;
        const int n = A.rows;
        const bool coarsest = l == static_cast<int>(levels_.size()) - 1;
        if (coarsest && !jacobi_coarse_)
        {
            APF_KERNEL("amg_coarse_solve", s);
            dense_matvec<<<nblocks((long long)n * 32, 256, 1024), 256, 0, s>>>(n, coarse_inv_.get(), b, x);
            return;
        }
        const int pre = coarsest ? kCoarseSweeps : opt_.smooth_steps;
        const int post = coarsest ? 0 : opt_.smooth_steps;
        // smoother weights: omega D^-1 (plain) or the level's per-row weights, one vector
        // for the first pre-smoothing sweep and one for the later sweeps; post-smoothing
        // applies the pre-smoothing weights in reverse order
        const bool own = L.w.size() != 0;
        const double om = own ? 1.0 : L.omega;
        auto weights = [&](int sweep) -> const double* {
            if (!own)
                return L.dinv.get();
            return sweep == 0 || L.w2.size() == 0 ? L.w.get() : L.w2.get();
        };
        // the iterate alternates between x and the level's scratch t; starting in the right
        // one makes the last of the pre + post smoothing writes land in x (no copies)
        double* cur = first_iterate(l, x);
        double* other = cur == x ? L.t.get() : x;
        if (!first_done)
        {
            APF_KERNEL("amg_jacobi_first", s);
            jacobi_first<<<nblocks(n, 256), 256, 0, s>>>(n, b, weights(0), om, cur);
        }
        const DeviceSell& A32 = *L.A32;
        for (int k = 1; k < pre; ++k)
        {
            jacobi_sweep(s, A32, cur, b, weights(k), om, other, coarsest ? "amg_coarse_sweep" : level_name(0, l));
            std::swap(cur, other);
        }
        if (coarsest)
            return;
        residual(s, A32, cur, b, L.r.get(), level_name(1, l));
        AmgLevel& C = levels_[static_cast<std::size_t>(l) + 1];
        const bool c_dense = l + 2 == static_cast<int>(levels_.size()) && !jacobi_coarse_;
        if (c_dense)
        {
            spmv(s, *L.R32, L.r.get(), C.b.get(), 1.0, 0.0, level_name(2, l));
            vcycle(s, l + 1, C.b.get(), C.x.get());
        }
        else
        {
            // restriction fused with the coarse level's first damped-Jacobi step from zero
            const bool cown = C.w.size() != 0;
            spmv_jacobi_first(s, *L.R32, L.r.get(), C.b.get(), cown ? C.w.get() : C.dinv.get(),
                              cown ? 1.0 : C.omega, first_iterate(l + 1, C.x.get()), level_name(2, l));
            vcycle(s, l + 1, C.b.get(), C.x.get(), true);
        }
        spmv(s, *L.P32, C.x.get(), cur, L.alpha, 1.0, level_name(3, l));
        for (int k = 0; k < post; ++k)
        {
            jacobi_sweep(s, A32, cur, b, weights(post - 1 - k), om, other, level_name(0, l));
            std::swap(cur, other);
        }
    }

    void Amg::set_smoother(int l, DeviceBuffer<double>&& w, DeviceBuffer<double>&& w2, double alpha)
    {
        require(l >= 0 && l < levels(), APF_ERR_INVALID, "AMG: no such level");
        AmgLevel& L = levels_[static_cast<std::size_t>(l)];
        const auto rows = static_cast<std::size_t>(L.A->rows);
        require((w.size() == 0 || w.size() == rows) && (w2.size() == 0 || w2.size() == rows) &&
                    !(w.size() == 0 && w2.size() != 0),
                APF_ERR_INVALID, "AMG: smoother weights of the wrong size");
        L.w = std::move(w);
        L.w2 = std::move(w2);
        L.alpha = alpha;
    }

    void Amg::reset_smoothers()
    {
        for (auto& L : levels_)
        {
            L.w.release();
            L.w2.release();
            L.alpha = 1.0;
        }
    }

    void Amg::apply(cudaStream_t s, const double* b, double* x)
    {
        vcycle(s, 0, b, x);
    }
}
