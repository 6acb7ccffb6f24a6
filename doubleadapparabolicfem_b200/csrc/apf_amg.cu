// Smoothed-aggregation AMG (see apf_amg.cuh).
//
// Setup per level: strength graph |a_ij| >= theta sqrt(a_ii a_jj); aggregates from a
// distance-1 maximal independent set (hash priorities, deterministic); tentative
// prolongator T (one 1 per row); P = (I - omega D_F^-1 A_F) T with the filtered
// operator A_F (weak entries lumped onto the diagonal); A_c = P^T A P.  The coarsest
// operator is inverted densely on the host once per setup.  The V-cycle uses the same
// number of damped-Jacobi sweeps before and after the coarse correction, so it is
// symmetric and positive definite.
#include <algorithm>
#include <cmath>
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

        __device__ __forceinline__ double diag_of(const int* rp, const int* ci, const double* va, int r)
        {
            double d = 0.0;
            for (int k = rp[r]; k < rp[r + 1]; ++k)
                if (ci[k] == r)
                    d += va[k];
            return d;
        }

        __global__ void diag_kernel(int n, const int* rp, const int* ci, const double* va, double* d)
        {
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
                d[r] = diag_of(rp, ci, va, r);
        }

        enum : int { UNDECIDED = 0, ROOT = 1, OUT = 2 };

        __global__ void mis_init(int n, const int* rp, const int* ci, const double* va, const double* diag, double theta,
                                 int* state)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                bool any = false;
                for (int k = rp[i]; k < rp[i + 1] && !any; ++k)
                {
                    const int j = ci[k];
                    any = j != i && fabs(va[k]) >= theta * sqrt(fabs(diag[i] * diag[j]));
                }
                state[i] = any ? UNDECIDED : ROOT;
            }
        }

        __global__ void mis_select(int n, const int* rp, const int* ci, const double* va, const double* diag, double theta,
                                   const int* sin, int* sout, int* undecided)
        {
            int cnt = 0;
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                const int st = sin[i];
                if (st != UNDECIDED)
                {
                    sout[i] = st;
                    continue;
                }
                bool is_max = true, has_root = false;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                {
                    const int j = ci[k];
                    if (j == i || fabs(va[k]) < theta * sqrt(fabs(diag[i] * diag[j])))
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

        __global__ void root_flags(int n, const int* state, int* flag)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                flag[i] = state[i] == ROOT;
        }

        // each non-root joins its strongest root neighbour (ties: smallest index)
        __global__ void assign_aggregates(int n, const int* rp, const int* ci, const double* va, const double* diag,
                                          double theta, const int* state, const int* root_pos, int* agg, int* status)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                if (state[i] == ROOT)
                {
                    agg[i] = root_pos[i];
                    continue;
                }
                int best = -1;
                double bv = -1.0;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                {
                    const int j = ci[k];
                    if (j == i || state[j] != ROOT || fabs(va[k]) < theta * sqrt(fabs(diag[i] * diag[j])))
                        continue;
                    const double v = fabs(va[k]);
                    if (v > bv || (v == bv && j < best))
                    {
                        bv = v;
                        best = j;
                    }
                }
                if (best < 0)
                {
                    atomicExch(status, APF_ERR_INTERNAL);
                    agg[i] = 0;
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

        // M = I - omega D_F^-1 A_F restricted to the strong pattern (+ diagonal)
        __global__ void filtered_count(int n, const int* rp, const int* ci, const double* va, const double* diag,
                                       double theta, int* cnt)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                int c = 1;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                {
                    const int j = ci[k];
                    if (j != i && fabs(va[k]) >= theta * sqrt(fabs(diag[i] * diag[j])))
                        ++c;
                }
                cnt[i] = c;
            }
        }

        __global__ void filtered_fill(int n, const int* rp, const int* ci, const double* va, const double* diag,
                                      double theta, double omega, const int* mp, int* mc, double* mv)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                double dF = 0.0;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                {
                    const int j = ci[k];
                    const bool strong = j != i && fabs(va[k]) >= theta * sqrt(fabs(diag[i] * diag[j]));
                    if (!strong)
                        dF += va[k]; // diagonal and lumped weak entries
                }
                const double s = dF != 0.0 ? omega / dF : 0.0;
                int o = mp[i];
                bool diag_done = false;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                {
                    const int j = ci[k];
                    if (!diag_done && j >= i)
                    {
                        mc[o] = i;
                        mv[o] = 1.0 - s * dF;
                        ++o;
                        diag_done = true;
                    }
                    if (j != i && fabs(va[k]) >= theta * sqrt(fabs(diag[i] * diag[j])))
                    {
                        mc[o] = j;
                        mv[o] = -s * va[k];
                        ++o;
                    }
                }
                if (!diag_done)
                {
                    mc[o] = i;
                    mv[o] = 1.0 - s * dF;
                }
            }
        }

        __global__ void scale_kernel(int n, const double* a, const double* d, double* y)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                y[i] = a[i] * d[i];
        }

        __global__ void init_random(int n, double* x)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                x[i] = 0.5 + (hash_u32(static_cast<unsigned>(i) * 2654435761u) & 0xffff) / 65536.0;
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

        int read_int(cudaStream_t s, const int* d)
        {
            int h = 0;
            APF_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, s));
            sync(s);
            return h;
        }

        // rho(D^-1 A) by power iteration
        double spectral_radius(cudaStream_t s, const DeviceCsr& A, const double* dinv, Workspace& w)
        {
            const int n = A.rows;
            DeviceBuffer<double> x(n, s), y(n, s);
            {
                APF_KERNEL("amg_init_random", s);
                init_random<<<nblocks(n, 256), 256, 0, s>>>(n, x.get());
            }
            double lam = 1.0;
            for (int it = 0; it < 12; ++it)
            {
                spmv(s, A, x.get(), y.get());
                {
                    APF_KERNEL("amg_scale", s);
                    scale_kernel<<<nblocks(n, 256), 256, 0, s>>>(n, y.get(), dinv, y.get());
                }
                const double yy = dot_host(s, w, n, y.get(), y.get());
                const double xx = dot_host(s, w, n, x.get(), x.get());
                lam = std::sqrt(yy / std::max(xx, 1e-300));
                axpby(s, n, 1.0 / std::sqrt(std::max(yy, 1e-300)), y.get(), 0.0, x.get());
            }
            return lam;
        }

        // dense SPD inverse via Cholesky (host, coarsest level only)
        void dense_spd_inverse(std::vector<double>& a, int n)
        {
            // a: row-major n x n, overwritten by its inverse
            std::vector<double> L(a);
            for (int j = 0; j < n; ++j)
            {
                double d = L[(size_t)j * n + j];
                for (int k = 0; k < j; ++k)
                    d -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
                if (!(d > 0.0))
                    throw Error(APF_ERR_NUMERIC, "AMG coarsest operator is not positive definite");
                d = std::sqrt(d);
                L[(size_t)j * n + j] = d;
                for (int i = j + 1; i < n; ++i)
                {
                    double v = L[(size_t)i * n + j];
                    const double* li = &L[(size_t)i * n];
                    const double* lj = &L[(size_t)j * n];
                    for (int k = 0; k < j; ++k)
                        v -= li[k] * lj[k];
                    L[(size_t)i * n + j] = v / d;
                }
            }
            // inverse column by column: solve L L^T x = e_c
            std::vector<double> col(n);
            for (int c = 0; c < n; ++c)
            {
                std::fill(col.begin(), col.end(), 0.0);
                col[c] = 1.0;
                for (int i = 0; i < n; ++i)
                {
                    double v = col[i];
                    for (int k = 0; k < i; ++k)
                        v -= L[(size_t)i * n + k] * col[k];
                    col[i] = v / L[(size_t)i * n + i];
                }
                for (int i = n - 1; i >= 0; --i)
                {
                    double v = col[i];
                    for (int k = i + 1; k < n; ++k)
                        v -= L[(size_t)k * n + i] * col[k];
                    col[i] = v / L[(size_t)i * n + i];
                }
                for (int i = 0; i < n; ++i)
                    a[(size_t)i * n + c] = col[i];
            }
        }
    }

    void Amg::setup(cudaStream_t s, const DeviceCsr& A, const AmgOptions& opt, Workspace& w)
    {
        opt_ = opt;
        levels_.clear();
        levels_.reserve(static_cast<std::size_t>(opt.max_levels));
        levels_.emplace_back();
        levels_[0].A = &A;
        w.ensure(s);
        bool force_dense = false;
        for (int l = 0;; ++l)
        {
            AmgLevel& L = levels_[static_cast<std::size_t>(l)];
            const DeviceCsr& Al = *L.A;
            const int n = Al.rows;
            L.x.allocate(n, s);
            L.b.allocate(n, s);
            L.r.allocate(n, s);
            L.t.allocate(n, s);
            if (force_dense || n <= opt.coarse_size || l + 1 >= opt.max_levels)
            {
                // dense inverse of the coarsest operator
                std::vector<int> rp(n + 1), ci(Al.nnz());
                std::vector<double> va(Al.nnz());
                APF_CUDA(cudaMemcpyAsync(rp.data(), Al.row_ptr.get(), (n + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
                if (Al.nnz())
                {
                    APF_CUDA(cudaMemcpyAsync(ci.data(), Al.col_idx.get(), Al.nnz() * sizeof(int), cudaMemcpyDeviceToHost, s));
                    APF_CUDA(cudaMemcpyAsync(va.data(), Al.values.get(), Al.nnz() * sizeof(double), cudaMemcpyDeviceToHost, s));
                }
                sync(s);
                require(n <= 6000, APF_ERR_CAPACITY, "AMG: coarsest level too large for the dense solve");
                std::vector<double> dense((size_t)n * n, 0.0);
                for (int r = 0; r < n; ++r)
                    for (int k = rp[r]; k < rp[r + 1]; ++k)
                        dense[(size_t)r * n + ci[k]] += va[k];
                dense_spd_inverse(dense, n);
                coarse_inv_.allocate(dense.size(), s);
                APF_CUDA(cudaMemcpyAsync(coarse_inv_.get(), dense.data(), dense.size() * sizeof(double),
                                         cudaMemcpyHostToDevice, s));
                sync(s);
                n_coarse_ = n;
                break;
            }
            inverse_diagonal(s, Al, L.dinv);
            DeviceBuffer<double> diag(n, s);
            {
                APF_KERNEL("amg_diag", s);
                diag_kernel<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(), diag.get());
            }
            const double rho = 1.05 * spectral_radius(s, Al, L.dinv.get(), w);
            L.omega = 4.0 / (3.0 * rho);
            // aggregation
            DeviceBuffer<int> st0(n, s), st1(n, s), cnt(1, s);
            {
                APF_KERNEL("amg_mis_init", s);
                mis_init<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(), diag.get(),
                                                         opt.strength, st0.get());
            }
            int* cur = st0.get();
            int* nxt = st1.get();
            for (int it = 0; it < 200; ++it)
            {
                cnt.zero();
                {
                    APF_KERNEL("amg_mis_select", s);
                    mis_select<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(),
                                                               diag.get(), opt.strength, cur, nxt, cnt.get());
                }
                std::swap(cur, nxt);
                if (read_int(s, cnt.get()) == 0)
                    break;
                require(it < 199, APF_ERR_INTERNAL, "AMG: independent-set selection did not finish");
            }
            DeviceBuffer<int> flag(n + 1, s), pos(n + 1, s), agg(n, s), status(1, s);
            status.zero();
            {
                APF_KERNEL("amg_root_flags", s);
                root_flags<<<nblocks(n, 256), 256, 0, s>>>(n, cur, flag.get());
            }
            const int nc = static_cast<int>(exclusive_scan(flag.get(), pos.get(), n, s));
            {
                APF_KERNEL("amg_assign", s);
                assign_aggregates<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(),
                                                                  diag.get(), opt.strength, cur, pos.get(), agg.get(),
                                                                  status.get());
            }
            require(read_int(s, status.get()) == 0, APF_ERR_INTERNAL, "AMG: a node has no aggregate");
            if (nc >= n || nc == 0)
            {
                // no coarsening possible: redo this level as the dense coarsest level
                force_dense = true;
                --l;
                continue;
            }
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
                filtered_count<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(),
                                                               diag.get(), opt.strength, mcnt.get());
            }
            M.row_ptr.allocate(n + 1, s);
            const long long mnnz = exclusive_scan(mcnt.get(), M.row_ptr.get(), n, s);
            M.col_idx.allocate(mnnz, s);
            M.values.allocate(mnnz, s);
            {
                APF_KERNEL("amg_filtered_fill", s);
                filtered_fill<<<nblocks(n, 256), 256, 0, s>>>(n, Al.row_ptr.get(), Al.col_idx.get(), Al.values.get(),
                                                              diag.get(), opt.strength, L.omega, M.row_ptr.get(),
                                                              M.col_idx.get(), M.values.get());
            }
            spgemm(s, M, T, L.P);
            transpose(s, L.P, L.R);
            DeviceCsr AP;
            spgemm(s, Al, L.P, AP);
            levels_.emplace_back();
            AmgLevel& C = levels_.back();
            AmgLevel& Lr = levels_[levels_.size() - 2];
            spgemm(s, Lr.R, AP, C.A_own);
            C.A = &C.A_own;
            sync(s);
        }
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

    void Amg::vcycle(cudaStream_t s, int l, const double* b, double* x)
    {
        AmgLevel& L = levels_[static_cast<std::size_t>(l)];
        const DeviceCsr& A = *L.A;
        const int n = A.rows;
        if (l == static_cast<int>(levels_.size()) - 1)
        {
            APF_KERNEL("amg_coarse_solve", s);
            dense_matvec<<<nblocks((long long)n * 32, 256, 1024), 256, 0, s>>>(n, coarse_inv_.get(), b, x);
            return;
        }
        // pre-smoothing from x = 0
        {
            APF_KERNEL("amg_jacobi_first", s);
            jacobi_first<<<nblocks(n, 256), 256, 0, s>>>(n, b, L.dinv.get(), L.omega, x);
        }
        for (int k = 1; k < opt_.smooth_steps; ++k)
        {
            jacobi_sweep(s, A, x, b, L.dinv.get(), L.omega, L.t.get());
            copy(s, n, L.t.get(), x);
        }
        residual(s, A, x, b, L.r.get());
        AmgLevel& C = levels_[static_cast<std::size_t>(l) + 1];
        spmv(s, L.R, L.r.get(), C.b.get());
        vcycle(s, l + 1, C.b.get(), C.x.get());
        spmv(s, L.P, C.x.get(), x, 1.0, 1.0);
        for (int k = 0; k < opt_.smooth_steps; ++k)
        {
            jacobi_sweep(s, A, x, b, L.dinv.get(), L.omega, L.t.get());
            copy(s, n, L.t.get(), x);
        }
    }

    void Amg::apply(cudaStream_t s, const double* b, double* x)
    {
        vcycle(s, 0, b, x);
    }
}
