// Block-preconditioned MINRES on the device.
//
// Restates the reference's solve path (src/linear_algebra/eigen_backend/preconditioners/
// parabolic_graph_norm_minres.hpp:232-369 with iterative_residual_acceptance.hpp:118-216):
//   * preconditioned MINRES (Paige & Saunders 1975, Lanczos form) on K = [A_y B^T; B C];
//   * block preconditioner P = blkdiag(A_y, Hhat): the reference factors both blocks with a
//     sparse Cholesky; here each block is applied as one symmetric smoothed-aggregation
//     AMG V-cycle (a fixed SPD operator), or the learned preconditioner built on it;
//   * backend stopping test ||r_0|| phibar_k / beta_1 < tol ||b||;
//   * batches of `true_residual_check_interval` iterations; after each batch the FP64
//     true residual ||K x - b|| / ||b|| accepts; if the backend had converged but the
//     true residual did not, the backend tolerance is multiplied by 0.1 (floor
//     max(eps, tol sqrt(eps))); the batch restarts from the current iterate (stacked
//     problems: a restart that needs no iteration tightens the tolerance again).
// All Lanczos scalars live in device memory; the host only reads the status every
// `kCheckEvery` iterations, so iterations run back to back on the stream.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <limits>

#include "apf_minres.cuh"

namespace apf
{
    namespace
    {
        struct MinresDev
        {
            double beta, oldb, alfa, dbar, epsln, phibar, cs, sn, gamma, delta, phi, oldeps;
            double beta1, r0n, bn, tol, err, bb;
            int done, bad, its, pad;
        };

        constexpr int kThreads = 256;
        constexpr int kCheckEvery = 8;

        int nb(long long n)
        {
            return static_cast<int>(std::max<long long>(1, std::min<long long>((n + kThreads - 1) / kThreads, kRedBlocks)));
        }

        __device__ __forceinline__ double block_sum(double v)
        {
            __shared__ double ws[kThreads / 32];
            for (int o = 16; o > 0; o >>= 1)
                v += __shfl_down_sync(0xffffffffu, v, o);
            if ((threadIdx.x & 31) == 0)
                ws[threadIdx.x >> 5] = v;
            __syncthreads();
            double t = 0.0;
            if (threadIdx.x == 0)
                for (int w = 0; w < kThreads / 32; ++w)
                    t += ws[w];
            return t;
        }

        // One MINRES iteration as a CUDA graph: its ~100 launches (Lanczos step, K SpMV,
        // both V-cycles on their two streams) are replayed with one launch.  The three
        // Lanczos vectors rotate with period 3, so a solve needs at most four graphs
        // (first iteration + three rotation phases).
        struct IterationGraph
        {
            cudaGraphExec_t exec = nullptr;
            long long kernels = 0;
            int batch = -1;
            ~IterationGraph()
            {
                if (exec)
                    cudaGraphExecDestroy(exec);
            }
            void reset()
            {
                if (exec)
                    cudaGraphExecDestroy(exec);
                exec = nullptr;
                kernels = 0;
                batch = -1;
            }
        };

        // Capture `body` (launches on s and streams forked from it) into g.
        template<class F>
        void capture_iteration(cudaStream_t s, IterationGraph& g, F&& body)
        {
            g.reset();
            const long long before = g_kernel_launches.load();
            APF_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            try
            {
                body();
            }
            catch (...)
            {
                cudaGraph_t partial = nullptr;
                cudaStreamEndCapture(s, &partial);
                if (partial)
                    cudaGraphDestroy(partial);
                cudaGetLastError();
                throw;
            }
            cudaGraph_t graph = nullptr;
            APF_CUDA(cudaStreamEndCapture(s, &graph));
            g.kernels = g_kernel_launches.load() - before;
            g_kernel_launches.fetch_sub(g.kernels);
            const cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
            cudaGraphDestroy(graph);
            APF_CUDA(e);
        }

        // Graphs are used unless per-launch event timing is on (the events bracket single
        // launches) or the caller's stream is the legacy default stream (not capturable).
        bool graphs_enabled(cudaStream_t s)
        {
            if (s == nullptr || s == cudaStreamLegacy)
                return false;
            return !(t_profiler && t_profiler->enabled && t_profiler->kernels);
        }

        // sum of squares of v over each segment (one block per segment, fixed order)
        __global__ void k_segment_sumsq(const int2* __restrict__ segs, const double* __restrict__ v,
                                        double* __restrict__ out)
        {
            const int2 r = segs[blockIdx.x];
            double acc = 0.0;
            for (int i = r.x + threadIdx.x; i < r.y; i += blockDim.x)
                acc += v[i] * v[i];
            const double t = block_sum(acc);
            if (threadIdx.x == 0)
                out[blockIdx.x] = t;
        }

        std::vector<double> part_norms2(cudaStream_t s, const Partition& P, const double* v, DeviceBuffer<double>& tmp)
        {
            const int nseg = 2 * P.n_parts;
            std::vector<double> seg(static_cast<std::size_t>(nseg)), out(static_cast<std::size_t>(P.n_parts));
            if (nseg == 0)
                return out;
            {
                APF_KERNEL("minres_part_norms", s);
                k_segment_sumsq<<<nseg, kThreads, 0, s>>>(P.segs.get(), v, tmp.get());
            }
            APF_CUDA(cudaGetLastError());
            APF_CUDA(cudaMemcpyAsync(seg.data(), tmp.get(), nseg * sizeof(double), cudaMemcpyDeviceToHost, s));
            sync(s);
            for (int p = 0; p < P.n_parts; ++p)
                out[p] = seg[2 * p] + seg[2 * p + 1];
            return out;
        }

        __global__ void k_vscale(int n, const double* __restrict__ z, double* __restrict__ v, const MinresDev* S)
        {
            if (S->done)
                return;
            const double s = 1.0 / S->beta;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
                v[i] = s * z[i];
        }

        // y -= (beta/oldb) r1 (not on the first iteration); partial sums of v.y
        __global__ void k_t1(int n, double* __restrict__ y, const double* __restrict__ r1, const double* __restrict__ v,
                             const MinresDev* S, int first, double* __restrict__ partials)
        {
            const double c = (first || S->done) ? 0.0 : S->beta / S->oldb;
            double acc = 0.0;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
            {
                const double yi = y[i] - c * r1[i];
                y[i] = yi;
                acc += v[i] * yi;
            }
            const double t = block_sum(acc);
            if (threadIdx.x == 0)
                partials[blockIdx.x] = t;
        }

        __global__ void k_alfa(int nparts, const double* __restrict__ partials, MinresDev* S)
        {
            __shared__ double ws[32];
            double s = 0.0;
            for (int i = threadIdx.x; i < nparts; i += blockDim.x)
                s += partials[i];
            for (int o = 16; o > 0; o >>= 1)
                s += __shfl_down_sync(0xffffffffu, s, o);
            if ((threadIdx.x & 31) == 0)
                ws[threadIdx.x >> 5] = s;
            __syncthreads();
            if (threadIdx.x == 0)
            {
                double t = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
                    t += ws[w];
                if (!S->done)
                    S->alfa = t;
            }
        }

        __global__ void k_t2(int n, double* __restrict__ y, const double* __restrict__ r2, const MinresDev* S)
        {
            if (S->done)
                return;
            const double c = S->alfa / S->beta;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
                y[i] -= c * r2[i];
        }

        __global__ void k_dot_partials(int n, const double* __restrict__ a, const double* __restrict__ b,
                                       double* __restrict__ partials)
        {
            double acc = 0.0;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
                acc += a[i] * b[i];
            const double t = block_sum(acc);
            if (threadIdx.x == 0)
                partials[blockIdx.x] = t;
        }

        // Lanczos / Givens recurrences after beta_{k+1}^2 = r2.z is known
        __global__ void k_scalars(int nparts, const double* __restrict__ partials, MinresDev* S)
        {
            __shared__ double ws[32];
            double s = 0.0;
            for (int i = threadIdx.x; i < nparts; i += blockDim.x)
                s += partials[i];
            for (int o = 16; o > 0; o >>= 1)
                s += __shfl_down_sync(0xffffffffu, s, o);
            if ((threadIdx.x & 31) == 0)
                ws[threadIdx.x >> 5] = s;
            __syncthreads();
            if (threadIdx.x != 0 || S->done)
                return;
            double bb = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
                bb += ws[w];
            S->bb = bb;
            if (!(bb >= 0.0) || !isfinite(bb))
            {
                S->bad = 1;
                S->done = 1;
                return;
            }
            S->oldb = S->beta;
            const double beta = sqrt(bb);
            S->beta = beta;
            S->oldeps = S->epsln;
            const double delta = S->cs * S->dbar + S->sn * S->alfa;
            const double gbar = S->sn * S->dbar - S->cs * S->alfa;
            S->delta = delta;
            S->epsln = S->sn * beta;
            S->dbar = -S->cs * beta;
            const double gamma = fmax(hypot(gbar, beta), 1e-300);
            S->gamma = gamma;
            S->cs = gbar / gamma;
            S->sn = beta / gamma;
            S->phi = S->cs * S->phibar;
            S->phibar = S->sn * S->phibar;
            S->its += 1;
            S->err = S->r0n * (S->phibar / S->beta1) / S->bn;
        }

        // w_new = (v - oldeps w1 - delta w2)/gamma; x += phi w_new; (w1, w2) <- (w2, w_new)
        __global__ void k_w(int n, const double* __restrict__ v, double* __restrict__ w1, double* __restrict__ w2,
                            double* __restrict__ x, MinresDev* S)
        {
            if (S->done)
                return;
            const double oe = S->oldeps, de = S->delta, ig = 1.0 / S->gamma, ph = S->phi;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
            {
                const double wn = (v[i] - oe * w1[i] - de * w2[i]) * ig;
                w1[i] = w2[i];
                w2[i] = wn;
                x[i] += ph * wn;
            }
        }

        // set done once the backend test passes (runs after k_w so the last update lands)
        __global__ void k_check(MinresDev* S, int max_its)
        {
            if (S->done)
                return;
            if (S->err < S->tol || S->beta == 0.0 || S->its >= max_its)
                S->done = 1;
        }
    }

    namespace
    {
        // Hhat_F: drop |h_ij| < tau sqrt(h_ii h_jj) (j != i) and add |h_ij| to h_ii.  Each
        // dropped pair adds [[|a|,-a],[-a,|a|]] >= 0, so Hhat_F >= Hhat > 0 stays SPD.
        __global__ void drop_count(int n, const int* rp, const int* ci, const double* va, double tau, int* cnt)
        {
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
            {
                double d = 0.0;
                for (int k = rp[r]; k < rp[r + 1]; ++k)
                    if (ci[k] == r)
                        d += va[k];
                int c = 0;
                for (int k = rp[r]; k < rp[r + 1]; ++k)
                {
                    const int j = ci[k];
                    if (j == r)
                    {
                        ++c;
                        continue;
                    }
                    double dj = 0.0;
                    for (int q = rp[j]; q < rp[j + 1]; ++q)
                        if (ci[q] == j)
                            dj += va[q];
                    c += fabs(va[k]) >= tau * sqrt(fabs(d * dj));
                }
                cnt[r] = c;
            }
        }

        __global__ void drop_fill(int n, const int* rp, const int* ci, const double* va, double tau, const int* fp,
                                  int* fc, double* fv)
        {
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
            {
                double d = 0.0;
                for (int k = rp[r]; k < rp[r + 1]; ++k)
                    if (ci[k] == r)
                        d += va[k];
                double lump = 0.0;
                int o = fp[r], diag_pos = -1;
                for (int k = rp[r]; k < rp[r + 1]; ++k)
                {
                    const int j = ci[k];
                    if (j == r)
                    {
                        diag_pos = o;
                        fc[o] = j;
                        fv[o] = 0.0;
                        ++o;
                        continue;
                    }
                    double dj = 0.0;
                    for (int q = rp[j]; q < rp[j + 1]; ++q)
                        if (ci[q] == j)
                            dj += va[q];
                    if (fabs(va[k]) >= tau * sqrt(fabs(d * dj)))
                    {
                        fc[o] = j;
                        fv[o] = va[k];
                        ++o;
                    }
                    else
                        lump += fabs(va[k]);
                }
                if (diag_pos >= 0)
                    fv[diag_pos] = d + lump;
            }
        }
    }

    void BlockPreconditioner::setup(cudaStream_t s, const DeviceCsr& A_y, const DeviceCsr& Hhat, const AmgOptions& opt,
                                    Workspace& w, const int* y_component, const int* x_component)
    {
        n_lambda = A_y.rows;
        n_u = Hhat.rows;
        if (!side_)
        {
            APF_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
            APF_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
            APF_CUDA(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming));
        }
        amg_a.setup(s, A_y, opt, w, y_component);
        // Hhat carries many couplings far below its diagonal scale (products of the
        // time-derivative columns that nearly cancel); the hierarchy is built on the
        // SPD filtered operator Hhat_F >= Hhat
        const int n = Hhat.rows;
        DeviceBuffer<int> cnt(static_cast<std::size_t>(n) + 1, s);
        const int blocks = static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 32)));
        if (n > 0)
        {
            APF_KERNEL("hhat_drop_count", s);
            drop_count<<<blocks, 256, 0, s>>>(n, Hhat.row_ptr.get(), Hhat.col_idx.get(), Hhat.values.get(), kHhatDrop,
                                             cnt.get());
        }
        hhat_f.rows = hhat_f.cols = n;
        hhat_f.row_ptr.allocate(static_cast<std::size_t>(n) + 1, s);
        const long long nnz = exclusive_scan(cnt.get(), hhat_f.row_ptr.get(), n, s);
        hhat_f.col_idx.allocate(static_cast<std::size_t>(nnz), s);
        hhat_f.values.allocate(static_cast<std::size_t>(nnz), s);
        if (n > 0)
        {
            APF_KERNEL("hhat_drop_fill", s);
            drop_fill<<<blocks, 256, 0, s>>>(n, Hhat.row_ptr.get(), Hhat.col_idx.get(), Hhat.values.get(), kHhatDrop,
                                            hhat_f.row_ptr.get(), hhat_f.col_idx.get(), hhat_f.values.get());
        }
        build_sell(s, hhat_f);
        amg_h.setup(s, hhat_f, opt, w, x_component);
        A_y_ = &A_y;
        H_ = &Hhat;
        vcycles = opt.vcycles;
        scale_a = scale_h = 1.0;
        if (vcycles == 2)
        {
            t_a_.allocate(n_lambda, s);
            w_a_.allocate(n_lambda, s);
            t_h_.allocate(n_u, s);
            w_h_.allocate(n_u, s);
        }
    }

    namespace
    {
        // a fixed start vector with entries in [-1, 1] (integer hash of the index)
        __global__ void hash_fill_kernel(int n, double* x)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                unsigned h = static_cast<unsigned>(i) * 2654435761u + 0x9e3779b9u;
                h ^= h >> 15;
                h *= 2246822519u;
                h ^= h >> 13;
                x[i] = static_cast<double>(h) / 2147483648.0 - 1.0;
            }
        }
    }

    void BlockPreconditioner::prepare(cudaStream_t s, Workspace& w)
    {
        if (vcycles != 2)
            return;
        // lambda_max(V A) by 15 power steps (V and A SPD: V A is similar to an SPD matrix, its
        // eigenvalues are positive, the power method converges to the largest from below; the
        // factor 1.1 and the two-step polynomial's margin (positive up to mu = 2) cover the gap)
        auto estimate = [&](Amg& amg, const DeviceCsr& A, int n, double* x, double* y) {
            if (n == 0)
                return 1.0;
            {
                APF_KERNEL("precond_power_start", s);
                hash_fill_kernel<<<static_cast<int>(std::min<long long>((n + 255) / 256, 148 * 16)), 256, 0, s>>>(n, x);
            }
            double nx = std::sqrt(dot_host(s, w, n, x, x));
            double lam = 1.0;
            for (int it = 0; it < 15; ++it)
            {
                spmv(s, A, x, y);      // y = A x
                amg.apply(s, y, x);    // x = V A x_old
                const double nz = std::sqrt(dot_host(s, w, n, x, x));
                require(std::isfinite(nz) && nz > 0.0, APF_ERR_NUMERIC, "preconditioner power iteration broke down");
                lam = nz / nx;
                axpby(s, n, 1.0 / nz, x, 0.0, x);
                nx = 1.0;
            }
            return lam;
        };
        scale_a = 1.0 / (1.1 * estimate(amg_a, *A_y_, n_lambda, t_a_.get(), w_a_.get()));
        scale_h = 1.0 / (1.1 * estimate(amg_h, *H_, n_u, t_h_.get(), w_h_.get()));
        APF_CUDA(cudaGetLastError());
    }

    void BlockPreconditioner::apply_block(cudaStream_t s, int block, const double* r, double* z)
    {
        Amg& amg = block == 0 ? amg_a : amg_h;
        if (vcycles != 2)
        {
            amg.apply(s, r, z);
            return;
        }
        // z = c V r;  z += c V (r - A z): the two-step iteration from zero, the operator
        // c V (2 I - c A V), symmetric, with the eigenvalues 2 mu - mu^2 > 0 of its product with
        // A for mu = c lambda(V A) in (0, 1)
        const int n = block == 0 ? n_lambda : n_u;
        const DeviceCsr& A = block == 0 ? *A_y_ : *H_;
        const double c = block == 0 ? scale_a : scale_h;
        double* t = block == 0 ? t_a_.get() : t_h_.get();
        double* v = block == 0 ? w_a_.get() : w_h_.get();
        amg.apply(s, r, z);
        axpby(s, n, c, z, 0.0, z);
        residual(s, A, z, r, t);
        amg.apply(s, t, v);
        axpby(s, n, c, v, 1.0, z);
    }

    BlockPreconditioner::~BlockPreconditioner()
    {
        if (side_)
            cudaStreamDestroy(side_);
        if (fork_)
            cudaEventDestroy(fork_);
        if (join_)
            cudaEventDestroy(join_);
    }

    void BlockPreconditioner::apply(cudaStream_t s, const double* r, double* z)
    {
        require(side_ != nullptr, APF_ERR_INVALID, "block preconditioner used before its setup");
        if (t_profiler && t_profiler->enabled && t_profiler->kernels)
        {
            // per-launch event timing: both V-cycles on the caller's stream, one after the
            // other, so that each launch's duration is its own (no overlap with the other
            // block's launches sharing the GPU)
            apply_block(s, 1, r + n_lambda, z + n_lambda);
            apply_block(s, 0, r, z);
            return;
        }
        APF_CUDA(cudaEventRecord(fork_, s));
        APF_CUDA(cudaStreamWaitEvent(side_, fork_, 0));
        apply_block(side_, 1, r + n_lambda, z + n_lambda);
        apply_block(s, 0, r, z);
        APF_CUDA(cudaEventRecord(join_, side_));
        APF_CUDA(cudaStreamWaitEvent(s, join_, 0));
    }

    MinresSummary minres_solve(cudaStream_t s, const DeviceCsr& K, Preconditioner& P, const double* b, double* x,
                               const MinresOptions& opt, Workspace& w)
    {
        const int n = K.rows;
        w.ensure(s);
        MinresSummary sum;
        DeviceBuffer<double> r1(n, s), r2(n, s), y(n, s), z(n, s), v(n, s), w1(n, s), w2(n, s), res(n, s);
        DeviceBuffer<MinresDev> S(1, s);
        DeviceBuffer<double> parts(kRedBlocks, s);
        const bool use_graphs = graphs_enabled(s);
        IterationGraph graphs[4];
        const double bn = std::sqrt(dot_host(s, w, n, b, b));
        if (bn == 0.0)
        {
            fill(s, n, 0.0, x);
            sum.converged = true;
            sum.true_residual = 0.0;
            if (opt.parts) // x = 0 solves every part exactly
                sum.part_residuals.assign(static_cast<std::size_t>(opt.parts->n_parts), 0.0);
            return sum;
        }
        DeviceBuffer<double> seg_tmp(opt.parts ? 2 * std::max(1, opt.parts->n_parts) : 1, s);
        std::vector<double> part_b2;
        if (opt.parts)
            part_b2 = part_norms2(s, *opt.parts, b, seg_tmp);
        auto true_residual = [&]() {
            residual(s, K, x, b, res.get());
            const double rel = std::sqrt(dot_host(s, w, n, res.get(), res.get())) / bn;
            if (!opt.parts)
                return rel;
            // every stacked problem must meet the tolerance on its own
            const std::vector<double> r2 = part_norms2(s, *opt.parts, res.get(), seg_tmp);
            sum.part_residuals.assign(r2.size(), 0.0);
            double worst = 0.0;
            for (std::size_t p = 0; p < r2.size(); ++p)
            {
                const double v = part_b2[p] > 0.0 ? std::sqrt(r2[p] / part_b2[p]) : std::sqrt(r2[p]);
                sum.part_residuals[p] = v;
                worst = std::max(worst, std::isfinite(v) ? v : std::numeric_limits<double>::infinity());
            }
            return std::max(rel, worst);
        };
        const int limit = std::max(1, opt.max_iterations);
        const int batch = std::min(limit, std::max(1, opt.batch));
        const double target = std::max(0.0, opt.tolerance);
        const double min_backend = std::max(std::numeric_limits<double>::epsilon(),
                                            target * std::sqrt(std::numeric_limits<double>::epsilon()));
        double backend_tol = target;
        while (sum.iterations < limit)
        {
            const int this_batch = std::min(batch, limit - sum.iterations);
            // --- one backend MINRES run from the current x ---
            residual(s, K, x, b, r1.get());
            P.apply(s, r1.get(), z.get());
            const double r0n = std::sqrt(dot_host(s, w, n, r1.get(), r1.get()));
            const double bb1 = dot_host(s, w, n, r1.get(), z.get());
            if (!(bb1 >= 0.0))
                throw Error(APF_ERR_NUMERIC, "MINRES: preconditioner is not positive definite");
            const double beta1 = std::sqrt(bb1);
            int its = 0;
            bool backend_conv = false;
            double backend_err = r0n / bn;
            if (beta1 == 0.0 || r0n <= backend_tol * bn)
            {
                backend_conv = true;
            }
            else
            {
                MinresDev h{};
                h.beta = beta1;
                h.oldb = 0.0;
                h.phibar = beta1;
                h.cs = -1.0;
                h.sn = 0.0;
                h.beta1 = beta1;
                h.r0n = r0n;
                h.bn = bn;
                h.tol = backend_tol;
                h.err = backend_err;
                APF_CUDA(cudaMemcpyAsync(S.get(), &h, sizeof(h), cudaMemcpyHostToDevice, s));
                copy(s, n, r1.get(), r2.get());
                fill(s, n, 0.0, w1.get());
                fill(s, n, 0.0, w2.get());
                double* pr1 = r1.get();
                double* pr2 = r2.get();
                double* py = y.get();
                int issued = 0;
                MinresDev hs{};
                while (issued < this_batch)
                {
                    const int chunk = std::min(kCheckEvery, this_batch - issued);
                    for (int c = 0; c < chunk; ++c)
                    {
                        const int first = issued == 0;
                        double* q1 = pr1;
                        double* q2 = pr2;
                        double* qy = py;
                        // vectors before the step: r1 = q1, r2 = q2, y = qy; after it the
                        // roles rotate (r1 <- r2, r2 <- y, y <- r1)
                        auto step = [&]() {
                            {
                                APF_KERNEL("minres_vscale", s);
                                k_vscale<<<nb(n), kThreads, 0, s>>>(n, z.get(), v.get(), S.get());
                            }
                            spmv(s, K, v.get(), qy, 1.0, 0.0, "minres_spmv_K");
                            {
                                APF_KERNEL("minres_t1", s);
                                k_t1<<<kRedBlocks, kThreads, 0, s>>>(n, qy, q1, v.get(), S.get(), first, parts.get());
                            }
                            {
                                APF_KERNEL("minres_alfa", s);
                                k_alfa<<<1, 256, 0, s>>>(kRedBlocks, parts.get(), S.get());
                            }
                            {
                                APF_KERNEL("minres_t2", s);
                                k_t2<<<nb(n), kThreads, 0, s>>>(n, qy, q2, S.get());
                            }
                            P.apply(s, qy, z.get());
                            {
                                APF_KERNEL("minres_dot", s);
                                k_dot_partials<<<kRedBlocks, kThreads, 0, s>>>(n, qy, z.get(), parts.get());
                            }
                            {
                                APF_KERNEL("minres_scalars", s);
                                k_scalars<<<1, 256, 0, s>>>(kRedBlocks, parts.get(), S.get());
                            }
                            {
                                APF_KERNEL("minres_w", s);
                                k_w<<<nb(n), kThreads, 0, s>>>(n, v.get(), w1.get(), w2.get(), x, S.get());
                            }
                            {
                                APF_KERNEL("minres_check", s);
                                k_check<<<1, 1, 0, s>>>(S.get(), this_batch);
                            }
                        };
                        if (use_graphs)
                        {
                            IterationGraph& g = first ? graphs[3] : graphs[issued % 3];
                            if (!g.exec || g.batch != this_batch)
                            {
                                capture_iteration(s, g, step);
                                g.batch = this_batch;
                            }
                            APF_CUDA(cudaGraphLaunch(g.exec, s));
                            g_kernel_launches.fetch_add(g.kernels);
                        }
                        else
                        {
                            step();
                        }
                        pr1 = q2;
                        pr2 = qy;
                        py = q1;
                        ++issued;
                    }
                    APF_CUDA(cudaMemcpyAsync(&hs, S.get(), sizeof(hs), cudaMemcpyDeviceToHost, s));
                    sync(s);
                    if (hs.bad)
                        throw Error(APF_ERR_NUMERIC, "MINRES: preconditioner is not positive definite");
                    if (hs.done)
                        break;
                }
                its = hs.its;
                backend_err = hs.err;
                backend_conv = hs.err < backend_tol || hs.beta == 0.0;
            }
            ++sum.batches;
            sum.iterations += its;
            sum.backend_error = backend_err;
            sum.backend_converged = backend_conv;
            const double rel = true_residual();
            sum.true_residual = rel;
            if (std::isfinite(rel) && rel <= target)
            {
                sum.converged = true;
                return sum;
            }
            if (!std::isfinite(rel) || !std::isfinite(backend_err))
                return sum;
            // a batch with no iteration: the backend test already held at the restart.  With
            // one problem that means the true residual met the target (returned above); with
            // stacked problems (parts) the global residual can be below the backend tolerance
            // while one problem's own residual is not, so the tolerance is tightened further
            // until its floor
            if (its <= 0 && (!opt.parts || backend_tol <= min_backend))
                return sum;
            if (backend_conv)
                backend_tol = std::max(min_backend, backend_tol * 0.1);
        }
        return sum;
    }
}
