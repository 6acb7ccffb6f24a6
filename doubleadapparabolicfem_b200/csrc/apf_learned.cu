// Learned smoother weights for the AMG blocks of the MINRES preconditioner: row features,
// the MLP forward pass (FP32 CUDA cores for training, BF16 tensor cores for inference), the
// installation of the weights in the V-cycles, and (further below) the loss of the
// stationary V-cycle iteration with its reverse-mode gradient.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "apf_learned.cuh"

namespace apf
{
    using namespace learned;

    namespace
    {
        int nblk(long long work, int threads, int cap = 148 * 16)
        {
            return static_cast<int>(std::max<long long>(1, std::min<long long>((work + threads - 1) / threads, cap)));
        }

        // one warp per row: scale-free features of row i of A (a_ii = 1 / dinv_i)
        //   f0 sum_j |a_ij| / a_ii        f1 max_j |a_ij| / a_ii      f2 sum_j a_ij / a_ii
        //   f3 sum_j a_ij^2 / (a_ii a_jj) f4 nnz / 32                 f5 share of positive a_ij
        //   f6 level / 8                  f7 block (0: A_y, 1: Hhat)            (j != i)
        __global__ void features_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                        const double* __restrict__ va, const double* __restrict__ dinv, float level,
                                        float block, float* __restrict__ feat)
        {
            const int lane = threadIdx.x & 31;
            const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            const int nw = (gridDim.x * blockDim.x) >> 5;
            for (int i = warp; i < n; i += nw)
            {
                const double di = dinv[i];
                double s_abs = 0.0, s_max = 0.0, s_sgn = 0.0, s_sq = 0.0, s_pos = 0.0;
                const int b = rp[i], e = rp[i + 1];
                for (int k = b + lane; k < e; k += 32)
                {
                    const int j = ci[k];
                    if (j == i)
                        continue;
                    const double a = va[k];
                    s_abs += fabs(a) * di;
                    s_max = fmax(s_max, fabs(a) * di);
                    s_sgn += a * di;
                    s_sq += a * a * di * dinv[j];
                    s_pos += a > 0.0 ? 1.0 : 0.0;
                }
                for (int o = 16; o > 0; o >>= 1)
                {
                    s_abs += __shfl_xor_sync(0xffffffffu, s_abs, o);
                    s_max = fmax(s_max, __shfl_xor_sync(0xffffffffu, s_max, o));
                    s_sgn += __shfl_xor_sync(0xffffffffu, s_sgn, o);
                    s_sq += __shfl_xor_sync(0xffffffffu, s_sq, o);
                    s_pos += __shfl_xor_sync(0xffffffffu, s_pos, o);
                }
                if (lane == 0)
                {
                    const int nnz = e - b;
                    float* f = feat + static_cast<long long>(i) * kFeatures;
                    f[0] = static_cast<float>(s_abs);
                    f[1] = static_cast<float>(s_max);
                    f[2] = static_cast<float>(s_sgn);
                    f[3] = static_cast<float>(s_sq);
                    f[4] = static_cast<float>(nnz) / 32.0f;
                    f[5] = nnz > 1 ? static_cast<float>(s_pos / (nnz - 1)) : 0.0f;
                    f[6] = level / 8.0f;
                    f[7] = block;
                }
            }
        }

        // FP32 forward pass, one thread per row; also used by the training pass
        __device__ __forceinline__ void mlp_fp32(const float* __restrict__ P, const float* f, float* h1, float* h2,
                                                 float* y)
        {
            for (int j = 0; j < kHidden; ++j)
            {
                float a = P[kB1 + j];
                for (int k = 0; k < kFeatures; ++k)
                    a = fmaf(P[kW1 + j * kFeatures + k], f[k], a);
                h1[j] = tanhf(a);
            }
            for (int j = 0; j < kHidden; ++j)
            {
                float a = P[kB2 + j];
                for (int k = 0; k < kHidden; ++k)
                    a = fmaf(P[kW2 + j * kHidden + k], h1[k], a);
                h2[j] = tanhf(a);
            }
            for (int o = 0; o < kOutputs; ++o)
            {
                float a = P[kB3 + o];
                for (int k = 0; k < kHidden; ++k)
                    a = fmaf(P[kW3 + o * kHidden + k], h2[k], a);
                y[o] = a;
            }
        }

        __global__ void forward_fp32_kernel(int n, const float* __restrict__ params, const float* __restrict__ feat,
                                            float* __restrict__ y)
        {
            __shared__ float P[kParams];
            for (int i = threadIdx.x; i < kParams; i += blockDim.x)
                P[i] = params[i];
            __syncthreads();
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                float f[kFeatures], h1[kHidden], h2[kHidden], out[kOutputs];
                for (int k = 0; k < kFeatures; ++k)
                    f[k] = feat[static_cast<long long>(i) * kFeatures + k];
                mlp_fp32(P, f, h1, h2, out);
                for (int o = 0; o < kOutputs; ++o)
                    y[static_cast<long long>(i) * kOutputs + o] = out[o];
            }
        }

        __device__ __forceinline__ unsigned pack_bf16(float lo, float hi)
        {
            const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
            unsigned u;
            memcpy(&u, &v, sizeof(u));
            return u;
        }

        __device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1)
        {
            asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                         "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                         : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                         : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
        }

        // BF16 forward pass on the tensor cores: one warp per tile of 16 rows.
        // Layer 1: [16 x 16 (8 features, zero padded)] x [16 x 32]; layer 2: [16 x 32] x [32 x 32];
        // the FP32 accumulator fragments of one layer are repacked in registers as the next
        // layer's BF16 operand fragments; the last layer (32 -> 2) is a quad shuffle reduction.
        __global__ void __launch_bounds__(128) forward_bf16_kernel(int n, const float* __restrict__ params,
                                                                   const float* __restrict__ feat, float* __restrict__ y)
        {
            const int lane = threadIdx.x & 31;
            const int g = lane >> 2, t = lane & 3;
            // B fragments of W1^T (k = feature, n = hidden unit) and W2^T, biases and w3 in the
            // accumulator layout (columns 2t, 2t+1 of each 8-wide tile)
            unsigned b1f[4][2], b2f[2][4][2];
            float bias1[4][2], bias2[4][2], w3[kOutputs][4][2];
            for (int nt = 0; nt < 4; ++nt)
            {
                const int col = nt * 8 + g;
                const int k0 = 2 * t;
                b1f[nt][0] = pack_bf16(params[kW1 + col * kFeatures + k0], params[kW1 + col * kFeatures + k0 + 1]);
                b1f[nt][1] = 0u; // features 8..15 are padding
                for (int ks = 0; ks < 2; ++ks)
                {
                    const int kk = ks * 16 + 2 * t;
                    b2f[ks][nt][0] = pack_bf16(params[kW2 + col * kHidden + kk], params[kW2 + col * kHidden + kk + 1]);
                    b2f[ks][nt][1] = pack_bf16(params[kW2 + col * kHidden + kk + 8], params[kW2 + col * kHidden + kk + 9]);
                }
                for (int c = 0; c < 2; ++c)
                {
                    bias1[nt][c] = params[kB1 + nt * 8 + 2 * t + c];
                    bias2[nt][c] = params[kB2 + nt * 8 + 2 * t + c];
                    for (int o = 0; o < kOutputs; ++o)
                        w3[o][nt][c] = params[kW3 + o * kHidden + nt * 8 + 2 * t + c];
                }
            }
            float b3[kOutputs];
            for (int o = 0; o < kOutputs; ++o)
                b3[o] = params[kB3 + o];
            const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            const int nw = (gridDim.x * blockDim.x) >> 5;
            const int tiles = (n + 15) / 16;
            for (int tile = warp; tile < tiles; tile += nw)
            {
                const int r0 = tile * 16 + g, r1 = r0 + 8;
                float f00 = 0.f, f01 = 0.f, f10 = 0.f, f11 = 0.f;
                if (r0 < n)
                {
                    f00 = feat[static_cast<long long>(r0) * kFeatures + 2 * t];
                    f01 = feat[static_cast<long long>(r0) * kFeatures + 2 * t + 1];
                }
                if (r1 < n)
                {
                    f10 = feat[static_cast<long long>(r1) * kFeatures + 2 * t];
                    f11 = feat[static_cast<long long>(r1) * kFeatures + 2 * t + 1];
                }
                const unsigned a1[4] = {pack_bf16(f00, f01), pack_bf16(f10, f11), 0u, 0u};
                float h1[4][4];
                for (int nt = 0; nt < 4; ++nt)
                {
                    h1[nt][0] = bias1[nt][0];
                    h1[nt][1] = bias1[nt][1];
                    h1[nt][2] = bias1[nt][0];
                    h1[nt][3] = bias1[nt][1];
                    mma_bf16(h1[nt], a1, b1f[nt][0], b1f[nt][1]);
                }
                unsigned a2[2][4];
                for (int ks = 0; ks < 2; ++ks)
                {
                    const int n0 = 2 * ks, n1 = 2 * ks + 1;
                    a2[ks][0] = pack_bf16(tanhf(h1[n0][0]), tanhf(h1[n0][1]));
                    a2[ks][1] = pack_bf16(tanhf(h1[n0][2]), tanhf(h1[n0][3]));
                    a2[ks][2] = pack_bf16(tanhf(h1[n1][0]), tanhf(h1[n1][1]));
                    a2[ks][3] = pack_bf16(tanhf(h1[n1][2]), tanhf(h1[n1][3]));
                }
                float acc0[kOutputs], acc1[kOutputs];
                for (int o = 0; o < kOutputs; ++o)
                    acc0[o] = acc1[o] = 0.f;
                for (int nt = 0; nt < 4; ++nt)
                {
                    float h2[4] = {bias2[nt][0], bias2[nt][1], bias2[nt][0], bias2[nt][1]};
                    mma_bf16(h2, a2[0], b2f[0][nt][0], b2f[0][nt][1]);
                    mma_bf16(h2, a2[1], b2f[1][nt][0], b2f[1][nt][1]);
                    const float t0 = tanhf(h2[0]), t1 = tanhf(h2[1]), t2 = tanhf(h2[2]), t3 = tanhf(h2[3]);
                    for (int o = 0; o < kOutputs; ++o)
                    {
                        acc0[o] = fmaf(w3[o][nt][0], t0, fmaf(w3[o][nt][1], t1, acc0[o]));
                        acc1[o] = fmaf(w3[o][nt][0], t2, fmaf(w3[o][nt][1], t3, acc1[o]));
                    }
                }
                for (int o = 0; o < kOutputs; ++o)
                {
                    acc0[o] += __shfl_xor_sync(0xffffffffu, acc0[o], 1);
                    acc0[o] += __shfl_xor_sync(0xffffffffu, acc0[o], 2);
                    acc1[o] += __shfl_xor_sync(0xffffffffu, acc1[o], 1);
                    acc1[o] += __shfl_xor_sync(0xffffffffu, acc1[o], 2);
                }
                if (t == 0)
                {
                    for (int o = 0; o < kOutputs; ++o)
                    {
                        if (r0 < n)
                            y[static_cast<long long>(r0) * kOutputs + o] = acc0[o] + b3[o];
                        if (r1 < n)
                            y[static_cast<long long>(r1) * kOutputs + o] = acc1[o] + b3[o];
                    }
                }
            }
        }

        // w_i = omega * dinv_i * exp(range * tanh(y_i^(o)))
        __global__ void weights_kernel(int n, const float* __restrict__ y, int o, const double* __restrict__ dinv,
                                       double omega, double* __restrict__ w)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                w[i] = omega * dinv[i] *
                       exp(static_cast<double>(kWeightRange) *
                           tanh(static_cast<double>(y[static_cast<long long>(i) * kOutputs + o])));
        }

        // symmetric Gershgorin row sums of W^1/2 A W^1/2, maximum via integer atomics on the
        // (non-negative) double bit pattern
        __global__ void gershgorin_sym_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                              const double* __restrict__ va, const double* __restrict__ w,
                                              unsigned long long* __restrict__ out)
        {
            double best = 0.0;
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                const double wi = w[i];
                double sum = 0.0;
                for (int k = rp[i]; k < rp[i + 1]; ++k)
                    sum += sqrt(wi * w[ci[k]]) * fabs(va[k]);
                best = fmax(best, sum);
            }
            for (int o = 16; o > 0; o >>= 1)
                best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
            if ((threadIdx.x & 31) == 0)
                atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(best)));
        }

        // w *= bound / g when the Gershgorin bound g (device, double bits) exceeds bound
        __global__ void bound_kernel(int n, const unsigned long long* __restrict__ gbits, double bound,
                                     double* __restrict__ w)
        {
            const double g = __longlong_as_double(static_cast<long long>(*gbits));
            if (!(g > bound))
                return;
            const double a = bound / g;
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                w[i] *= a;
        }

        // weights of sweep class o on one level from model outputs y, bounded on the device
        void bounded_weights(cudaStream_t s, const AmgLevel& L, const float* y, int o, DeviceBuffer<double>& w)
        {
            const DeviceCsr& A = *L.A;
            const int n = A.rows;
            w.allocate(n, s);
            {
                APF_KERNEL("learned_weights", s);
                weights_kernel<<<nblk(n, 256), 256, 0, s>>>(n, y, o, L.dinv.get(), L.omega, w.get());
            }
            DeviceBuffer<unsigned long long> gmax(1, s);
            gmax.zero();
            {
                APF_KERNEL("learned_gershgorin", s);
                gershgorin_sym_kernel<<<nblk(n, 256, 1024), 256, 0, s>>>(n, A.row_ptr.get(), A.col_idx.get(),
                                                                         A.values.get(), w.get(), gmax.get());
            }
            {
                APF_KERNEL("learned_bound", s);
                bound_kernel<<<nblk(n, 256), 256, 0, s>>>(n, gmax.get(), kSmootherBound, w.get());
            }
        }

        double alpha_of(const LearnedModel& m, int block, int level)
        {
            const float th = m.params[kAlpha + block * kMaxLevels + std::min(level, kMaxLevels - 1)];
            return 2.0 / (1.0 + std::exp(-static_cast<double>(th)));
        }
    }

    void learned_features(cudaStream_t s, const DeviceCsr& A, const double* dinv, int level, int block, float* feat)
    {
        if (A.rows == 0)
            return;
        APF_KERNEL("learned_features", s);
        features_kernel<<<nblk(static_cast<long long>(A.rows) * 32, 256), 256, 0, s>>>(
            A.rows, A.row_ptr.get(), A.col_idx.get(), A.values.get(), dinv, static_cast<float>(level),
            static_cast<float>(block), feat);
    }

    void learned_forward(cudaStream_t s, const float* params, int n, const float* feat, float* y, int precision)
    {
        if (n == 0)
            return;
        if (precision == 0)
        {
            APF_KERNEL("learned_forward_fp32", s);
            forward_fp32_kernel<<<nblk(n, 128), 128, 0, s>>>(n, params, feat, y);
        }
        else
        {
            APF_KERNEL("learned_forward_bf16_mma", s);
            forward_bf16_kernel<<<nblk((static_cast<long long>(n) + 15) / 16 * 32, 128), 128, 0, s>>>(n, params, feat, y);
        }
    }

    void apply_learned_smoothers(cudaStream_t s, const LearnedModel& model, Amg& amg, int block)
    {
        DeviceBuffer<float> dparams(kParams, s);
        dparams.upload(model.params.data(), kParams);
        const int nl = amg.levels();
        for (int l = 0; l + 1 < nl; ++l)
        {
            const AmgLevel& L = amg.level(l);
            const int n = L.A->rows;
            DeviceBuffer<float> feat(static_cast<std::size_t>(n) * kFeatures, s), y(static_cast<std::size_t>(n) * kOutputs, s);
            learned_features(s, *L.A, L.dinv.get(), l, block, feat.get());
            learned_forward(s, dparams.get(), n, feat.get(), y.get(), 1);
            DeviceBuffer<double> w, w2;
            bounded_weights(s, L, y.get(), 0, w);
            bounded_weights(s, L, y.get(), 1, w2);
            amg.set_smoother(l, std::move(w), std::move(w2), alpha_of(model, block, l));
        }
    }
}

// ---------------------------------------------------------------------------------------
// Training: loss of the stationary V-cycle iteration and its reverse-mode gradient
// ---------------------------------------------------------------------------------------
namespace apf
{
    namespace
    {
        __global__ void mul_kernel(int n, const double* __restrict__ a, const double* __restrict__ b,
                                   double* __restrict__ y)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                y[i] = a[i] * b[i];
        }

        // y += a (.) b
        __global__ void fma_kernel(int n, const double* __restrict__ a, const double* __restrict__ b,
                                   double* __restrict__ y)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                y[i] += a[i] * b[i];
        }

        // ybar_i^(o) = wbar_i * dw_i / dy_i^(o) = wbar_i * w_i * range * (1 - tanh^2 y_i^(o))
        __global__ void ybar_kernel(int n, int o, const double* __restrict__ wbar, const double* __restrict__ w,
                                    const float* __restrict__ y, float* __restrict__ ybar)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                const long long k = static_cast<long long>(i) * kOutputs + o;
                const double th = tanh(static_cast<double>(y[k]));
                ybar[k] = static_cast<float>(wbar[i] * w[i] * kWeightRange * (1.0 - th * th));
            }
        }

        // counter-based standard normal numbers (splitmix64 + Box-Muller)
        __device__ __forceinline__ unsigned long long splitmix(unsigned long long x)
        {
            x += 0x9e3779b97f4a7c15ull;
            x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
            x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
            return x ^ (x >> 31);
        }

        __global__ void normal_kernel(int n, unsigned long long seed, double* __restrict__ y)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            {
                const unsigned long long h1 = splitmix(seed * 0x632be59bd9b4e019ull + 2ull * i);
                const unsigned long long h2 = splitmix(seed * 0x632be59bd9b4e019ull + 2ull * i + 1ull);
                const double u1 = (static_cast<double>(h1 >> 11) + 0.5) * (1.0 / 9007199254740992.0);
                const double u2 = static_cast<double>(h2 >> 11) * (1.0 / 9007199254740992.0);
                y[i] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
            }
        }

        // MLP backward over rows: per-block partial gradients (deterministic order).  A tile of
        // kTile rows is run forward and backward by kTile threads (one row each); the block
        // then forms the tile's weight-gradient outer products from shared memory, each
        // thread owning fixed gradient entries.
        constexpr int kTile = 64;
        constexpr int kBackThreads = 256;

        __global__ void __launch_bounds__(kBackThreads) mlp_backward_kernel(int n, const float* __restrict__ params,
                                                                           const float* __restrict__ feat,
                                                                           const float* __restrict__ ybar,
                                                                           float* __restrict__ partial)
        {
            __shared__ float P[kParams];
            __shared__ float sf[kTile][kFeatures];
            __shared__ float sh1[kTile][kHidden + 1];
            __shared__ float sd1[kTile][kHidden + 1];
            __shared__ float sh2[kTile][kHidden + 1];
            __shared__ float sd2[kTile][kHidden + 1];
            __shared__ float syb[kTile][kOutputs];
            const int tid = threadIdx.x;
            for (int i = tid; i < kParams; i += blockDim.x)
                P[i] = params[i];
            float gW2[4] = {0.f, 0.f, 0.f, 0.f};
            float gW1 = 0.f, gB1 = 0.f, gB2 = 0.f, gW3 = 0.f, gB3 = 0.f;
            __syncthreads();
            const int tiles = (n + kTile - 1) / kTile;
            for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x)
            {
                if (tid < kTile)
                {
                    const int r = tile * kTile + tid;
                    float f[kFeatures], h1[kHidden], h2[kHidden], y[kOutputs];
                    float yb[kOutputs];
                    for (int o = 0; o < kOutputs; ++o)
                        yb[o] = 0.f;
                    if (r < n)
                    {
                        for (int k = 0; k < kFeatures; ++k)
                            f[k] = feat[static_cast<long long>(r) * kFeatures + k];
                        for (int o = 0; o < kOutputs; ++o)
                            yb[o] = ybar[static_cast<long long>(r) * kOutputs + o];
                    }
                    else
                        for (int k = 0; k < kFeatures; ++k)
                            f[k] = 0.f;
                    mlp_fp32(P, f, h1, h2, y);
                    float d2[kHidden];
                    for (int j = 0; j < kHidden; ++j)
                    {
                        float a = 0.f;
                        for (int o = 0; o < kOutputs; ++o)
                            a = fmaf(yb[o], P[kW3 + o * kHidden + j], a);
                        d2[j] = a * (1.f - h2[j] * h2[j]);
                    }
                    for (int k = 0; k < kHidden; ++k)
                    {
                        float a = 0.f;
                        for (int j = 0; j < kHidden; ++j)
                            a = fmaf(P[kW2 + j * kHidden + k], d2[j], a);
                        sd1[tid][k] = a * (1.f - h1[k] * h1[k]);
                        sh1[tid][k] = h1[k];
                        sh2[tid][k] = h2[k];
                        sd2[tid][k] = d2[k];
                    }
                    for (int k = 0; k < kFeatures; ++k)
                        sf[tid][k] = f[k];
                    for (int o = 0; o < kOutputs; ++o)
                        syb[tid][o] = yb[o];
                }
                __syncthreads();
                // W2[j][k]: entries tid, tid + 256, tid + 512, tid + 768
                for (int q = 0; q < 4; ++q)
                {
                    const int e = tid + q * kBackThreads, j = e / kHidden, k = e % kHidden;
                    float a = 0.f;
                    for (int r = 0; r < kTile; ++r)
                        a = fmaf(sd2[r][j], sh1[r][k], a);
                    gW2[q] += a;
                }
                {
                    const int j = tid / kFeatures, k = tid % kFeatures; // W1[j][k], 256 entries
                    float a = 0.f;
                    for (int r = 0; r < kTile; ++r)
                        a = fmaf(sd1[r][j], sf[r][k], a);
                    gW1 += a;
                }
                if (tid < kHidden)
                {
                    float a1 = 0.f, a2 = 0.f;
                    for (int r = 0; r < kTile; ++r)
                    {
                        a1 += sd1[r][tid];
                        a2 += sd2[r][tid];
                    }
                    gB1 += a1;
                    gB2 += a2;
                }
                if (tid < kOutputs * kHidden) // W3[o][j]
                {
                    const int o = tid / kHidden, j = tid % kHidden;
                    float a = 0.f;
                    for (int r = 0; r < kTile; ++r)
                        a = fmaf(syb[r][o], sh2[r][j], a);
                    gW3 += a;
                }
                if (tid < kOutputs)
                {
                    float a = 0.f;
                    for (int r = 0; r < kTile; ++r)
                        a += syb[r][tid];
                    gB3 += a;
                }
                __syncthreads();
            }
            float* out = partial + static_cast<long long>(blockIdx.x) * kParams;
            for (int q = 0; q < 4; ++q)
                out[kW2 + tid + q * kBackThreads] = gW2[q];
            out[kW1 + tid] = gW1;
            if (tid < kHidden)
            {
                out[kB1 + tid] = gB1;
                out[kB2 + tid] = gB2;
            }
            if (tid < kOutputs * kHidden)
                out[kW3 + tid] = gW3;
            if (tid < kOutputs)
                out[kB3 + tid] = gB3;
        }

        static_assert(kHidden * kHidden == 4 * kBackThreads, "W2 gradient ownership");
        static_assert(kHidden * kFeatures == kBackThreads, "W1 gradient ownership");

        // sum of the per-block partial gradients in block order
        __global__ void reduce_partials_kernel(int blocks, const float* __restrict__ partial, float* __restrict__ out)
        {
            for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kAlpha; p += gridDim.x * blockDim.x)
            {
                float a = 0.f;
                for (int b = 0; b < blocks; ++b)
                    a += partial[static_cast<long long>(b) * kParams + p];
                out[p] = a;
            }
        }

        struct LevelTape
        {
            // per application: the input b, the residuals b - A x before every pre-smoothing
            // sweep after the first and before every post-smoothing sweep, and P x_c
            std::vector<DeviceBuffer<double>> b, pxc;
            std::vector<std::vector<DeviceBuffer<double>>> pre_r, post_r;
        };

        // V-cycle with recorded intermediates and its reverse pass: `sweeps` damped-Jacobi
        // sweeps with the level's weights w before and after the coarse correction, which is
        // scaled by alpha (the structure of Amg::vcycle with a learned smoother)
        class TapedVcycle
        {
        public:
            TapedVcycle(cudaStream_t s, Amg& amg, int applications, int sweeps, Workspace& w)
                : s_(s), amg_(amg), ws_(w), sweeps_(sweeps)
            {
                const int nl = amg.levels();
                tape_.resize(nl);
                scratch_.resize(nl);
                wbar_.resize(nl);
                abar_.assign(nl, 0.0);
                for (int l = 0; l + 1 < nl; ++l)
                {
                    const int n = amg.level(l).A->rows;
                    auto& T = tape_[l];
                    T.pre_r.resize(applications);
                    T.post_r.resize(applications);
                    for (int a = 0; a < applications; ++a)
                    {
                        T.b.emplace_back(n, s);
                        T.pxc.emplace_back(n, s);
                        for (int k = 0; k < sweeps; ++k)
                        {
                            T.pre_r[a].emplace_back(k == 0 ? 0 : n, s);
                            T.post_r[a].emplace_back(n, s);
                        }
                    }
                    for (int o = 0; o < kOutputs; ++o)
                    {
                        wbar_[l].emplace_back(n, s);
                        wbar_[l].back().zero();
                    }
                }
                // per level: 6 work vectors, then the level's input [6] and output [7] as seen
                // from the finer level
                for (int l = 0; l < nl; ++l)
                {
                    const int n = amg.level(l).A->rows;
                    for (int k = 0; k < 8; ++k)
                        scratch_[l].emplace_back(n, s);
                }
            }

            void forward(int app, const double* b, double* x) { fwd(0, app, b, x); }
            void reverse(int app, const double* xbar, double* bbar) { rev(0, app, xbar, bbar); }
            DeviceBuffer<double>& wbar(int l, int o) { return wbar_[l][o]; }
            double abar(int l) const { return abar_[l]; }

        private:
            int g(int n) const { return nblk(n, 256); }
            // sweep class of pre-smoothing sweep k and its weights (post-smoothing sweep k in
            // time order is pre-smoothing sweep sweeps - 1 - k)
            static int cls(int k) { return k == 0 ? 0 : 1; }
            static const double* W(const AmgLevel& L, int o) { return o == 0 ? L.w.get() : L.w2.get(); }

            void mul(int n, const double* a, const double* b, double* y)
            {
                APF_KERNEL("learned_train_mul", s_);
                mul_kernel<<<g(n), 256, 0, s_>>>(n, a, b, y);
            }
            void fma(int n, const double* a, const double* b, double* y)
            {
                APF_KERNEL("learned_train_fma", s_);
                fma_kernel<<<g(n), 256, 0, s_>>>(n, a, b, y);
            }

            void fwd(int l, int app, const double* b, double* x)
            {
                Amg& M = amg_;
                if (l == M.levels() - 1)
                {
                    M.coarse_apply(s_, b, x);
                    return;
                }
                AmgLevel& L = M.level(l);
                const DeviceCsr& A = *L.A;
                const int n = A.rows;
                double* r1 = scratch_[l][1].get();
                double* bc = scratch_[l + 1][6].get();
                double* xc = scratch_[l + 1][7].get();
                auto& T = tape_[l];
                copy(s_, n, b, T.b[app].get());
                mul(n, W(L, 0), b, x);                         // first pre-smoothing sweep from 0
                for (int k = 1; k < sweeps_; ++k)
                {
                    double* r = T.pre_r[app][k].get();
                    residual(s_, A, x, b, r);
                    fma(n, W(L, cls(k)), r, x);
                }
                residual(s_, A, x, b, r1);
                spmv(s_, L.R, r1, bc);
                fwd(l + 1, app, bc, xc);
                spmv(s_, L.P, xc, T.pxc[app].get());
                axpby(s_, n, L.alpha, T.pxc[app].get(), 1.0, x);
                for (int k = 0; k < sweeps_; ++k)
                {
                    double* r = T.post_r[app][k].get();
                    residual(s_, A, x, b, r);
                    fma(n, W(L, cls(sweeps_ - 1 - k)), r, x);
                }
            }

            void rev(int l, int app, const double* xbar_in, double* bb)
            {
                Amg& M = amg_;
                if (l == M.levels() - 1)
                {
                    M.coarse_apply(s_, xbar_in, bb); // symmetric linear map: its own adjoint
                    return;
                }
                AmgLevel& L = M.level(l);
                const DeviceCsr& A = *L.A;
                const int n = A.rows;
                auto& sc = scratch_[l];
                double* xb = sc[0].get();   // running adjoint of the iterate
                double* rb = sc[1].get();
                double* tmp = sc[2].get();
                double* xcb = scratch_[l + 1][6].get();
                double* bcb = scratch_[l + 1][7].get();
                auto& T = tape_[l];
                copy(s_, n, xbar_in, xb);
                fill(s_, n, 0.0, bb);
                // one sweep x+ = x + W r, r = b - A x, read backwards:
                //   wbar += xb (.) r;  rb = W xb;  bb += rb;  xb = xb - A rb
                auto sweep_back = [&](const double* r, int o) {
                    fma(n, xb, r, wbar_[l][o].get());
                    mul(n, W(L, o), xb, rb);
                    axpby(s_, n, 1.0, rb, 1.0, bb);
                    residual(s_, A, rb, xb, tmp);
                    std::swap(xb, tmp);
                };
                for (int k = sweeps_ - 1; k >= 0; --k)
                    sweep_back(T.post_r[app][k].get(), cls(sweeps_ - 1 - k));
                // coarse correction x+ = x + alpha P V(R (b - A x))
                abar_[l] += dot_host(s_, ws_, n, xb, T.pxc[app].get());
                spmv(s_, L.R, xb, xcb, L.alpha, 0.0);
                rev(l + 1, app, xcb, bcb);
                spmv(s_, L.P, bcb, rb);
                axpby(s_, n, 1.0, rb, 1.0, bb);
                residual(s_, A, rb, xb, tmp);
                std::swap(xb, tmp);
                for (int k = sweeps_ - 1; k >= 1; --k)
                    sweep_back(T.pre_r[app][k].get(), cls(k));
                // first sweep x = W b
                fma(n, W(L, 0), xb, bb);
                fma(n, xb, T.b[app].get(), wbar_[l][0].get());
            }

            cudaStream_t s_;
            Amg& amg_;
            Workspace& ws_;
            int sweeps_;
            std::vector<LevelTape> tape_;
            std::vector<std::vector<DeviceBuffer<double>>> scratch_;
            std::vector<std::vector<DeviceBuffer<double>>> wbar_;
            std::vector<double> abar_;
        };

        struct LevelModelState
        {
            DeviceBuffer<float> feat, y;
        };
    }

    double learned_loss_and_grad(cudaStream_t s, const LearnedModel& model, BlockPreconditioner& P,
                                 const DeviceCsr& target_a, const DeviceCsr& target_h, int samples, int steps,
                                 int burn_in, unsigned long long seed, const double* start_vectors, float* grad,
                                 Workspace& ws)
    {
        require(samples >= 1 && steps >= 1 && burn_in >= 0, APF_ERR_INVALID,
                "learned loss: samples and steps must be positive, burn_in non-negative");
        ws.ensure(s);
        DeviceBuffer<float> dparams(kParams, s);
        dparams.upload(model.params.data(), kParams);
        std::vector<float> g(kParams, 0.0f);
        double loss = 0.0;
        const int nlam = P.n_lambda;
        for (int block = 0; block < 2; ++block)
        {
            Amg& amg = block == 0 ? P.amg_a : P.amg_h;
            const DeviceCsr& T = block == 0 ? target_a : target_h;
            const int n = T.rows;
            const int nl = amg.levels();
            // model outputs on every non-coarsest level (FP32 forward), weights installed; the
            // Gershgorin rescale is a constant factor (no gradient through the bound)
            std::vector<LevelModelState> st(std::max(0, nl - 1));
            for (int l = 0; l + 1 < nl; ++l)
            {
                AmgLevel& L = amg.level(l);
                const int nr = L.A->rows;
                st[l].feat.allocate(static_cast<std::size_t>(nr) * kFeatures, s);
                st[l].y.allocate(static_cast<std::size_t>(nr) * kOutputs, s);
                learned_features(s, *L.A, L.dinv.get(), l, block, st[l].feat.get());
                learned_forward(s, dparams.get(), nr, st[l].feat.get(), st[l].y.get(), 0);
                DeviceBuffer<double> w, w2;
                bounded_weights(s, L, st[l].y.get(), 0, w);
                bounded_weights(s, L, st[l].y.get(), 1, w2);
                amg.set_smoother(l, std::move(w), std::move(w2), alpha_of(model, block, l));
            }
            TapedVcycle V(s, amg, steps, amg.smooth_steps(), ws);
            DeviceBuffer<double> e(n, s), a(n, s), v(n, s), te(n, s), ebar(n, s), abarv(n, s);
            double block_loss = 0.0;
            for (int smp = 0; smp < samples; ++smp)
            {
                if (start_vectors)
                    copy(s, n, start_vectors + static_cast<long long>(smp) * (nlam + P.n_u) + (block == 0 ? 0 : nlam),
                         e.get());
                else
                {
                    APF_KERNEL("learned_train_normal", s);
                    normal_kernel<<<nblk(n, 256), 256, 0, s>>>(n, seed * 2654435761ull + 2ull * smp + block, e.get());
                }
                // burn-in (no gradient): e <- E^burn_in e, rescaled to unit energy
                for (int j = 0; j < burn_in; ++j)
                {
                    spmv(s, T, e.get(), a.get());
                    amg.apply(s, a.get(), v.get());
                    axpby(s, n, -1.0, v.get(), 1.0, e.get());
                }
                spmv(s, T, e.get(), te.get());
                double q0 = dot_host(s, ws, n, e.get(), te.get());
                require(q0 > 0.0 && std::isfinite(q0), APF_ERR_NUMERIC, "learned loss: start vector with no energy");
                if (burn_in > 0)
                {
                    axpby(s, n, 0.0, e.get(), 1.0 / std::sqrt(q0), e.get());
                    q0 = 1.0;
                }
                for (int j = 0; j < steps; ++j)
                {
                    spmv(s, T, e.get(), a.get());
                    V.forward(j, a.get(), v.get());
                    axpby(s, n, -1.0, v.get(), 1.0, e.get());
                }
                spmv(s, T, e.get(), te.get());
                const double qk = dot_host(s, ws, n, e.get(), te.get());
                require(qk > 0.0 && std::isfinite(qk), APF_ERR_NUMERIC, "learned loss: iteration lost all energy");
                block_loss += (std::log(qk) - std::log(q0)) / steps;
                if (!grad)
                    continue;
                // ebar_k = (2 / k) T e_k / q_k; then for j = k-1..0: vbar = -ebar, abar = V^T vbar,
                // ebar += T abar
                copy(s, n, te.get(), ebar.get());
                axpby(s, n, 0.0, te.get(), 2.0 / (steps * qk), ebar.get());
                for (int j = steps - 1; j >= 0; --j)
                {
                    copy(s, n, ebar.get(), v.get());
                    axpby(s, n, 0.0, ebar.get(), -1.0, v.get());
                    V.reverse(j, v.get(), abarv.get());
                    spmv(s, T, abarv.get(), ebar.get(), 1.0, 1.0);
                }
            }
            loss += block_loss / samples;
            if (!grad)
                continue;
            // parameter gradients: alpha logits on the host, MLP weights by the backward kernel
            for (int l = 0; l + 1 < nl; ++l)
            {
                const double al = amg.level(l).alpha;
                const double ab = V.abar(l) / samples;
                g[kAlpha + block * kMaxLevels + std::min(l, kMaxLevels - 1)] += static_cast<float>(ab * al * (1.0 - al / 2.0));
                const int nr = amg.level(l).A->rows;
                DeviceBuffer<float> yb(static_cast<std::size_t>(nr) * kOutputs, s);
                for (int o = 0; o < kOutputs; ++o)
                {
                    DeviceBuffer<double>& wb = V.wbar(l, o);
                    axpby(s, nr, 0.0, wb.get(), 1.0 / samples, wb.get());
                    APF_KERNEL("learned_train_ybar", s);
                    ybar_kernel<<<nblk(nr, 256), 256, 0, s>>>(nr, o, wb.get(),
                                                              o == 0 ? amg.level(l).w.get() : amg.level(l).w2.get(),
                                                              st[l].y.get(), yb.get());
                }
                const int blocks = std::max(1, std::min(148 * 2, (nr + kTile - 1) / kTile));
                DeviceBuffer<float> partial(static_cast<std::size_t>(blocks) * kParams, s), sum(kParams, s);
                {
                    APF_KERNEL("learned_mlp_backward", s);
                    mlp_backward_kernel<<<blocks, kBackThreads, 0, s>>>(nr, dparams.get(), st[l].feat.get(), yb.get(),
                                                                      partial.get());
                }
                {
                    APF_KERNEL("learned_reduce_partials", s);
                    reduce_partials_kernel<<<nblk(kAlpha, 256), 256, 0, s>>>(blocks, partial.get(), sum.get());
                }
                std::vector<float> h(kParams);
                APF_CUDA(cudaMemcpyAsync(h.data(), sum.get(), kAlpha * sizeof(float), cudaMemcpyDeviceToHost, s));
                sync(s);
                for (int p = 0; p < kAlpha; ++p)
                    g[p] += h[p];
            }
        }
        if (grad)
            std::memcpy(grad, g.data(), sizeof(float) * kParams);
        return loss;
    }
}
