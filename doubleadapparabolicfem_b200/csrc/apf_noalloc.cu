// Allocation-free true-residual check.
//
// apf_true_residual_noalloc computes ||b - K x||_2 / ||b||_2 (the acceptance test of the
// MINRES batches) for a CSR matrix that the caller already holds on the device, without
// allocating any device memory.  It is meant for callers that cannot call cudaMalloc at
// the point where they need the check: for example a solver loop that owns all device
// memory through its own pool and forbids the runtime allocator, or a job that runs the
// GPU so close to full that an allocation at the end of a long solve could fail.
//
// Scratch: the per-block partial sums live in one file-scope device array shared by every
// call on a device (and held by every GPU that loads the library until the process exits).
// Its size fixes the largest matrix: kRowsPerBlock rows per block and at most kMaxBlocks
// blocks, i.e. kMaxRows rows.  Larger matrices are rejected with APF_ERR_CAPACITY.
// Each call writes every partial slot it later reads, so nothing has to be cleared between
// calls; calls whose work overlaps on the GPU (different streams, no ordering) race on the
// shared array and must not be issued.  The first call on a device looks the array up and
// loads this file's kernels (which may take device memory for their code); make it before
// any stream capture, and before the point where nothing may be allocated any more.
#include <mutex>

#include "apf_internal.hpp"

namespace
{
    constexpr int kRowsPerBlock = 4096;
    constexpr int kMaxBlocks = 4096;
    constexpr long long kMaxRows = static_cast<long long>(kRowsPerBlock) * kMaxBlocks; // 16,777,216
    constexpr int kThreads = 256;

    // [0, kMaxBlocks): partial sums of r_i^2; [kMaxBlocks, 2 kMaxBlocks): of b_i^2;
    // [2 kMaxBlocks, 2 kMaxBlocks + 2): absolute and relative residual of the last call
    static __device__ __align__(256) double g_residual_scratch[2 * kMaxBlocks + 2];

    template<int G>
    __global__ void residual_partials(int rows, const int* __restrict__ rp, const int* __restrict__ ci,
                                      const double* __restrict__ va, const double* __restrict__ x,
                                      const double* __restrict__ b, double* scratch);
    __global__ void residual_finish(int nblocks, double* scratch);

    // Device address of g_residual_scratch, looked up once per device.  The same one-time
    // set-up also loads the five kernels of this file onto the device: under CUDA's lazy
    // module loading a kernel's code is otherwise loaded (and device memory taken for it) at
    // its first launch, so a later call that picks another lanes-per-row variant could still
    // allocate.  After the first call on a device nothing here allocates.
    std::mutex g_setup_mutex;
    double* g_scratch_addr[64] = {};

    template<class K>
    void force_load(K kernel)
    {
        cudaFuncAttributes attr{};
        const cudaError_t e = cudaFuncGetAttributes(&attr, kernel);
        if (e != cudaSuccess)
            throw apf::Error(APF_ERR_CUDA, std::string("cudaFuncGetAttributes(residual kernel): ") +
                                               cudaGetErrorString(e));
    }

    double* scratch_address(int device)
    {
        apf::require(device >= 0 && device < 64, APF_ERR_INVALID, "device index out of range");
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[device])
        {
            void* p = nullptr;
            // the context's device is current here (the C-ABI layer made it so)
            const cudaError_t e = cudaGetSymbolAddress(&p, g_residual_scratch);
            if (e != cudaSuccess || p == nullptr)
                throw apf::Error(APF_ERR_CUDA, std::string("cudaGetSymbolAddress(residual scratch): ") +
                                                   cudaGetErrorString(e));
            force_load(residual_partials<4>);
            force_load(residual_partials<8>);
            force_load(residual_partials<16>);
            force_load(residual_partials<32>);
            force_load(residual_finish);
            g_scratch_addr[device] = static_cast<double*>(p);
        }
        return g_scratch_addr[device];
    }

    // One block per kRowsPerBlock rows; G lanes per row (same row summation as the
    // library's residual kernel), block-level partial sums written to the scratch.
    template<int G>
    __global__ void residual_partials(int rows, const int* __restrict__ rp, const int* __restrict__ ci,
                                      const double* __restrict__ va, const double* __restrict__ x,
                                      const double* __restrict__ b, double* scratch)
    {
        constexpr int RPW = 32 / G;
        __shared__ double s_rr[kThreads / 32], s_bb[kThreads / 32];
        const int lane = threadIdx.x & (G - 1);
        const int sub = (threadIdx.x & 31) / G;
        const int warp = threadIdx.x >> 5;
        const long long first = static_cast<long long>(blockIdx.x) * kRowsPerBlock;
        const long long last = min(first + kRowsPerBlock, static_cast<long long>(rows));
        double rr = 0.0, bb = 0.0;
        for (long long base = first + warp * RPW; base < last; base += (kThreads / 32) * RPW)
        {
            const long long r = base + sub;
            double sum = 0.0;
            if (r < last)
            {
                const int s0 = rp[r], e = rp[r + 1];
                for (int k = s0 + lane; k < e; k += G)
                    sum += va[k] * __ldg(x + ci[k]);
            }
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1)
                sum += __shfl_down_sync(0xffffffffu, sum, o, G);
            if (lane == 0 && r < last)
            {
                const double ri = b[r] - sum;
                rr += ri * ri;
                bb += b[r] * b[r];
            }
        }
        for (int o = 16; o > 0; o >>= 1)
        {
            rr += __shfl_down_sync(0xffffffffu, rr, o);
            bb += __shfl_down_sync(0xffffffffu, bb, o);
        }
        if ((threadIdx.x & 31) == 0)
        {
            s_rr[warp] = rr;
            s_bb[warp] = bb;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            double t = 0.0, u = 0.0;
            for (int w = 0; w < kThreads / 32; ++w)
            {
                t += s_rr[w];
                u += s_bb[w];
            }
            scratch[blockIdx.x] = t;
            scratch[kMaxBlocks + blockIdx.x] = u;
        }
    }

    // fixed-order sum of the partials written by this call
    __global__ void residual_finish(int nblocks, double* scratch)
    {
        if (threadIdx.x != 0 || blockIdx.x != 0)
            return;
        double rr = 0.0, bb = 0.0;
        for (int i = 0; i < nblocks; ++i)
        {
            rr += scratch[i];
            bb += scratch[kMaxBlocks + i];
        }
        const double rn = sqrt(rr), bn = sqrt(bb);
        scratch[2 * kMaxBlocks] = rn;
        scratch[2 * kMaxBlocks + 1] = rn / (bn > 0.0 ? bn : 1.0); // zero rhs: report the absolute norm
    }
}

namespace apf
{
    void true_residual_noalloc(int device, cudaStream_t s, int rows, const int* row_ptr, const int* col_idx,
                               const double* values, const double* x, const double* b, double* absolute,
                               double* relative)
    {
        require(rows >= 0, APF_ERR_INVALID, "negative row count");
        require(rows <= kMaxRows, APF_ERR_CAPACITY,
                "apf_true_residual_noalloc: " + std::to_string(rows) + " rows exceed the fixed scratch limit of " +
                    std::to_string(kMaxRows) + " rows");
        require(rows == 0 || (row_ptr && col_idx && values && x && b), APF_ERR_INVALID, "null input pointer");
        double* scratch = scratch_address(device);
        const int nblocks = rows == 0 ? 1 : static_cast<int>((rows + kRowsPerBlock - 1) / kRowsPerBlock);
        if (rows > 0)
        {
            // the same lanes-per-row choice as the library's residual kernel
            int nnz = 0;
            APF_CUDA(cudaMemcpyAsync(&nnz, row_ptr + rows, sizeof(int), cudaMemcpyDeviceToHost, s));
            APF_CUDA(cudaStreamSynchronize(s));
            const double avg = static_cast<double>(nnz) / rows;
            APF_KERNEL("residual_partials_noalloc", s);
            if (avg <= 6)
                residual_partials<4><<<nblocks, kThreads, 0, s>>>(rows, row_ptr, col_idx, values, x, b, scratch);
            else if (avg <= 14)
                residual_partials<8><<<nblocks, kThreads, 0, s>>>(rows, row_ptr, col_idx, values, x, b, scratch);
            else if (avg <= 40)
                residual_partials<16><<<nblocks, kThreads, 0, s>>>(rows, row_ptr, col_idx, values, x, b, scratch);
            else
                residual_partials<32><<<nblocks, kThreads, 0, s>>>(rows, row_ptr, col_idx, values, x, b, scratch);
        }
        else
        {
            APF_CUDA(cudaMemsetAsync(scratch, 0, 2 * sizeof(double), s));
            APF_CUDA(cudaMemsetAsync(scratch + kMaxBlocks, 0, sizeof(double), s));
        }
        {
            APF_KERNEL("residual_finish_noalloc", s);
            residual_finish<<<1, 32, 0, s>>>(nblocks, scratch);
        }
        APF_CUDA(cudaGetLastError());
        double out[2] = {0.0, 0.0};
        APF_CUDA(cudaMemcpyAsync(out, scratch + 2 * kMaxBlocks, sizeof(out), cudaMemcpyDeviceToHost, s));
        APF_CUDA(cudaStreamSynchronize(s));
        if (absolute)
            *absolute = out[0];
        if (relative)
            *relative = out[1];
    }
}
