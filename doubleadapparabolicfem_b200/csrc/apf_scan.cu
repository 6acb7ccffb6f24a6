// Exclusive prefix sum of int32 counts into int32 offsets (three-phase block scan).
#include "apf_internal.hpp"

namespace apf
{
    namespace
    {
        constexpr int kScanBlock = 1024;

        __global__ void scan_block_sums(const int* __restrict__ in, int n, long long* __restrict__ sums)
        {
            __shared__ long long warp_sums[32];
            const int i = blockIdx.x * kScanBlock + threadIdx.x;
            long long v = i < n ? in[i] : 0;
            for (int o = 16; o > 0; o >>= 1)
                v += __shfl_down_sync(0xffffffffu, v, o);
            if ((threadIdx.x & 31) == 0)
                warp_sums[threadIdx.x >> 5] = v;
            __syncthreads();
            if (threadIdx.x < 32)
            {
                long long w = warp_sums[threadIdx.x];
                for (int o = 16; o > 0; o >>= 1)
                    w += __shfl_down_sync(0xffffffffu, w, o);
                if (threadIdx.x == 0)
                    sums[blockIdx.x] = w;
            }
        }

        // Sequential exclusive scan of the (few) block sums in one thread block.
        __global__ void scan_sums_serial(long long* __restrict__ sums, int nb, long long* __restrict__ total)
        {
            __shared__ long long buf[kScanBlock];
            long long carry = 0;
            for (int base = 0; base < nb; base += kScanBlock)
            {
                const int i = base + threadIdx.x;
                long long v = i < nb ? sums[i] : 0;
                buf[threadIdx.x] = v;
                __syncthreads();
                for (int o = 1; o < kScanBlock; o <<= 1)
                {
                    long long add = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
                    __syncthreads();
                    buf[threadIdx.x] += add;
                    __syncthreads();
                }
                if (i < nb)
                    sums[i] = carry + buf[threadIdx.x] - v;
                const long long block_total = buf[kScanBlock - 1];
                __syncthreads();
                carry += block_total;
            }
            if (threadIdx.x == 0)
                *total = carry;
        }

        __global__ void scan_apply(const int* __restrict__ in, int n, const long long* __restrict__ sums,
                                   const long long* __restrict__ total, int* __restrict__ out)
        {
            __shared__ long long warp_tot[32];
            const int i = blockIdx.x * kScanBlock + threadIdx.x;
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            long long v = i < n ? in[i] : 0;
            long long x = v;
            for (int o = 1; o < 32; o <<= 1)
            {
                const long long y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) warp_tot[wid] = x;
            __syncthreads();
            if (wid == 0)
            {
                long long w = warp_tot[lane];
                for (int o = 1; o < 32; o <<= 1)
                {
                    const long long y = __shfl_up_sync(0xffffffffu, w, o);
                    if (lane >= o) w += y;
                }
                warp_tot[lane] = w;
            }
            __syncthreads();
            const long long warp_prefix = wid > 0 ? warp_tot[wid - 1] : 0;
            const long long excl = sums[blockIdx.x] + warp_prefix + x - v;
            if (i < n)
                out[i] = static_cast<int>(excl);
            if (i == n - 1 || (n == 0 && i == 0))
                out[n] = static_cast<int>(*total);
        }
    }

    long long exclusive_scan(const int* counts, int* out, int n, cudaStream_t s)
    {
        const int nb = n > 0 ? (n + kScanBlock - 1) / kScanBlock : 1;
        DeviceBuffer<long long> sums(static_cast<std::size_t>(nb) + 1, s);
        long long* total = sums.get() + nb;
        if (n == 0)
        {
            APF_CUDA(cudaMemsetAsync(out, 0, sizeof(int), s));
            return 0;
        }
        {
            APF_KERNEL("scan_block_sums", s);
            scan_block_sums<<<nb, kScanBlock, 0, s>>>(counts, n, sums.get());
        }
        {
            APF_KERNEL("scan_sums_serial", s);
            scan_sums_serial<<<1, kScanBlock, 0, s>>>(sums.get(), nb, total);
        }
        {
            APF_KERNEL("scan_apply", s);
            scan_apply<<<nb, kScanBlock, 0, s>>>(counts, n, sums.get(), total, out);
        }
        APF_CUDA(cudaGetLastError());
        long long h_total = 0;
        APF_CUDA(cudaMemcpyAsync(&h_total, total, sizeof(long long), cudaMemcpyDeviceToHost, s));
        APF_CUDA(cudaStreamSynchronize(s));
        if (h_total > 0x7fffffffll)
            throw Error(APF_ERR_CAPACITY, "exclusive_scan: total exceeds int32 range");
        return h_total;
    }
}
