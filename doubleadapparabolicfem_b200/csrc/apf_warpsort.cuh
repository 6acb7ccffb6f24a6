// Warp-level sort of 64-bit keys in shared memory (used by the row-gather kernels).
#pragma once

#include <cuda_runtime.h>

namespace apf
{
    // key = col (high 32) | seq (17 bits) | slot (15 bits): sorting by key orders the
    // candidates of a row by column and, within a column, by a deterministic sequence
    // number; the slot points back to the candidate's value.
    constexpr int kSlotBits = 15;
    constexpr int kSeqBits = 17;

    __device__ __forceinline__ unsigned long long make_key(int col, int seq, int slot)
    {
        return (static_cast<unsigned long long>(static_cast<unsigned>(col)) << 32) |
               (static_cast<unsigned long long>(seq & ((1 << kSeqBits) - 1)) << kSlotBits) |
               static_cast<unsigned long long>(slot);
    }

    // In-place ascending bitonic sort of n (power of two) keys by one warp.
    __device__ __forceinline__ void warp_bitonic_sort(unsigned long long* keys, int n)
    {
        const int lane = threadIdx.x & 31;
        for (int k = 2; k <= n; k <<= 1)
        {
            for (int j = k >> 1; j > 0; j >>= 1)
            {
                for (int i = lane; i < n; i += 32)
                {
                    const int ixj = i ^ j;
                    if (ixj > i)
                    {
                        const unsigned long long a = keys[i], b = keys[ixj];
                        const bool up = (i & k) == 0;
                        if ((a > b) == up)
                        {
                            keys[i] = b;
                            keys[ixj] = a;
                        }
                    }
                }
                __syncwarp();
            }
        }
    }

    __device__ __forceinline__ int next_pow2(int n)
    {
        int p = 1;
        while (p < n)
            p <<= 1;
        return p;
    }
}
