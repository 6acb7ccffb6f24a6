// Warp-per-row sparse accumulation helpers: a shared-memory hash set of a row's distinct
// columns, segment search over flattened candidate lists, and sums in candidate order.
#pragma once

#include <cuda_runtime.h>

namespace apf
{
    // candidate segments flattened per pass, and the per-warp shared memory of the segment
    // offsets (int[kSeg + 2]) and staged values (double[32]), rounded up to 16 bytes so that
    // every warp's region starts 16-byte aligned
    constexpr int kSeg = 256;
    constexpr int kRowExtra = (((kSeg + 2) * 4 + 32 * 8) + 15) / 16 * 16;

    __device__ __forceinline__ unsigned hash_slot(int col, int hbits)
    {
        return (static_cast<unsigned>(col) * 2654435761u) >> (32 - hbits);
    }

    __device__ __forceinline__ void hash_insert(int* tkeys, int col, int hbits)
    {
        const int H = 1 << hbits;
        unsigned h = hash_slot(col, hbits);
        while (true)
        {
            const int prev = atomicCAS(tkeys + h, -1, col);
            if (prev == -1 || prev == col)
                break;
            h = (h + 1) & (H - 1);
        }
    }

    // insert col; true when it was not in the table yet
    __device__ __forceinline__ bool hash_insert_new(int* tkeys, int col, int hbits)
    {
        const int H = 1 << hbits;
        unsigned h = hash_slot(col, hbits);
        while (true)
        {
            const int prev = atomicCAS(tkeys + h, -1, col);
            if (prev == -1)
                return true;
            if (prev == col)
                return false;
            h = (h + 1) & (H - 1);
        }
    }

    // slot of col in the table, inserting it when absent (fresh = it was absent)
    __device__ __forceinline__ int hash_slot_of(int* tkeys, int col, int hbits, bool& fresh)
    {
        const int H = 1 << hbits;
        unsigned h = hash_slot(col, hbits);
        while (true)
        {
            const int prev = atomicCAS(tkeys + h, -1, col);
            if (prev == -1 || prev == col)
            {
                fresh = prev == -1;
                return static_cast<int>(h);
            }
            h = (h + 1) & (H - 1);
        }
    }

    __device__ __forceinline__ int hash_rank(const int* tkeys, const int* tranks, int col, int hbits)
    {
        const int H = 1 << hbits;
        unsigned h = hash_slot(col, hbits);
        while (tkeys[h] != col)
            h = (h + 1) & (H - 1);
        return tranks[h];
    }

    // segment index lo with seg[lo] <= t < seg[lo + 1]
    __device__ __forceinline__ int find_segment(const int* seg, int cnt, int t)
    {
        int lo = 0, hi = cnt;
        while (hi - lo > 1)
        {
            const int mid = (lo + hi) >> 1;
            if (seg[mid] <= t)
                lo = mid;
            else
                hi = mid;
        }
        return lo;
    }

    // add each ok lane's value to acc[rank] in lane order (the lowest lane of a rank adds
    // its group's values one by one)
    __device__ __forceinline__ void ordered_add(double* acc, double* stage, bool ok, int r, double v, int lane)
    {
        const unsigned grp = __match_any_sync(0xffffffffu, ok ? r : -1 - lane);
        stage[lane] = v;
        __syncwarp();
        if (ok && lane == __ffs(grp) - 1)
        {
            double a = acc[r];
            for (unsigned m = grp; m; m &= m - 1)
                a += stage[__ffs(m) - 1];
            acc[r] = a;
        }
        __syncwarp();
    }
}
