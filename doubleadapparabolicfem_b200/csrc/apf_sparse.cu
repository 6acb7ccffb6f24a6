// Sparse/vector building blocks (see apf_sparse.cuh).
#include <algorithm>
#include <type_traits>

#include "apf_sparse.cuh"
#include "apf_warpsort.cuh"
#include "apf_rowhash.cuh"

namespace apf
{
    namespace
    {
        int blocks_for(long long work, int threads, int cap = 148 * 32)
        {
            long long g = (work + threads - 1) / threads;
            return static_cast<int>(std::max<long long>(1, std::min<long long>(g, cap)));
        }

        // G lanes per row; the row loop is warp-uniform so the shuffles see all 32 lanes.
        // Each lane keeps four predicated loads of the row in flight per step (the row
        // pointer, column, value and x gathers form one dependent chain per step, so the
        // number of steps per row, not the bytes, sets the time on L2-resident levels).
        // MODE 0: y = alpha A x + beta y;  1: y = b - A x;  2: y = x + alpha dinv (b - A x);
        // 3: y = alpha A x and z = beta dinv y (a restriction fused with the coarse level's
        // first damped-Jacobi step from zero)
        template<int G, int MODE, class V = double>
        __global__ void __launch_bounds__(256) spmv_kernel(int rows, const int* __restrict__ rp, const int* __restrict__ ci,
                                                           const V* __restrict__ va, const double* __restrict__ x,
                                                           const double* __restrict__ b, double* __restrict__ y,
                                                           double alpha, double beta, const double* __restrict__ dinv,
                                                           double* __restrict__ z)
        {
            constexpr int RPW = 32 / G; // rows per warp and step
            const int lane = threadIdx.x & (G - 1);
            const int sub = (threadIdx.x & 31) / G;
            const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
            const long long nwarps = (gridDim.x * (long long)blockDim.x) >> 5;
            for (long long base = warp * RPW; base < rows; base += nwarps * RPW)
            {
                const long long r = base + sub;
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                if (r < rows)
                {
                    const int e = rp[r + 1];
                    for (int k = rp[r] + lane; k < e; k += 4 * G)
                    {
                        const bool p1 = k + G < e, p2 = k + 2 * G < e, p3 = k + 3 * G < e;
                        const int c0 = ci[k];
                        const int c1 = p1 ? ci[k + G] : 0;
                        const int c2 = p2 ? ci[k + 2 * G] : 0;
                        const int c3 = p3 ? ci[k + 3 * G] : 0;
                        const double v0 = static_cast<double>(va[k]);
                        const double v1 = p1 ? static_cast<double>(va[k + G]) : 0.0;
                        const double v2 = p2 ? static_cast<double>(va[k + 2 * G]) : 0.0;
                        const double v3 = p3 ? static_cast<double>(va[k + 3 * G]) : 0.0;
                        s0 += v0 * __ldg(x + c0);
                        if (p1)
                            s1 += v1 * __ldg(x + c1);
                        if (p2)
                            s2 += v2 * __ldg(x + c2);
                        if (p3)
                            s3 += v3 * __ldg(x + c3);
                    }
                }
                double sum = (s0 + s1) + (s2 + s3);
#pragma unroll
                for (int o = G / 2; o > 0; o >>= 1)
                    sum += __shfl_down_sync(0xffffffffu, sum, o, G);
                if (lane == 0 && r < rows)
                {
                    if (MODE == 1)
                        y[r] = b[r] - sum;
                    else if (MODE == 2)
                        y[r] = x[r] + alpha * dinv[r] * (b[r] - sum);
                    else if (MODE == 3)
                    {
                        const double v = alpha * sum;
                        y[r] = v;
                        z[r] = beta * dinv[r] * v;
                    }
                    else
                        y[r] = beta == 0.0 ? alpha * sum : alpha * sum + beta * y[r];
                }
            }
        }

        // SELL-32 SpMV: one thread per row, one warp per slice (same MODEs as spmv_kernel).
        // Bounded to 32 registers (eight blocks of 256 threads per SM): the kernel is
        // latency-bound and warps in flight set its bandwidth; the few spilled values live
        // in L1.  Measured at outer level 6 against 40 registers and six blocks: K SpMV 0.86
        // -> 0.94 of the HBM copy bandwidth, finest-level sweeps 0.59 -> 0.64; a variant
        // with two accumulators and no spills lost both gains.  The f32 operators (the
        // V-cycle levels) use the paired layout of sell_fill: each load request carries two
        // entries (8 bytes), as the f64 operator's values do; with the group loop kept
        // rolled that took the finest-level sweeps from 0.68 to 0.80 of the copy bandwidth
        // on the locally refined workload (the scalar layout: 68-72 bytes of spills, the
        // paired one 24-28).
        template<int MODE, class V>
        __global__ void __launch_bounds__(256, 8) sell_kernel(int rows, int slices, const int* __restrict__ sp,
                                                           const int* __restrict__ col, const V* __restrict__ val,
                                                           const double* __restrict__ x, const double* __restrict__ b,
                                                           double* __restrict__ y, double alpha, double beta,
                                                           const double* __restrict__ dinv, const int* __restrict__ perm,
                                                           double* __restrict__ z)
        {
            const int lane = threadIdx.x & 31;
            const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            const int nwarps = (gridDim.x * blockDim.x) >> 5;
            for (int sl = warp; sl < slices; sl += nwarps)
            {
                const int base = sp[sl];
                const int width = (sp[sl + 1] - base) >> 5;
                const V* v = val + base + lane;
                const int* c = col + base + lane;
                // the row index (and, for y = a A x + b y, the old y) is requested before
                // the loop, so its latency overlaps the matrix loads; the sweeps' operands
                // b, x and the weights are read after it (hoisting them too cost the
                // sweeps more in registers than it saved in latency)
                const int rs = sl * 32 + lane;
                const bool live = rs < rows;
                const int r = live ? (perm ? __ldg(perm + rs) : rs) : 0;
                double pre_y = 0.0;
                if (MODE == 0 && live && beta != 0.0)
                    pre_y = y[r];
                // four independent load chains in flight per thread; the matrix streams
                // through once (evict-first loads), x stays cached for the gathers
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                int j = 0;
                if constexpr (std::is_same_v<V, float>)
                {
                    // paired f32 layout (even width): one 8-byte column load and one 8-byte
                    // value load per two entries, twice the bytes per outstanding request of
                    // the scalar layout at the same register count
                    const int2* cp = reinterpret_cast<const int2*>(col + base) + lane;
                    const float2* vp = reinterpret_cast<const float2*>(val + base) + lane;
#pragma unroll 1
                    for (; j + 3 < width; j += 4)
                    {
                        const int2 ca = __ldcs(cp + 16 * j), cb = __ldcs(cp + 16 * j + 32);
                        const float2 va = __ldcs(vp + 16 * j), vb = __ldcs(vp + 16 * j + 32);
                        const double x0 = __ldg(x + ca.x), x1 = __ldg(x + ca.y), x2 = __ldg(x + cb.x),
                                     x3 = __ldg(x + cb.y);
                        s0 += static_cast<double>(va.x) * x0;
                        s1 += static_cast<double>(va.y) * x1;
                        s2 += static_cast<double>(vb.x) * x2;
                        s3 += static_cast<double>(vb.y) * x3;
                    }
                    if (j < width)
                    {
                        const int2 ca = __ldcs(cp + 16 * j);
                        const float2 va = __ldcs(vp + 16 * j);
                        s0 += static_cast<double>(va.x) * __ldg(x + ca.x);
                        s0 += static_cast<double>(va.y) * __ldg(x + ca.y);
                    }
                }
                else
                {
                    for (; j + 3 < width; j += 4)
                    {
                        const int c0 = __ldcs(c + 32 * j), c1 = __ldcs(c + 32 * j + 32);
                        const int c2 = __ldcs(c + 32 * j + 64), c3 = __ldcs(c + 32 * j + 96);
                        const V v0 = __ldcs(v + 32 * j), v1 = __ldcs(v + 32 * j + 32);
                        const V v2 = __ldcs(v + 32 * j + 64), v3 = __ldcs(v + 32 * j + 96);
                        const double x0 = __ldg(x + c0), x1 = __ldg(x + c1), x2 = __ldg(x + c2), x3 = __ldg(x + c3);
                        s0 += static_cast<double>(v0) * x0;
                        s1 += static_cast<double>(v1) * x1;
                        s2 += static_cast<double>(v2) * x2;
                        s3 += static_cast<double>(v3) * x3;
                    }
                    for (; j < width; ++j)
                        s0 += static_cast<double>(__ldcs(v + 32 * j)) * __ldg(x + __ldcs(c + 32 * j));
                }
                const double sum = (s0 + s1) + (s2 + s3);
                if (live)
                {
                    if (MODE == 1)
                        y[r] = b[r] - sum;
                    else if (MODE == 2)
                        y[r] = x[r] + alpha * dinv[r] * (b[r] - sum);
                    else if (MODE == 3)
                    {
                        const double v = alpha * sum;
                        y[r] = v;
                        z[r] = beta * dinv[r] * v;
                    }
                    else
                        y[r] = beta == 0.0 ? alpha * sum : alpha * sum + beta * pre_y;
                }
            }
        }

        __global__ void to_f32_kernel(long long n, const double* __restrict__ a, float* __restrict__ b)
        {
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
                b[i] = static_cast<float>(a[i]);
        }

        // slice widths x 32 (element counts per slice)
        // rows sorted by decreasing length inside windows of kSellWindow rows (ties by row
        // index): perm[sorted position] = row.  One block of 256 threads per window, bitonic
        // sort of (length, row) keys in shared memory.
        constexpr int kSellWindow = 512;
        __global__ void __launch_bounds__(256) sell_sort_rows(int rows, const int* __restrict__ rp, int* __restrict__ perm)
        {
            __shared__ unsigned long long key[kSellWindow];
            const int w0 = blockIdx.x * kSellWindow;
            for (int k = threadIdx.x; k < kSellWindow; k += blockDim.x)
            {
                const int r = w0 + k;
                const unsigned len = r < rows ? static_cast<unsigned>(rp[r + 1] - rp[r]) : 0u;
                // descending length first, real rows before the window's padding, then index
                const unsigned hi = r < rows ? 0x7fffffffu - min(len, 0x7ffffffeu) : 0xffffffffu;
                key[k] = (static_cast<unsigned long long>(hi) << 32) | static_cast<unsigned>(k);
            }
            __syncthreads();
            for (int size = 2; size <= kSellWindow; size <<= 1)
                for (int stride = size >> 1; stride > 0; stride >>= 1)
                {
                    for (int t = threadIdx.x; t < kSellWindow / 2; t += blockDim.x)
                    {
                        const int i = 2 * t - (t & (stride - 1));
                        const int j = i + stride;
                        const bool up = (i & size) == 0;
                        const unsigned long long a = key[i], b = key[j];
                        if ((a > b) == up)
                        {
                            key[i] = b;
                            key[j] = a;
                        }
                    }
                    __syncthreads();
                }
            for (int k = threadIdx.x; k < kSellWindow; k += blockDim.x)
                if (w0 + k < rows)
                    perm[w0 + k] = w0 + static_cast<int>(key[k] & 0xffffffffu);
        }

        // even = 1: widths rounded up to an even count (the paired f32 layout)
        __global__ void sell_count(int rows, int slices, const int* __restrict__ rp, const int* __restrict__ perm,
                                   int* __restrict__ cnt, int even)
        {
            const int lane = threadIdx.x & 31;
            const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            const int nwarps = (gridDim.x * blockDim.x) >> 5;
            for (int sl = warp; sl < slices; sl += nwarps)
            {
                const int rs = sl * 32 + lane;
                const int r = rs < rows ? perm[rs] : 0;
                int len = rs < rows ? rp[r + 1] - rp[r] : 0;
                for (int o = 16; o > 0; o >>= 1)
                    len = max(len, __shfl_xor_sync(0xffffffffu, len, o));
                if (lane == 0)
                    cnt[sl] = 32 * (even ? (len + 1) & ~1 : len);
            }
        }

        template<class V>
        __global__ void sell_fill(int rows, int slices, const int* __restrict__ rp, const int* __restrict__ ci,
                                  const double* __restrict__ va, const int* __restrict__ sp, const int* __restrict__ perm,
                                  int* __restrict__ col, V* __restrict__ val)
        {
            const int lane = threadIdx.x & 31;
            const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            const int nwarps = (gridDim.x * blockDim.x) >> 5;
            for (int sl = warp; sl < slices; sl += nwarps)
            {
                const int base = sp[sl];
                const int width = (sp[sl + 1] - base) >> 5;
                const int rs = sl * 32 + lane;
                const int r = rs < rows ? perm[rs] : 0;
                const int b = rs < rows ? rp[r] : 0;
                const int len = rs < rows ? rp[r + 1] - b : 0;
                for (int j = 0; j < width; ++j)
                {
                    // f64: entry j of the slice's 32 rows contiguous; f32: pairs of entries
                    // (2q, 2q + 1) of a row adjacent, pair q of the 32 rows contiguous
                    const int o = std::is_same_v<V, float> ? base + 64 * (j >> 1) + 2 * lane + (j & 1)
                                                           : base + 32 * j + lane;
                    col[o] = j < len ? ci[b + j] : 0;
                    val[o] = static_cast<V>(j < len ? va[b + j] : 0.0);
                }
            }
        }

        __global__ void dot_partials(int n, const double* __restrict__ a, const double* __restrict__ b,
                                     double* __restrict__ partials)
        {
            __shared__ double ws[kRedThreads / 32];
            double s = 0.0;
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
                s += b ? a[i] * b[i] : a[i];
            for (int o = 16; o > 0; o >>= 1)
                s += __shfl_down_sync(0xffffffffu, s, o);
            if ((threadIdx.x & 31) == 0)
                ws[threadIdx.x >> 5] = s;
            __syncthreads();
            if (threadIdx.x == 0)
            {
                double t = 0.0;
                for (int w = 0; w < kRedThreads / 32; ++w)
                    t += ws[w];
                partials[blockIdx.x] = t;
            }
        }

        __global__ void sum_partials(int n, const double* __restrict__ partials, double* __restrict__ out)
        {
            __shared__ double ws[32];
            double s = 0.0;
            for (int i = threadIdx.x; i < n; i += blockDim.x)
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
                *out = t;
            }
        }

        __global__ void axpby_kernel(int n, double a, const double* __restrict__ x, double b, double* __restrict__ y)
        {
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
                y[i] = a * x[i] + (b == 0.0 ? 0.0 : b * y[i]);
        }

        __global__ void fill_kernel(int n, double v, double* __restrict__ y)
        {
            for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
                y[i] = v;
        }

        __global__ void inv_diag_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                        const double* __restrict__ va, double* __restrict__ inv)
        {
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
            {
                double d = 0.0;
                for (int k = rp[r]; k < rp[r + 1]; ++k)
                    if (ci[k] == r)
                        d += va[k];
                inv[r] = d != 0.0 ? 1.0 / d : 0.0;
            }
        }

        // ---- sparse product C = A B ---------------------------------------------
        // candidate products per row of A B (cand[r]) and their maximum (*out)
        __global__ void spgemm_bound(int rows, const int* __restrict__ ap, const int* __restrict__ ac,
                                     const int* __restrict__ bp, int* __restrict__ out, int* __restrict__ cand)
        {
            int m = 0;
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
            {
                int n = 0;
                for (int k = ap[r]; k < ap[r + 1]; ++k)
                    n += bp[ac[k] + 1] - bp[ac[k]];
                m = max(m, n);
                cand[r] = n;
            }
            for (int o = 16; o > 0; o >>= 1)
                m = max(m, __shfl_down_sync(0xffffffffu, m, o));
            if ((threadIdx.x & 31) == 0)
                atomicMax(out, m);
        }

        struct GemmArgs
        {
            int rows;
            const int *ap, *ac;
            const double* av;
            const int *bp, *bc;
            const double* bv;
            int* count;
            const int* cp;
            int* cc;
            double* cv;
            const int* list; // rows to process (null: all rows)
            int nlist;
        };

        // One warp per row of A B with at most CAP candidate products, processed 32 at a time
        // in generation order (A's row order, then B's row order) with the warp's lanes spread
        // over all of them (the B rows of up to kSeg A entries are flattened through a
        // prefix sum of their lengths).  The distinct columns go through a shared-memory hash
        // set (at most half full) and only those are sorted; each product is then added to
        // its column's accumulator in generation order (within a group of 32, the lowest lane
        // of each column adds its group's products in lane order), so the sums are those of a
        // stable sort of the candidates.  Output: the row's sorted distinct columns and sums
        // at cp[row], their number in count[row].
        // Shared memory per warp: table keys int[2 CAP], ranks int[2 CAP], sorted keys /
        // accumulators 8 B x CAP, segment offsets int[kSeg + 2], staged products double[32].

        template<int CAP>
        __global__ void __launch_bounds__(256) spgemm_rows(GemmArgs A)
        {
            extern __shared__ unsigned char smem_raw[];
            const int warps = blockDim.x >> 5;
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            unsigned char* mine = smem_raw + (size_t)w * (24 * CAP + kRowExtra);
            int* tkeys = reinterpret_cast<int*>(mine);
            int* tranks = tkeys + 2 * CAP;
            unsigned long long* ukeys = reinterpret_cast<unsigned long long*>(tranks + 2 * CAP);
            double* acc = reinterpret_cast<double*>(ukeys);
            int* seg = reinterpret_cast<int*>(ukeys + CAP);
            double* stage = reinterpret_cast<double*>(seg + kSeg + 2);
            const int nrows = A.list ? A.nlist : A.rows;
            for (int idx = blockIdx.x * warps + w; idx < nrows; idx += gridDim.x * warps)
            {
                const int row = A.list ? A.list[idx] : idx;
                const int ab = A.ap[row], ae = A.ap[row + 1];
                int n = 0;
                for (int k = ab; k < ae; ++k)
                    n += A.bp[A.ac[k] + 1] - A.bp[A.ac[k]];
                // table at most half full: 2 min(n, CAP) slots (CAP bounds the distinct columns;
                // a row with more is marked count = -1 and left for a larger CAP)
                int hbits = 6;
                while ((1 << hbits) < 2 * min(n, CAP))
                    ++hbits;
                const int H = 1 << hbits;
                for (int t = lane; t < H; t += 32)
                    tkeys[t] = -1;
                __syncwarp();
                // every product (ok, column, value) in generation order, 32 lanes at a time
                auto for_each = [&](auto&& f) {
                    for (int kb = ab; kb < ae; kb += kSeg)
                    {
                        const int cnt = min(ae - kb, kSeg);
                        for (int i = lane; i < cnt; i += 32)
                            seg[i + 1] = A.bp[A.ac[kb + i] + 1] - A.bp[A.ac[kb + i]];
                        __syncwarp();
                        for (int i0 = 0, carry = 0; i0 < cnt; i0 += 32)
                        {
                            int v = i0 + lane < cnt ? seg[i0 + lane + 1] : 0;
                            for (int o = 1; o < 32; o <<= 1)
                            {
                                const int u = __shfl_up_sync(0xffffffffu, v, o);
                                if (lane >= o)
                                    v += u;
                            }
                            __syncwarp();
                            if (i0 + lane < cnt)
                                seg[i0 + lane + 1] = carry + v;
                            carry += __shfl_sync(0xffffffffu, v, 31);
                            __syncwarp();
                        }
                        if (lane == 0)
                            seg[0] = 0;
                        __syncwarp();
                        const int nb = seg[cnt];
                        for (int t0 = 0; t0 < nb; t0 += 32)
                        {
                            const int t = t0 + lane;
                            const bool ok = t < nb;
                            int col = 0;
                            double v = 0.0;
                            if (ok)
                            {
                                const int i = find_segment(seg, cnt, t);
                                const int k = kb + i;
                                const int q = A.bp[A.ac[k]] + (t - seg[i]);
                                col = A.bc[q];
                                v = A.av[k] * A.bv[q];
                            }
                            f(ok, col, v);
                        }
                        __syncwarp();
                    }
                };
                int distinct = 0;
                bool overflow = false;
                for_each([&](bool ok, int col, double) {
                    const bool fresh = ok && !overflow && hash_insert_new(tkeys, col, hbits);
                    distinct += __popc(__ballot_sync(0xffffffffu, fresh));
                    overflow = overflow || distinct > CAP;
                });
                __syncwarp();
                if (overflow)
                {
                    if (lane == 0)
                        A.count[row] = -1;
                    __syncwarp();
                    continue;
                }
                // compact and sort the distinct columns: key = column (high) | table slot (low)
                int u = 0;
                for (int t0 = 0; t0 < H; t0 += 32)
                {
                    const int t = t0 + lane;
                    const int key = tkeys[t];
                    const unsigned m = __ballot_sync(0xffffffffu, key != -1);
                    if (key != -1)
                        ukeys[u + __popc(m & ((1u << lane) - 1))] =
                            (static_cast<unsigned long long>(static_cast<unsigned>(key)) << 32) | static_cast<unsigned>(t);
                    u += __popc(m);
                }
                const int np = next_pow2(u);
                for (int k = u + lane; k < np; k += 32)
                    ukeys[k] = ~0ull;
                __syncwarp();
                warp_bitonic_sort(ukeys, np);
                const int base = A.cp[row];
                for (int k = lane; k < u; k += 32)
                {
                    const unsigned long long key = ukeys[k];
                    tranks[static_cast<unsigned>(key)] = k;
                    A.cc[base + k] = static_cast<int>(key >> 32);
                }
                __syncwarp();
                for (int k = lane; k < u; k += 32)
                    acc[k] = 0.0;
                __syncwarp();
                for_each([&](bool ok, int col, double v) {
                    const int r = ok ? hash_rank(tkeys, tranks, col, hbits) : 0;
                    ordered_add(acc, stage, ok, r, v, lane);
                });
                for (int k = lane; k < u; k += 32)
                    A.cv[base + k] = acc[k];
                if (lane == 0)
                    A.count[row] = u;
                __syncwarp();
            }
        }

        // rows (of list, or all) whose count is the overflow mark -1, and their list
        __global__ void overflow_rows(int n, const int* __restrict__ list, const int* __restrict__ counts,
                                      int* __restrict__ flag)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                flag[i] = counts[list ? list[i] : i] < 0 ? 1 : 0;
        }

        __global__ void overflow_list(int n, const int* __restrict__ list, const int* __restrict__ flag,
                                      const int* __restrict__ pos, int* __restrict__ out)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                if (flag[i])
                    out[pos[i]] = list ? list[i] : i;
        }

        // class of every row; per-block histograms in shared memory, one global atomic per
        // class and block
        __global__ void bucket_count_kernel(int rows, const int* __restrict__ cand, const int* __restrict__ caps,
                                            int ncaps, int* __restrict__ cls, int* __restrict__ counts)
        {
            __shared__ int h[17];
            if (threadIdx.x < 17)
                h[threadIdx.x] = 0;
            __syncthreads();
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
            {
                int b = 0;
                while (b < ncaps && cand[r] > caps[b])
                    ++b;
                cls[r] = b;
                atomicAdd(h + b, 1);
            }
            __syncthreads();
            if (threadIdx.x <= ncaps && h[threadIdx.x])
                atomicAdd(counts + threadIdx.x, h[threadIdx.x]);
        }

        // rows into their class ranges: each block reserves its slots per class with one
        // global atomic, then places its rows through shared-memory cursors
        __global__ void bucket_fill_kernel(int rows, const int* __restrict__ cls, const int* __restrict__ base,
                                           int* __restrict__ cursor, int* __restrict__ list)
        {
            __shared__ int h[17], off[17];
            const int r0 = blockIdx.x * blockDim.x * 8, r1 = min(rows, r0 + static_cast<int>(blockDim.x) * 8);
            if (threadIdx.x < 17)
                h[threadIdx.x] = 0;
            __syncthreads();
            for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x)
                atomicAdd(h + cls[r], 1);
            __syncthreads();
            if (threadIdx.x < 17)
            {
                off[threadIdx.x] = h[threadIdx.x] ? base[threadIdx.x] + atomicAdd(cursor + threadIdx.x, h[threadIdx.x]) : 0;
                h[threadIdx.x] = 0;
            }
            __syncthreads();
            for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x)
            {
                const int b = cls[r];
                list[off[b] + atomicAdd(h + b, 1)] = r;
            }
        }

        // one warp per row: move the row's distinct entries from its candidate segment of
        // the staging arrays to the compressed result
        __global__ void spgemm_compact(int rows, const int* __restrict__ cand_ptr, const int* __restrict__ tc,
                                       const double* __restrict__ tv, const int* __restrict__ cp, int* __restrict__ cc,
                                       double* __restrict__ cv)
        {
            const int lane = threadIdx.x & 31;
            const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            const int nw = (gridDim.x * blockDim.x) >> 5;
            for (int r = warp; r < rows; r += nw)
            {
                const int src = cand_ptr[r], dst = cp[r], len = cp[r + 1] - dst;
                for (int k = lane; k < len; k += 32)
                {
                    cc[dst + k] = tc[src + k];
                    cv[dst + k] = tv[src + k];
                }
            }
        }

        // ---- transpose -----------------------------------------------------------
        __global__ void col_count(int nnz, const int* __restrict__ ci, int* __restrict__ cnt)
        {
            for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz; k += (long long)gridDim.x * blockDim.x)
                atomicAdd(&cnt[ci[k]], 1);
        }

        __global__ void transpose_fill(int rows, const int* __restrict__ rp, const int* __restrict__ ci,
                                       const double* __restrict__ va, const int* __restrict__ tp, int* __restrict__ cursor,
                                       int* __restrict__ tc, double* __restrict__ tv)
        {
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
                for (int k = rp[r]; k < rp[r + 1]; ++k)
                {
                    const int c = ci[k];
                    const int pos = tp[c] + atomicAdd(&cursor[c], 1);
                    tc[pos] = r;
                    tv[pos] = va[k];
                }
        }

        // sort every row segment by column (one warp per row; rows up to CAP long)
        template<int CAP>
        __global__ void __launch_bounds__(256) sort_rows(int rows, const int* __restrict__ rp, int* __restrict__ ci,
                                                         double* __restrict__ va)
        {
            extern __shared__ unsigned char smem_raw[];
            const int warps = blockDim.x >> 5;
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            unsigned long long* keys = reinterpret_cast<unsigned long long*>(smem_raw) + (size_t)w * CAP;
            double* vals = reinterpret_cast<double*>(reinterpret_cast<unsigned long long*>(smem_raw) + (size_t)warps * CAP) +
                           (size_t)w * CAP;
            for (int row = blockIdx.x * warps + w; row < rows; row += gridDim.x * warps)
            {
                const int b = rp[row], n = rp[row + 1] - b;
                for (int k = lane; k < n; k += 32)
                {
                    keys[k] = (static_cast<unsigned long long>(static_cast<unsigned>(ci[b + k])) << 32) | (unsigned)k;
                    vals[k] = va[b + k];
                }
                const int np = next_pow2(n);
                for (int k = n + lane; k < np; k += 32)
                    keys[k] = ~0ull;
                __syncwarp();
                warp_bitonic_sort(keys, np);
                for (int k = lane; k < n; k += 32)
                {
                    ci[b + k] = static_cast<int>(keys[k] >> 32);
                    va[b + k] = vals[keys[k] & 0xffffffffu];
                }
                __syncwarp();
            }
        }

        __global__ void max_len_kernel(int n, const int* __restrict__ p, int* __restrict__ out)
        {
            int m = 0;
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                m = max(m, p[i + 1] - p[i]);
            for (int o = 16; o > 0; o >>= 1)
                m = max(m, __shfl_down_sync(0xffffffffu, m, o));
            if ((threadIdx.x & 31) == 0)
                atomicMax(out, m);
        }

        int read_int(cudaStream_t s, const int* d)
        {
            int h = 0;
            APF_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, s));
            sync(s);
            return h;
        }

        template<class F>
        void with_cap(int n, F&& f)
        {
            if (n <= 64) f(std::integral_constant<int, 64>{});
            else if (n <= 256) f(std::integral_constant<int, 256>{});
            else if (n <= 1024) f(std::integral_constant<int, 1024>{});
            else if (n <= 4096) f(std::integral_constant<int, 4096>{});
            else if (n <= 8192) f(std::integral_constant<int, 8192>{});
            else throw Error(APF_ERR_CAPACITY, "sparse product: a row has more than 8192 candidate entries");
        }

        template<int CAP>
        int warps_for_cap()
        {
            return std::max(1, std::min(8, (96 * 1024) / (CAP * 16)));
        }
    }

    namespace
    {
        // G lanes per row: about four to eight entries per lane (one or two unrolled steps
        // per row), then more lanes while the launch would not fill the GPU once
        template<class F>
        void with_lanes(long long rows, double avg, F&& go)
        {
            int g = 4;
            while (g < 32 && avg > 6.0 * g)
                g *= 2;
            while (g < 32 && rows * g < 148LL * 2048)
                g *= 2;
            if (g == 4) go(std::integral_constant<int, 4>{});
            else if (g == 8) go(std::integral_constant<int, 8>{});
            else if (g == 16) go(std::integral_constant<int, 16>{});
            else go(std::integral_constant<int, 32>{});
        }

        template<int MODE>
        void sell_launch(cudaStream_t s, const DeviceSell& S, const double* x, const double* b, double* y, double alpha,
                         double beta, const double* dinv, double* z = nullptr)
        {
            if (S.csr_rp)
            {
                // CSR layout with f32 values (short or wide-row operators)
                with_lanes(S.rows, S.avg_row, [&](auto g) {
                    constexpr int G = decltype(g)::value;
                    spmv_kernel<G, MODE, float><<<blocks_for((long long)S.rows * G, 256, 148 * 64), 256, 0, s>>>(
                        S.rows, S.csr_rp, S.csr_ci, S.val32.get(), x, b, y, alpha, beta, dinv, z);
                });
                APF_CUDA(cudaGetLastError());
                return;
            }
            const int grid = blocks_for((long long)S.slices * 32, 256, 148 * 64);
            if (S.val32.size())
                sell_kernel<MODE, float><<<grid, 256, 0, s>>>(S.rows, S.slices, S.slice_ptr.get(), S.col.get(),
                                                              S.val32.get(), x, b, y, alpha, beta, dinv, S.perm.get(), z);
            else
                sell_kernel<MODE, double><<<grid, 256, 0, s>>>(S.rows, S.slices, S.slice_ptr.get(), S.col.get(),
                                                               S.val.get(), x, b, y, alpha, beta, dinv, S.perm.get(), z);
            APF_CUDA(cudaGetLastError());
        }

        template<int MODE>
        void spmv_dispatch(cudaStream_t s, const DeviceCsr& A, const double* x, const double* b, double* y, double alpha,
                           double beta, const double* dinv = nullptr, const char* name = nullptr)
        {
            if (A.rows == 0)
                return;
            const double avg = static_cast<double>(A.nnz()) / A.rows;
            const int threads = 256;
            APF_KERNEL(name ? name : (MODE == 1 ? "residual" : (MODE == 2 ? "jacobi_sweep" : "spmv")), s);
            if (A.sell)
            {
                sell_launch<MODE>(s, *A.sell, x, b, y, alpha, beta, dinv);
                return;
            }
            with_lanes(A.rows, avg, [&](auto g) {
                constexpr int G = decltype(g)::value;
                spmv_kernel<G, MODE><<<blocks_for((long long)A.rows * G, threads, 148 * 64), threads, 0, s>>>(
                    A.rows, A.row_ptr.get(), A.col_idx.get(), A.values.get(), x, b, y, alpha, beta, dinv, nullptr);
            });
            APF_CUDA(cudaGetLastError());
        }
    }

    bool build_sell(cudaStream_t s, DeviceCsr& A, double max_padding)
    {
        A.sell.reset();
        if (A.rows == 0 || A.nnz() == 0)
            return false;
        const int slices = (A.rows + 31) / 32;
        DeviceBuffer<int> cnt(slices, s);
        const int grid = blocks_for((long long)slices * 32, 256, 148 * 32);
        auto S = std::make_unique<DeviceSell>();
        S->perm.allocate(static_cast<std::size_t>(A.rows), s);
        {
            APF_KERNEL("sell_sort_rows", s);
            sell_sort_rows<<<(A.rows + kSellWindow - 1) / kSellWindow, 256, 0, s>>>(A.rows, A.row_ptr.get(), S->perm.get());
        }
        {
            APF_KERNEL("sell_count", s);
            sell_count<<<grid, 256, 0, s>>>(A.rows, slices, A.row_ptr.get(), S->perm.get(), cnt.get(), 0);
        }
        S->rows = A.rows;
        S->slices = slices;
        S->slice_ptr.allocate(static_cast<std::size_t>(slices) + 1, s);
        const long long total = exclusive_scan(cnt.get(), S->slice_ptr.get(), slices, s);
        if (total > static_cast<long long>(max_padding * static_cast<double>(A.nnz())) || total >= (1ll << 31))
            return false;
        S->col.allocate(static_cast<std::size_t>(total), s);
        S->val.allocate(static_cast<std::size_t>(total), s);
        {
            APF_KERNEL("sell_fill", s);
            sell_fill<double><<<grid, 256, 0, s>>>(A.rows, slices, A.row_ptr.get(), A.col_idx.get(), A.values.get(),
                                                  S->slice_ptr.get(), S->perm.get(), S->col.get(), S->val.get());
        }
        APF_CUDA(cudaGetLastError());
        A.sell = std::move(S);
        return true;
    }

    std::unique_ptr<DeviceSell> make_sell32(cudaStream_t s, const DeviceCsr& A)
    {
        auto S = std::make_unique<DeviceSell>();
        S->rows = A.rows;
        S->avg_row = A.rows ? static_cast<double>(A.nnz()) / A.rows : 0.0;
        if (A.rows < kSellMinRows || S->avg_row > kSellMaxRow)
        {
            // few rows or long rows: one thread per row would leave the GPU idle or
            // serialise long loops; keep the CSR arrays and lanes per row, f32 values
            S->csr_rp = A.row_ptr.get();
            S->csr_ci = A.col_idx.get();
            S->val32.allocate(static_cast<std::size_t>(A.nnz()), s);
            if (A.nnz())
            {
                APF_KERNEL("sell_fill", s);
                to_f32_kernel<<<blocks_for(A.nnz(), 256, 148 * 32), 256, 0, s>>>(A.nnz(), A.values.get(), S->val32.get());
            }
            APF_CUDA(cudaGetLastError());
            return S;
        }
        S->slices = (A.rows + 31) / 32;
        S->slice_ptr.allocate(static_cast<std::size_t>(S->slices) + 1, s);
        if (A.rows == 0)
            return S;
        DeviceBuffer<int> cnt(S->slices, s);
        const int grid = blocks_for((long long)S->slices * 32, 256, 148 * 32);
        S->perm.allocate(static_cast<std::size_t>(A.rows), s);
        {
            APF_KERNEL("sell_sort_rows", s);
            sell_sort_rows<<<(A.rows + kSellWindow - 1) / kSellWindow, 256, 0, s>>>(A.rows, A.row_ptr.get(), S->perm.get());
        }
        {
            APF_KERNEL("sell_count", s);
            sell_count<<<grid, 256, 0, s>>>(A.rows, S->slices, A.row_ptr.get(), S->perm.get(), cnt.get(), 1);
        }
        const long long total = exclusive_scan(cnt.get(), S->slice_ptr.get(), S->slices, s);
        S->col.allocate(static_cast<std::size_t>(total), s);
        S->val32.allocate(static_cast<std::size_t>(total), s);
        if (total)
        {
            APF_KERNEL("sell_fill", s);
            sell_fill<float><<<grid, 256, 0, s>>>(A.rows, S->slices, A.row_ptr.get(), A.col_idx.get(), A.values.get(),
                                                 S->slice_ptr.get(), S->perm.get(), S->col.get(), S->val32.get());
        }
        APF_CUDA(cudaGetLastError());
        return S;
    }

    void spmv(cudaStream_t s, const DeviceSell& A, const double* x, double* y, double alpha, double beta,
              const char* name)
    {
        if (A.rows == 0)
            return;
        APF_KERNEL(name ? name : "spmv", s);
        sell_launch<0>(s, A, x, nullptr, y, alpha, beta, nullptr);
    }

    void spmv_jacobi_first(cudaStream_t s, const DeviceSell& A, const double* x, double* y, const double* w,
                           double omega, double* z, const char* name)
    {
        if (A.rows == 0)
            return;
        APF_KERNEL(name ? name : "spmv", s);
        sell_launch<3>(s, A, x, nullptr, y, 1.0, omega, w, z);
    }

    void jacobi_sweep(cudaStream_t s, const DeviceSell& A, const double* x, const double* b, const double* dinv,
                      double omega, double* y, const char* name)
    {
        if (A.rows == 0)
            return;
        APF_KERNEL(name ? name : "jacobi_sweep", s);
        sell_launch<2>(s, A, x, b, y, omega, 0.0, dinv);
    }

    void residual(cudaStream_t s, const DeviceSell& A, const double* x, const double* b, double* r, const char* name)
    {
        if (A.rows == 0)
            return;
        APF_KERNEL(name ? name : "residual", s);
        sell_launch<1>(s, A, x, b, r, 1.0, 0.0, nullptr);
    }

    void spmv(cudaStream_t s, const DeviceCsr& A, const double* x, double* y, double alpha, double beta, const char* name)
    {
        spmv_dispatch<0>(s, A, x, nullptr, y, alpha, beta, nullptr, name);
    }

    void jacobi_sweep(cudaStream_t s, const DeviceCsr& A, const double* x, const double* b, const double* dinv,
                      double omega, double* y)
    {
        spmv_dispatch<2>(s, A, x, b, y, omega, 0.0, dinv);
    }

    void residual(cudaStream_t s, const DeviceCsr& A, const double* x, const double* b, double* r)
    {
        spmv_dispatch<1>(s, A, x, b, r, 1.0, 0.0);
    }

    void dot_device(cudaStream_t s, Workspace& w, int n, const double* a, const double* b, double* out)
    {
        w.ensure(s);
        {
            APF_KERNEL("dot_partials", s);
            dot_partials<<<kRedBlocks, kRedThreads, 0, s>>>(n, a, b, w.partials.get());
        }
        {
            APF_KERNEL("sum_partials", s);
            sum_partials<<<1, 256, 0, s>>>(kRedBlocks, w.partials.get(), out);
        }
        APF_CUDA(cudaGetLastError());
    }

    double dot_host(cudaStream_t s, Workspace& w, int n, const double* a, const double* b)
    {
        w.ensure(s);
        dot_device(s, w, n, a, b, w.scalars.get());
        double h = 0.0;
        APF_CUDA(cudaMemcpyAsync(&h, w.scalars.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
        sync(s);
        return h;
    }

    void axpby(cudaStream_t s, int n, double a, const double* x, double b, double* y)
    {
        APF_KERNEL("axpby", s);
        axpby_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, a, x, b, y);
    }

    void copy(cudaStream_t s, int n, const double* x, double* y)
    {
        if (n)
            APF_CUDA(cudaMemcpyAsync(y, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }

    void fill(cudaStream_t s, int n, double v, double* y)
    {
        APF_KERNEL("fill", s);
        fill_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, v, y);
    }

    void inverse_diagonal(cudaStream_t s, const DeviceCsr& A, DeviceBuffer<double>& inv)
    {
        inv.allocate(static_cast<std::size_t>(A.rows), s);
        APF_KERNEL("inv_diag", s);
        inv_diag_kernel<<<blocks_for(A.rows, 256), 256, 0, s>>>(A.rows, A.row_ptr.get(), A.col_idx.get(), A.values.get(),
                                                                 inv.get());
    }

    void bucket_rows(cudaStream_t s, int rows, const int* cand, const int* caps, int ncaps, RowBuckets& out)
    {
        require(ncaps >= 1 && ncaps <= 16, APF_ERR_INVALID, "bucket_rows: 1 to 16 classes");
        DeviceBuffer<int> dcaps(ncaps, s), cls(static_cast<std::size_t>(std::max(rows, 1)), s), counts(ncaps + 1, s),
            base(ncaps + 1, s), cursor(ncaps + 1, s);
        dcaps.upload(caps, ncaps);
        counts.zero();
        cursor.zero();
        if (rows > 0)
        {
            APF_KERNEL("bucket_rows", s);
            bucket_count_kernel<<<blocks_for(rows, 256), 256, 0, s>>>(rows, cand, dcaps.get(), ncaps, cls.get(), counts.get());
        }
        std::vector<int> h(ncaps + 1, 0);
        APF_CUDA(cudaMemcpyAsync(h.data(), counts.get(), (ncaps + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
        sync(s);
        require(h[ncaps] == 0, APF_ERR_CAPACITY, "sparse product: a row has more candidates than the largest class");
        out.offsets.assign(ncaps + 1, 0);
        for (int b = 0; b < ncaps; ++b)
            out.offsets[b + 1] = out.offsets[b] + h[b];
        base.upload(out.offsets.data(), ncaps + 1);
        out.list.allocate(static_cast<std::size_t>(std::max(rows, 1)), s);
        if (rows > 0)
        {
            APF_KERNEL("bucket_rows", s);
            bucket_fill_kernel<<<(rows + 256 * 8 - 1) / (256 * 8), 256, 0, s>>>(rows, cls.get(), base.get(), cursor.get(),
                                                                                out.list.get());
        }
        APF_CUDA(cudaGetLastError());
    }

    void spgemm(cudaStream_t s, const DeviceCsr& A, const DeviceCsr& B, DeviceCsr& C)
    {
        require(A.cols == B.rows, APF_ERR_INVALID, "spgemm: inner dimensions differ");
        C.rows = A.rows;
        C.cols = B.cols;
        C.row_ptr.allocate(static_cast<std::size_t>(A.rows) + 1, s);
        if (A.rows == 0)
        {
            APF_CUDA(cudaMemsetAsync(C.row_ptr.get(), 0, sizeof(int), s));
            return;
        }
        // one sorting pass: each row's distinct products go to its candidate segment of
        // staging arrays (sized by the candidate counts), then a compaction
        DeviceBuffer<int> bound(1, s), cand(static_cast<std::size_t>(A.rows) + 1, s),
            cand_ptr(static_cast<std::size_t>(A.rows) + 1, s);
        bound.zero();
        {
            APF_KERNEL("spgemm_bound", s);
            spgemm_bound<<<blocks_for(A.rows, 256, 148 * 8), 256, 0, s>>>(A.rows, A.row_ptr.get(), A.col_idx.get(),
                                                                           B.row_ptr.get(), bound.get(), cand.get());
        }
        const long long total = exclusive_scan(cand.get(), cand_ptr.get(), A.rows, s);
        DeviceBuffer<int> count(static_cast<std::size_t>(A.rows) + 1, s), tc(static_cast<std::size_t>(std::max(total, 1ll)), s);
        DeviceBuffer<double> tv(static_cast<std::size_t>(std::max(total, 1ll)), s);
        GemmArgs g{A.rows, A.row_ptr.get(), A.col_idx.get(), A.values.get(), B.row_ptr.get(), B.col_idx.get(),
                   B.values.get(), count.get(), cand_ptr.get(), tc.get(), tv.get(), nullptr, 0};
        // every row with room for 128 distinct columns (the candidates stream through), then
        // the rows that had more with 1024, then 8192
        auto launch = [&](auto tag) {
            constexpr int CAP = decltype(tag)::value;
            const int warps = std::max(1, std::min(8, (96 * 1024) / (CAP * 24 + kRowExtra)));
            const size_t smem = (size_t)warps * (CAP * 24 + kRowExtra);
            const int blocks = blocks_for(g.list ? g.nlist : A.rows, warps, 148 * 32);
            APF_CUDA(cudaFuncSetAttribute(spgemm_rows<CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            APF_KERNEL("spgemm_fill", s);
            spgemm_rows<CAP><<<blocks, warps * 32, smem, s>>>(g);
            APF_CUDA(cudaGetLastError());
        };
        g.list = nullptr;
        g.nlist = A.rows;
        launch(std::integral_constant<int, 128>{});
        DeviceBuffer<int> oflag(static_cast<std::size_t>(A.rows) + 1, s), opos(static_cast<std::size_t>(A.rows) + 1, s),
            olist(1, s);
        for (int pass = 0; pass < 3; ++pass)
        {
            const int nin = g.list ? g.nlist : A.rows;
            {
                APF_KERNEL("spgemm_overflow_rows", s);
                overflow_rows<<<blocks_for(nin, 256), 256, 0, s>>>(nin, g.list, count.get(), oflag.get());
            }
            const int nover = static_cast<int>(exclusive_scan(oflag.get(), opos.get(), nin, s));
            if (nover == 0)
                break;
            require(pass < 2, APF_ERR_CAPACITY, "sparse product: a row has more than 8192 distinct columns");
            DeviceBuffer<int> next(static_cast<std::size_t>(nover), s);
            {
                APF_KERNEL("spgemm_overflow_rows", s);
                overflow_list<<<blocks_for(nin, 256), 256, 0, s>>>(nin, g.list, oflag.get(), opos.get(), next.get());
            }
            olist = std::move(next);
            g.list = olist.get();
            g.nlist = nover;
            if (pass == 0)
                launch(std::integral_constant<int, 1024>{});
            else
                launch(std::integral_constant<int, 8192>{});
        }
        const long long nnz = exclusive_scan(count.get(), C.row_ptr.get(), A.rows, s);
        C.col_idx.allocate(static_cast<std::size_t>(nnz), s);
        C.values.allocate(static_cast<std::size_t>(nnz), s);
        {
            APF_KERNEL("spgemm_compact", s);
            spgemm_compact<<<blocks_for((long long)A.rows * 32, 256, 148 * 16), 256, 0, s>>>(
                A.rows, cand_ptr.get(), tc.get(), tv.get(), C.row_ptr.get(), C.col_idx.get(), C.values.get());
        }
        APF_CUDA(cudaGetLastError());
    }

    void transpose(cudaStream_t s, const DeviceCsr& A, DeviceCsr& T)
    {
        T.rows = A.cols;
        T.cols = A.rows;
        DeviceBuffer<int> cnt(static_cast<std::size_t>(A.cols) + 1, s);
        cnt.zero();
        if (A.nnz())
        {
            APF_KERNEL("col_count", s);
            col_count<<<blocks_for(A.nnz(), 256), 256, 0, s>>>(static_cast<int>(A.nnz()), A.col_idx.get(), cnt.get());
        }
        T.row_ptr.allocate(static_cast<std::size_t>(A.cols) + 1, s);
        const long long nnz = exclusive_scan(cnt.get(), T.row_ptr.get(), A.cols, s);
        T.col_idx.allocate(static_cast<std::size_t>(nnz), s);
        T.values.allocate(static_cast<std::size_t>(nnz), s);
        cnt.zero();
        if (A.rows)
        {
            APF_KERNEL("transpose_fill", s);
            transpose_fill<<<blocks_for(A.rows, 256), 256, 0, s>>>(A.rows, A.row_ptr.get(), A.col_idx.get(),
                                                                    A.values.get(), T.row_ptr.get(), cnt.get(),
                                                                    T.col_idx.get(), T.values.get());
        }
        DeviceBuffer<int> mx(1, s);
        mx.zero();
        if (T.rows)
        {
            APF_KERNEL("max_len", s);
            max_len_kernel<<<blocks_for(T.rows, 256, 1024), 256, 0, s>>>(T.rows, T.row_ptr.get(), mx.get());
        }
        const int longest = read_int(s, mx.get());
        if (T.rows == 0 || longest <= 1)
            return;
        with_cap(longest, [&](auto tag) {
            constexpr int CAP = decltype(tag)::value;
            const int warps = warps_for_cap<CAP>();
            const size_t smem = (size_t)warps * CAP * 16;
            APF_CUDA(cudaFuncSetAttribute(sort_rows<CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            APF_KERNEL("sort_rows", s);
            sort_rows<CAP><<<blocks_for(T.rows, warps, 148 * 32), warps * 32, smem, s>>>(T.rows, T.row_ptr.get(),
                                                                                          T.col_idx.get(), T.values.get());
            APF_CUDA(cudaGetLastError());
        });
    }
}
