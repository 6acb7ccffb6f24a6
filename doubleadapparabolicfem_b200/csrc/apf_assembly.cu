// Main-system assembly on the device: A_y, B, B^T, C_signed, f, g, K, and the
// parabolic graph-norm block Hhat = -C_signed + B_dt diag(A_y)^-1 B_dt^T + A_x.
//
// Design (B200): assembly is "pull" (row gather), not triplet scatter.
//   1. incidence lists: true DOF -> (cell, local index, restriction entry), built
//      with a count / scan / fill pass;
//   2. one warp per matrix row gathers every candidate (column, value) of that row
//      from its incident cells -- local entries recomputed in closed form from the
//      cell geometry (affine prisms, cell-constant M) and filtered with
//      |a_ij| > zero_tol exactly like scatter.hpp:66-115 -- sorts the candidates
//      in shared memory (bitonic, key = column | deterministic sequence number)
//      and sums duplicates in a fixed order.  One sorting pass writes each row's
//      distinct columns and values into its segment
//      of staging arrays sized by the row's candidate count; a scan of the distinct counts
//      gives row_ptr and a compaction writes the block.
// The result is the reference's compressed pattern bit for bit (setFromTriplets
// keeps summed explicit zeros, so does this) and deterministic values with no
// floating-point atomics.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <type_traits>

#include "apf_device.cuh"
#include "apf_quad1d.cuh"
#include "apf_warpsort.cuh"
#include "apf_rowhash.cuh"
#include "apf_internal.hpp"
#include "apf_system.hpp"

namespace apf
{
    __constant__ RefTables c_tab[2];

    std::atomic<long long> g_kernel_launches{0};
    thread_local Profiler* t_profiler = nullptr;

    namespace
    {
        // ------------------------------------------------------------------
        // incidence lists
        // ------------------------------------------------------------------
        // An "assembly cell" a (index into cell_list or the identity) takes its
        // row restriction from source cell src(a) = src_map ? src_map[cell] : cell.
        struct IncidenceSpec
        {
            int n_asm;                 // number of assembly cells
            const int* cell_list;      // optional: assembly cell -> cell index
            const int* src_map;        // optional: cell -> restriction source cell
            const int* offsets;        // restriction offsets [n_src*ndof+1]
            const int* dofs;
            int ndof;
        };

        __device__ __forceinline__ int asm_cell(const IncidenceSpec& s, int a)
        {
            return s.cell_list ? s.cell_list[a] : a;
        }
        __device__ __forceinline__ int src_cell(const IncidenceSpec& s, int c)
        {
            return s.src_map ? s.src_map[c] : c;
        }

        __global__ void incidence_count(IncidenceSpec s, int* __restrict__ count)
        {
            const long long total = static_cast<long long>(s.n_asm) * s.ndof;
            for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
                 k += (long long)gridDim.x * blockDim.x)
            {
                const int a = static_cast<int>(k / s.ndof), i = static_cast<int>(k % s.ndof);
                const int c = asm_cell(s, a);
                const int r = src_cell(s, c) * s.ndof + i;
                for (int e = s.offsets[r]; e < s.offsets[r + 1]; ++e)
                    atomicAdd(&count[s.dofs[e]], 1);
            }
        }

        __global__ void incidence_fill(IncidenceSpec s, const int* __restrict__ ptr, int* __restrict__ cursor,
                                       int2* __restrict__ inc)
        {
            const long long total = static_cast<long long>(s.n_asm) * s.ndof;
            for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
                 k += (long long)gridDim.x * blockDim.x)
            {
                const int a = static_cast<int>(k / s.ndof), i = static_cast<int>(k % s.ndof);
                const int c = asm_cell(s, a);
                const int r = src_cell(s, c) * s.ndof + i;
                for (int e = s.offsets[r]; e < s.offsets[r + 1]; ++e)
                {
                    const int d = s.dofs[e];
                    const int pos = ptr[d] + atomicAdd(&cursor[d], 1);
                    inc[pos] = make_int2(c * s.ndof + i, e);
                }
            }
        }

        __global__ void max_row_length(const int* __restrict__ ptr, int n, int* __restrict__ out)
        {
            int m = 0;
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                m = max(m, ptr[i + 1] - ptr[i]);
            for (int o = 16; o > 0; o >>= 1)
                m = max(m, __shfl_down_sync(0xffffffffu, m, o));
            if ((threadIdx.x & 31) == 0)
                atomicMax(out, m);
        }

        // ------------------------------------------------------------------
        // local block evaluators
        // ------------------------------------------------------------------
        struct AsmData
        {
            int p;
            int dim; // 1: quads (geometry rows x0 x1 t0 t1, one M value per cell), 2: prisms
            const double* y_geo;
            const double* x_geo;
            const int* y_to_x;
            const double* m_y; // per Y cell or null
            const double* m_x; // per X cell or null
            const int* y_off;
            const int* y_dofs;
            const double* y_w;
            const int* x_off;
            const int* x_dofs;
            const double* x_w;
            double zero_tol;
        };

        // 1+1D local entry (P1 x P1 quadrilaterals, see apf_quad1d.cuh)
        __device__ double local_entry_1d(const AsmData& d, int kind, int c, int i, int j)
        {
            const int s = i >> 1, a = i & 1, r = j >> 1, b = j & 1;
            if (kind == K_AY || kind == K_AX)
            {
                const q1d::Quad g = q1d::load(kind == K_AY ? d.y_geo : d.x_geo, c);
                const double* m = kind == K_AY ? d.m_y : d.m_x;
                const double mc = m ? m[c] : 1.0;
                return mc * (g.k / g.h) * q1d::stiff(s, r) * q1d::mass(a, b);
            }
            if (kind == K_C)
            {
                const q1d::Quad g = q1d::load(d.x_geo, c);
                return (a == 0 && b == 0) ? -(g.h * q1d::mass(s, r)) : 0.0;
            }
            int ix = i, jy = j;
            if (kind == K_BT || kind == K_BDTT)
            {
                ix = j;
                jy = i;
            }
            const int cx = d.y_to_x[c];
            const q1d::Quad gy = q1d::load(d.y_geo, c);
            const q1d::Quad gx = q1d::load(d.x_geo, cx);
            const double mc = d.m_y ? d.m_y[c] : 1.0;
            return q1d::mixed(gy, gx, q1d::same(d.y_geo, c, d.x_geo, cx), mc, ix, jy,
                              kind == K_BDT || kind == K_BDTT);
        }

        // local entry L_c(i, j) of block `kind` on assembly cell c
        __device__ double local_entry(const AsmData& d, int kind, int c, int i, int j)
        {
            if (d.dim == 1)
                return local_entry_1d(d, kind, c, i, j);
            const RefTables& t = c_tab[d.p - 1];
            if (kind == K_AY || kind == K_AX)
            {
                const double* geo = kind == K_AY ? d.y_geo : d.x_geo;
                const double* m = kind == K_AY ? d.m_y : d.m_x;
                const CellGeo g = load_geo(geo, c);
                double q00, q01, q11;
                q_form(g, m, c, q00, q01, q11);
                const int s = i / t.nt, a = i % t.nt, r = j / t.nt, b = j % t.nt;
                return g.det * g.ht * t.Mt[a][b] * ks(t, q00, q01, q11, s, r);
            }
            if (kind == K_C)
            {
                const CellGeo g = load_geo(d.x_geo, c);
                const int s = i / t.nt, a = i % t.nt, r = j / t.nt, b = j % t.nt;
                return -(g.det * t.Mx[s][r] * t.S0[a] * t.S0[b]);
            }
            // mixed blocks: row index of B is the X-local index
            int ix = i, jy = j;
            if (kind == K_BT || kind == K_BDTT)
            {
                ix = j;
                jy = i;
            }
            const bool dt_only = kind == K_BDT || kind == K_BDTT;
            const int cx = d.y_to_x[c];
            const CellGeo gy = load_geo(d.y_geo, c);
            double q00, q01, q11;
            q_form(gy, d.m_y, c, q00, q01, q11);
            if (same_geometry(d.y_geo, c, d.x_geo, cx))
                return b_same(t, gy, q00, q01, q11, ix, jy, dt_only);
            const CellGeo gx = load_geo(d.x_geo, cx);
            double v = 0.0;
            for (int k = 0; k < t.ndof; ++k)
                v += transfer(t, gy, gx, ix, k) * b_same(t, gy, q00, q01, q11, k, jy, dt_only);
            return v;
        }

        // column restriction of local column j on assembly cell c
        __device__ __forceinline__ void col_restriction(const AsmData& d, int kind, int c, int j, int ndof,
                                                        const int*& dofs, const double*& w, int& b, int& e)
        {
            if (kind == K_AY || kind == K_B || kind == K_BDT)
            {
                const int r = c * ndof + j;
                b = d.y_off[r];
                e = d.y_off[r + 1];
                dofs = d.y_dofs;
                w = d.y_w;
                return;
            }
            const int cx = (kind == K_BT || kind == K_BDTT) ? d.y_to_x[c] : c;
            const int r = cx * ndof + j;
            b = d.x_off[r];
            e = d.x_off[r + 1];
            dofs = d.x_dofs;
            w = d.x_w;
        }

        __device__ __forceinline__ const double* row_weights(const AsmData& d, int kind)
        {
            return (kind == K_AY || kind == K_BT || kind == K_BDTT) ? d.y_w : d.x_w;
        }

        // ------------------------------------------------------------------
        // warp-level candidate sort / reduce
        // ------------------------------------------------------------------
        struct Term
        {
            int kind;
            const int* inc_ptr;
            const int2* inc;
            int col_offset;
        };

        struct GatherArgs
        {
            AsmData d;
            int n_rows;
            int ndof;
            int n_terms;
            Term term[2];
            int* row_count;      // count pass output
            const int* row_ptr;  // fill pass input
            int* col_out;
            double* val_out;
            int* status;         // nonzero on overflow
            const int* list;     // rows to process (null: all)
            int nlist;
            int kmax;            // restriction entries per local row (at most kMaxRestrictionEntries)
        };

        // One warp per row with at most UCAP distinct columns, in one pass over the candidates:
        // per term, the row's incidences staged and ordered by (cell * ndof + i); then every
        // (incidence, local column j, restriction entry q) candidate with |local| > zero_tol,
        // 32 items at a time, is added to its column's slot of a shared-memory hash table
        // (at most half full) in generation order (within 32 items: by restriction entry,
        // then lane); at the end only the distinct columns are sorted.  A row with more than
        // UCAP distinct columns is marked row_count = -1 and left for a larger UCAP.
        // Shared memory per warp: incidences int[2 kIncCap + 2], table keys int[2 UCAP],
        // table sums double[2 UCAP], sorted keys 8 B x UCAP, staged values double[32].
        constexpr int kGatherIncCap = 256;
        // longest restriction row accepted (hanging-node chains of adaptive meshes: the
        // reference's 1-irregular refinement gives at most about 9)
        constexpr int kMaxRestrictionEntries = 16;

        template<int UCAP>
        __host__ __device__ constexpr std::size_t gather_u_warp_bytes()
        {
            return ((sizeof(int) * (2 * kGatherIncCap + 2) + 32 * UCAP + 32 * 8) + 15) / 16 * 16;
        }

        // Every candidate (ok, column, value) of one row in generation order: per term, the
        // row's incidences staged in incs and ordered by (cell * ndof + i); then every
        // (incidence, local column j, restriction entry q) item, 32 at a time (within a
        // batch: by restriction entry, then lane), ok = |local| > zero_tol.  All lanes of
        // the warp call f with the same sequence.  A row with more than kGatherIncCap
        // incidences in a term sets too_many_inc and stops.
        template<class F>
        __device__ __forceinline__ void row_candidates(const GatherArgs& A, int row, int lane, int* incs,
                                                       bool& too_many_inc, F&& f)
        {
            const int ndof = A.ndof;
            for (int tt = 0; tt < A.n_terms; ++tt)
            {
                const Term T = A.term[tt];
                const int ib = T.inc_ptr[row], ie = T.inc_ptr[row + 1];
                const int n_inc = ie - ib;
                if (n_inc > kGatherIncCap)
                {
                    too_many_inc = true;
                    return;
                }
                for (int k = lane; k < n_inc; k += 32)
                {
                    const int2 v = T.inc[ib + k];
                    incs[k] = v.x;
                    incs[kGatherIncCap + k] = v.y;
                }
                __syncwarp();
                int my_ci[8], my_e[8], my_rank[8];
                int nm = 0;
                for (int k = lane; k < n_inc; k += 32, ++nm)
                {
                    const int ci = incs[k];
                    int rank = 0;
                    for (int q = 0; q < n_inc; ++q)
                        rank += incs[q] < ci;
                    my_ci[nm] = ci;
                    my_e[nm] = incs[kGatherIncCap + k];
                    my_rank[nm] = rank;
                }
                __syncwarp();
                for (int q = 0; q < nm; ++q)
                {
                    incs[my_rank[q]] = my_ci[q];
                    incs[kGatherIncCap + my_rank[q]] = my_e[q];
                }
                __syncwarp();
                const double* rw = row_weights(A.d, T.kind);
                const int items = n_inc * ndof;
                for (int it0 = 0; it0 < items; it0 += 32)
                {
                    const int it = it0 + lane;
                    bool ok = false;
                    double v = 0.0, wi = 0.0;
                    const int* cd = nullptr;
                    const double* cw = nullptr;
                    int b = 0, e = 0;
                    if (it < items)
                    {
                        const int t_idx = it / ndof, j = it % ndof;
                        const int ci = incs[t_idx];
                        const int c = ci / ndof, i = ci % ndof;
                        wi = rw[incs[kGatherIncCap + t_idx]];
                        v = local_entry(A.d, T.kind, c, i, j);
                        ok = fabs(v) > A.d.zero_tol;
                        if (ok)
                            col_restriction(A.d, T.kind, c, j, ndof, cd, cw, b, e);
                    }
                    for (int q = 0; q < A.kmax; ++q)
                    {
                        const bool has = ok && b + q < e;
                        f(has, has ? cd[b + q] + T.col_offset : 0, has ? wi * cw[b + q] * v : 0.0);
                    }
                }
                __syncwarp();
            }
        }

        // Numeric pass on a kept pattern (the two-pass full saddle assembly): one warp per
        // row; the row's candidates, in row_candidates' order and with its zero_tol filter,
        // are added into the pattern's slots (the column's position among the row's sorted
        // columns) with ordered_add, so each slot receives exactly the sum the gather forms
        // for that column.  Slots that no candidate reaches stay 0.  A candidate whose column
        // is missing from the pattern sets status APF_ERR_INVALID.
        constexpr int kFillWarps = 4;
        constexpr int kFillWarpBytes = sizeof(int) * (2 * kGatherIncCap + 2) + 32 * sizeof(double);

        __global__ void __launch_bounds__(kFillWarps * 32) fill_rows_on_pattern(GatherArgs A, int row_base,
                                                                                const int* __restrict__ prow,
                                                                                const int* __restrict__ pcol,
                                                                                double* __restrict__ pval)
        {
            __shared__ __align__(16) unsigned char smem[kFillWarps * kFillWarpBytes];
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            int* incs = reinterpret_cast<int*>(smem + w * kFillWarpBytes);
            double* stage = reinterpret_cast<double*>(incs + 2 * kGatherIncCap + 2);
            for (int row = blockIdx.x * kFillWarps + w; row < A.n_rows; row += gridDim.x * kFillWarps)
            {
                const int b = prow[row_base + row], e = prow[row_base + row + 1];
                for (int k = b + lane; k < e; k += 32)
                    pval[k] = 0.0;
                __syncwarp();
                bool too_many_inc = false;
                row_candidates(A, row, lane, incs, too_many_inc, [&](bool ok, int col, double v) {
                    int slot = 0;
                    bool live = ok;
                    if (ok)
                    {
                        int lo = b, hi = e;
                        while (lo < hi)
                        {
                            const int mid = (lo + hi) >> 1;
                            if (pcol[mid] < col)
                                lo = mid + 1;
                            else
                                hi = mid;
                        }
                        if (lo < e && pcol[lo] == col)
                            slot = lo - b;
                        else
                        {
                            live = false;
                            atomicExch(A.status, APF_ERR_INVALID);
                        }
                    }
                    ordered_add(pval + b, stage, live, slot, v, lane);
                });
                if (too_many_inc && lane == 0)
                    atomicExch(A.status, APF_ERR_CAPACITY);
                __syncwarp();
            }
        }

        // entries with |value| > tol per row (prune(1.0, tol) keeps exactly those)
        __global__ void prune_count(int rows, const int* __restrict__ rp, const double* __restrict__ val, double tol,
                                    int* __restrict__ cnt)
        {
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
            {
                int c = 0;
                for (int k = rp[r]; k < rp[r + 1]; ++k)
                    c += fabs(val[k]) > tol;
                cnt[r] = c;
            }
        }

        // one warp per row: the kept entries in order (ballot compaction)
        __global__ void prune_fill(int rows, const int* __restrict__ rp, const int* __restrict__ ci,
                                   const double* __restrict__ val, double tol, const int* __restrict__ out_rp,
                                   int* __restrict__ out_ci, double* __restrict__ out_val)
        {
            const int lane = threadIdx.x & 31;
            const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            const int nwarps = (gridDim.x * blockDim.x) >> 5;
            for (int r = warp; r < rows; r += nwarps)
            {
                int o = out_rp[r];
                for (int k0 = rp[r]; k0 < rp[r + 1]; k0 += 32)
                {
                    const int k = k0 + lane;
                    const bool keep = k < rp[r + 1] && fabs(val[k]) > tol;
                    const unsigned m = __ballot_sync(0xffffffffu, keep);
                    if (keep)
                    {
                        const int at = o + __popc(m & ((1u << lane) - 1));
                        out_ci[at] = ci[k];
                        out_val[at] = val[k];
                    }
                    o += __popc(m);
                }
            }
        }

        // row pointers of two CSR row blocks stacked (the second block's shifted by the
        // first's nonzeros)
        __global__ void stack_row_ptr(int n_top, const int* __restrict__ top, int n_bottom,
                                      const int* __restrict__ bottom, int* __restrict__ out)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n_top + n_bottom; i += gridDim.x * blockDim.x)
                out[i] = i <= n_top ? top[i] : top[n_top] + bottom[i - n_top];
        }

        template<int UCAP>
        __global__ void __launch_bounds__(128) gather_rows_u(GatherArgs A)
        {
            extern __shared__ unsigned char smem_raw[];
            const int warps = blockDim.x >> 5;
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            unsigned char* mine = smem_raw + (size_t)w * gather_u_warp_bytes<UCAP>();
            int* incs = reinterpret_cast<int*>(mine);
            int* tkeys = incs + 2 * kGatherIncCap + 2;
            double* tvals = reinterpret_cast<double*>(tkeys + 2 * UCAP);
            unsigned long long* ukeys = reinterpret_cast<unsigned long long*>(tvals + 2 * UCAP);
            double* stage = reinterpret_cast<double*>(ukeys + UCAP);
            const int ndof = A.ndof;
            const int nrows = A.list ? A.nlist : A.n_rows;
            for (int idx = blockIdx.x * warps + w; idx < nrows; idx += gridDim.x * warps)
            {
                const int row = A.list ? A.list[idx] : idx;
                bool too_many_inc = false;
                auto for_each = [&](auto&& f) { row_candidates(A, row, lane, incs, too_many_inc, f); };
                int n = 0;
                for (int tt = 0; tt < A.n_terms; ++tt)
                    n += (A.term[tt].inc_ptr[row + 1] - A.term[tt].inc_ptr[row]) * ndof * A.kmax;
                int hbits = 6;
                while ((1 << hbits) < 2 * min(n, UCAP))
                    ++hbits;
                const int H = 1 << hbits;
                for (int t = lane; t < H; t += 32)
                {
                    tkeys[t] = -1;
                    tvals[t] = 0.0;
                }
                __syncwarp();
                int distinct = 0;
                bool overflow = false;
                for_each([&](bool ok, int col, double v) {
                    bool fresh = false;
                    const bool live = ok && !overflow;
                    const int h = live ? hash_slot_of(tkeys, col, hbits, fresh) : 0;
                    distinct += __popc(__ballot_sync(0xffffffffu, fresh));
                    ordered_add(tvals, stage, live, h, v, lane);
                    overflow = overflow || distinct > UCAP;
                });
                __syncwarp();
                if (too_many_inc)
                {
                    if (lane == 0)
                    {
                        atomicExch(A.status, APF_ERR_CAPACITY);
                        A.row_count[row] = 0;
                    }
                    __syncwarp();
                    continue;
                }
                if (overflow)
                {
                    if (lane == 0)
                        A.row_count[row] = -1;
                    __syncwarp();
                    continue;
                }
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
                const int out_base = A.row_ptr[row];
                for (int k = lane; k < u; k += 32)
                {
                    const unsigned long long key = ukeys[k];
                    A.col_out[out_base + k] = static_cast<int>(key >> 32);
                    A.val_out[out_base + k] = tvals[static_cast<unsigned>(key)];
                }
                if (lane == 0)
                    A.row_count[row] = u;
                __syncwarp();
            }
        }

        // ------------------------------------------------------------------
        // vectors f, g (one thread per row; deterministic order after sorting)
        // ------------------------------------------------------------------
        struct VecArgs
        {
            AsmData d;
            int n_rows;
            int ndof;
            const int* inc_ptr;
            const int2* inc;
            int which;            // 0 = f (Y cells, ell), 1 = g (bottom X cells, u0)
            const double* ell;    // per Y cell
            int u0_kind;
            double g_scale;
            double* out;
            int* status;
        };

        __device__ double u0_value(int kind, double x, double y)
        {
            if (kind == APF_U0_SIN_SIN)
                return sinpi(x) * sinpi(y);
            if (kind == APF_U0_ONE)
                return 1.0;
            return 0.0;
        }

        struct XIndArgs
        {
            int p, n_y, n_x, n_bottom, u0_kind;
            const double *y_geo, *x_geo, *m_y;
            const int *y_off, *y_dofs, *x_off, *x_dofs, *bottom;
            const double *y_w, *x_w, *lambda, *u;
            double *lam_y, *trace_x;
        };

        __device__ double u0_value_1d(int kind, double x)
        {
            if (kind == APF_U0_SIN_SIN)
                return sinpi(x);
            if (kind == APF_U0_ONE)
                return 1.0;
            return 0.0;
        }

        __device__ double local_vector(const VecArgs& A, int c, int i)
        {
            if (A.d.dim == 1)
            {
                if (A.which == 0)
                {
                    if (!A.ell)
                        return 0.0;
                    const q1d::Quad g = q1d::load(A.d.y_geo, c);
                    return A.ell[c] * g.h * g.k * 0.25;
                }
                const int kind = A.u0_kind;
                return q1d::initial_load(q1d::load(A.d.x_geo, c), i, A.g_scale,
                                         [kind](double x) { return u0_value_1d(kind, x); });
            }
            const RefTables& t = c_tab[A.d.p - 1];
            const int s = i / t.nt, a = i % t.nt;
            if (A.which == 0)
            {
                if (!A.ell)
                    return 0.0;
                const CellGeo g = load_geo(A.d.y_geo, c);
                return A.ell[c] * g.det * g.ht * t.ix[s] * t.it[a];
            }
            const CellGeo g = load_geo(A.d.x_geo, c);
            double acc = 0.0;
            for (int q = 0; q < t.nbq; ++q)
            {
                const double xi = t.bq_pts[q][0], eta = t.bq_pts[q][1];
                const double x = g.x0 + g.J00 * xi + g.J01 * eta;
                const double y = g.y0 + g.J10 * xi + g.J11 * eta;
                acc += A.g_scale * u0_value(A.u0_kind, x, y) * (t.bq_T[q][s] * t.S0[a]) * (g.det * t.bq_w[q]);
            }
            return acc;
        }

        __global__ void gather_vector(VecArgs A)
        {
            constexpr int kMaxInc = 64;
            for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < A.n_rows; row += gridDim.x * blockDim.x)
            {
                const int b = A.inc_ptr[row], e = A.inc_ptr[row + 1];
                if (e - b > kMaxInc)
                {
                    atomicExch(A.status, APF_ERR_CAPACITY);
                    continue;
                }
                // visit incidences in ascending (cell*ndof+i) order
                int last = -1;
                double s = 0.0;
                for (int step = 0; step < e - b; ++step)
                {
                    int best = 0x7fffffff, best_e = -1;
                    for (int q = b; q < e; ++q)
                    {
                        const int ci = A.inc[q].x;
                        if (ci > last && ci < best)
                        {
                            best = ci;
                            best_e = A.inc[q].y;
                        }
                    }
                    last = best;
                    const int c = best / A.ndof, i = best % A.ndof;
                    const double v = local_vector(A, c, i);
                    if (fabs(v) > A.d.zero_tol)
                    {
                        const double* w = A.which == 0 ? A.d.y_w : A.d.x_w;
                        s += w[best_e] * v;
                    }
                }
                A.out[row] = s;
            }
        }

        // ------------------------------------------------------------------
        // CSR algebra: K = [A B^T; B C] and Hhat
        // ------------------------------------------------------------------
        __global__ void k_row_counts(int n_lambda, int n_u, const int* __restrict__ a_ptr, const int* __restrict__ bt_ptr,
                                     const int* __restrict__ b_ptr, const int* __restrict__ c_ptr, int* __restrict__ cnt)
        {
            const int n = n_lambda + n_u;
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
            {
                if (r < n_lambda)
                    cnt[r] = (a_ptr[r + 1] - a_ptr[r]) + (bt_ptr[r + 1] - bt_ptr[r]);
                else
                {
                    const int q = r - n_lambda;
                    cnt[r] = (b_ptr[q + 1] - b_ptr[q]) + (c_ptr[q + 1] - c_ptr[q]);
                }
            }
        }

        // one warp per row: copy two CSR row segments (second shifted by n_lambda)
        __global__ void k_row_fill(int n_lambda, int n_u, const int* __restrict__ k_ptr,
                                   const int* a_ptr, const int* a_col, const double* a_val,
                                   const int* bt_ptr, const int* bt_col, const double* bt_val,
                                   const int* b_ptr, const int* b_col, const double* b_val,
                                   const int* c_ptr, const int* c_col, const double* c_val,
                                   int* __restrict__ k_col, double* __restrict__ k_val)
        {
            const int n = n_lambda + n_u;
            const int lane = threadIdx.x & 31;
            const int warps_total = (gridDim.x * blockDim.x) >> 5;
            for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += warps_total)
            {
                const int* p1; const int* c1; const double* v1;
                const int* p2; const int* c2; const double* v2;
                int q = r;
                if (r < n_lambda) { p1 = a_ptr; c1 = a_col; v1 = a_val; p2 = bt_ptr; c2 = bt_col; v2 = bt_val; }
                else { q = r - n_lambda; p1 = b_ptr; c1 = b_col; v1 = b_val; p2 = c_ptr; c2 = c_col; v2 = c_val; }
                int o = k_ptr[r];
                const int b1 = p1[q], e1 = p1[q + 1];
                for (int k = b1 + lane; k < e1; k += 32)
                {
                    k_col[o + k - b1] = c1[k];
                    k_val[o + k - b1] = v1[k];
                }
                o += e1 - b1;
                const int b2 = p2[q], e2 = p2[q + 1];
                for (int k = b2 + lane; k < e2; k += 32)
                {
                    k_col[o + k - b2] = c2[k] + n_lambda;
                    k_val[o + k - b2] = v2[k];
                }
            }
        }

        __global__ void csr_diagonal(int n, const int* __restrict__ ptr, const int* __restrict__ col,
                                     const double* __restrict__ val, double diag_tol, double* __restrict__ inv_diag,
                                     int* __restrict__ status)
        {
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
            {
                double d = 0.0;
                for (int k = ptr[r]; k < ptr[r + 1]; ++k)
                    if (col[k] == r)
                        d += val[k];
                if (!(d > diag_tol))
                {
                    atomicExch(status, APF_ERR_NUMERIC);
                    inv_diag[r] = 0.0;
                }
                else
                    inv_diag[r] = 1.0 / d;
            }
        }

        struct HhatArgs
        {
            int n_u;
            const int *c_ptr, *c_col; const double* c_val;        // C_signed
            const int *ax_ptr, *ax_col; const double* ax_val;     // A_x
            const int *bd_ptr, *bd_col; const double* bd_val;     // B_dt (rows u)
            const int *bt_ptr, *bt_col; const double* bt_val;     // B_dt^T (rows lambda)
            const double* inv_diag;                                // 1/A_y(c,c)
            int* row_count;
            const int* row_ptr;
            int* col_out;
            double* val_out;
            int* status;
            const int* list; // rows to process (null: all)
            int nlist;
        };

        // max over rows of |C row| + sum_{c in B_dt row} |B_dt^T row c| + |A_x row|
        // candidates per row (cand[row]) and their maximum (*out)
        __global__ void hhat_row_bound(HhatArgs A, int* __restrict__ out, int* __restrict__ cand)
        {
            int m = 0;
            for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < A.n_u; row += gridDim.x * blockDim.x)
            {
                int n = (A.c_ptr[row + 1] - A.c_ptr[row]) + (A.ax_ptr[row + 1] - A.ax_ptr[row]);
                for (int k = A.bd_ptr[row]; k < A.bd_ptr[row + 1]; ++k)
                {
                    const int c = A.bd_col[k];
                    n += A.bt_ptr[c + 1] - A.bt_ptr[c];
                }
                m = max(m, n);
                cand[row] = n;
            }
            for (int o = 16; o > 0; o >>= 1)
                m = max(m, __shfl_down_sync(0xffffffffu, m, o));
            if ((threadIdx.x & 31) == 0)
                atomicMax(out, m);
        }

        // Candidates: (col, value, is_ax).  Reference semantics
        // (schur_approximations.hpp:107-200, sparse_matrix_ops.hpp:286-316 with zero_tol 0):
        //   hpar = setFromTriplets(-C[nz], (1/A_cc * B_ic) * B_jc for B_ic, B_jc != 0)
        //   Hhat = setFromTriplets(hpar[nz], A_x[nz])
        // One warp per row with at most CAP candidates: the -C row, the Schur terms
        // (inv_c B_dt(row, c)) B_dt(j, c) for the nonzero B_dt entries of the row (the B_dt^T
        // rows of up to kSeg of them flattened through a prefix sum of their lengths), then
        // the A_x row, 32 at a time in that order.  Distinct columns of the kept candidates
        // go through a shared-memory hash set; only those are sorted; every candidate is then
        // added to its column's two accumulators (-C and Schur: hpar; A_x) in generation
        // order, the order in which the reference's setFromTriplets passes sum them.  Shared
        // memory per warp: table keys int[2 CAP], ranks int[2 CAP], sorted keys / (hpar, A_x)
        // accumulators 16 B x CAP, sorted columns int[CAP], then kRowExtra.
        template<int CAP>
        __global__ void __launch_bounds__(256) hhat_rows(HhatArgs A)
        {
            // CAP bounds the row's distinct columns (not its candidates, which stream through):
            // a row with more is marked (row_count = -1) and left for a larger CAP
            extern __shared__ unsigned char smem_raw[];
            const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
            unsigned char* mine = smem_raw + (size_t)w * (CAP * 36 + kRowExtra);
            int* tkeys = reinterpret_cast<int*>(mine);
            int* tranks = tkeys + 2 * CAP;
            unsigned long long* ukeys = reinterpret_cast<unsigned long long*>(tranks + 2 * CAP);
            double2* acc = reinterpret_cast<double2*>(ukeys);
            int* ucols = reinterpret_cast<int*>(acc + CAP);
            int* seg = ucols + CAP;
            double* stage = reinterpret_cast<double*>(seg + kSeg + 2);
            double* hs = reinterpret_cast<double*>(acc);
            const int nrows = A.list ? A.nlist : A.n_u;
            for (int idx = blockIdx.x * (blockDim.x >> 5) + w; idx < nrows; idx += gridDim.x * (blockDim.x >> 5))
            {
                const int row = A.list ? A.list[idx] : idx;
                // every candidate (ok, column, value, is_ax) in generation order, 32 lanes at a time
                auto for_each = [&](auto&& f) {
                    {
                        const int b = A.c_ptr[row], e = A.c_ptr[row + 1];
                        for (int k0 = b; k0 < e; k0 += 32)
                        {
                            const int k = k0 + lane;
                            const bool ok = k < e && A.c_val[k] != 0.0;
                            f(ok, ok ? A.c_col[k] : 0, ok ? -A.c_val[k] : 0.0, false);
                        }
                    }
                    const int db = A.bd_ptr[row], de = A.bd_ptr[row + 1];
                    for (int kb = db; kb < de; kb += kSeg)
                    {
                        const int cnt = min(de - kb, kSeg);
                        for (int i = lane; i < cnt; i += 32)
                        {
                            const int c = A.bd_col[kb + i];
                            seg[i + 1] = A.bd_val[kb + i] != 0.0 ? A.bt_ptr[c + 1] - A.bt_ptr[c] : 0;
                        }
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
                            bool ok = false;
                            int col = 0;
                            double contrib = 0.0;
                            if (t < nb)
                            {
                                const int i = find_segment(seg, cnt, t);
                                const int k = kb + i;
                                const int c = A.bd_col[k];
                                const int q = A.bt_ptr[c] + (t - seg[i]);
                                const double vj = A.bt_val[q];
                                contrib = (A.inv_diag[c] * A.bd_val[k]) * vj;
                                ok = vj != 0.0 && fabs(contrib) > 0.0;
                                col = A.bt_col[q];
                            }
                            f(ok, col, contrib, false);
                        }
                        __syncwarp();
                    }
                    {
                        const int b = A.ax_ptr[row], e = A.ax_ptr[row + 1];
                        for (int k0 = b; k0 < e; k0 += 32)
                        {
                            const int k = k0 + lane;
                            const bool ok = k < e && A.ax_val[k] != 0.0;
                            f(ok, ok ? A.ax_col[k] : 0, ok ? A.ax_val[k] : 0.0, true);
                        }
                    }
                };
                int n = (A.c_ptr[row + 1] - A.c_ptr[row]) + (A.ax_ptr[row + 1] - A.ax_ptr[row]);
                for (int k = A.bd_ptr[row]; k < A.bd_ptr[row + 1]; ++k)
                    n += A.bt_ptr[A.bd_col[k] + 1] - A.bt_ptr[A.bd_col[k]];
                // table at most half full: 2 min(n, CAP) slots (+ one group of 32 beyond CAP
                // before the overflow is seen)
                int hbits = 6;
                while ((1 << hbits) < 2 * min(n, CAP))
                    ++hbits;
                const int H = 1 << hbits;
                for (int t = lane; t < H; t += 32)
                    tkeys[t] = -1;
                __syncwarp();
                int distinct = 0;
                bool overflow = false;
                for_each([&](bool ok, int col, double, bool) {
                    const bool fresh = ok && !overflow && hash_insert_new(tkeys, col, hbits);
                    distinct += __popc(__ballot_sync(0xffffffffu, fresh));
                    overflow = overflow || distinct > CAP;
                });
                __syncwarp();
                if (overflow)
                {
                    if (lane == 0)
                        A.row_count[row] = -1;
                    __syncwarp();
                    continue;
                }
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
                for (int k = lane; k < u; k += 32)
                {
                    const unsigned long long key = ukeys[k];
                    tranks[static_cast<unsigned>(key)] = k;
                    ucols[k] = static_cast<int>(key >> 32);
                }
                __syncwarp();
                for (int k = lane; k < u; k += 32)
                    acc[k] = make_double2(0.0, 0.0);
                __syncwarp();
                // hpar and A_x sums of each column live side by side: rank r -> hs[2 r] / hs[2 r + 1]
                for_each([&](bool ok, int col, double v, bool is_ax) {
                    const int r = ok ? hash_rank(tkeys, tranks, col, hbits) : 0;
                    ordered_add(hs, stage, ok, 2 * r + (is_ax ? 1 : 0), v, lane);
                });
                // kept entries (hpar or A_x nonzero) in column order to the row's segment
                const int out_base = A.row_ptr[row];
                int kept = 0;
                for (int k0 = 0; k0 < u; k0 += 32)
                {
                    const int k = k0 + lane;
                    double h = 0.0, a = 0.0;
                    if (k < u)
                    {
                        h = acc[k].x;
                        a = acc[k].y;
                    }
                    const bool keep = k < u && (h != 0.0 || a != 0.0);
                    const unsigned km = __ballot_sync(0xffffffffu, keep);
                    if (keep)
                    {
                        const int pos = out_base + kept + __popc(km & ((1u << lane) - 1));
                        A.col_out[pos] = ucols[k];
                        A.val_out[pos] = h + a;
                    }
                    kept += __popc(km);
                }
                if (lane == 0)
                    A.row_count[row] = kept;
                __syncwarp();
            }
        }

        // rows (of list, or all) whose count is the overflow mark -1
        __global__ void overflow_flags(int n, const int* __restrict__ list, const int* __restrict__ counts,
                                       int* __restrict__ flag)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                flag[i] = counts[list ? list[i] : i] < 0 ? 1 : 0;
        }

        __global__ void overflow_compact(int n, const int* __restrict__ list, const int* __restrict__ flag,
                                         const int* __restrict__ pos, int* __restrict__ out)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                if (flag[i])
                    out[pos[i]] = list ? list[i] : i;
        }

        // one warp per row: the row's kept entries from its staging segment to the result
        __global__ void hhat_compact(int rows, const int* __restrict__ cand_ptr, const int* __restrict__ tc,
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

        int grid_for(long long work, int block, int max_blocks = 148 * 32)
        {
            long long g = (work + block - 1) / block;
            if (g < 1) g = 1;
            if (g > max_blocks) g = max_blocks;
            return static_cast<int>(g);
        }
    } // namespace

    // ----------------------------------------------------------------------
    // host orchestration
    // ----------------------------------------------------------------------
    void upload_tables_once(int device)
    {
        static bool done[64] = {};
        if (device >= 0 && device < 64 && done[device])
            return;
        RefTables t[2] = {make_ref_tables(1), make_ref_tables(2)};
        APF_CUDA(cudaMemcpyToSymbol(c_tab, t, sizeof(t)));
        if (device >= 0 && device < 64)
            done[device] = true;
    }

    Incidence build_incidence(cudaStream_t s, int n_dofs, int n_asm, const int* cell_list, const int* src_map,
                              const int* offsets, const int* dofs, int ndof)
    {
        Incidence inc;
        inc.ptr.allocate(static_cast<std::size_t>(n_dofs) + 1, s);
        DeviceBuffer<int> count(static_cast<std::size_t>(n_dofs) + 1, s);
        count.zero();
        IncidenceSpec spec{n_asm, cell_list, src_map, offsets, dofs, ndof};
        const long long work = static_cast<long long>(n_asm) * ndof;
        if (work > 0)
        {
            {
                APF_KERNEL("incidence_count", s);
                incidence_count<<<grid_for(work, 256), 256, 0, s>>>(spec, count.get());
            }
        }
        APF_CUDA(cudaGetLastError());
        const long long total = exclusive_scan(count.get(), inc.ptr.get(), n_dofs, s);
        inc.entries.allocate(static_cast<std::size_t>(std::max<long long>(total, 1)), s);
        count.zero();
        if (work > 0)
        {
            {
                APF_KERNEL("incidence_fill", s);
                incidence_fill<<<grid_for(work, 256), 256, 0, s>>>(spec, inc.ptr.get(), count.get(), inc.entries.get());
            }
        }
        APF_CUDA(cudaGetLastError());
        DeviceBuffer<int> mx(1, s);
        mx.zero();
        if (n_dofs > 0)
        {
            {
                APF_KERNEL("max_row_length", s);
                max_row_length<<<grid_for(n_dofs, 256, 1024), 256, 0, s>>>(inc.ptr.get(), n_dofs, mx.get());
            }
        }
        APF_CUDA(cudaMemcpyAsync(&inc.max_len, mx.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        sync(s);
        return inc;
    }

    namespace
    {
        AsmData make_asm_data(const SystemInputs& in, double zero_tol)
        {
            AsmData d{};
            d.p = in.p;
            d.dim = in.dim;
            d.y_geo = in.y_geo.get();
            d.x_geo = in.x_geo.get();
            d.y_to_x = in.y_to_x.get();
            d.m_y = in.m_y.size() ? in.m_y.get() : nullptr;
            d.m_x = in.m_x.size() ? in.m_x.get() : nullptr;
            d.y_off = in.y_off.get();
            d.y_dofs = in.y_dofs.get();
            d.y_w = in.y_w.get();
            d.x_off = in.x_off.get();
            d.x_dofs = in.x_dofs.get();
            d.x_w = in.x_w.get();
            d.zero_tol = zero_tol;
            return d;
        }

        // candidates of each row: incidences x local DOFs x restriction entries per term
        __global__ void gather_candidates(int n_rows, Term t0, Term t1, int n_terms, int per_incidence,
                                          int* __restrict__ cand)
        {
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += gridDim.x * blockDim.x)
            {
                int n = (t0.inc_ptr[r + 1] - t0.inc_ptr[r]);
                if (n_terms > 1)
                    n += t1.inc_ptr[r + 1] - t1.inc_ptr[r];
                cand[r] = n * per_incidence;
            }
        }

        __global__ void gather_compact(int rows, const int* __restrict__ cand_ptr, const int* __restrict__ tc,
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

        int check_status(DeviceBuffer<int>& st, cudaStream_t s)
        {
            int h = 0;
            APF_CUDA(cudaMemcpyAsync(&h, st.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
            sync(s);
            return h;
        }
    }

    // Build one CSR block from up to two gather terms.
    void gather_csr(cudaStream_t s, const SystemInputs& in, double zero_tol, int n_rows, int n_cols, int n_terms,
                    const int* kinds, const Incidence* const* incs, const int* col_offsets, int kmax, DeviceCsr& out)
    {
        GatherArgs a{};
        a.d = make_asm_data(in, zero_tol);
        a.n_rows = n_rows;
        a.ndof = in.ndof;
        a.n_terms = n_terms;
        int cap = 0;
        for (int t = 0; t < n_terms; ++t)
        {
            a.term[t] = Term{kinds[t], incs[t]->ptr.get(), incs[t]->entries.get(), col_offsets[t]};
            require(incs[t]->max_len <= 256, APF_ERR_CAPACITY, "a DOF has more than 256 cell incidences");
            cap += incs[t]->max_len * in.ndof * kmax;
        }
        require(kmax <= kMaxRestrictionEntries, APF_ERR_CAPACITY, "restriction rows with more than 16 entries are not supported");
        DeviceBuffer<int> status(1, s);
        status.zero();
        a.status = status.get();
        // one sorting pass: each row's distinct entries go to its candidate segment of
        // staging arrays (sized by incidences x local DOFs x restriction entries), then a
        // compaction into the CSR block
        DeviceBuffer<int> counts(static_cast<std::size_t>(n_rows) + 1, s), cand(static_cast<std::size_t>(n_rows) + 1, s),
            cand_ptr(static_cast<std::size_t>(n_rows) + 1, s);
        if (n_rows > 0)
        {
            APF_KERNEL("gather_candidates", s);
            gather_candidates<<<grid_for(n_rows, 256), 256, 0, s>>>(n_rows, a.term[0], a.term[n_terms > 1 ? 1 : 0],
                                                                    n_terms, in.ndof * kmax, cand.get());
        }
        const long long total = exclusive_scan(cand.get(), cand_ptr.get(), n_rows, s);
        DeviceBuffer<int> tc(static_cast<std::size_t>(std::max(total, 1ll)), s);
        DeviceBuffer<double> tv(static_cast<std::size_t>(std::max(total, 1ll)), s);
        a.row_count = counts.get();
        a.row_ptr = cand_ptr.get();
        a.col_out = tc.get();
        a.val_out = tv.get();
        // every row with room for 128 distinct columns (the candidates stream through), then
        // the rows that had more with 1024, then 4096
        (void)cap;
        a.kmax = kmax;
        auto run = [&](auto tag) {
            constexpr int UCAP = decltype(tag)::value;
            const int warps = std::max(1, std::min(4, static_cast<int>((96 * 1024) / gather_u_warp_bytes<UCAP>())));
            const size_t smem = warps * gather_u_warp_bytes<UCAP>();
            const int blocks = grid_for(a.list ? a.nlist : n_rows, warps, 148 * 64);
            APF_CUDA(cudaFuncSetAttribute(gather_rows_u<UCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            APF_KERNEL("gather_rows_fill", s);
            gather_rows_u<UCAP><<<blocks, warps * 32, smem, s>>>(a);
            APF_CUDA(cudaGetLastError());
        };
        a.list = nullptr;
        a.nlist = n_rows;
        if (n_rows > 0)
            run(std::integral_constant<int, 128>{});
        DeviceBuffer<int> oflag(static_cast<std::size_t>(n_rows) + 1, s), opos(static_cast<std::size_t>(n_rows) + 1, s),
            olist(1, s);
        for (int pass = 0; pass < 3 && n_rows > 0; ++pass)
        {
            const int nin = a.list ? a.nlist : n_rows;
            {
                APF_KERNEL("gather_overflow_rows", s);
                overflow_flags<<<grid_for(nin, 256), 256, 0, s>>>(nin, a.list, counts.get(), oflag.get());
            }
            const int nover = static_cast<int>(exclusive_scan(oflag.get(), opos.get(), nin, s));
            if (nover == 0)
                break;
            require(pass < 2, APF_ERR_CAPACITY, "assembly: a row has more than 4096 distinct columns");
            DeviceBuffer<int> next(static_cast<std::size_t>(nover), s);
            {
                APF_KERNEL("gather_overflow_rows", s);
                overflow_compact<<<grid_for(nin, 256), 256, 0, s>>>(nin, a.list, oflag.get(), opos.get(), next.get());
            }
            olist = std::move(next);
            a.list = olist.get();
            a.nlist = nover;
            if (pass == 0)
                run(std::integral_constant<int, 1024>{});
            else
                run(std::integral_constant<int, 4096>{});
        }
        out.rows = n_rows;
        out.cols = n_cols;
        out.row_ptr.allocate(static_cast<std::size_t>(n_rows) + 1, s);
        const long long nnz = exclusive_scan(counts.get(), out.row_ptr.get(), n_rows, s);
        if (check_status(status, s) != 0)
            throw Error(APF_ERR_CAPACITY, "assembly: per-row candidate buffer overflow");
        out.col_idx.allocate(static_cast<std::size_t>(nnz), s);
        out.values.allocate(static_cast<std::size_t>(nnz), s);
        if (n_rows > 0)
        {
            APF_KERNEL("gather_compact", s);
            gather_compact<<<grid_for((long long)n_rows * 32, 256, 148 * 16), 256, 0, s>>>(
                n_rows, cand_ptr.get(), tc.get(), tv.get(), out.row_ptr.get(), out.col_idx.get(), out.values.get());
        }
        APF_CUDA(cudaGetLastError());
    }

    void gather_vector_host(cudaStream_t s, const SystemInputs& in, double zero_tol, int which, const Incidence& inc,
                            int n_rows, const double* ell, int u0_kind, double g_scale, DeviceBuffer<double>& out)
    {
        VecArgs a{};
        a.d = make_asm_data(in, zero_tol);
        a.n_rows = n_rows;
        a.ndof = in.ndof;
        a.inc_ptr = inc.ptr.get();
        a.inc = inc.entries.get();
        a.which = which;
        a.ell = ell;
        a.u0_kind = u0_kind;
        a.g_scale = g_scale;
        out.allocate(static_cast<std::size_t>(n_rows), s);
        a.out = out.get();
        DeviceBuffer<int> status(1, s);
        status.zero();
        a.status = status.get();
        if (n_rows > 0)
        {
            {
                APF_KERNEL("gather_vector", s);
                gather_vector<<<grid_for(n_rows, 128), 128, 0, s>>>(a);
            }
            APF_CUDA(cudaGetLastError());
        }
        if (check_status(status, s) != 0)
            throw Error(APF_ERR_CAPACITY, "assembly: more than 64 incidences for a vector row");
    }

    void build_k(cudaStream_t s, int n_lambda, int n_u, const DeviceCsr& a, const DeviceCsr& bt, const DeviceCsr& b,
                 const DeviceCsr& c, DeviceCsr& k)
    {
        const int n = n_lambda + n_u;
        DeviceBuffer<int> cnt(static_cast<std::size_t>(n) + 1, s);
        {
            APF_KERNEL("k_row_counts", s);
            k_row_counts<<<grid_for(n, 256), 256, 0, s>>>(n_lambda, n_u, a.row_ptr.get(), bt.row_ptr.get(), b.row_ptr.get(),
                                                          c.row_ptr.get(), cnt.get());
        }
        APF_CUDA(cudaGetLastError());
        k.rows = k.cols = n;
        k.row_ptr.allocate(static_cast<std::size_t>(n) + 1, s);
        const long long nnz = exclusive_scan(cnt.get(), k.row_ptr.get(), n, s);
        k.col_idx.allocate(static_cast<std::size_t>(nnz), s);
        k.values.allocate(static_cast<std::size_t>(nnz), s);
        {
            APF_KERNEL("k_row_fill", s);
            k_row_fill<<<grid_for((long long)n * 32, 256), 256, 0, s>>>(
                n_lambda, n_u, k.row_ptr.get(), a.row_ptr.get(), a.col_idx.get(), a.values.get(), bt.row_ptr.get(),
                bt.col_idx.get(), bt.values.get(), b.row_ptr.get(), b.col_idx.get(), b.values.get(), c.row_ptr.get(),
                c.col_idx.get(), c.values.get(), k.col_idx.get(), k.values.get());
        }
        APF_CUDA(cudaGetLastError());
    }

    void full_saddle_pattern(cudaStream_t s, const SystemInputs& in, const Incidence& inc_y, const Incidence& inc_xy,
                             const Incidence& inc_xb, DeviceBuffer<int>& row_ptr, DeviceBuffer<int>& col_idx)
    {
        const int n_lambda = in.n_lambda, n_u = in.n_u, n = n_lambda + n_u;
        // a negative filter keeps every candidate: the structural union of the restricted
        // couplings (the values of this pass are not used)
        DeviceCsr top, bottom;
        {
            const int kinds[2] = {K_AY, K_BT};
            const Incidence* incs[2] = {&inc_y, &inc_y};
            const int offs[2] = {0, n_lambda};
            gather_csr(s, in, -1.0, n_lambda, n, 2, kinds, incs, offs, in.kmax, top);
        }
        {
            const int kinds[2] = {K_B, K_C};
            const Incidence* incs[2] = {&inc_xy, &inc_xb};
            const int offs[2] = {0, n_lambda};
            gather_csr(s, in, -1.0, n_u, n, 2, kinds, incs, offs, in.kmax, bottom);
        }
        row_ptr.allocate(static_cast<std::size_t>(n) + 1, s);
        {
            APF_KERNEL("stack_row_ptr", s);
            stack_row_ptr<<<grid_for(n + 1, 256), 256, 0, s>>>(n_lambda, top.row_ptr.get(), n_u, bottom.row_ptr.get(),
                                                               row_ptr.get());
        }
        APF_CUDA(cudaGetLastError());
        const std::size_t nt = top.col_idx.size(), nb = bottom.col_idx.size();
        col_idx.allocate(nt + nb, s);
        if (nt)
            APF_CUDA(cudaMemcpyAsync(col_idx.get(), top.col_idx.get(), nt * sizeof(int), cudaMemcpyDeviceToDevice, s));
        if (nb)
            APF_CUDA(cudaMemcpyAsync(col_idx.get() + nt, bottom.col_idx.get(), nb * sizeof(int),
                                     cudaMemcpyDeviceToDevice, s));
    }

    void full_saddle_numeric(cudaStream_t s, const SystemInputs& in, const Incidence& inc_y, const Incidence& inc_xy,
                             const Incidence& inc_xb, const int* row_ptr, const int* col_idx, long long nnz_pattern,
                             DeviceCsr& K)
    {
        const int n_lambda = in.n_lambda, n_u = in.n_u, n = n_lambda + n_u;
        require(in.kmax <= kMaxRestrictionEntries, APF_ERR_CAPACITY, "restriction rows with more than 16 entries are not supported");
        DeviceBuffer<double> vals(static_cast<std::size_t>(std::max(nnz_pattern, 1ll)), s);
        DeviceBuffer<int> status(1, s);
        status.zero();
        auto fill = [&](int n_rows, int row_base, int k0, const Incidence& i0, int k1, const Incidence& i1) {
            if (n_rows == 0)
                return;
            require(i0.max_len <= kGatherIncCap && i1.max_len <= kGatherIncCap, APF_ERR_CAPACITY,
                    "a DOF has more than 256 cell incidences");
            GatherArgs a{};
            a.d = make_asm_data(in, in.zero_tol);
            a.n_rows = n_rows;
            a.ndof = in.ndof;
            a.n_terms = 2;
            a.term[0] = Term{k0, i0.ptr.get(), i0.entries.get(), 0};
            a.term[1] = Term{k1, i1.ptr.get(), i1.entries.get(), n_lambda};
            a.status = status.get();
            a.kmax = in.kmax;
            APF_KERNEL("fill_rows_on_pattern", s);
            fill_rows_on_pattern<<<grid_for(n_rows, kFillWarps, 148 * 64), kFillWarps * 32, 0, s>>>(
                a, row_base, row_ptr, col_idx, vals.get());
            APF_CUDA(cudaGetLastError());
        };
        fill(n_lambda, 0, K_AY, inc_y, K_BT, inc_y);
        fill(n_u, n_lambda, K_B, inc_xy, K_C, inc_xb);
        const int st = check_status(status, s);
        if (st == APF_ERR_INVALID)
            throw Error(APF_ERR_INVALID, "two-pass assembly: a coupling lies outside the cached pattern "
                                         "(the pattern belongs to another mesh)");
        if (st != 0)
            throw Error(APF_ERR_CAPACITY, "two-pass assembly: more than 256 cell incidences for a DOF");
        // prune(1.0, zero_tol): keep |value| > zero_tol
        DeviceBuffer<int> cnt(static_cast<std::size_t>(n) + 1, s);
        if (n > 0)
        {
            APF_KERNEL("prune_count", s);
            prune_count<<<grid_for(n, 256), 256, 0, s>>>(n, row_ptr, vals.get(), in.zero_tol, cnt.get());
            APF_CUDA(cudaGetLastError());
        }
        K.rows = K.cols = n;
        K.row_ptr.allocate(static_cast<std::size_t>(n) + 1, s);
        const long long nnz = exclusive_scan(cnt.get(), K.row_ptr.get(), n, s);
        K.col_idx.allocate(static_cast<std::size_t>(nnz), s);
        K.values.allocate(static_cast<std::size_t>(nnz), s);
        if (n > 0)
        {
            APF_KERNEL("prune_fill", s);
            prune_fill<<<grid_for((long long)n * 32, 256, 148 * 16), 256, 0, s>>>(
                n, row_ptr, col_idx, vals.get(), in.zero_tol, K.row_ptr.get(), K.col_idx.get(), K.values.get());
            APF_CUDA(cudaGetLastError());
        }
    }

    void build_hhat(cudaStream_t s, const DeviceCsr& A_y, const DeviceCsr& C, const DeviceCsr& A_x, const DeviceCsr& B_dt,
                    const DeviceCsr& B_dtT, double diag_tol, DeviceCsr& H, DeviceBuffer<double>& inv_diag)
    {
        const int n_u = C.rows;
        DeviceBuffer<int> status(1, s);
        status.zero();
        inv_diag.allocate(static_cast<std::size_t>(A_y.rows), s);
        {
            APF_KERNEL("csr_diagonal", s);
            csr_diagonal<<<grid_for(A_y.rows, 256), 256, 0, s>>>(A_y.rows, A_y.row_ptr.get(), A_y.col_idx.get(),
                                                                 A_y.values.get(), diag_tol, inv_diag.get(), status.get());
        }
        APF_CUDA(cudaGetLastError());
        if (check_status(status, s) != 0)
            throw Error(APF_ERR_NUMERIC, "diagonal_schur_approximation: A_y diagonal must be positive.");
        HhatArgs a{};
        a.n_u = n_u;
        a.c_ptr = C.row_ptr.get(); a.c_col = C.col_idx.get(); a.c_val = C.values.get();
        a.ax_ptr = A_x.row_ptr.get(); a.ax_col = A_x.col_idx.get(); a.ax_val = A_x.values.get();
        a.bd_ptr = B_dt.row_ptr.get(); a.bd_col = B_dt.col_idx.get(); a.bd_val = B_dt.values.get();
        a.bt_ptr = B_dtT.row_ptr.get(); a.bt_col = B_dtT.col_idx.get(); a.bt_val = B_dtT.values.get();
        a.inv_diag = inv_diag.get();
        a.status = status.get();
        DeviceBuffer<int> counts(static_cast<std::size_t>(n_u) + 1, s);
        a.row_count = counts.get();
        // candidates per row -> shared-memory capacity and the staging segments of the one
        // sorting pass (each row's kept entries land in its segment, then a compaction)
        DeviceBuffer<int> bound(1, s), cand(static_cast<std::size_t>(n_u) + 1, s),
            cand_ptr(static_cast<std::size_t>(n_u) + 1, s);
        bound.zero();
        if (n_u > 0)
        {
            APF_KERNEL("hhat_row_bound", s);
            hhat_row_bound<<<grid_for(n_u, 256, 148 * 8), 256, 0, s>>>(a, bound.get(), cand.get());
        }
        const long long total = exclusive_scan(cand.get(), cand_ptr.get(), n_u, s);
        DeviceBuffer<int> tc(static_cast<std::size_t>(std::max(total, 1ll)), s);
        DeviceBuffer<double> tv(static_cast<std::size_t>(std::max(total, 1ll)), s);
        auto run = [&](auto cap_tag) {
            constexpr int CAP = decltype(cap_tag)::value;
            const int warps = std::max(1, std::min(8, (96 * 1024) / (CAP * 36 + kRowExtra)));
            const int threads = warps * 32;
            const size_t smem = (size_t)warps * (CAP * 36 + kRowExtra);
            const int blocks = grid_for(a.list ? a.nlist : n_u, warps, 148 * 32);
            APF_CUDA(cudaFuncSetAttribute(hhat_rows<CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            APF_KERNEL("hhat_rows_fill", s);
            hhat_rows<CAP><<<blocks, threads, smem, s>>>(a);
            APF_CUDA(cudaGetLastError());
        };
        a.row_ptr = cand_ptr.get();
        a.col_out = tc.get();
        a.val_out = tv.get();
        // every row with room for 128 distinct columns (the candidates stream through), then
        // the rows that had more with 1024, then 4096
        a.list = nullptr;
        a.nlist = n_u;
        if (n_u > 0)
            run(std::integral_constant<int, 128>{});
        DeviceBuffer<int> oflag(static_cast<std::size_t>(n_u) + 1, s), opos(static_cast<std::size_t>(n_u) + 1, s),
            olist(static_cast<std::size_t>(std::max(n_u, 1)), s);
        for (int pass = 0; pass < 2 && n_u > 0; ++pass)
        {
            {
                APF_KERNEL("hhat_overflow_rows", s);
                overflow_flags<<<grid_for(n_u, 256), 256, 0, s>>>(a.list ? a.nlist : n_u, a.list, counts.get(),
                                                                 oflag.get());
            }
            const int nover = static_cast<int>(exclusive_scan(oflag.get(), opos.get(), a.list ? a.nlist : n_u, s));
            if (nover == 0)
                break;
            DeviceBuffer<int> next(static_cast<std::size_t>(nover), s);
            {
                APF_KERNEL("hhat_overflow_rows", s);
                overflow_compact<<<grid_for(n_u, 256), 256, 0, s>>>(a.list ? a.nlist : n_u, a.list, oflag.get(),
                                                                   opos.get(), next.get());
            }
            olist = std::move(next);
            a.list = olist.get();
            a.nlist = nover;
            if (pass == 0)
                run(std::integral_constant<int, 1024>{});
            else
                run(std::integral_constant<int, 4096>{});
        }
        if (n_u > 0 && a.list)
        {
            APF_KERNEL("hhat_overflow_rows", s);
            overflow_flags<<<grid_for(n_u, 256), 256, 0, s>>>(a.nlist, a.list, counts.get(), oflag.get());
            if (exclusive_scan(oflag.get(), opos.get(), a.nlist, s) != 0)
                throw Error(APF_ERR_CAPACITY, "graph norm: a row has more than 4096 distinct columns");
        }
        H.rows = H.cols = n_u;
        H.row_ptr.allocate(static_cast<std::size_t>(n_u) + 1, s);
        const long long nnz = exclusive_scan(counts.get(), H.row_ptr.get(), n_u, s);
        if (check_status(status, s) != 0)
            throw Error(APF_ERR_CAPACITY, "graph norm: per-row candidate buffer overflow");
        H.col_idx.allocate(static_cast<std::size_t>(nnz), s);
        H.values.allocate(static_cast<std::size_t>(nnz), s);
        if (n_u > 0)
        {
            APF_KERNEL("hhat_compact", s);
            hhat_compact<<<grid_for((long long)n_u * 32, 256, 148 * 16), 256, 0, s>>>(
                n_u, cand_ptr.get(), tc.get(), tv.get(), H.row_ptr.get(), H.col_idx.get(), H.values.get());
        }
        APF_CUDA(cudaGetLastError());
    }

    // M per X cell, taken from the Y cells it contains (M is cell-constant).
    namespace
    {
        // mw values of M per cell (3 in 2+1D: m00 m01 m11; 1 in 1+1D)
        __global__ void scatter_m_to_x(int ny, int mw, const int* __restrict__ y_to_x, const double* __restrict__ m_y,
                                       double* __restrict__ m_x)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ny; c += gridDim.x * blockDim.x)
            {
                const int x = y_to_x[c];
                for (int k = 0; k < mw; ++k)
                    m_x[(long long)mw * x + k] = m_y[(long long)mw * c + k];
            }
        }

        // gw doubles per geometry row; t0 at offset gw - 2
        __global__ void mark_bottom(int nx, int gw, const double* __restrict__ x_geo, int* __restrict__ flag)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nx; c += gridDim.x * blockDim.x)
                flag[c] = x_geo[(long long)gw * c + gw - 2] == 0.0 ? 1 : 0;
        }

        __global__ void compact_flags(int n, const int* __restrict__ flag, const int* __restrict__ pos,
                                      int* __restrict__ list)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
                if (flag[c])
                    list[pos[c]] = c;
        }

        __global__ void max_restr_row(int n, const int* __restrict__ off, int* __restrict__ out)
        {
            int m = 0;
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                m = max(m, off[i + 1] - off[i]);
            for (int o = 16; o > 0; o >>= 1)
                m = max(m, __shfl_down_sync(0xffffffffu, m, o));
            if ((threadIdx.x & 31) == 0)
                atomicMax(out, m);
        }
    }

    namespace
    {
        // time coordinate of every true DOF named by a restriction row, quantized to 2^-20
        // (dyadic mesh times are exact): DOFs on one time level share a component
        __global__ void dof_time_component(int rows, int ndof, int p, int gw, const double* __restrict__ geo,
                                           const int* __restrict__ off, const int* __restrict__ dofs,
                                           int* __restrict__ comp)
        {
            for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
            {
                const int c = r / ndof, a = (r % ndof) % (p + 1);
                const double t0 = geo[(long long)gw * c + gw - 2], t1 = geo[(long long)gw * c + gw - 1];
                const int level = static_cast<int>(llround((t0 + (t1 - t0) * a / p) * 1048576.0));
                for (int e = off[r]; e < off[r + 1]; ++e)
                    comp[dofs[e]] = level;
            }
        }
    }

    void dof_time_components(cudaStream_t s, const SystemInputs& in, bool y_space, DeviceBuffer<int>& comp)
    {
        const int n = y_space ? in.n_lambda : in.n_u;
        comp.allocate(static_cast<std::size_t>(n), s);
        comp.zero();
        const int rows = (y_space ? in.n_y_cells : in.n_x_cells) * in.ndof;
        if (rows > 0)
        {
            APF_KERNEL("dof_time_component", s);
            dof_time_component<<<grid_for(rows, 256), 256, 0, s>>>(
                rows, in.ndof, in.p, in.dim == 1 ? 4 : 8, y_space ? in.y_geo.get() : in.x_geo.get(),
                y_space ? in.y_off.get() : in.x_off.get(),
                y_space ? in.y_dofs.get() : in.x_dofs.get(), comp.get());
        }
        APF_CUDA(cudaGetLastError());
    }

    void prepare_inputs(cudaStream_t s, SystemInputs& in)
    {
        // M on X cells
        const int mw = in.dim == 1 ? 1 : 3, gw = in.dim == 1 ? 4 : 8;
        if (in.m_y.size())
        {
            in.m_x.allocate(static_cast<std::size_t>(in.n_x_cells) * mw, s);
            std::vector<double> ident;
            // default identity for X cells not covered (should not happen for a valid Y/X pair)
            ident.resize(static_cast<std::size_t>(in.n_x_cells) * mw);
            for (int c = 0; c < in.n_x_cells; ++c)
            {
                if (mw == 1)
                    ident[c] = 1.0;
                else
                {
                    ident[3 * c] = 1.0; ident[3 * c + 1] = 0.0; ident[3 * c + 2] = 1.0;
                }
            }
            APF_CUDA(cudaMemcpyAsync(in.m_x.get(), ident.data(), ident.size() * sizeof(double), cudaMemcpyHostToDevice, s));
            {
                APF_KERNEL("scatter_m_to_x", s);
                scatter_m_to_x<<<grid_for(in.n_y_cells, 256), 256, 0, s>>>(in.n_y_cells, mw, in.y_to_x.get(), in.m_y.get(),
                                                                           in.m_x.get());
            }
            APF_CUDA(cudaGetLastError());
            sync(s);
        }
        // bottom X cells (temporal boundary at t = 0)
        DeviceBuffer<int> flag(static_cast<std::size_t>(in.n_x_cells) + 1, s);
        DeviceBuffer<int> pos(static_cast<std::size_t>(in.n_x_cells) + 1, s);
        if (in.n_x_cells > 0)
        {
            {
                APF_KERNEL("mark_bottom", s);
                mark_bottom<<<grid_for(in.n_x_cells, 256), 256, 0, s>>>(in.n_x_cells, gw, in.x_geo.get(), flag.get());
            }
        }
        const long long nb = exclusive_scan(flag.get(), pos.get(), in.n_x_cells, s);
        in.n_bottom = static_cast<int>(nb);
        in.bottom_list.allocate(static_cast<std::size_t>(std::max<long long>(nb, 1)), s);
        if (in.n_x_cells > 0)
        {
            {
                APF_KERNEL("compact_flags", s);
                compact_flags<<<grid_for(in.n_x_cells, 256), 256, 0, s>>>(in.n_x_cells, flag.get(), pos.get(), in.bottom_list.get());
            }
        }
        // max entries per restriction row
        DeviceBuffer<int> mx(1, s);
        mx.zero();
        const int ny_rows = in.n_y_cells * in.ndof, nx_rows = in.n_x_cells * in.ndof;
        if (ny_rows > 0)
            {
                APF_KERNEL("max_restr_row", s);
                max_restr_row<<<grid_for(ny_rows, 256, 1024), 256, 0, s>>>(ny_rows, in.y_off.get(), mx.get());
            }
        if (nx_rows > 0)
            {
                APF_KERNEL("max_restr_row", s);
                max_restr_row<<<grid_for(nx_rows, 256, 1024), 256, 0, s>>>(nx_rows, in.x_off.get(), mx.get());
            }
        APF_CUDA(cudaGetLastError());
        APF_CUDA(cudaMemcpyAsync(&in.kmax, mx.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        sync(s);
        if (in.kmax < 1)
            in.kmax = 1;
    }
}

// ---------------------------------------------------------------------------------------
// X-marking indicators of the adaptive driver (algorithm/detail/indicator_utilities.hpp:
// compute_x_marking_indicator_components :443-473, compute_spatial_energy_squared_by_active_cell
// :115-171, aggregate_to_x_active_cells :405-433, compute_initial_trace_mismatch_squared_by_x_cell
// :336-400)
// ---------------------------------------------------------------------------------------
namespace apf
{
    namespace
    {
        // nodal values of a true-DOF vector on local DOF i of cell c (restriction row)
        __device__ __forceinline__ double local_value(const int* off, const int* dofs, const double* w, const double* v,
                                                      long long row)
        {
            double s = 0.0;
            for (int e = off[row]; e < off[row + 1]; ++e)
                s += w[e] * v[dofs[e]];
            return s;
        }

        // lambda_y^2_K = int_K grad_x lambda . M grad_x lambda: the local A_y energy of lambda_delta
        __global__ void lambda_energy_kernel(XIndArgs A)
        {
            const RefTables& t = c_tab[A.p - 1];
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.n_y; c += gridDim.x * blockDim.x)
            {
                double lam[kMaxNs * kMaxNt];
                for (int i = 0; i < t.ndof; ++i)
                    lam[i] = local_value(A.y_off, A.y_dofs, A.y_w, A.lambda, static_cast<long long>(c) * t.ndof + i);
                const CellGeo g = load_geo(A.y_geo, c);
                double q00, q01, q11;
                q_form(g, A.m_y, c, q00, q01, q11);
                double e = 0.0;
                for (int i = 0; i < t.ndof; ++i)
                {
                    const int s = i / t.nt, a = i % t.nt;
                    double row = 0.0;
                    for (int j = 0; j < t.ndof; ++j)
                    {
                        const int r = j / t.nt, b = j % t.nt;
                        row += t.Mt[a][b] * ks(t, q00, q01, q11, s, r) * lam[j];
                    }
                    e += lam[i] * row;
                }
                A.lam_y[c] = g.det * g.ht * e;
            }
        }

        // ||u0 - u_delta(., 0)||^2 on the bottom face of every X cell at t = 0 (bottom Duffy rule)
        __global__ void initial_trace_kernel(XIndArgs A)
        {
            const RefTables& t = c_tab[A.p - 1];
            for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < A.n_bottom; k += gridDim.x * blockDim.x)
            {
                const int c = A.bottom[k];
                double u[kMaxNs * kMaxNt];
                for (int i = 0; i < t.ndof; ++i)
                    u[i] = local_value(A.x_off, A.x_dofs, A.x_w, A.u, static_cast<long long>(c) * t.ndof + i);
                const CellGeo g = load_geo(A.x_geo, c);
                double acc = 0.0;
                for (int q = 0; q < t.nbq; ++q)
                {
                    const double xi = t.bq_pts[q][0], eta = t.bq_pts[q][1];
                    const double x = g.x0 + g.J00 * xi + g.J01 * eta;
                    const double y = g.y0 + g.J10 * xi + g.J11 * eta;
                    double uh = 0.0;
                    for (int s = 0; s < t.ns; ++s)
                        for (int a = 0; a < t.nt; ++a)
                            uh += u[s * t.nt + a] * t.bq_T[q][s] * t.S0[a];
                    const double d = u0_value(A.u0_kind, x, y) - uh;
                    acc += d * d * g.det * t.bq_w[q];
                }
                A.trace_x[c] = acc;
            }
        }

        // 1+1D: lambda_y^2_K = m (k / h) sum_ij D_sr Mt_ab lambda_i lambda_j
        __global__ void lambda_energy_1d_kernel(XIndArgs A)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.n_y; c += gridDim.x * blockDim.x)
            {
                double lam[4];
                for (int i = 0; i < 4; ++i)
                    lam[i] = local_value(A.y_off, A.y_dofs, A.y_w, A.lambda, 4ll * c + i);
                const q1d::Quad g = q1d::load(A.y_geo, c);
                const double m = A.m_y ? A.m_y[c] : 1.0;
                double e = 0.0;
                for (int i = 0; i < 4; ++i)
                {
                    double row = 0.0;
                    for (int j = 0; j < 4; ++j)
                        row += q1d::stiff(i >> 1, j >> 1) * q1d::mass(i & 1, j & 1) * lam[j];
                    e += lam[i] * row;
                }
                A.lam_y[c] = m * (g.k / g.h) * e;
            }
        }

        // 1+1D: ||u0 - u_delta(., 0)||^2 on the bottom edge, 3-point Gauss rule
        __global__ void initial_trace_1d_kernel(XIndArgs A)
        {
            for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < A.n_bottom; k += gridDim.x * blockDim.x)
            {
                const int c = A.bottom[k];
                const double u0l = local_value(A.x_off, A.x_dofs, A.x_w, A.u, 4ll * c + 0);
                const double u0r = local_value(A.x_off, A.x_dofs, A.x_w, A.u, 4ll * c + 2);
                const q1d::Quad g = q1d::load(A.x_geo, c);
                double acc = 0.0;
                for (int q = 0; q < 3; ++q)
                {
                    const double xi = q1d::gauss_x(q);
                    const double uh = u0l * (1.0 - xi) + u0r * xi;
                    const double d = u0_value_1d(A.u0_kind, g.x0 + g.h * xi) - uh;
                    acc += d * d * g.h * q1d::gauss_w(q);
                }
                A.trace_x[c] = acc;
            }
        }

        __global__ void child_count_kernel(int n_y, const int* __restrict__ y_to_x, int* __restrict__ cnt)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_y; c += gridDim.x * blockDim.x)
                atomicAdd(cnt + y_to_x[c], 1);
        }

        __global__ void child_fill_kernel(int n_y, const int* __restrict__ y_to_x, const int* __restrict__ ptr,
                                          int* __restrict__ cursor, int* __restrict__ child)
        {
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_y; c += gridDim.x * blockDim.x)
            {
                const int x = y_to_x[c];
                child[ptr[x] + atomicAdd(cursor + x, 1)] = c;
            }
        }

        // per X cell: sum of its Y children's lambda energies in ascending Y order (children
        // sorted in place: the fill order of the atomics is not deterministic), plus the trace
        __global__ void aggregate_kernel(int n_x, const int* __restrict__ ptr, int* __restrict__ child,
                                         const double* __restrict__ lam_y, const double* __restrict__ trace_x,
                                         double* __restrict__ lam_x, double* __restrict__ eta_x)
        {
            for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n_x; x += gridDim.x * blockDim.x)
            {
                const int b = ptr[x], e = ptr[x + 1];
                for (int i = b + 1; i < e; ++i)
                {
                    const int v = child[i];
                    int j = i - 1;
                    while (j >= b && child[j] > v)
                    {
                        child[j + 1] = child[j];
                        --j;
                    }
                    child[j + 1] = v;
                }
                double s = 0.0;
                for (int i = b; i < e; ++i)
                    s += lam_y[child[i]];
                lam_x[x] = s;
                eta_x[x] = s + trace_x[x];
            }
        }
    }

    void y_cell_energy(cudaStream_t s, const SystemInputs& in, const double* v, double* out)
    {
        XIndArgs a{};
        a.p = in.p;
        a.n_y = in.n_y_cells;
        a.y_geo = in.y_geo.get();
        a.m_y = in.m_y.size() ? in.m_y.get() : nullptr;
        a.y_off = in.y_off.get();
        a.y_dofs = in.y_dofs.get();
        a.y_w = in.y_w.get();
        a.lambda = v;
        a.lam_y = out;
        if (in.n_y_cells > 0)
        {
            APF_KERNEL("y_cell_energy", s);
            if (in.dim == 1)
                lambda_energy_1d_kernel<<<grid_for(in.n_y_cells, 128), 128, 0, s>>>(a);
            else
                lambda_energy_kernel<<<grid_for(in.n_y_cells, 128), 128, 0, s>>>(a);
        }
        APF_CUDA(cudaGetLastError());
    }

    namespace
    {
        // dst[c][k] = sum_i src[src_index[c]][i] phi_i(node_k of dst cell c): the local
        // function of the source prism evaluated at the nodes of the destination prism (the
        // destination lies inside the source, so this represents it exactly)
        __global__ void nodal_transfer_kernel(int p, int n, const double* __restrict__ dst_geo,
                                              const int* __restrict__ src_index, const double* __restrict__ src_geo,
                                              const double* __restrict__ src, double* __restrict__ dst)
        {
            const RefTables& t = c_tab[p - 1];
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
            {
                const int sc = src_index ? src_index[c] : c;
                const double* in = src + static_cast<long long>(sc) * t.ndof;
                double* out = dst + static_cast<long long>(c) * t.ndof;
                if (same_geometry(dst_geo, c, src_geo, sc))
                {
                    for (int k = 0; k < t.ndof; ++k)
                        out[k] = in[k];
                    continue;
                }
                const CellGeo gd = load_geo(dst_geo, c);
                const CellGeo gs = load_geo(src_geo, sc);
                for (int k = 0; k < t.ndof; ++k)
                {
                    double v = 0.0;
                    for (int i = 0; i < t.ndof; ++i)
                        v += transfer(t, gd, gs, i, k) * in[i];
                    out[k] = v;
                }
            }
        }

        // out[c] = v_c^T A_c v_c with the local A_y block of prism c and nodal values v_c
        __global__ void nodal_energy_kernel(int p, int n, const double* __restrict__ geo, const double* __restrict__ m,
                                            const double* __restrict__ v, double* __restrict__ out)
        {
            const RefTables& t = c_tab[p - 1];
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
            {
                const double* lam = v + static_cast<long long>(c) * t.ndof;
                const CellGeo g = load_geo(geo, c);
                double q00, q01, q11;
                q_form(g, m, c, q00, q01, q11);
                double e = 0.0;
                for (int i = 0; i < t.ndof; ++i)
                {
                    const int s = i / t.nt, a = i % t.nt;
                    double row = 0.0;
                    for (int j = 0; j < t.ndof; ++j)
                    {
                        const int r = j / t.nt, b = j % t.nt;
                        row += t.Mt[a][b] * ks(t, q00, q01, q11, s, r) * lam[j];
                    }
                    e += lam[i] * row;
                }
                out[c] = g.det * g.ht * e;
            }
        }
    }

    namespace
    {
        // owner[dof]: the smallest local row (cell * nd + k) whose restriction row is the single
        // entry (dof, 1) -- an unconstrained occurrence of the true DOF
        __global__ void true_dof_owner_kernel(long long rows, const int* __restrict__ off, const int* __restrict__ dofs,
                                              const double* __restrict__ w, int* __restrict__ owner)
        {
            for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows;
                 r += (long long)gridDim.x * blockDim.x)
            {
                const int a = off[r];
                if (off[r + 1] - a == 1 && w[a] == 1.0)
                    atomicMin(owner + dofs[a], static_cast<int>(r));
            }
        }

        constexpr int kNoOwner = 0x7f7f7f7f; // the byte pattern 0x7f in every byte of an int

        __global__ void unowned_kernel(int n, const int* __restrict__ owner, int* __restrict__ count)
        {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
                if (owner[i] == kNoOwner)
                    atomicAdd(count, 1);
        }

        // out[dof] for every true DOF of the degree-q space (restriction off/dofs, cells with
        // geometry dst_geo): the degree-p function v (true DOFs through the source restriction
        // soff/sdofs/sw of the source cells src_index[c], geometry src_geo) at the DOF's node,
        // evaluated in the owner row's cell only (one deterministic writer per DOF)
        __global__ void interpolate_kernel(int n, int q, int p, const double* __restrict__ dst_geo,
                                           const int* __restrict__ src_index, const double* __restrict__ src_geo,
                                           const int* __restrict__ soff, const int* __restrict__ sdofs,
                                           const double* __restrict__ sw, const double* __restrict__ v,
                                           const int* __restrict__ off, const int* __restrict__ dofs,
                                           const int* __restrict__ owner, double* __restrict__ out)
        {
            const RefTables& tq = c_tab[q - 1];
            const RefTables& tp = c_tab[p - 1];
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
            {
                const int sc = src_index ? src_index[c] : c;
                double loc[kMaxNs * kMaxNt];
                for (int i = 0; i < tp.ndof; ++i)
                {
                    const long long row = static_cast<long long>(sc) * tp.ndof + i;
                    double a = 0.0;
                    for (int e = soff[row]; e < soff[row + 1]; ++e)
                        a += sw[e] * v[sdofs[e]];
                    loc[i] = a;
                }
                const CellGeo gd = load_geo(dst_geo, c);
                const CellGeo gs = load_geo(src_geo, sc);
                for (int k = 0; k < tq.ndof; ++k)
                {
                    const long long row = static_cast<long long>(c) * tq.ndof + k;
                    const int a = off[row];
                    if (off[row + 1] - a != 1 || owner[dofs[a]] != static_cast<int>(row))
                        continue;
                    double val = 0.0;
                    for (int i = 0; i < tp.ndof; ++i)
                        val += loc[i] * transfer_between(tq, tp, gd, gs, i, k);
                    out[dofs[a]] = val;
                }
            }
        }
    }

    void interpolate_to_space(cudaStream_t s, int q, int p, int n, const double* dst_geo, const int* src_index,
                              const double* src_geo, const int* soff, const int* sdofs, const double* sw,
                              const double* v, const int* off, const int* dofs, const double* w, int n_true,
                              double* out)
    {
        require(q >= 1 && q <= 2 && p >= 1 && p <= q, APF_ERR_INVALID, "interpolate_to_space: degrees");
        if (n_true <= 0)
            return;
        const int ndq = (q + 1) * (q + 2) / 2 * (q + 1);
        const long long rows = static_cast<long long>(n) * ndq;
        require(rows < kNoOwner, APF_ERR_CAPACITY, "interpolate_to_space: too many local rows");
        DeviceBuffer<int> owner(n_true, s), count(1, s);
        APF_CUDA(cudaMemsetAsync(owner.get(), 0x7f, sizeof(int) * n_true, s)); // kNoOwner, above every row
        count.zero();
        {
            APF_KERNEL("true_dof_owner", s);
            true_dof_owner_kernel<<<grid_for(rows, 256), 256, 0, s>>>(rows, off, dofs, w, owner.get());
        }
        {
            APF_KERNEL("true_dof_unowned", s);
            unowned_kernel<<<grid_for(n_true, 256), 256, 0, s>>>(n_true, owner.get(), count.get());
        }
        int unowned = 0;
        APF_CUDA(cudaMemcpyAsync(&unowned, count.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        sync(s);
        require(unowned == 0, APF_ERR_INVALID,
                "interpolate_to_space: a true DOF has no unconstrained occurrence in the restriction");
        if (n > 0)
        {
            APF_KERNEL("interpolate_nodal", s);
            interpolate_kernel<<<grid_for(n, 128), 128, 0, s>>>(n, q, p, dst_geo, src_index, src_geo, soff, sdofs, sw, v,
                                                                off, dofs, owner.get(), out);
        }
        APF_CUDA(cudaGetLastError());
    }

    void nodal_transfer(cudaStream_t s, int p, int n, const double* dst_geo, const int* src_index, const double* src_geo,
                        const double* src, double* dst)
    {
        if (n <= 0)
            return;
        APF_KERNEL("nodal_transfer", s);
        nodal_transfer_kernel<<<grid_for(n, 128), 128, 0, s>>>(p, n, dst_geo, src_index, src_geo, src, dst);
        APF_CUDA(cudaGetLastError());
    }

    void nodal_energy(cudaStream_t s, int p, int n, const double* geo, const double* m, const double* v, double* out)
    {
        if (n <= 0)
            return;
        APF_KERNEL("nodal_energy", s);
        nodal_energy_kernel<<<grid_for(n, 128), 128, 0, s>>>(p, n, geo, m, v, out);
        APF_CUDA(cudaGetLastError());
    }

    void x_indicators(cudaStream_t s, const SystemInputs& in, const double* lambda, const double* u, double* lam_y,
                      double* lam_x, double* trace_x, double* eta_x)
    {
        XIndArgs a{};
        a.p = in.p;
        a.n_y = in.n_y_cells;
        a.n_x = in.n_x_cells;
        a.n_bottom = in.n_bottom;
        a.y_geo = in.y_geo.get();
        a.x_geo = in.x_geo.get();
        a.m_y = in.m_y.size() ? in.m_y.get() : nullptr;
        a.y_off = in.y_off.get();
        a.y_dofs = in.y_dofs.get();
        a.y_w = in.y_w.get();
        a.x_off = in.x_off.get();
        a.x_dofs = in.x_dofs.get();
        a.x_w = in.x_w.get();
        a.bottom = in.bottom_list.get();
        a.u0_kind = in.u0_kind;
        a.lambda = lambda;
        a.u = u;
        a.lam_y = lam_y;
        a.trace_x = trace_x;
        if (in.n_x_cells > 0)
            APF_CUDA(cudaMemsetAsync(trace_x, 0, sizeof(double) * in.n_x_cells, s));
        if (in.n_y_cells > 0)
        {
            APF_KERNEL("xind_lambda_energy", s);
            if (in.dim == 1)
                lambda_energy_1d_kernel<<<grid_for(in.n_y_cells, 128), 128, 0, s>>>(a);
            else
                lambda_energy_kernel<<<grid_for(in.n_y_cells, 128), 128, 0, s>>>(a);
        }
        if (in.n_bottom > 0)
        {
            APF_KERNEL("xind_initial_trace", s);
            if (in.dim == 1)
                initial_trace_1d_kernel<<<grid_for(in.n_bottom, 128), 128, 0, s>>>(a);
            else
                initial_trace_kernel<<<grid_for(in.n_bottom, 128), 128, 0, s>>>(a);
        }
        DeviceBuffer<int> cnt(static_cast<std::size_t>(in.n_x_cells) + 1, s), ptr(static_cast<std::size_t>(in.n_x_cells) + 1, s),
            cursor(static_cast<std::size_t>(in.n_x_cells) + 1, s), child(static_cast<std::size_t>(std::max(in.n_y_cells, 1)), s);
        cnt.zero();
        cursor.zero();
        if (in.n_y_cells > 0)
        {
            APF_KERNEL("xind_child_count", s);
            child_count_kernel<<<grid_for(in.n_y_cells, 256), 256, 0, s>>>(in.n_y_cells, in.y_to_x.get(), cnt.get());
        }
        exclusive_scan(cnt.get(), ptr.get(), in.n_x_cells, s);
        if (in.n_y_cells > 0)
        {
            APF_KERNEL("xind_child_fill", s);
            child_fill_kernel<<<grid_for(in.n_y_cells, 256), 256, 0, s>>>(in.n_y_cells, in.y_to_x.get(), ptr.get(),
                                                                         cursor.get(), child.get());
        }
        if (in.n_x_cells > 0)
        {
            APF_KERNEL("xind_aggregate", s);
            aggregate_kernel<<<grid_for(in.n_x_cells, 256), 256, 0, s>>>(in.n_x_cells, ptr.get(), child.get(), lam_y,
                                                                        trace_x, lam_x, eta_x);
        }
        APF_CUDA(cudaGetLastError());
    }
}
