// extern "C" entry points of libapf_b200 (declared in include/apf_b200.h) and the
// host-side drivers that sequence the device kernels.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <numeric>
#include <vector>
#include <array>
#include <memory>
#include <new>
#include <string>

#include "apf_internal.hpp"
#include "apf_estimator.cuh"
#include "apf_gdelta.cuh"
#include "apf_learned.cuh"
#include "apf_system.hpp"

struct apf_ctx
{
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string last_error;
    apf::Profiler profiler;
    std::string report;
    std::unique_ptr<apf::LearnedModel> learned; // model of APF_PRECOND_LEARNED set-ups
    unsigned long long learned_version = 0;
    int patch_precision = APF_PATCH_FP64; // apf_ctx_set_patch_precision
    apf::PatchTuner tuner;                // apf_ctx_set_autotune
    std::string tune_report;
};

struct apf_learned_model
{
    apf::LearnedModel model;
};

struct apf_system
{
    apf_ctx* ctx = nullptr;
    apf::System sys;
};

namespace
{
    template<class F>
    int guarded(apf_ctx* ctx, F&& f)
    {
        struct ProfilerScope
        {
            explicit ProfilerScope(apf_ctx* c) { apf::t_profiler = c ? &c->profiler : nullptr; }
            ~ProfilerScope() { apf::t_profiler = nullptr; }
        } scope(ctx);
        try
        {
            if (ctx)
            {
                int cur = -1;
                cudaGetDevice(&cur);
                if (cur != ctx->device)
                    APF_CUDA(cudaSetDevice(ctx->device));
            }
            f();
            if (ctx)
                ctx->last_error.clear();
            return APF_OK;
        }
        catch (const apf::Error& e)
        {
            if (ctx)
                ctx->last_error = e.what();
            return e.code;
        }
        catch (const std::exception& e)
        {
            if (ctx)
                ctx->last_error = e.what();
            return APF_ERR_INTERNAL;
        }
    }

    // Keep the stream-ordered pool at 1.5x the largest footprint seen so far, reserved as one
    // block: carving each call's buffers from one block avoids the pool mapping fresh memory
    // for fragmented requests (seen as stalls of up to seconds between identical calls).
    void ensure_pool(apf_ctx* ctx)
    {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) != cudaSuccess)
            return;
        std::uint64_t reserved = 0, used_high = 0;
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &used_high);
        const std::uint64_t gib = 1ull << 30;
        std::uint64_t target = ((used_high + used_high / 2 + gib - 1) / gib) * gib;
        std::size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
            target = std::min<std::uint64_t>(target, (total_b / 10) * 7);
        if (used_high == 0 || reserved >= target)
            return;
        void* p = nullptr;
        if (cudaMallocAsync(&p, target, ctx->stream) == cudaSuccess)
        {
            cudaFreeAsync(p, ctx->stream);
            cudaStreamSynchronize(ctx->stream);
            // the reservation is not footprint: measure the next calls from here
            std::uint64_t zero = 0;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero);
        }
        cudaGetLastError(); // a failed reservation only costs the optimisation
    }

    template<class T>
    void stage(apf::DeviceBuffer<T>& dst, const T* src, std::size_t n, bool on_device, cudaStream_t s)
    {
        dst.allocate(n, s);
        if (n == 0)
            return;
        apf::require(src != nullptr, APF_ERR_INVALID, "null input array");
        APF_CUDA(cudaMemcpyAsync(dst.get(), src, n * sizeof(T),
                                 on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    }
}

struct apf_two_pass_cache
{
    apf_ctx* ctx = nullptr;
    bool valid = false;
    std::array<long long, 12> key{};
    apf::DeviceBuffer<int> row_ptr, col_idx;
    long long pattern_builds = 0, pattern_reuses = 0;
};

namespace
{
    using TwoPassKey = std::array<long long, 12>;

    __device__ __forceinline__ unsigned long long mix64(unsigned long long z)
    {
        // splitmix64 finaliser
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }

    // order-independent fingerprint of an int array: sum over i of mix(tag, i, a[i])
    __global__ void fingerprint_add(const int* __restrict__ a, long long n, unsigned tag,
                                    unsigned long long* __restrict__ acc)
    {
        unsigned long long h = 0;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
            h += mix64((static_cast<unsigned long long>(tag) << 56) ^ (static_cast<unsigned long long>(i) << 24) ^
                       static_cast<unsigned long long>(static_cast<unsigned>(a[i])) * 0x9e3779b97f4a7c15ull);
        for (int o = 16; o > 0; o >>= 1)
            h += __shfl_xor_sync(0xffffffffu, h, o);
        if ((threadIdx.x & 31) == 0)
            atomicAdd(acc, h);
    }

    TwoPassKey two_pass_key(cudaStream_t s, const apf::SystemInputs& in)
    {
        apf::DeviceBuffer<unsigned long long> acc(1, s);
        APF_CUDA(cudaMemsetAsync(acc.get(), 0, sizeof(unsigned long long), s));
        const apf::DeviceBuffer<int>* arrays[6] = {&in.y_off, &in.y_dofs, &in.x_off, &in.x_dofs, &in.y_to_x,
                                                   &in.bottom_list};
        for (unsigned t = 0; t < 6; ++t)
        {
            const long long n = static_cast<long long>(arrays[t]->size());
            if (n == 0)
                continue;
            APF_KERNEL("pattern_fingerprint", s);
            fingerprint_add<<<static_cast<int>(std::min<long long>((n + 255) / 256, 148 * 8)), 256, 0, s>>>(
                arrays[t]->get(), n, t + 1, acc.get());
            APF_CUDA(cudaGetLastError());
        }
        unsigned long long h = 0;
        APF_CUDA(cudaMemcpyAsync(&h, acc.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
        apf::sync(s);
        return TwoPassKey{in.p, in.dim, in.ndof, in.n_y_cells, in.n_x_cells, in.n_lambda, in.n_u,
                          static_cast<long long>(in.y_dofs.size()), static_cast<long long>(in.x_dofs.size()),
                          in.n_bottom, static_cast<long long>(h >> 1), static_cast<long long>(h & 1)};
    }

    // problem descriptor -> device inputs of a system (validation as the reference's
    // assembly preconditions)
    void stage_problem(apf_ctx* ctx, const apf_problem_desc* d, int inputs_on_device, apf::System& S)
    {
        const int dim = d->dim_space == 0 ? 2 : d->dim_space;
        apf::require(dim == 1 || dim == 2, APF_ERR_INVALID, "dim_space must be 1 or 2");
        apf::require(d->p == 1 || (d->p == 2 && dim == 2), APF_ERR_INVALID,
                     "p must be 1 or 2 (2+1D) or 1 (1+1D)");
        apf::require(d->n_y_cells >= 0 && d->n_x_cells >= 0 && d->n_lambda >= 0 && d->n_u >= 0, APF_ERR_INVALID,
                     "negative sizes");
        apf::require(d->u0_kind >= 0 && d->u0_kind <= 2, APF_ERR_INVALID, "unknown u0_kind");
        S.stream = ctx->stream;
        auto& in = S.in;
        in.p = d->p;
        in.dim = dim;
        in.ndof = dim == 1 ? (d->p + 1) * (d->p + 1) : (d->p + 1) * (d->p + 2) / 2 * (d->p + 1);
        in.n_y_cells = d->n_y_cells;
        in.n_x_cells = d->n_x_cells;
        in.n_lambda = d->n_lambda;
        in.n_u = d->n_u;
        in.u0_kind = d->u0_kind;
        in.zero_tol = d->zero_tol;
        in.g_scale = d->g_scale;
        const bool dev = inputs_on_device != 0;
        cudaStream_t s = ctx->stream;
        const std::size_t ny = static_cast<std::size_t>(d->n_y_cells), nx = static_cast<std::size_t>(d->n_x_cells);
        const std::size_t gw = dim == 1 ? 4 : 8, mw = dim == 1 ? 1 : 3;
        stage(in.y_geo, d->y_geometry, ny * gw, dev, s);
        stage(in.x_geo, d->x_geometry, nx * gw, dev, s);
        stage(in.y_to_x, d->y_to_x, ny, dev, s);
        stage(in.y_off, d->y_restr_offsets, ny * in.ndof + 1, dev, s);
        stage(in.y_dofs, d->y_restr_dofs, static_cast<std::size_t>(d->y_restr_nnz), dev, s);
        stage(in.y_w, d->y_restr_weights, static_cast<std::size_t>(d->y_restr_nnz), dev, s);
        stage(in.x_off, d->x_restr_offsets, nx * in.ndof + 1, dev, s);
        stage(in.x_dofs, d->x_restr_dofs, static_cast<std::size_t>(d->x_restr_nnz), dev, s);
        stage(in.x_w, d->x_restr_weights, static_cast<std::size_t>(d->x_restr_nnz), dev, s);
        if (d->m_cells)
            stage(in.m_y, d->m_cells, ny * mw, dev, s);
        if (d->ell_cells)
            stage(in.ell, d->ell_cells, ny, dev, s);
    }
}

namespace apf
{
    void assemble_main(System& S)
    {
        cudaStream_t s = S.stream;
        SystemInputs& in = S.in;
        prepare_inputs(s, in);
        const int nd = in.ndof;
        S.inc_y = build_incidence(s, in.n_lambda, in.n_y_cells, nullptr, nullptr, in.y_off.get(), in.y_dofs.get(), nd);
        S.inc_xy = build_incidence(s, in.n_u, in.n_y_cells, nullptr, in.y_to_x.get(), in.x_off.get(), in.x_dofs.get(), nd);
        S.inc_xb = build_incidence(s, in.n_u, in.n_bottom, in.bottom_list.get(), nullptr, in.x_off.get(), in.x_dofs.get(), nd);
        {
            const int kinds[1] = {K_AY};
            const Incidence* incs[1] = {&S.inc_y};
            const int offs[1] = {0};
            gather_csr(s, in, in.zero_tol, in.n_lambda, in.n_lambda, 1, kinds, incs, offs, in.kmax, S.blocks[APF_BLOCK_A_Y]);
        }
        {
            const int kinds[1] = {K_BT};
            const Incidence* incs[1] = {&S.inc_y};
            const int offs[1] = {0};
            gather_csr(s, in, in.zero_tol, in.n_lambda, in.n_u, 1, kinds, incs, offs, in.kmax, S.blocks[APF_BLOCK_BT]);
        }
        {
            const int kinds[1] = {K_B};
            const Incidence* incs[1] = {&S.inc_xy};
            const int offs[1] = {0};
            gather_csr(s, in, in.zero_tol, in.n_u, in.n_lambda, 1, kinds, incs, offs, in.kmax, S.blocks[APF_BLOCK_B]);
        }
        {
            const int kinds[1] = {K_C};
            const Incidence* incs[1] = {&S.inc_xb};
            const int offs[1] = {0};
            gather_csr(s, in, in.zero_tol, in.n_u, in.n_u, 1, kinds, incs, offs, in.kmax, S.blocks[APF_BLOCK_C]);
        }
        S.have[APF_BLOCK_A_Y] = S.have[APF_BLOCK_BT] = S.have[APF_BLOCK_B] = S.have[APF_BLOCK_C] = true;
        gather_vector_host(s, in, in.zero_tol, 0, S.inc_y, in.n_lambda, in.ell.size() ? in.ell.get() : nullptr,
                           in.u0_kind, in.g_scale, S.f);
        gather_vector_host(s, in, in.zero_tol, 1, S.inc_xb, in.n_u, nullptr, in.u0_kind, in.g_scale, S.g);
        build_k(s, in.n_lambda, in.n_u, S.blocks[APF_BLOCK_A_Y], S.blocks[APF_BLOCK_BT], S.blocks[APF_BLOCK_B],
                S.blocks[APF_BLOCK_C], S.blocks[APF_BLOCK_K]);
        S.have[APF_BLOCK_K] = true;
        sync(s);
    }

    void assemble_graph_norm(System& S, double diag_tol)
    {
        require(S.have[APF_BLOCK_A_Y] && S.have[APF_BLOCK_C], APF_ERR_INVALID,
                "assemble_graph_norm: assemble the main system first");
        cudaStream_t s = S.stream;
        SystemInputs& in = S.in;
        const int nd = in.ndof;
        // The graph-norm blocks are assembled with the same local filter as the main
        // system (parabolic_graph_norm.hpp:22-65 passes zero_tol through).
        S.inc_x = build_incidence(s, in.n_u, in.n_x_cells, nullptr, nullptr, in.x_off.get(), in.x_dofs.get(), nd);
        {
            const int kinds[1] = {K_AX};
            const Incidence* incs[1] = {&S.inc_x};
            const int offs[1] = {0};
            gather_csr(s, in, in.zero_tol, in.n_u, in.n_u, 1, kinds, incs, offs, in.kmax, S.blocks[APF_BLOCK_AX]);
        }
        {
            const int kinds[1] = {K_BDT};
            const Incidence* incs[1] = {&S.inc_xy};
            const int offs[1] = {0};
            gather_csr(s, in, in.zero_tol, in.n_u, in.n_lambda, 1, kinds, incs, offs, in.kmax, S.blocks[APF_BLOCK_BDT]);
        }
        DeviceCsr bdtT;
        {
            const int kinds[1] = {K_BDTT};
            const Incidence* incs[1] = {&S.inc_y};
            const int offs[1] = {0};
            gather_csr(s, in, in.zero_tol, in.n_lambda, in.n_u, 1, kinds, incs, offs, in.kmax, bdtT);
        }
        S.have[APF_BLOCK_AX] = S.have[APF_BLOCK_BDT] = true;
        build_hhat(s, S.blocks[APF_BLOCK_A_Y], S.blocks[APF_BLOCK_C], S.blocks[APF_BLOCK_AX], S.blocks[APF_BLOCK_BDT],
                   bdtT, diag_tol, S.blocks[APF_BLOCK_HHAT], S.inv_diag_ay);
        S.have[APF_BLOCK_HHAT] = true;
        sync(s);
    }
}

namespace
{
    // n values of one array into host memory (a device array through the context's stream)
    template<class T>
    std::vector<T> fetch_host(apf_ctx* ctx, const T* p, int n, bool on_device)
    {
        std::vector<T> h(static_cast<std::size_t>(n));
        if (n == 0)
            return h;
        apf::require(p != nullptr, APF_ERR_INVALID, "artifact writer: null array");
        if (on_device)
        {
            APF_CUDA(cudaMemcpyAsync(h.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx->stream));
            APF_CUDA(cudaStreamSynchronize(ctx->stream));
        }
        else
            std::memcpy(h.data(), p, sizeof(T) * n);
        return h;
    }

    // entry order of the reference's writers: decreasing total, ties by increasing cell id
    // (CellwiseSquaredError::sorted_descending), or the given order
    std::vector<int> artifact_order(const std::vector<int32_t>& ids, const std::vector<double>& key, bool sort)
    {
        std::vector<int> order(ids.size());
        std::iota(order.begin(), order.end(), 0);
        if (sort)
            std::sort(order.begin(), order.end(), [&](int a, int b) {
                if (key[a] != key[b])
                    return key[a] > key[b];
                return ids[a] < ids[b];
            });
        return order;
    }

    void write_artifact(const char* path, const std::vector<int32_t>& header, const std::vector<int32_t>& ids,
                        const std::vector<const std::vector<double>*>& columns, const std::vector<int>& order)
    {
        std::ofstream f(path, std::ios::binary | std::ios::trunc);
        apf::require(f.is_open(), APF_ERR_INVALID, std::string("artifact writer: cannot open ") + path);
        f.write(reinterpret_cast<const char*>(header.data()), static_cast<std::streamsize>(header.size() * 4));
        std::vector<int32_t> oid(order.size());
        for (std::size_t k = 0; k < order.size(); ++k)
            oid[k] = ids[static_cast<std::size_t>(order[k])];
        // empty blocks are not written (write_binary_block skips empty vectors)
        if (!oid.empty())
            f.write(reinterpret_cast<const char*>(oid.data()), static_cast<std::streamsize>(oid.size() * 4));
        std::vector<double> col(order.size());
        for (const auto* c : columns)
        {
            for (std::size_t k = 0; k < order.size(); ++k)
                col[k] = (*c)[static_cast<std::size_t>(order[k])];
            if (!col.empty())
                f.write(reinterpret_cast<const char*>(col.data()), static_cast<std::streamsize>(col.size() * 8));
        }
        apf::require(static_cast<bool>(f), APF_ERR_INTERNAL, std::string("artifact writer: write failed: ") + path);
    }

    template<class F>
    int host_guarded(apf_ctx* ctx, F&& f)
    {
        if (ctx)
            return guarded(ctx, std::forward<F>(f));
        try
        {
            f();
            return APF_OK;
        }
        catch (const apf::Error& e)
        {
            return e.code;
        }
        catch (const std::exception&)
        {
            return APF_ERR_INTERNAL;
        }
    }
}

extern "C" {

int apf_ctx_create(int device, void* stream, apf_ctx** out)
{
    if (!out)
        return APF_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        return APF_ERR_NO_DEVICE;
    if (device < 0 || device >= n)
        return APF_ERR_INVALID;
    auto ctx = std::make_unique<apf_ctx>();
    ctx->device = device;
    const int rc = guarded(ctx.get(), [&] {
        APF_CUDA(cudaSetDevice(device));
        if (stream)
            ctx->stream = static_cast<cudaStream_t>(stream);
        else
        {
            APF_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
            ctx->own_stream = true;
        }
        apf::upload_tables_once(device);
        // The library's buffers come from this process's default stream-ordered pool.  Its
        // default release threshold (0) hands freed memory back to the driver at every
        // synchronisation, so each inner iteration would map its GBs of assembly, AMG and
        // estimator buffers afresh; keeping freed memory in the pool makes the next
        // iteration's allocations cheap.  (Process-local; released at exit.)
        cudaMemPool_t pool;
        APF_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        std::uint64_t keep = UINT64_MAX;
        APF_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    });
    if (rc != APF_OK)
        return rc;
    *out = ctx.release();
    return APF_OK;
}

void apf_ctx_destroy(apf_ctx* ctx)
{
    if (!ctx)
        return;
    cudaSetDevice(ctx->device);
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream && ctx->stream)
        cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* apf_ctx_last_error(const apf_ctx* ctx)
{
    return ctx ? ctx->last_error.c_str() : "null context";
}

int apf_ctx_synchronize(apf_ctx* ctx)
{
    return guarded(ctx, [&] { APF_CUDA(cudaStreamSynchronize(ctx->stream)); });
}

int64_t apf_ctx_kernel_launches(const apf_ctx*)
{
    return apf::g_kernel_launches.load();
}

int apf_ctx_set_timing(apf_ctx* ctx, int enable)
{
    if (!ctx)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        ctx->profiler.flush();
        ctx->profiler.enabled = enable != 0;
        ctx->profiler.kernels = enable != 2;
        ctx->profiler.totals.clear();
    });
}

int apf_ctx_reserve_pool(apf_ctx* ctx, int64_t bytes)
{
    if (!ctx || bytes < 0)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        if (bytes == 0)
            return;
        void* p = nullptr;
        APF_CUDA(cudaMallocAsync(&p, static_cast<std::size_t>(bytes), ctx->stream));
        APF_CUDA(cudaFreeAsync(p, ctx->stream));
        APF_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int apf_ctx_pool_stats(apf_ctx* ctx, int64_t* reserved, int64_t* reserved_high, int64_t* used, int64_t* used_high)
{
    if (!ctx)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        cudaMemPool_t pool;
        APF_CUDA(cudaDeviceGetDefaultMemPool(&pool, ctx->device));
        auto get = [&](cudaMemPoolAttr attr, int64_t* out) {
            if (!out)
                return;
            std::uint64_t v = 0;
            APF_CUDA(cudaMemPoolGetAttribute(pool, attr, &v));
            *out = static_cast<int64_t>(v);
        };
        get(cudaMemPoolAttrReservedMemCurrent, reserved);
        get(cudaMemPoolAttrReservedMemHigh, reserved_high);
        get(cudaMemPoolAttrUsedMemCurrent, used);
        get(cudaMemPoolAttrUsedMemHigh, used_high);
    });
}

const char* apf_ctx_timing_report(apf_ctx* ctx)
{
    if (!ctx)
        return "{}";
    ctx->profiler.flush();
    std::string r = "{";
    bool first = true;
    for (const auto& [name, v] : ctx->profiler.totals)
    {
        char buf[256];
        std::snprintf(buf, sizeof(buf), "%s\"%s\": [%lld, %.6f]", first ? "" : ", ", name.c_str(), v.first, v.second);
        r += buf;
        first = false;
    }
    r += "}";
    ctx->report = r;
    return ctx->report.c_str();
}

int apf_assemble_main_system(apf_ctx* ctx, const apf_problem_desc* d, int inputs_on_device, apf_system** out)
{
    if (!ctx || !d || !out)
        return APF_ERR_INVALID;
    *out = nullptr;
    auto h = std::make_unique<apf_system>();
    h->ctx = ctx;
    const int rc = guarded(ctx, [&] {
        APF_HOST_RANGE("call_assemble_main_system");
        ensure_pool(ctx);
        stage_problem(ctx, d, inputs_on_device, h->sys);
        apf::assemble_main(h->sys);
    });
    if (rc != APF_OK)
        return rc;
    *out = h.release();
    return APF_OK;
}

int apf_two_pass_cache_create(apf_ctx* ctx, apf_two_pass_cache** out)
{
    if (!ctx || !out)
        return APF_ERR_INVALID;
    *out = new apf_two_pass_cache;
    (*out)->ctx = ctx;
    return APF_OK;
}

void apf_two_pass_cache_destroy(apf_two_pass_cache* cache)
{
    if (!cache)
        return;
    cudaSetDevice(cache->ctx->device);
    cudaStreamSynchronize(cache->ctx->stream);
    delete cache;
}

int apf_two_pass_cache_stats(const apf_two_pass_cache* cache, int64_t* pattern_builds, int64_t* pattern_reuses,
                             int64_t* pattern_entries)
{
    if (!cache)
        return APF_ERR_INVALID;
    if (pattern_builds)
        *pattern_builds = cache->pattern_builds;
    if (pattern_reuses)
        *pattern_reuses = cache->pattern_reuses;
    if (pattern_entries)
        *pattern_entries = cache->valid ? static_cast<int64_t>(cache->col_idx.size()) : 0;
    return APF_OK;
}

int apf_assemble_full_saddle_two_pass(apf_ctx* ctx, const apf_problem_desc* d, int inputs_on_device,
                                      apf_two_pass_cache* cache, apf_system** out)
{
    if (!ctx || !d || !out || (cache && cache->ctx != ctx))
        return APF_ERR_INVALID;
    *out = nullptr;
    auto h = std::make_unique<apf_system>();
    h->ctx = ctx;
    const int rc = guarded(ctx, [&] {
        APF_HOST_RANGE("call_assemble_full_saddle_two_pass");
        ensure_pool(ctx);
        auto& S = h->sys;
        apf::require(d->dim_space == 0 || d->dim_space == 2, APF_ERR_INVALID,
                     "the two-pass full saddle assembly is for 2+1D problems");
        stage_problem(ctx, d, inputs_on_device, S);
        cudaStream_t s = S.stream;
        auto& in = S.in;
        apf::prepare_inputs(s, in);
        const int nd = in.ndof;
        S.inc_y = apf::build_incidence(s, in.n_lambda, in.n_y_cells, nullptr, nullptr, in.y_off.get(), in.y_dofs.get(), nd);
        S.inc_xy = apf::build_incidence(s, in.n_u, in.n_y_cells, nullptr, in.y_to_x.get(), in.x_off.get(),
                                        in.x_dofs.get(), nd);
        S.inc_xb = apf::build_incidence(s, in.n_u, in.n_bottom, in.bottom_list.get(), nullptr, in.x_off.get(),
                                        in.x_dofs.get(), nd);
        apf::DeviceBuffer<int> own_rp, own_ci;
        const int* rp = nullptr;
        const int* ci = nullptr;
        long long nnz_pattern = 0;
        // the pattern is kept while the mesh and its DOF maps are unchanged: sizes plus a
        // fingerprint of the restriction rows, the Y -> X map and the bottom-cell list
        // (the reference keys its cache on the spaces' version counters)
        TwoPassKey key{};
        if (cache)
            key = two_pass_key(s, in);
        if (cache && cache->valid && cache->key == key)
        {
            ++cache->pattern_reuses;
        }
        else
        {
            if (cache)
                cache->valid = false; // a pass that throws leaves no stale pattern behind
            apf::DeviceBuffer<int>& prp = cache ? cache->row_ptr : own_rp;
            apf::DeviceBuffer<int>& pci = cache ? cache->col_idx : own_ci;
            apf::full_saddle_pattern(s, in, S.inc_y, S.inc_xy, S.inc_xb, prp, pci);
            if (cache)
            {
                cache->key = key;
                cache->valid = true;
                ++cache->pattern_builds;
            }
        }
        rp = cache ? cache->row_ptr.get() : own_rp.get();
        ci = cache ? cache->col_idx.get() : own_ci.get();
        nnz_pattern = static_cast<long long>(cache ? cache->col_idx.size() : own_ci.size());
        apf::full_saddle_numeric(s, in, S.inc_y, S.inc_xy, S.inc_xb, rp, ci, nnz_pattern, S.blocks[APF_BLOCK_K]);
        S.have[APF_BLOCK_K] = true;
        apf::gather_vector_host(s, in, in.zero_tol, 0, S.inc_y, in.n_lambda, in.ell.size() ? in.ell.get() : nullptr,
                                in.u0_kind, in.g_scale, S.f);
        apf::gather_vector_host(s, in, in.zero_tol, 1, S.inc_xb, in.n_u, nullptr, in.u0_kind, in.g_scale, S.g);
        apf::sync(s);
    });
    if (rc != APF_OK)
        return rc;
    *out = h.release();
    return APF_OK;
}

int apf_assemble_graph_norm(apf_ctx* ctx, apf_system* sys, double diagonal_tolerance)
{
    if (!ctx || !sys)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        APF_HOST_RANGE("call_assemble_graph_norm");
        apf::assemble_graph_norm(sys->sys, diagonal_tolerance);
    });
}

int apf_system_block_info(const apf_system* sys, int block, int32_t* rows, int32_t* cols, int64_t* nnz)
{
    if (!sys || block < 0 || block >= APF_N_BLOCKS || !sys->sys.have[block])
        return APF_ERR_INVALID;
    const auto& b = sys->sys.blocks[block];
    if (rows) *rows = b.rows;
    if (cols) *cols = b.cols;
    if (nnz) *nnz = b.nnz();
    return APF_OK;
}

int apf_system_block_copy(apf_ctx* ctx, const apf_system* sys, int block, int32_t* row_ptr, int32_t* col_idx,
                          double* values, int to_device)
{
    if (!ctx || !sys || block < 0 || block >= APF_N_BLOCKS || !sys->sys.have[block])
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        const auto& b = sys->sys.blocks[block];
        const cudaMemcpyKind k = to_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        if (row_ptr)
            APF_CUDA(cudaMemcpyAsync(row_ptr, b.row_ptr.get(), (b.rows + 1) * sizeof(int), k, ctx->stream));
        if (col_idx && b.nnz())
            APF_CUDA(cudaMemcpyAsync(col_idx, b.col_idx.get(), b.nnz() * sizeof(int), k, ctx->stream));
        if (values && b.nnz())
            APF_CUDA(cudaMemcpyAsync(values, b.values.get(), b.nnz() * sizeof(double), k, ctx->stream));
        APF_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int apf_system_block_device_ptrs(const apf_system* sys, int block, const int32_t** row_ptr, const int32_t** col_idx,
                                 const double** values)
{
    if (!sys || block < 0 || block >= APF_N_BLOCKS || !sys->sys.have[block])
        return APF_ERR_INVALID;
    const auto& b = sys->sys.blocks[block];
    if (row_ptr) *row_ptr = b.row_ptr.get();
    if (col_idx) *col_idx = b.col_idx.get();
    if (values) *values = b.values.get();
    return APF_OK;
}

int apf_system_vector_copy(apf_ctx* ctx, const apf_system* sys, int which, double* out, int to_device)
{
    if (!ctx || !sys || !out || (which != APF_VEC_F && which != APF_VEC_G))
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        const auto& v = which == APF_VEC_F ? sys->sys.f : sys->sys.g;
        if (v.size())
            APF_CUDA(cudaMemcpyAsync(out, v.get(), v.size() * sizeof(double),
                                     to_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, ctx->stream));
        APF_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

void apf_solver_options_default(apf_solver_options* opt)
{
    if (!opt)
        return;
    opt->tolerance = 1e-8;
    opt->max_iterations = 20000;
    opt->use_true_residual_batching = 1;
    opt->true_residual_check_interval = 100;
    opt->preconditioner = APF_PRECOND_AMG_BLOCK;
    opt->amg_smooth_steps = 2;
    opt->amg_strength = 0.08;
    opt->amg_coarse_size = 256;
    opt->amg_aggressive_levels = 1;
    opt->amg_vcycles = 1;
}

namespace
{
    apf::AmgOptions amg_options(const apf_solver_options* o)
    {
        apf::AmgOptions a;
        a.smooth_steps = std::max(1, o->amg_smooth_steps);
        a.strength = o->amg_strength;
        a.coarse_size = std::max(16, o->amg_coarse_size);
        a.aggressive_levels = std::max(0, o->amg_aggressive_levels);
        a.vcycles = std::min(2, std::max(1, o->amg_vcycles));
        return a;
    }

    // smoother weights of the set-up hierarchy: plain omega D^-1, or the learned model's
    void install_smoothers(apf_ctx* ctx, apf::System& S, int kind)
    {
        apf::require(kind == APF_PRECOND_AMG_BLOCK || kind == APF_PRECOND_LEARNED, APF_ERR_INVALID,
                     "unknown preconditioner");
        if (kind == APF_PRECOND_LEARNED)
        {
            apf::require(ctx->learned != nullptr, APF_ERR_INVALID,
                         "APF_PRECOND_LEARNED needs a model (apf_ctx_set_learned_model)");
            if (S.precond_kind == APF_PRECOND_LEARNED && S.precond_model_version == ctx->learned_version)
                return;
            APF_HOST_RANGE("learned_install");
            apf::apply_learned_smoothers(ctx->stream, *ctx->learned, S.precond->amg_a, 0);
            apf::apply_learned_smoothers(ctx->stream, *ctx->learned, S.precond->amg_h, 1);
            S.precond_model_version = ctx->learned_version;
        }
        else if (S.precond_kind != APF_PRECOND_AMG_BLOCK)
        {
            S.precond->amg_a.reset_smoothers();
            S.precond->amg_h.reset_smoothers();
        }
        S.precond_kind = kind;
    }

    void setup_precond(apf_ctx* ctx, apf_system* h, const apf_solver_options* opt)
    {
        auto& S = h->sys;
        apf::require(S.have[APF_BLOCK_HHAT], APF_ERR_INVALID,
                     "ParabolicGraphNorm requires graph-norm block context from assembly (call apf_assemble_graph_norm)");
        APF_HOST_RANGE("setup_preconditioner");
        const auto t0 = std::chrono::steady_clock::now();
        S.precond.reset();
        auto p = std::make_unique<apf::BlockPreconditioner>();
        S.precond_opts = amg_options(opt);
        if (!S.blocks[APF_BLOCK_A_Y].sell)
            apf::build_sell(ctx->stream, S.blocks[APF_BLOCK_A_Y]);
        apf::DeviceBuffer<int> y_comp, x_comp;
        apf::dof_time_components(ctx->stream, S.in, true, y_comp);
        apf::dof_time_components(ctx->stream, S.in, false, x_comp);
        p->setup(ctx->stream, S.blocks[APF_BLOCK_A_Y], S.blocks[APF_BLOCK_HHAT], S.precond_opts, S.ws, y_comp.get(),
                 x_comp.get());
        apf::sync(ctx->stream);
        S.precond = std::move(p); // only a fully set-up preconditioner is kept
        S.precond_kind = APF_PRECOND_AMG_BLOCK;
        install_smoothers(ctx, S, opt->preconditioner);
        S.precond_setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
}

int apf_setup_preconditioner(apf_ctx* ctx, apf_system* sys, const apf_solver_options* opt)
{
    if (!ctx || !sys || !opt)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] { setup_precond(ctx, sys, opt); });
}

namespace
{
    // MINRES on the system's K; rhs NULL = the assembled [f; g].  correction: initial_guess
    // is x0, MINRES solves K d = rhs - K x0 from zero and the solution is x0 + d.
    int solve_minres(apf_ctx* ctx, apf_system* sys, const apf_solver_options* opt, const double* rhs,
                     const double* initial_guess, double* solution, int pointers_on_device,
                     apf_solver_diagnostics* diag, bool correction = false);
}

int apf_solve_minres(apf_ctx* ctx, apf_system* sys, const apf_solver_options* opt, const double* initial_guess,
                     double* solution, int pointers_on_device, apf_solver_diagnostics* diag)
{
    return solve_minres(ctx, sys, opt, nullptr, initial_guess, solution, pointers_on_device, diag);
}

int apf_solve_minres_with_rhs(apf_ctx* ctx, apf_system* sys, const apf_solver_options* opt, const double* rhs,
                              const double* initial_guess, double* solution, int pointers_on_device,
                              apf_solver_diagnostics* diag)
{
    if (!rhs)
        return APF_ERR_INVALID;
    return solve_minres(ctx, sys, opt, rhs, initial_guess, solution, pointers_on_device, diag);
}

int apf_solve_minres_correction(apf_ctx* ctx, apf_system* sys, const apf_solver_options* opt, const double* x0,
                                double* solution, int pointers_on_device, apf_solver_diagnostics* diag)
{
    if (!x0)
        return APF_ERR_INVALID;
    return solve_minres(ctx, sys, opt, nullptr, x0, solution, pointers_on_device, diag, true);
}

namespace
{
int solve_minres(apf_ctx* ctx, apf_system* sys, const apf_solver_options* opt, const double* rhs,
                 const double* initial_guess, double* solution, int pointers_on_device, apf_solver_diagnostics* diag,
                 bool correction)
{
    if (!ctx || !sys || !opt)
        return APF_ERR_INVALID;
    apf::MinresSummary summary;
    double solve_seconds = 0.0;
    int used = -1, fallback = 0;
    int rc = guarded(ctx, [&] {
        APF_HOST_RANGE("call_solve_minres");
        auto& S = sys->sys;
        cudaStream_t s = ctx->stream;
        apf::require(opt->tolerance >= 0.0, APF_ERR_INVALID, "negative tolerance");
        if (!S.precond)
            setup_precond(ctx, sys, opt);
        else
            install_smoothers(ctx, S, opt->preconditioner);
        const int nl = S.in.n_lambda, nu = S.in.n_u, n = nl + nu;
        S.rhs.allocate(n, s);
        if (rhs)
            APF_CUDA(cudaMemcpyAsync(S.rhs.get(), rhs, n * sizeof(double),
                                     pointers_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
        else
        {
            apf::copy(s, nl, S.f.get(), S.rhs.get());
            apf::copy(s, nu, S.g.get(), S.rhs.get() + nl);
        }
        S.solution.allocate(n, s);
        if (!S.blocks[APF_BLOCK_K].sell)
            apf::build_sell(s, S.blocks[APF_BLOCK_K]);
        apf::DeviceBuffer<double> x0;
        if (correction)
        {
            // the correction equation K d = b - K x0 (d from zero), x = x0 + d afterwards
            x0.allocate(n, s);
            APF_CUDA(cudaMemcpyAsync(x0.get(), initial_guess, n * sizeof(double),
                                     pointers_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
            apf::spmv(s, S.blocks[APF_BLOCK_K], x0.get(), S.rhs.get(), -1.0, 1.0);
            apf::fill(s, n, 0.0, S.solution.get());
        }
        else if (initial_guess)
            APF_CUDA(cudaMemcpyAsync(S.solution.get(), initial_guess, n * sizeof(double),
                                     pointers_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
        else
            apf::fill(s, n, 0.0, S.solution.get());
        apf::MinresOptions mo;
        mo.tolerance = opt->tolerance;
        mo.max_iterations = opt->max_iterations;
        mo.batch = opt->use_true_residual_batching ? opt->true_residual_check_interval : opt->max_iterations;
        mo.parts = S.partition.n_parts > 0 ? &S.partition : nullptr;
        const auto t0 = std::chrono::steady_clock::now();
        S.precond->prepare(s, S.ws);
        summary = apf::minres_solve(s, S.blocks[APF_BLOCK_K], *S.precond, S.rhs.get(), S.solution.get(), mo, S.ws);
        used = S.precond_kind;
        if (!summary.converged && S.precond_kind == APF_PRECOND_LEARNED)
        {
            // the plain block preconditioner is the fallback: a fresh run from the learned
            // run's iterate
            install_smoothers(ctx, S, APF_PRECOND_AMG_BLOCK);
            S.precond->prepare(s, S.ws);
            const apf::MinresSummary first = summary;
            summary = apf::minres_solve(s, S.blocks[APF_BLOCK_K], *S.precond, S.rhs.get(), S.solution.get(), mo, S.ws);
            summary.iterations += first.iterations;
            summary.batches += first.batches;
            used = APF_PRECOND_AMG_BLOCK;
            fallback = 1;
        }
        solve_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (correction)
            apf::axpby(s, n, 1.0, x0.get(), 1.0, S.solution.get());
        if (solution)
            APF_CUDA(cudaMemcpyAsync(solution, S.solution.get(), n * sizeof(double),
                                     pointers_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
        apf::sync(s);
    });
    if (diag)
    {
        *diag = apf_solver_diagnostics{};
        sys->sys.part_residuals = summary.part_residuals;
        diag->iterations = summary.iterations;
        diag->residual_check_batches = summary.batches;
        diag->converged = summary.converged ? 1 : 0;
        diag->backend_converged = summary.backend_converged ? 1 : 0;
        diag->backend_reported_error = summary.backend_error;
        diag->final_true_residual = summary.true_residual;
        diag->setup_seconds = sys->sys.precond_setup_seconds;
        diag->solve_seconds = solve_seconds;
        diag->preconditioner_used = used;
        diag->learned_fallback = fallback;
        if (sys->sys.precond)
        {
            diag->amg_levels_lambda = sys->sys.precond->amg_a.levels();
            diag->amg_levels_u = sys->sys.precond->amg_h.levels();
            diag->amg_nnz_lambda = sys->sys.precond->amg_a.operator_nnz();
            diag->amg_nnz_u = sys->sys.precond->amg_h.operator_nnz();
        }
    }
    if (rc == APF_OK && !summary.converged)
    {
        char buf[256];
        std::snprintf(buf, sizeof(buf),
                      "MINRES(ParabolicGraphNorm) solve failed. iterations=%d, error=%.12e, true_relative_residual=%.12e",
                      summary.iterations, summary.backend_error, summary.true_residual);
        ctx->last_error = buf;
        rc = APF_ERR_NOT_CONVERGED;
    }
    return rc;
}
}

int apf_system_set_solution(apf_ctx* ctx, apf_system* sys, const double* x, int pointers_on_device)
{
    if (!ctx || !sys || !x)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        auto& S = sys->sys;
        const int n = S.in.n_lambda + S.in.n_u;
        S.solution.allocate(static_cast<std::size_t>(n), ctx->stream);
        APF_CUDA(cudaMemcpyAsync(S.solution.get(), x, n * sizeof(double),
                                 pointers_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
        apf::sync(ctx->stream);
    });
}

int apf_system_residual_norms(apf_ctx* ctx, apf_system* sys, const double* x, int pointers_on_device,
                              double* residual_norm, double* rhs_norm)
{
    if (!ctx || !sys || !residual_norm || !rhs_norm)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        auto& S = sys->sys;
        cudaStream_t s = ctx->stream;
        const int nl = S.in.n_lambda, nu = S.in.n_u, n = nl + nu;
        apf::require(x != nullptr || S.solution.size() == static_cast<std::size_t>(n), APF_ERR_INVALID,
                     "apf_system_residual_norms: no solution held (solve first or pass x)");
        apf::DeviceBuffer<double> b(n, s), r(n, s), xd;
        apf::copy(s, nl, S.f.get(), b.get());
        apf::copy(s, nu, S.g.get(), b.get() + nl);
        const double* xp = S.solution.get();
        if (x)
        {
            xd.allocate(n, s);
            APF_CUDA(cudaMemcpyAsync(xd.get(), x, n * sizeof(double),
                                     pointers_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
            xp = xd.get();
        }
        apf::residual(s, S.blocks[APF_BLOCK_K], xp, b.get(), r.get());
        const double rr = apf::dot_host(s, S.ws, n, r.get(), r.get());
        const double bb = apf::dot_host(s, S.ws, n, b.get(), b.get());
        *residual_norm = rr >= 0.0 ? std::sqrt(rr) : std::numeric_limits<double>::quiet_NaN();
        *rhs_norm = bb >= 0.0 ? std::sqrt(bb) : std::numeric_limits<double>::quiet_NaN();
    });
}

int apf_system_keep_flux(apf_ctx* ctx, apf_system* sys, int keep)
{
    if (!ctx || !sys)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        auto& S = sys->sys;
        S.keep_flux = keep != 0;
        if (!S.keep_flux)
        {
            S.flux_cells = 0;
            S.flux_sigma = apf::DeviceBuffer<double>();
            S.flux_geo = apf::DeviceBuffer<double>();
            S.flux_slab.clear();
            S.flux_source.clear();
        }
    });
}

int apf_flux_cells(apf_ctx* ctx, const apf_system* sys, int32_t* n_cells, int32_t* slab, int32_t* source_y_cell)
{
    if (!ctx || !sys || !n_cells)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        const auto& S = sys->sys;
        *n_cells = S.flux_cells;
        for (int c = 0; c < S.flux_cells; ++c)
        {
            if (slab)
                slab[c] = S.flux_slab[static_cast<std::size_t>(c)];
            if (source_y_cell)
                source_y_cell[c] = S.flux_source[static_cast<std::size_t>(c)];
        }
    });
}

int apf_flux_sample(apf_ctx* ctx, apf_system* sys, int32_t n_points, const int32_t* cell, const double* points,
                    double* values, int pointers_on_device)
{
    if (!ctx || !sys || n_points < 0 || (n_points > 0 && (!cell || !points || !values)))
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        APF_HOST_RANGE("call_flux_sample");
        apf::flux_sample(ctx->stream, sys->sys, n_points, cell, points, values, pointers_on_device != 0);
    });
}

int apf_preconditioner_apply(apf_ctx* ctx, apf_system* sys, int block, const double* r, double* z,
                             int pointers_on_device)
{
    if (!ctx || !sys || !r || !z || block < 0 || block > 2)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        auto& S = sys->sys;
        apf::require(S.precond != nullptr, APF_ERR_INVALID, "preconditioner has not been set up");
        cudaStream_t s = ctx->stream;
        const int nl = S.in.n_lambda, nu = S.in.n_u;
        const int n = block == 0 ? nl : (block == 1 ? nu : nl + nu);
        apf::DeviceBuffer<double> dr(n, s), dz(n, s);
        APF_CUDA(cudaMemcpyAsync(dr.get(), r, n * sizeof(double),
                                 pointers_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
        S.precond->prepare(s, S.ws);
        if (block < 2)
            S.precond->apply_block(s, block, dr.get(), dz.get());
        else
            S.precond->apply(s, dr.get(), dz.get());
        APF_CUDA(cudaMemcpyAsync(z, dz.get(), n * sizeof(double),
                                 pointers_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
        apf::sync(s);
    });
}

int apf_system_set_partition(apf_ctx* ctx, apf_system* sys, int n_parts, const int32_t* lambda_offsets,
                             const int32_t* u_offsets)
{
    if (!ctx || !sys || n_parts < 0 || (n_parts > 0 && (!lambda_offsets || !u_offsets)))
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        auto& S = sys->sys;
        const int nl = S.in.n_lambda, nu = S.in.n_u;
        std::vector<int2> segs(2 * static_cast<std::size_t>(n_parts));
        if (n_parts > 0)
            apf::require(lambda_offsets[0] == 0 && u_offsets[0] == 0 && lambda_offsets[n_parts] == nl &&
                             u_offsets[n_parts] == nu,
                         APF_ERR_INVALID, "partition offsets must start at 0 and end at n_lambda / n_u");
        for (int p = 0; p < n_parts; ++p)
        {
            apf::require(lambda_offsets[p] <= lambda_offsets[p + 1] && u_offsets[p] <= u_offsets[p + 1],
                         APF_ERR_INVALID, "partition offsets must not decrease");
            segs[2 * p] = make_int2(lambda_offsets[p], lambda_offsets[p + 1]);
            segs[2 * p + 1] = make_int2(nl + u_offsets[p], nl + u_offsets[p + 1]);
        }
        S.partition.n_parts = n_parts;
        S.partition.segs.allocate(std::max<std::size_t>(segs.size(), 1), ctx->stream);
        if (!segs.empty())
            S.partition.segs.upload(segs.data(), segs.size());
        S.part_residuals.clear();
    });
}

int apf_system_part_residuals(apf_ctx* ctx, const apf_system* sys, double* out)
{
    if (!ctx || !sys || !out)
        return APF_ERR_INVALID;
    const auto& r = sys->sys.part_residuals;
    if (static_cast<int>(r.size()) != sys->sys.partition.n_parts)
        return APF_ERR_INVALID;
    std::copy(r.begin(), r.end(), out);
    return APF_OK;
}

int apf_ctx_set_autotune(apf_ctx* ctx, int enable)
{
    if (!ctx)
        return APF_ERR_INVALID;
    ctx->tuner.enabled = enable != 0;
    if (enable < 0)
        ctx->tuner = apf::PatchTuner{};
    return APF_OK;
}

const char* apf_ctx_autotune_report(apf_ctx* ctx)
{
    if (!ctx)
        return "";
    std::string r = "{";
    bool first = true;
    const auto& t = ctx->tuner;
    for (int p = 0; p < 2; ++p)
        for (int f = 0; f < 2; ++f)
            for (int b = 0; b < apf::kPatchBuckets; ++b)
            {
                if (t.width[p][f][b] == 0)
                    continue;
                char buf[256];
                std::snprintf(buf, sizeof(buf),
                              "%s\"p%d_%s_n%d\": {\"warps_per_patch\": %d, \"patches\": %d, \"ms_w1_w2_w4\": [%.3f, %.3f, %.3f]}",
                              first ? "" : ", ", p + 1, f ? "fp32_refined" : "fp64", apf::kPatchBucketMax[b],
                              t.width[p][f][b], t.patches[p][f][b], t.ms[p][f][b][0], t.ms[p][f][b][1],
                              t.ms[p][f][b][2]);
                r += buf;
                first = false;
            }
    r += "}";
    ctx->tune_report = r;
    return ctx->tune_report.c_str();
}

int apf_ctx_set_patch_precision(apf_ctx* ctx, int precision)
{
    if (!ctx || (precision != APF_PATCH_FP64 && precision != APF_PATCH_FP32_REFINED))
        return APF_ERR_INVALID;
    ctx->patch_precision = precision;
    return APF_OK;
}

int apf_estimate(apf_ctx* ctx, apf_system* sys, const int32_t* y_vertex_ids, int pointers_on_device,
                 double* flux_squared, double* divergence_squared, double* reconstruction_squared, double* eta_squared,
                 apf_estimator_result* result)
{
    if (!ctx || !sys || (!y_vertex_ids && sys->sys.in.dim != 1))
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        APF_HOST_RANGE("call_estimate");
        auto& S = sys->sys;
        apf::EstimatorTotals t;
        if (S.in.dim == 1)
        {
            t = apf::estimate_1d(ctx->stream, S, flux_squared, divergence_squared, reconstruction_squared, eta_squared,
                                 pointers_on_device != 0);
        }
        else
        {
            const std::size_t n = 3ull * static_cast<std::size_t>(S.in.n_y_cells);
            std::vector<int> vids(n);
            if (n)
                APF_CUDA(cudaMemcpyAsync(vids.data(), y_vertex_ids, n * sizeof(int),
                                         pointers_on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost,
                                         ctx->stream));
            apf::sync(ctx->stream);
            t = apf::estimate(ctx->stream, S, vids, flux_squared, divergence_squared, reconstruction_squared,
                              eta_squared, pointers_on_device != 0, ctx->patch_precision, &ctx->tuner);
        }
        if (result)
        {
            result->flux_squared = t.flux;
            result->divergence_squared = t.div;
            result->reconstruction_squared = t.recon;
            result->eta_squared = t.eta;
            result->n_slabs = t.n_slabs;
            result->n_patches = t.n_patches;
            result->max_patch_cells = t.max_patch_cells;
            result->reconstruction_iterations = t.recon_iterations;
            result->reconstruction_residual = t.recon_residual;
        }
    });
}

int apf_x_indicators(apf_ctx* ctx, apf_system* sys, int pointers_on_device, double* lambda_by_y, double* lambda_by_x,
                     double* trace_by_x, double* eta_by_x, apf_x_indicator_totals* totals)
{
    if (!ctx || !sys)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        auto& S = sys->sys;
        const auto& in = S.in;
        apf::require(S.solution.size() == static_cast<std::size_t>(in.n_lambda) + in.n_u, APF_ERR_INVALID,
                     "X indicators: solve the main system first");
        cudaStream_t s = ctx->stream;
        const int ny = in.n_y_cells, nx = in.n_x_cells;
        apf::DeviceBuffer<double> ly(ny, s), lx(nx, s), tx(nx, s), ex(nx, s);
        apf::x_indicators(s, in, S.solution.get(), S.solution.get() + in.n_lambda, ly.get(), lx.get(), tx.get(),
                          ex.get());
        const cudaMemcpyKind kind = pointers_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        if (lambda_by_y && ny) APF_CUDA(cudaMemcpyAsync(lambda_by_y, ly.get(), ny * sizeof(double), kind, s));
        if (lambda_by_x && nx) APF_CUDA(cudaMemcpyAsync(lambda_by_x, lx.get(), nx * sizeof(double), kind, s));
        if (trace_by_x && nx) APF_CUDA(cudaMemcpyAsync(trace_by_x, tx.get(), nx * sizeof(double), kind, s));
        if (eta_by_x && nx) APF_CUDA(cudaMemcpyAsync(eta_by_x, ex.get(), nx * sizeof(double), kind, s));
        if (totals)
        {
            S.ws.ensure(s);
            totals->lambda_y_squared = apf::dot_host(s, S.ws, nx, lx.get(), nullptr);
            totals->initial_trace_squared = apf::dot_host(s, S.ws, nx, tx.get(), nullptr);
            totals->eta_squared = totals->lambda_y_squared + totals->initial_trace_squared;
        }
        apf::sync(s);
    });
}

int apf_y_estimator_threshold_squared(double rho, double lambda_y_squared, double initial_trace_squared,
                                      double* threshold_squared)
{
    if (!threshold_squared || !(rho > 0.0))
        return APF_ERR_INVALID;
    const double shifted = rho + 0.5;
    *threshold_squared = rho * rho * (lambda_y_squared + (1.0 + 1.0 / (shifted * shifted)) * initial_trace_squared);
    return APF_OK;
}

int apf_g_estimator(apf_ctx* ctx, apf_system* sys, int32_t n_g, const int32_t* g_restr_offsets,
                    const int32_t* g_restr_dofs, const double* g_restr_weights, int32_t g_restr_nnz, double tolerance,
                    apf_g_estimator_result* result)
{
    if (!ctx || !sys || !g_restr_offsets || !result || n_g < 0 || g_restr_nnz < 0 || !(tolerance > 0.0) ||
        (g_restr_nnz > 0 && (!g_restr_dofs || !g_restr_weights)))
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        APF_HOST_RANGE("call_g_estimator");
        auto& S = sys->sys;
        const std::size_t rows = static_cast<std::size_t>(S.in.n_y_cells) * 18;
        apf::require(S.in.p == 1 && S.in.dim == 2, APF_ERR_INVALID,
                     "G^delta estimator: 2+1D systems of degree 1 (G of degree 2)");
        const std::vector<int> off(g_restr_offsets, g_restr_offsets + rows + 1);
        const std::vector<int> dofs(g_restr_dofs, g_restr_dofs + g_restr_nnz);
        const std::vector<double> w(g_restr_weights, g_restr_weights + g_restr_nnz);
        const apf::GDeltaResult r = apf::g_delta(ctx->stream, S, n_g, off, dofs, w, tolerance);
        *result = apf_g_estimator_result{};
        result->lambda_difference_squared = r.lambda_difference_squared;
        result->solve_relative_residual = r.relative_residual;
        result->solve_iterations = r.iterations;
        result->n_g = r.n_g;
    });
}

int apf_write_cellwise_error_binary(apf_ctx* ctx, const char* path, int32_t n_cells, const int32_t* cell_ids,
                                    const double* values, int pointers_on_device, int sort_descending)
{
    if (!path || n_cells < 0 || (pointers_on_device && !ctx))
        return APF_ERR_INVALID;
    return host_guarded(ctx, [&] {
        const auto ids = fetch_host(ctx, cell_ids, n_cells, pointers_on_device != 0);
        const auto v = fetch_host(ctx, values, n_cells, pointers_on_device != 0);
        // header: format version 1, entry count
        write_artifact(path, {1, n_cells}, ids, {&v}, artifact_order(ids, v, sort_descending != 0));
    });
}

int apf_write_cellwise_error_components_binary(apf_ctx* ctx, const char* path, int32_t n_cells,
                                               const int32_t* cell_ids, const double* flux, const double* recon,
                                               const double* divergence, const double* eta, int pointers_on_device,
                                               int sort_descending)
{
    if (!path || n_cells < 0 || (pointers_on_device && !ctx))
        return APF_ERR_INVALID;
    return host_guarded(ctx, [&] {
        const bool dev = pointers_on_device != 0;
        const auto ids = fetch_host(ctx, cell_ids, n_cells, dev);
        const auto f = fetch_host(ctx, flux, n_cells, dev);
        const auto r = fetch_host(ctx, recon, n_cells, dev);
        const auto d = fetch_host(ctx, divergence, n_cells, dev);
        const auto e = fetch_host(ctx, eta, n_cells, dev);
        // header: format version 1, entry count, 4 components
        write_artifact(path, {1, n_cells, 4}, ids, {&f, &r, &d, &e}, artifact_order(ids, e, sort_descending != 0));
    });
}

int apf_write_x_indicator_components_binary(apf_ctx* ctx, const char* path, int32_t n_x_cells,
                                            const int32_t* x_cell_ids, const double* lambda_by_x,
                                            const double* trace_by_x, const double* eta_by_x, int pointers_on_device)
{
    if (!path || n_x_cells < 0 || (pointers_on_device && !ctx))
        return APF_ERR_INVALID;
    return host_guarded(ctx, [&] {
        const bool dev = pointers_on_device != 0;
        const auto ids = fetch_host(ctx, x_cell_ids, n_x_cells, dev);
        const auto l = fetch_host(ctx, lambda_by_x, n_x_cells, dev);
        const auto t = fetch_host(ctx, trace_by_x, n_x_cells, dev);
        const auto e = fetch_host(ctx, eta_by_x, n_x_cells, dev);
        // header: format version 1, entry count, 3 components; always by decreasing eta
        write_artifact(path, {1, n_x_cells, 3}, ids, {&l, &t, &e}, artifact_order(ids, e, true));
    });
}

int apf_true_residual_noalloc(apf_ctx* ctx, int32_t rows, const int32_t* row_ptr, const int32_t* col_idx,
                              const double* values, const double* x, const double* b, double* absolute_residual,
                              double* relative_residual)
{
    if (!ctx)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        apf::true_residual_noalloc(ctx->device, ctx->stream, rows, row_ptr, col_idx, values, x, b, absolute_residual,
                                   relative_residual);
    });
}

int apf_system_solution_device_ptr(const apf_system* sys, const double** solution)
{
    if (!sys || !solution || !sys->sys.solution.size())
        return APF_ERR_INVALID;
    *solution = sys->sys.solution.get();
    return APF_OK;
}

void apf_system_destroy(apf_system* sys)
{
    if (!sys)
        return;
    if (sys->ctx)
    {
        cudaSetDevice(sys->ctx->device);
        cudaStreamSynchronize(sys->ctx->stream);
    }
    delete sys;
}

} // extern "C"

// ---- learned preconditioner ----------------------------------------------------------

int apf_learned_model_create(apf_learned_model** out)
{
    if (!out)
        return APF_ERR_INVALID;
    *out = new (std::nothrow) apf_learned_model();
    return *out ? APF_OK : APF_ERR_INTERNAL;
}

int apf_learned_model_destroy(apf_learned_model* model)
{
    delete model;
    return APF_OK;
}

int apf_learned_model_set_params(apf_learned_model* model, const float* params, int n)
{
    if (!model || !params || n != apf::learned::kParams)
        return APF_ERR_INVALID;
    std::memcpy(model->model.params.data(), params, sizeof(float) * n);
    return APF_OK;
}

int apf_learned_model_get_params(const apf_learned_model* model, float* params, int n)
{
    if (!model || !params || n != apf::learned::kParams)
        return APF_ERR_INVALID;
    std::memcpy(params, model->model.params.data(), sizeof(float) * n);
    return APF_OK;
}

int apf_ctx_set_learned_model(apf_ctx* ctx, const apf_learned_model* model)
{
    if (!ctx)
        return APF_ERR_INVALID;
    if (model)
        ctx->learned = std::make_unique<apf::LearnedModel>(model->model);
    else
        ctx->learned.reset();
    ++ctx->learned_version;
    return APF_OK;
}

int apf_learned_loss_and_grad(apf_ctx* ctx, apf_system* sys, const apf_learned_model* model, int samples, int steps,
                              int burn_in, uint64_t seed, const double* start_vectors, int pointers_on_device,
                              double* loss, float* grad)
{
    if (!ctx || !sys || !model)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        auto& S = sys->sys;
        apf::require(S.precond != nullptr, APF_ERR_INVALID, "learned loss: set up the preconditioner first");
        cudaStream_t s = ctx->stream;
        const long long n = static_cast<long long>(S.in.n_lambda) + S.in.n_u;
        apf::DeviceBuffer<double> starts;
        const double* sv = nullptr;
        if (start_vectors)
        {
            if (pointers_on_device)
                sv = start_vectors;
            else
            {
                starts.allocate(static_cast<std::size_t>(n) * std::max(1, samples), s);
                starts.upload(start_vectors, static_cast<std::size_t>(n) * std::max(1, samples));
                sv = starts.get();
            }
        }
        const double L = apf::learned_loss_and_grad(s, model->model, *S.precond, S.blocks[APF_BLOCK_A_Y],
                                                     S.blocks[APF_BLOCK_HHAT], samples, steps, burn_in, seed, sv, grad,
                                                     S.ws);
        apf::sync(s);
        S.precond_kind = -2; // FP32-model weights installed: the next solve re-installs
        if (loss)
            *loss = L;
    });
}

int apf_learned_forward(apf_ctx* ctx, const apf_learned_model* model, int n, const float* features, float* y,
                        int precision, int pointers_on_device)
{
    if (!ctx || !model || n < 0 || (n > 0 && (!features || !y)) || (precision != 0 && precision != 1))
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        cudaStream_t s = ctx->stream;
        apf::DeviceBuffer<float> dp(apf::learned::kParams, s);
        dp.upload(model->model.params.data(), apf::learned::kParams);
        apf::DeviceBuffer<float> f, out;
        const float* fp = features;
        float* yp = y;
        if (!pointers_on_device)
        {
            f.allocate(static_cast<std::size_t>(n) * apf::learned::kFeatures, s);
            f.upload(features, static_cast<std::size_t>(n) * apf::learned::kFeatures);
            out.allocate(static_cast<std::size_t>(n) * apf::learned::kOutputs, s);
            fp = f.get();
            yp = out.get();
        }
        apf::learned_forward(s, dp.get(), n, fp, yp, precision);
        if (!pointers_on_device && n > 0)
            APF_CUDA(cudaMemcpyAsync(y, out.get(), static_cast<std::size_t>(n) * apf::learned::kOutputs * sizeof(float),
                                     cudaMemcpyDeviceToHost, s));
        apf::sync(s);
    });
}

namespace
{
    apf::Amg& amg_of(apf_system* sys, int block)
    {
        auto& S = sys->sys;
        apf::require(S.precond != nullptr, APF_ERR_INVALID, "no preconditioner set up");
        apf::require(block == 0 || block == 1, APF_ERR_INVALID, "block must be 0 (A_y) or 1 (Hhat)");
        return block == 0 ? S.precond->amg_a : S.precond->amg_h;
    }

    apf::AmgLevel& level_of(apf_system* sys, int block, int level)
    {
        apf::Amg& amg = amg_of(sys, block);
        apf::require(level >= 0 && level < amg.levels(), APF_ERR_INVALID, "no such AMG level");
        return amg.level(level);
    }
}

int apf_amg_info(apf_ctx* ctx, apf_system* sys, int block, int* levels, int* dense_coarse, int* coarse_sweeps,
                 int* smooth_steps)
{
    if (!ctx || !sys)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        apf::Amg& amg = amg_of(sys, block);
        if (levels) *levels = amg.levels();
        if (dense_coarse) *dense_coarse = amg.dense_coarse() ? 1 : 0;
        if (coarse_sweeps) *coarse_sweeps = apf::Amg::coarse_sweeps();
        if (smooth_steps) *smooth_steps = sys->sys.precond_opts.smooth_steps;
    });
}

int apf_amg_level_info(apf_ctx* ctx, apf_system* sys, int block, int level, int* rows, int64_t* nnz_a,
                       int64_t* nnz_p, double* omega, double* alpha)
{
    if (!ctx || !sys)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        apf::AmgLevel& L = level_of(sys, block, level);
        if (rows) *rows = L.A->rows;
        if (nnz_a) *nnz_a = L.A->nnz();
        if (nnz_p) *nnz_p = L.P.nnz();
        if (omega) *omega = L.omega;
        if (alpha) *alpha = L.alpha;
    });
}

int apf_amg_level_copy(apf_ctx* ctx, apf_system* sys, int block, int level, int which, int32_t* row_ptr,
                       int32_t* col_idx, double* values)
{
    if (!ctx || !sys || (which != 0 && which != 1))
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        apf::AmgLevel& L = level_of(sys, block, level);
        const apf::DeviceCsr& M = which == 0 ? *L.A : L.P;
        cudaStream_t s = ctx->stream;
        if (row_ptr && M.row_ptr.size())
            APF_CUDA(cudaMemcpyAsync(row_ptr, M.row_ptr.get(), M.row_ptr.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
        if (col_idx && M.nnz())
            APF_CUDA(cudaMemcpyAsync(col_idx, M.col_idx.get(), M.nnz() * sizeof(int), cudaMemcpyDeviceToHost, s));
        if (values && M.nnz())
            APF_CUDA(cudaMemcpyAsync(values, M.values.get(), M.nnz() * sizeof(double), cudaMemcpyDeviceToHost, s));
        apf::sync(s);
    });
}

int apf_amg_level_weights(apf_ctx* ctx, apf_system* sys, int block, int level, int o, double* weights)
{
    if (!ctx || !sys || !weights || (o != 0 && o != 1))
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        apf::AmgLevel& L = level_of(sys, block, level);
        cudaStream_t s = ctx->stream;
        const int n = L.A->rows;
        apf::require(L.dinv.size() == static_cast<std::size_t>(n), APF_ERR_INTERNAL, "AMG level without its diagonal");
        const apf::DeviceBuffer<double>& W = (o == 1 && L.w2.size()) ? L.w2 : L.w;
        if (W.size())
            APF_CUDA(cudaMemcpyAsync(weights, W.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
        else
        {
            apf::DeviceBuffer<double> t(n, s);
            apf::axpby(s, n, L.omega, L.dinv.get(), 0.0, t.get());
            APF_CUDA(cudaMemcpyAsync(weights, t.get(), n * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        apf::sync(s);
    });
}

int apf_amg_level_features(apf_ctx* ctx, apf_system* sys, int block, int level, float* features)
{
    if (!ctx || !sys || !features)
        return APF_ERR_INVALID;
    return guarded(ctx, [&] {
        apf::AmgLevel& L = level_of(sys, block, level);
        cudaStream_t s = ctx->stream;
        const int n = L.A->rows;
        apf::require(L.dinv.size() == static_cast<std::size_t>(n), APF_ERR_INTERNAL, "AMG level without its diagonal");
        apf::DeviceBuffer<float> f(static_cast<std::size_t>(n) * apf::learned::kFeatures, s);
        apf::learned_features(s, *L.A, L.dinv.get(), level, block, f.get());
        if (n)
            APF_CUDA(cudaMemcpyAsync(features, f.get(), f.size() * sizeof(float), cudaMemcpyDeviceToHost, s));
        apf::sync(s);
    });
}
