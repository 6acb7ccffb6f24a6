// Internal definitions shared by the CUDA translation units of libapf_b200.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/apf_b200.h"

namespace apf
{
    // Error raised inside the library; the C-ABI layer converts it to a status code
    // plus a message retrievable with apf_last_error().
    struct Error : std::runtime_error
    {
        int code;
        Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
    };

#define APF_CUDA(call)                                                                      \
    do                                                                                      \
    {                                                                                       \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            throw ::apf::Error(APF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

    inline void require(bool ok, int code, const std::string& msg)
    {
        if (!ok)
            throw Error(code, msg);
    }
    // literal messages: no string is built unless the check fails (hot host loops)
    inline void require(bool ok, int code, const char* msg)
    {
        if (!ok)
            throw Error(code, msg);
    }

    // Stream-ordered device buffer (cudaMallocAsync / cudaFreeAsync on the owning stream).
    template<class T>
    class DeviceBuffer
    {
    public:
        DeviceBuffer() = default;
        DeviceBuffer(std::size_t n, cudaStream_t s) { allocate(n, s); }
        DeviceBuffer(const DeviceBuffer&) = delete;
        DeviceBuffer& operator=(const DeviceBuffer&) = delete;
        DeviceBuffer(DeviceBuffer&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) { o.p_ = nullptr; o.n_ = 0; }
        DeviceBuffer& operator=(DeviceBuffer&& o) noexcept
        {
            if (this != &o)
            {
                release();
                p_ = o.p_; n_ = o.n_; s_ = o.s_;
                o.p_ = nullptr; o.n_ = 0;
            }
            return *this;
        }
        ~DeviceBuffer() { release(); }

        void allocate(std::size_t n, cudaStream_t s)
        {
            release();
            s_ = s;
            n_ = n;
            if (n > 0)
                APF_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p_), n * sizeof(T), s));
        }
        void release() noexcept
        {
            if (p_)
                cudaFreeAsync(p_, s_);
            p_ = nullptr;
            n_ = 0;
        }
        void zero()
        {
            if (n_)
                APF_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s_));
        }
        void upload(const T* host, std::size_t n)
        {
            if (n != n_)
                allocate(n, s_);
            if (n)
                APF_CUDA(cudaMemcpyAsync(p_, host, n * sizeof(T), cudaMemcpyHostToDevice, s_));
        }
        T* get() const noexcept { return p_; }
        std::size_t size() const noexcept { return n_; }
        cudaStream_t stream() const noexcept { return s_; }

    private:
        T* p_ = nullptr;
        std::size_t n_ = 0;
        cudaStream_t s_ = nullptr;
    };

    // Sliced-ELLPACK copy of a CSR matrix for the SpMV: rows sorted by decreasing length
    // inside windows of 512 (perm: sorted position -> row), slices of 32 sorted rows, each
    // slice stored column-major at its own width (one thread per row, coalesced loads),
    // padding entries have value 0 and column 0.
    struct DeviceSell
    {
        int rows = 0;
        int slices = 0;
        DeviceBuffer<int> perm;      // sorted position -> row
        DeviceBuffer<int> slice_ptr; // slices + 1 element offsets
        DeviceBuffer<int> col;
        DeviceBuffer<double> val;    // f64 values, or empty when val32 holds them
        DeviceBuffer<float> val32;   // f32 values (preconditioner copies; products accumulate in f64)
        // CSR layout instead of slices (operators with few or long rows): row pointers and
        // column indices of the source matrix, which must outlive this copy
        const int* csr_rp = nullptr;
        const int* csr_ci = nullptr;
        double avg_row = 0.0;
    };
    constexpr int kSellMinRows = 148 * 32 * 8; // below: too few slices to fill the GPU
    constexpr double kSellMaxRow = 40.0;       // above: one thread per row serialises

    // Row-compressed sparse matrix resident on the device (int32 indices, f64 values).
    // `sell`, when built (build_sell), is used by the SpMV kernels instead of the CSR arrays;
    // it must be rebuilt if the values change.
    struct DeviceCsr
    {
        int rows = 0;
        int cols = 0;
        DeviceBuffer<int> row_ptr;
        DeviceBuffer<int> col_idx;
        DeviceBuffer<double> values;
        std::unique_ptr<DeviceSell> sell;
        std::int64_t nnz() const noexcept { return static_cast<std::int64_t>(col_idx.size()); }
    };

    extern std::atomic<long long> g_kernel_launches;

    // Optional per-kernel CUDA-event timing (enabled per context with apf_ctx_set_timing).
    struct Profiler
    {
        bool enabled = false;
        bool kernels = true; // false: host ranges only (no per-launch events)
        struct Rec
        {
            const char* name;
            cudaEvent_t a, b;
        };
        std::vector<Rec> pending;
        std::map<std::string, std::pair<long long, double>> totals; // name -> (launches, ms)

        void flush()
        {
            for (auto& r : pending)
            {
                float ms = 0.f;
                cudaEventSynchronize(r.b);
                cudaEventElapsedTime(&ms, r.a, r.b);
                auto& t = totals[r.name];
                t.first += 1;
                t.second += ms;
                cudaEventDestroy(r.a);
                cudaEventDestroy(r.b);
            }
            pending.clear();
        }
    };

    // Profiler of the context whose call is running on this thread (set by the C-ABI layer).
    extern thread_local Profiler* t_profiler;

    // Counts a kernel launch and, when timing is on, brackets it with CUDA events
    // recorded on the launching stream.
    class KernelTimer
    {
    public:
        KernelTimer(const char* name, cudaStream_t s) : s_(s)
        {
            g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
            if (t_profiler && t_profiler->enabled && t_profiler->kernels)
            {
                rec_.name = name;
                cudaEventCreate(&rec_.a);
                cudaEventCreate(&rec_.b);
                cudaEventRecord(rec_.a, s);
                on_ = true;
            }
        }
        ~KernelTimer()
        {
            if (on_)
            {
                cudaEventRecord(rec_.b, s_);
                t_profiler->pending.push_back(rec_);
            }
        }

    private:
        cudaStream_t s_;
        Profiler::Rec rec_{};
        bool on_ = false;
    };

    // Host wall time of a stretch of host-side work (patch topology, set-up loops), recorded
    // as "host:<name>" beside the kernel times when timing is on.
    class HostRange
    {
    public:
        explicit HostRange(const char* name) : name_(name)
        {
            if (t_profiler && t_profiler->enabled)
            {
                on_ = true;
                t0_ = std::chrono::steady_clock::now();
            }
        }
        ~HostRange()
        {
            if (on_)
            {
                const double ms =
                    std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count();
                auto& t = t_profiler->totals[std::string("host:") + name_];
                t.first += 1;
                t.second += ms;
            }
        }

    private:
        const char* name_;
        bool on_ = false;
        std::chrono::steady_clock::time_point t0_;
    };

#define APF_KT_CAT2(a, b) a##b
#define APF_KT_CAT(a, b) APF_KT_CAT2(a, b)
#define APF_KERNEL(name, stream) ::apf::KernelTimer APF_KT_CAT(apf_kt_, __LINE__)(name, stream)
#define APF_HOST_RANGE(name) ::apf::HostRange APF_KT_CAT(apf_hr_, __LINE__)(name)

    // Exclusive scan of n int32 counts into out[0..n] (out[n] = total); returns the total.
    long long exclusive_scan(const int* counts, int* out, int n, cudaStream_t s);

    // Block until the stream is idle and surface any asynchronous error.
    inline void sync(cudaStream_t s)
    {
        APF_CUDA(cudaStreamSynchronize(s));
    }
}
