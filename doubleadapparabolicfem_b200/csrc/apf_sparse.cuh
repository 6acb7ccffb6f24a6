// Sparse/vector building blocks on the device (CSR f64/int32): SpMV, sparse products
// by per-row gather + warp sort, transposes, deterministic reductions.
#pragma once

#include <vector>

#include "apf_internal.hpp"

namespace apf
{
    // Deterministic reductions: fixed grid, per-block partials, fixed-order final sum.
    constexpr int kRedBlocks = 592; // 4 x 148 SMs
    constexpr int kRedThreads = 256;

    struct Workspace
    {
        DeviceBuffer<double> partials; // kRedBlocks * 4
        DeviceBuffer<double> scalars;  // scratch device scalars
        void ensure(cudaStream_t s)
        {
            if (!partials.size())
                partials.allocate(kRedBlocks * 4, s);
            if (!scalars.size())
                scalars.allocate(64, s);
        }
    };

    // Build A.sell (sliced ELLPACK) unless its padding would exceed max_padding x nnz;
    // returns whether it was built.
    bool build_sell(cudaStream_t s, DeviceCsr& A, double max_padding = 1.35);
    // A sliced-ELLPACK copy of A with f32 values (always built): for the V-cycle operators,
    // whose rounding to f32 keeps them symmetric and fixed.
    std::unique_ptr<DeviceSell> make_sell32(cudaStream_t s, const DeviceCsr& A);
    // the SpMV family on such a copy (same semantics as the DeviceCsr versions below)
    void spmv(cudaStream_t s, const DeviceSell& A, const double* x, double* y, double alpha = 1.0, double beta = 0.0,
              const char* name = nullptr);
    void jacobi_sweep(cudaStream_t s, const DeviceSell& A, const double* x, const double* b, const double* dinv,
                      double omega, double* y, const char* name = nullptr);
    void residual(cudaStream_t s, const DeviceSell& A, const double* x, const double* b, double* r,
                  const char* name = nullptr);
    // y = A x and z = omega w y in one pass (a restriction fused with the first damped-Jacobi
    // step from zero on the coarse level)
    void spmv_jacobi_first(cudaStream_t s, const DeviceSell& A, const double* x, double* y, const double* w,
                           double omega, double* z, const char* name = nullptr);
    // y = alpha * A x + beta * y   (beta == 0 ignores y's old contents)
    void spmv(cudaStream_t s, const DeviceCsr& A, const double* x, double* y, double alpha = 1.0, double beta = 0.0,
              const char* name = nullptr);
    // y = x + omega * dinv * (b - A x)   (one damped-Jacobi sweep; y must not alias x)
    void jacobi_sweep(cudaStream_t s, const DeviceCsr& A, const double* x, const double* b, const double* dinv,
                      double omega, double* y);
    // r = b - A x
    void residual(cudaStream_t s, const DeviceCsr& A, const double* x, const double* b, double* r);
    // out = dot(a, b) written to a device scalar (deterministic); b = null: the sum of a
    void dot_device(cudaStream_t s, Workspace& w, int n, const double* a, const double* b, double* out);
    double dot_host(cudaStream_t s, Workspace& w, int n, const double* a, const double* b);
    // C = A * B (pattern = all candidate products, duplicates summed in a fixed order)
    void spgemm(cudaStream_t s, const DeviceCsr& A, const DeviceCsr& B, DeviceCsr& C);
    // T = A^T (rows sorted)
    void transpose(cudaStream_t s, const DeviceCsr& A, DeviceCsr& T);
    // inverse diagonal of a square CSR
    void inverse_diagonal(cudaStream_t s, const DeviceCsr& A, DeviceBuffer<double>& inv);
    // Rows grouped by their candidate count into capacity classes caps[0] < caps[1] < ...:
    // list holds the rows of class 0, then class 1, ...; offsets (host) has ncaps + 1 entries.
    // Rows above the last class are an error (APF_ERR_CAPACITY).
    struct RowBuckets
    {
        DeviceBuffer<int> list;
        std::vector<int> offsets;
    };
    void bucket_rows(cudaStream_t s, int rows, const int* cand, const int* caps, int ncaps, RowBuckets& out);
    // vector helpers
    void axpby(cudaStream_t s, int n, double a, const double* x, double b, double* y); // y = a x + b y
    void copy(cudaStream_t s, int n, const double* x, double* y);
    void fill(cudaStream_t s, int n, double v, double* y);
}
