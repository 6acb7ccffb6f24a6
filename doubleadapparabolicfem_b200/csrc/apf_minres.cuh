// Block-preconditioned MINRES on the device (see apf_minres.cu).
#pragma once

#include <vector>

#include "apf_amg.cuh"

namespace apf
{
    // z = P^{-1} r for a fixed SPD operator P (full saddle size n_lambda + n_u).
    class Preconditioner
    {
    public:
        virtual ~Preconditioner() = default;
        virtual void apply(cudaStream_t s, const double* r, double* z) = 0;
    };

    // blkdiag(A_y, Hhat)^{-1} approximated by one AMG V-cycle per block.  The two V-cycles
    // are independent: the Hhat one runs on a second stream forked from and joined back
    // into the caller's stream, so the latency-bound coarse levels of both overlap.
    class BlockPreconditioner : public Preconditioner
    {
    public:
        BlockPreconditioner() = default;
        BlockPreconditioner(const BlockPreconditioner&) = delete;
        BlockPreconditioner& operator=(const BlockPreconditioner&) = delete;
        ~BlockPreconditioner() override;
        // y_component / x_component: time level of every Y / X DOF (device) or null
        void setup(cudaStream_t s, const DeviceCsr& A_y, const DeviceCsr& Hhat, const AmgOptions& opt, Workspace& w,
                   const int* y_component = nullptr, const int* x_component = nullptr);
        void apply(cudaStream_t s, const double* r, double* z) override;
        // one block's operator alone (block 0: A_y part, 1: Hhat part)
        void apply_block(cudaStream_t s, int block, const double* r, double* z);
        // before a solve (outside any stream capture): with two V-cycles per application,
        // the scale 1 / (1.1 lambda_max(V A)) of each block from a power iteration on the
        // current smoothers
        void prepare(cudaStream_t s, Workspace& w);
        int n_lambda = 0, n_u = 0;
        Amg amg_a, amg_h;
        DeviceCsr hhat_f; // filtered SPD operator the Hhat hierarchy is built on
        static constexpr double kHhatDrop = 0.01;
        int vcycles = 1;
        double scale_a = 1.0, scale_h = 1.0;

    private:
        cudaStream_t side_ = nullptr;
        cudaEvent_t fork_ = nullptr, join_ = nullptr;
        const DeviceCsr* A_y_ = nullptr;
        const DeviceCsr* H_ = nullptr;
        DeviceBuffer<double> t_a_, w_a_, t_h_, w_h_;
    };

    // Independent problems stacked block-diagonally in K: segment 2p covers part p's lambda
    // rows, segment 2p + 1 its u rows (offsets into the full vector).  With a partition the
    // true-residual acceptance uses the largest per-part relative residual.
    struct Partition
    {
        int n_parts = 0;
        DeviceBuffer<int2> segs; // [2 n_parts] (begin, end)
    };

    struct MinresOptions
    {
        double tolerance = 1e-8;
        int max_iterations = 20000;
        int batch = 100; // true_residual_check_interval (0 or negative: no batching)
        const Partition* parts = nullptr;
    };

    struct MinresSummary
    {
        int iterations = 0;
        int batches = 0;
        double backend_error = 0.0;
        bool backend_converged = false;
        double true_residual = 0.0;
        bool converged = false;
        std::vector<double> part_residuals; // per part, with a partition
    };

    MinresSummary minres_solve(cudaStream_t s, const DeviceCsr& K, Preconditioner& P, const double* b, double* x,
                               const MinresOptions& opt, Workspace& w);
}
