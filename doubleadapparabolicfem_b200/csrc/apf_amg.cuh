// Smoothed-aggregation algebraic multigrid on the device, used as an SPD block
// preconditioner (one symmetric V-cycle = a fixed SPD linear operator, so MINRES
// remains a short-recurrence method).
#pragma once

#include <vector>

#include "apf_sparse.cuh"

namespace apf
{
    struct AmgOptions
    {
        double strength = 0.08;   // strong: |a_ij| >= strength * sqrt(a_ii a_jj)
        int smooth_steps = 2;     // damped-Jacobi sweeps before and after the coarse correction
        int coarse_size = 1024;   // dense solve at or below this size
        int max_levels = 20;
        // levels (from the finest) whose aggregates come from a distance-2 independent set
        // (roots two strong edges apart: larger aggregates, fewer coarse unknowns)
        int aggressive_levels = 0;
        // V-cycles per application in the block preconditioner (1, or 2: the scaled two-step
        // iteration, see BlockPreconditioner::apply)
        int vcycles = 1;
    };

    struct AmgLevel
    {
        DeviceCsr A_own;              // level operator (coarse levels own theirs)
        const DeviceCsr* A = nullptr; // finest level references the caller's matrix
        DeviceCsr P;                  // prolongation (n x n_coarse)
        DeviceCsr R;                  // restriction = P^T
        DeviceBuffer<double> dinv;    // 1 / diag(A)
        double omega = 0.0;           // Jacobi damping 4 / (3 rho(D^-1 A))
        DeviceBuffer<int> comp;       // component of each unknown (empty: one component)
        DeviceBuffer<double> x, b, r, t;
        DeviceBuffer<double> w;       // per-row weights of the first pre-smoothing sweep (empty: omega D^-1)
        DeviceBuffer<double> w2;      // weights of the later pre-smoothing sweeps (empty: w)
        double alpha = 1.0;           // coarse-correction scale
        // f32-valued sliced-ELLPACK copies of A, P, R for the V-cycle's SpMVs
        std::unique_ptr<DeviceSell> A32, P32, R32;
    };

    class Amg
    {
    public:
        // component (optional, device, A.rows values): unknowns of different components are
        // never aggregated together.
        void setup(cudaStream_t s, const DeviceCsr& A, const AmgOptions& opt, Workspace& w,
                   const int* component = nullptr);
        // x = V-cycle(b); x and b are device vectors of the finest size.
        void apply(cudaStream_t s, const double* b, double* x);
        int levels() const { return static_cast<int>(levels_.size()); }
        long long operator_nnz() const;
        std::vector<int> level_rows() const;
        // level access for the learned smoother weights and their training
        AmgLevel& level(int l) { return levels_[static_cast<std::size_t>(l)]; }
        const AmgLevel& level(int l) const { return levels_[static_cast<std::size_t>(l)]; }
        bool dense_coarse() const { return !jacobi_coarse_; }
        int smooth_steps() const { return opt_.smooth_steps; }
        const double* coarse_inverse() const { return coarse_inv_.get(); }
        static constexpr int coarse_sweeps() { return kCoarseSweeps; }
        // Replace level l's Jacobi weights omega D^-1 by per-row weights (device, moved in):
        // w for the first pre-smoothing sweep, w2 for the later ones (post-smoothing runs the
        // same weights in reverse order), and scale its coarse correction by alpha; the
        // V-cycle stays symmetric.
        void set_smoother(int l, DeviceBuffer<double>&& w, DeviceBuffer<double>&& w2, double alpha);
        // back to omega D^-1 and alpha = 1 on every level
        void reset_smoothers();
        // x = the coarsest level's solve of b (dense inverse or fixed Jacobi sweeps; a
        // symmetric linear map)
        void coarse_apply(cudaStream_t s, const double* b, double* x) { vcycle(s, levels() - 1, b, x); }

    private:
        // first_done: the caller already wrote level l's first damped-Jacobi iterate from
        // zero (a restriction fused with it)
        void vcycle(cudaStream_t s, int l, const double* b, double* x, bool first_done = false);
        double* first_iterate(int l, double* x);
        std::vector<AmgLevel> levels_;
        DeviceBuffer<double> coarse_inv_; // dense inverse of the coarsest operator, row-major
        int n_coarse_ = 0;
        bool jacobi_coarse_ = false;      // coarsest level smoothed only (too large for a dense solve)
        static constexpr int kCoarseSweeps = 8;
        static constexpr int kMaxDense = 1500; // largest coarsest level inverted densely (device Gauss-Jordan, n launches)
        AmgOptions opt_{};
    };
}
