// Learned smoother weights for the AMG V-cycle blocks of the MINRES preconditioner.
//
// A small MLP maps scale-free features of each matrix row (per AMG level, per block) to
// multiplicative corrections of the plain damped-Jacobi weight, one per smoothing sweep
// class (the first sweep, and the later ones), and per-level logits give the
// coarse-correction scale:
//   w_i^(o) = omega_l / a_ii * exp(kWeightRange * tanh(y_i^(o))),  y_i = MLP(f_i), o = 0, 1
//   alpha_l = 2 sigmoid(theta_{block,l})
// Pre-smoothing sweep k uses w^(min(k,1)); post-smoothing runs the same weights in reverse
// order, so the V-cycle stays symmetric (each sweep's error propagation I - W A is
// A-self-adjoint and the post-smoother is the A-adjoint of the pre-smoother) and the
// preconditioner remains a fixed SPD operator for MINRES; a symmetric Gershgorin bound
// rescales each weight vector when needed so that every sweep stays convergent whatever
// the network outputs.
#pragma once

#include "apf_minres.cuh"

namespace apf
{
    namespace learned
    {
        constexpr int kFeatures = 8;
        constexpr int kHidden = 32;
        constexpr int kOutputs = 2; // weight of the first sweep, weight of the later sweeps
        constexpr int kMaxLevels = 16;
        constexpr float kWeightRange = 0.5f;
        constexpr double kSmootherBound = 1.9; // max symmetric Gershgorin row sum of W^1/2 A W^1/2
        // flat FP32 parameter layout
        constexpr int kW1 = 0;                         // [kHidden][kFeatures]
        constexpr int kB1 = kW1 + kHidden * kFeatures; // [kHidden]
        constexpr int kW2 = kB1 + kHidden;             // [kHidden][kHidden]
        constexpr int kB2 = kW2 + kHidden * kHidden;   // [kHidden]
        constexpr int kW3 = kB2 + kHidden;             // [kOutputs][kHidden]
        constexpr int kB3 = kW3 + kOutputs * kHidden;  // [kOutputs]
        constexpr int kAlpha = kB3 + kOutputs;         // [2][kMaxLevels]
        constexpr int kParams = kAlpha + 2 * kMaxLevels;
        static_assert(kParams == APF_LEARNED_NUM_PARAMS, "parameter count of the C ABI");
    }

    struct LearnedModel
    {
        std::vector<float> params = std::vector<float>(learned::kParams, 0.0f);
    };

    // Row features of a level operator: f[i][0..7] (FP32, row-major), see apf_learned.cu.
    void learned_features(cudaStream_t s, const DeviceCsr& A, const double* dinv, int level, int block, float* feat);

    // y[i][0..1] = MLP(f_i): precision 0 = FP32 on the CUDA cores, 1 = BF16 operands with
    // FP32 accumulation on the tensor cores (mma.sync m16n8k16).  params: device, FP32.
    void learned_forward(cudaStream_t s, const float* params, int n, const float* feat, float* y, int precision);

    // Install the learned weights on every non-coarsest level of amg (block 0 = A_y, 1 = Hhat);
    // params: host copy of the model.
    void apply_learned_smoothers(cudaStream_t s, const LearnedModel& model, Amg& amg, int block);

    // Loss of the stationary V-cycle iteration of both blocks and its gradient with respect to
    // the model parameters:
    //   L = sum_block mean_sample (1/k) log(||E^k e||_T^2 / ||e||_T^2),  E = I - V T
    // with T the block the V-cycle stands for (target_a = A_y, target_h = Hhat), k = steps,
    // and e = E^burn_in e0 (burn-in without gradient: the loss then measures the slowly
    // contracting modes, the ones that set the preconditioned spectrum's spread).
    // start vectors: device, [samples][n_lambda + n_u] (lambda part, then u part), or null
    // for seeded normal vectors.  grad (host, kParams floats) may be null.  Leaves the
    // FP32-model weights installed in P's V-cycles.
    double learned_loss_and_grad(cudaStream_t s, const LearnedModel& model, BlockPreconditioner& P,
                                 const DeviceCsr& target_a, const DeviceCsr& target_h, int samples, int steps,
                                 int burn_in, unsigned long long seed, const double* start_vectors, float* grad,
                                 Workspace& w);
}
