// The adaptive driver's G^delta estimator on the device (see apf_gdelta.cu).
#pragma once

#include <vector>

#include "apf_sparse.cuh"
#include "apf_system.hpp"

namespace apf
{
    struct GDeltaResult
    {
        double lambda_difference_squared = 0.0; // ||lambda_G - lambda_delta||^2 in the A_G energy
        double relative_residual = 0.0;         // of the CG solve for lambda_G
        int iterations = 0;
        int n_g = 0;
    };

    // For the solved system S (p = 1): the space G of degree 2 on S's Y cells given by its
    // restriction (host arrays: off [n_y_cells * 18 + 1], dofs, weights; n_g true DOFs).
    GDeltaResult g_delta(cudaStream_t s, System& S, int n_g, const std::vector<int>& off, const std::vector<int>& dofs,
                         const std::vector<double>& w, double tol);
}
