// Equilibrated-flux estimator (see apf_estimator.cu).
#pragma once

#include <vector>

#include "apf_system.hpp"

namespace apf
{
    // Vertex patches of every time slab; patches of slabs with identical spatial meshes
    // share one topology entry.
    struct PatchSet
    {
        int n_slabs = 0;
        int max_cells = 0;
        int max_n = 0;                  // largest patch system (flux + scalar + constraint)
        std::vector<int> slab_ptr;      // slab -> range in slab_cells
        std::vector<int> slab_cells;    // Y cell ids grouped by slab
        std::vector<int> topo_ptr;      // topology patch -> range of patch cells
        std::vector<int> topo_cell;     // local cell index in the slab's cell list
        std::vector<int> topo_center;   // local vertex index of the patch vertex
        std::vector<int> topo_edge;     // 3 per patch cell: free edge id | sign bit 30
        std::vector<int> topo_nfree;
        std::vector<int> topo_boundary;
        std::vector<int> patch_slab;    // patch -> slab
        std::vector<int> patch_topo;    // patch -> topology patch
    };

    struct EstimatorTotals
    {
        double flux = 0.0, div = 0.0, recon = 0.0, eta = 0.0;
        int n_slabs = 0, n_patches = 0, max_patch_cells = 0, recon_iterations = 0;
        double recon_residual = 0.0;
    };

    // times: [n_cells][2] (t0, t1) of every cell; vids: [n_cells][3] spatial vertex ids
    void build_patches(const std::vector<double>& times, const std::vector<int>& vids, int n_cells, PatchSet& ps);

    // Launch-shape autotuner of the patch solves (one per context): for every (degree,
    // precision, patch-size bucket) the first estimate that meets it times the candidate
    // team widths (1, 2, 4 warps per patch) on that bucket's own patches and keeps the
    // fastest; later estimates reuse the choice.
    struct PatchTuner
    {
        bool enabled = true;
        int width[2][2][7] = {};     // [p - 1][FP32][bucket] -> warps per patch (0: not tuned)
        float ms[2][2][7][3] = {};   // candidate times of the tuning launch
        int patches[2][2][7] = {};   // patches in the bucket when it was tuned
    };
    // patch-size buckets (largest system size of each): the patch matrix's shared-memory
    // slice, and so the teams per SM, follows the bucket, so the ladder is fine where the
    // common sizes lie (P1: 29 unknowns at valence-4 vertices, 57 at valence 8)
    constexpr int kPatchBuckets = 7;
    constexpr int kPatchBucketMax[kPatchBuckets] = {30, 40, 48, 58, 64, 96, 144};

    // patch_precision: APF_PATCH_FP64 or APF_PATCH_FP32_REFINED (p = 1)
    EstimatorTotals estimate(cudaStream_t s, System& S, const std::vector<int>& vids_host, double* flux, double* div,
                                double* recon, double* eta, bool out_on_device, int patch_precision = APF_PATCH_FP64,
                                PatchTuner* tuner = nullptr);

    // sigma_x, sigma_y, div sigma (values: [n][3]) of the flux kept by the last estimate
    // (System::keep_flux) at physical points (x, y, t) ([n][3]), point i in estimator cell
    // cell[i] (0 <= cell[i] < S.flux_cells)
    void flux_sample(cudaStream_t s, const System& S, int n, const int* cell, const double* points, double* values,
                     bool on_device);

    // lambda~ of the slab reconstruction: A_y lambda~ = f - B^T u by PCG with the A_y
    // V-cycle from lambda_delta (relative residual 1e-14, at most 400 iterations)
    void reconstruct_lambda(cudaStream_t s, System& S, DeviceBuffer<double>& lt, EstimatorTotals& tot);

    // 1+1D (P1) edge-patch estimator
    EstimatorTotals estimate_1d(cudaStream_t s, System& S, double* flux, double* div, double* recon, double* eta,
                                bool out_on_device);
}
