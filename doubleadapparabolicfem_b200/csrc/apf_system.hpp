// Device-resident problem inputs and assembled system (internal).
#pragma once

#include <atomic>
#include <memory>

#include "apf_internal.hpp"
#include "apf_minres.cuh"

namespace apf
{
    // local-block kinds of the row gather
    enum Kind : int
    {
        K_AY = 0,   // rows Y, cols Y, cells Y
        K_BT = 1,   // rows Y, cols X (ancestor), cells Y: B(j, i)
        K_B = 2,    // rows X (ancestor), cols Y, cells Y
        K_C = 3,    // rows X, cols X, cells bottom X
        K_AX = 4,   // rows X, cols X, cells X
        K_BDT = 5,  // as K_B, time-derivative part only
        K_BDTT = 6, // as K_BT, time-derivative part only
    };

    // true DOF -> list of (cell*ndof + local, restriction entry)
    struct Incidence
    {
        DeviceBuffer<int> ptr;
        DeviceBuffer<int2> entries;
        int max_len = 0;
    };

    struct SystemInputs
    {
        int p = 1, ndof = 6;
        int dim = 2; // space dimension: 2 (prisms, geometry rows of 8) or 1 (quads, rows of 4)
        int n_y_cells = 0, n_x_cells = 0, n_lambda = 0, n_u = 0;
        DeviceBuffer<double> y_geo, x_geo;
        DeviceBuffer<int> y_to_x;
        DeviceBuffer<int> y_off, y_dofs, x_off, x_dofs;
        DeviceBuffer<double> y_w, x_w;
        DeviceBuffer<double> m_y, m_x, ell;
        DeviceBuffer<int> bottom_list;
        int n_bottom = 0;
        int kmax = 1;
        int u0_kind = 0;
        double zero_tol = 1e-15, g_scale = -1.0;
    };

    struct System
    {
        cudaStream_t stream = nullptr;
        SystemInputs in;
        Incidence inc_y, inc_xy, inc_xb, inc_x;
        DeviceCsr blocks[APF_N_BLOCKS];
        bool have[APF_N_BLOCKS] = {};
        DeviceBuffer<double> f, g;
        DeviceBuffer<double> inv_diag_ay;
        // solve state
        Workspace ws;
        std::unique_ptr<BlockPreconditioner> precond;
        AmgOptions precond_opts{};
        DeviceBuffer<double> rhs, solution;
        double precond_setup_seconds = 0.0;
        int precond_kind = -1;                    // APF_PRECOND_* installed in precond's V-cycles
        unsigned long long precond_model_version = 0; // learned model the weights came from
        Partition partition;                 // stacked independent problems (apf_system_set_partition)
        std::vector<double> part_residuals;  // per-part true relative residuals of the last solve
        // the equilibrated flux of the last 2+1D estimate, kept when keep_flux is set: per
        // estimator cell (the Y cells, or the slab cells they are cut into) the flux
        // coefficients of its three vertex-patch slots, its geometry, time slab and source Y cell
        bool keep_flux = false;
        int flux_p = 0, flux_cells = 0;
        DeviceBuffer<double> flux_sigma, flux_geo;
        std::vector<int> flux_slab, flux_source;
    };

    void upload_tables_once(int device);
    // quantized time coordinate of every Y (y_space) or X DOF: the AMG coarsens each time
    // level separately (its low-energy modes are arbitrary in time, smooth in space)
    void dof_time_components(cudaStream_t s, const SystemInputs& in, bool y_space, DeviceBuffer<int>& comp);
    void prepare_inputs(cudaStream_t s, SystemInputs& in);
    // per Y cell: v_K^T A_y,K v_K, the local A_y energy (int_K grad_x v . M grad_x v) of a
    // Y-space true-DOF vector v (device)
    void y_cell_energy(cudaStream_t s, const SystemInputs& in, const double* v, double* out);
    // dst[c][k] (n cells, ndof nodal values each) = the local function src[src_index[c]] of
    // a source prism (geometry src_geo) evaluated at the nodes of prism c (geometry dst_geo),
    // which lies inside it; src_index NULL = identity.  Exact for nested prisms.
    void nodal_transfer(cudaStream_t s, int p, int n, const double* dst_geo, const int* src_index, const double* src_geo,
                        const double* src, double* dst);
    // true-DOF values of a degree-q space (restriction off/dofs/w on n cells of geometry
    // dst_geo) interpolating the degree-p function v (true DOFs through the restriction
    // soff/sdofs/sw of the source cells src_index[c] (NULL = c), geometry src_geo) at its
    // nodes; each DOF is written from its first unconstrained occurrence (deterministic).
    // Exact when the source function lies in the degree-q space (nested cells, p <= q).
    void interpolate_to_space(cudaStream_t s, int q, int p, int n, const double* dst_geo, const int* src_index,
                              const double* src_geo, const int* soff, const int* sdofs, const double* sw,
                              const double* v, const int* off, const int* dofs, const double* w, int n_true,
                              double* out);
    // out[c] = v_c^T A_c v_c: the local A_y energy (int grad_x v . M grad_x v) of nodal values
    // v_c on prism c (m: 3 per cell or NULL = identity)
    void nodal_energy(cudaStream_t s, int p, int n, const double* geo, const double* m, const double* v, double* out);
    // X-marking indicators from lambda_delta (Y true DOFs) and u_delta (X true DOFs), all
    // device arrays: per Y cell lambda energy, per X cell its aggregate, the initial-trace
    // mismatch (0 off the t = 0 layer) and their sum
    void x_indicators(cudaStream_t s, const SystemInputs& in, const double* lambda, const double* u, double* lam_y,
                      double* lam_x, double* trace_x, double* eta_x);
    Incidence build_incidence(cudaStream_t s, int n_dofs, int n_asm, const int* cell_list, const int* src_map,
                              const int* offsets, const int* dofs, int ndof);
    void gather_csr(cudaStream_t s, const SystemInputs& in, double zero_tol, int n_rows, int n_cols, int n_terms,
                    const int* kinds, const Incidence* const* incs, const int* col_offsets, int kmax, DeviceCsr& out);
    void gather_vector_host(cudaStream_t s, const SystemInputs& in, double zero_tol, int which, const Incidence& inc,
                            int n_rows, const double* ell, int u0_kind, double g_scale, DeviceBuffer<double>& out);
    void build_k(cudaStream_t s, int n_lambda, int n_u, const DeviceCsr& a, const DeviceCsr& bt, const DeviceCsr& b,
                 const DeviceCsr& c, DeviceCsr& k);
    // Two-pass full saddle assembly (the direct-solver path's K = [A_y B^T; B C_signed]):
    // the structural pattern (union of the restricted couplings, no value filter), then
    // the numeric pass into that pattern and the prune of |value| <= zero_tol
    void full_saddle_pattern(cudaStream_t s, const SystemInputs& in, const Incidence& inc_y, const Incidence& inc_xy,
                             const Incidence& inc_xb, DeviceBuffer<int>& row_ptr, DeviceBuffer<int>& col_idx);
    void full_saddle_numeric(cudaStream_t s, const SystemInputs& in, const Incidence& inc_y, const Incidence& inc_xy,
                             const Incidence& inc_xb, const int* row_ptr, const int* col_idx, long long nnz_pattern,
                             DeviceCsr& K);
    void build_hhat(cudaStream_t s, const DeviceCsr& A_y, const DeviceCsr& C, const DeviceCsr& A_x, const DeviceCsr& B_dt,
                    const DeviceCsr& B_dtT, double diag_tol, DeviceCsr& H, DeviceBuffer<double>& inv_diag);

    // ||b - K x||_2 and ||b - K x||_2 / ||b||_2 with no device allocation (apf_noalloc.cu)
    void true_residual_noalloc(int device, cudaStream_t s, int rows, const int* row_ptr, const int* col_idx,
                               const double* values, const double* x, const double* b, double* absolute,
                               double* relative);

    // assembly drivers (apf_capi.cu)
    void assemble_main(System& sys);
    void assemble_graph_norm(System& sys, double diag_tol);
}
