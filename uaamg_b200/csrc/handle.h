// The C-ABI handle (include/uaamg.h) and the helpers that api.cpp and runtime.cpp
// share: error recording and the mapping of engine errors to uaamg_status.
#pragma once
#include <string>

#include "../../include/uaamg.h"
#include "engine.h"

struct uaamg_handle {
    int device = 0;
    cudaStream_t stream = 0;
    int dirichlet = 0;
    int dim = 0, nx = 0, ny = 0, nz = 0;
    double dx = 1, dy = 1, dz = 1;
    size_t n = 0;
    uint8_t* d_solid = nullptr;
    double* d_rhs = nullptr;  // staging for the host-array entry points
    double* d_p = nullptr;
    double* d_hist = nullptr;
    double* d_face[3] = {nullptr, nullptr, nullptr};  // face velocities of uaamg_project
    double* d_lap[3] = {nullptr, nullptr, nullptr};   // lap_diag, lap_off_x, lap_off_y
    bool lap_on = false;                              // uaamg_set_variable_laplacian
    long lap_version = 0;                             // bumped on every upload
    cudaStream_t copy_stream = nullptr;  // uaamg_solve: p's upload beside the solve
    cudaEvent_t p_ready = nullptr;
    size_t face_n[3] = {0, 0, 0};
    int hist_cap = 0;
    int last_iters = 0;
    uaamg::Engine* eng[3] = {nullptr, nullptr, nullptr};
    bool ready[3] = {false, false, false};
    int sweeps = 0;  // V-cycle kernels (uaamg_set_vcycle_kernels): 0 fused marches +
                     // small-level kernel, 1 sweeps, 2 fused marches on every level,
                     // 3 four marches a level + small-level kernel, 4 four marches on
                     // every level
    int autotune = 0;
    int nu_fine = 1, nu_coarse = 1;  // smoothing sweeps (uaamg_set_smoothing)
    long long batch_group_cells = 0; // batch problems of at most this many padded cells
                                     // share one CUDA graph per step (0: none)
    std::string err;
    struct BatchPool* batch = nullptr;  // runtime.cpp: per-problem slots of uaamg_solve_batch
};

namespace uaamg {
namespace api {

uaamg_status fail(uaamg_handle* h, uaamg_status s, const std::string& msg);
uaamg_status cuda_fail(uaamg_handle* h, cudaError_t e, const char* where);
uaamg_status map_engine(uaamg_handle* h, int e, const char* where,
                        const uaamg::Engine* eng = nullptr);
// uaamg_stats from an engine result (CG_* status mapped to uaamg_status).
uaamg_status fill_stats(const uaamg::Engine* eng, const uaamg::SolveResult& r, uaamg_stats* st);
// Frees the batch slots of a handle (runtime.cpp).
void free_batch(uaamg_handle* h);

// The engine flags of a V-cycle kernel mode (uaamg_set_vcycle_kernels).
inline void apply_vcycle_mode(uaamg::Engine* e, int mode) {
    e->set_vcycle_sweeps(mode == 1);
    e->set_small_levels(mode == 0 || mode == 3);
    e->set_fused(mode == 0 || mode == 2);
}

}  // namespace api
}  // namespace uaamg
