// Host-side interface between the C-ABI layer (api.cpp) and the per-precision
// engines (kernels_f64.cu, kernels_f32.cu).  No CUDA device code here.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace uaamg {

// Engine precision modes (match uaamg_precision in include/uaamg.h).
enum Precision : int { PREC_FP64 = 0, PREC_FP32 = 1, PREC_MIXED = 2 };

struct SolveArgs {
    const double* rhs;   // device, padded FP64 right-hand side of  lap(p) = rhs
    double* x;           // device, padded FP64 pressure: in = accumulate target / warm start
    int max_iter;
    double tol;
    int tol_mode;        // 0 absolute (the reference), 1 relative to ||b||
    int warm;            // 1: r0 = b - A x_in
    int replace_every;   // mixed: residual replacement period (iterations)
    int project_mean;    // subtract the fluid mean of the result (FP64)
    int precond;         // 1 UAAMG V-cycle, 0 identity (plain CG)
    double* hist;        // optional device array, max_iter+1: ||r_k|| per update
    const uint8_t* ref_solid;  // the caller's mask (reference layout), for project_mean
    cudaEvent_t x_ready = nullptr;  // optional: x holds its input once this event completes
                                    // (waited on just before x is first read)
};

struct SolveResult {
    int status;          // CG_* (common.cuh)
    int iterations;
    int replacements;
    double rr;           // recursive r.r at exit
    double rr_true;      // FP64 ||b - A x||^2 at exit
    double bnorm;        // ||b||
    double r0;           // ||r0||
    double tol_abs;
};

// Error codes returned by engine calls (0 = success), mapped to uaamg_status
// by the C-ABI layer.
enum EngineError : int { E_OK = 0, E_OOM = 1, E_CUDA = 2, E_ARG = 3, E_NOPROB = 4 };

// Aggregated in-situ timing of one kernel class on one level.
struct KernelTime {
    int cls;
    const char* name;
    int level;
    int launches;
    double total_ms;
    double bytes;  // algorithmic bytes per launch
};

class Engine {
public:
    virtual ~Engine() {}
    // The CUDA error behind the last E_CUDA result (cudaSuccess when none).
    cudaError_t cuda_error = cudaSuccess;
    // Builds the level hierarchy for a padded level-0 mask already on the device.
    virtual int set_problem(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                            const uint8_t* d_solid, int dirichlet) = 0;
    // z = M^{-1} r (one V(1,1) cycle); FP64 device arrays, padded.
    virtual int precond_apply(const double* d_r, double* d_z) = 0;
    virtual int solve(const SolveArgs& a, SolveResult* res) = 0;
    // The solve in stages, for engines that share the GPU (batch, serving):
    // begin queues the set-up and the first preconditioner application; step
    // queues two iterations; poll reports whether the device has stopped (wait:
    // block on the oldest queued step); end queues the output and blocks for the
    // result.  All on the engine's stream.
    virtual int solve_begin(const SolveArgs& a) = 0;
    virtual int solve_step() = 0;
    virtual int solve_poll(bool wait, bool* stopped) = 0;
    virtual int solve_inflight() const = 0;
    virtual int solve_end(SolveResult* res) = 0;
    // solve_end in two halves for a caller that must not block: enqueue queues the
    // exit work (FP64 true residual, solution export, state copy) on the engine's
    // stream; collect reads the result once that work has completed (e.g. after an
    // event recorded behind it reports done), and then does not wait.
    virtual int solve_end_enqueue() = 0;
    // After solve_begin: queue one step (two PCG iterations) on stream s, without a
    // graph, then copy the device 'done' flag into flag_dst (pinned host memory).
    // For capturing the steps of many engines into one CUDA graph (batches); the
    // engine's own step bookkeeping (solve_step / solve_poll) is not used then.
    virtual int enqueue_step(cudaStream_t s, int* flag_dst) = 0;
    virtual int solve_end_collect(SolveResult* res) = 0;
    virtual int nlevels() const = 0;
    virtual void level_dims(int l, int* nx, int* ny, int* nz) const = 0;
    // Host copies of level l: mask and FP64 views of cx, cy, cz (nullable).
    virtual int copy_level(int l, uint8_t* solid, double* cx, double* cy, double* cz) = 0;
    // boxes of level l run by the whole-tile box kernels, and how many are trimmed
    virtual int level_trim(int l, int* boxes, int* trimmed) = 0;
    virtual void set_stream(cudaStream_t s) = 0;
    virtual size_t device_bytes() const = 0;
    // Number of kernel launches issued by the last solve() (for launch accounting).
    virtual long launches() const = 0;
    // V-cycle as per-colour sweep kernels (the cross-check) instead of the fused kernels.
    virtual void set_vcycle_sweeps(bool on) = 0;
    // Marches: run the small levels and the coarsest solve as one single-block
    // kernel (default on; off: marches on every level).
    virtual void set_small_levels(bool on) = 0;
    // Marches: two fused marches per level (fused.cuh: down = forward sweep, residual
    // and restriction; up = prolongation and reverse sweep) instead of four
    // (march.cuh).  Default on.
    virtual void set_fused(bool on) = 0;
    // Pre- and post-smoothing sweeps on the finest level and on the coarse levels
    // (V(nu, nu) cycles; the reference's V(1,1) is 1, 1, the default).  More than one
    // sweep runs the four-march level with the extra sweeps as colour-sweep kernels.
    virtual void set_smoothing(int fine, int coarse) = 0;
    // 2D variable-coefficient outer-CG operator (the lap_diag / lap_off_x / lap_off_y
    // branch of PCG::solve, pcg.cpp:35-46): device arrays in the caller's padded
    // layout with row stride sx, read in place by every solve until changed;
    // nullptr: the uniform operator.  The V-cycle keeps its own couplings.  version
    // changes whenever the arrays' contents do (the FP32 forms keep converted copies).
    virtual void set_operator(const double* d, const double* ox, const double* oy, int sx,
                              long version) = 0;
    // Replay each pair of PCG iterations as one CUDA graph (default on).
    virtual void set_graphs(bool on) = 0;
    // 1: the next set_problem times each level's marches for a few z-chunk lengths
    // and keeps the fastest (cached per level shape for the process).
    virtual void set_autotune(bool on) = 0;
    // Per-launch CUDA-event timing of subsequent solves (adds two events per launch).
    virtual void set_profiling(bool on) = 0;
    virtual int profile_results(std::vector<KernelTime>& out) = 0;
    // Non-zero if a kernel of the last call gave up waiting for its TMA loads.
    virtual int timed_out() = 0;
};

// The autotuner's persistent choices (tunecache.cpp): an id of the current GPU, and
// lookup / store of integer lists by key (in memory; also in the JSON file set by
// uaamg_set_tune_cache).
std::string tune_gpu_id();
bool tune_lookup(const std::string& key, std::vector<int>* val);
void tune_store(const std::string& key, const std::vector<int>& val);

Engine* create_engine_f64();
Engine* create_engine_f32(int mixed);

}  // namespace uaamg
