/* uaamg.h -- C-ABI of the B200-native UAAMG-preconditioned CG pressure solver.
 *
 * Drop-in boundary for the reference's pressure-solve path (A-006/UAAMGPCG):
 * a host C++ Solver / Solver3D subclass (or any FFI) calls these functions in
 * place of PCG(UAAMGPreconditioner)::solve.  Plain pointers and sizes only.
 *
 * Data contract (the reference's, include/core/mesh.h:30-35, mesh_3d.h:38):
 * every cell array is ghost-padded and column-major with i fastest,
 *   2D: (nx+2)*(ny+2) cells, id = i + j*(nx+2)
 *   3D: (nx+2)*(ny+2)*(nz+2) cells, id = i + j*(nx+2) + k*(nx+2)*(ny+2)
 * interior cells are 1..nx etc.  The solid mask is one byte per padded cell
 * (non-zero = solid), the expansion of Grid::solid (std::vector<bool>) that the
 * reference's GPU adapter uploads (src/solver/cuda/cuda_pcg_solver.cu:45-49).
 *
 * Sign and null-space convention: identical to PCG::solve (src/solver/pcg.cpp:
 * 18-33, pcg_3d.cpp:18-36): the solver solves lap(p) = rhs on fluid cells with
 * Neumann walls and solids, after removing the fluid mean of rhs; the pressure is
 * accumulated into p (callers zero it first, src/pressure/pressure.cpp:17).
 *
 * Every call returns a uaamg_status; none prints or aborts.  A handle is not
 * thread-safe: one host thread per handle (as the reference's per-object GPU
 * buffers, include/solver/cuda/cuda_pcg_3d.h:36-40).  All GPU work of a handle is
 * issued on its stream (uaamg_set_stream; default: the legacy default stream).
 */
#ifndef UAAMG_H
#define UAAMG_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define UAAMG_API __attribute__((visibility("default")))
#else
#define UAAMG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum uaamg_status {
    UAAMG_OK = 0,             /* converged (or operation succeeded) */
    UAAMG_NOT_CONVERGED = 1,  /* max_iter reached; result is the last iterate */
    UAAMG_BREAKDOWN = 2,      /* p.Ap below the breakdown threshold (pcg.cpp:100) */
    UAAMG_NAN = 3,            /* a NaN/Inf appeared in a reduction */
    UAAMG_OOM = 4,            /* device allocation failed */
    UAAMG_INVALID_ARG = 5,
    UAAMG_CUDA_ERROR = 6,
    UAAMG_TIMEOUT = 7,        /* reserved for bounded device waits */
    UAAMG_NO_PROBLEM = 8      /* solve before uaamg_set_problem_* */
} uaamg_status;

typedef enum uaamg_precision {
    UAAMG_FP64 = 0,   /* reference-exact: FP64 everywhere (CudaPCG3D::solve analogue) */
    UAAMG_FP32 = 1,   /* plain FP32 PCG: FP32 vectors and V-cycle, FP64 reductions */
    UAAMG_MIXED = 2   /* FP32 CG + FP32 V-cycle, FP64 reductions, FP64 solution with
                         true-residual replacement every replace_every iterations */
} uaamg_precision;

typedef enum uaamg_tol_mode {
    UAAMG_TOL_ABS = 0, /* stop when sqrt(r.r) < tol (PCG::solve, pcg.cpp:111-112) */
    UAAMG_TOL_REL = 1  /* stop when sqrt(r.r) < tol * ||b||, b the normalised RHS */
} uaamg_tol_mode;

typedef struct uaamg_options {
    int precision;      /* uaamg_precision, default UAAMG_FP64 */
    int tol_mode;       /* uaamg_tol_mode, default UAAMG_TOL_ABS */
    int max_iter;       /* default 2000 (Config::solve_iters, include/config/config.h:30) */
    double tol;         /* default 1e-6 (Config::solve_tol, config.h:31) */
    int warm_start;     /* 0: r0 = b and p is accumulated into (the reference);
                           1: r0 = b - A p_in, the result is p_in + correction */
    int replace_every;  /* UAAMG_MIXED residual-replacement period, default 10 */
    int project_mean;   /* 1: subtract the fluid mean of the result in FP64 */
    int preconditioner; /* 1: UAAMG V(1,1) (Factory key "pcg_uaamg"); 0: identity ("cg") */
} uaamg_options;

typedef struct uaamg_stats {
    int status;                 /* uaamg_status of the solve */
    int iterations;             /* x/r updates performed */
    int replacements;           /* FP64 residual replacements (UAAMG_MIXED) */
    int levels;                 /* multigrid levels */
    double residual;            /* FP64 true ||b - A p|| at exit (fluid cells) */
    double rel_residual;        /* residual / ||b|| */
    double recursive_residual;  /* the CG's recursive ||r|| at exit */
    double rhs_norm;            /* ||b|| */
    double solve_ms;            /* wall time of the call, host clock */
    long long kernel_launches;  /* kernels launched by the call */
} uaamg_stats;

typedef struct uaamg_handle uaamg_handle;

/* Fills *o with the defaults above. */
UAAMG_API void uaamg_default_options(uaamg_options* o);

/* Creates a solver handle on CUDA device `device`.  Replaces construction of
 * CudaPCGSolver / CudaPCGSolver3D (include/solver/cuda_pcg_solver.h:14-32,
 * cuda_pcg_solver_3d.h:14-32). */
UAAMG_API uaamg_status uaamg_create(uaamg_handle** out, int device);
UAAMG_API uaamg_status uaamg_destroy(uaamg_handle* h);

/* Work stream of the handle (a cudaStream_t passed as void*). */
UAAMG_API uaamg_status uaamg_set_stream(uaamg_handle* h, void* stream);

/* Problem (grid + solid mask) set-up: builds the level masks and Galerkin
 * coefficients on the device for every precision, once per mask.  Replaces the
 * per-apply set-up of UAAMGPreconditioner[3D]::apply (uaamg_preconditioner.cpp:
 * 183-189, uaamg_preconditioner_3d.cpp:205-214) and the GPU adapter's mask
 * upload (cuda_pcg_solver.cu:27-49).  `solid` is a HOST byte mask (padded). */
UAAMG_API uaamg_status uaamg_set_problem_2d(uaamg_handle* h, int nx, int ny, double dx, double dy,
                                  const uint8_t* solid);
UAAMG_API uaamg_status uaamg_set_problem_3d(uaamg_handle* h, int nx, int ny, int nz, double dx,
                                  double dy, double dz, const uint8_t* solid);
/* Same, mask already on the device. */
UAAMG_API uaamg_status uaamg_set_problem_device(uaamg_handle* h, int dim, int nx, int ny, int nz,
                                      double dx, double dy, double dz,
                                      const uint8_t* d_solid);
/* Variable-coefficient Laplacian for the outer CG, 2D (Grid::init_variable_lap and
 * Grid::lap_diag / lap_off_x / lap_off_y, include/core/grid.h:23-31,
 * src/core/grid.cpp:12-17, as PCG::solve applies them, src/solver/pcg.cpp:35-46):
 * padded (nx+2)(ny+2) FP64 HOST arrays, copied to the device.  Every later solve of
 * the current problem (uaamg_solve*, uaamg_project*, uaamg_static_pressure*) uses
 *   A v = lap_diag v_C + lap_off_x (v_L + v_R) + lap_off_y (v_B + v_T)
 * on fluid cells (a solid or out-of-domain neighbour reads v_C; solid rows 0) for its
 * search directions and FP64 residuals; the UAAMG V-cycle keeps its uniform
 * couplings, as the reference's does.  All three NULL: back to the uniform
 * operator.  uaamg_solve_batch and the server keep the uniform operator.  UAAMG_INVALID_ARG for a 3D problem (Grid3D has no such arrays) or when
 * only some are NULL; UAAMG_NO_PROBLEM before uaamg_set_problem_*, which clears the
 * coefficients. */
UAAMG_API uaamg_status uaamg_set_variable_laplacian(uaamg_handle* h, const double* lap_diag,
                                          const double* lap_off_x,
                                          const double* lap_off_y);
/* Cell-centred Dirichlet p = 0 on every domain wall instead of Neumann (the
 * standalone Ax=b check of test/solver/test_amgpcg.cpp:29-70, on the MAC grid).
 * Takes effect at the next uaamg_set_problem_*. */
UAAMG_API uaamg_status uaamg_set_dirichlet_walls(uaamg_handle* h, int on);

/* V-cycle kernels of this handle: 0 (default) = z marches, two per level (the way
 * down: forward sweep, residual and restriction; the way up: prolongation and the
 * reverse sweep), each streaming the level's planes through TMA-filled shared
 * memory, down to the first level of at most 1024 cells; that level, the smaller
 * ones and the coarsest solve run as ONE single-block kernel with the levels in
 * shared memory;
 * 1 = one kernel per colour sweep, restriction and prolongation, step by step as
 * UAAMGPreconditioner3D::vCycle (uaamg_preconditioner_3d.cpp:183-196);
 * 2 = the two-march levels on every level and a separate coarsest-level kernel;
 * 3 = as 0 with four marches per level (forward sweep; residual + restriction;
 * prolongation + even colour; odd colour);
 * 4 = four marches per level on every level and a separate coarsest-level kernel.
 * All give identical results in FP64; 1 to 4 exist to cross-check 0. */
UAAMG_API uaamg_status uaamg_set_vcycle_kernels(uaamg_handle* h, int sweeps);

/* Smoothing schedule of this handle's V-cycle: pre- and post-smoothing sweeps (1 to 4)
 * on the finest level and on the coarse levels, i.e. V(nu, nu) cycles; 1, 1 (default)
 * is the reference's V(1,1) (UAAMGPreconditioner3D::vCycle, uaamg_preconditioner_3d.cpp:
 * 183-196; its CUDA path fixes NU = 1, cuda_uaamg_preconditioner_3d_opt_f.cu:444).  More
 * sweeps make a different (still symmetric) preconditioner; the batch autotuner
 * (uaamg_set_autotune) may choose them per problem class.  Takes effect at the next
 * solve. */
UAAMG_API uaamg_status uaamg_set_smoothing(uaamg_handle* h, int sweeps_fine, int sweeps_coarse);

/* Solve lap(p) = rhs with HOST FP64 arrays (padded): the Solver::solve /
 * Solver3D::solve drop-in (include/solver/solver.h:18-34, solver_3d.h:7-12;
 * CudaPCGSolver::solve, cuda_pcg_solver.cu:21-63).  Host<->device copies are
 * part of the call.  opts may be NULL (defaults); stats may be NULL. */
UAAMG_API uaamg_status uaamg_solve(uaamg_handle* h, const double* rhs, double* p,
                         const uaamg_options* opts, uaamg_stats* stats);

/* Same with DEVICE FP64 arrays (CudaPCG3D::solve_optimized's device-pointer
 * form, include/solver/cuda/cuda_pcg_3d.h:10-13). */
UAAMG_API uaamg_status uaamg_solve_device(uaamg_handle* h, const double* d_rhs, double* d_p,
                                const uaamg_options* opts, uaamg_stats* stats);

/* Pressure projection with DEVICE arrays: the PressureProjection::project /
 * PressureProjection3D::project drop-in (src/pressure/pressure.cpp:5-33,
 * pressure_3d.cpp:5-40) run on the GPU around the solve.  rhs = div(u)/dt on fluid
 * interior cells (fvc::divergence, include/core/grid.h:44-47), p = 0 (kept as the
 * initial guess when opts->warm_start), the solve as uaamg_solve_device, then
 * u -= dt * grad p on every face between two fluid cells (pressure.cpp:21-32,
 * pressure_3d.cpp:21-39).  FP64 face arrays, i fastest: d_u (nx+1)(ny+2)[(nz+2)],
 * d_v (nx+2)(ny+1)[(nz+2)], d_w (nx+2)(ny+2)(nz+1) (3D; NULL in 2D); d_p padded
 * cells.  Divergence and corrected velocities are the reference's FP64 expressions,
 * bit for bit.  Returns the solve's status; as in the reference, the velocities are
 * corrected whatever the solve's outcome (not after an argument or CUDA error). */
UAAMG_API uaamg_status uaamg_project_device(uaamg_handle* h, double dt, double* d_u, double* d_v,
                                  double* d_w, double* d_p, const uaamg_options* opts,
                                  uaamg_stats* stats);

/* The same with HOST arrays (the velocities and p are copied in and out). */
UAAMG_API uaamg_status uaamg_project(uaamg_handle* h, double dt, double* u, double* v, double* w,
                           double* p, const uaamg_options* opts, uaamg_stats* stats);

/* Static pressure recovery with DEVICE arrays: the
 * PressureProjection::recoverStaticPressure drop-in (src/pressure/pressure.cpp:35-66;
 * the second pressure solve of each LFM cycle, src/lfm/lfm_simulator.cpp:199), 2D:
 * rhs = -(du/dx^2 + 2 du/dy dv/dx + dv/dy^2) from cell-centre velocities (cross
 * derivatives dropped next to solids), p = 0, then the solve as uaamg_solve_device on
 * the current problem's hierarchy.  d_u (nx+1)(ny+2), d_v (nx+2)(ny+1), d_p padded;
 * the right-hand side is the reference's FP64 expression, bit for bit. */
UAAMG_API uaamg_status uaamg_static_pressure_device(uaamg_handle* h, const double* d_u,
                                          const double* d_v, double* d_p,
                                          const uaamg_options* opts, uaamg_stats* stats);

/* The same with HOST arrays (u and v copied in, p out). */
UAAMG_API uaamg_status uaamg_static_pressure(uaamg_handle* h, const double* u, const double* v,
                                   double* p, const uaamg_options* opts, uaamg_stats* stats);

/* One V(1,1) cycle z = M^{-1} r with HOST FP64 arrays: the
 * Preconditioner[3D]::apply drop-in (include/solver/preconditioner/
 * preconditioner_3d.h:18-33, UAAMGPreconditioner3D::apply). */
UAAMG_API uaamg_status uaamg_precond_apply(uaamg_handle* h, int precision, const double* r, double* z);

/* Residual history of the last solve: hist[k] = ||r_k|| for k = 0..iterations
 * (recursive residual; hist[0] = ||r0||).  n = capacity. */
UAAMG_API uaamg_status uaamg_residual_history(uaamg_handle* h, double* hist, int n);

/* Hierarchy inspection (bit-exact parity checks): number of levels, level dims,
 * and host copies of level l's padded mask and couplings (FP64 values of the
 * given precision's hierarchy; cz ignored in 2D; any pointer may be NULL). */
UAAMG_API uaamg_status uaamg_num_levels(uaamg_handle* h, int* nlevels);
UAAMG_API uaamg_status uaamg_level_dims(uaamg_handle* h, int l, int* nx, int* ny, int* nz);
UAAMG_API uaamg_status uaamg_copy_level(uaamg_handle* h, int precision, int l, uint8_t* solid,
                              double* cx, double* cy, double* cz);
/* Trimming of level l (3D levels of at most 64^3 cells, run as whole 8^3-tile boxes):
 * *boxes = the level's boxes (0 on other levels), *trimmed = those whose tile and
 * 2-cell ring are interior fluid with one diagonal and one coupling per axis, which
 * the box kernels run without loading diagonals, couplings or codes (the reference's
 * tile trimming, cuda_uaamg_preconditioner_3d.cu:81-99 and :357-375; results are
 * identical either way).  UAAMG_NO_TRIM=1 in the environment turns trimming off for
 * engines created afterwards. */
UAAMG_API uaamg_status uaamg_level_trim(uaamg_handle* h, int precision, int l, int* boxes,
                                        int* trimmed);

/* In-situ kernel timing: runs uaamg_solve_device with a CUDA event pair around
 * every kernel launch and returns, per (kernel class, level), the launch count,
 * total device time and algorithmic bytes per launch (the compulsory traffic the
 * roofline is computed from).  Up to cap entries are written; *count receives
 * the number available.  The extra events make this solve slightly slower than
 * an unprofiled one.  (No reference counterpart: the reference times whole
 * solves with host clocks, src/solver/cuda/test_paper_bench.cu:21-28.) */
typedef struct uaamg_kernel_time {
    char name[32];
    int level;
    int launches;
    double total_ms;
    double bytes_per_launch;
} uaamg_kernel_time;
UAAMG_API uaamg_status uaamg_profile_solve(uaamg_handle* h, const double* d_rhs, double* d_p,
                                           const uaamg_options* opts, uaamg_stats* stats,
                                           uaamg_kernel_time* out, int cap, int* count);

/* Allocation-free residual check, for callers that cannot call cudaMalloc:
 * code running during CUDA-graph stream capture, inside host callbacks or
 * allocator hooks, or in applications that own every device allocation.  No
 * handle, no allocation: d_out[0] = ||b - A p|| and d_out[1] = ||b|| (FP64,
 * fluid interior cells), b = -(rhs - mean_fluid(rhs)) as PCG::solve forms it and
 * A the PCG operator with Neumann walls and solids.  All arrays are DEVICE
 * arrays in the padded reference layout; d_out holds 2 doubles.  Work is queued
 * on `stream` (a cudaStream_t) and the call returns without waiting.
 * Scratch is a 16.4 KiB file-scope device array (held by every GPU that loads the
 * library until exit); grids of 2^31 padded cells or more are rejected.  The
 * first call on a device looks up that array and should come before any stream
 * capture (after a device reset, the first call in the new context looks it up
 * again); calls that overlap on the GPU share the array and race.
 * This entry point has no counterpart in the reference. */
UAAMG_API uaamg_status uaamg_residual_noalloc(int dim, int nx, int ny, int nz, double dx,
                                              double dy, double dz, const uint8_t* d_solid,
                                              const double* d_rhs, const double* d_p,
                                              double* d_out, void* stream);

/* Device memory held by the handle, bytes. */
UAAMG_API uaamg_status uaamg_device_bytes(uaamg_handle* h, size_t* bytes);

/* Text of the last error on this handle (never NULL). */
UAAMG_API const char* uaamg_last_error(uaamg_handle* h);
UAAMG_API const char* uaamg_status_string(int status);

/* ---- Batched uneven solves (uaamg_solve_batch) ---------------------------------
 * One problem of a batch: HOST arrays in the reference layout of Grid / Grid3D
 * (include/core/mesh.h:35, mesh_3d.h:38), padded, column-major i-fastest.  p
 * follows Solver::solve (include/solver/solver.h:18-34): 0 on entry, or the
 * initial guess when options.warm_start is set; the result is written into it. */
typedef struct uaamg_problem {
    int dim, nx, ny, nz;  /* nz ignored for dim = 2 */
    double dx, dy, dz;
    const uint8_t* solid;
    const double* rhs;
    double* p;
} uaamg_problem;

/* Solves n independent problems of any mix of sizes together on the handle's
 * device: each problem keeps its own hierarchy, CG state and stream (reused by
 * the next batch when its shape matches), and the host interleaves the problems'
 * two-iteration CUDA graphs so that small problems fill the GPU together.  The
 * handle's own problem (uaamg_set_problem_*) is untouched.  stats[i] (may be
 * NULL) receives problem i's statistics.  Returns UAAMG_OK when every problem
 * converged, else the first non-OK status in problem order.  The reference has
 * no batch entry point; each problem matches uaamg_solve on it alone bit for bit. */
UAAMG_API uaamg_status uaamg_solve_batch(uaamg_handle* h, int n, const uaamg_problem* problems,
                                         const uaamg_options* opts, uaamg_stats* stats);

/* 1: before its first solve, every hierarchy times its V-cycle marches at each
 * level for a few z-chunk lengths (planes per block) and keeps the fastest;
 * results are cached per level shape for the process.  0 (default): fixed rule.
 * No reference counterpart (the reference's kernels have fixed shapes). */
UAAMG_API uaamg_status uaamg_set_autotune(uaamg_handle* h, int on);

/* Process-wide file (JSON) that keeps the autotuner's choices -- z-chunk lengths per
 * level shape, and for batches the smoothing schedule per problem class (GPU,
 * precision, shape, solid fraction to 0.05) -- so later processes reuse them; NULL:
 * memory only (the default).  An existing file is read at once and rewritten as
 * choices are added.  No counterpart in the reference, whose CUDA kernels fix tile
 * shapes and smoothing at compile time. */
UAAMG_API uaamg_status uaamg_set_tune_cache(const char* path);

/* uaamg_solve_batch: the problems of at most max_cells padded cells share ONE CUDA
 * graph per step (two PCG iterations of each, on their own streams, forked and
 * joined inside the graph) instead of one graph each; 0 (default): every problem
 * runs its own graph.  Results are the same either way.  No counterpart in the
 * reference. */
UAAMG_API uaamg_status uaamg_set_batch_group(uaamg_handle* h, long long max_cells);

/* ---- Serving (uaamg_server_{start,submit,poll,stop}) --------------------------
 * A device-resident request loop on one GPU.  Requests carry a simulation id; the
 * server keeps each id's hierarchy and FP64 pressure on the device and
 * warm-starts the id's next request from it.  Requests are admitted while fewer
 * than max_active solves run and the device bytes of all resident ids stay within
 * hbm_budget_bytes (idle ids are evicted least-recently-used first); admitted
 * solves run concurrently, each on its own stream, and new requests join as
 * slots free up (continuous batching).  A request of an id waits for that id's
 * previous request. */
typedef struct uaamg_server uaamg_server;

typedef struct uaamg_server_config {
    int device;
    int precision;            /* uaamg_precision */
    double tol;               /* relative to ||b|| (UAAMG_TOL_REL) */
    int max_iter;
    int replace_every;        /* mixed precision residual replacement period */
    int warm_start;           /* 1: start from the id's previous pressure */
    int max_active;           /* concurrent solves */
    size_t hbm_budget_bytes;  /* device bytes all resident ids may hold */
} uaamg_server_config;

typedef struct uaamg_request {
    long long sim_id;
    int dim, nx, ny, nz;
    double dx, dy, dz;
    const uint8_t* solid;     /* host, copied by submit */
    const double* rhs;        /* host, copied by submit (see flags) */
    double* p_out;            /* host, may be NULL: receives the padded pressure (reference
                                 layout) when the solve finishes; must stay valid until then */
    int flags;                /* UAAMG_REQUEST_* bits, 0 by default */
} uaamg_request;

/* uaamg_request.flags: rhs (and p_out, when given) are lent to the server instead of
 * copied -- the right-hand side is copied to the device straight from rhs and the
 * pressure straight into p_out; the caller keeps both valid, and rhs unmodified, until
 * the ticket is polled done.  Page-locked (pinned) buffers make both copies
 * asynchronous; no host copy of either array is made. */
#define UAAMG_REQUEST_BORROW 1

typedef struct uaamg_result {
    long long ticket;
    long long sim_id;
    int status;               /* uaamg_status */
    int iterations;
    double rel_residual;      /* FP64 true ||b - A p|| / ||b|| */
    double wait_ms;           /* submit -> admitted */
    double latency_ms;        /* submit -> result on the host */
    int warm;                 /* 1 when warm-started from the id's previous pressure */
} uaamg_result;

UAAMG_API void uaamg_server_default_config(uaamg_server_config* cfg);
UAAMG_API uaamg_status uaamg_server_start(uaamg_server** out, const uaamg_server_config* cfg);
/* Copies the request's arrays and queues it; *ticket identifies it. */
UAAMG_API uaamg_status uaamg_server_submit(uaamg_server* s, const uaamg_request* req,
                                           long long* ticket);
/* *done = 1 once the ticket's solve finished (its p_out is written): res is
 * filled and the ticket is released.  Non-blocking; an unknown or already
 * released ticket is UAAMG_INVALID_ARG. */
UAAMG_API uaamg_status uaamg_server_poll(uaamg_server* s, long long ticket, uaamg_result* res,
                                         int* done);
/* Blocks until every submitted request has finished. */
UAAMG_API uaamg_status uaamg_server_drain(uaamg_server* s);
/* Device bytes held by resident ids, resident id count, completed requests. */
UAAMG_API uaamg_status uaamg_server_info(uaamg_server* s, size_t* device_bytes, int* resident,
                                         long long* completed);
UAAMG_API uaamg_status uaamg_server_stop(uaamg_server* s);

#ifdef __cplusplus
}
#endif
#endif /* UAAMG_H */
