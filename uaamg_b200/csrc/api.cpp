// C-ABI layer (include/uaamg.h): handle, problem staging, host<->device copies,
// dispatch to the per-precision engines.
#include "../../include/uaamg.h"

#include <chrono>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "engine.h"
#include "handle.h"

namespace uaamg {
namespace api {

uaamg_status fail(uaamg_handle* h, uaamg_status s, const std::string& msg) {
    if (h) h->err = msg;
    return s;
}

uaamg_status cuda_fail(uaamg_handle* h, cudaError_t e, const char* where) {
    return fail(h, UAAMG_CUDA_ERROR, std::string(where) + ": " + cudaGetErrorString(e));
}

uaamg_status map_engine(uaamg_handle* h, int e, const char* where, const uaamg::Engine* eng) {
    switch (e) {
        case uaamg::E_OK: return UAAMG_OK;
        case uaamg::E_OOM: return fail(h, UAAMG_OOM, std::string(where) + ": device allocation failed");
        case uaamg::E_ARG: return fail(h, UAAMG_INVALID_ARG, std::string(where) + ": invalid argument");
        case uaamg::E_NOPROB: return fail(h, UAAMG_NO_PROBLEM, std::string(where) + ": no problem set");
        default: {
            cudaError_t ce = eng && eng->cuda_error != cudaSuccess ? eng->cuda_error : cudaGetLastError();
            return fail(h, UAAMG_CUDA_ERROR, std::string(where) + ": CUDA error " +
                                                 (ce != cudaSuccess ? cudaGetErrorString(ce) : ""));
        }
    }
}

uaamg_status fill_stats(const uaamg::Engine* eng, const uaamg::SolveResult& r, uaamg_stats* st) {
    uaamg_status out;
    switch (r.status) {
        case 1: out = UAAMG_OK; break;            // CG_CONVERGED
        case 3: out = UAAMG_BREAKDOWN; break;
        case 4: out = UAAMG_NAN; break;
        default: out = UAAMG_NOT_CONVERGED; break; // CG_MAXITER / never started
    }
    if (st) {
        st->status = out;
        st->iterations = r.iterations;
        st->replacements = r.replacements;
        st->levels = eng->nlevels();
        st->residual = r.rr_true >= 0 ? __builtin_sqrt(r.rr_true) : 0.0;
        st->rhs_norm = r.bnorm;
        st->rel_residual = r.bnorm > 0 ? st->residual / r.bnorm : st->residual;
        st->recursive_residual = r.rr >= 0 ? __builtin_sqrt(r.rr) : 0.0;
        st->kernel_launches = eng->launches();
    }
    return out;
}

}  // namespace api
}  // namespace uaamg

namespace {

using uaamg::api::fail;
using uaamg::api::cuda_fail;
using uaamg::api::map_engine;

void free_problem(uaamg_handle* h) {
    if (h->stream) cudaStreamSynchronize(h->stream);
    else cudaDeviceSynchronize();
    cudaFree(h->d_solid); h->d_solid = nullptr;
    cudaFree(h->d_rhs); h->d_rhs = nullptr;
    cudaFree(h->d_p); h->d_p = nullptr;
    cudaFree(h->d_hist); h->d_hist = nullptr;
    for (int a = 0; a < 3; ++a) {
        cudaFree(h->d_face[a]);
        h->d_face[a] = nullptr;
        h->face_n[a] = 0;
        cudaFree(h->d_lap[a]);
        h->d_lap[a] = nullptr;
    }
    h->lap_on = false;
    h->hist_cap = 0;
    h->n = 0;
    h->dim = 0;
    for (int q = 0; q < 3; ++q) h->ready[q] = false;
}

// Engine of precision p with the current problem's hierarchy built.
uaamg_status engine_for(uaamg_handle* h, int p, uaamg::Engine** out) {
    if (p < 0 || p > 2) return fail(h, UAAMG_INVALID_ARG, "unknown precision");
    if (!h->dim) return fail(h, UAAMG_NO_PROBLEM, "no problem set (call uaamg_set_problem_*)");
    if (!h->eng[p]) {
        h->eng[p] = p == uaamg::PREC_FP64 ? uaamg::create_engine_f64()
                                          : uaamg::create_engine_f32(p == uaamg::PREC_MIXED);
        if (!h->eng[p]) return fail(h, UAAMG_OOM, "engine allocation failed");
    }
    h->eng[p]->set_stream(h->stream);
    uaamg::api::apply_vcycle_mode(h->eng[p], h->sweeps);
    h->eng[p]->set_smoothing(h->nu_fine, h->nu_coarse);
    h->eng[p]->set_autotune(h->autotune != 0);
    if (h->lap_on)
        h->eng[p]->set_operator(h->d_lap[0], h->d_lap[1], h->d_lap[2], h->nx + 2, h->lap_version);
    else
        h->eng[p]->set_operator(nullptr, nullptr, nullptr, 0, h->lap_version);
    if (!h->ready[p]) {
        int e = h->eng[p]->set_problem(h->dim, h->nx, h->ny, h->nz, h->dx, h->dy, h->dz,
                                       h->d_solid, h->dirichlet);
        if (e != uaamg::E_OK) return map_engine(h, e, "hierarchy set-up", h->eng[p]);
        h->ready[p] = true;
    }
    *out = h->eng[p];
    return UAAMG_OK;
}

uaamg_status set_problem(uaamg_handle* h, int dim, int nx, int ny, int nz, double dx, double dy,
                         double dz, const uint8_t* solid, bool solid_on_device) {
    if (!h) return UAAMG_INVALID_ARG;
    if (dim != 2 && dim != 3) return fail(h, UAAMG_INVALID_ARG, "dim must be 2 or 3");
    if (dim == 2) { nz = 0; dz = 1.0; }
    if (nx < 2 || ny < 2 || (dim == 3 && nz < 2))
        return fail(h, UAAMG_INVALID_ARG, "every axis needs at least 2 interior cells");
    if (!(dx > 0) || !(dy > 0) || !(dz > 0))
        return fail(h, UAAMG_INVALID_ARG, "spacing must be positive");
    const size_t n = (size_t)(nx + 2) * (ny + 2) * (dim == 3 ? (size_t)(nz + 2) : 1);
    if (n >= (size_t)1 << 31) return fail(h, UAAMG_INVALID_ARG, "grid exceeds 2^31 padded cells");
    if (!solid) return fail(h, UAAMG_INVALID_ARG, "solid mask is NULL");
    cudaSetDevice(h->device);
    free_problem(h);
    cudaError_t e;
    if ((e = cudaMalloc(&h->d_solid, n)) != cudaSuccess ||
        (e = cudaMalloc(&h->d_rhs, n * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&h->d_p, n * sizeof(double))) != cudaSuccess) {
        cudaGetLastError();
        free_problem(h);
        return fail(h, UAAMG_OOM, "problem buffers: device allocation failed");
    }
    e = cudaMemcpyAsync(h->d_solid, solid, n,
                        solid_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { free_problem(h); return cuda_fail(h, e, "mask upload"); }
    h->dim = dim; h->nx = nx; h->ny = ny; h->nz = nz;
    h->dx = dx; h->dy = dy; h->dz = dz;
    h->n = n;
    return UAAMG_OK;
}

uaamg_status ensure_hist(uaamg_handle* h, int max_iter) {
    if (max_iter + 1 <= h->hist_cap) return UAAMG_OK;
    cudaFree(h->d_hist);
    h->d_hist = nullptr;
    h->hist_cap = 0;
    if (cudaMalloc(&h->d_hist, sizeof(double) * (size_t)(max_iter + 1)) != cudaSuccess) {
        cudaGetLastError();
        return fail(h, UAAMG_OOM, "residual history allocation failed");
    }
    h->hist_cap = max_iter + 1;
    return UAAMG_OK;
}

uaamg_status solve_dev(uaamg_handle* h, const double* d_rhs, double* d_p, const uaamg_options* o,
                       uaamg_stats* st, cudaEvent_t p_ready = nullptr) {
    uaamg_options opts;
    uaamg_default_options(&opts);
    if (o) opts = *o;
    if (opts.max_iter < 0 || !(opts.tol >= 0) || opts.tol_mode < 0 || opts.tol_mode > 1)
        return fail(h, UAAMG_INVALID_ARG, "bad options");
    if (!d_rhs || !d_p) return fail(h, UAAMG_INVALID_ARG, "NULL array");
    uaamg::Engine* eng = nullptr;
    uaamg_status s = engine_for(h, opts.precision, &eng);
    if (s != UAAMG_OK) return s;
    if ((s = ensure_hist(h, opts.max_iter)) != UAAMG_OK) return s;
    cudaMemsetAsync(h->d_hist, 0, sizeof(double) * (size_t)h->hist_cap, h->stream);
    uaamg::SolveArgs a;
    a.rhs = d_rhs;
    a.x = d_p;
    a.max_iter = opts.max_iter;
    a.tol = opts.tol;
    a.tol_mode = opts.tol_mode;
    a.warm = opts.warm_start;
    a.replace_every = opts.replace_every;
    a.project_mean = opts.project_mean;
    a.precond = opts.preconditioner;
    a.hist = h->d_hist;
    a.ref_solid = h->d_solid;
    a.x_ready = p_ready;
    uaamg::SolveResult r;
    std::memset(&r, 0, sizeof(r));
    int e = eng->solve(a, &r);
    if (e != uaamg::E_OK) return map_engine(h, e, "solve", eng);
    if (eng->timed_out())
        return fail(h, UAAMG_TIMEOUT, "solve: a kernel gave up waiting for its tile loads");
    h->last_iters = r.iterations;
    return uaamg::api::fill_stats(eng, r, st);
}

}  // namespace

extern "C" {

void uaamg_default_options(uaamg_options* o) {
    if (!o) return;
    o->precision = UAAMG_FP64;
    o->tol_mode = UAAMG_TOL_ABS;
    o->max_iter = 2000;
    o->tol = 1e-6;
    o->warm_start = 0;
    o->replace_every = 10;
    o->project_mean = 0;
    o->preconditioner = 1;
}

uaamg_status uaamg_create(uaamg_handle** out, int device) {
    if (!out) return UAAMG_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return UAAMG_INVALID_ARG;
    }
    if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return UAAMG_CUDA_ERROR; }
    uaamg_handle* h = new (std::nothrow) uaamg_handle();
    if (!h) return UAAMG_OOM;
    h->device = device;
    *out = h;
    return UAAMG_OK;
}

uaamg_status uaamg_destroy(uaamg_handle* h) {
    if (!h) return UAAMG_INVALID_ARG;
    cudaSetDevice(h->device);
    free_problem(h);
    uaamg::api::free_batch(h);
    for (auto*& e : h->eng) { delete e; e = nullptr; }
    if (h->p_ready) cudaEventDestroy(h->p_ready);
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    delete h;
    return UAAMG_OK;
}

uaamg_status uaamg_set_stream(uaamg_handle* h, void* stream) {
    if (!h) return UAAMG_INVALID_ARG;
    h->stream = static_cast<cudaStream_t>(stream);
    for (auto* e : h->eng) if (e) e->set_stream(h->stream);
    return UAAMG_OK;
}

uaamg_status uaamg_set_vcycle_kernels(uaamg_handle* h, int sweeps) {
    if (!h) return UAAMG_INVALID_ARG;
    if (sweeps < 0 || sweeps > 4) return fail(h, UAAMG_INVALID_ARG, "V-cycle kernels: 0 to 4");
    h->sweeps = sweeps;
    return UAAMG_OK;
}

uaamg_status uaamg_set_smoothing(uaamg_handle* h, int sweeps_fine, int sweeps_coarse) {
    if (!h) return UAAMG_INVALID_ARG;
    if (sweeps_fine < 1 || sweeps_fine > 4 || sweeps_coarse < 1 || sweeps_coarse > 4)
        return fail(h, UAAMG_INVALID_ARG, "smoothing sweeps: 1 to 4");
    h->nu_fine = sweeps_fine;
    h->nu_coarse = sweeps_coarse;
    return UAAMG_OK;
}

uaamg_status uaamg_set_variable_laplacian(uaamg_handle* h, const double* lap_diag,
                                          const double* lap_off_x, const double* lap_off_y) {
    if (!h) return UAAMG_INVALID_ARG;
    const int given = (lap_diag != nullptr) + (lap_off_x != nullptr) + (lap_off_y != nullptr);
    if (given != 0 && given != 3)
        return fail(h, UAAMG_INVALID_ARG, "variable Laplacian: give all three arrays or none");
    if (!h->dim) return fail(h, UAAMG_NO_PROBLEM, "no problem set (call uaamg_set_problem_*)");
    if (h->dim != 2)
        return fail(h, UAAMG_INVALID_ARG, "variable Laplacian: 2D problems only");
    if (!given) {
        h->lap_on = false;
        return UAAMG_OK;
    }
    cudaSetDevice(h->device);
    const double* src[3] = {lap_diag, lap_off_x, lap_off_y};
    const size_t bytes = h->n * sizeof(double);
    for (int a = 0; a < 3; ++a) {
        if (!h->d_lap[a] && cudaMalloc(&h->d_lap[a], bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(h, UAAMG_OOM, "variable Laplacian: device allocation failed");
        }
    }
    // the solves in flight may still read the previous coefficients
    cudaError_t e = h->stream ? cudaStreamSynchronize(h->stream) : cudaDeviceSynchronize();
    for (int a = 0; a < 3 && e == cudaSuccess; ++a)
        e = cudaMemcpyAsync(h->d_lap[a], src[a], bytes, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        h->lap_on = false;
        return cuda_fail(h, e, "variable Laplacian upload");
    }
    h->lap_on = true;
    ++h->lap_version;
    return UAAMG_OK;
}

uaamg_status uaamg_set_dirichlet_walls(uaamg_handle* h, int on) {
    if (!h) return UAAMG_INVALID_ARG;
    h->dirichlet = on ? 1 : 0;
    for (int q = 0; q < 3; ++q) h->ready[q] = false;
    return UAAMG_OK;
}

uaamg_status uaamg_set_problem_2d(uaamg_handle* h, int nx, int ny, double dx, double dy,
                                  const uint8_t* solid) {
    return set_problem(h, 2, nx, ny, 0, dx, dy, 1.0, solid, false);
}

uaamg_status uaamg_set_problem_3d(uaamg_handle* h, int nx, int ny, int nz, double dx, double dy,
                                  double dz, const uint8_t* solid) {
    return set_problem(h, 3, nx, ny, nz, dx, dy, dz, solid, false);
}

uaamg_status uaamg_set_problem_device(uaamg_handle* h, int dim, int nx, int ny, int nz, double dx,
                                      double dy, double dz, const uint8_t* d_solid) {
    return set_problem(h, dim, nx, ny, nz, dx, dy, dz, d_solid, true);
}

uaamg_status uaamg_solve(uaamg_handle* h, const double* rhs, double* p, const uaamg_options* opts,
                         uaamg_stats* stats) {
    if (!h) return UAAMG_INVALID_ARG;
    if (!h->dim) return fail(h, UAAMG_NO_PROBLEM, "no problem set (call uaamg_set_problem_*)");
    if (!rhs || !p) return fail(h, UAAMG_INVALID_ARG, "NULL array");
    cudaSetDevice(h->device);
    auto t0 = std::chrono::steady_clock::now();
    const size_t bytes = h->n * sizeof(double);
    cudaError_t e = cudaMemcpyAsync(h->d_rhs, rhs, bytes, cudaMemcpyHostToDevice, h->stream);
    // p is read only when the solve adds its result to it (or at the start of a warm
    // start): without a warm start it is uploaded on a side stream while the solve runs
    cudaEvent_t p_ready = nullptr;
    if (e == cudaSuccess && !(opts && opts->warm_start)) {
        if (!h->copy_stream && cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
            h->copy_stream = nullptr;
        if (h->copy_stream && !h->p_ready &&
            cudaEventCreateWithFlags(&h->p_ready, cudaEventDisableTiming) != cudaSuccess)
            h->p_ready = nullptr;
        if (h->copy_stream && h->p_ready) {
            e = cudaMemcpyAsync(h->d_p, p, bytes, cudaMemcpyHostToDevice, h->copy_stream);
            if (e == cudaSuccess) e = cudaEventRecord(h->p_ready, h->copy_stream);
            if (e == cudaSuccess) p_ready = h->p_ready;
        }
    }
    if (e == cudaSuccess && !p_ready) e = cudaMemcpyAsync(h->d_p, p, bytes, cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "upload");
    uaamg_status s = solve_dev(h, h->d_rhs, h->d_p, opts, stats, p_ready);
    if (p_ready) cudaEventSynchronize(p_ready);  // the upload has finished whatever the outcome
    if (s == UAAMG_OK || s == UAAMG_NOT_CONVERGED || s == UAAMG_BREAKDOWN || s == UAAMG_NAN) {
        e = cudaMemcpyAsync(p, h->d_p, bytes, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "download");
    }
    if (stats)
        stats->solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return s;
}

uaamg_status uaamg_solve_device(uaamg_handle* h, const double* d_rhs, double* d_p,
                                const uaamg_options* opts, uaamg_stats* stats) {
    if (!h) return UAAMG_INVALID_ARG;
    cudaSetDevice(h->device);
    auto t0 = std::chrono::steady_clock::now();
    uaamg_status s = solve_dev(h, d_rhs, d_p, opts, stats);
    if (stats)
        stats->solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return s;
}

uaamg_status uaamg_precond_apply(uaamg_handle* h, int precision, const double* r, double* z) {
    if (!h) return UAAMG_INVALID_ARG;
    if (!r || !z) return fail(h, UAAMG_INVALID_ARG, "NULL array");
    cudaSetDevice(h->device);
    uaamg::Engine* eng = nullptr;
    uaamg_status s = engine_for(h, precision, &eng);
    if (s != UAAMG_OK) return s;
    const size_t bytes = h->n * sizeof(double);
    cudaError_t e = cudaMemcpyAsync(h->d_rhs, r, bytes, cudaMemcpyHostToDevice, h->stream);
    // z is written on interior cells only (UAAMGPreconditioner3D::apply,
    // uaamg_preconditioner_3d.cpp:225-228); its ghost cells come back as 0
    if (e == cudaSuccess) e = cudaMemsetAsync(h->d_p, 0, bytes, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "upload");
    int ee = eng->precond_apply(h->d_rhs, h->d_p);
    if (ee != uaamg::E_OK) return map_engine(h, ee, "precond_apply", eng);
    if (eng->timed_out())
        return fail(h, UAAMG_TIMEOUT, "precond_apply: a kernel gave up waiting for its tile loads");
    e = cudaMemcpyAsync(z, h->d_p, bytes, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "download");
    return UAAMG_OK;
}

uaamg_status uaamg_residual_history(uaamg_handle* h, double* hist, int n) {
    if (!h || !hist || n < 0) return UAAMG_INVALID_ARG;
    if (!h->d_hist) return fail(h, UAAMG_NO_PROBLEM, "no solve yet");
    int m = h->last_iters + 1;
    if (m > n) m = n;
    if (m > h->hist_cap) m = h->hist_cap;
    cudaSetDevice(h->device);
    cudaError_t e = cudaMemcpyAsync(hist, h->d_hist, sizeof(double) * (size_t)m,
                                    cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return e == cudaSuccess ? UAAMG_OK : cuda_fail(h, e, "history");
}

uaamg_status uaamg_num_levels(uaamg_handle* h, int* nlevels) {
    if (!h || !nlevels) return UAAMG_INVALID_ARG;
    uaamg::Engine* eng = nullptr;
    uaamg_status s = engine_for(h, UAAMG_FP64, &eng);
    if (s != UAAMG_OK) return s;
    *nlevels = eng->nlevels();
    return UAAMG_OK;
}

uaamg_status uaamg_level_dims(uaamg_handle* h, int l, int* nx, int* ny, int* nz) {
    if (!h || !nx || !ny || !nz) return UAAMG_INVALID_ARG;
    uaamg::Engine* eng = nullptr;
    uaamg_status s = engine_for(h, UAAMG_FP64, &eng);
    if (s != UAAMG_OK) return s;
    if (l < 0 || l >= eng->nlevels()) return fail(h, UAAMG_INVALID_ARG, "level out of range");
    eng->level_dims(l, nx, ny, nz);
    return UAAMG_OK;
}

uaamg_status uaamg_level_trim(uaamg_handle* h, int precision, int l, int* boxes, int* trimmed) {
    if (!h || !boxes || !trimmed) return UAAMG_INVALID_ARG;
    cudaSetDevice(h->device);
    uaamg::Engine* eng = nullptr;
    uaamg_status s = engine_for(h, precision, &eng);
    if (s != UAAMG_OK) return s;
    if (l < 0 || l >= eng->nlevels()) return fail(h, UAAMG_INVALID_ARG, "level out of range");
    return map_engine(h, eng->level_trim(l, boxes, trimmed), "level_trim");
}

uaamg_status uaamg_copy_level(uaamg_handle* h, int precision, int l, uint8_t* solid, double* cx,
                              double* cy, double* cz) {
    if (!h) return UAAMG_INVALID_ARG;
    cudaSetDevice(h->device);
    uaamg::Engine* eng = nullptr;
    uaamg_status s = engine_for(h, precision, &eng);
    if (s != UAAMG_OK) return s;
    int e = eng->copy_level(l, solid, cx, cy, cz);
    return map_engine(h, e, "copy_level");
}

uaamg_status uaamg_profile_solve(uaamg_handle* h, const double* d_rhs, double* d_p,
                                 const uaamg_options* opts, uaamg_stats* stats,
                                 uaamg_kernel_time* out, int cap, int* count) {
    if (!h || !count || (cap > 0 && !out)) return UAAMG_INVALID_ARG;
    cudaSetDevice(h->device);
    uaamg_options o;
    uaamg_default_options(&o);
    if (opts) o = *opts;
    uaamg::Engine* eng = nullptr;
    uaamg_status s = engine_for(h, o.precision, &eng);
    if (s != UAAMG_OK) return s;
    eng->set_profiling(true);
    auto t0 = std::chrono::steady_clock::now();
    s = solve_dev(h, d_rhs, d_p, &o, stats);
    if (stats)
        stats->solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::vector<uaamg::KernelTime> kt;
    int e = eng->profile_results(kt);
    eng->set_profiling(false);
    if (e != uaamg::E_OK) return map_engine(h, e, "profile");
    *count = (int)kt.size();
    for (int q = 0; q < cap && q < (int)kt.size(); ++q) {
        std::memset(out[q].name, 0, sizeof(out[q].name));
        std::strncpy(out[q].name, kt[q].name, sizeof(out[q].name) - 1);
        out[q].level = kt[q].level;
        out[q].launches = kt[q].launches;
        out[q].total_ms = kt[q].total_ms;
        out[q].bytes_per_launch = kt[q].bytes;
    }
    return s;
}

uaamg_status uaamg_device_bytes(uaamg_handle* h, size_t* bytes) {
    if (!h || !bytes) return UAAMG_INVALID_ARG;
    size_t b = h->n * (1 + 2 * sizeof(double)) + sizeof(double) * (size_t)h->hist_cap;
    for (auto* e : h->eng) if (e) b += e->device_bytes();
    *bytes = b;
    return UAAMG_OK;
}

const char* uaamg_last_error(uaamg_handle* h) {
    if (!h) return "NULL handle";
    return h->err.c_str();
}

const char* uaamg_status_string(int s) {
    switch (s) {
        case UAAMG_OK: return "ok";
        case UAAMG_NOT_CONVERGED: return "not converged";
        case UAAMG_BREAKDOWN: return "breakdown";
        case UAAMG_NAN: return "nan";
        case UAAMG_OOM: return "out of device memory";
        case UAAMG_INVALID_ARG: return "invalid argument";
        case UAAMG_CUDA_ERROR: return "cuda error";
        case UAAMG_TIMEOUT: return "timeout";
        case UAAMG_NO_PROBLEM: return "no problem set";
        default: return "unknown status";
    }
}

}  // extern "C"
