// Pressure projection around the solve with every array on the GPU: the
// PressureProjection::project / PressureProjection3D::project drop-in
// (src/pressure/pressure.cpp:5-33, pressure_3d.cpp:5-40) --
//   rhs = div(u) / dt on fluid interior cells, 0 elsewhere (pressure.cpp:10-14 with
//         fvc::divergence, include/core/grid.h:44-47; operators.h:18-21, operators_3d.h:17-21)
//   p = 0, solve lap(p) = rhs (uaamg_solve_device)
//   u -= dt * dp/dx on the faces between two fluid cells (pressure.cpp:21-32,
//         pressure_3d.cpp:21-39), likewise v and w.
// The per-cell and per-face expressions are the reference's, evaluated in FP64 in the
// same order (this unit is built with -fmad=false), so the divergence and the
// corrected velocities are bit-identical to the reference's for the same pressure.
//
// Face arrays are FP64, i fastest: u (nx+1)(ny+2)[(nz+2)], v (nx+2)(ny+1)[(nz+2)],
// w (nx+2)(ny+2)(nz+1) (3D only); face (i, j, k) of u lies between cells (i, j, k)
// and (i+1, j, k) of the padded cell layout.
#include <chrono>
#include <cstring>

#include "handle.h"

using uaamg::api::cuda_fail;
using uaamg::api::fail;

namespace {

constexpr int kProjThreads = 128;

// Grid over an array of rows: x covers a row of fx entries, y the rows j, z the
// planes k (one block row a thread row; no index division).
inline dim3 row_grid(int fx, int fy, int fz) {
    return dim3((unsigned)((fx + kProjThreads - 1) / kProjThreads), (unsigned)fy, (unsigned)fz);
}

// rhs over the whole padded cell array (0 on ghost and solid cells).
__global__ void k_divergence(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                             const uint8_t* __restrict__ solid, const double* __restrict__ u,
                             const double* __restrict__ v, const double* __restrict__ w, double dt,
                             double* __restrict__ rhs) {
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x), j = (int)blockIdx.y;
    const int k = dim == 3 ? (int)blockIdx.z : 0;
    if (i > nx + 1) return;
    {
        const long long id = i + (long long)(nx + 2) * (j + (long long)(ny + 2) * k);
        double out = 0.0;
        const bool inner = i >= 1 && i <= nx && j >= 1 && j <= ny && (dim == 2 || (k >= 1 && k <= nz));
        if (inner && !solid[id]) {
            if (dim == 3) {
                const long long su = nx + 1, suv = (long long)(nx + 1) * (ny + 2);
                const long long sv = nx + 2, svv = (long long)(nx + 2) * (ny + 1);
                const long long sw = nx + 2, sww = (long long)(nx + 2) * (ny + 2);
                const double div = (u[i + j * su + k * suv] - u[(i - 1) + j * su + k * suv]) / dx +
                                   (v[i + j * sv + k * svv] - v[i + (j - 1) * sv + k * svv]) / dy +
                                   (w[i + j * sw + k * sww] - w[i + j * sw + (k - 1) * sww]) / dz;
                out = div / dt;
            } else {
                const long long su = nx + 1, sv = nx + 2;
                const double div = (u[i + j * su] - u[(i - 1) + j * su]) / dx +
                                   (v[i + j * sv] - v[i + (j - 1) * sv]) / dy;
                out = div / dt;
            }
        }
        rhs[id] = out;
    }
}

// One face array (axis 0: u, 1: v, 2: w): f -= dt * (p_hi - p_lo) / h on the interior
// faces whose two cells are fluid.
__global__ void k_correct_faces(int dim, int axis, int nx, int ny, int nz, double h,
                                const uint8_t* __restrict__ solid, const double* __restrict__ p,
                                double dt, double* __restrict__ f) {
    const int fx = axis == 0 ? nx + 1 : nx + 2;
    const int fy = axis == 1 ? ny + 1 : ny + 2;
    const long long csx = nx + 2, csxy = (long long)(nx + 2) * (ny + 2);
    const long long step = axis == 0 ? 1 : (axis == 1 ? csx : csxy);
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x), j = (int)blockIdx.y;
    const int k = dim == 3 ? (int)blockIdx.z : 0;
    if (i >= fx) return;
    {
        const long long t = i + (long long)fx * (j + (long long)fy * k);
        bool ok;
        if (axis == 0) ok = i >= 1 && i <= nx - 1 && j >= 1 && j <= ny;
        else if (axis == 1) ok = i >= 1 && i <= nx && j >= 1 && j <= ny - 1;
        else ok = i >= 1 && i <= nx && j >= 1 && j <= ny && k >= 1 && k <= nz - 1;
        if (dim == 3 && axis != 2) ok = ok && k >= 1 && k <= nz;
        if (!ok) return;
        const long long c0 = i + j * csx + k * csxy, c1 = c0 + step;
        if (solid[c0] || solid[c1]) return;
        f[t] -= dt * (p[c1] - p[c0]) / h;
    }
}

// Cell-centre velocities of recoverStaticPressure, indices clamped to the interior.
__device__ __forceinline__ double st_uc(const double* u, int nx, int ny, int i, int j) {
    i = i < 1 ? 1 : (i > nx ? nx : i);
    j = j < 1 ? 1 : (j > ny ? ny : j);
    const long long su = nx + 1;
    return 0.5 * (u[i + j * su] + u[(i - 1) + j * su]);
}
__device__ __forceinline__ double st_vc(const double* v, int nx, int ny, int i, int j) {
    i = i < 1 ? 1 : (i > nx ? nx : i);
    j = j < 1 ? 1 : (j > ny ? ny : j);
    const long long sv = nx + 2;
    return 0.5 * (v[i + j * sv] + v[i + (j - 1) * sv]);
}

// Right-hand side of PressureProjection::recoverStaticPressure (pressure.cpp:35-66),
// 2D: rhs = -(du/dx^2 + 2 du/dy dv/dx + dv/dy^2) on fluid cells, the cross
// derivatives dropped next to a solid; 0 on ghost and solid cells.
__global__ void k_static_rhs(int nx, int ny, double dx, double dy, const uint8_t* __restrict__ solid,
                             const double* __restrict__ u, const double* __restrict__ v,
                             double* __restrict__ rhs) {
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x), j = (int)blockIdx.y;
    if (i > nx + 1) return;
    const long long sp = nx + 2, su = nx + 1, sv = nx + 2;
    const long long id = i + j * sp;
    double out = 0.0;
    if (i >= 1 && i <= nx && j >= 1 && j <= ny && !solid[id]) {
        const double du_dx = (u[i + j * su] - u[(i - 1) + j * su]) / dx;
        const double dv_dy = (v[i + j * sv] - v[i + (j - 1) * sv]) / dy;
        const bool sL = solid[id - 1], sR = solid[id + 1], sB = solid[id - sp], sT = solid[id + sp];
        const double du_dy =
            (sB || sT) ? 0.0 : (st_uc(u, nx, ny, i, j + 1) - st_uc(u, nx, ny, i, j - 1)) / (2 * dy);
        const double dv_dx =
            (sL || sR) ? 0.0 : (st_vc(v, nx, ny, i + 1, j) - st_vc(v, nx, ny, i - 1, j)) / (2 * dx);
        out = -(du_dx * du_dx + 2.0 * du_dy * dv_dx + dv_dy * dv_dy);
    }
    rhs[id] = out;
}

long long face_count(int dim, int nx, int ny, int nz, int axis) {
    const long long zz = dim == 3 ? nz + 2 : 1;
    if (axis == 0) return (long long)(nx + 1) * (ny + 2) * zz;
    if (axis == 1) return (long long)(nx + 2) * (ny + 1) * zz;
    return (long long)(nx + 2) * (ny + 2) * (nz + 1);
}

// Whether a solve that returned s left a pressure to correct the velocities with: as
// the reference's project() corrects after any solve (pressure.cpp:17-32), every
// solver outcome counts (converged, max_iter, breakdown, NaN), errors do not.
bool solved(uaamg_status s) {
    return s == UAAMG_OK || s == UAAMG_NOT_CONVERGED || s == UAAMG_BREAKDOWN || s == UAAMG_NAN;
}

// Divergence into the handle's staging RHS, p zeroed unless a warm start, the solve,
// the face correction; everything on the handle's stream.
uaamg_status project_dev(uaamg_handle* h, double dt, double* d_u, double* d_v, double* d_w,
                         double* d_p, const uaamg_options* opts, uaamg_stats* stats) {
    if (!h->dim) return fail(h, UAAMG_NO_PROBLEM, "no problem set (call uaamg_set_problem_*)");
    if (!d_u || !d_v || !d_p || (h->dim == 3 && !d_w)) return fail(h, UAAMG_INVALID_ARG, "NULL array");
    if (!(dt > 0.0)) return fail(h, UAAMG_INVALID_ARG, "dt must be positive");
    const int dim = h->dim, nx = h->nx, ny = h->ny, nz = h->nz;
    if (ny + 2 > 65535 || (dim == 3 && nz + 2 > 65535))
        return fail(h, UAAMG_INVALID_ARG, "projection: more than 65533 cells along y or z");
    const long long n = (long long)h->n;
    k_divergence<<<row_grid(nx + 2, ny + 2, dim == 3 ? nz + 2 : 1), kProjThreads, 0, h->stream>>>(
        dim, nx, ny, nz, h->dx, h->dy, h->dz, h->d_solid, d_u, d_v, d_w, dt, h->d_rhs);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "divergence");
    const bool warm = opts && opts->warm_start;
    if (!warm && (e = cudaMemsetAsync(d_p, 0, (size_t)n * sizeof(double), h->stream)) != cudaSuccess)
        return cuda_fail(h, e, "zero p");
    const uaamg_status s = uaamg_solve_device(h, h->d_rhs, d_p, opts, stats);
    if (!solved(s)) return s;
    double* f[3] = {d_u, d_v, d_w};
    const double hh[3] = {h->dx, h->dy, h->dz};
    for (int a = 0; a < dim; ++a) {
        const int fx = a == 0 ? nx + 1 : nx + 2, fy = a == 1 ? ny + 1 : ny + 2;
        const int fz = dim == 3 ? (a == 2 ? nz + 1 : nz + 2) : 1;
        k_correct_faces<<<row_grid(fx, fy, fz), kProjThreads, 0, h->stream>>>(dim, a, nx, ny, nz, hh[a],
                                                                              h->d_solid, d_p, dt, f[a]);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(h, e, "velocity correction");
    return s;
}

// recoverStaticPressure: its right-hand side into the handle's staging RHS, p = 0,
// the solve (the hierarchy of the current problem is reused).
uaamg_status static_dev(uaamg_handle* h, const double* d_u, const double* d_v, double* d_p,
                        const uaamg_options* opts, uaamg_stats* stats) {
    if (!h->dim) return fail(h, UAAMG_NO_PROBLEM, "no problem set (call uaamg_set_problem_*)");
    if (h->dim != 2) return fail(h, UAAMG_INVALID_ARG, "static pressure recovery is 2D (as in the reference)");
    if (!d_u || !d_v || !d_p) return fail(h, UAAMG_INVALID_ARG, "NULL array");
    if (h->ny + 2 > 65535) return fail(h, UAAMG_INVALID_ARG, "static pressure: more than 65533 rows");
    k_static_rhs<<<row_grid(h->nx + 2, h->ny + 2, 1), kProjThreads, 0, h->stream>>>(
        h->nx, h->ny, h->dx, h->dy, h->d_solid, d_u, d_v, h->d_rhs);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(h, e, "static rhs");
    if ((e = cudaMemsetAsync(d_p, 0, h->n * sizeof(double), h->stream)) != cudaSuccess)
        return cuda_fail(h, e, "zero p");
    return uaamg_solve_device(h, h->d_rhs, d_p, opts, stats);
}

// Device copies of the face arrays for the host-array entry point, sized on demand.
uaamg_status ensure_faces(uaamg_handle* h) {
    for (int a = 0; a < h->dim; ++a) {
        const size_t want = (size_t)face_count(h->dim, h->nx, h->ny, h->nz, a);
        if (h->d_face[a] && h->face_n[a] == want) continue;
        cudaFree(h->d_face[a]);
        h->d_face[a] = nullptr;
        h->face_n[a] = 0;
        cudaError_t e = cudaMalloc(&h->d_face[a], want * sizeof(double));
        if (e != cudaSuccess) {
            h->d_face[a] = nullptr;
            return e == cudaErrorMemoryAllocation ? fail(h, UAAMG_OOM, "face arrays")
                                                  : cuda_fail(h, e, "face arrays");
        }
        h->face_n[a] = want;
    }
    return UAAMG_OK;
}

}  // namespace

extern "C" {

uaamg_status uaamg_project_device(uaamg_handle* h, double dt, double* d_u, double* d_v, double* d_w,
                                  double* d_p, const uaamg_options* opts, uaamg_stats* stats) {
    if (!h) return UAAMG_INVALID_ARG;
    cudaSetDevice(h->device);
    const auto t0 = std::chrono::steady_clock::now();
    const uaamg_status s = project_dev(h, dt, d_u, d_v, d_w, d_p, opts, stats);
    if (stats)
        stats->solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return s;
}

uaamg_status uaamg_project(uaamg_handle* h, double dt, double* u, double* v, double* w, double* p,
                           const uaamg_options* opts, uaamg_stats* stats) {
    if (!h) return UAAMG_INVALID_ARG;
    if (!h->dim) return fail(h, UAAMG_NO_PROBLEM, "no problem set (call uaamg_set_problem_*)");
    if (!u || !v || !p || (h->dim == 3 && !w)) return fail(h, UAAMG_INVALID_ARG, "NULL array");
    cudaSetDevice(h->device);
    const auto t0 = std::chrono::steady_clock::now();
    uaamg_status s = ensure_faces(h);
    if (s != UAAMG_OK) return s;
    double* host[3] = {u, v, w};
    cudaError_t e = cudaSuccess;
    for (int a = 0; a < h->dim && e == cudaSuccess; ++a)
        e = cudaMemcpyAsync(h->d_face[a], host[a], h->face_n[a] * sizeof(double), cudaMemcpyHostToDevice,
                            h->stream);
    if (e == cudaSuccess && opts && opts->warm_start)
        e = cudaMemcpyAsync(h->d_p, p, h->n * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "upload");
    s = project_dev(h, dt, h->d_face[0], h->d_face[1], h->dim == 3 ? h->d_face[2] : nullptr, h->d_p,
                    opts, stats);
    if (!solved(s)) return s;
    for (int a = 0; a < h->dim && e == cudaSuccess; ++a)
        e = cudaMemcpyAsync(host[a], h->d_face[a], h->face_n[a] * sizeof(double), cudaMemcpyDeviceToHost,
                            h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p, h->d_p, h->n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "download");
    if (stats)
        stats->solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return s;
}

}  // extern "C"

extern "C" {

uaamg_status uaamg_static_pressure_device(uaamg_handle* h, const double* d_u, const double* d_v,
                                          double* d_p, const uaamg_options* opts, uaamg_stats* stats) {
    if (!h) return UAAMG_INVALID_ARG;
    cudaSetDevice(h->device);
    return static_dev(h, d_u, d_v, d_p, opts, stats);
}

uaamg_status uaamg_static_pressure(uaamg_handle* h, const double* u, const double* v, double* p,
                                   const uaamg_options* opts, uaamg_stats* stats) {
    if (!h) return UAAMG_INVALID_ARG;
    if (!h->dim) return fail(h, UAAMG_NO_PROBLEM, "no problem set (call uaamg_set_problem_*)");
    if (h->dim != 2) return fail(h, UAAMG_INVALID_ARG, "static pressure recovery is 2D (as in the reference)");
    if (!u || !v || !p) return fail(h, UAAMG_INVALID_ARG, "NULL array");
    cudaSetDevice(h->device);
    uaamg_status s = ensure_faces(h);
    if (s != UAAMG_OK) return s;
    cudaError_t e = cudaMemcpyAsync(h->d_face[0], u, h->face_n[0] * sizeof(double), cudaMemcpyHostToDevice,
                                    h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->d_face[1], v, h->face_n[1] * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "upload");
    s = static_dev(h, h->d_face[0], h->d_face[1], h->d_p, opts, stats);
    if (!solved(s)) return s;
    e = cudaMemcpyAsync(p, h->d_p, h->n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "download");
    return s;
}

}  // extern "C"
