// Test infrastructure only: a C-ABI shim around the reference's OWN CUDA 3D solver
// (CudaPCG3D, include/solver/cuda/cuda_pcg_3d.h), compiled together with the
// reference's unmodified CUDA sources by `make -C oracle ref-gpu` into
// oracle/_ref/libuaamg_ref_gpu.so.  It times the reference's GPU path on the same
// device as this library, as a second reference beside its CPU solver; nothing in
// the product links it.
//
// Reference code driven here:
//   CudaGrid3D::allocate                     include/solver/cuda/cuda_common_3d.h:17-37
//   CudaPCG3D::solve_optimized               src/solver/cuda/cuda_pcg_3d_opt.cu:335-433
//   CudaPCG3D::solve_mixed (FP32 V-cycle)    src/solver/cuda/cuda_pcg_3d_opt.cu:326-330
// Both stop on ||r|| / ||r0|| < tol with r0 the zero-mean, negated right-hand side,
// which for a cold start is the relative rule ||r|| < tol ||b|| of this library.
#include "solver/cuda/cuda_pcg_3d.h"

#include <cuda_runtime.h>

#include <cstdint>

extern "C" {

// One 3D problem solved `reps` times (after one untimed solve) by the reference's GPU
// PCG: mode 0 solve_optimized (FP64), 1 solve_mixed (FP32 V-cycle).  solid, rhs and p
// are padded (nx+2)(ny+2)(nz+2) HOST arrays; p receives the last solution.  ms_out:
// mean CUDA-event time of one solve (device work and the solver's own host syncs);
// iters_out / relres_out: the solver's last_iters / last_rel_res.  Returns 0, or a
// CUDA error code.
int ref_gpu_pcg3d(int nx, int ny, int nz, double dx, double dy, double dz,
                  const uint8_t* solid, const double* rhs, double* p, int max_iter, double tol,
                  int mode, int reps, double* ms_out, int* iters_out, double* relres_out) {
    const size_t n = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    CudaGrid3D g;
    g.allocate(nx, ny, nz, dx, dy, dz);
    double *d_rhs = nullptr, *d_p = nullptr;
    cudaError_t e = cudaMalloc(&d_rhs, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_p, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(g.solid, solid, n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_rhs, rhs, n * sizeof(double), cudaMemcpyHostToDevice);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    CudaPCG3D pcg;
    float total = 0.0f;
    for (int r = 0; e == cudaSuccess && r <= reps; ++r) {
        cudaMemset(d_p, 0, n * sizeof(double));
        cudaEventRecord(t0);
        if (mode == 1) pcg.solve_mixed(g, d_p, d_rhs, max_iter, tol);
        else pcg.solve_optimized(g, d_p, d_rhs, max_iter, tol);
        cudaEventRecord(t1);
        e = cudaEventSynchronize(t1);
        if (e == cudaSuccess) e = cudaGetLastError();
        float ms = 0.0f;
        if (e == cudaSuccess && r > 0) {
            cudaEventElapsedTime(&ms, t0, t1);
            total += ms;
        }
    }
    if (e == cudaSuccess) e = cudaMemcpy(p, d_p, n * sizeof(double), cudaMemcpyDeviceToHost);
    if (ms_out) *ms_out = reps > 0 ? total / reps : 0.0;
    if (iters_out) *iters_out = pcg.last_iters;
    if (relres_out) *relres_out = pcg.last_rel_res;
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(d_rhs);
    cudaFree(d_p);
    g.free();
    return (int)e;
}

}  // extern "C"
