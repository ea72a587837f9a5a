// Shared device-side definitions of the B200 UAAMG-PCG engine.
//
// Memory layout (the reference's, include/core/mesh_3d.h:38 and mesh.h:35): every
// per-cell array of a level is ghost-padded and column-major with i fastest,
// id = i + j*(nx+2) + k*(nx+2)*(ny+2).  2D levels have no z ghosts: the interior
// is the single plane k = 0.  Ghost entries of vectors and coefficient channels
// stay 0, which is what makes Neumann walls need no special-casing in the
// V-cycle kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace uaamg {

// Cell code bits (one byte a cell, vec.cuh k_codes): interior fluid cell, colour
// (i + j + k odd); on the finest level bits 0-5 mark the +x,-x,+y,-y,+z,-z
// neighbours that are interior fluid cells.
constexpr uint32_t kActive = 64u, kOdd = 128u;

struct Geom {
    int nx, ny, nz;  // interior cells; nz == 0 for a 2D level
    int sx, sxy;     // strides in cells: sx = nx+2, sxy = (nx+2)(ny+2)
    int n;           // padded cell count
};

// The reference's layout: row pitch nx+2.
inline Geom make_geom(int dim, int nx, int ny, int nz) {
    Geom g;
    g.nx = nx; g.ny = ny; g.nz = dim == 3 ? nz : 0;
    g.sx = nx + 2;
    g.sxy = (nx + 2) * (ny + 2);
    g.n = dim == 3 ? g.sxy * (nz + 2) : g.sxy;
    return g;
}

// The engines' internal layout: the same ghost-padded i-fastest order with the row
// pitch rounded up to a multiple of 16 cells, so every row of every array starts
// on a 16-byte boundary (a tensor-map requirement for TMA, and 128-bit loads).
// Columns nx+2 .. sx-1 are padding and stay 0.
constexpr int kPitchAlign = 16;
inline Geom make_geom_pitched(int dim, int nx, int ny, int nz) {
    Geom g = make_geom(dim, nx, ny, nz);
    g.sx = (nx + 2 + kPitchAlign - 1) / kPitchAlign * kPitchAlign;
    g.sxy = g.sx * (ny + 2);
    g.n = dim == 3 ? g.sxy * (nz + 2) : g.sxy;
    return g;
}

// Run status written by the device-side finalisers (CGState::status).
enum : int {
    CG_RUNNING = 0,
    CG_CONVERGED = 1,
    CG_MAXITER = 2,
    CG_BREAKDOWN = 3,
    CG_NAN = 4,
};

// Device-resident PCG state.  All scalars are FP64; the loop never copies a
// scalar to the host: alpha/beta/stopping decisions are taken by the last block
// of the kernel that finishes each reduction.
struct CGState {
    double rz_old;     // r.z of the previous iteration
    double pap;        // p.Ap
    double alpha, beta;
    double rr;         // recursive r.r
    double rr_true;    // FP64 true residual b - A x (residual replacement / exit)
    double r0;         // ||r0||
    double tol_abs;    // stop when sqrt(r.r) < tol_abs
    double mean_z;     // fluid mean of z (null-space projection)
    double nfluid;     // fluid cell count
    double sum0, sum1; // scratch sums (RHS normalisation)
    double bnorm;      // ||b|| of the normalised right-hand side
    double breakdown;  // p.Ap below this stops the solve (the reference's 1e-15)
    int done;          // 1 once the solve stopped; every loop kernel then returns at once
    int status;        // CG_* above
    int iter;          // completed x/r updates
    int cand;          // mixed mode: recursive residual met tol, confirm with the true one
    int max_iter;
    int replace_every; // mixed mode residual-replacement period (0 = off)
    int replacements;  // replacements performed
    int dirichlet;     // 1: no null space (skip mean projections)
    int init;          // 1 while forming p0 = z0 (beta = 0)
    int fold;          // mixed mode: the next x update first folds x_lo into x_hi
    unsigned int counter[8];  // last-block counters, one per reduction site
};

// q = a / d and r = a % d for 0 <= a < 2^31, 0 < d, from a reciprocal 1/d computed
// once (rd): the double-precision estimate is off by at most one and one exact
// correction step fixes it.  A fraction of the instructions of an integer division
// by a value known only at run time, which the grid-stride walks would otherwise
// pay per item.
__device__ __forceinline__ int divmod_rcp(int a, int d, double rd, int& r) {
    int q = (int)((double)a * rd);
    r = a - q * d;
    if (r < 0) { --q; r += d; }
    else if (r >= d) { ++q; r -= d; }
    return q;
}

// Programmatic dependent launch: the engine launches its kernels so that each may
// be scheduled while its predecessor on the stream is still finishing.  Every
// kernel therefore first waits until the preceding grid has completed and its
// memory operations are visible (a no-op when it was launched without the
// attribute), and then lets its own successor be launched.
__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Host-visible launch helpers ------------------------------------------------

template <int DIM>
inline dim3 cell_block() { return DIM == 3 ? dim3(32, 4, 2) : dim3(32, 8, 1); }

template <int DIM>
inline dim3 cell_grid(int nx, int ny, int nz) {
    dim3 b = cell_block<DIM>();
    return dim3((nx + b.x - 1) / b.x, (ny + b.y - 1) / b.y,
                DIM == 3 ? (nz + b.z - 1) / b.z : 1);
}

inline size_t grid_blocks(dim3 g) { return (size_t)g.x * g.y * g.z; }

}  // namespace uaamg
