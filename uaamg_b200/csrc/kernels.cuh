// Device kernels of the B200 UAAMG-PCG engine, templated on the dimension (2 or 3)
// and the arithmetic type T (double for the reference-exact mode, float for the
// FP32 and mixed modes).  Included by kernels_f64.cu (built with -fmad=false so
// every a*b+c rounds twice, as the reference's x86-64 build does) and by
// kernels_f32.cu; everything here has internal linkage so each translation unit
// owns its copy.
//
// Reference algorithm (A-006/UAAMGPCG, src/solver/preconditioner/
// uaamg_preconditioner_3d.cpp and uaamg_preconditioner.cpp; src/solver/pcg_3d.cpp
// and pcg.cpp).  Per-cell arithmetic follows the reference's operation order so the
// FP64 mode reproduces it bit for bit; reductions are FP64, deterministic
// (fixed block partials + fixed-order last-block sum) but ordered differently
// from the reference's sequential loops.
#pragma once
#include "common.cuh"

namespace uaamg {
namespace {

// ---------------------------------------------------------------------------
// helpers

template <int DIM>
__device__ __forceinline__ bool thread_cell(const Geom& g, int& i, int& j, int& k) {
    i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    j = 1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
    k = DIM == 3 ? 1 + (int)(blockIdx.z * blockDim.z + threadIdx.z) : 0;
    return i <= g.nx && j <= g.ny && (DIM == 2 || k <= g.nz);
}

__device__ __forceinline__ int cidx(const Geom& g, int i, int j, int k) {
    return i + j * g.sx + k * g.sxy;
}

// Deterministic block + grid reduction of NV FP64 values.  Every thread of every
// block must call it (out-of-range threads contribute 0).  Each block writes its
// partial sums to partials[block*NV + q]; the last block to arrive (atomic
// counter) re-reads all partials in a fixed order and returns true in its thread 0
// with the totals in tot.  The counter is reset for the next launch.
template <int NV>
__device__ __forceinline__ bool reduce_last(double (&v)[NV], double* partials,
                                            unsigned int* counter, double (&tot)[NV]) {
    __shared__ double sm[32][NV];
    __shared__ int am_last;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, warp = tid >> 5, nwarp = (nthr + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q)
        for (int off = 16; off > 0; off >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], off);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) sm[warp][q] = v[q];
    __syncthreads();
    const unsigned nblk = gridDim.x * gridDim.y * gridDim.z;
    const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = 0.0;
            for (int w = 0; w < nwarp; ++w) s += sm[w][q];
            partials[(size_t)bid * NV + q] = s;
        }
        __threadfence();
        unsigned prev = atomicAdd(counter, 1u);
        am_last = (prev == nblk - 1) ? 1 : 0;
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] = 0.0;
    // partials b = tid, tid + nthr, ... added in that order; the loads of four are
    // issued together (a launch of thousands of blocks would otherwise pay one L2
    // round trip per partial here, in one block, at its end)
    unsigned b = tid;
    for (; b + 3 * nthr < nblk; b += 4 * nthr) {
        double t[4][NV];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int q = 0; q < NV; ++q) t[u][q] = __ldcg(&partials[(size_t)(b + u * nthr) * NV + q]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int q = 0; q < NV; ++q) acc[q] += t[u][q];
    }
    for (; b < nblk; b += nthr)
#pragma unroll
        for (int q = 0; q < NV; ++q) acc[q] += __ldcg(&partials[(size_t)b * NV + q]);
#pragma unroll
    for (int q = 0; q < NV; ++q)
        for (int off = 16; off > 0; off >>= 1) acc[q] += __shfl_down_sync(0xffffffffu, acc[q], off);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; ++q) sm[warp][q] = acc[q];
    __syncthreads();
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = 0.0;
            for (int w = 0; w < nwarp; ++w) s += sm[w][q];
            tot[q] = s;
        }
        *counter = 0u;
        return true;
    }
    return false;
}

// ---------------------------------------------------------------------------
// Hierarchy set-up

// Coarse cell solid iff at least half of its 2^DIM children are solid
// (uaamg_preconditioner_3d.cpp:34-45; uaamg_preconditioner.cpp:43-53).
template <int DIM>
__global__ void k_restrict_solid(Geom f, const uint8_t* __restrict__ fs, Geom c,
                                 uint8_t* __restrict__ cs) {
    pdl_entry();
    int ic, jc, kc;
    if (!thread_cell<DIM>(c, ic, jc, kc)) return;
    const int i_f = 2 * ic - 1, j_f = 2 * jc - 1, k_f = DIM == 3 ? 2 * kc - 1 : 0;
    int sc = 0;
#pragma unroll
    for (int di = 0; di < 2; ++di)
#pragma unroll
        for (int dj = 0; dj < 2; ++dj)
#pragma unroll
            for (int dk = 0; dk < (DIM == 3 ? 2 : 1); ++dk)
                sc += fs[cidx(f, i_f + di, j_f + dj, k_f + dk)] != 0;
    cs[cidx(c, ic, jc, kc)] = (uint8_t)(2 * sc >= (DIM == 3 ? 8 : 4));
}

// Finest-level couplings from the mask (uaamg_preconditioner_3d.cpp:50-66):
// cx[c] = h_x^-2 when c and c+e_x are fluid and i < nx.  Channels are zeroed
// beforehand.  wd (optional) is the Dirichlet-wall diagonal channel.
template <int DIM, class T>
__global__ void k_fine_coeffs(Geom g, const uint8_t* __restrict__ s, T* cx, T* cy, T* cz, T* wd,
                              T idx2, T idy2, T idz2) {
    pdl_entry();
    int i, j, k;
    if (!thread_cell<DIM>(g, i, j, k)) return;
    const int id = cidx(g, i, j, k);
    if (s[id]) return;
    if (i < g.nx && !s[id + 1]) cx[id] = idx2;
    if (j < g.ny && !s[id + g.sx]) cy[id] = idy2;
    if (DIM == 3 && k < g.nz && !s[id + g.sxy]) cz[id] = idz2;
    if (wd) {
        T w = T(0);
        if (i == 1) w += T(2) * idx2;
        if (i == g.nx) w += T(2) * idx2;
        if (j == 1) w += T(2) * idy2;
        if (j == g.ny) w += T(2) * idy2;
        if (DIM == 3 && k == 1) w += T(2) * idz2;
        if (DIM == 3 && k == g.nz) w += T(2) * idz2;
        wd[id] = w;
    }
}

// Galerkin coarse couplings (uaamg_preconditioner_3d.cpp:81-106): the coarse +x
// coupling is the sum of the fine +x couplings across the shared face, summed in
// the reference's (dj, dk) order.  The wall channel sums over all children.
template <int DIM, class T>
__global__ void k_galerkin(Geom f, const T* __restrict__ fcx, const T* __restrict__ fcy,
                           const T* __restrict__ fcz, const T* __restrict__ fwd, Geom c,
                           const uint8_t* __restrict__ cs, T* ccx, T* ccy, T* ccz, T* cwd) {
    pdl_entry();
    int ic, jc, kc;
    if (!thread_cell<DIM>(c, ic, jc, kc)) return;
    const int id = cidx(c, ic, jc, kc);
    if (cs[id]) return;
    const int i_f = 2 * ic - 1, j_f = 2 * jc - 1, k_f = DIM == 3 ? 2 * kc - 1 : 0;
    constexpr int KC = DIM == 3 ? 2 : 1;
    T sx = T(0), sy = T(0), sz = T(0), sw = T(0);
    for (int dj = 0; dj < 2; ++dj)
        for (int dk = 0; dk < KC; ++dk) sx += fcx[cidx(f, i_f + 1, j_f + dj, k_f + dk)];
    for (int di = 0; di < 2; ++di)
        for (int dk = 0; dk < KC; ++dk) sy += fcy[cidx(f, i_f + di, j_f + 1, k_f + dk)];
    if (DIM == 3)
        for (int di = 0; di < 2; ++di)
            for (int dj = 0; dj < 2; ++dj) sz += fcz[cidx(f, i_f + di, j_f + dj, k_f + 1)];
    if (cwd) {
        for (int di = 0; di < 2; ++di)
            for (int dj = 0; dj < 2; ++dj)
                for (int dk = 0; dk < KC; ++dk) sw += fwd[cidx(f, i_f + di, j_f + dj, k_f + dk)];
        cwd[id] = sw;
    }
    ccx[id] = sx;
    ccy[id] = sy;
    if (DIM == 3) ccz[id] = sz;
}

// Level arrays as seen by the V-cycle kernels.
template <class T>
struct LevelView {
    Geom g;
    const uint8_t* solid;
    const T* cx;
    const T* cy;
    const T* cz;
    const T* wd;  // nullptr unless Dirichlet walls
    T* x;
    const T* b;
};

// Diagonal in the reference's summation order (uaamg_preconditioner_3d.cpp:72-74).
template <int DIM, class T>
__device__ __forceinline__ T diag_at(const LevelView<T>& L, int id) {
    T d = L.cx[id] + L.cx[id - 1] + L.cy[id] + L.cy[id - L.g.sx];
    if (DIM == 3) d = d + L.cz[id] + L.cz[id - L.g.sxy];
    if (L.wd) d = d + L.wd[id];
    return d;
}

// ---------------------------------------------------------------------------
// V-cycle kernels

// One colour of red-black Gauss-Seidel (uaamg_preconditioner_3d.cpp:123-138):
// x = (b + sum c*x_nb)/diag on cells with (i+j+k)&1 == parity, skipping solid
// cells and diag < 1e-30.  One thread per x-pair of cells.
template <int DIM, class T>
__global__ void k_sweep(LevelView<T> L, int parity, const int* __restrict__ done) {
    pdl_entry();
    if (done && *done) return;
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = 1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
    const int k = DIM == 3 ? 1 + (int)(blockIdx.z * blockDim.z + threadIdx.z) : 0;
    if (j > L.g.ny || (DIM == 3 && k > L.g.nz)) return;
    const int i0 = (((1 + j + k) & 1) == parity) ? 1 : 2;
    const int i = i0 + 2 * t;
    if (i > L.g.nx) return;
    const int id = cidx(L.g, i, j, k);
    if (L.solid[id]) return;
    const T d = diag_at<DIM>(L, id);
    if (d < T(1e-30)) return;
    const int sx = L.g.sx, sxy = L.g.sxy;
    T nb = L.cx[id] * L.x[id + 1] + L.cx[id - 1] * L.x[id - 1]
         + L.cy[id] * L.x[id + sx] + L.cy[id - sx] * L.x[id - sx];
    if (DIM == 3) nb = nb + L.cz[id] * L.x[id + sxy] + L.cz[id - sxy] * L.x[id - sxy];
    L.x[id] = (L.b[id] + nb) / d;
}

// Residual restriction b_c = sum over fluid children of (b - A x)
// (uaamg_preconditioner_3d.cpp:144-165).  One thread per coarse cell.
template <int DIM, class T>
__global__ void k_restrict(LevelView<T> F, Geom cg, const uint8_t* __restrict__ cs, T* cb,
                           const int* __restrict__ done) {
    pdl_entry();
    if (done && *done) return;
    int ic, jc, kc;
    if (!thread_cell<DIM>(cg, ic, jc, kc)) return;
    const int cid = cidx(cg, ic, jc, kc);
    if (cs[cid]) return;
    const int i_f = 2 * ic - 1, j_f = 2 * jc - 1, k_f = DIM == 3 ? 2 * kc - 1 : 0;
    const int sx = F.g.sx, sxy = F.g.sxy;
    T sum = T(0);
    for (int di = 0; di < 2; ++di)
        for (int dj = 0; dj < 2; ++dj)
            for (int dk = 0; dk < (DIM == 3 ? 2 : 1); ++dk) {
                const int fid = cidx(F.g, i_f + di, j_f + dj, k_f + dk);
                if (F.solid[fid]) continue;
                const T d = diag_at<DIM>(F, fid);
                T ax = d * F.x[fid] - F.cx[fid] * F.x[fid + 1] - F.cx[fid - 1] * F.x[fid - 1]
                     - F.cy[fid] * F.x[fid + sx] - F.cy[fid - sx] * F.x[fid - sx];
                if (DIM == 3) ax = ax - F.cz[fid] * F.x[fid + sxy] - F.cz[fid - sxy] * F.x[fid - sxy];
                sum += F.b[fid] - ax;
            }
    cb[cid] = sum;
}

// Prolongation x_f += 2 x_c for fluid coarse/fluid fine cells
// (uaamg_preconditioner_3d.cpp:168-181).
template <int DIM, class T>
__global__ void k_prolong(Geom cg, const uint8_t* __restrict__ cs, const T* __restrict__ cx_,
                          Geom fg, const uint8_t* __restrict__ fs, T* fx,
                          const int* __restrict__ done) {
    pdl_entry();
    if (done && *done) return;
    int ic, jc, kc;
    if (!thread_cell<DIM>(cg, ic, jc, kc)) return;
    const int cid = cidx(cg, ic, jc, kc);
    if (cs[cid]) return;
    const T val = T(2) * cx_[cid];
    const int i_f = 2 * ic - 1, j_f = 2 * jc - 1, k_f = DIM == 3 ? 2 * kc - 1 : 0;
    for (int di = 0; di < 2; ++di)
        for (int dj = 0; dj < 2; ++dj)
            for (int dk = 0; dk < (DIM == 3 ? 2 : 1); ++dk) {
                const int fid = cidx(fg, i_f + di, j_f + dj, k_f + dk);
                if (!fs[fid]) fx[fid] += val;
            }
}

// Coarsest level: 10 x (forward + reverse) RBGS sweeps (uaamg_preconditioner_3d.cpp:
// 185-186) in ONE block; colours are separated by __syncthreads, which makes the
// block's global-memory writes visible to all its threads.
template <int DIM, class T>
__global__ void k_coarsest(LevelView<T> L, const int* __restrict__ done) {
    pdl_entry();
    if (done && *done) return;
    const int nx = L.g.nx, ny = L.g.ny, nzi = DIM == 3 ? L.g.nz : 1;
    const int ncell = nx * ny * nzi;
    const int sx = L.g.sx, sxy = L.g.sxy;
    for (int s = 0; s < 10; ++s)
        for (int h = 0; h < 4; ++h) {
            const int parity = (h == 0 || h == 3) ? 1 : 0;  // fwd: 1,0  rev: 0,1
            for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
                const int i = 1 + c % nx;
                const int j = 1 + (c / nx) % ny;
                const int k = DIM == 3 ? 1 + c / (nx * ny) : 0;
                if (((i + j + k) & 1) != parity) continue;
                const int id = cidx(L.g, i, j, k);
                if (L.solid[id]) continue;
                const T d = diag_at<DIM>(L, id);
                if (d < T(1e-30)) continue;
                T nb = L.cx[id] * L.x[id + 1] + L.cx[id - 1] * L.x[id - 1]
                     + L.cy[id] * L.x[id + sx] + L.cy[id - sx] * L.x[id - sx];
                if (DIM == 3) nb = nb + L.cz[id] * L.x[id + sxy] + L.cz[id - sxy] * L.x[id - sxy];
                L.x[id] = (L.b[id] + nb) / d;
            }
            __syncthreads();
        }
}

// ---------------------------------------------------------------------------
// PCG kernels

struct Stencil {
    double idx2, idy2, idz2, diag;
    int dirichlet;
    // 2D variable-coefficient operator (Grid::lap_diag / lap_off_x / lap_off_y,
    // include/core/grid.h:23-31), the caller's padded arrays in the reference
    // layout (index i + j * vsx); vd == nullptr: the uniform operator
    int vsx;
    const double* __restrict__ vd;
    const double* __restrict__ vox;
    const double* __restrict__ voy;
    // FP32 forms: per-cell copies in the level's own layout (index id) of
    // s = d + 2 ox + 2 oy, ox and oy, for the difference form of the operator
    const float* __restrict__ fs;
    const float* __restrict__ fx;
    const float* __restrict__ fy;
};


// The variable-coefficient branch of PCG::solve's operator (pcg.cpp:35-46):
// A v = d v_C + ox (v_L + v_R) + oy (v_B + v_T) with the same neighbour rule as the
// uniform operator, summed in the reference's order.
template <class T>
__device__ __forceinline__ T var_op(const Stencil& st, int i, int j, T vc, T vL, T vR, T vB, T vT) {
    const long long q = i + (long long)j * st.vsx;
    return (T)st.vd[q] * vc + (T)st.vox[q] * (vL + vR) + (T)st.voy[q] * (vB + vT);
}

// Reference PCG operator (pcg_3d.cpp:38-55, pcg.cpp:47-59): a solid or out-of-domain
// neighbour reads p_C (Neumann; -p_C for a Dirichlet wall); solid rows are 0.
template <int DIM, class T>
__device__ __forceinline__ T apply_A(const Geom& g, const uint8_t* __restrict__ s,
                                     const T* __restrict__ v, int i, int j, int k, int id,
                                     T idx2, T idy2, T idz2, T diag, int dirichlet) {
    const T vc = v[id];
    const T wall = dirichlet ? -vc : vc;
    const int sx = g.sx, sxy = g.sxy;
    const T vL = i > 1 ? (!s[id - 1] ? v[id - 1] : vc) : wall;
    const T vR = i < g.nx ? (!s[id + 1] ? v[id + 1] : vc) : wall;
    const T vB = j > 1 ? (!s[id - sx] ? v[id - sx] : vc) : wall;
    const T vT = j < g.ny ? (!s[id + sx] ? v[id + sx] : vc) : wall;
    if (DIM == 3) {
        const T vF = k > 1 ? (!s[id - sxy] ? v[id - sxy] : vc) : wall;
        const T vK = k < g.nz ? (!s[id + sxy] ? v[id + sxy] : vc) : wall;
        return diag * vc - (vL + vR) * idx2 - (vB + vT) * idy2 - (vF + vK) * idz2;
    }
    return diag * vc - (vL + vR) * idx2 - (vB + vT) * idy2;
}

// Grid-stride walk over the interior in rows of 32 cells along x: a warp owns 32
// consecutive cells of one row.  Blocks are (32, 8); the grid is capped at a few
// blocks per SM, which keeps a reduction's last-block combine short.
template <int DIM, class F>
__device__ __forceinline__ void for_cells(const Geom& g, F&& f) {
    const int nxc = (g.nx + 31) >> 5;
    const int nrows = g.ny * (DIM == 3 ? g.nz : 1);
    const int nitems = nrows * nxc;  // < 2^26: padded grids have fewer than 2^31 cells
    const double rx = 1.0 / nxc, ry = 1.0 / g.ny;
    for (int it = (int)(blockIdx.x * blockDim.y + threadIdx.y); it < nitems;
         it += (int)(gridDim.x * blockDim.y)) {
        int ch, jr = 0;
        const int row = divmod_rcp(it, nxc, rx, ch);
        const int i = 1 + (ch << 5) + (int)threadIdx.x;
        if (i > g.nx) continue;
        int kr = 0;
        if (DIM == 3) kr = divmod_rcp(row, g.ny, ry, jr);
        else jr = row;
        f(i, 1 + jr, DIM == 3 ? 1 + kr : 0, cidx(g, i, 1 + jr, DIM == 3 ? 1 + kr : 0));
    }
}

// s = d + 2 ox + 2 oy (FP64), ox, oy of every interior cell as FP32 in the level's
// layout, from the caller's padded arrays (reference layout, row stride st.vsx).
__global__ void k_var_coeffs(Geom g, Stencil st, float* fs, float* fx, float* fy) {
    pdl_entry();
    for_cells<2>(g, [&](int i, int j, int, int id) {
        const long long q = i + (long long)j * st.vsx;
        const double d = st.vd[q], ox = st.vox[q], oy = st.voy[q];
        fs[id] = (float)(d + 2.0 * ox + 2.0 * oy);
        fx[id] = (float)ox;
        fy[id] = (float)oy;
    });
}

// Sum and count over fluid interior cells of a FP64 field: cg->sum0, cg->nfluid.
template <int DIM>
__global__ void k_sum_count(Geom g, const uint8_t* __restrict__ s, const double* __restrict__ v,
                            double* partials, CGState* cg, int slot) {
    pdl_entry();
    double acc[2] = {0.0, 0.0};
    for_cells<DIM>(g, [&](int, int, int, int id) {
        if (!s[id]) { acc[0] += v[id]; acc[1] += 1.0; }
    });
    double tot[2];
    if (reduce_last<2>(acc, partials, &cg->counter[slot], tot)) {
        cg->sum0 = tot[0];
        cg->nfluid = tot[1];
    }
}

// b = -(rhs - mean) on fluid interior cells, 0 elsewhere (pcg_3d.cpp:22-36);
// mean = sum0/nfluid unless Dirichlet.  b may alias rhs (each cell reads its own
// value before writing it).
template <int DIM>
__global__ void k_rhs_negate(Geom g, const uint8_t* __restrict__ s, const double* rhs, double* b,
                             const CGState* cg) {
    pdl_entry();
    double mean = cg->nfluid > 0.0 ? cg->sum0 / cg->nfluid : 0.0;
    if (cg->dirichlet) mean = 0.0;
    for_cells<DIM>(g, [&](int, int, int, int id) {
        b[id] = s[id] ? 0.0 : -(rhs[id] - mean);
    });
}

// v -= mean over fluid cells (pcg_3d.cpp:66-77), mean = sum0/nfluid.
template <int DIM>
__global__ void k_sub_mean(Geom g, const uint8_t* __restrict__ s, double* v, const CGState* cg) {
    pdl_entry();
    if (cg->dirichlet) return;
    const double mean = cg->nfluid > 0.0 ? cg->sum0 / cg->nfluid : 0.0;
    for_cells<DIM>(g, [&](int, int, int, int id) {
        if (!s[id]) v[id] -= mean;
    });
}

// The last block's bookkeeping of a true residual r.r (rr): mode 0 the initial
// residual (r0, the absolute tolerance); mode 1 a residual replacement; 2 and 3
// record it only.
__device__ __forceinline__ void true_residual_done(CGState* cg, double rr, int mode, double tol,
                                                   int tol_mode) {
    cg->rr_true = rr;
    if (mode == 0) {
        cg->r0 = sqrt(rr);
        cg->rr = rr;
        cg->tol_abs = tol_mode ? tol * cg->bnorm : tol;
        if (rr == 0.0) { cg->status = CG_CONVERGED; cg->done = 1; }  // b = 0: x = 0 exactly
    } else if (mode == 1) {
        // a true residual more than twice the recursive one means the FP32
        // recurrence drifted: the next search direction restarts (beta = 0),
        // since beta = r.z / r.z_old would mix the replaced residual with
        // directions built for the drifted one
        if (rr > 4.0 * cg->rr) cg->init = 1;
        cg->rr = rr;
        cg->replacements += 1;
        if (cg->cand) {
            cg->cand = 0;
            if (sqrt(rr) < cg->tol_abs) { cg->status = CG_CONVERGED; cg->done = 1; }
        }
        if (!(rr == rr)) { cg->status = CG_NAN; cg->done = 1; }
    }
}

// Mixed-mode residual replacement due now: every replace_every iterations, or when
// the recursive residual met the tolerance (a candidate to confirm).
__device__ __forceinline__ bool replacement_due(const CGState* cg) {
    return !cg->done && (cg->cand || (cg->replace_every > 0 && cg->iter > 0 &&
                                      cg->iter % cg->replace_every == 0));
}

// r = b - A x (FP64), copied into the working residual rw (type T), with
// ||r||^2 reduced.  mode 0: initial residual (sets r0, and tol_abs = tol or
// tol*||b|| for the relative rule, ||b|| being the RHS norm, not ||r0||);
// mode 1: residual replacement; mode 2: exit diagnostics only (the solve loop and
// its exit use k_resid_x64 for both); mode 3: plain b <- b - A x for a warm start (rw may alias b: each cell reads
// its own b before writing it).  When x == nullptr the residual is b itself.
template <int DIM, class T>
__global__ void k_true_residual(Geom g, const uint8_t* __restrict__ s, const double* b,
                                const double* __restrict__ x, T* rw, Stencil st, double* partials,
                                CGState* cg, int slot, int mode, double tol, int tol_mode) {
    pdl_entry();
    if (mode == 1 && !replacement_due(cg)) return;
    double acc[1] = {0.0};
    for_cells<DIM>(g, [&](int i, int j, int k, int id) {
        if (!s[id]) {
            double r = b[id];
            if (x && DIM == 2 && st.vd) {
                const double vc = x[id], wall = st.dirichlet ? -vc : vc;
                const double vL = i > 1 ? (!s[id - 1] ? x[id - 1] : vc) : wall;
                const double vR = i < g.nx ? (!s[id + 1] ? x[id + 1] : vc) : wall;
                const double vB = j > 1 ? (!s[id - g.sx] ? x[id - g.sx] : vc) : wall;
                const double vT = j < g.ny ? (!s[id + g.sx] ? x[id + g.sx] : vc) : wall;
                r = r - var_op<double>(st, i, j, vc, vL, vR, vB, vT);
            } else if (x) {
                r = r - apply_A<DIM, double>(g, s, x, i, j, k, id, st.idx2, st.idy2, st.idz2,
                                             st.diag, st.dirichlet);
            }
            if (rw) rw[id] = (T)r;
            acc[0] += r * r;
        } else if (rw) {
            rw[id] = T(0);
        }
    });
    double tot[1];
    if (reduce_last<1>(acc, partials, &cg->counter[slot], tot))
        true_residual_done(cg, tot[0], mode, tol, tol_mode);
}

// FP64 true residual r = b - A x of the finest level with x = x_hi + x_lo (either
// part may be absent), the reference's operator (pcg_3d.cpp:38-55: a neighbour that
// is not an interior fluid cell reads x_C, or -x_C across a Dirichlet wall),
// neighbours from the cell codes.  A block of 32 x 8 threads takes tiles of as many
// (i, j) columns and zc planes in turn (the grid is a few blocks per SM, so a
// launch with no replacement due ends quickly); a thread walks its column's planes,
// keeping x of the planes below, at and above in registers; every load of a step
// is independent of the others.  Writes r as T to rw (0 on solid cells) when
// given, reduces r.r; mode 1 (residual replacement, gated as replacement_due) also
// asks the next x update to fold x_lo into x_hi; mode 2: exit diagnostics.
template <int DIM, class T>
__global__ void __launch_bounds__(256) k_resid_x64(Geom g, const uint8_t* __restrict__ code,
                                                   const double* __restrict__ b,
                                                   const double* __restrict__ xhi,
                                                   const T* __restrict__ xlo, T* __restrict__ rw,
                                                   Stencil st, int zc, double* partials, CGState* cg,
                                                   int slot, int mode, double tol, int tol_mode) {
    pdl_entry();
    if (mode == 1 && !replacement_due(cg)) return;
    double acc[1] = {0.0};
    const int tx = (g.nx + 31) / 32, ty = (g.ny + 7) / 8, tz = DIM == 3 ? (g.nz + zc - 1) / zc : 1;
    for (int w = blockIdx.x; w < tx * ty * tz; w += gridDim.x) {
        const int i = 1 + 32 * (w % tx) + (int)threadIdx.x;
        const int j = 1 + 8 * ((w / tx) % ty) + (int)threadIdx.y;
        if (i > g.nx || j > g.ny) continue;
        const int kb = DIM == 3 ? 1 + (w / (tx * ty)) * zc : 0;
        const int ke = DIM == 3 ? min(kb + zc, g.nz + 1) : 1;
        auto X = [&](int q) -> double {
            if (xhi && xlo) return xhi[q] + (double)xlo[q];
            return xhi ? xhi[q] : (double)xlo[q];
        };
        const double idx2 = st.idx2, idy2 = st.idy2, idz2 = st.idz2, diag = st.diag;
        const int sx = g.sx, sxy = g.sxy;
        int id = cidx(g, i, j, kb);
        double xm = DIM == 3 ? X(id - sxy) : 0.0, xc = X(id);
        for (int k = kb; k < ke; ++k, id += sxy) {
            const double xp = DIM == 3 ? X(id + sxy) : 0.0;
            const uint32_t c = code[id];
            const double bb = b[id];
            const double xl = X(id - 1), xr = X(id + 1), xb = X(id - sx), xt = X(id + sx);
            const double wall = st.dirichlet ? -xc : xc;
            const double vL = (c & 2u) ? xl : (i > 1 ? xc : wall);
            const double vR = (c & 1u) ? xr : (i < g.nx ? xc : wall);
            const double vB = (c & 8u) ? xb : (j > 1 ? xc : wall);
            const double vT = (c & 4u) ? xt : (j < g.ny ? xc : wall);
            double ax;
            if (DIM == 3) {
                const double vF = (c & 32u) ? xm : (k > 1 ? xc : wall);
                const double vK = (c & 16u) ? xp : (k < g.nz ? xc : wall);
                ax = diag * xc - (vL + vR) * idx2 - (vB + vT) * idy2 - (vF + vK) * idz2;
            } else if (st.vd) {
                ax = (c & kActive) ? var_op<double>(st, i, j, xc, vL, vR, vB, vT) : 0.0;
            } else {
                ax = diag * xc - (vL + vR) * idx2 - (vB + vT) * idy2;
            }
            const double r = (c & kActive) ? bb - ax : 0.0;
            acc[0] += r * r;
            if (rw) rw[id] = (T)r;
            xm = xc;
            xc = xp;
        }
    }
    double tot[1];
    if (reduce_last<1>(acc, partials, &cg->counter[slot], tot)) {
        if (mode == 1) cg->fold = 1;
        true_residual_done(cg, tot[0], mode, tol, tol_mode);
        // a replacement at max_iter that did not confirm convergence ends the solve
        if (mode == 1 && !cg->done && cg->iter >= cg->max_iter) {
            cg->status = CG_MAXITER;
            cg->done = 1;
        }
    }
}

// 2D search direction, the same fused step as the z march k_pmatvec (march.cuh):
// p = (z - m) + beta p_old on fluid cells (pcg.cpp:113-122), Ap from the new p of
// the neighbours, formed on the fly (a solid or out-of-domain neighbour reads p_C;
// pcg.cpp:47-59), p.Ap reduced; the last block sets alpha = rz_old / p.Ap or stops
// on breakdown (pcg.cpp:97-99).  The operator is the uniform one, or with st.vd the
// variable-coefficient one, Ap = d p_C + ox (p_L + p_R) + oy (p_B + p_T)
// (pcg.cpp:35-46).  FP64 evaluates the reference's expressions (on its arrays);
// FP32 the difference forms (the variable one on FP32 copies st.fs, fx, fy).  In 2D
// a march has a single plane to pipeline, and this flat walk is the faster kernel.
// A thread owns the vertical pair (i, j), (i, j+1) -- j odd -- and a warp 32 such
// columns; every load of a step (z and p_old of the pair, its side neighbours and
// the rows below and above, codes, coefficients) is issued before any is used, the
// pair sharing its vertical neighbours.  Reads of ghost or solid cells are harmless
// (the padded arrays hold them) and discarded by the neighbour rule.  p_old and
// p_new are distinct buffers.
template <class T>
__global__ void __launch_bounds__(256) k_pmatvec_2d(Geom g, const uint8_t* __restrict__ code,
                                                     const T* __restrict__ z,
                                                     const T* __restrict__ pold,
                                                     T* __restrict__ pnew, T* __restrict__ ap,
                                                     Stencil st, double* partials, CGState* cg) {
    pdl_entry();
    if (cg->done) return;
    const T m = (T)cg->mean_z, beta = (T)cg->beta;
    const T idx2 = (T)st.idx2, idy2 = (T)st.idy2, diag = (T)st.diag;
    double acc[1] = {0.0};
    const int sx = g.sx;
    const int nxc = (g.nx + 31) >> 5;
    const int nitems = ((g.ny + 1) >> 1) * nxc;  // < 2^26
    const double rx = 1.0 / nxc;
    for (int it = (int)(blockIdx.x * blockDim.y + threadIdx.y); it < nitems;
         it += (int)(gridDim.x * blockDim.y)) {
        int ch;
        const int pr = divmod_rcp(it, nxc, rx, ch);
        const int i = 1 + (ch << 5) + (int)threadIdx.x;
        if (i > g.nx) continue;
        const int j = 1 + 2 * pr;
        const bool hb = j < g.ny;  // (i, j+1) is an interior cell
        const int id = cidx(g, i, j, 0);
        const int sb = hb ? sx : 0;            // second cell, or the first again
        const int s2 = hb ? 2 * sx : sx;       // the row above the pair (a ghost at most)
        // 0: below A, 1: A, 2: B (above A), 3: above B, 4/5: A -x/+x, 6/7: B -x/+x
        const int off[8] = {-sx, 0, sb, s2, -1, 1, sb - 1, sb + 1};
        T zz[8], qq[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            zz[e] = z[id + off[e]];
            qq[e] = pold[id + off[e]];
        }
        const uint32_t cc[2] = {code[id], code[id + sb]};
        const bool var = st.vd != nullptr;  // the same for the whole launch
        T k0[2] = {T(0), T(0)}, kx[2] = {T(0), T(0)}, ky[2] = {T(0), T(0)};
        if (!var) {
        } else if constexpr (sizeof(T) == 8) {
            const long long q = i + (long long)j * st.vsx, qb = hb ? st.vsx : 0;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                k0[e] = st.vd[q + e * qb];
                kx[e] = st.vox[q + e * qb];
                ky[e] = st.voy[q + e * qb];
            }
        } else {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                k0[e] = st.fs[id + e * sb];
                kx[e] = st.fx[id + e * sb];
                ky[e] = st.fy[id + e * sb];
            }
        }
        T pp[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) pp[e] = (zz[e] - m) + beta * qq[e];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            if (e == 1 && !hb) break;
            const uint32_t c = cc[e];
            const int jj = j + e, cid = id + e * sx;
            if (!(c & kActive)) {
                pnew[cid] = T(0);
                ap[cid] = T(0);
                continue;
            }
            const T p0 = pp[1 + e];
            const T wall = st.dirichlet ? -p0 : p0;
            const T vL = (c & 2u) ? pp[4 + 2 * e] : (i > 1 ? p0 : wall);
            const T vR = (c & 1u) ? pp[5 + 2 * e] : (i < g.nx ? p0 : wall);
            const T vB = (c & 8u) ? pp[e] : (jj > 1 ? p0 : wall);
            const T vT = (c & 4u) ? pp[2 + e] : (jj < g.ny ? p0 : wall);
            T a;
            if (!var) {
                // the march's expressions: the reference's in FP64, differences in FP32
                a = sizeof(T) == 8 ? diag * p0 - (vL + vR) * idx2 - (vB + vT) * idy2
                                   : ((p0 - vL) + (p0 - vR)) * idx2 + ((p0 - vB) + (p0 - vT)) * idy2;
            } else if constexpr (sizeof(T) == 8) {
                // the reference's expression and order
                a = k0[e] * p0 + kx[e] * (vL + vR) + ky[e] * (vB + vT);
            } else {
                // the same operator as (d + 2 ox + 2 oy) p_C - ox ((p_C - p_L) + (p_C - p_R))
                // - oy (...): no cancellation of O(1/h^2) terms in FP32
                a = k0[e] * p0 - kx[e] * ((p0 - vL) + (p0 - vR)) - ky[e] * ((p0 - vB) + (p0 - vT));
            }
            pnew[cid] = p0;
            ap[cid] = a;
            acc[0] += (double)p0 * (double)a;
        }
    }
    double tot[1];
    if (reduce_last<1>(acc, partials, &cg->counter[0], tot)) {
        const double pap = tot[0];
        cg->pap = pap;
        if (!(pap == pap)) { cg->status = CG_NAN; cg->done = 1; }
        else if (pap < cg->breakdown) { cg->status = CG_BREAKDOWN; cg->done = 1; }
        else cg->alpha = cg->rz_old / pap;
    }
}

// ||b||^2 over fluid cells -> cg->bnorm (FP64).
template <int DIM>
__global__ void k_norm(Geom g, const uint8_t* __restrict__ s, const double* __restrict__ b,
                       double* partials, CGState* cg, int slot) {
    pdl_entry();
    double acc[1] = {0.0};
    for_cells<DIM>(g, [&](int, int, int, int id) {
        if (!s[id]) acc[0] += b[id] * b[id];
    });
    double tot[1];
    if (reduce_last<1>(acc, partials, &cg->counter[slot], tot)) cg->bnorm = sqrt(tot[0]);
}

// Null-space projection of z and the new r.z (pcg_3d.cpp:112-123), given the
// fluid sums of z, r*z and r: with m = mean_fluid(z), r.(z - m) = r.z - m*sum(r).
// Sets beta = rz/rz_old (0 when forming p0) and rz_old = rz.
__device__ __forceinline__ void finish_zdot(CGState* cg, const double (&tot)[3]) {
    double m = 0.0, rz = tot[1];
    if (!cg->dirichlet) {
        m = cg->nfluid > 0.0 ? tot[0] / cg->nfluid : 0.0;
        rz = tot[1] - m * tot[2];
    }
    cg->mean_z = m;
    cg->beta = cg->init ? 0.0 : rz / cg->rz_old;
    cg->rz_old = rz;
    cg->init = 0;
    if (!(rz == rz)) { cg->status = CG_NAN; cg->done = 1; }
}

// The sums above as a separate pass (used with the per-level sweep V-cycle; the
// fused V-cycle computes them in its last kernel).
template <int DIM, class T>
__global__ void k_zdot(Geom g, const uint8_t* __restrict__ s, const T* __restrict__ r,
                       const T* __restrict__ z, double* partials, CGState* cg) {
    pdl_entry();
    if (cg->done) return;
    double acc[3] = {0.0, 0.0, 0.0};
    for_cells<DIM>(g, [&](int, int, int, int id) {
        if (!s[id]) {
            const double zv = (double)z[id], rv = (double)r[id];
            acc[0] += zv;
            acc[1] += rv * zv;
            acc[2] += rv;
        }
    });
    double tot[3];
    if (reduce_last<3>(acc, partials, &cg->counter[2], tot)) finish_zdot(cg, tot);
}

}  // namespace
}  // namespace uaamg
