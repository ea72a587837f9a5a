// Fused V-cycle level kernels: per level, ONE kernel on the way down (forward
// red-black Gauss-Seidel sweep from x = 0, residual b - A x, Galerkin restriction
// to the next level's b) and ONE on the way up (prolongation x += 2 x_coarse,
// reverse red-black sweep), each on a block-resident tile of TX x TY x TZ cells
// with a 2-cell halo in shared memory.  Reference steps fused here:
// uaamg_preconditioner_3d.cpp:123-141 (smooth), 144-165 (restrictResidual),
// 168-181 (prolongateAdd), 183-196 (vCycle).
//
// Why a 2-cell halo is enough and why the pre-smoothed x is never stored:
//  * Down: with x = 0 on entry, the forward sweep's first colour (odd i+j+k) is
//    x = (b + 0)/d, a function of the cell alone; the second colour needs its odd
//    neighbours (1 cell out, whose diagonals need the mask 1 further); the residual
//    needs both colours 1 cell out.  Only the coarse b leaves the kernel.
//  * Up: the reverse sweep overwrites every even cell from its odd neighbours,
//    whose values are (b + 0)/d + 2 x_coarse -- recomputed here from b -- and then
//    every odd cell from its even neighbours.  The pre-smoothed even values are
//    dead, so the down kernel writes no fine x at all.
// Every per-cell expression keeps the reference's operation order, so the FP64
// instantiation (compiled with -fmad=false) reproduces the reference bit for bit.
//
// Coefficients: on the finest level they follow from the mask (a coupling exists
// iff both cells are interior fluid cells: uaamg_preconditioner_3d.cpp:50-66) and
// no coefficient array is read; coarse levels read their Galerkin arrays.
#pragma once
#include "kernels.cuh"

namespace uaamg {
namespace {

template <class T>
struct VLevel {
    Geom g;
    const uint8_t* solid;
    const T* cx;   // nullptr on the finest level: couplings from the mask
    const T* cy;
    const T* cz;
    const T* wd;   // Dirichlet wall diagonal (coarse levels), or nullptr
    T idx2, idy2, idz2;
    int dirichlet;
};

template <int DIM, int TX, int TY, int TZ>
struct TileGeo {
    static constexpr int H = 2;
    static constexpr int AX = TX + 2 * H, AY = TY + 2 * H, AZ = DIM == 3 ? TZ + 2 * H : 1;
    static constexpr int NA = AX * AY * AZ;                                // b, x region
    static constexpr int BX = AX + 2, BY = AY + 2, BZ = DIM == 3 ? AZ + 2 : 1;
    static constexpr int NB = BX * BY * BZ;                                // mask region
    template <class T>
    static constexpr size_t smem_bytes() {
        return 2 * sizeof(T) * NA + ((NB + 15) / 16) * 16;
    }
};

// Loads the tile's active flags (interior fluid) over the mask region and b over
// the value region.  i0, j0, k0: first interior cell of the tile.
template <int DIM, class T, int TX, int TY, int TZ>
__device__ __forceinline__ void tile_load(const VLevel<T>& L, const T* __restrict__ b, int i0,
                                          int j0, int k0, T* sb, uint8_t* sa) {
    using G = TileGeo<DIM, TX, TY, TZ>;
    const Geom& g = L.g;
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int q = tid; q < G::NB; q += nthr) {
        const int a = q % G::BX, bb = (q / G::BX) % G::BY, cc = q / (G::BX * G::BY);
        const int i = i0 - G::H - 1 + a, j = j0 - G::H - 1 + bb;
        const int k = DIM == 3 ? k0 - G::H - 1 + cc : 0;
        const bool in = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny &&
                        (DIM == 2 || (k >= 1 && k <= g.nz));
        sa[q] = (in && !L.solid[cidx(g, i, j, k)]) ? 1 : 0;
    }
    __syncthreads();
    for (int q = tid; q < G::NA; q += nthr) {
        const int a = q % G::AX, bb = (q / G::AX) % G::AY, cc = q / (G::AX * G::AY);
        const int i = i0 - G::H + a, j = j0 - G::H + bb, k = DIM == 3 ? k0 - G::H + cc : 0;
        const int qa = (a + 1) + G::BX * ((bb + 1) + G::BY * (DIM == 3 ? cc + 1 : 0));
        sb[q] = sa[qa] ? b[cidx(g, i, j, k)] : T(0);
    }
}

// Couplings of an active cell (local value-region index q, mask index qa, global
// id and coordinates) in the reference's order: +x, -x, +y, -y[, +z, -z].
template <int DIM, class T, int TX, int TY, int TZ>
__device__ __forceinline__ void couplings(const VLevel<T>& L, const uint8_t* sa, int qa, int id,
                                          T (&c)[6]) {
    using G = TileGeo<DIM, TX, TY, TZ>;
    if (!L.cx) {
        c[0] = sa[qa + 1] ? L.idx2 : T(0);
        c[1] = sa[qa - 1] ? L.idx2 : T(0);
        c[2] = sa[qa + G::BX] ? L.idy2 : T(0);
        c[3] = sa[qa - G::BX] ? L.idy2 : T(0);
        if (DIM == 3) {
            c[4] = sa[qa + G::BX * G::BY] ? L.idz2 : T(0);
            c[5] = sa[qa - G::BX * G::BY] ? L.idz2 : T(0);
        }
    } else {
        const Geom& g = L.g;
        c[0] = L.cx[id];
        c[1] = L.cx[id - 1];
        c[2] = L.cy[id];
        c[3] = L.cy[id - g.sx];
        if (DIM == 3) {
            c[4] = L.cz[id];
            c[5] = L.cz[id - g.sxy];
        }
    }
}

// Diagonal = sum of the couplings in the reference's order (+ Dirichlet walls).
template <int DIM, class T>
__device__ __forceinline__ T diag_of(const VLevel<T>& L, const T (&c)[6], int i, int j, int k,
                                     int id) {
    T d = c[0] + c[1] + c[2] + c[3];
    if (DIM == 3) d = d + c[4] + c[5];
    if (L.dirichlet) {
        if (!L.cx) {  // finest level: walls from the coordinates (as k_fine_coeffs)
            T w = T(0);
            const Geom& g = L.g;
            if (i == 1) w += T(2) * L.idx2;
            if (i == g.nx) w += T(2) * L.idx2;
            if (j == 1) w += T(2) * L.idy2;
            if (j == g.ny) w += T(2) * L.idy2;
            if (DIM == 3 && k == 1) w += T(2) * L.idz2;
            if (DIM == 3 && k == g.nz) w += T(2) * L.idz2;
            d = d + w;
        } else {
            d = d + L.wd[id];
        }
    }
    return d;
}

// sum c * x_nb in the reference's order (uaamg_preconditioner_3d.cpp:133-135).
template <int DIM, class T, int TX, int TY, int TZ>
__device__ __forceinline__ T neighbour_sum(const T (&c)[6], const T* sx, int q) {
    using G = TileGeo<DIM, TX, TY, TZ>;
    T nb = c[0] * sx[q + 1] + c[1] * sx[q - 1] + c[2] * sx[q + G::AX] + c[3] * sx[q - G::AX];
    if (DIM == 3) nb = nb + c[4] * sx[q + G::AX * G::AY] + c[5] * sx[q - G::AX * G::AY];
    return nb;
}

template <int DIM, int TX, int TY, int TZ>
__device__ __forceinline__ void tile_origin(int tile, int ntx, int nty, int& i0, int& j0, int& k0) {
    const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tile / (ntx * nty);
    i0 = 1 + tx * TX;
    j0 = 1 + ty * TY;
    k0 = DIM == 3 ? 1 + tz * TZ : 0;
}

// Local value-region decode: q -> (a, bb, cc), global (i, j, k), mask index qa.
template <int DIM, int TX, int TY, int TZ>
__device__ __forceinline__ void decode(int q, int i0, int j0, int k0, int& i, int& j, int& k,
                                       int& qa) {
    using G = TileGeo<DIM, TX, TY, TZ>;
    const int a = q % G::AX, bb = (q / G::AX) % G::AY, cc = q / (G::AX * G::AY);
    i = i0 - G::H + a;
    j = j0 - G::H + bb;
    k = DIM == 3 ? k0 - G::H + cc : 0;
    qa = (a + 1) + G::BX * ((bb + 1) + G::BY * (DIM == 3 ? cc + 1 : 0));
}

// Down: forward sweep from x = 0, residual, restriction into the coarse b.
template <int DIM, class T, int TX, int TY, int TZ>
__global__ void __launch_bounds__(256) k_vdown(VLevel<T> L, const T* __restrict__ b, Geom cgm,
                                               const uint8_t* __restrict__ cs, T* cb,
                                               int ntx, int nty, int ntiles,
                                               const int* __restrict__ done) {
    if (done && *done) return;
    using G = TileGeo<DIM, TX, TY, TZ>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sb = reinterpret_cast<T*>(smem_raw);
    T* sx = sb + G::NA;
    uint8_t* sa = reinterpret_cast<uint8_t*>(sx + G::NA);
    const Geom& g = L.g;
    const int tid = threadIdx.x, nthr = blockDim.x;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int i0, j0, k0;
        tile_origin<DIM, TX, TY, TZ>(tile, ntx, nty, i0, j0, k0);
        tile_load<DIM, T, TX, TY, TZ>(L, b, i0, j0, k0, sb, sa);
        __syncthreads();
        // first colour (odd), whole value region: x = (b + 0)/d
        for (int q = tid; q < G::NA; q += nthr) {
            int i, j, k, qa;
            decode<DIM, TX, TY, TZ>(q, i0, j0, k0, i, j, k, qa);
            T xv = T(0);
            if (sa[qa] && ((i + j + k) & 1)) {
                T c[6];
                const int id = cidx(g, i, j, k);
                couplings<DIM, T, TX, TY, TZ>(L, sa, qa, id, c);
                const T d = diag_of<DIM, T>(L, c, i, j, k, id);
                if (!(d < T(1e-30))) xv = (sb[q] + T(0)) / d;
            }
            sx[q] = xv;
        }
        __syncthreads();
        // second colour (even), one cell beyond the tile
        for (int q = tid; q < G::NA; q += nthr) {
            const int a = q % G::AX, bb = (q / G::AX) % G::AY, cc = q / (G::AX * G::AY);
            if (a < 1 || a > G::AX - 2 || bb < 1 || bb > G::AY - 2) continue;
            if (DIM == 3 && (cc < 1 || cc > G::AZ - 2)) continue;
            int i, j, k, qa;
            decode<DIM, TX, TY, TZ>(q, i0, j0, k0, i, j, k, qa);
            if (!sa[qa] || ((i + j + k) & 1)) continue;
            T c[6];
            const int id = cidx(g, i, j, k);
            couplings<DIM, T, TX, TY, TZ>(L, sa, qa, id, c);
            const T d = diag_of<DIM, T>(L, c, i, j, k, id);
            if (d < T(1e-30)) continue;
            sx[q] = (sb[q] + neighbour_sum<DIM, T, TX, TY, TZ>(c, sx, q)) / d;
        }
        __syncthreads();
        // restriction: coarse cells whose children lie in this tile
        constexpr int CX = TX / 2, CY = TY / 2, CZ = DIM == 3 ? TZ / 2 : 1;
        for (int cq = tid; cq < CX * CY * CZ; cq += nthr) {
            const int ca = cq % CX, cbb = (cq / CX) % CY, ccc = cq / (CX * CY);
            const int ic = (i0 + 1) / 2 + ca, jc = (j0 + 1) / 2 + cbb;
            const int kc = DIM == 3 ? (k0 + 1) / 2 + ccc : 0;
            if (ic > cgm.nx || jc > cgm.ny || (DIM == 3 && kc > cgm.nz)) continue;
            const int cid = cidx(cgm, ic, jc, kc);
            if (cs[cid]) continue;
            T sum = T(0);
            for (int di = 0; di < 2; ++di)
                for (int dj = 0; dj < 2; ++dj)
                    for (int dk = 0; dk < (DIM == 3 ? 2 : 1); ++dk) {
                        const int a = 2 * ca + di + G::H, bb = 2 * cbb + dj + G::H;
                        const int cc = DIM == 3 ? 2 * ccc + dk + G::H : 0;
                        const int q = a + G::AX * (bb + G::AY * cc);
                        int i, j, k, qa;
                        decode<DIM, TX, TY, TZ>(q, i0, j0, k0, i, j, k, qa);
                        if (!sa[qa]) continue;
                        T c[6];
                        const int id = cidx(g, i, j, k);
                        couplings<DIM, T, TX, TY, TZ>(L, sa, qa, id, c);
                        const T d = diag_of<DIM, T>(L, c, i, j, k, id);
                        T ax = d * sx[q] - c[0] * sx[q + 1] - c[1] * sx[q - 1]
                             - c[2] * sx[q + G::AX] - c[3] * sx[q - G::AX];
                        if (DIM == 3)
                            ax = ax - c[4] * sx[q + G::AX * G::AY] - c[5] * sx[q - G::AX * G::AY];
                        sum += sb[q] - ax;
                    }
            cb[cid] = sum;
        }
        __syncthreads();
    }
}

// Up: prolongation of the coarse correction and the reverse sweep; writes the
// level's x (interior cells of the tile; solid cells 0).  ZDOT (finest level
// only): also reduces sum z, sum r*z, sum r over fluid cells (r = this level's b)
// and finishes the CG's null-space projection / beta (pcg_3d.cpp:112-123).
template <int DIM, class T, int TX, int TY, int TZ, bool ZDOT>
__global__ void __launch_bounds__(256) k_vup(VLevel<T> L, const T* __restrict__ b, Geom cgm,
                                             const uint8_t* __restrict__ cs,
                                             const T* __restrict__ xc, T* __restrict__ x,
                                             int ntx, int nty, int ntiles,
                                             const int* __restrict__ done, double* partials,
                                             CGState* cg) {
    if (done && *done) return;
    using G = TileGeo<DIM, TX, TY, TZ>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sb = reinterpret_cast<T*>(smem_raw);
    T* sx = sb + G::NA;
    uint8_t* sa = reinterpret_cast<uint8_t*>(sx + G::NA);
    const Geom& g = L.g;
    const int tid = threadIdx.x, nthr = blockDim.x;
    double acc[3] = {0.0, 0.0, 0.0};
    // coarse parent of fine (i, j, k): children 2ic-1, 2ic (uaamg_preconditioner_3d.cpp:176)
    auto prolong = [&](int i, int j, int k) -> T {
        if (i > 2 * cgm.nx || j > 2 * cgm.ny || (DIM == 3 && k > 2 * cgm.nz)) return T(0);
        const int cid = cidx(cgm, (i + 1) >> 1, (j + 1) >> 1, DIM == 3 ? (k + 1) >> 1 : 0);
        return cs[cid] ? T(0) : T(2) * xc[cid];
    };
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int i0, j0, k0;
        tile_origin<DIM, TX, TY, TZ>(tile, ntx, nty, i0, j0, k0);
        tile_load<DIM, T, TX, TY, TZ>(L, b, i0, j0, k0, sb, sa);
        __syncthreads();
        // odd cells, whole value region: pre-smoothed (b + 0)/d plus the prolongation
        for (int q = tid; q < G::NA; q += nthr) {
            int i, j, k, qa;
            decode<DIM, TX, TY, TZ>(q, i0, j0, k0, i, j, k, qa);
            T xv = T(0);
            if (sa[qa] && ((i + j + k) & 1)) {
                T c[6];
                const int id = cidx(g, i, j, k);
                couplings<DIM, T, TX, TY, TZ>(L, sa, qa, id, c);
                const T d = diag_of<DIM, T>(L, c, i, j, k, id);
                if (!(d < T(1e-30))) xv = (sb[q] + T(0)) / d;
                xv = xv + prolong(i, j, k);
            }
            sx[q] = xv;
        }
        __syncthreads();
        // reverse sweep, first colour (even), one cell beyond the tile
        for (int q = tid; q < G::NA; q += nthr) {
            const int a = q % G::AX, bb = (q / G::AX) % G::AY, cc = q / (G::AX * G::AY);
            if (a < 1 || a > G::AX - 2 || bb < 1 || bb > G::AY - 2) continue;
            if (DIM == 3 && (cc < 1 || cc > G::AZ - 2)) continue;
            int i, j, k, qa;
            decode<DIM, TX, TY, TZ>(q, i0, j0, k0, i, j, k, qa);
            if (!sa[qa] || ((i + j + k) & 1)) continue;
            T c[6];
            const int id = cidx(g, i, j, k);
            couplings<DIM, T, TX, TY, TZ>(L, sa, qa, id, c);
            const T d = diag_of<DIM, T>(L, c, i, j, k, id);
            // a cell the smoother skips keeps its pre-smoothed 0 plus the prolongation
            sx[q] = d < T(1e-30) ? T(0) + prolong(i, j, k)
                                 : (sb[q] + neighbour_sum<DIM, T, TX, TY, TZ>(c, sx, q)) / d;
        }
        __syncthreads();
        // second colour (odd) on the tile, then write the tile
        for (int q = tid; q < G::NA; q += nthr) {
            const int a = q % G::AX, bb = (q / G::AX) % G::AY, cc = q / (G::AX * G::AY);
            if (a < G::H || a >= G::H + TX || bb < G::H || bb >= G::H + TY) continue;
            if (DIM == 3 && (cc < G::H || cc >= G::H + TZ)) continue;
            int i, j, k, qa;
            decode<DIM, TX, TY, TZ>(q, i0, j0, k0, i, j, k, qa);
            if (i > g.nx || j > g.ny || (DIM == 3 && k > g.nz)) continue;
            const int id = cidx(g, i, j, k);
            T xv = T(0);
            if (sa[qa]) {
                xv = sx[q];
                if ((i + j + k) & 1) {
                    T c[6];
                    couplings<DIM, T, TX, TY, TZ>(L, sa, qa, id, c);
                    const T d = diag_of<DIM, T>(L, c, i, j, k, id);
                    if (!(d < T(1e-30))) xv = (sb[q] + neighbour_sum<DIM, T, TX, TY, TZ>(c, sx, q)) / d;
                }
                if (ZDOT) {
                    const double zv = (double)xv, rv = (double)sb[q];
                    acc[0] += zv;
                    acc[1] += rv * zv;
                    acc[2] += rv;
                }
            }
            x[id] = xv;
        }
        __syncthreads();
    }
    if (ZDOT) {
        double tot[3];
        if (reduce_last<3>(acc, partials, &cg->counter[2], tot)) finish_zdot(cg, tot);
    }
}

}  // namespace
}  // namespace uaamg
