// Fused stencil kernels on TMA-staged tiles: per multigrid level ONE kernel on
// the way down (forward red-black Gauss-Seidel sweep from x = 0, residual
// b - A x, Galerkin restriction to the next level's b) and ONE on the way up
// (prolongation x += 2 x_coarse, reverse red-black sweep), plus the CG's
// search-direction update fused with the operator and p.Ap.  Each block walks
// its share of tiles of TX x TY x TZ cells; the tile's value box (with halo) and
// cell-code box are staged in shared memory by cp.async.bulk.tensor loads
// (tma.cuh) into a two-stage ring, so the next tile's loads fly while the current
// one is computed.  Reference steps fused here:
// uaamg_preconditioner_3d.cpp:123-141 (smooth), 144-165 (restrictResidual),
// 168-181 (prolongateAdd), 183-196 (vCycle); pcg_3d.cpp:38-55 (matvec),
// 94-99 (p.Ap, alpha), 113-122 (mean projection, p = z + beta p).
//
// Why a 2-cell halo is enough and why the pre-smoothed x is never stored:
//  * Down: with x = 0 on entry, the forward sweep's first colour (odd i+j+k) is
//    x = (b + 0)/d, a function of the cell alone; the second colour needs its odd
//    neighbours; the residual needs both colours 1 cell out.  Only the coarse b
//    leaves the kernel.
//  * Up: the reverse sweep overwrites every even cell from its odd neighbours,
//    whose values are (b + 0)/d + 2 x_coarse -- recomputed here from b -- and then
//    every odd cell from its even neighbours.  The pre-smoothed even values are
//    dead, so the down kernel writes no fine x at all.
//
// Cell codes (one byte per cell, built once per problem by k_codes): bit 6 the
// cell is an interior fluid cell, bit 7 its colour (i+j+k odd), and on the finest
// level bits 0-5 whether its +x,-x,+y,-y,+z,-z neighbour is an interior fluid
// cell -- exactly when the reference's coupling exists
// (uaamg_preconditioner_3d.cpp:50-66).  Finest-level diagonals then come from a
// 64-entry table summed in the reference's order; coarse levels read their
// Galerkin arrays and a diagonal array.
//
// Arithmetic: the FP64 instantiation (compiled with -fmad=false) keeps every
// per-cell expression of the reference, including the division by the diagonal,
// so it reproduces the reference bit for bit.  The FP32 instantiation multiplies
// by the reciprocal diagonal instead (within one FP32 rounding of the division).
#pragma once
#include "kernels.cuh"
#include "tma.cuh"

namespace uaamg {
namespace {

constexpr uint32_t kActive = 64u, kOdd = 128u;

template <class T>
struct VLevel {
    Geom g;
    const T* cx;   // nullptr on the finest level: couplings from the cell codes
    const T* cy;
    const T* cz;
    const T* dg;   // coarse levels: diagonal
    const T* rdg;  // coarse levels: 1/diagonal (0 where the smoother skips the cell)
    T idx2, idy2, idz2;
    int dirichlet;
};

// x-extent of a box of elements E covering cells [i0 - halo, i0 + TX - 1 + halo]
// for tiles starting at i0 = 1 + t*TX (TX a multiple of 16): the start is rounded
// down to a 16-byte boundary, `off` cells before the first needed cell.
template <class E, int TX, int HALO>
struct XBox {
    static constexpr int a = 16 / (int)sizeof(E);
    static constexpr int off = ((1 - HALO) % a + a) % a;
    static constexpr int W = (TX + 2 * HALO + off + a - 1) / a * a;
};

__host__ __device__ constexpr size_t align128(size_t b) { return (b + 127) / 128 * 128; }

// Shared-memory plan of the V-cycle kernels: value box and code box with a 2-cell
// halo, two stages, plus the x scratch and the diagonal tables.
template <int DIM, class T, int TX, int TY, int TZ>
struct VPlan {
    static constexpr int H = 2;
    static constexpr int RX = TX + 2 * H, RY = TY + 2 * H, RZ = DIM == 3 ? TZ + 2 * H : 1;
    using XB = XBox<T, TX, H>;
    using XC = XBox<uint8_t, TX, H>;
    static constexpr int BW = XB::W, BY = RY, BZ = RZ;
    static constexpr int CW = XC::W, CY = RY, CZ = RZ;
    static constexpr size_t NB = (size_t)BW * BY * BZ, NC = (size_t)CW * CY * CZ;
    static constexpr size_t STAGE = align128(NB * sizeof(T)) + align128(NC);
    static constexpr size_t OFF_S0 = 128, OFF_S1 = OFF_S0 + STAGE;
    static constexpr size_t OFF_X = OFF_S1 + STAGE;
    static constexpr size_t OFF_L = OFF_X + align128(NB * sizeof(T));
    static constexpr size_t BYTES = OFF_L + align128(128 * sizeof(T)) + 128;  // + base alignment
    static constexpr uint32_t TX_BYTES = (uint32_t)(NB * sizeof(T) + NC);
};

// Shared-memory plan of the search-direction kernel: z and p_old with a 1-cell
// halo, the tile's codes, two stages.
template <int DIM, class T, int TX, int TY, int TZ>
struct PPlan {
    static constexpr int RX = TX + 2, RY = TY + 2, RZ = DIM == 3 ? TZ + 2 : 1;
    using XB = XBox<T, TX, 1>;
    using XC = XBox<uint8_t, TX, 0>;
    static constexpr int BW = XB::W, BY = RY, BZ = RZ;
    static constexpr int CW = XC::W, CY = TY, CZ = DIM == 3 ? TZ : 1;
    static constexpr size_t NB = (size_t)BW * BY * BZ, NC = (size_t)CW * CY * CZ;
    static constexpr size_t STAGE = 2 * align128(NB * sizeof(T)) + align128(NC);
    static constexpr size_t OFF_S0 = 128, OFF_S1 = OFF_S0 + STAGE;
    static constexpr size_t BYTES = OFF_S1 + STAGE + 128;
    static constexpr uint32_t TX_BYTES = (uint32_t)(2 * NB * sizeof(T) + NC);
};

__device__ __forceinline__ unsigned char* aligned_smem(unsigned char* raw) {
    const uintptr_t p = reinterpret_cast<uintptr_t>(raw);
    return reinterpret_cast<unsigned char*>((p + 127) & ~uintptr_t(127));
}

template <int DIM, int TX, int TY, int TZ>
__device__ __forceinline__ void tile_origin(int tile, int ntx, int nty, int& i0, int& j0, int& k0) {
    const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tile / (ntx * nty);
    i0 = 1 + tx * TX;
    j0 = 1 + ty * TY;
    k0 = DIM == 3 ? 1 + tz * TZ : 0;
}

// Couplings of an active cell in the reference's order +x, -x, +y, -y[, +z, -z].
template <int DIM, class T>
__device__ __forceinline__ void couplings(const VLevel<T>& L, uint32_t code, int id, T (&c)[6]) {
    if (!L.cx) {
        c[0] = (code & 1u) ? L.idx2 : T(0);
        c[1] = (code & 2u) ? L.idx2 : T(0);
        c[2] = (code & 4u) ? L.idy2 : T(0);
        c[3] = (code & 8u) ? L.idy2 : T(0);
        if (DIM == 3) {
            c[4] = (code & 16u) ? L.idz2 : T(0);
            c[5] = (code & 32u) ? L.idz2 : T(0);
        }
    } else {
        c[0] = __ldg(&L.cx[id]);
        c[1] = __ldg(&L.cx[id - 1]);
        c[2] = __ldg(&L.cy[id]);
        c[3] = __ldg(&L.cy[id - L.g.sx]);
        if (DIM == 3) {
            c[4] = __ldg(&L.cz[id]);
            c[5] = __ldg(&L.cz[id - L.g.sxy]);
        }
    }
}

// Dirichlet wall diagonal of a finest-level cell (as k_fine_coeffs).
template <int DIM, class T>
__device__ __forceinline__ T wall_diag(const VLevel<T>& L, int i, int j, int k) {
    T w = T(0);
    const Geom& g = L.g;
    if (i == 1) w += T(2) * L.idx2;
    if (i == g.nx) w += T(2) * L.idx2;
    if (j == 1) w += T(2) * L.idy2;
    if (j == g.ny) w += T(2) * L.idy2;
    if (DIM == 3 && k == 1) w += T(2) * L.idz2;
    if (DIM == 3 && k == g.nz) w += T(2) * L.idz2;
    return w;
}

// Diagonal d of an active cell and the factor that turns (b + sum) into the
// smoothed value: returns false when the reference's smoother skips the cell
// (d < 1e-30).  FP64: x = num / d; FP32: x = num * rd.
template <int DIM, class T>
__device__ __forceinline__ bool diag_of(const VLevel<T>& L, const T* lut, uint32_t code, int i,
                                        int j, int k, int id, T& d, T& rd) {
    if (L.cx) {
        d = __ldg(&L.dg[id]);
        if (sizeof(T) == 4) rd = __ldg(&L.rdg[id]);
    } else if (!L.dirichlet) {
        d = lut[code & 63u];
        if (sizeof(T) == 4) rd = lut[64 + (code & 63u)];
    } else {
        d = lut[code & 63u] + wall_diag<DIM, T>(L, i, j, k);
        if (sizeof(T) == 4) rd = d < T(1e-30) ? T(0) : T(1) / d;
    }
    return !(d < T(1e-30));
}

template <class T>
__device__ __forceinline__ T smoothed(T num, T d, T rd) {
    return sizeof(T) == 4 ? num * rd : num / d;
}

// lut[0..63]: diagonal by neighbour code, summed in the reference's order
// (uaamg_preconditioner_3d.cpp:72-74); lut[64..127]: its reciprocal (FP32).
template <int DIM, class T>
__device__ __forceinline__ void build_lut(const VLevel<T>& L, T* lut) {
    for (int c = threadIdx.x; c < 64; c += blockDim.x) {
        T v[6];
        v[0] = (c & 1) ? L.idx2 : T(0);
        v[1] = (c & 2) ? L.idx2 : T(0);
        v[2] = (c & 4) ? L.idy2 : T(0);
        v[3] = (c & 8) ? L.idy2 : T(0);
        v[4] = (c & 16) ? L.idz2 : T(0);
        v[5] = (c & 32) ? L.idz2 : T(0);
        T d = v[0] + v[1] + v[2] + v[3];
        if (DIM == 3) d = d + v[4] + v[5];
        lut[c] = d;
        lut[64 + c] = d < T(1e-30) ? T(0) : T(1) / d;
    }
}

template <int DIM, class T, class P>
__device__ __forceinline__ T nb_sum(const T (&c)[6], const T* sx, int qb) {
    T nb = c[0] * sx[qb + 1] + c[1] * sx[qb - 1] + c[2] * sx[qb + P::BW] + c[3] * sx[qb - P::BW];
    if (DIM == 3) nb = nb + c[4] * sx[qb + P::BW * P::BY] + c[5] * sx[qb - P::BW * P::BY];
    return nb;
}

// Issues a V-cycle tile's loads (thread 0 only).
template <int DIM, class P>
__device__ __forceinline__ void vissue(const CUtensorMap* mb, const CUtensorMap* mc, void* sb,
                                       void* sc, uint64_t* bar, int i0, int j0, int k0) {
    fence_proxy_async();
    mbar_expect_tx(bar, P::TX_BYTES);
    tma_load<DIM>(sb, mb, i0 - P::H - P::XB::off, j0 - P::H, k0 - P::H, bar);
    tma_load<DIM>(sc, mc, i0 - P::H - P::XC::off, j0 - P::H, k0 - P::H, bar);
}

// Waits for a stage; one block-wide verdict.  On a timeout the error word is set
// and the caller leaves.
__device__ __forceinline__ bool stage_wait(uint64_t* bar, uint32_t& phase, int* err) {
    const bool ok = mbar_wait(bar, phase, kTmaWaitLimit);
    phase ^= 1u;
    const bool all = __syncthreads_and(ok ? 1 : 0) != 0;
    if (!all && threadIdx.x == 0) atomicExch(err, 1);
    return all;
}

// Down: forward sweep from x = 0, residual, restriction into the coarse b.
template <int DIM, class T, int TX, int TY, int TZ>
__global__ void __launch_bounds__(256) k_vdown(const __grid_constant__ CUtensorMap map_b,
                                               const __grid_constant__ CUtensorMap map_c,
                                               VLevel<T> L, Geom cgm,
                                               const uint8_t* __restrict__ cs, T* cb, int ntx,
                                               int nty, int ntiles, const int* __restrict__ done,
                                               int* err) {
    if (done && *done) return;
    using P = VPlan<DIM, T, TX, TY, TZ>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* sm0 = aligned_smem(smem_raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm0);
    auto stage = [&](int q) { return sm0 + P::OFF_S0 + (size_t)q * P::STAGE; };
    T* sx = reinterpret_cast<T*>(sm0 + P::OFF_X);
    T* lut = reinterpret_cast<T*>(sm0 + P::OFF_L);
    const Geom& g = L.g;
    const int tid = threadIdx.x, nthr = blockDim.x;
    if (tid == 0) { mbar_init(&bars[0], 1); mbar_init(&bars[1], 1); }
    build_lut<DIM, T>(L, lut);
    __syncthreads();
    uint32_t phase[2] = {0u, 0u};
    int tile = blockIdx.x, s = 0;
    if (tile < ntiles && tid == 0) {
        int i0, j0, k0;
        tile_origin<DIM, TX, TY, TZ>(tile, ntx, nty, i0, j0, k0);
        vissue<DIM, P>(&map_b, &map_c, stage(0), stage(0) + align128(P::NB * sizeof(T)), &bars[0],
                       i0, j0, k0);
    }
    for (; tile < ntiles; tile += gridDim.x, s ^= 1) {
        int i0, j0, k0;
        tile_origin<DIM, TX, TY, TZ>(tile, ntx, nty, i0, j0, k0);
        const int next = tile + gridDim.x;
        if (next < ntiles && tid == 0) {
            int a0, b0, c0;
            tile_origin<DIM, TX, TY, TZ>(next, ntx, nty, a0, b0, c0);
            vissue<DIM, P>(&map_b, &map_c, stage(s ^ 1),
                           stage(s ^ 1) + align128(P::NB * sizeof(T)), &bars[s ^ 1], a0, b0, c0);
        }
        if (!stage_wait(&bars[s], phase[s], err)) return;
        const T* sb = reinterpret_cast<const T*>(stage(s));
        const uint8_t* scd = stage(s) + align128(P::NB * sizeof(T));
        const int ib = i0 - P::H, jb = j0 - P::H, kb = DIM == 3 ? k0 - P::H : 0;
        // first colour (odd), whole value region: x = (b + 0)/d
        for (int p = tid; p < P::RX * P::RY; p += nthr) {
            const int a = p % P::RX, bb = p / P::RX;
            for (int cc = 0; cc < P::RZ; ++cc) {
                const int qb = a + P::XB::off + P::BW * (bb + P::BY * cc);
                const int qc = a + P::XC::off + P::CW * (bb + P::CY * cc);
                const uint32_t code = scd[qc];
                T xv = T(0);
                if ((code & (kActive | kOdd)) == (kActive | kOdd)) {
                    const int i = ib + a, j = jb + bb, k = kb + cc;
                    T d, rd;
                    if (diag_of<DIM, T>(L, lut, code, i, j, k, cidx(g, i, j, k), d, rd))
                        xv = smoothed<T>(sb[qb] + T(0), d, rd);
                }
                sx[qb] = xv;
            }
        }
        __syncthreads();
        // second colour (even), one cell beyond the tile
        for (int p = tid; p < (P::RX - 2) * (P::RY - 2); p += nthr) {
            const int a = 1 + p % (P::RX - 2), bb = 1 + p / (P::RX - 2);
            for (int cc = DIM == 3 ? 1 : 0; cc < (DIM == 3 ? P::RZ - 1 : 1); ++cc) {
                const int qc = a + P::XC::off + P::CW * (bb + P::CY * cc);
                const uint32_t code = scd[qc];
                if ((code & (kActive | kOdd)) != kActive) continue;
                const int qb = a + P::XB::off + P::BW * (bb + P::BY * cc);
                const int i = ib + a, j = jb + bb, k = kb + cc;
                const int id = cidx(g, i, j, k);
                T d, rd;
                if (!diag_of<DIM, T>(L, lut, code, i, j, k, id, d, rd)) continue;
                T c[6];
                couplings<DIM, T>(L, code, id, c);
                sx[qb] = smoothed<T>(sb[qb] + nb_sum<DIM, T, P>(c, sx, qb), d, rd);
            }
        }
        __syncthreads();
        // restriction: coarse cells whose children lie in this tile, children in the
        // reference's (di, dj, dk) order
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
                        const int a = 2 * ca + di + P::H, bb = 2 * cbb + dj + P::H;
                        const int cc = DIM == 3 ? 2 * ccc + dk + P::H : 0;
                        const int qc = a + P::XC::off + P::CW * (bb + P::CY * cc);
                        const uint32_t code = scd[qc];
                        if (!(code & kActive)) continue;
                        const int qb = a + P::XB::off + P::BW * (bb + P::BY * cc);
                        const int i = ib + a, j = jb + bb, k = kb + cc;
                        const int id = cidx(g, i, j, k);
                        T d, rd;
                        diag_of<DIM, T>(L, lut, code, i, j, k, id, d, rd);
                        T c[6];
                        couplings<DIM, T>(L, code, id, c);
                        T ax = d * sx[qb] - c[0] * sx[qb + 1] - c[1] * sx[qb - 1]
                             - c[2] * sx[qb + P::BW] - c[3] * sx[qb - P::BW];
                        if (DIM == 3)
                            ax = ax - c[4] * sx[qb + P::BW * P::BY] - c[5] * sx[qb - P::BW * P::BY];
                        sum += sb[qb] - ax;
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
__global__ void __launch_bounds__(256) k_vup(const __grid_constant__ CUtensorMap map_b,
                                             const __grid_constant__ CUtensorMap map_c,
                                             VLevel<T> L, Geom cgm,
                                             const uint8_t* __restrict__ cs,
                                             const T* __restrict__ xc, T* __restrict__ x,
                                             int ntx, int nty, int ntiles,
                                             const int* __restrict__ done, int* err,
                                             double* partials, CGState* cg) {
    if (done && *done) return;
    using P = VPlan<DIM, T, TX, TY, TZ>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* sm0 = aligned_smem(smem_raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm0);
    auto stage = [&](int q) { return sm0 + P::OFF_S0 + (size_t)q * P::STAGE; };
    T* sx = reinterpret_cast<T*>(sm0 + P::OFF_X);
    T* lut = reinterpret_cast<T*>(sm0 + P::OFF_L);
    const Geom& g = L.g;
    const int tid = threadIdx.x, nthr = blockDim.x;
    double acc[3] = {0.0, 0.0, 0.0};
    // coarse parent of fine (i, j, k): children 2ic-1, 2ic (uaamg_preconditioner_3d.cpp:176)
    auto prolong = [&](int i, int j, int k) -> T {
        if (i > 2 * cgm.nx || j > 2 * cgm.ny || (DIM == 3 && k > 2 * cgm.nz)) return T(0);
        const int cid = cidx(cgm, (i + 1) >> 1, (j + 1) >> 1, DIM == 3 ? (k + 1) >> 1 : 0);
        return cs[cid] ? T(0) : T(2) * __ldg(&xc[cid]);
    };
    if (tid == 0) { mbar_init(&bars[0], 1); mbar_init(&bars[1], 1); }
    build_lut<DIM, T>(L, lut);
    __syncthreads();
    uint32_t phase[2] = {0u, 0u};
    bool failed = false;
    int tile = blockIdx.x, s = 0;
    if (tile < ntiles && tid == 0) {
        int i0, j0, k0;
        tile_origin<DIM, TX, TY, TZ>(tile, ntx, nty, i0, j0, k0);
        vissue<DIM, P>(&map_b, &map_c, stage(0), stage(0) + align128(P::NB * sizeof(T)), &bars[0],
                       i0, j0, k0);
    }
    for (; tile < ntiles; tile += gridDim.x, s ^= 1) {
        int i0, j0, k0;
        tile_origin<DIM, TX, TY, TZ>(tile, ntx, nty, i0, j0, k0);
        const int next = tile + gridDim.x;
        if (next < ntiles && tid == 0) {
            int a0, b0, c0;
            tile_origin<DIM, TX, TY, TZ>(next, ntx, nty, a0, b0, c0);
            vissue<DIM, P>(&map_b, &map_c, stage(s ^ 1),
                           stage(s ^ 1) + align128(P::NB * sizeof(T)), &bars[s ^ 1], a0, b0, c0);
        }
        if (!stage_wait(&bars[s], phase[s], err)) { failed = true; break; }
        const T* sb = reinterpret_cast<const T*>(stage(s));
        const uint8_t* scd = stage(s) + align128(P::NB * sizeof(T));
        const int ib = i0 - P::H, jb = j0 - P::H, kb = DIM == 3 ? k0 - P::H : 0;
        // odd cells, whole value region: pre-smoothed (b + 0)/d plus the prolongation
        for (int p = tid; p < P::RX * P::RY; p += nthr) {
            const int a = p % P::RX, bb = p / P::RX;
            for (int cc = 0; cc < P::RZ; ++cc) {
                const int qb = a + P::XB::off + P::BW * (bb + P::BY * cc);
                const int qc = a + P::XC::off + P::CW * (bb + P::CY * cc);
                const uint32_t code = scd[qc];
                T xv = T(0);
                if ((code & (kActive | kOdd)) == (kActive | kOdd)) {
                    const int i = ib + a, j = jb + bb, k = kb + cc;
                    T d, rd;
                    if (diag_of<DIM, T>(L, lut, code, i, j, k, cidx(g, i, j, k), d, rd))
                        xv = smoothed<T>(sb[qb] + T(0), d, rd);
                    xv = xv + prolong(i, j, k);
                }
                sx[qb] = xv;
            }
        }
        __syncthreads();
        // reverse sweep, first colour (even), one cell beyond the tile
        for (int p = tid; p < (P::RX - 2) * (P::RY - 2); p += nthr) {
            const int a = 1 + p % (P::RX - 2), bb = 1 + p / (P::RX - 2);
            for (int cc = DIM == 3 ? 1 : 0; cc < (DIM == 3 ? P::RZ - 1 : 1); ++cc) {
                const int qc = a + P::XC::off + P::CW * (bb + P::CY * cc);
                const uint32_t code = scd[qc];
                if ((code & (kActive | kOdd)) != kActive) continue;
                const int qb = a + P::XB::off + P::BW * (bb + P::BY * cc);
                const int i = ib + a, j = jb + bb, k = kb + cc;
                const int id = cidx(g, i, j, k);
                T d, rd;
                if (!diag_of<DIM, T>(L, lut, code, i, j, k, id, d, rd)) {
                    // a cell the smoother skips keeps its pre-smoothed 0 plus the prolongation
                    sx[qb] = T(0) + prolong(i, j, k);
                } else {
                    T c[6];
                    couplings<DIM, T>(L, code, id, c);
                    sx[qb] = smoothed<T>(sb[qb] + nb_sum<DIM, T, P>(c, sx, qb), d, rd);
                }
            }
        }
        __syncthreads();
        // second colour (odd) on the tile, then write the tile
        for (int p = tid; p < TX * TY; p += nthr) {
            const int a = P::H + p % TX, bb = P::H + p / TX;
            const int i = ib + a, j = jb + bb;
            if (i > g.nx || j > g.ny) continue;
            for (int cc = DIM == 3 ? P::H : 0; cc < (DIM == 3 ? P::H + TZ : 1); ++cc) {
                const int k = kb + cc;
                if (DIM == 3 && k > g.nz) break;
                const int qb = a + P::XB::off + P::BW * (bb + P::BY * cc);
                const int qc = a + P::XC::off + P::CW * (bb + P::CY * cc);
                const int id = cidx(g, i, j, k);
                const uint32_t code = scd[qc];
                T xv = T(0);
                if (code & kActive) {
                    xv = sx[qb];
                    if (code & kOdd) {
                        T d, rd;
                        if (diag_of<DIM, T>(L, lut, code, i, j, k, id, d, rd)) {
                            T c[6];
                            couplings<DIM, T>(L, code, id, c);
                            xv = smoothed<T>(sb[qb] + nb_sum<DIM, T, P>(c, sx, qb), d, rd);
                        }
                    }
                    if (ZDOT) {
                        const double zv = (double)xv, rv = (double)sb[qb];
                        acc[0] += zv;
                        acc[1] += rv * zv;
                        acc[2] += rv;
                    }
                }
                x[id] = xv;
            }
        }
        __syncthreads();
    }
    if (ZDOT && !failed) {
        double tot[3];
        if (reduce_last<3>(acc, partials, &cg->counter[2], tot)) finish_zdot(cg, tot);
    }
}

// Search direction fused with the operator: p = (z - m) + beta p_old on fluid
// cells (pcg_3d.cpp:113-122), Ap with the neighbours' new p formed on the fly
// from the staged z and p_old, p.Ap reduced; the last block sets
// alpha = rz_old / p.Ap or stops on breakdown (pcg_3d.cpp:94-99).  A solid or
// out-of-domain neighbour reads p_C (Neumann; -p_C for a Dirichlet wall).
// p_old and p_new are distinct buffers.
template <int DIM, class T, int TX, int TY, int TZ>
__global__ void __launch_bounds__(256) k_pmatvec_tile(const __grid_constant__ CUtensorMap map_z,
                                                      const __grid_constant__ CUtensorMap map_p,
                                                      const __grid_constant__ CUtensorMap map_c,
                                                      Geom g, T* __restrict__ pnew,
                                                      T* __restrict__ ap, Stencil st, int ntx,
                                                      int nty, int ntiles, double* partials,
                                                      CGState* cg, int* err) {
    if (cg->done) return;
    using P = PPlan<DIM, T, TX, TY, TZ>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* sm0 = aligned_smem(smem_raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm0);
    auto stage = [&](int q) { return sm0 + P::OFF_S0 + (size_t)q * P::STAGE; };
    constexpr size_t OZ = 0, OP = align128(P::NB * sizeof(T)), OC = 2 * align128(P::NB * sizeof(T));
    const int tid = threadIdx.x, nthr = blockDim.x;
    const T m = (T)cg->mean_z, beta = (T)cg->beta;
    const T idx2 = (T)st.idx2, idy2 = (T)st.idy2, idz2 = (T)st.idz2, diag = (T)st.diag;
    double acc[1] = {0.0};
    auto issue = [&](int t, int sidx) {
        int i0, j0, k0;
        tile_origin<DIM, TX, TY, TZ>(t, ntx, nty, i0, j0, k0);
        fence_proxy_async();
        mbar_expect_tx(&bars[sidx], P::TX_BYTES);
        tma_load<DIM>(stage(sidx) + OZ, &map_z, i0 - 1 - P::XB::off, j0 - 1, k0 - 1, &bars[sidx]);
        tma_load<DIM>(stage(sidx) + OP, &map_p, i0 - 1 - P::XB::off, j0 - 1, k0 - 1, &bars[sidx]);
        tma_load<DIM>(stage(sidx) + OC, &map_c, i0 - P::XC::off, j0, k0, &bars[sidx]);
    };
    if (tid == 0) { mbar_init(&bars[0], 1); mbar_init(&bars[1], 1); }
    __syncthreads();
    uint32_t phase[2] = {0u, 0u};
    bool failed = false;
    int tile = blockIdx.x, s = 0;
    if (tile < ntiles && tid == 0) issue(tile, 0);
    for (; tile < ntiles; tile += gridDim.x, s ^= 1) {
        int i0, j0, k0;
        tile_origin<DIM, TX, TY, TZ>(tile, ntx, nty, i0, j0, k0);
        const int next = tile + gridDim.x;
        if (next < ntiles && tid == 0) issue(next, s ^ 1);
        if (!stage_wait(&bars[s], phase[s], err)) { failed = true; break; }
        const T* sz = reinterpret_cast<const T*>(stage(s) + OZ);
        const T* spo = reinterpret_cast<const T*>(stage(s) + OP);
        const uint8_t* scd = stage(s) + OC;
        auto pv = [&](int q) -> T { return (sz[q] - m) + beta * spo[q]; };
        constexpr int ZB = P::BW * P::BY;
        for (int p = tid; p < TX * TY; p += nthr) {
            const int a = p % TX, bb = p / TX;
            const int i = i0 + a, j = j0 + bb;
            if (i > g.nx || j > g.ny) continue;
            for (int cc = 0; cc < (DIM == 3 ? TZ : 1); ++cc) {
                const int k = DIM == 3 ? k0 + cc : 0;
                if (DIM == 3 && k > g.nz) break;
                const int id = cidx(g, i, j, k);
                const uint32_t code = scd[a + P::XC::off + P::CW * (bb + P::CY * cc)];
                if (!(code & kActive)) {
                    ap[id] = T(0);
                    pnew[id] = T(0);
                    continue;
                }
                const int qb = (a + 1) + P::XB::off + P::BW * ((bb + 1) + P::BY * (DIM == 3 ? cc + 1 : 0));
                const T pc = pv(qb);
                const T wall = st.dirichlet ? -pc : pc;
                const T vL = (code & 2u) ? pv(qb - 1) : (i > 1 ? pc : wall);
                const T vR = (code & 1u) ? pv(qb + 1) : (i < g.nx ? pc : wall);
                const T vB = (code & 8u) ? pv(qb - P::BW) : (j > 1 ? pc : wall);
                const T vT = (code & 4u) ? pv(qb + P::BW) : (j < g.ny ? pc : wall);
                T a_;
                if (DIM == 3) {
                    const T vF = (code & 32u) ? pv(qb - ZB) : (k > 1 ? pc : wall);
                    const T vK = (code & 16u) ? pv(qb + ZB) : (k < g.nz ? pc : wall);
                    a_ = diag * pc - (vL + vR) * idx2 - (vB + vT) * idy2 - (vF + vK) * idz2;
                } else {
                    a_ = diag * pc - (vL + vR) * idx2 - (vB + vT) * idy2;
                }
                pnew[id] = pc;
                ap[id] = a_;
                acc[0] += (double)pc * (double)a_;
            }
        }
        __syncthreads();
    }
    if (failed) return;
    double tot[1];
    if (reduce_last<1>(acc, partials, &cg->counter[0], tot)) {
        const double pap = tot[0];
        cg->pap = pap;
        if (!(pap == pap)) { cg->status = CG_NAN; cg->done = 1; }
        else if (pap < cg->breakdown) { cg->status = CG_BREAKDOWN; cg->done = 1; }
        else cg->alpha = cg->rz_old / pap;
    }
}

// x += alpha p, r -= alpha Ap over the whole padded array with 16-byte vectors
// (p and Ap are 0 outside fluid cells, r starts at 0 there), then r.r; the last
// block applies the stopping rule sqrt(r.r) < tol_abs (pcg_3d.cpp:99-110).  In
// mixed mode meeting the rule only marks a candidate for the FP64 residual
// replacement to confirm.
template <class T>
struct Vec16;
template <> struct Vec16<float> { using V = float4; static constexpr int N = 4; };
template <> struct Vec16<double> { using V = double2; static constexpr int N = 2; };

template <class T>
__device__ __forceinline__ void vaxpy_rr(typename Vec16<T>::V& x, typename Vec16<T>::V& r,
                                         const typename Vec16<T>::V& p,
                                         const typename Vec16<T>::V& a, T alpha, double& rr);
template <>
__device__ __forceinline__ void vaxpy_rr<float>(float4& x, float4& r, const float4& p,
                                                const float4& a, float alpha, double& rr) {
    x.x += alpha * p.x; x.y += alpha * p.y; x.z += alpha * p.z; x.w += alpha * p.w;
    r.x = r.x - alpha * a.x; r.y = r.y - alpha * a.y; r.z = r.z - alpha * a.z; r.w = r.w - alpha * a.w;
    rr += (double)r.x * (double)r.x + (double)r.y * (double)r.y;
    rr += (double)r.z * (double)r.z + (double)r.w * (double)r.w;
}
template <>
__device__ __forceinline__ void vaxpy_rr<double>(double2& x, double2& r, const double2& p,
                                                 const double2& a, double alpha, double& rr) {
    x.x += alpha * p.x; x.y += alpha * p.y;
    r.x = r.x - alpha * a.x; r.y = r.y - alpha * a.y;
    rr += r.x * r.x;
    rr += r.y * r.y;
}

template <class T>
__global__ void __launch_bounds__(256) k_update_flat(long long nvec, T* x, T* r,
                                                     const T* __restrict__ p,
                                                     const T* __restrict__ ap, double* partials,
                                                     CGState* cg, double* hist) {
    if (cg->done) return;
    using V = typename Vec16<T>::V;
    const T alpha = (T)cg->alpha;
    V* xv = reinterpret_cast<V*>(x);
    V* rv = reinterpret_cast<V*>(r);
    const V* pv = reinterpret_cast<const V*>(p);
    const V* av = reinterpret_cast<const V*>(ap);
    double acc[1] = {0.0};
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nvec; t += stride) {
        V xx = xv[t], rr_ = rv[t];
        const V pp = __ldg(&pv[t]), aa = __ldg(&av[t]);
        vaxpy_rr<T>(xx, rr_, pp, aa, alpha, acc[0]);
        xv[t] = xx;
        rv[t] = rr_;
    }
    double tot[1];
    if (reduce_last<1>(acc, partials, &cg->counter[1], tot)) {
        const double rr = tot[0];
        cg->rr = rr;
        cg->iter += 1;
        if (hist) {
            if (cg->iter == 1) hist[0] = cg->r0;
            hist[cg->iter] = sqrt(rr);
        }
        if (!(rr == rr)) { cg->status = CG_NAN; cg->done = 1; }
        else if (sqrt(rr) < cg->tol_abs) {
            if (cg->replace_every > 0) cg->cand = 1;
            else { cg->status = CG_CONVERGED; cg->done = 1; }
        } else if (cg->iter >= cg->max_iter && cg->replace_every == 0) {
            cg->status = CG_MAXITER; cg->done = 1;
        }
    }
}

// Mixed mode fold over the whole padded array (x_lo is 0 outside fluid cells).
template <class T>
__global__ void k_fold_flat(long long n, double* xhi, T* xlo, const CGState* cg, int force) {
    if (!force) {
        if (cg->done) return;
        if (!(cg->cand || (cg->replace_every > 0 && cg->iter > 0 &&
                           cg->iter % cg->replace_every == 0)))
            return;
    }
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const T v = xlo[t];
        if (v != T(0)) {
            xhi[t] += (double)v;
            xlo[t] = T(0);
        }
    }
}

// Layout conversions between the reference's layout (gr) and the pitched one (g).
template <int DIM, class T>
__global__ void k_import(Geom g, Geom gr, const double* __restrict__ src, T* dst) {
    for_cells<DIM>(g, [&](int i, int j, int k, int id) { dst[id] = (T)src[cidx(gr, i, j, k)]; });
}
template <int DIM>
__global__ void k_import_mask(Geom g, Geom gr, const uint8_t* __restrict__ src, uint8_t* dst) {
    for_cells<DIM>(g, [&](int i, int j, int k, int id) {
        dst[id] = src[cidx(gr, i, j, k)] ? 1 : 0;
    });
}
// dst (reference layout) = src on interior cells (overwrite) or += src (accumulate).
template <int DIM, class T>
__global__ void k_export(Geom g, Geom gr, const T* __restrict__ src, double* dst, int accumulate) {
    for_cells<DIM>(g, [&](int i, int j, int k, int id) {
        const int rid = cidx(gr, i, j, k);
        dst[rid] = accumulate ? dst[rid] + (double)src[id] : (double)src[id];
    });
}

// Cell codes of a level (see the top of this file): fine = 1 adds the neighbour
// bits of the finest level.
template <int DIM>
__global__ void k_codes(Geom g, const uint8_t* __restrict__ s, uint8_t* code, int fine) {
    for_cells<DIM>(g, [&](int i, int j, int k, int id) {
        uint32_t c = ((i + j + k) & 1) ? kOdd : 0u;
        if (!s[id]) {
            c |= kActive;
            if (fine) {
                if (i < g.nx && !s[id + 1]) c |= 1u;
                if (i > 1 && !s[id - 1]) c |= 2u;
                if (j < g.ny && !s[id + g.sx]) c |= 4u;
                if (j > 1 && !s[id - g.sx]) c |= 8u;
                if (DIM == 3) {
                    if (k < g.nz && !s[id + g.sxy]) c |= 16u;
                    if (k > 1 && !s[id - g.sxy]) c |= 32u;
                }
            }
        }
        code[id] = (uint8_t)c;
    });
}

// Diagonal of every fluid cell of a coarse level (reference order, + walls) and
// its reciprocal (0 where the smoother skips the cell: d < 1e-30).
template <int DIM, class T>
__global__ void k_diag(Geom g, const uint8_t* __restrict__ s, const T* __restrict__ cx,
                       const T* __restrict__ cy, const T* __restrict__ cz,
                       const T* __restrict__ wd, T* dg, T* rdg) {
    for_cells<DIM>(g, [&](int, int, int, int id) {
        if (s[id]) return;
        T d = cx[id] + cx[id - 1] + cy[id] + cy[id - g.sx];
        if (DIM == 3) d = d + cz[id] + cz[id - g.sxy];
        if (wd) d = d + wd[id];
        dg[id] = d;
        rdg[id] = d < T(1e-30) ? T(0) : T(1) / d;
    });
}

}  // namespace
}  // namespace uaamg
