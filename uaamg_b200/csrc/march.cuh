// Stencil kernels that march along z through a level: a block owns a 32 x 8
// column tile of (i, j) cells and walks a chunk of z planes; each plane of every
// input array arrives as one TMA box (the tile plus a 1-cell ring) in a ring of
// shared-memory stages, kept several planes ahead of the compute so that the
// block always has loads in flight.  A z neighbour is the same column one
// stage up or down, so nothing along z is loaded twice, and a cell's value
// that needs a division (a pre-smoothed value) is computed once per plane into
// a shared plane buffer that the in-plane neighbours read.
//
// One V-cycle level = four marches (uaamg_preconditioner_3d.cpp:183-196):
//   k_fwd_smooth   forward red-black sweep from x = 0 (smooth(L,1,false),
//                  123-141): odd cells x = b/d, then even cells from them.
//   k_restrict_res residual b - A x and its restriction to the coarse b
//                  (restrictResidual, 144-165).
//   k_up_even      prolongation x += 2 x_coarse (prolongateAdd, 168-181) and
//                  the first colour (even) of the reverse sweep.
//   k_up_odd       the second colour (odd) of the reverse sweep, in place; on
//                  the finest level also the CG's z sums (pcg_3d.cpp:112-123).
// plus the CG search-direction march k_pmatvec (pcg_3d.cpp:38-55, 94-99,
// 113-122).
//
// Finest level: the couplings are the constants 1/h^2 wherever the neighbour is
// an interior fluid cell (uaamg_preconditioner_3d.cpp:50-66), and every other
// neighbour holds x = 0, so c_n x_n = (1/h^2) x_n for every neighbour; the
// diagonal comes from the cell-code bits in the reference's summation order.
// Coarse levels read their Galerkin coefficients and diagonal from TMA boxes.
//
// Arithmetic: every per-cell expression is the reference's, operand for operand
// and in its order, including the division by the diagonal; with the FP64
// instantiation compiled with -fmad=false the V-cycle reproduces the reference
// bit for bit.
#pragma once
#include "kernels.cuh"
#include "tma.cuh"

namespace uaamg {
namespace {

constexpr uint32_t kActive = 64u, kOdd = 128u;
constexpr int kMX = 32, kMY = 8;                   // column tile; one thread per column
constexpr int kHalo = 2 * (kMX + 2) + 2 * kMY;     // cells of the 1-cell ring: 84

__host__ __device__ constexpr size_t align128(size_t b) { return (b + 127) / 128 * 128; }

// Plane box of a level array: cells i in [i0-1, i0+32], j in [j0-1, j0+8] of one
// plane, where i0 = 1 + 32 bx, j0 = 1 + 8 by.  The start column i0-1 = 32 bx sits
// on a 16-byte boundary for every element size; the width is padded to 16 bytes.
template <class E>
struct PBox {
    static constexpr int W = ((kMX + 2) * (int)sizeof(E) + 15) / 16 * 16 / (int)sizeof(E);
    static constexpr int H = kMY + 2;
    static constexpr int N = W * H;
    static constexpr uint32_t BYTES = (uint32_t)(N * sizeof(E));
};
// Parent box: the next-coarser level's cells under a plane box, i.e. coarse
// columns [16 bx, 16 bx + 17], rows [4 by, 4 by + 5] of coarse plane (k+1)/2.
template <class E>
struct QBox {
    static constexpr int W = ((kMX / 2 + 2) * (int)sizeof(E) + 15) / 16 * 16 / (int)sizeof(E);
    static constexpr int H = kMY / 2 + 2;
    static constexpr uint32_t BYTES = (uint32_t)(W * H * sizeof(E));
};

// One ring stage: value boxes of T in slot order b, [x], [cx, cy, (cz), dg], the
// code box, optionally the parent box.
template <int DIM, class T, bool HASX, bool COEF, bool XC>
struct MPlan {
    static constexpr int NCOEF = COEF ? (DIM == 3 ? 4 : 3) : 0;
    static constexpr int QB = 0, QX = 1, QC0 = HASX ? 2 : 1;
    static constexpr int QCX = QC0, QCY = QC0 + 1, QCZ = QC0 + 2, QDG = QC0 + (DIM == 3 ? 3 : 2);
    static constexpr int NV = 1 + (HASX ? 1 : 0) + NCOEF;
    static constexpr bool XCB = XC;
    static constexpr size_t VB = align128(PBox<T>::BYTES);
    static constexpr size_t OFF_CODE = NV * VB;
    static constexpr size_t OFF_XC = OFF_CODE + align128(PBox<uint8_t>::BYTES);
    static constexpr size_t STAGE = OFF_XC + (XC ? align128(QBox<T>::BYTES) : 0);
    static constexpr uint32_t TX_BYTES =
        NV * PBox<T>::BYTES + PBox<uint8_t>::BYTES + (XC ? QBox<T>::BYTES : 0);
};

// Tensor maps of one march, in the stage's slot order.
struct MarchMaps {
    CUtensorMap v[6];
    CUtensorMap code;
    CUtensorMap xc;
};

template <class T>
struct MLevel {
    Geom g;          // this level
    Geom cg;         // next-coarser level (restriction target / prolongation source)
    T idx2, idy2, idz2;
    int dirichlet;   // finest level: add the Dirichlet wall diagonal
    int zc;          // planes per block (even)
};

__device__ __forceinline__ unsigned char* aligned_smem(unsigned char* raw) {
    const uintptr_t p = reinterpret_cast<uintptr_t>(raw);
    return reinterpret_cast<unsigned char*>((p + 127) & ~uintptr_t(127));
}

template <class E>
__device__ __forceinline__ E boxv(const unsigned char* st, size_t off, int q) {
    return reinterpret_cast<const E*>(st + off)[q];
}

// Ring position of the h-th cell of the 1-cell ring (h < kHalo).
__device__ __forceinline__ void halo_cell(int h, int& a, int& r) {
    if (h < kMX + 2) { a = h; r = 0; }
    else if (h < 2 * (kMX + 2)) { a = h - (kMX + 2); r = kMY + 1; }
    else if (h < 2 * (kMX + 2) + kMY) { a = 0; r = 1 + h - 2 * (kMX + 2); }
    else { a = kMX + 1; r = 1 + h - 2 * (kMX + 2) - kMY; }
}

// Finest-level diagonal from the neighbour bits, summed in the reference's order
// (uaamg_preconditioner_3d.cpp:72-74).
template <int DIM, class T>
__device__ __forceinline__ T fine_diag(uint32_t c, T idx2, T idy2, T idz2) {
    T d = ((c & 1u) ? idx2 : T(0)) + ((c & 2u) ? idx2 : T(0)) + ((c & 4u) ? idy2 : T(0)) +
          ((c & 8u) ? idy2 : T(0));
    if (DIM == 3) d = d + ((c & 16u) ? idz2 : T(0)) + ((c & 32u) ? idz2 : T(0));
    return d;
}

// Dirichlet wall diagonal of a finest-level cell (as k_fine_coeffs).
template <int DIM, class T>
__device__ __forceinline__ T wall_diag_at(const MLevel<T>& L, int i, int j, int k) {
    T w = T(0);
    if (i == 1) w += T(2) * L.idx2;
    if (i == L.g.nx) w += T(2) * L.idx2;
    if (j == 1) w += T(2) * L.idy2;
    if (j == L.g.ny) w += T(2) * L.idy2;
    if (DIM == 3 && k == 1) w += T(2) * L.idz2;
    if (DIM == 3 && k == L.g.nz) w += T(2) * L.idz2;
    return w;
}

// Diagonal of the cell at box position q of stage st (cell (i, j, k)).
template <int DIM, class T, class P, bool FINE>
__device__ __forceinline__ T mdiag(const MLevel<T>& L, const unsigned char* st, uint32_t c, int q,
                                   int i, int j, int k) {
    if constexpr (FINE) {
        T d = fine_diag<DIM, T>(c, L.idx2, L.idy2, L.idz2);
        if (L.dirichlet) d = d + wall_diag_at<DIM, T>(L, i, j, k);
        return d;
    } else {
        return boxv<T>(st, P::QDG * P::VB, q);
    }
}

// Couplings of the cell at box position q in the reference's order
// +x, -x, +y, -y, +z, -z (stc: this plane's stage, stm: the plane below).
template <int DIM, class T, class P, bool FINE>
__device__ __forceinline__ void mcoup(const MLevel<T>& L, const unsigned char* stc,
                                      const unsigned char* stm, int q, T (&c)[6]) {
    constexpr int W = PBox<T>::W;
    if constexpr (FINE) {
        c[0] = c[1] = L.idx2;
        c[2] = c[3] = L.idy2;
        c[4] = c[5] = L.idz2;
    } else {
        const T* cx = reinterpret_cast<const T*>(stc + P::QCX * P::VB);
        const T* cy = reinterpret_cast<const T*>(stc + P::QCY * P::VB);
        c[0] = cx[q];
        c[1] = cx[q - 1];
        c[2] = cy[q];
        c[3] = cy[q - W];
        if constexpr (DIM == 3) {
            c[4] = reinterpret_cast<const T*>(stc + P::QCZ * P::VB)[q];
            c[5] = reinterpret_cast<const T*>(stm + P::QCZ * P::VB)[q];
        } else {
            c[4] = c[5] = T(0);
        }
    }
}

// sum c_n v_n in the reference's order; v is a plane in PBox<T> layout, vp / vm the
// values one plane up / down.
template <int DIM, class T>
__device__ __forceinline__ T nbsum(const T (&c)[6], const T* v, int q, T vp, T vm) {
    constexpr int W = PBox<T>::W;
    T nb = c[0] * v[q + 1] + c[1] * v[q - 1] + c[2] * v[q + W] + c[3] * v[q - W];
    if (DIM == 3) nb = nb + c[4] * vp + c[5] * vm;
    return nb;
}

// Pre-smoothed value of the cell at box position q: an odd active cell smoothed
// from x = 0 has x = (b + 0)/d (skipped, x = 0, when d < 1e-30); every other cell 0.
template <int DIM, class T, class P, bool FINE>
__device__ __forceinline__ T presmooth(const MLevel<T>& L, const unsigned char* st, int a, int r,
                                       int i, int j, int k) {
    const uint32_t c = st[P::OFF_CODE + r * PBox<uint8_t>::W + a];
    if ((c & (kActive | kOdd)) != (kActive | kOdd)) return T(0);
    const int q = r * PBox<T>::W + a;
    const T d = mdiag<DIM, T, P, FINE>(L, st, c, q, i, j, k);
    if (d < T(1e-30)) return T(0);
    return (boxv<T>(st, P::QB * P::VB, q) + T(0)) / d;
}

// Prolongation 2 x_coarse of the fine cell at box position (a, r): the parent box
// holds 0 at solid and ghost coarse cells, so every fine cell may add it.
template <class T, class P>
__device__ __forceinline__ T prolong_at(const unsigned char* st, int a, int r) {
    return T(2) * boxv<T>(st, P::OFF_XC, ((r + 1) >> 1) * QBox<T>::W + ((a + 1) >> 1));
}

// March bookkeeping shared by the kernels: planes p0 .. plast pass through S
// stages; plane p uses stage (p - p0) % S for the ((p - p0) / S)-th time.
template <int S>
struct MRing {
    uint64_t* bars;
    unsigned char* base;
    size_t stage;
    int p0;
    __device__ unsigned char* at(int p) const { return base + (size_t)((p - p0) % S) * stage; }
    __device__ bool wait(int p) const {
        const int u = p - p0;
        return mbar_wait(&bars[u % S], (uint32_t)((u / S) & 1), kTmaWaitLimit);
    }
};

template <int DIM, class P>
__device__ __forceinline__ void issue_plane(const MarchMaps& M, unsigned char* st, uint64_t* bar,
                                            int k) {
    const int x0 = kMX * (int)blockIdx.x, y0 = kMY * (int)blockIdx.y;
    fence_proxy_async();
    mbar_expect_tx(bar, P::TX_BYTES);
#pragma unroll
    for (int q = 0; q < P::NV; ++q) tma_load<DIM>(st + q * P::VB, &M.v[q], x0, y0, k, bar);
    tma_load<DIM>(st + P::OFF_CODE, &M.code, x0, y0, k, bar);
    if constexpr (P::XCB) tma_load<DIM>(st + P::OFF_XC, &M.xc, x0 / 2, y0 / 2, (k + 1) >> 1, bar);
}

// Sets up the ring (thread 0 initialises the barriers and issues the first
// planes) and returns it; all threads return after a barrier.
template <int DIM, int S, class P>
__device__ __forceinline__ MRing<S> ring_start(const MarchMaps& M, unsigned char* sm, int p0,
                                               int plast) {
    MRing<S> R;
    R.bars = reinterpret_cast<uint64_t*>(sm);
    R.base = sm + 128;
    R.stage = P::STAGE;
    R.p0 = p0;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&R.bars[s], 1);
        for (int p = p0; p < p0 + S && p <= plast; ++p)
            issue_plane<DIM, P>(M, R.at(p), &R.bars[(p - p0) % S], p);
    }
    __syncthreads();
    return R;
}

// End of a march step: one block-wide verdict on the waits of the step, then the
// stage of plane `freed` is refilled with plane freed + S.
template <int DIM, int S, class P>
__device__ __forceinline__ bool ring_step(const MarchMaps& M, const MRing<S>& R, bool ok, int freed,
                                          int plast, int* err) {
    if (!__syncthreads_and(ok ? 1 : 0)) {
        if (threadIdx.x == 0 && threadIdx.y == 0) atomicExch(err, 1);
        return false;
    }
    if (threadIdx.x == 0 && threadIdx.y == 0 && freed >= R.p0 && freed + S <= plast)
        issue_plane<DIM, P>(M, R.at(freed + S), &R.bars[(freed - R.p0) % S], freed + S);
    return true;
}

// Dynamic shared memory of each march (ring + plane buffers + 128 B barriers + 128 B
// alignment slack).
template <int DIM, class T, bool FINE> struct FwdCfg {
    using P = MPlan<DIM, T, false, !FINE, false>;
    static constexpr int S = FINE ? 6 : 4;
    static constexpr size_t BYTES = 256 + S * P::STAGE + 2 * align128(PBox<T>::BYTES);
};
template <int DIM, class T, bool FINE> struct ResCfg {
    using P = MPlan<DIM, T, true, !FINE, false>;
    static constexpr int S = FINE ? 5 : 4;
    static constexpr size_t BYTES = 256 + S * P::STAGE + align128(2 * kMX * kMY * sizeof(T));
};
template <int DIM, class T, bool FINE> struct UpeCfg {
    using P = MPlan<DIM, T, false, !FINE, true>;
    static constexpr int S = FINE ? 6 : 4;
    static constexpr size_t BYTES = 256 + S * P::STAGE + 2 * align128(PBox<T>::BYTES);
};
template <int DIM, class T, bool FINE> struct UpoCfg {
    using P = MPlan<DIM, T, true, !FINE, false>;
    static constexpr int S = FINE ? 5 : 4;
    static constexpr size_t BYTES = 256 + S * P::STAGE;
};
template <int DIM, class T> struct PmvCfg {
    using P = MPlan<DIM, T, true, false, false>;
    static constexpr int S = 5;
    static constexpr size_t BYTES = 256 + S * P::STAGE;
};

// z range of this block: planes kb .. ke-1 (3D); the single plane 0 (2D).
template <int DIM>
__device__ __forceinline__ void zrange(const Geom& g, int zc, int& kb, int& ke) {
    if (DIM == 3) {
        kb = 1 + (int)blockIdx.z * zc;
        ke = min(kb + zc, g.nz + 1);
    } else {
        kb = 0;
        ke = 1;
    }
}

// ---------------------------------------------------------------------------
// Forward sweep from x = 0: x = (b + 0)/d on odd cells, then
// x = (b + sum c_n x_n)/d on even cells; writes x on every interior cell.
template <int DIM, class T, bool FINE>
__global__ void __launch_bounds__(256) k_fwd_smooth(const __grid_constant__ MarchMaps M,
                                                    MLevel<T> L, T* __restrict__ x,
                                                    const int* __restrict__ done, int* err) {
    if (done && *done) return;
    using C = FwdCfg<DIM, T, FINE>;
    using P = typename C::P;
    constexpr int S = C::S, W = PBox<T>::W, N = PBox<T>::N;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* sm = aligned_smem(smem_raw);
    T* Yb = reinterpret_cast<T*>(sm + 128 + S * P::STAGE);
    const Geom& g = L.g;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kMX * ty;
    const int i = 1 + kMX * (int)blockIdx.x + tx, j = 1 + kMY * (int)blockIdx.y + ty;
    const bool own = i <= g.nx && j <= g.ny;
    const int q = (ty + 1) * W + tx + 1;
    int ha = 0, hr = 0;
    if (tid < kHalo) halo_cell(tid, ha, hr);
    const int hq = hr * W + ha, hi = i - tx - 1 + ha, hj = j - ty - 1 + hr;
    int kb, ke;
    zrange<DIM>(g, L.zc, kb, ke);
    const int p0 = DIM == 3 ? kb - 1 : 0, plast = DIM == 3 ? ke : 0;
    MRing<S> R = ring_start<DIM, S, P>(M, sm, p0, plast);
    bool ok = R.wait(p0);
    // y: pre-smoothed values of this column at planes k-1, k, k+1
    T ym = T(0), y0 = T(0), yp = T(0);
    if (DIM == 3) y0 = presmooth<DIM, T, P, FINE>(L, R.at(p0), tx + 1, ty + 1, i, j, p0);
#pragma unroll 1
    for (int k = p0; k < ke; ++k) {
        const int kn = DIM == 3 ? k + 1 : 0;  // plane whose y plane is built this step
        if (DIM == 3) ok &= R.wait(kn);
        {
            const unsigned char* sn = R.at(kn);
            T* Yn = Yb + (kn & 1) * N;
            yp = presmooth<DIM, T, P, FINE>(L, sn, tx + 1, ty + 1, i, j, kn);
            Yn[q] = yp;
            if (tid < kHalo) Yn[hq] = presmooth<DIM, T, P, FINE>(L, sn, ha, hr, hi, hj, kn);
        }
        if (DIM == 2) {
            y0 = yp;
            __syncthreads();
        }
        if (k >= kb) {
            const unsigned char* sc = R.at(k);
            const uint32_t c = sc[P::OFF_CODE + (ty + 1) * PBox<uint8_t>::W + tx + 1];
            T xv = T(0);
            if (c & kActive) {
                if (c & kOdd) {
                    xv = y0;
                } else {
                    const T d = mdiag<DIM, T, P, FINE>(L, sc, c, q, i, j, k);
                    if (!(d < T(1e-30))) {
                        T cc[6];
                        mcoup<DIM, T, P, FINE>(L, sc, DIM == 3 ? R.at(k - 1) : sc, q, cc);
                        const T* Yc = Yb + (k & 1) * N;
                        xv = (boxv<T>(sc, P::QB * P::VB, q) + nbsum<DIM, T>(cc, Yc, q, yp, ym)) / d;
                    }
                }
            }
            if (own) x[cidx(g, i, j, k)] = xv;
        }
        if (DIM == 2) break;
        ym = y0;
        y0 = yp;
        if (!ring_step<DIM, S, P>(M, R, ok, k - 1, plast, err)) return;
    }
    if (DIM == 2 && !__syncthreads_and(ok ? 1 : 0) && tid == 0) atomicExch(err, 1);
}

// Residual r = b - A x of every fluid cell and its restriction
// b_c = sum over the 2x2(x2) children, in the reference's (di, dj, dk) order; the
// children of a coarse cell sit in two adjacent columns, two adjacent rows and
// two consecutive planes of one block, and meet in shared memory.
template <int DIM, class T, bool FINE>
__global__ void __launch_bounds__(256) k_restrict_res(const __grid_constant__ MarchMaps M,
                                                      MLevel<T> L, const uint8_t* __restrict__ ccode,
                                                      T* __restrict__ cb,
                                                      const int* __restrict__ done, int* err) {
    if (done && *done) return;
    using C = ResCfg<DIM, T, FINE>;
    using P = typename C::P;
    constexpr int S = C::S, W = PBox<T>::W;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* sm = aligned_smem(smem_raw);
    T* Rb = reinterpret_cast<T*>(sm + 128 + S * P::STAGE);  // [ty][tx][dk]
    const Geom& g = L.g;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kMX * ty;
    const int i = 1 + kMX * (int)blockIdx.x + tx, j = 1 + kMY * (int)blockIdx.y + ty;
    const int q = (ty + 1) * W + tx + 1;
    int kb, ke;
    zrange<DIM>(g, L.zc, kb, ke);
    const int p0 = DIM == 3 ? kb - 1 : 0, plast = DIM == 3 ? ke : 0;
    MRing<S> R = ring_start<DIM, S, P>(M, sm, p0, plast);
    bool ok = R.wait(p0);
    if (DIM == 3) ok &= R.wait(kb);
    T rlo = T(0);
#pragma unroll 1
    for (int k = kb; k < ke; ++k) {
        if (DIM == 3) ok &= R.wait(k + 1);
        const unsigned char* sc = R.at(k);
        const uint32_t c = sc[P::OFF_CODE + (ty + 1) * PBox<uint8_t>::W + tx + 1];
        T rv = T(0);
        if (c & kActive) {
            const T* xb = reinterpret_cast<const T*>(sc + P::QX * P::VB);
            const T d = mdiag<DIM, T, P, FINE>(L, sc, c, q, i, j, k);
            T cc[6];
            mcoup<DIM, T, P, FINE>(L, sc, DIM == 3 ? R.at(k - 1) : sc, q, cc);
            T ax = d * xb[q] - cc[0] * xb[q + 1] - cc[1] * xb[q - 1] - cc[2] * xb[q + W] -
                   cc[3] * xb[q - W];
            if (DIM == 3)
                ax = ax - cc[4] * boxv<T>(R.at(k + 1), P::QX * P::VB, q) -
                     cc[5] * boxv<T>(R.at(k - 1), P::QX * P::VB, q);
            rv = boxv<T>(sc, P::QB * P::VB, q) - ax;
        }
        // children with dk = 0 live on odd planes (k = 2 kc - 1); the pair is complete
        // on the even plane that follows
        const bool pair = DIM == 2 || (k & 1) == 0;
        if (DIM == 3 && !pair) rlo = rv;
        if (pair) {
            Rb[2 * tid] = DIM == 3 ? rlo : rv;
            Rb[2 * tid + 1] = rv;
        }
        if (DIM == 3) {
            if (!ring_step<DIM, S, P>(M, R, ok, k - 1, plast, err)) return;
        } else if (!__syncthreads_and(ok ? 1 : 0)) {
            if (tid == 0) atomicExch(err, 1);
            return;
        }
        if (pair && tid < (kMX / 2) * (kMY / 2)) {
            const int ca = tid % (kMX / 2), cr = tid / (kMX / 2);
            const int ic = kMX / 2 * (int)blockIdx.x + 1 + ca;
            const int jc = kMY / 2 * (int)blockIdx.y + 1 + cr;
            const int kc = DIM == 3 ? k / 2 : 0;
            if (ic <= L.cg.nx && jc <= L.cg.ny) {
                const int cid = cidx(L.cg, ic, jc, kc);
                T s = T(0);
                for (int di = 0; di < 2; ++di)
                    for (int dj = 0; dj < 2; ++dj) {
                        const int t = (2 * cr + dj) * kMX + 2 * ca + di;
                        s += Rb[2 * t];
                        if (DIM == 3) s += Rb[2 * t + 1];
                    }
                cb[cid] = (ccode[cid] & kActive) ? s : T(0);
            }
        }
        // Rb is rewritten two steps later, after another block-wide barrier
    }
}

// Prolongation and the first (even) colour of the reverse sweep.  Odd cells hold
// their pre-smoothed value plus the prolongation, (b + 0)/d + 2 x_c; even cells are
// smoothed from those: x = (b + sum c_n x_n)/d (a skipped even cell keeps
// 0 + 2 x_c).  Writes x on every interior cell.
template <int DIM, class T, bool FINE>
__global__ void __launch_bounds__(256) k_up_even(const __grid_constant__ MarchMaps M, MLevel<T> L,
                                                 T* __restrict__ x, const int* __restrict__ done,
                                                 int* err) {
    if (done && *done) return;
    using C = UpeCfg<DIM, T, FINE>;
    using P = typename C::P;
    constexpr int S = C::S, W = PBox<T>::W, N = PBox<T>::N;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* sm = aligned_smem(smem_raw);
    T* Yb = reinterpret_cast<T*>(sm + 128 + S * P::STAGE);
    const Geom& g = L.g;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + kMX * ty;
    const int i = 1 + kMX * (int)blockIdx.x + tx, j = 1 + kMY * (int)blockIdx.y + ty;
    const bool own = i <= g.nx && j <= g.ny;
    const int q = (ty + 1) * W + tx + 1;
    int ha = 0, hr = 0;
    if (tid < kHalo) halo_cell(tid, ha, hr);
    const int hq = hr * W + ha, hi = i - tx - 1 + ha, hj = j - ty - 1 + hr;
    // odd cells: pre-smoothed value + prolongation; others 0
    auto oddval = [&](const unsigned char* st, int qq, int a, int r, int ci, int cj, int ck) -> T {
        const uint32_t c = st[P::OFF_CODE + r * PBox<uint8_t>::W + a];
        if ((c & (kActive | kOdd)) != (kActive | kOdd)) return T(0);
        const T d = mdiag<DIM, T, P, FINE>(L, st, c, qq, ci, cj, ck);
        const T pre = d < T(1e-30) ? T(0) : (boxv<T>(st, P::QB * P::VB, qq) + T(0)) / d;
        return pre + prolong_at<T, P>(st, a, r);
    };
    int kb, ke;
    zrange<DIM>(g, L.zc, kb, ke);
    const int p0 = DIM == 3 ? kb - 1 : 0, plast = DIM == 3 ? ke : 0;
    MRing<S> R = ring_start<DIM, S, P>(M, sm, p0, plast);
    bool ok = R.wait(p0);
    T ym = T(0), y0 = T(0), yp = T(0);
    if (DIM == 3) y0 = oddval(R.at(p0), q, tx + 1, ty + 1, i, j, p0);
#pragma unroll 1
    for (int k = p0; k < ke; ++k) {
        const int kn = DIM == 3 ? k + 1 : 0;
        if (DIM == 3) ok &= R.wait(kn);
        {
            const unsigned char* sn = R.at(kn);
            T* Yn = Yb + (kn & 1) * N;
            yp = oddval(sn, q, tx + 1, ty + 1, i, j, kn);
            Yn[q] = yp;
            if (tid < kHalo) Yn[hq] = oddval(sn, hq, ha, hr, hi, hj, kn);
        }
        if (DIM == 2) {
            y0 = yp;
            __syncthreads();
        }
        if (k >= kb) {
            const unsigned char* sc = R.at(k);
            const uint32_t c = sc[P::OFF_CODE + (ty + 1) * PBox<uint8_t>::W + tx + 1];
            T xv = T(0);
            if (c & kActive) {
                if (c & kOdd) {
                    xv = y0;
                } else {
                    const T d = mdiag<DIM, T, P, FINE>(L, sc, c, q, i, j, k);
                    if (d < T(1e-30)) {
                        xv = T(0) + prolong_at<T, P>(sc, tx + 1, ty + 1);
                    } else {
                        T cc[6];
                        mcoup<DIM, T, P, FINE>(L, sc, DIM == 3 ? R.at(k - 1) : sc, q, cc);
                        const T* Yc = Yb + (k & 1) * N;
                        xv = (boxv<T>(sc, P::QB * P::VB, q) + nbsum<DIM, T>(cc, Yc, q, yp, ym)) / d;
                    }
                }
            }
            if (own) x[cidx(g, i, j, k)] = xv;
        }
        if (DIM == 2) break;
        ym = y0;
        y0 = yp;
        if (!ring_step<DIM, S, P>(M, R, ok, k - 1, plast, err)) return;
    }
    if (DIM == 2 && !__syncthreads_and(ok ? 1 : 0) && tid == 0) atomicExch(err, 1);
}

// Second (odd) colour of the reverse sweep, in place: odd cells read only even
// neighbours, which this kernel does not write.  ZDOT (finest level): also the
// fluid sums of z, r*z and r (r = this level's b) and the CG's projection / beta.
template <int DIM, class T, bool FINE, bool ZDOT>
__global__ void __launch_bounds__(256) k_up_odd(const __grid_constant__ MarchMaps M, MLevel<T> L,
                                                T* x, const int* __restrict__ done, int* err,
                                                double* partials, CGState* cg) {
    if (done && *done) return;
    using C = UpoCfg<DIM, T, FINE>;
    using P = typename C::P;
    constexpr int S = C::S, W = PBox<T>::W;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* sm = aligned_smem(smem_raw);
    const Geom& g = L.g;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = 1 + kMX * (int)blockIdx.x + tx, j = 1 + kMY * (int)blockIdx.y + ty;
    const bool own = i <= g.nx && j <= g.ny;
    const int q = (ty + 1) * W + tx + 1;
    double acc[3] = {0.0, 0.0, 0.0};
    int kb, ke;
    zrange<DIM>(g, L.zc, kb, ke);
    const int p0 = DIM == 3 ? kb - 1 : 0, plast = DIM == 3 ? ke : 0;
    MRing<S> R = ring_start<DIM, S, P>(M, sm, p0, plast);
    bool ok = R.wait(p0);
    if (DIM == 3) ok &= R.wait(kb);
    bool failed = false;
#pragma unroll 1
    for (int k = kb; k < ke; ++k) {
        if (DIM == 3) ok &= R.wait(k + 1);
        const unsigned char* sc = R.at(k);
        const uint32_t c = sc[P::OFF_CODE + (ty + 1) * PBox<uint8_t>::W + tx + 1];
        if (c & kActive) {
            const T* xb = reinterpret_cast<const T*>(sc + P::QX * P::VB);
            T xv = xb[q];
            if (c & kOdd) {
                const T d = mdiag<DIM, T, P, FINE>(L, sc, c, q, i, j, k);
                if (!(d < T(1e-30))) {
                    T cc[6];
                    mcoup<DIM, T, P, FINE>(L, sc, DIM == 3 ? R.at(k - 1) : sc, q, cc);
                    const T vp = DIM == 3 ? boxv<T>(R.at(k + 1), P::QX * P::VB, q) : T(0);
                    const T vm = DIM == 3 ? boxv<T>(R.at(k - 1), P::QX * P::VB, q) : T(0);
                    xv = (boxv<T>(sc, P::QB * P::VB, q) + nbsum<DIM, T>(cc, xb, q, vp, vm)) / d;
                    if (own) x[cidx(g, i, j, k)] = xv;
                }
            }
            if (ZDOT && own) {
                const double zv = (double)xv, rv = (double)boxv<T>(sc, P::QB * P::VB, q);
                acc[0] += zv;
                acc[1] += rv * zv;
                acc[2] += rv;
            }
        }
        if (DIM == 3) {
            if (!ring_step<DIM, S, P>(M, R, ok, k - 1, plast, err)) { failed = true; break; }
        } else if (!__syncthreads_and(ok ? 1 : 0)) {
            if (tx == 0 && ty == 0) atomicExch(err, 1);
            failed = true;
        }
    }
    if (ZDOT && !failed) {
        double tot[3];
        if (reduce_last<3>(acc, partials, &cg->counter[2], tot)) finish_zdot(cg, tot);
    }
}

// CG search direction fused with the operator: p = (z - m) + beta p_old on fluid
// cells (pcg_3d.cpp:113-122) and Ap from the new p of the neighbours, formed on
// the fly from the staged z and p_old (a solid or out-of-domain neighbour reads
// p_C -- Neumann -- or -p_C at a Dirichlet wall; pcg_3d.cpp:38-55); p.Ap is
// reduced and the last block sets alpha = rz_old / p.Ap or stops on breakdown
// (pcg_3d.cpp:94-99).  p_old and p_new are distinct buffers.
template <int DIM, class T>
__global__ void __launch_bounds__(256) k_pmatvec(const __grid_constant__ MarchMaps M, Geom g,
                                                 int zc, T* __restrict__ pnew, T* __restrict__ ap,
                                                 Stencil st, double* partials, CGState* cg,
                                                 int* err) {
    if (cg->done) return;
    using C = PmvCfg<DIM, T>;
    using P = typename C::P;
    constexpr int S = C::S, W = PBox<T>::W;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* sm = aligned_smem(smem_raw);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = 1 + kMX * (int)blockIdx.x + tx, j = 1 + kMY * (int)blockIdx.y + ty;
    const bool own = i <= g.nx && j <= g.ny;
    const int q = (ty + 1) * W + tx + 1;
    const T m = (T)cg->mean_z, beta = (T)cg->beta;
    const T idx2 = (T)st.idx2, idy2 = (T)st.idy2, idz2 = (T)st.idz2, diag = (T)st.diag;
    double acc[1] = {0.0};
    int kb, ke;
    zrange<DIM>(g, zc, kb, ke);
    const int p0 = DIM == 3 ? kb - 1 : 0, plast = DIM == 3 ? ke : 0;
    MRing<S> R = ring_start<DIM, S, P>(M, sm, p0, plast);
    bool ok = R.wait(p0);
    if (DIM == 3) ok &= R.wait(kb);
    bool failed = false;
    auto pv = [&](const unsigned char* s_, int qq) -> T {
        return (boxv<T>(s_, P::QB * P::VB, qq) - m) + beta * boxv<T>(s_, P::QX * P::VB, qq);
    };
#pragma unroll 1
    for (int k = kb; k < ke; ++k) {
        if (DIM == 3) ok &= R.wait(k + 1);
        const unsigned char* sc = R.at(k);
        const uint32_t c = sc[P::OFF_CODE + (ty + 1) * PBox<uint8_t>::W + tx + 1];
        T pc = T(0), a_ = T(0);
        if (c & kActive) {
            pc = pv(sc, q);
            const T wall = st.dirichlet ? -pc : pc;
            const T vL = (c & 2u) ? pv(sc, q - 1) : (i > 1 ? pc : wall);
            const T vR = (c & 1u) ? pv(sc, q + 1) : (i < g.nx ? pc : wall);
            const T vB = (c & 8u) ? pv(sc, q - W) : (j > 1 ? pc : wall);
            const T vT = (c & 4u) ? pv(sc, q + W) : (j < g.ny ? pc : wall);
            if (DIM == 3) {
                const T vF = (c & 32u) ? pv(R.at(k - 1), q) : (k > 1 ? pc : wall);
                const T vK = (c & 16u) ? pv(R.at(k + 1), q) : (k < g.nz ? pc : wall);
                a_ = diag * pc - (vL + vR) * idx2 - (vB + vT) * idy2 - (vF + vK) * idz2;
            } else {
                a_ = diag * pc - (vL + vR) * idx2 - (vB + vT) * idy2;
            }
            acc[0] += (double)pc * (double)a_;
        }
        if (own) {
            const int id = cidx(g, i, j, k);
            pnew[id] = pc;
            ap[id] = a_;
        }
        if (DIM == 3) {
            if (!ring_step<DIM, S, P>(M, R, ok, k - 1, plast, err)) { failed = true; break; }
        } else if (!__syncthreads_and(ok ? 1 : 0)) {
            if (tx == 0 && ty == 0) atomicExch(err, 1);
            failed = true;
        }
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

}  // namespace
}  // namespace uaamg
