// Stencil kernels that march along z through a level: a block owns a 32 x 16
// column tile of (i, j) cells (256 threads, each owning a pair of cells (i, j),
// (i, j+1) -- one of each colour, so a warp never splits on the red-black
// parity) and walks a chunk of z planes; each plane of every input array arrives as one TMA box (the tile plus
// a 1-cell ring) in a ring of shared-memory stages, issued several planes ahead
// of the compute so that the block always has loads in flight.  One thread waits
// on the stage's mbarrier for the plane the next step needs and the step's block
// barrier hands it to everyone.  A z neighbour is the same column one stage up
// or down, so nothing along z is loaded twice, and a value that needs a division
// (a pre-smoothed cell) is computed once per plane into a shared plane buffer
// that the in-plane neighbours read.
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
// diagonal is a 64-entry table indexed by the cell-code neighbour bits, summed
// in the reference's order.  Coarse levels read their Galerkin coefficients and
// diagonal from TMA boxes.
//
// Arithmetic: every per-cell expression is the reference's, operand for operand
// and in its order, including the division by the diagonal; with the FP64
// instantiation compiled with -fmad=false the V-cycle reproduces the reference
// bit for bit.
#pragma once
#include <cuda_fp16.h>

#include <type_traits>

#include "kernels.cuh"
#include "tma.cuh"

namespace uaamg {
namespace {

constexpr int kMX = 32, kMY = 16;                  // column tile
constexpr int kThreads = 256;                      // one thread per x-pair of the tile
constexpr int kHaloOdd = 2 * (kMX / 2 + 1) + kMY;  // odd cells of the 1-cell ring: 50

__host__ __device__ constexpr size_t align128(size_t b) { return (b + 127) / 128 * 128; }

// Plane box of a level array: cells i in [i0-1, i0+32], j in [j0-1, j0+16] of one
// plane, where i0 = 1 + 32 bx, j0 = 1 + 16 by.  The start column i0-1 = 32 bx sits
// on a 16-byte boundary for every element size; the width is padded to 16 bytes.
template <class E>
struct PBox {
    static constexpr int W = ((kMX + 2) * (int)sizeof(E) + 15) / 16 * 16 / (int)sizeof(E);
    static constexpr int H = kMY + 2;
    static constexpr int N = W * H;
    static constexpr uint32_t BYTES = (uint32_t)(N * sizeof(E));
};
// Parent box: the next-coarser level's cells under a plane box, i.e. coarse
// columns [16 bx, 16 bx + 17], rows [8 by, 8 by + 9] of coarse plane (k+1)/2.
template <class E>
struct QBox {
    static constexpr int W = ((kMX / 2 + 2) * (int)sizeof(E) + 15) / 16 * 16 / (int)sizeof(E);
    static constexpr int H = kMY / 2 + 2;
    static constexpr uint32_t BYTES = (uint32_t)(W * H * sizeof(E));
};

// One ring stage: value boxes of T in slot order b, [x], [dg], then (coarse levels)
// the coupling boxes cx, cy, [cz] of the coupling storage type CS, the code box,
// optionally the parent box.  Slot q's map is MarchMaps::v[q].
template <int DIM, class T, bool HASX, bool COEF, bool XC, class CS = T>
struct MPlan {
    static constexpr int NT = 1 + (HASX ? 1 : 0) + (COEF ? 1 : 0);  // boxes of T
    static constexpr int NCS = COEF ? (DIM == 3 ? 3 : 2) : 0;       // boxes of CS
    static constexpr int NV = NT + NCS;
    static constexpr int QB = 0, QX = 1, QDG = NT - 1;
    static constexpr bool XCB = XC;
    static constexpr size_t VB = align128(PBox<T>::BYTES);
    static constexpr size_t CB = align128(PBox<CS>::BYTES);
    static constexpr size_t OFF_CX = NT * VB, OFF_CY = OFF_CX + CB, OFF_CZ = OFF_CY + CB;
    static constexpr size_t OFF_CODE = NT * VB + NCS * CB;
    static constexpr size_t OFF_XC = OFF_CODE + align128(PBox<uint8_t>::BYTES);
    static constexpr size_t STAGE = OFF_XC + (XC ? align128(QBox<T>::BYTES) : 0);
    static constexpr uint32_t TX_BYTES = NT * PBox<T>::BYTES + NCS * PBox<CS>::BYTES +
                                         PBox<uint8_t>::BYTES + (XC ? QBox<T>::BYTES : 0);
    __host__ __device__ static constexpr size_t box_off(int q) {
        return q < NT ? (size_t)q * VB : NT * VB + (size_t)(q - NT) * CB;
    }
};

// Shared memory of a march: 128 B of barriers, the diagonal table, S stages, then
// the plane buffers.
template <class T, int S, class P>
struct MLayout {
    static constexpr size_t OFF_LUT = 128;
    static constexpr size_t OFF_RING = OFF_LUT + align128(64 * sizeof(T));
    static constexpr size_t OFF_EXTRA = OFF_RING + S * P::STAGE;
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
    T csx, csy, csz; // coarse levels: coupling = stored value * cs (1 when stored in T)
    int dirichlet;   // finest level: add the Dirichlet wall diagonal
    int zc;          // planes per block (even)
};

// A stored coupling as T: FP16 couplings hold the coupling / cs (a face count).
template <class T, class CS>
__device__ __forceinline__ T coupling(CS v, T cs) {
    if constexpr (std::is_same<CS, T>::value) {
        return v;
    } else {
        return (T)__half2float(v) * cs;
    }
}

// The dynamic shared memory of a march, declared 128-byte aligned (every TMA box
// sits at a multiple of 128 bytes from it).  Used directly -- never through an
// integer -- so that every access compiles to a 32-bit shared-memory address.  A
// base that is not 128-byte aligned sets the error word to 2 and the block returns
// before it issues a load.
#define UAAMG_MARCH_SMEM(sm, err)                                                 \
    extern __shared__ __align__(128) unsigned char smem_raw[];                   \
    unsigned char* sm = smem_raw;                                                \
    if (smem_u32(sm) & 127u) {                                                   \
        if (threadIdx.x == 0) atomicExch(err, 2);                                \
        return;                                                                  \
    }

template <class E>
__device__ __forceinline__ E boxv(const unsigned char* st, size_t off, int q) {
    return reinterpret_cast<const E*>(st + off)[q];
}

// Box position of the h-th odd cell of the 1-cell ring (h < kHaloOdd), where the
// box's corner cell (i0-1, j0-1, k) has parity s0: the odd cells of the bottom and
// top rows (17 each), then of the left and right columns (8 each).
__device__ __forceinline__ void halo_odd(int h, int s0, int& a, int& r) {
    constexpr int R = kMX / 2 + 1;
    if (h < R) { r = 0; a = 2 * h + (1 - s0); }
    else if (h < 2 * R) { r = kMY + 1; a = 2 * (h - R) + s0; }
    else if (h < 2 * R + kMY / 2) { a = 0; r = 1 + 2 * (h - 2 * R) + s0; }
    else { a = kMX + 1; r = 1 + 2 * (h - 2 * R - kMY / 2) + (1 - s0); }
}

// Finest-level diagonal table: entry c is the diagonal of a cell whose neighbour
// bits are c, summed in the reference's order (uaamg_preconditioner_3d.cpp:72-74).
template <int DIM, class T>
__device__ __forceinline__ void build_lut(T* lut, T idx2, T idy2, T idz2) {
    const int t = threadIdx.x + blockDim.x * threadIdx.y;
    if (t < 64) {
        const uint32_t c = (uint32_t)t;
        T d = ((c & 1u) ? idx2 : T(0)) + ((c & 2u) ? idx2 : T(0)) + ((c & 4u) ? idy2 : T(0)) +
              ((c & 8u) ? idy2 : T(0));
        if (DIM == 3) d = d + ((c & 16u) ? idz2 : T(0)) + ((c & 32u) ? idz2 : T(0));
        lut[t] = d;
    }
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

// Diagonal of the cell with code c at box position q of stage st (cell (i, j, k)).
template <int DIM, class T, class P, bool FINE>
__device__ __forceinline__ T mdiag(const MLevel<T>& L, const T* lut, const unsigned char* st,
                                   uint32_t c, int q, int i, int j, int k) {
    if constexpr (FINE) {
        T d = lut[c & 63u];
        if (L.dirichlet) d = d + wall_diag_at<DIM, T>(L, i, j, k);
        return d;
    } else {
        return boxv<T>(st, P::box_off(P::QDG), q);
    }
}

// Couplings of the cell at box column a, row r in the reference's order
// +x, -x, +y, -y, +z, -z (stc: this plane's stage, stm: the plane below).
template <int DIM, class T, class P, bool FINE, class CS>
__device__ __forceinline__ void mcoup(const MLevel<T>& L, const unsigned char* stc,
                                      const unsigned char* stm, int a, int r, T (&c)[6]) {
    if constexpr (FINE) {
        c[0] = c[1] = L.idx2;
        c[2] = c[3] = L.idy2;
        c[4] = c[5] = L.idz2;
    } else {
        constexpr int W = PBox<CS>::W;
        const int q = r * W + a;
        const CS* cx = reinterpret_cast<const CS*>(stc + P::OFF_CX);
        const CS* cy = reinterpret_cast<const CS*>(stc + P::OFF_CY);
        c[0] = coupling<T, CS>(cx[q], L.csx);
        c[1] = coupling<T, CS>(cx[q - 1], L.csx);
        c[2] = coupling<T, CS>(cy[q], L.csy);
        c[3] = coupling<T, CS>(cy[q - W], L.csy);
        if constexpr (DIM == 3) {
            c[4] = coupling<T, CS>(reinterpret_cast<const CS*>(stc + P::OFF_CZ)[q], L.csz);
            c[5] = coupling<T, CS>(reinterpret_cast<const CS*>(stm + P::OFF_CZ)[q], L.csz);
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

// A smoother's quotient num / d.  The mixed form (couplings stored in FP16)
// divides with the fast reciprocal, within 2 ulp: its V-cycle is only a
// preconditioner, and every cell's diagonal is perturbed the same way in each
// sweep, so the cycle stays symmetric.  Plain FP32 keeps IEEE division and FP64
// the reference's (bit-exact) division.
template <class T, class CS>
__device__ __forceinline__ T mdiv(T num, T d) {
    if constexpr (!std::is_same<CS, T>::value) return __fdividef(num, d);
    else return num / d;
}

// Pre-smoothed value of the cell at box position (a, r): an odd active cell
// smoothed from x = 0 has x = (b + 0)/d (skipped, x = 0, when d < 1e-30); every
// other cell 0.
template <int DIM, class T, class P, bool FINE, class CS>
__device__ __forceinline__ T presmooth(const MLevel<T>& L, const T* lut, const unsigned char* st,
                                       int a, int r, int i, int j, int k) {
    const uint32_t c = st[P::OFF_CODE + r * PBox<uint8_t>::W + a];
    if ((c & (kActive | kOdd)) != (kActive | kOdd)) return T(0);
    const int q = r * PBox<T>::W + a;
    const T d = mdiag<DIM, T, P, FINE>(L, lut, st, c, q, i, j, k);
    if (d < T(1e-30)) return T(0);
    return mdiv<T, CS>(boxv<T>(st, P::QB * P::VB, q) + T(0), d);
}

// Prolongation 2 x_coarse of the fine cell at box position (a, r): the parent box
// holds 0 at solid and ghost coarse cells, so every fine cell may add it.
template <class T, class P>
__device__ __forceinline__ T prolong_at(const unsigned char* st, int a, int r) {
    return T(2) * boxv<T>(st, P::OFF_XC, ((r + 1) >> 1) * QBox<T>::W + ((a + 1) >> 1));
}

template <int DIM, class P>
__device__ __forceinline__ void issue_plane(const MarchMaps& M, unsigned char* st, uint64_t* bar,
                                            int k) {
    const int x0 = kMX * (int)blockIdx.x, y0 = kMY * (int)blockIdx.y;
    fence_proxy_async();
    mbar_expect_tx(bar, P::TX_BYTES);
#pragma unroll
    for (int q = 0; q < P::NV; ++q) tma_load<DIM>(st + P::box_off(q), &M.v[q], x0, y0, k, bar);
    tma_load<DIM>(st + P::OFF_CODE, &M.code, x0, y0, k, bar);
    if constexpr (P::XCB) tma_load<DIM>(st + P::OFF_XC, &M.xc, x0 / 2, y0 / 2, (k + 1) >> 1, bar);
}

// March bookkeeping: planes p0 .. plast pass through S stages; plane p uses stage
// (p - p0) % S for the ((p - p0) / S)-th time.  Thread 0 issues every load and is
// the only thread that waits on the stage barriers.
template <int DIM, int S, class P>
struct MRing {
    uint64_t* bars;
    unsigned char* base;
    int p0, plast;
    __device__ unsigned char* at(int p) const { return base + (size_t)((p - p0) % S) * P::STAGE; }
    __device__ bool wait(int p) const {
        const int u = p - p0;
        return mbar_wait(&bars[u % S], (uint32_t)((u / S) & 1), kTmaWaitLimit);
    }
    // thread 0: barriers and the first S planes
    __device__ void start(const MarchMaps& M) const {
        for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
        for (int p = p0; p < p0 + S && p <= plast; ++p) issue_plane<DIM, P>(M, at(p), &bars[(p - p0) % S], p);
    }
    // thread 0, after a block barrier: refill the stage of plane `freed`
    __device__ void refill(const MarchMaps& M, int freed) const {
        if (freed >= p0 && freed + S <= plast)
            issue_plane<DIM, P>(M, at(freed + S), &bars[(freed - p0) % S], freed + S);
    }
};

// Block-wide verdict on thread 0's waits; on a timeout the error word is set.
__device__ __forceinline__ bool step_barrier(bool ok, int* err) {
    if (__syncthreads_and(ok ? 1 : 0)) return true;
    if (threadIdx.x == 0 && threadIdx.y == 0) atomicExch(err, 1);
    return false;
}

// A x of one cell in FP32, as a sum of couplings times differences,
// sum_n c_n (x - x_n) (+ the Dirichlet wall share of the diagonal times x): the
// same value as d x - sum_n c_n x_n in exact arithmetic, but the differences of
// nearby values are exact in floating point, so smooth fields keep their relative
// accuracy instead of cancelling d x against the neighbour sum (an error of
// eps / (k h)^2, several per cent on the smoothest modes of a 2048 x 1024 grid).
// On the finest level a term exists where the code bit says the coupling does.
template <int DIM, class T, bool FINE>
__device__ __forceinline__ T fp32_ax(const MLevel<T>& L, uint32_t c, T d, const T (&cc)[6], T x,
                                     T xr, T xl, T xt, T xb, T xk, T xf) {
    if constexpr (FINE) {
        const T tx = ((c & 1u) ? x - xr : T(0)) + ((c & 2u) ? x - xl : T(0));
        const T ty = ((c & 4u) ? x - xt : T(0)) + ((c & 8u) ? x - xb : T(0));
        T ax = tx * L.idx2 + ty * L.idy2;
        T sum = ((c & 1u) ? L.idx2 : T(0)) + ((c & 2u) ? L.idx2 : T(0)) +
                ((c & 4u) ? L.idy2 : T(0)) + ((c & 8u) ? L.idy2 : T(0));
        if (DIM == 3) {
            const T tz = ((c & 16u) ? x - xk : T(0)) + ((c & 32u) ? x - xf : T(0));
            ax = ax + tz * L.idz2;
            sum = sum + ((c & 16u) ? L.idz2 : T(0)) + ((c & 32u) ? L.idz2 : T(0));
        }
        return ax + (d - sum) * x;  // d - sum: the Dirichlet wall share (0 with Neumann walls)
    } else {
        T ax = cc[0] * (x - xr) + cc[1] * (x - xl) + cc[2] * (x - xt) + cc[3] * (x - xb);
        T sum = cc[0] + cc[1] + cc[2] + cc[3];
        if (DIM == 3) {
            ax = ax + cc[4] * (x - xk) + cc[5] * (x - xf);
            sum = sum + cc[4] + cc[5];
        }
        return ax + (d - sum) * x;  // d - sum: the Galerkin wall channel (0 with Neumann walls)
    }
}

// Per-march ring depth and dynamic shared-memory size.  A 2D march reads one plane;
// in 3D the depths trade prefetch distance against blocks per SM (measured on the
// 256^3 benchmark: 6 / 5 stages on the finest level beat 8 / 6 and 5 / 4).
template <int DIM, class T, bool FINE, class CS = T> struct FwdCfg {
    using P = MPlan<DIM, T, false, !FINE, false, CS>;
    static constexpr int S = DIM == 2 ? 1 : FINE ? 6 : 4;
    using Lay = MLayout<T, S, P>;
    static constexpr size_t BYTES = Lay::OFF_EXTRA + 2 * align128(PBox<T>::BYTES);
};
template <int DIM, class T, bool FINE, class CS = T> struct ResCfg {
    using P = MPlan<DIM, T, true, !FINE, false, CS>;
    static constexpr int S = DIM == 2 ? 1 : FINE && sizeof(T) == 4 ? 5 : 4;
    using Lay = MLayout<T, S, P>;
    static constexpr size_t BYTES = Lay::OFF_EXTRA;
};
template <int DIM, class T, bool FINE, class CS = T> struct UpeCfg {
    using P = MPlan<DIM, T, false, !FINE, true, CS>;
    static constexpr int S = DIM == 2 ? 1 : FINE ? 6 : 4;
    using Lay = MLayout<T, S, P>;
    static constexpr size_t BYTES = Lay::OFF_EXTRA + 2 * align128(PBox<T>::BYTES);
};
template <int DIM, class T, bool FINE, class CS = T> struct UpoCfg {
    using P = MPlan<DIM, T, true, !FINE, false, CS>;
    static constexpr int S = DIM == 2 ? 1 : FINE && sizeof(T) == 4 ? 5 : 4;
    using Lay = MLayout<T, S, P>;
    static constexpr size_t BYTES = Lay::OFF_EXTRA;
};
// The search-direction march forms each plane's p into one of two plane buffers
// and frees the plane's stage at once, so 3 stages keep two planes in flight.
// MINB: six resident blocks (40 registers) in FP32; compiled for eight (32
// registers) it ran slower (256^3: 85.9 against 78.6 us a launch, 69.0 M warp
// instructions).
template <int DIM, class T> struct PmvCfg {
    using P = MPlan<DIM, T, true, false, false>;
    static constexpr int S = DIM == 2 ? 1 : 3;
    static constexpr int MINB = sizeof(T) == 4 ? 6 : 1;
    using Lay = MLayout<T, S, P>;
    static constexpr size_t BYTES = Lay::OFF_EXTRA + 2 * align128(PBox<T>::BYTES);
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

// The thread's pair: cells A = (i, j) and B = (i, j + 1), lane = column, warp w =
// tile rows 2w and 2w + 1.  A and B have opposite colours on every plane; the
// lanes of a warp read consecutive words of a box row.
struct Pair {
    int i, j, lane, w;
    int a, rb;         // box column and row of A (B: row rb + 1)
    int qa, ca;        // box positions of A in the value and code boxes
    bool ina, inb;     // inside the level
    int gid;           // cidx(g, i, j, 0)
};

template <class T>
__device__ __forceinline__ Pair own_pair(const Geom& g) {
    Pair o;
    const int t = threadIdx.x;
    o.lane = t & 31;
    o.w = t >> 5;
    o.i = 1 + kMX * (int)blockIdx.x + o.lane;
    o.j = 1 + kMY * (int)blockIdx.y + 2 * o.w;
    o.a = o.lane + 1;
    o.rb = 2 * o.w + 1;
    o.qa = o.rb * PBox<T>::W + o.a;
    o.ca = o.rb * PBox<uint8_t>::W + o.a;
    o.ina = o.i <= g.nx && o.j <= g.ny;
    o.inb = o.i <= g.nx && o.j + 1 <= g.ny;
    o.gid = o.i + o.j * g.sx;
    return o;
}

// Stage pointers of planes k-1, k, k+1, advanced once per step.
struct Stages {
    const unsigned char *m, *c, *n;
};

template <int DIM, int S, class P>
__device__ __forceinline__ Stages stages_at(const MRing<DIM, S, P>& R, int k) {
    Stages s;
    s.c = R.at(k);
    s.m = DIM == 3 && k > R.p0 ? R.at(k - 1) : s.c;
    s.n = DIM == 3 ? R.at(k + 1) : s.c;
    return s;
}

template <int DIM, int S, class P>
__device__ __forceinline__ void stages_next(const MRing<DIM, S, P>& R, Stages& s, int k) {
    s.m = s.c;
    s.c = s.n;
    s.n = R.at(k + 2);  // k: the step just finished
}

// ---------------------------------------------------------------------------
// Forward sweep from x = 0: x = (b + 0)/d on odd cells, then
// x = (b + sum c_n x_n)/d on even cells; writes x on every interior cell.
// Step k builds plane k+1's odd values (the pair's odd cell and the ring's odd
// cells) into a plane buffer and smooths plane k's even cells from plane k's
// buffer and the odd values of their own column one plane up and down (registers).
template <int DIM, class T, bool FINE, class CS>
__global__ void __launch_bounds__(kThreads) k_fwd_smooth(const __grid_constant__ MarchMaps M,
                                                         MLevel<T> L, T* __restrict__ x,
                                                         const int* __restrict__ done, int* err) {
    pdl_entry();
    if (done && *done) return;
    using C = FwdCfg<DIM, T, FINE, CS>;
    using P = typename C::P;
    using Lay = typename C::Lay;
    constexpr int S = C::S, N = PBox<T>::N, W = PBox<T>::W, WC = PBox<uint8_t>::W;
    UAAMG_MARCH_SMEM(sm, err)
    T* lut = reinterpret_cast<T*>(sm + Lay::OFF_LUT);
    T* Yb = reinterpret_cast<T*>(sm + Lay::OFF_EXTRA);
    const Geom& g = L.g;
    const int tid = threadIdx.x;
    const Pair o = own_pair<T>(g);
    const int ib = kMX * (int)blockIdx.x, jb = kMY * (int)blockIdx.y;  // box corner cell
    // the last warps also build the odd cells of the plane buffer's ring; their box
    // positions for a corner cell of either parity
    const bool hal = tid >= kThreads - kHaloOdd;
    int ha0 = 0, hr0 = 0, ha1 = 0, hr1 = 0;
    if (hal) {
        halo_odd(tid - (kThreads - kHaloOdd), 0, ha0, hr0);
        halo_odd(tid - (kThreads - kHaloOdd), 1, ha1, hr1);
    }
    int kb, ke;
    zrange<DIM>(g, L.zc, kb, ke);
    MRing<DIM, S, P> R{reinterpret_cast<uint64_t*>(sm), sm + Lay::OFF_RING,
                       DIM == 3 ? kb - 1 : 0, DIM == 3 ? ke : 0};
    if (FINE) build_lut<DIM, T>(lut, L.idx2, L.idy2, L.idz2);
    bool ok = true;
    if (tid == 0) {
        R.start(M);
        ok = R.wait(R.p0) && (DIM == 2 || R.wait(R.p0 + 1));
    }
    if (!step_barrier(ok, err)) return;
    // odd value of the pair at plane p (stage st), placed in its column (0: A, 1: B);
    // bo = 1 when B is the odd cell
    auto odd_pair = [&](const unsigned char* st, int p, int bo, T& ya, T& yb) -> T {
        const T v = presmooth<DIM, T, P, FINE, CS>(L, lut, st, o.a, o.rb + bo, o.i, o.j + bo, p);
        ya = bo ? T(0) : v;
        yb = bo ? v : T(0);
        return v;
    };
    Stages sg = stages_at<DIM, S, P>(R, R.p0);
    int par = (o.i + o.j + R.p0) & 1;  // 1: A is odd at plane k
    T yma = T(0), ymb = T(0), y0a = T(0), y0b = T(0), ypa = T(0), ypb = T(0);
    if (DIM == 3) odd_pair(sg.c, R.p0, par ^ 1, y0a, y0b);
#pragma unroll 1
    for (int k = R.p0; k < ke; ++k) {
        const int kn = DIM == 3 ? k + 1 : 0;  // plane whose odd values are built this step
        const int pn = DIM == 3 ? par ^ 1 : par;
        {
            T* Yn = Yb + (kn & 1) * N;
            const T v = odd_pair(sg.n, kn, pn ^ 1, ypa, ypb);
            Yn[o.qa + (pn ? 0 : W)] = v;
            if (hal) {
                const int s0 = (ib + jb + kn) & 1, a = s0 ? ha1 : ha0, r = s0 ? hr1 : hr0;
                Yn[r * W + a] = presmooth<DIM, T, P, FINE, CS>(L, lut, sg.n, a, r, ib + a, jb + r, kn);
            }
        }
        if (DIM == 2) {
            y0a = ypa;
            y0b = ypb;
            __syncthreads();
        }
        if (k >= kb) {
            const T* Yc = Yb + (k & 1) * N;
            const int e = par;  // 1: B is the even cell
            const int q = o.qa + (e ? W : 0);
            const uint32_t c = sg.c[P::OFF_CODE + o.ca + (e ? WC : 0)];
            T xe = T(0);
            if (c & kActive) {
                const T d = mdiag<DIM, T, P, FINE>(L, lut, sg.c, c, q, o.i, o.j + e, k);
                if (!(d < T(1e-30))) {
                    T cc[6];
                    mcoup<DIM, T, P, FINE, CS>(L, sg.c, sg.m, o.a, o.rb + e, cc);
                    xe = mdiv<T, CS>(boxv<T>(sg.c, P::QB * P::VB, q) +
                                         nbsum<DIM, T>(cc, Yc, q, e ? ypb : ypa, e ? ymb : yma), d);
                }
            }
            const int base = o.gid + k * g.sxy;
            if (o.ina) x[base] = e ? y0a : xe;
            if (o.inb) x[base + g.sx] = e ? xe : y0b;
        }
        if (DIM == 2) break;
        yma = y0a; ymb = y0b;
        y0a = ypa; y0b = ypb;
        par ^= 1;
        if (tid == 0 && k + 2 <= R.plast) ok = R.wait(k + 2);
        if (!step_barrier(ok, err)) return;
        if (tid == 0) R.refill(M, k - 1);
        stages_next<DIM, S, P>(R, sg, k);
    }
}

// Residual r = b - A x of every fluid cell and its restriction
// b_c = sum over the 2x2(x2) children in the reference's (di, dj, dk) order.  A
// thread's pair is the dj = 0, 1 children of one coarse column, the di = 1 children
// are the next lane's pair, dk = 0, 1 are consecutive planes.
template <int DIM, class T, bool FINE, class CS>
__global__ void __launch_bounds__(kThreads) k_restrict_res(const __grid_constant__ MarchMaps M,
                                                           MLevel<T> L,
                                                           const uint8_t* __restrict__ ccode,
                                                           T* __restrict__ cb,
                                                           const int* __restrict__ done, int* err) {
    pdl_entry();
    if (done && *done) return;
    using C = ResCfg<DIM, T, FINE, CS>;
    using P = typename C::P;
    using Lay = typename C::Lay;
    constexpr int S = C::S, W = PBox<T>::W, WC = PBox<uint8_t>::W;
    UAAMG_MARCH_SMEM(sm, err)
    T* lut = reinterpret_cast<T*>(sm + Lay::OFF_LUT);
    const Geom& g = L.g;
    const int tid = threadIdx.x;
    const Pair o = own_pair<T>(g);
    int kb, ke;
    zrange<DIM>(g, L.zc, kb, ke);
    MRing<DIM, S, P> R{reinterpret_cast<uint64_t*>(sm), sm + Lay::OFF_RING,
                       DIM == 3 ? kb - 1 : 0, DIM == 3 ? ke : 0};
    if (FINE) build_lut<DIM, T>(lut, L.idx2, L.idy2, L.idz2);
    bool ok = true;
    if (tid == 0) {
        R.start(M);
        ok = R.wait(R.p0) && (DIM == 2 || (R.wait(kb) && R.wait(kb + 1)));
    }
    if (!step_barrier(ok, err)) return;
    const int ic = kMX / 2 * (int)blockIdx.x + 1 + (o.lane >> 1);
    const int jc = kMY / 2 * (int)blockIdx.y + 1 + o.w;
    const bool writer = (o.lane & 1) == 0 && ic <= L.cg.nx && jc <= L.cg.ny;
    Stages sg = stages_at<DIM, S, P>(R, kb);
    T rlo[2] = {T(0), T(0)};
#pragma unroll 1
    for (int k = kb; k < ke; ++k) {
        const T* xb = reinterpret_cast<const T*>(sg.c + P::QX * P::VB);
        T rv[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int q = o.qa + e * W;
            const uint32_t c = sg.c[P::OFF_CODE + o.ca + e * WC];
            rv[e] = T(0);
            if (c & kActive) {
                const T d = mdiag<DIM, T, P, FINE>(L, lut, sg.c, c, q, o.i, o.j + e, k);
                T cc[6];
                mcoup<DIM, T, P, FINE, CS>(L, sg.c, sg.m, o.a, o.rb + e, cc);
                const T xp = DIM == 3 ? boxv<T>(sg.n, P::QX * P::VB, q) : T(0);
                const T xm = DIM == 3 ? boxv<T>(sg.m, P::QX * P::VB, q) : T(0);
                T ax;
                if constexpr (sizeof(T) == 8) {  // the reference's expression (bit-exact)
                    ax = d * xb[q] - cc[0] * xb[q + 1] - cc[1] * xb[q - 1] - cc[2] * xb[q + W] -
                         cc[3] * xb[q - W];
                    if (DIM == 3) ax = ax - cc[4] * xp - cc[5] * xm;
                } else {
                    ax = fp32_ax<DIM, T, FINE>(L, c, d, cc, xb[q], xb[q + 1], xb[q - 1], xb[q + W],
                                               xb[q - W], xp, xm);
                }
                rv[e] = boxv<T>(sg.c, P::QB * P::VB, q) - ax;
            }
        }
        // children with dk = 0 live on odd planes (k = 2 kc - 1); the set is complete
        // on the even plane that follows
        if (DIM == 3 && (k & 1)) {
            rlo[0] = rv[0];
            rlo[1] = rv[1];
        } else {
            T pr[2][2];  // the di = 1 partner's values [dj][dk]
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                pr[e][0] = __shfl_down_sync(0xffffffffu, DIM == 3 ? rlo[e] : rv[e], 1);
                pr[e][1] = __shfl_down_sync(0xffffffffu, rv[e], 1);
            }
            if (writer) {
                const int kc = DIM == 3 ? k / 2 : 0;
                const int cid = cidx(L.cg, ic, jc, kc);
                T s = T(0);
                if (DIM == 3) {
                    s += rlo[0]; s += rv[0]; s += rlo[1]; s += rv[1];
                    s += pr[0][0]; s += pr[0][1]; s += pr[1][0]; s += pr[1][1];
                } else {
                    s += rv[0]; s += rv[1];
                    s += pr[0][1]; s += pr[1][1];
                }
                cb[cid] = (ccode[cid] & kActive) ? s : T(0);
            }
        }
        if (DIM == 2) break;
        if (tid == 0 && k + 2 <= R.plast) ok = R.wait(k + 2);
        if (!step_barrier(ok, err)) return;
        if (tid == 0) R.refill(M, k - 1);
        stages_next<DIM, S, P>(R, sg, k);
    }
}

// Prolongation and the first (even) colour of the reverse sweep.  Odd cells hold
// their pre-smoothed value plus the prolongation, (b + 0)/d + 2 x_c; even cells are
// smoothed from those: x = (b + sum c_n x_n)/d (a skipped even cell keeps
// 0 + 2 x_c).  Writes x on every interior cell.
template <int DIM, class T, bool FINE, class CS>
__global__ void __launch_bounds__(kThreads) k_up_even(const __grid_constant__ MarchMaps M,
                                                      MLevel<T> L, T* __restrict__ x,
                                                      const int* __restrict__ done, int* err) {
    pdl_entry();
    if (done && *done) return;
    using C = UpeCfg<DIM, T, FINE, CS>;
    using P = typename C::P;
    using Lay = typename C::Lay;
    constexpr int S = C::S, N = PBox<T>::N, W = PBox<T>::W, WC = PBox<uint8_t>::W;
    UAAMG_MARCH_SMEM(sm, err)
    T* lut = reinterpret_cast<T*>(sm + Lay::OFF_LUT);
    T* Yb = reinterpret_cast<T*>(sm + Lay::OFF_EXTRA);
    const Geom& g = L.g;
    const int tid = threadIdx.x;
    const Pair o = own_pair<T>(g);
    const int ib = kMX * (int)blockIdx.x, jb = kMY * (int)blockIdx.y;
    const bool hal = tid >= kThreads - kHaloOdd;
    int ha0 = 0, hr0 = 0, ha1 = 0, hr1 = 0;
    if (hal) {
        halo_odd(tid - (kThreads - kHaloOdd), 0, ha0, hr0);
        halo_odd(tid - (kThreads - kHaloOdd), 1, ha1, hr1);
    }
    // odd cell at box position (a, r): pre-smoothed value + prolongation (0 if not
    // an active odd cell)
    auto oddval = [&](const unsigned char* st, int a, int r, int ci, int cj, int ck) -> T {
        const uint32_t c = st[P::OFF_CODE + r * WC + a];
        if ((c & (kActive | kOdd)) != (kActive | kOdd)) return T(0);
        const int qq = r * W + a;
        const T d = mdiag<DIM, T, P, FINE>(L, lut, st, c, qq, ci, cj, ck);
        const T pre = d < T(1e-30) ? T(0) : mdiv<T, CS>(boxv<T>(st, P::QB * P::VB, qq) + T(0), d);
        return pre + prolong_at<T, P>(st, a, r);
    };
    int kb, ke;
    zrange<DIM>(g, L.zc, kb, ke);
    MRing<DIM, S, P> R{reinterpret_cast<uint64_t*>(sm), sm + Lay::OFF_RING,
                       DIM == 3 ? kb - 1 : 0, DIM == 3 ? ke : 0};
    if (FINE) build_lut<DIM, T>(lut, L.idx2, L.idy2, L.idz2);
    bool ok = true;
    if (tid == 0) {
        R.start(M);
        ok = R.wait(R.p0) && (DIM == 2 || R.wait(R.p0 + 1));
    }
    if (!step_barrier(ok, err)) return;
    auto odd_pair = [&](const unsigned char* st, int p, int bo, T& ya, T& yb) -> T {
        const T v = oddval(st, o.a, o.rb + bo, o.i, o.j + bo, p);
        ya = bo ? T(0) : v;
        yb = bo ? v : T(0);
        return v;
    };
    Stages sg = stages_at<DIM, S, P>(R, R.p0);
    int par = (o.i + o.j + R.p0) & 1;
    T yma = T(0), ymb = T(0), y0a = T(0), y0b = T(0), ypa = T(0), ypb = T(0);
    if (DIM == 3) odd_pair(sg.c, R.p0, par ^ 1, y0a, y0b);
#pragma unroll 1
    for (int k = R.p0; k < ke; ++k) {
        const int kn = DIM == 3 ? k + 1 : 0;
        const int pn = DIM == 3 ? par ^ 1 : par;
        {
            T* Yn = Yb + (kn & 1) * N;
            const T v = odd_pair(sg.n, kn, pn ^ 1, ypa, ypb);
            Yn[o.qa + (pn ? 0 : W)] = v;
            if (hal) {
                const int s0 = (ib + jb + kn) & 1, a = s0 ? ha1 : ha0, r = s0 ? hr1 : hr0;
                Yn[r * W + a] = oddval(sg.n, a, r, ib + a, jb + r, kn);
            }
        }
        if (DIM == 2) {
            y0a = ypa;
            y0b = ypb;
            __syncthreads();
        }
        if (k >= kb) {
            const T* Yc = Yb + (k & 1) * N;
            const int e = par;
            const int q = o.qa + (e ? W : 0);
            const uint32_t c = sg.c[P::OFF_CODE + o.ca + (e ? WC : 0)];
            T xe = T(0);
            if (c & kActive) {
                const T d = mdiag<DIM, T, P, FINE>(L, lut, sg.c, c, q, o.i, o.j + e, k);
                if (d < T(1e-30)) {
                    // a skipped even cell keeps its pre-smoothed 0 plus the prolongation
                    xe = T(0) + prolong_at<T, P>(sg.c, o.a, o.rb + e);
                } else {
                    T cc[6];
                    mcoup<DIM, T, P, FINE, CS>(L, sg.c, sg.m, o.a, o.rb + e, cc);
                    xe = mdiv<T, CS>(boxv<T>(sg.c, P::QB * P::VB, q) +
                                         nbsum<DIM, T>(cc, Yc, q, e ? ypb : ypa, e ? ymb : yma), d);
                }
            }
            const int base = o.gid + k * g.sxy;
            if (o.ina) x[base] = e ? y0a : xe;
            if (o.inb) x[base + g.sx] = e ? xe : y0b;
        }
        if (DIM == 2) break;
        yma = y0a; ymb = y0b;
        y0a = ypa; y0b = ypb;
        par ^= 1;
        if (tid == 0 && k + 2 <= R.plast) ok = R.wait(k + 2);
        if (!step_barrier(ok, err)) return;
        if (tid == 0) R.refill(M, k - 1);
        stages_next<DIM, S, P>(R, sg, k);
    }
}

// Second (odd) colour of the reverse sweep, in place: odd cells read only even
// neighbours, which this kernel does not write.  ZDOT (finest level): also the
// fluid sums of z, r*z and r (r = this level's b) and the CG's projection / beta.
template <int DIM, class T, bool FINE, bool ZDOT, class CS>
__global__ void __launch_bounds__(kThreads) k_up_odd(const __grid_constant__ MarchMaps M,
                                                     MLevel<T> L, T* x,
                                                     const int* __restrict__ done, int* err,
                                                     double* partials, CGState* cg) {
    pdl_entry();
    if (done && *done) return;
    using C = UpoCfg<DIM, T, FINE, CS>;
    using P = typename C::P;
    using Lay = typename C::Lay;
    constexpr int S = C::S, W = PBox<T>::W, WC = PBox<uint8_t>::W;
    UAAMG_MARCH_SMEM(sm, err)
    T* lut = reinterpret_cast<T*>(sm + Lay::OFF_LUT);
    const Geom& g = L.g;
    const int tid = threadIdx.x;
    const Pair o = own_pair<T>(g);
    double acc[3] = {0.0, 0.0, 0.0};
    int kb, ke;
    zrange<DIM>(g, L.zc, kb, ke);
    MRing<DIM, S, P> R{reinterpret_cast<uint64_t*>(sm), sm + Lay::OFF_RING,
                       DIM == 3 ? kb - 1 : 0, DIM == 3 ? ke : 0};
    if (FINE) build_lut<DIM, T>(lut, L.idx2, L.idy2, L.idz2);
    bool ok = true;
    if (tid == 0) {
        R.start(M);
        ok = R.wait(R.p0) && (DIM == 2 || (R.wait(kb) && R.wait(kb + 1)));
    }
    if (!step_barrier(ok, err)) return;
    Stages sg = stages_at<DIM, S, P>(R, kb);
    int par = (o.i + o.j + kb) & 1;  // 1: A is odd
#pragma unroll 1
    for (int k = kb; k < ke; ++k) {
        const T* xb = reinterpret_cast<const T*>(sg.c + P::QX * P::VB);
        const int od = par ^ 1;  // 1: B is the odd cell
        T za = xb[o.qa], zb = xb[o.qa + W];
        const uint32_t ca = sg.c[P::OFF_CODE + o.ca], cbb = sg.c[P::OFF_CODE + o.ca + WC];
        {
            const int q = o.qa + (od ? W : 0);
            const uint32_t c = od ? cbb : ca;
            if (c & kActive) {
                const T d = mdiag<DIM, T, P, FINE>(L, lut, sg.c, c, q, o.i, o.j + od, k);
                if (!(d < T(1e-30))) {
                    T cc[6];
                    mcoup<DIM, T, P, FINE, CS>(L, sg.c, sg.m, o.a, o.rb + od, cc);
                    const T vp = DIM == 3 ? boxv<T>(sg.n, P::QX * P::VB, q) : T(0);
                    const T vm = DIM == 3 ? boxv<T>(sg.m, P::QX * P::VB, q) : T(0);
                    const T xv = mdiv<T, CS>(boxv<T>(sg.c, P::QB * P::VB, q) + nbsum<DIM, T>(cc, xb, q, vp, vm), d);
                    if (od) zb = xv; else za = xv;
                    if (od ? o.inb : o.ina) x[o.gid + k * g.sxy + (od ? g.sx : 0)] = xv;
                }
            }
        }
        if (ZDOT) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const uint32_t c = e ? cbb : ca;
                if ((c & kActive) && (e ? o.inb : o.ina)) {
                    const double zv = (double)(e ? zb : za);
                    const double rv = (double)boxv<T>(sg.c, P::QB * P::VB, o.qa + e * W);
                    acc[0] += zv;
                    acc[1] += rv * zv;
                    acc[2] += rv;
                }
            }
        }
        if (DIM == 2) break;
        par ^= 1;
        if (tid == 0 && k + 2 <= R.plast) ok = R.wait(k + 2);
        if (!step_barrier(ok, err)) return;
        if (tid == 0) R.refill(M, k - 1);
        stages_next<DIM, S, P>(R, sg, k);
    }
    if (ZDOT) {
        double tot[3];
        if (reduce_last<3>(acc, partials, &cg->counter[2], tot)) finish_zdot(cg, tot);
    }
}

// The t-th cell of a plane box's 1-cell ring (t < 100) as box column a and row r:
// rows 0 and 17 (34 cells each), then columns 0 and 33 of rows 1-16.
__device__ __forceinline__ bool ring_cell(int t, int& a, int& r) {
    constexpr int kRow = kMX + 2;
    if (t >= 2 * kRow + 2 * kMY) return false;
    if (t < 2 * kRow) {
        a = t % kRow;
        r = t < kRow ? 0 : kMY + 1;
    } else {
        const int u = t - 2 * kRow;
        a = u < kMY ? 0 : kMX + 1;
        r = 1 + u % kMY;
    }
    return true;
}

// CG search direction fused with the operator: p = (z - m) + beta p_old on fluid
// cells (pcg_3d.cpp:113-122) and Ap from the new p of the neighbours (a solid or
// out-of-domain neighbour reads p_C -- Neumann -- or -p_C at a Dirichlet wall;
// pcg_3d.cpp:38-55); p.Ap is reduced and the last block sets alpha = rz_old / p.Ap
// or stops on breakdown (pcg_3d.cpp:94-99).  p_old and p_new are distinct buffers.
// DIRW: the problem has Dirichlet walls (with Neumann walls a missing neighbour
// always reads p_C, so the wall tests drop out; the selected values are the same).
//
// Each plane's p is formed once, into a shared plane buffer (two, alternating):
// step k forms plane k+1 (every thread its own pair and the pair's codes, threads
// 0-99 the 1-cell ring) while it applies the stencil on plane k, whose p the
// previous step formed; the step barrier hands the new plane to the in-plane
// neighbours.  The pair's own column at k-1, k, k+1 stays in registers, so the z
// neighbours need no shared-memory read, and a plane's ring stage is free as soon
// as its p is formed: three stages keep two planes in flight.
template <int DIM, class T, bool DIRW = true>
__global__ void __launch_bounds__(kThreads, DIRW ? 1 : PmvCfg<DIM, T>::MINB)
    k_pmatvec(const __grid_constant__ MarchMaps M, Geom g, int zc, T* __restrict__ pnew,
              T* __restrict__ ap, Stencil st, double* partials, CGState* cg, int* err) {
    pdl_entry();
    if (cg->done) return;
    using C = PmvCfg<DIM, T>;
    using P = typename C::P;
    using Lay = typename C::Lay;
    constexpr int S = C::S, W = PBox<T>::W, WC = PBox<uint8_t>::W;
    UAAMG_MARCH_SMEM(sm, err)
    T* pbuf0 = reinterpret_cast<T*>(sm + Lay::OFF_EXTRA);
    T* pbuf1 = reinterpret_cast<T*>(sm + Lay::OFF_EXTRA + align128(PBox<T>::BYTES));
    const int tid = threadIdx.x;
    const Pair o = own_pair<T>(g);
    const T m = (T)cg->mean_z, beta = (T)cg->beta;
    const T idx2 = (T)st.idx2, idy2 = (T)st.idy2, idz2 = (T)st.idz2, diag = (T)st.diag;
    double acc[1] = {0.0};
    int kb, ke;
    zrange<DIM>(g, zc, kb, ke);
    MRing<DIM, S, P> R{reinterpret_cast<uint64_t*>(sm), sm + Lay::OFF_RING,
                       DIM == 3 ? kb - 1 : 0, DIM == 3 ? ke : 0};
    bool ok = true;
    if (tid == 0) {
        R.start(M);
        ok = R.wait(R.p0) && (DIM == 2 || (R.wait(kb) && R.wait(kb + 1)));
    }
    if (!step_barrier(ok, err)) return;
    int rq = -1, ra, rr;
    if (ring_cell(tid, ra, rr)) rq = rr * W + ra;
    auto pv = [&](const unsigned char* s_, int qq) -> T {
        return (boxv<T>(s_, P::QB * P::VB, qq) - m) + beta * boxv<T>(s_, P::QX * P::VB, qq);
    };
    // p of the staged plane s_ into the buffer pb: the pair's cells (also returned,
    // with their codes, B's in bits 8-15) and this thread's ring cell
    auto form = [&](const unsigned char* s_, T* pb, T (&out)[2], uint32_t& code) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            out[e] = pv(s_, o.qa + e * W);
            pb[o.qa + e * W] = out[e];
        }
        code = (uint32_t)s_[P::OFF_CODE + o.ca] | ((uint32_t)s_[P::OFF_CODE + o.ca + WC] << 8);
        if (rq >= 0) pb[rq] = pv(s_, rq);
    };
    T pm[2] = {T(0), T(0)}, pc[2], pn[2] = {T(0), T(0)};
    uint32_t cc, cn = 0u;
    if (DIM == 3) {
#pragma unroll
        for (int e = 0; e < 2; ++e) pm[e] = pv(R.at(kb - 1), o.qa + e * W);
    }
    form(R.at(kb), pbuf0, pc, cc);
    __syncthreads();
    if (DIM == 3 && tid == 0) {
        R.refill(M, kb - 1);
        R.refill(M, kb);
    }
    T* pbc = pbuf0;
    T* pbn = pbuf1;
#pragma unroll 1
    for (int k = kb; k < ke; ++k) {
        if (DIM == 3) form(R.at(k + 1), pbn, pn, cn);
        T a_[2] = {T(0), T(0)};
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const uint32_t c = (cc >> (8 * e)) & 0xffu;
            if (c & kActive) {
                const int q = o.qa + e * W, i = o.i, j = o.j + e;
                const T p0 = pc[e];
                const T wall = DIRW && st.dirichlet ? -p0 : p0;
                const T vL = (c & 2u) ? pbc[q - 1] : (!DIRW || i > 1 ? p0 : wall);
                const T vR = (c & 1u) ? pbc[q + 1] : (!DIRW || i < g.nx ? p0 : wall);
                // the pair's other cell is the +y (A) or -y (B) neighbour
                const T vB = (c & 8u) ? (e ? pc[0] : pbc[q - W]) : (!DIRW || j > 1 ? p0 : wall);
                const T vT = (c & 4u) ? (e ? pbc[q + W] : pc[1]) : (!DIRW || j < g.ny ? p0 : wall);
                if (DIM == 3) {
                    const T vF = (c & 32u) ? pm[e] : (!DIRW || k > 1 ? p0 : wall);
                    const T vK = (c & 16u) ? pn[e] : (!DIRW || k < g.nz ? p0 : wall);
                    a_[e] = sizeof(T) == 8
                                ? diag * p0 - (vL + vR) * idx2 - (vB + vT) * idy2 - (vF + vK) * idz2
                                : ((p0 - vL) + (p0 - vR)) * idx2 + ((p0 - vB) + (p0 - vT)) * idy2 +
                                      ((p0 - vF) + (p0 - vK)) * idz2;
                } else {
                    a_[e] = sizeof(T) == 8 ? diag * p0 - (vL + vR) * idx2 - (vB + vT) * idy2
                                           : ((p0 - vL) + (p0 - vR)) * idx2 + ((p0 - vB) + (p0 - vT)) * idy2;
                }
                acc[0] += (double)p0 * (double)a_[e];
            }
        }
        const int id = o.gid + k * g.sxy;
        if (o.ina) { pnew[id] = (cc & kActive) ? pc[0] : T(0); ap[id] = a_[0]; }
        if (o.inb) { pnew[id + g.sx] = (cc & (kActive << 8)) ? pc[1] : T(0); ap[id + g.sx] = a_[1]; }
        if (DIM == 2) break;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            pm[e] = pc[e];
            pc[e] = pn[e];
        }
        cc = cn;
        T* t = pbc;
        pbc = pbn;
        pbn = t;
        if (tid == 0 && k + 2 <= R.plast) ok = R.wait(k + 2);
        if (!step_barrier(ok, err)) return;
        if (tid == 0) R.refill(M, k + 1);
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

// ---------------------------------------------------------------------------
// FP64 residual replacement of the mixed 3D solve as a z march: r = b - A x with
// x = x_hi + x_lo (pcg_3d.cpp:38-55 operator, the arithmetic of k_resid_x64), r
// written as T (0 on solid cells), r.r reduced; the last block asks the next x
// update to fold x_lo into x_hi and runs the convergence test.  Each plane of b,
// x_hi (FP64), x_lo (T) and the codes arrives as one TMA box per array; step k
// forms x of plane k+1 once into one of two FP64 plane buffers (pairs and ring,
// as in k_pmatvec), keeps the pair's own x at k-1, k, k+1 and b at k, k+1 in
// registers, and applies the operator on plane k.
template <class T>
struct RPlan {
    static constexpr int NV = 3;  // b, x_hi (FP64), x_lo (T)
    static constexpr size_t DB = align128(PBox<double>::BYTES);
    static constexpr size_t OFF_XH = DB, OFF_XL = 2 * DB;
    static constexpr size_t OFF_CODE = OFF_XL + align128(PBox<T>::BYTES);
    static constexpr size_t STAGE = OFF_CODE + align128(PBox<uint8_t>::BYTES);
    static constexpr bool XCB = false;
    static constexpr uint32_t TX_BYTES =
        2 * PBox<double>::BYTES + PBox<T>::BYTES + PBox<uint8_t>::BYTES;
    __host__ __device__ static constexpr size_t box_off(int q) {
        return q == 0 ? 0 : q == 1 ? OFF_XH : OFF_XL;
    }
};
template <class T> struct RxCfg {
    using P = RPlan<T>;
    static constexpr int S = 3;
    using Lay = MLayout<double, S, P>;
    static constexpr size_t BYTES = Lay::OFF_EXTRA + 2 * align128(PBox<double>::BYTES);
};

template <class T, bool DIRW = true>
__global__ void __launch_bounds__(kThreads) k_resid_march(const __grid_constant__ MarchMaps M, Geom g,
                                                          int zc, T* __restrict__ rw, Stencil st,
                                                          double* partials, CGState* cg, int slot,
                                                          double tol, int tol_mode, int* err) {
    pdl_entry();
    if (!replacement_due(cg)) return;
    using C = RxCfg<T>;
    using P = typename C::P;
    using Lay = typename C::Lay;
    constexpr int S = C::S, WD = PBox<double>::W, WT = PBox<T>::W, WC = PBox<uint8_t>::W;
    UAAMG_MARCH_SMEM(sm, err)
    double* xbuf0 = reinterpret_cast<double*>(sm + Lay::OFF_EXTRA);
    double* xbuf1 = reinterpret_cast<double*>(sm + Lay::OFF_EXTRA + align128(PBox<double>::BYTES));
    const int tid = threadIdx.x;
    const Pair o = own_pair<T>(g);
    const int qd = o.rb * WD + o.a, qt = o.rb * WT + o.a;  // A in the FP64 and T boxes
    const double idx2 = st.idx2, idy2 = st.idy2, idz2 = st.idz2, diag = st.diag;
    double acc[1] = {0.0};
    int kb, ke;
    zrange<3>(g, zc, kb, ke);
    MRing<3, S, P> R{reinterpret_cast<uint64_t*>(sm), sm + Lay::OFF_RING, kb - 1, ke};
    bool ok = true;
    if (tid == 0) {
        R.start(M);
        ok = R.wait(R.p0) && R.wait(kb) && R.wait(kb + 1);
    }
    if (!step_barrier(ok, err)) return;
    int rqd = -1, rqt = 0, ra, rr;
    if (ring_cell(tid, ra, rr)) {
        rqd = rr * WD + ra;
        rqt = rr * WT + ra;
    }
    auto X = [&](const unsigned char* s_, int q_d, int q_t) -> double {
        return boxv<double>(s_, P::OFF_XH, q_d) + (double)boxv<T>(s_, P::OFF_XL, q_t);
    };
    // x of the staged plane s_ into the buffer xb (the pair's cells also returned,
    // with b and the codes, B's in bits 8-15) and this thread's ring cell
    auto form = [&](const unsigned char* s_, double* xb, double (&xo)[2], double (&bo)[2],
                    uint32_t& code) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            xo[e] = X(s_, qd + e * WD, qt + e * WT);
            xb[qd + e * WD] = xo[e];
            bo[e] = boxv<double>(s_, 0, qd + e * WD);
        }
        code = (uint32_t)s_[P::OFF_CODE + o.ca] | ((uint32_t)s_[P::OFF_CODE + o.ca + WC] << 8);
        if (rqd >= 0) xb[rqd] = X(s_, rqd, rqt);
    };
    double xm[2], xc[2], xn[2] = {0.0, 0.0}, bc[2], bn[2] = {0.0, 0.0};
    uint32_t cc, cn = 0u;
    {
        const unsigned char* s0 = R.at(kb - 1);
#pragma unroll
        for (int e = 0; e < 2; ++e) xm[e] = X(s0, qd + e * WD, qt + e * WT);
    }
    form(R.at(kb), xbuf0, xc, bc, cc);
    __syncthreads();
    if (tid == 0) {
        R.refill(M, kb - 1);
        R.refill(M, kb);
    }
    double* xbc = xbuf0;
    double* xbn = xbuf1;
#pragma unroll 1
    for (int k = kb; k < ke; ++k) {
        form(R.at(k + 1), xbn, xn, bn, cn);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const uint32_t c = (cc >> (8 * e)) & 0xffu;
            const int q = qd + e * WD, i = o.i, j = o.j + e;
            const double x0 = xc[e];
            const double wall = DIRW && st.dirichlet ? -x0 : x0;
            const double vL = (c & 2u) ? xbc[q - 1] : (!DIRW || i > 1 ? x0 : wall);
            const double vR = (c & 1u) ? xbc[q + 1] : (!DIRW || i < g.nx ? x0 : wall);
            // the pair's other cell is the +y (A) or -y (B) neighbour
            const double vB = (c & 8u) ? (e ? xc[0] : xbc[q - WD]) : (!DIRW || j > 1 ? x0 : wall);
            const double vT = (c & 4u) ? (e ? xbc[q + WD] : xc[1]) : (!DIRW || j < g.ny ? x0 : wall);
            const double vF = (c & 32u) ? xm[e] : (!DIRW || k > 1 ? x0 : wall);
            const double vK = (c & 16u) ? xn[e] : (!DIRW || k < g.nz ? x0 : wall);
            const double ax = diag * x0 - (vL + vR) * idx2 - (vB + vT) * idy2 - (vF + vK) * idz2;
            const double r = (c & kActive) ? bc[e] - ax : 0.0;
            if (e ? o.inb : o.ina) {
                acc[0] += r * r;
                rw[o.gid + k * g.sxy + (e ? g.sx : 0)] = (T)r;
            }
        }
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            xm[e] = xc[e];
            xc[e] = xn[e];
            bc[e] = bn[e];
        }
        cc = cn;
        double* t = xbc;
        xbc = xbn;
        xbn = t;
        if (tid == 0 && k + 2 <= R.plast) ok = R.wait(k + 2);
        if (!step_barrier(ok, err)) return;
        if (tid == 0) R.refill(M, k + 1);
    }
    double tot[1];
    if (reduce_last<1>(acc, partials, &cg->counter[slot], tot)) {
        cg->fold = 1;
        true_residual_done(cg, tot[0], 1, tol, tol_mode);
        // a replacement at max_iter that did not confirm convergence ends the solve
        if (!cg->done && cg->iter >= cg->max_iter) {
            cg->status = CG_MAXITER;
            cg->done = 1;
        }
    }
}

#undef UAAMG_MARCH_SMEM

}  // namespace
}  // namespace uaamg
