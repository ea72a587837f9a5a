// Fused V-cycle level kernels: ONE z march for the way down through a level and
// ONE for the way up (uaamg_preconditioner_3d.cpp:183-196; 2D
// uaamg_preconditioner.cpp:162-175), instead of the four marches of march.cuh.
//
//   k_level_down  forward red-black sweep from x = 0 (smooth(L,1,false),
//                 _3d.cpp:123-141), the residual b - A x (restrictResidual,
//                 144-165) and its restriction to the coarse b.  The smoothed x
//                 is never stored: odd cells hold b/d and even cells a function of
//                 the b of their neighbours, so the block recomputes x on its tile
//                 and a 2-cell ring from the staged b, and writes only the coarse b.
//   k_level_up    prolongation x += 2 x_coarse (prolongateAdd, 168-181) and the
//                 reverse sweep (even colour, then odd), writing the final x; on
//                 the finest level also the CG's z sums (pcg_3d.cpp:112-123).
//
// Block: a 32 x 16 column tile (256 threads, each owning the cell pair (i, j),
// (i, j+1) -- one cell of each colour), marching a chunk of z planes.  Every plane
// of b, the cell codes (coarse levels: diagonal and couplings; way up: the parent
// x) arrives by TMA as a box of the tile plus a 2-cell ring, into a ring of
// shared-memory stages.  Step s of the march computes three things:
//   1. the odd-colour value of plane s+1 (tile and 2-cell ring),
//   2. the even-colour value of plane s (tile and 1-cell ring), from the odd
//      values of plane s in shared memory and plane s +- 1 in registers,
//   3. the final result of plane s-1 on the tile (way down: residual and
//      restriction; way up: the odd colour of the reverse sweep and the store).
// A z neighbour is the same column one step up or down, so each thread keeps its
// column's recent values in registers; in-plane neighbours are read from three
// shared x planes written one step earlier, so one block barrier per step
// suffices.  The first 104 threads also own a pair of ring cells (50 pairs of
// the 1-cell ring, 54 of the 2-cell ring).
//
// Arithmetic: every per-cell value is the reference's expression in its order
// (the forward even update (b + sum c_n x_n)/d, the residual b - (d x - sum c_n
// x_n), the restriction's child order), so the FP64 instantiation (built with
// -fmad=false) reproduces the reference's V-cycle bit for bit.  The FP32 forms
// take the residual of the forward sweep from its exact form: an even cell was
// just relaxed, so its residual is 0, and an odd cell's is sum_n c_n x_n over its
// (even) neighbours, since d x = b there; cells with d < 1e-30 (skipped by the
// smoother) keep r = b.
#pragma once
#include "march.cuh"

namespace uaamg {
namespace {

// Box of element type E around a tile with a 2-cell ring: cells
// i in [i0-2, i0+33], j in [j0-2, j0+17] (i0 = 1 + 32 bx, j0 = 1 + 16 by) of one
// plane.  The start column 32 bx - A is the 16-byte boundary at or below i0 - 2.
template <class E>
struct RBox {
    static constexpr int A = 16 / (int)sizeof(E);          // elements per 16 bytes
    static constexpr int W = (A + 35 + A - 1) / A * A;      // row width (elements)
    static constexpr int H = kMY + 4;
    static constexpr uint32_t BYTES = (uint32_t)(W * H * sizeof(E));
    // position of the cell (i0 + di, j0 + dj), di in [-2, 33], dj in [-2, 17]
    __host__ __device__ static constexpr int pos(int di, int dj) { return (dj + 2) * W + A + 1 + di; }
};

// Tensor maps of a fused march (boxes of RBox geometry; xc: the parent level's x
// in QBox geometry).
struct FMaps {
    CUtensorMap b, code, dg, cx, cy, cz, xc;
};

// One ring stage: b, codes, [diagonal, couplings], [parent x].
template <int DIM, class T, class CS, bool FINE, bool UP>
struct FPlan {
    static constexpr int NC = FINE ? 0 : (DIM == 3 ? 3 : 2);
    static constexpr size_t OFF_B = 0;
    static constexpr size_t OFF_CODE = align128(RBox<T>::BYTES);
    static constexpr size_t OFF_DG = OFF_CODE + align128(RBox<uint8_t>::BYTES);
    static constexpr size_t OFF_CX = OFF_DG + (FINE ? 0 : align128(RBox<T>::BYTES));
    static constexpr size_t CB = align128(RBox<CS>::BYTES);
    static constexpr size_t OFF_CY = OFF_CX + CB, OFF_CZ = OFF_CY + CB;
    static constexpr size_t OFF_XC = OFF_CX + NC * CB;
    static constexpr size_t STAGE = OFF_XC + (UP ? align128(QBox<T>::BYTES) : 0);
    static constexpr uint32_t TX = RBox<T>::BYTES + RBox<uint8_t>::BYTES +
                                   (FINE ? 0u : RBox<T>::BYTES + NC * RBox<CS>::BYTES) +
                                   (UP ? QBox<T>::BYTES : 0u);
};

// Ring depth and shared memory.  LAG: planes behind the step that stay resident
// (the coarse levels read the -z coupling of plane s-2 in step 3); S >= LAG + 3
// keeps the plane of the next step in flight during the current one.
template <int DIM, class T, class CS, bool FINE, bool UP>
struct FCfg {
    using P = FPlan<DIM, T, CS, FINE, UP>;
    static constexpr int LAG = FINE ? 1 : 2;
    static constexpr int S = DIM == 2 ? 1 : LAG + 3 + (FINE ? (UP ? 2 : 3) : 1);
    static constexpr int NXP = DIM == 2 ? 1 : 3;  // shared x planes
    static constexpr size_t OFF_LUT = 128;          // after the stage barriers
    // finest level in FP32: the per-code table of the branch-free cell updates
    static constexpr bool LEAN = FINE && sizeof(T) == 4;
    static constexpr size_t OFF_TAB = OFF_LUT + align128(64 * sizeof(T));
    static constexpr size_t OFF_RING = OFF_TAB + (LEAN ? 128 * sizeof(float2) : 0);
    static constexpr size_t OFF_X = OFF_RING + S * P::STAGE;
    static constexpr size_t XB = align128(RBox<T>::BYTES);
    static constexpr size_t BYTES = OFF_X + NXP * XB;
    // resident blocks per SM the finest FP32 level is compiled for (registers): 3D,
    // five on the way down (its shared memory fits five) and four on the way up (at 48
    // registers the compiler recomputed values: 256^3, 74.3 M against 58.0 M warp
    // instructions, 101 against 89 us a launch; the way down at four, 73 against
    // 69 us); 2D, eight (a full SM of 256-thread
    // blocks; the 2D way up at five blocks and 48 registers: 2048 x 1024 solve 10.24
    // against 9.99 ms)
    static constexpr int MINB = LEAN ? (DIM == 3 ? (UP ? 4 : 5) : 8) : 1;
    static_assert(S <= 16, "stage barriers: 128 bytes");
};

// A cell of a task: box positions in the T, code and coupling boxes, the parent
// box position, its global offset in a level plane, whether it lies in the level,
// and its colour on plane 0 ((i + j) & 1).
struct FCell {
    int qt, qc, qs, qq;
    int gid;
    bool in;
    int par;
};

template <class T, class CS>
__device__ __forceinline__ FCell fcell(const Geom& g, int i0, int j0, int di, int dj) {
    FCell c;
    c.qt = RBox<T>::pos(di, dj);
    c.qc = RBox<uint8_t>::pos(di, dj);
    c.qs = RBox<CS>::pos(di, dj);
    c.qq = ((dj + 2) >> 1) * QBox<T>::W + ((di + 2) >> 1);
    const int i = i0 + di, j = j0 + dj;
    c.gid = i + j * g.sx;
    c.in = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny;
    c.par = (i + j) & 1;
    return c;
}

// The ring tasks: pair t (t < 104) of the 1-cell ring (t < 50) or the 2-cell ring;
// both cells of a pair are neighbours, so they have opposite colours.
__device__ __forceinline__ void ring_pair(int t, int& d1i, int& d1j, int& d2i, int& d2j) {
    if (t < 17) { d1i = 2 * t - 1; d2i = 2 * t; d1j = d2j = -1; }
    else if (t < 34) { const int u = t - 17; d1i = 2 * u - 1; d2i = 2 * u; d1j = d2j = kMY; }
    else if (t < 42) { const int u = t - 34; d1i = d2i = -1; d1j = 2 * u; d2j = 2 * u + 1; }
    else if (t < 50) { const int u = t - 42; d1i = d2i = kMX; d1j = 2 * u; d2j = 2 * u + 1; }
    else if (t < 68) { const int u = t - 50; d1i = 2 * u - 2; d2i = 2 * u - 1; d1j = d2j = -2; }
    else if (t < 86) { const int u = t - 68; d1i = 2 * u - 2; d2i = 2 * u - 1; d1j = d2j = kMY + 1; }
    else if (t < 95) { const int u = t - 86; d1i = d2i = -2; d1j = 2 * u - 1; d2j = 2 * u; }
    else { const int u = t - 95; d1i = d2i = kMX + 1; d1j = 2 * u - 1; d2j = 2 * u; }
}
constexpr int kRing1Tasks = 50, kRingTasks = 104;

template <int DIM, class T, class CS, bool FINE, bool UP>
__device__ __forceinline__ void f_issue(const FMaps& M, unsigned char* st, uint64_t* bar, int k) {
    using P = FPlan<DIM, T, CS, FINE, UP>;
    const int x0 = kMX * (int)blockIdx.x, y0 = kMY * (int)blockIdx.y - 1;
    fence_proxy_async();
    mbar_expect_tx(bar, P::TX);
    tma_load<DIM>(st + P::OFF_B, &M.b, x0 - RBox<T>::A, y0, k, bar);
    tma_load<DIM>(st + P::OFF_CODE, &M.code, x0 - RBox<uint8_t>::A, y0, k, bar);
    if constexpr (!FINE) {
        tma_load<DIM>(st + P::OFF_DG, &M.dg, x0 - RBox<T>::A, y0, k, bar);
        tma_load<DIM>(st + P::OFF_CX, &M.cx, x0 - RBox<CS>::A, y0, k, bar);
        tma_load<DIM>(st + P::OFF_CY, &M.cy, x0 - RBox<CS>::A, y0, k, bar);
        if constexpr (DIM == 3) tma_load<DIM>(st + P::OFF_CZ, &M.cz, x0 - RBox<CS>::A, y0, k, bar);
    }
    if constexpr (UP)
        tma_load<DIM>(st + P::OFF_XC, &M.xc, x0 / 2, (y0 + 1) / 2, (k + 1) >> 1, bar);
}

// Planes p0 .. plast pass through S stages; plane p uses stage (p - p0) mod S.
// Thread 0 issues every load and is the only thread that waits on the barriers.
template <int DIM, class T, class CS, bool FINE, bool UP, int S>
struct FRing {
    using P = FPlan<DIM, T, CS, FINE, UP>;
    uint64_t* bars;
    unsigned char* base;
    int p0, plast;
    // stage of plane p (p >= p0 - S; planes below p0 are never read)
    __device__ unsigned char* at(int p) const {
        return base + (size_t)((p - p0 + 2 * S) % S) * P::STAGE;
    }
    __device__ bool wait(int p) const {
        const int u = p - p0;
        return mbar_wait(&bars[u % S], (uint32_t)((u / S) & 1), kTmaWaitLimit);
    }
    __device__ void start(const FMaps& M) const {
        for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
        for (int p = p0; p < p0 + S && p <= plast; ++p)
            f_issue<DIM, T, CS, FINE, UP>(M, at(p), &bars[(p - p0) % S], p);
    }
    // after a block barrier: plane `freed` is no longer read; load plane freed + S
    __device__ void refill(const FMaps& M, int freed) const {
        if (freed >= p0 && freed + S <= plast)
            f_issue<DIM, T, CS, FINE, UP>(M, at(freed + S), &bars[(freed - p0) % S], freed + S);
    }
};

// Recent values of one column: the last two odd-colour values and the last
// even-colour value computed for it.
template <class T>
struct FHist {
    T o1, o2, e1;
};

// The dynamic shared memory of a fused march (128-byte aligned; see march.cuh).
#define UAAMG_FUSED_SMEM(sm, err)                                                 \
    extern __shared__ __align__(128) unsigned char smem_raw[];                   \
    unsigned char* sm = smem_raw;                                                \
    if (smem_u32(sm) & 127u) {                                                   \
        if (threadIdx.x == 0) atomicExch(err, 2);                                \
        return;                                                                  \
    }

template <int DIM, class T, bool FINE, class CS, bool UP, bool ZDOT>
__global__ void __launch_bounds__(kThreads, (FCfg<DIM, T, CS, FINE, UP>::MINB))
    k_level_fused(const __grid_constant__ FMaps M, MLevel<T> L, T* __restrict__ out,
                  const int* __restrict__ done, int* err, double* partials, CGState* cg) {
    pdl_entry();
    if (done && *done) return;
    using C = FCfg<DIM, T, CS, FINE, UP>;
    using P = typename C::P;
    constexpr int S = C::S, WT = RBox<T>::W, WS = RBox<CS>::W;
    constexpr bool kFull = sizeof(T) == 8;  // the reference's residual expression
    UAAMG_FUSED_SMEM(sm, err)
    T* lut = reinterpret_cast<T*>(sm + C::OFF_LUT);
    const Geom& g = L.g;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int i0 = 1 + kMX * (int)blockIdx.x, j0 = 1 + kMY * (int)blockIdx.y;
    if (FINE) build_lut<DIM, T>(lut, L.idx2, L.idy2, L.idz2);
    // Finest level in FP32 (no Dirichlet walls: those problems take the four-march
    // level): every cell update is a multiply-add driven by the table entry of its
    // code's low 7 bits (neighbour bits, interior-fluid bit): x = 1/d for an interior
    // fluid cell the smoother relaxes (d >= 1e-30), else 0; y = 1 for an interior
    // fluid cell it skips (d < 1e-30), else 0.
    constexpr bool LEAN = C::LEAN;
    const float2* tab = reinterpret_cast<const float2*>(sm + C::OFF_TAB);
    if constexpr (LEAN) {
        if (tid < 128) {
            const uint32_t c = (uint32_t)tid;
            float d = ((c & 1u) ? (float)L.idx2 : 0.f) + ((c & 2u) ? (float)L.idx2 : 0.f) +
                      ((c & 4u) ? (float)L.idy2 : 0.f) + ((c & 8u) ? (float)L.idy2 : 0.f);
            if (DIM == 3) d = d + ((c & 16u) ? (float)L.idz2 : 0.f) + ((c & 32u) ? (float)L.idz2 : 0.f);
            const bool act = (c & kActive) != 0, skip = act && d < 1e-30f;
            float2 e;
            e.x = act && !skip ? mdiv<float, CS>(1.0f, d) : 0.f;
            e.y = skip ? 1.f : 0.f;
            reinterpret_cast<float2*>(sm + C::OFF_TAB)[tid] = e;
        }
    }

    // --- per-cell arithmetic --------------------------------------------------
    auto code_at = [&](const unsigned char* st, const FCell& c) -> uint32_t {
        return st[P::OFF_CODE + c.qc];
    };
    auto b_at = [&](const unsigned char* st, const FCell& c) -> T {
        return reinterpret_cast<const T*>(st + P::OFF_B)[c.qt];
    };
    // (a finest level with Dirichlet walls never runs here: no wall diagonal)
    auto diag_of = [&](const unsigned char* st, const FCell& c, uint32_t code, int k) -> T {
        if constexpr (FINE) {
            return lut[code & 63u];
        } else {
            return reinterpret_cast<const T*>(st + P::OFF_DG)[c.qt];
        }
    };
    // couplings +x, -x, +y, -y, +z, -z (stc: this plane, stm: the plane below)
    auto coup = [&](const unsigned char* stc, const unsigned char* stm, const FCell& c, T (&cc)[6]) {
        if constexpr (FINE) {
            cc[0] = cc[1] = L.idx2;
            cc[2] = cc[3] = L.idy2;
            cc[4] = cc[5] = L.idz2;
        } else {
            const CS* cx = reinterpret_cast<const CS*>(stc + P::OFF_CX);
            const CS* cy = reinterpret_cast<const CS*>(stc + P::OFF_CY);
            cc[0] = coupling<T, CS>(cx[c.qs], L.csx);
            cc[1] = coupling<T, CS>(cx[c.qs - 1], L.csx);
            cc[2] = coupling<T, CS>(cy[c.qs], L.csy);
            cc[3] = coupling<T, CS>(cy[c.qs - WS], L.csy);
            if constexpr (DIM == 3) {
                cc[4] = coupling<T, CS>(reinterpret_cast<const CS*>(stc + P::OFF_CZ)[c.qs], L.csz);
                cc[5] = coupling<T, CS>(reinterpret_cast<const CS*>(stm + P::OFF_CZ)[c.qs], L.csz);
            } else {
                cc[4] = cc[5] = T(0);
            }
        }
    };
    // sum c_n v_n in the reference's order (v: a shared x plane)
    auto nbsum2 = [&](const T (&cc)[6], const T* v, int q, T vp, T vm) -> T {
        T nb = cc[0] * v[q + 1] + cc[1] * v[q - 1] + cc[2] * v[q + WT] + cc[3] * v[q - WT];
        if (DIM == 3) nb = nb + cc[4] * vp + cc[5] * vm;
        return nb;
    };
    auto prolong = [&](const unsigned char* st, const FCell& c) -> T {
        return T(2) * reinterpret_cast<const T*>(st + P::OFF_XC)[c.qq];
    };
    // odd-colour value at plane k: pre-smoothed (b + 0)/d, plus the prolongation on
    // the way up; 0 on cells that are not interior fluid
    auto oval = [&](const unsigned char* st, const FCell& c, int k) -> T {
        if constexpr (LEAN) {
            const uint32_t code = code_at(st, c);
            const float2 t = tab[code & 127u];
            if constexpr (UP) return b_at(st, c) * t.x + ((code & kActive) ? prolong(st, c) : T(0));
            else return b_at(st, c) * t.x;
        }
        const uint32_t code = code_at(st, c);
        if (!(code & kActive)) return T(0);
        const T d = diag_of(st, c, code, k);
        const T pre = d < T(1e-30) ? T(0) : mdiv<T, CS>(b_at(st, c) + T(0), d);
        if constexpr (UP) return pre + prolong(st, c);
        else return pre;
    };
    // even-colour value at plane k from the odd values around it: forward sweep
    // (way down) or first colour of the reverse sweep (way up; a skipped cell keeps
    // 0 + the prolongation)
    auto evalc = [&](const unsigned char* st, const unsigned char* stm, const T* xv, const FCell& c,
                     int k, T op, T om) -> T {
        if constexpr (LEAN) {
            const float2 t = tab[code_at(st, c) & 127u];
            const int q = c.qt;
            T nb = L.idx2 * (xv[q + 1] + xv[q - 1]) + L.idy2 * (xv[q + WT] + xv[q - WT]);
            if (DIM == 3) nb = nb + L.idz2 * (op + om);
            if constexpr (UP) return (b_at(st, c) + nb) * t.x + t.y * prolong(st, c);
            else return (b_at(st, c) + nb) * t.x;
        }
        const uint32_t code = code_at(st, c);
        if (!(code & kActive)) return T(0);
        const T d = diag_of(st, c, code, k);
        if (d < T(1e-30)) {
            if constexpr (UP) return T(0) + prolong(st, c);
            else return T(0);
        }
        T cc[6];
        coup(st, stm, c, cc);
        return mdiv<T, CS>(b_at(st, c) + nbsum2(cc, xv, c.qt, op, om), d);
    };

    // --- tasks ---------------------------------------------------------------
    // tile pair: A = (i0 + lane, j0 + 2w), B = (i0 + lane, j0 + 2w + 1)
    const FCell cA = fcell<T, CS>(g, i0, j0, lane, 2 * w);
    const FCell cB = fcell<T, CS>(g, i0, j0, lane, 2 * w + 1);
    const bool ring = tid < kRingTasks, ring1 = tid < kRing1Tasks;
    FCell cR1, cR2;
    {
        int d1i = 0, d1j = 0, d2i = 0, d2j = 0;
        if (ring) ring_pair(tid, d1i, d1j, d2i, d2j);
        cR1 = fcell<T, CS>(g, i0, j0, d1i, d1j);
        cR2 = fcell<T, CS>(g, i0, j0, d2i, d2j);
    }
    int kb, ke;
    zrange<DIM>(g, L.zc, kb, ke);
    T* xpl = reinterpret_cast<T*>(sm + C::OFF_X);
    double acc[3] = {0.0, 0.0, 0.0};
    const int ic = kMX / 2 * (int)blockIdx.x + 1 + (lane >> 1);
    const int jc = kMY / 2 * (int)blockIdx.y + 1 + w;
    const bool writer = !UP && (lane & 1) == 0 && ic <= L.cg.nx && jc <= L.cg.ny;

    // Final step on the tile pair at plane k, in colour order: cO / cE are the pair's
    // odd and even cells there, vO / vE their x values, zp* / zm* their columns'
    // values at k+1 and k-1; aOdd: A is the odd cell.  rlo: the way down's dk = 0
    // residuals, kept from the odd plane below.
    auto final_pair = [&](auto kodd, const unsigned char* st, const unsigned char* stm, const T* xv,
                          int k, const FCell& cO, const FCell& cE, bool aOdd, T vO, T vE, T zpO,
                          T zmO, T zpE, T zmE, T (&rlo)[2]) {
        constexpr bool KODD = decltype(kodd)::value;  // plane k is odd (3D)
        const uint32_t kO = code_at(st, cO), kE = code_at(st, cE);
        T resO = UP ? vO : T(0), resE = UP ? vE : T(0);
        if constexpr (LEAN) {
            const float2 tO = tab[kO & 127u];
            const int q = cO.qt;
            T nb = L.idx2 * (xv[q + 1] + xv[q - 1]) + L.idy2 * (xv[q + WT] + xv[q - WT]);
            if (DIM == 3) nb = nb + L.idz2 * (zpO + zmO);
            if constexpr (UP) {
                resO = (b_at(st, cO) + nb) * tO.x + tO.y * vO;  // a skipped cell keeps vO
            } else {
                const float2 tE = tab[kE & 127u];
                resO = (tO.x != 0.f ? nb : T(0)) + tO.y * b_at(st, cO);
                resE = tE.y * b_at(st, cE);
            }
        } else if (kO & kActive) {  // odd cell: reverse-sweep update / residual
            const T d = diag_of(st, cO, kO, k);
            if constexpr (UP) {
                if (!(d < T(1e-30))) {
                    T cc[6];
                    coup(st, stm, cO, cc);
                    resO = mdiv<T, CS>(b_at(st, cO) + nbsum2(cc, xv, cO.qt, zpO, zmO), d);
                }
            } else if constexpr (kFull) {
                T cc[6];
                coup(st, stm, cO, cc);
                T ax = d * vO - cc[0] * xv[cO.qt + 1] - cc[1] * xv[cO.qt - 1] -
                       cc[2] * xv[cO.qt + WT] - cc[3] * xv[cO.qt - WT];
                if (DIM == 3) ax = ax - cc[4] * zpO - cc[5] * zmO;
                resO = b_at(st, cO) - ax;
            } else {
                if (d < T(1e-30)) {
                    resO = b_at(st, cO);
                } else {
                    T cc[6];
                    coup(st, stm, cO, cc);
                    resO = nbsum2(cc, xv, cO.qt, zpO, zmO);
                }
            }
        }
        if constexpr (!UP && !LEAN) {
            if (kE & kActive) {  // even cell: residual (0 after its relaxation in FP32)
                const T d = diag_of(st, cE, kE, k);
                if constexpr (kFull) {
                    T cc[6];
                    coup(st, stm, cE, cc);
                    T ax = d * vE - cc[0] * xv[cE.qt + 1] - cc[1] * xv[cE.qt - 1] -
                           cc[2] * xv[cE.qt + WT] - cc[3] * xv[cE.qt - WT];
                    if (DIM == 3) ax = ax - cc[4] * zpE - cc[5] * zmE;
                    resE = b_at(st, cE) - ax;
                } else {
                    if (d < T(1e-30)) resE = b_at(st, cE);
                }
            }
        }
        if constexpr (UP) {
            const int base = k * g.sxy;
            const bool inO = cO.in, inE = cE.in;
            if (inO) out[cO.gid + base] = resO;
            if (inE) out[cE.gid + base] = resE;
            if (ZDOT) {
                if constexpr (LEAN) {
                    // z and b are 0 on every cell that is not interior fluid (ghosts,
                    // padding and cells past the level included)
                    const double zo = (double)resO, ro = (double)b_at(st, cO);
                    const double ze = (double)resE, re = (double)b_at(st, cE);
                    acc[0] += zo;
                    acc[1] += ro * zo;
                    acc[2] += ro;
                    acc[0] += ze;
                    acc[1] += re * ze;
                    acc[2] += re;
                } else {
                    if ((kO & kActive) && inO) {
                        const double zv = (double)resO, rv = (double)b_at(st, cO);
                        acc[0] += zv;
                        acc[1] += rv * zv;
                        acc[2] += rv;
                    }
                    if ((kE & kActive) && inE) {
                        const double zv = (double)resE, rv = (double)b_at(st, cE);
                        acc[0] += zv;
                        acc[1] += rv * zv;
                        acc[2] += rv;
                    }
                }
            }
        } else {
            const T res[2] = {aOdd ? resO : resE, aOdd ? resE : resO};  // [dj]
            // restriction: children dk = 0 on odd planes; the set is complete on the
            // even plane that follows (2D: one plane)
            if (DIM == 3 && KODD) {
                rlo[0] = res[0];
                rlo[1] = res[1];
            } else {
                T pr[2][2];  // the di = 1 partner's values [dj][dk]
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    pr[e][0] = __shfl_down_sync(0xffffffffu, DIM == 3 ? rlo[e] : res[e], 1);
                    pr[e][1] = __shfl_down_sync(0xffffffffu, res[e], 1);
                }
                if (writer) {
                    const int kc = DIM == 3 ? k / 2 : 0;
                    const int cid = cidx(L.cg, ic, jc, kc);
                    T sum = T(0);
                    if (DIM == 3) {
                        sum += rlo[0]; sum += res[0]; sum += rlo[1]; sum += res[1];
                        sum += pr[0][0]; sum += pr[0][1]; sum += pr[1][0]; sum += pr[1][1];
                    } else {
                        sum += res[0]; sum += res[1];
                        sum += pr[0][1]; sum += pr[1][1];
                    }
                    // also written on solid coarse cells, where no kernel reads b
                    out[cid] = sum;
                }
            }
        }
    };

    T rlo[2] = {T(0), T(0)};
    if constexpr (DIM == 2) {
        // one plane: odd values, barrier, even values, barrier, final
        unsigned char* st = sm + C::OFF_RING;
        uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
        bool ok = true;
        if (tid == 0) {
            mbar_init(bar, 1);
            f_issue<DIM, T, CS, FINE, UP>(M, st, bar, 0);
            ok = mbar_wait(bar, 0u, kTmaWaitLimit);
        }
        if (!step_barrier(ok, err)) return;
        // A is odd when i + j is odd; ring pairs likewise
        const bool oddA = cA.par != 0;
        const FCell tO = oddA ? cA : cB, tE = oddA ? cB : cA;
        const bool odd1 = cR1.par != 0;
        const FCell rO = odd1 ? cR1 : cR2, rE = odd1 ? cR2 : cR1;
        const T ot = oval(st, tO, 0);
        xpl[tO.qt] = ot;
        if (ring) xpl[rO.qt] = oval(st, rO, 0);
        __syncthreads();
        const T et = evalc(st, st, xpl, tE, 0, T(0), T(0));
        xpl[tE.qt] = et;
        if (ring1) xpl[rE.qt] = evalc(st, st, xpl, rE, 0, T(0), T(0));
        __syncthreads();
        final_pair(std::false_type(), st, st, xpl, 0, tO, tE, oddA, ot, et, T(0), T(0), T(0), T(0),
                   rlo);
    } else {
        // steps s = kb-3 .. ke: odd values of planes kb-2 .. ke+1, even values of
        // kb-1 .. ke, final results of kb .. ke-1
        const int s0 = kb - 3;
        FRing<DIM, T, CS, FINE, UP, S> R{reinterpret_cast<uint64_t*>(sm), sm + C::OFF_RING, kb - 2,
                                         ke + 1};
        bool ok = true;
        if (tid == 0) {
            R.start(M);
            ok = R.wait(R.p0);
        }
        if (!step_barrier(ok, err)) return;
        // role 0 is the cell that is even on planes s0, s0+2, ... (odd on s0+1, ...)
        const bool aRole0 = ((cA.par + s0) & 1) == 0;
        const FCell t0 = aRole0 ? cA : cB, t1 = aRole0 ? cB : cA;
        const bool r1Role0 = ((cR1.par + s0) & 1) == 0;
        const FCell q0 = r1Role0 ? cR1 : cR2, q1 = r1Role0 ? cR2 : cR1;
        FHist<T> ht[2] = {{T(0), T(0), T(0)}, {T(0), T(0), T(0)}};
        T hr[2] = {T(0), T(0)};  // ring columns: last odd value
        // stages of planes s+1, s, s-1, s-2 and the shared x planes s+1, s, s-1,
        // rotated once per step (planes below p0 are never read)
        const unsigned char* ring_end = sm + C::OFF_RING + S * P::STAGE;
        const unsigned char* sp1 = R.at(s0 + 1);
        const unsigned char* s00 = R.at(s0);
        const unsigned char* sm1 = R.at(s0 - 1);
        const unsigned char* sm2 = R.at(s0 - 2);
        T* xn = xpl + (size_t)((s0 + 4) % 3) * (C::XB / sizeof(T));
        T* xc = xpl + (size_t)((s0 + 3) % 3) * (C::XB / sizeof(T));
        T* xo = xpl + (size_t)((s0 + 5) % 3) * (C::XB / sizeof(T));
        // one step; R0c: the role whose cell is even at plane s; PHc: the phases it runs
        // (2: odd and even values, 3: all three; 0: decided at run time from s) --
        // compile-time
        auto step = [&](int s, auto R0c, auto PHc) -> bool {
            constexpr int RC = decltype(R0c)::value, RO = 1 - RC, PH = decltype(PHc)::value;
            const bool run_even = PH == 0 ? s >= kb - 1 : PH >= 2;
            const bool run_final = PH == 0 ? s >= kb + 1 : PH == 3;
            const FCell& tc = RC == 0 ? t0 : t1;
            const FCell& qc = RC == 0 ? q0 : q1;
            // 1. odd values of plane s+1
            const T on = oval(sp1, tc, s + 1);
            xn[tc.qt] = on;
            T onr = T(0);
            if (ring) {
                onr = oval(sp1, qc, s + 1);
                xn[qc.qt] = onr;
            }
            // 2. even values of plane s
            T en = T(0);
            if (run_even) {
                en = evalc(s00, sm1, xc, tc, s, on, ht[RC].o1);
                xc[tc.qt] = en;
                if (ring1) xc[qc.qt] = evalc(s00, sm1, xc, qc, s, onr, hr[RC]);
            }
            // 3. final results of plane s-1: the role-RC cell is odd there (plane s-1 is
            // odd for role 0: s0 = kb - 3 is even)
            if (run_final) {
                const int p = s - 1;
                const T vR = ht[RC].o1, vO = ht[RO].e1;   // x at p
                const T zpR = en, zmR = ht[RC].e1;         // role RC: even values at p+1, p-1
                const T zpO = ht[RO].o1, zmO = ht[RO].o2;  // role RO: odd values at p+1, p-1
                const FCell& to = RC == 0 ? t1 : t0;
                final_pair(std::integral_constant<bool, RC == 0>(), sm1, sm2, xo, p, tc, to,
                           aRole0 == (RC == 0), vR, vO, zpR, zmR, zpO, zmO, rlo);
            }
            ht[RC].o2 = ht[RC].o1;
            ht[RC].o1 = on;
            ht[RC].e1 = en;
            hr[RC] = onr;
            sm2 = sm1;
            sm1 = s00;
            s00 = sp1;
            sp1 += P::STAGE;
            if (sp1 == ring_end) sp1 = sm + C::OFF_RING;
            {
                T* t = xo;
                xo = xc;
                xc = xn;
                xn = t;
            }
            bool okk = true;
            if (tid == 0 && s + 2 <= R.plast) okk = R.wait(s + 2);
            if (!step_barrier(okk, err)) return false;
            if (tid == 0) R.refill(M, s - C::LAG);
            return true;
        };
        using R0 = std::integral_constant<int, 0>;
        using R1 = std::integral_constant<int, 1>;
        if constexpr (UP) {
            // one loop, phases by s (fewer registers than two loops here)
#pragma unroll 1
            for (int s = s0; s <= ke; s += 2) {
                if (!step(s, R0(), std::integral_constant<int, 0>())) return;
                if (s + 1 <= ke && !step(s + 1, R1(), std::integral_constant<int, 0>())) return;
            }
        } else {
            // steps kb-3 .. kb fill the pipeline: odd and even values only (the even
            // values of planes kb-3, kb-2 are not needed; their shared positions are
            // written again before any read); then ke >= kb + 1 steps run all three
#pragma unroll 1
            for (int s = s0; s <= kb; s += 2) {
                if (!step(s, R0(), std::integral_constant<int, 2>())) return;
                if (!step(s + 1, R1(), std::integral_constant<int, 2>())) return;
            }
#pragma unroll 1
            for (int s = kb + 1; s <= ke; s += 2) {
                if (!step(s, R0(), std::integral_constant<int, 3>())) return;
                if (s + 1 <= ke && !step(s + 1, R1(), std::integral_constant<int, 3>())) return;
            }
        }
    }
    if constexpr (UP && ZDOT) {
        double tot[3];
        if (reduce_last<3>(acc, partials, &cg->counter[2], tot)) finish_zdot(cg, tot);
    }
}

// ---------------------------------------------------------------------------
// Small 3D levels (a few 8^3 tiles): the same two steps per level as whole-tile
// boxes instead of z marches, whose pipeline never fills on a handful of planes.  A
// block owns an 8 x 8 x 8 tile; one TMA load per array brings the tile and a 2-cell
// ring (12^3 cells) into shared memory; then (1) the odd-colour values on the whole
// box, (2) the even-colour values on the tile and the inner ring, (3) the final
// results on the tile (way down: residual and restriction; way up: odd colour of
// the reverse sweep, the store, and on the finest level the z sums), with one block
// barrier between the phases.  Per-cell expressions are those of k_level_fused.
constexpr int kBT = 8;               // tile edge
constexpr int kBB = kBT + 4;         // box edge (2-cell ring)

// Box of element type E: cells i in [i0-2, i0+9] (i0 = 1 + 8 bx), the start column
// 8 bx - A rounded to 16 bytes; rows and planes 12.
template <class E>
struct BBox {
    static constexpr int A = 16 / (int)sizeof(E);
    static constexpr int W = (A + kBB - 1 + A - 1) / A * A;
    static constexpr uint32_t BYTES = (uint32_t)(W * kBB * kBB * sizeof(E));
    __host__ __device__ static constexpr int pos(int di, int dj, int dk) {
        return ((dk + 2) * kBB + (dj + 2)) * W + A + 1 + di;
    }
};
// Parent box (coarse x under the box): coarse cells [4 bx, 4 bx + 5] per axis.
template <class T>
struct BQBox {
    static constexpr int W = (6 * (int)sizeof(T) + 15) / 16 * 16 / (int)sizeof(T);
    static constexpr uint32_t BYTES = (uint32_t)(W * 6 * 6 * sizeof(T));
};

template <class T, class CS, bool FINE, bool UP>
struct BPlan {
    static constexpr size_t OFF_B = 0;
    static constexpr size_t OFF_CODE = align128(BBox<T>::BYTES);
    static constexpr size_t OFF_DG = OFF_CODE + align128(BBox<uint8_t>::BYTES);
    static constexpr size_t CB = align128(BBox<CS>::BYTES);
    static constexpr size_t OFF_CX = OFF_DG + (FINE ? 0 : align128(BBox<T>::BYTES));
    static constexpr size_t OFF_CY = OFF_CX + CB, OFF_CZ = OFF_CY + CB;
    static constexpr size_t OFF_XC = OFF_CX + (FINE ? 0 : 3 * CB);
    static constexpr size_t OFF_X = OFF_XC + (UP ? align128(BQBox<T>::BYTES) : 0);
    static constexpr size_t OFF_BAR = OFF_X + align128(BBox<T>::BYTES);
    static constexpr size_t OFF_LUT = OFF_BAR + 128;
    static constexpr size_t BYTES = OFF_LUT + align128(64 * sizeof(T));
    static constexpr uint32_t TX = BBox<T>::BYTES + BBox<uint8_t>::BYTES +
                                   (FINE ? 0u : BBox<T>::BYTES + 3 * BBox<CS>::BYTES) +
                                   (UP ? BQBox<T>::BYTES : 0u);
};

// Tensor maps of a box kernel: b, codes, diagonal, couplings (BBox geometry), and the
// parent level's x (BQBox geometry).
struct BMaps {
    CUtensorMap b, code, dg, cx, cy, cz, xc;
    // coarse levels: per box the default stencil {d, c_x, c_y, c_z} (as T) when every
    // cell of the box and its 2-cell ring is interior fluid with that diagonal and
    // those couplings (a trimmed box), else d = 0 (k_box_trim); null: no trimming
    const void* trim;
};

// Trimming of a coarse box level (the reference's tile trimming,
// cuda_uaamg_preconditioner_3d.cu:81-99 and :357-375, on this kernel's 8^3 tiles): a
// box whose 12^3 cells (tile and 2-cell ring) are all interior fluid and share one
// diagonal and one coupling per axis needs none of its diagonal, coupling or code
// boxes: the box kernel loads b (and the parent x) only and uses the four values.
// The values are the stored ones, so results are identical with and without
// trimming.  One block of 256 threads per box; rec[4 box + 0] = d or 0.
template <class E>
__device__ __forceinline__ bool same_bits(E a, E b) {
    if constexpr (sizeof(E) == 2) return __half_as_ushort(a) == __half_as_ushort(b);
    else if constexpr (sizeof(E) == 4) return __float_as_uint(a) == __float_as_uint(b);
    else return __double_as_longlong(a) == __double_as_longlong(b);
}

template <class T, class CS>
__global__ void __launch_bounds__(256) k_box_trim(Geom g, const uint8_t* __restrict__ code,
                                                  const T* __restrict__ dg, const CS* __restrict__ cx,
                                                  const CS* __restrict__ cy, const CS* __restrict__ cz,
                                                  T csx, T csy, T csz, T* rec) {
    pdl_entry();
    const int i0 = 1 + kBT * (int)blockIdx.x, j0 = 1 + kBT * (int)blockIdx.y,
              k0 = 1 + kBT * (int)blockIdx.z;
    const bool inside = i0 - 2 >= 1 && j0 - 2 >= 1 && k0 - 2 >= 1 && i0 + kBT + 1 <= g.nx &&
                        j0 + kBT + 1 <= g.ny && k0 + kBT + 1 <= g.nz;
    bool ok = inside;
    T d0 = T(0);
    CS x0{}, y0{}, z0{};
    if (inside) {
        const int id0 = cidx(g, i0, j0, k0);
        d0 = dg[id0];
        x0 = cx[id0];
        y0 = cy[id0];
        z0 = cz[id0];
        ok = !(d0 < T(1e-30));
        for (int c = threadIdx.x; ok && c < kBB * kBB * kBB; c += blockDim.x) {
            const int i = i0 - 2 + c % kBB, j = j0 - 2 + (c / kBB) % kBB, k = k0 - 2 + c / (kBB * kBB);
            const int id = cidx(g, i, j, k);
            ok = (code[id] & kActive) && same_bits(dg[id], d0) && same_bits(cx[id], x0) &&
                 same_bits(cy[id], y0) && same_bits(cz[id], z0);
        }
    }
    ok = __syncthreads_and(ok) != 0;
    if (threadIdx.x == 0) {
        const size_t r = 4 * (((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x);
        rec[r] = ok ? d0 : T(0);
        rec[r + 1] = ok ? coupling<T, CS>(x0, csx) : T(0);
        rec[r + 2] = ok ? coupling<T, CS>(y0, csy) : T(0);
        rec[r + 3] = ok ? coupling<T, CS>(z0, csz) : T(0);
    }
}

template <class T, bool FINE, class CS, bool UP, bool ZDOT>
__global__ void __launch_bounds__(kThreads)
    k_level_box(const __grid_constant__ BMaps M, MLevel<T> L, T* __restrict__ out,
                const int* __restrict__ done, int* err, double* partials, CGState* cg) {
    pdl_entry();
    if (done && *done) return;
    using P = BPlan<T, CS, FINE, UP>;
    constexpr int WT = BBox<T>::W, WS = BBox<CS>::W;
    constexpr int PT = WT * kBB, PS = WS * kBB;  // plane strides
    constexpr bool kFull = sizeof(T) == 8;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* sm = smem_raw;
    if (smem_u32(sm) & 127u) {
        if (threadIdx.x == 0) atomicExch(err, 2);
        return;
    }
    const Geom& g = L.g;
    const int tid = threadIdx.x;
    const int bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
    const int i0 = 1 + kBT * bx, j0 = 1 + kBT * by, k0 = 1 + kBT * bz;
    T* lut = reinterpret_cast<T*>(sm + P::OFF_LUT);
    T* xs = reinterpret_cast<T*>(sm + P::OFF_X);
    const T* bs = reinterpret_cast<const T*>(sm + P::OFF_B);
    const unsigned char* cs = sm + P::OFF_CODE;
    const T* dgs = reinterpret_cast<const T*>(sm + P::OFF_DG);
    const CS* cxs = reinterpret_cast<const CS*>(sm + P::OFF_CX);
    const CS* cys = reinterpret_cast<const CS*>(sm + P::OFF_CY);
    const CS* czs = reinterpret_cast<const CS*>(sm + P::OFF_CZ);
    const T* xcs = reinterpret_cast<const T*>(sm + P::OFF_XC);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + P::OFF_BAR);
    if (FINE) build_lut<3, T>(lut, L.idx2, L.idy2, L.idz2);
    // a trimmed coarse box: its default stencil (d > 0), read before any load
    T trim[4] = {T(0), T(0), T(0), T(0)};
    if constexpr (!FINE) {
        if (M.trim) {
            const T* r = reinterpret_cast<const T*>(M.trim) + 4 * ((bz * gridDim.y + by) * gridDim.x + bx);
#pragma unroll
            for (int q = 0; q < 4; ++q) trim[q] = r[q];
        }
    }
    const bool tr = !FINE && trim[0] != T(0);
    // The code box starts at the 16-byte boundary at or below its first column (x0 - 1
    // in the padded array): x0 - 16 when bx is even, x0 - 8 when it is odd.  Every other
    // box starts at x0 - A, a 16-byte boundary for its element size.
    const int aC = kBT * bx - 16 * ((kBT * bx - 1) >> 4);
    static_assert(16 + kBT + 2 < BBox<uint8_t>::W, "code box: tile and ring at the widest offset");
    bool ok = true;
    if (tid == 0) {
        mbar_init(bar, 1);
        const int x0 = kBT * bx, y0 = kBT * by - 1, z0 = kBT * bz - 1;
        fence_proxy_async();
        constexpr uint32_t kTrimTX = BBox<T>::BYTES + (UP ? BQBox<T>::BYTES : 0u);
        mbar_expect_tx(bar, tr ? kTrimTX : P::TX);
        tma_load<3>(sm + P::OFF_B, &M.b, x0 - BBox<T>::A, y0, z0, bar);
        if (!tr) {
            tma_load<3>(sm + P::OFF_CODE, &M.code, x0 - aC, y0, z0, bar);
            if constexpr (!FINE) {
                tma_load<3>(sm + P::OFF_DG, &M.dg, x0 - BBox<T>::A, y0, z0, bar);
                tma_load<3>(sm + P::OFF_CX, &M.cx, x0 - BBox<CS>::A, y0, z0, bar);
                tma_load<3>(sm + P::OFF_CY, &M.cy, x0 - BBox<CS>::A, y0, z0, bar);
                tma_load<3>(sm + P::OFF_CZ, &M.cz, x0 - BBox<CS>::A, y0, z0, bar);
            }
        }
        if constexpr (UP) tma_load<3>(sm + P::OFF_XC, &M.xc, x0 / 2, (y0 + 1) / 2, (z0 + 1) / 2, bar);
        ok = mbar_wait(bar, 0u, kTmaWaitLimit);
    }
    if (!step_barrier(ok, err)) return;

    // per-cell helpers on box offsets (di, dj, dk) in [-2, 9]
    auto qT = [](int di, int dj, int dk) { return BBox<T>::pos(di, dj, dk); };
    auto qC = [aC](int di, int dj, int dk) {
        return BBox<uint8_t>::pos(di, dj, dk) - BBox<uint8_t>::A + aC;
    };
    auto qS = [](int di, int dj, int dk) { return BBox<CS>::pos(di, dj, dk); };
    auto nbsum = [&](const T (&cc)[6], int q) -> T {
        return cc[0] * xs[q + 1] + cc[1] * xs[q - 1] + cc[2] * xs[q + WT] + cc[3] * xs[q - WT] +
               cc[4] * xs[q + PT] + cc[5] * xs[q - PT];
    };
    auto prolong = [&](int di, int dj, int dk) -> T {
        return T(2) * xcs[(((dk + 2) >> 1) * 6 + ((dj + 2) >> 1)) * BQBox<T>::W + ((di + 2) >> 1)];
    };
    // colour of a box cell: (i + j + k) & 1 with i0 + j0 + k0 odd
    const int par0 = (i0 + j0 + k0) & 1;

    // The three steps; TR: a trimmed box (every cell interior fluid, the stencil in
    // trim[]), whose codes, diagonals and couplings were not loaded.
    auto run = [&](auto trimc) {
        constexpr bool TR = decltype(trimc)::value;
        auto code_at = [&](int di, int dj, int dk) -> uint32_t {
            if constexpr (TR) return kActive;
            else return cs[qC(di, dj, dk)];
        };
        auto diag = [&](uint32_t code, int q) -> T {
            if constexpr (TR) return trim[0];
            else if constexpr (FINE) return lut[code & 63u];
            else return dgs[q];
        };
        auto coup = [&](int qs, T (&cc)[6]) {
            if constexpr (TR) {
                cc[0] = cc[1] = trim[1];
                cc[2] = cc[3] = trim[2];
                cc[4] = cc[5] = trim[3];
            } else if constexpr (FINE) {
                cc[0] = cc[1] = L.idx2;
                cc[2] = cc[3] = L.idy2;
                cc[4] = cc[5] = L.idz2;
            } else {
                cc[0] = coupling<T, CS>(cxs[qs], L.csx);
                cc[1] = coupling<T, CS>(cxs[qs - 1], L.csx);
                cc[2] = coupling<T, CS>(cys[qs], L.csy);
                cc[3] = coupling<T, CS>(cys[qs - WS], L.csy);
                cc[4] = coupling<T, CS>(czs[qs], L.csz);
                cc[5] = coupling<T, CS>(czs[qs - PS], L.csz);
            }
        };

        // Cells are enumerated by colour: the rows (dj, dk) of a region hold
        // alternating colours, so the k-th cell of a colour in a row is di = first +
        // 2 m + s with s fixed by the row's parity.  A thread steps its enumeration
        // index by the block size, updating (m, row) incrementally.
        static_assert(kThreads == 256, "incremental colour enumeration assumes 256 threads");
        // 1. odd values on the whole box: 144 rows of 12 cells, 6 odd per row; a step
        // of 256 is 42 rows (3 planes and 6 rows) and 4 cells
        {
            int m = tid % 6, jj = (tid / 6) % kBB, kk = tid / (6 * kBB);
            while (kk < kBB) {
                const int dj = jj - 2, dk = kk - 2;
                const int di = -2 + 2 * m + ((1 + dj + dk + par0) & 1);
                const int q = qT(di, dj, dk);
                const uint32_t code = code_at(di, dj, dk);
                T v = T(0);
                if (code & kActive) {
                    const T d = diag(code, q);
                    v = d < T(1e-30) ? T(0) : mdiv<T, CS>(bs[q] + T(0), d);
                    if constexpr (UP) v = v + prolong(di, dj, dk);
                }
                xs[q] = v;
                m += 4;
                jj += 6;
                kk += 3;
                if (m >= 6) { m -= 6; jj += 1; }
                if (jj >= kBB) { jj -= kBB; kk += 1; }
            }
        }
        __syncthreads();
        // 2. even values on the tile and the inner ring: 100 rows of 10 cells, 5 even
        // per row; a step of 256 is 51 rows (5 planes and 1 row) and 1 cell
        {
            constexpr int R = kBT + 2;
            int m = tid % 5, jj = (tid / 5) % R, kk = tid / (5 * R);
            while (kk < R) {
                const int dj = jj - 1, dk = kk - 1;
                const int di = -1 + 2 * m + ((1 + dj + dk + par0) & 1);
                const int q = qT(di, dj, dk);
                const uint32_t code = code_at(di, dj, dk);
                T v = T(0);
                if (code & kActive) {
                    const T d = diag(code, q);
                    if (d < T(1e-30)) {
                        if constexpr (UP) v = T(0) + prolong(di, dj, dk);
                    } else {
                        T cc[6];
                        coup(qS(di, dj, dk), cc);
                        v = mdiv<T, CS>(bs[q] + nbsum(cc, q), d);
                    }
                }
                xs[q] = v;
                m += 1;
                jj += 1;
                kk += 5;
                if (m >= 5) { m -= 5; jj += 1; }
                if (jj >= R) { jj -= R; kk += 1; }
            }
        }
        __syncthreads();
        // 3. final results on the tile: thread = the x pair (2 m, 2 m + 1) of row (dj,
        // dk); u = 0 its odd cell, u = 1 its even cell (no lane diverges on colour)
        double acc[3] = {0.0, 0.0, 0.0};
        T* rs = reinterpret_cast<T*>(sm + P::OFF_B);  // way down: residuals replace b (tile only)
        T res[2];
        int resq[2];
        const int pm = tid & 3, pj = (tid >> 2) & 7, pk = tid >> 5;
        const int sO = (1 + pj + pk + par0) & 1;  // the odd cell is di = 2 pm + sO
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const bool odd = u == 0;
            const int di = 2 * pm + (u == 0 ? sO : 1 - sO), dj = pj, dk = pk;
            const int q = qT(di, dj, dk);
            const uint32_t code = code_at(di, dj, dk);
            const T x0 = xs[q];
            T v = UP ? x0 : T(0);
            if (code & kActive) {
                const T d = diag(code, q);
                if constexpr (UP) {
                    if (odd && !(d < T(1e-30))) {
                        T cc[6];
                        coup(qS(di, dj, dk), cc);
                        v = mdiv<T, CS>(bs[q] + nbsum(cc, q), d);
                    }
                } else if constexpr (kFull) {
                    T cc[6];
                    coup(qS(di, dj, dk), cc);
                    const T ax = d * x0 - cc[0] * xs[q + 1] - cc[1] * xs[q - 1] - cc[2] * xs[q + WT] -
                                 cc[3] * xs[q - WT] - cc[4] * xs[q + PT] - cc[5] * xs[q - PT];
                    v = bs[q] - ax;
                } else {
                    if (d < T(1e-30)) {
                        v = bs[q];
                    } else if (odd) {
                        T cc[6];
                        coup(qS(di, dj, dk), cc);
                        v = nbsum(cc, q);
                    }
                }
            }
            res[u] = v;
            resq[u] = q;
            if constexpr (UP) {
                const int i = i0 + di, j = j0 + dj, k = k0 + dk;
                if (i <= g.nx && j <= g.ny && k <= g.nz) {
                    out[cidx(g, i, j, k)] = v;
                    if (ZDOT && (code & kActive)) {
                        const double zv = (double)v, rv = (double)bs[q];
                        acc[0] += zv;
                        acc[1] += rv * zv;
                        acc[2] += rv;
                    }
                }
            }
        }
        if constexpr (!UP) {
            __syncthreads();  // every b of the tile has been read
#pragma unroll
            for (int u = 0; u < 2; ++u) rs[resq[u]] = res[u];
            __syncthreads();
            // restriction: 4^3 coarse cells, the 2x2x2 children in (di, dj, dk) order
            if (tid < (kBT / 2) * (kBT / 2) * (kBT / 2)) {
                const int ci = tid % 4, cj = (tid / 4) % 4, ck = tid / 16;
                const int ic = kBT / 2 * bx + 1 + ci, jc = kBT / 2 * by + 1 + cj,
                          kc = kBT / 2 * bz + 1 + ck;
                if (ic <= L.cg.nx && jc <= L.cg.ny && kc <= L.cg.nz) {
                    T sum = T(0);
#pragma unroll
                    for (int a = 0; a < 2; ++a)
#pragma unroll
                        for (int b2 = 0; b2 < 2; ++b2)
#pragma unroll
                            for (int e = 0; e < 2; ++e) sum += rs[qT(2 * ci + a, 2 * cj + b2, 2 * ck + e)];
                    // also written on solid coarse cells, where no kernel reads b
                    out[cidx(L.cg, ic, jc, kc)] = sum;
                }
            }
        }
        if constexpr (UP && ZDOT) {
            double tot[3];
            if (reduce_last<3>(acc, partials, &cg->counter[2], tot)) finish_zdot(cg, tot);
        }
    };
    if constexpr (FINE) {
        run(std::false_type{});
    } else {
        if (tr) run(std::true_type{});
        else run(std::false_type{});
    }
}

#undef UAAMG_FUSED_SMEM

}  // namespace
}  // namespace uaamg
