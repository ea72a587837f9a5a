// The V-cycle's small levels in ONE thread block: from the first level of at most
// kTailCells cells down to the coarsest and back up, in one launch instead of four
// z marches per level plus the coarsest solve (whose launches are mostly start-up
// latency at these sizes).  Every small level's x and b live in shared memory (the
// level's interior plus a zero ghost ring); codes, couplings and diagonals are read
// from global memory through L1.  The phases -- forward sweep, residual
// restriction, the coarsest level's 10 x (forward + reverse) sweeps, prolongation
// with the even colour, the odd colour -- are separated by block barriers.  The
// first level's b comes in from global memory and its x goes back out (the next
// finer level's prolongation reads it).
//
// Per cell the arithmetic is the marches' (march.cuh), in the reference's order:
//   forward sweep from x = 0   uaamg_preconditioner_3d.cpp:123-138 (smooth, colour
//                              1 then 0; odd cells see x = 0, so x = (b + 0)/d)
//   residual restriction       uaamg_preconditioner_3d.cpp:144-165
//   coarsest 10 x (fwd + rev)  uaamg_preconditioner_3d.cpp:185-186
//   prolongation x += 2 x_c    uaamg_preconditioner_3d.cpp:168-181
//   reverse sweep colour 0, 1  uaamg_preconditioner_3d.cpp:123-138
// so the FP64 engine stays bit-exact with the reference (built with -fmad=false).
#pragma once
#include "march.cuh"

namespace uaamg {
namespace {

// Largest level the tail takes: one block walks a level's cells a few a thread,
// each waiting on its codes and couplings from L2, which outgrows four z-march
// launches beyond about a thousand cells.
constexpr int kTailCells = 1024;
constexpr int kTailMaxLevels = 16;
constexpr size_t kTailSmemBytes = 200 * 1024;    // x and b of every tail level

template <class T>
constexpr int tail_threads() { return sizeof(T) == 8 ? 512 : 1024; }

template <class T>
struct TailLevel {
    Geom g;          // the level's global (pitched) layout
    int csx, csxy;   // shared-memory layout: (nx + 2) x (ny + 2) [x (nz + 2)]
    int xs, bs;      // offsets of x and b in the shared array (elements)
    const uint8_t* code;
    const T* cx;
    const T* cy;
    const T* cz;
    const T* dg;
    T* x;            // global x and b: used for the first level only
    const T* b;
    float rnx, rny;  // 1/nx, 1/ny (cell number -> (i, j, k))
};

template <class T>
struct TailArgs {
    int nlev;                         // levels in the tail; the last is the coarsest
    int smem_elems;                   // shared array length (elements of T)
    TailLevel<T> lv[kTailMaxLevels];  // lv[0]: the first (finest) level of the tail
};

template <int DIM>
__device__ __forceinline__ int tail_ncell(const Geom& g) {
    return g.nx * g.ny * (DIM == 3 ? g.nz : 1);
}

// Shared-memory view of one level: global index id (couplings, codes) and local
// index s (x, b) of a cell, and its neighbours' strides in both.
template <int DIM, class T>
struct TailView {
    const TailLevel<T>& L;
    T* x;
    T* b;
    __device__ __forceinline__ int gid(int i, int j, int k) const { return cidx(L.g, i, j, k); }
    __device__ __forceinline__ int sid(int i, int j, int k) const { return i + j * L.csx + k * L.csxy; }
};

// Couplings of the cell at global index id in the reference's order +x, -x, +y,
// -y, +z, -z.
template <int DIM, class T>
__device__ __forceinline__ void tail_coup(const TailLevel<T>& L, int id, T (&c)[6]) {
    c[0] = __ldg(L.cx + id);
    c[1] = __ldg(L.cx + id - 1);
    c[2] = __ldg(L.cy + id);
    c[3] = __ldg(L.cy + id - L.g.sx);
    if (DIM == 3) {
        c[4] = __ldg(L.cz + id);
        c[5] = __ldg(L.cz + id - L.g.sxy);
    } else {
        c[4] = c[5] = T(0);
    }
}

template <int DIM, class T>
__device__ __forceinline__ T tail_nb(const T (&c)[6], T xr, T xl, T xt, T xb, T xk, T xf) {
    T nb = c[0] * xr + c[1] * xl + c[2] * xt + c[3] * xb;
    if (DIM == 3) nb = nb + c[4] * xk + c[5] * xf;
    return nb;
}

// q = a / d, r = a % d for 0 <= a < 2^24, 0 < d, from the reciprocal rd = 1/d
// rounded to single precision (computed on the host): the estimate is off by at most
// one, and one exact correction step fixes it (every phase maps each thread's cell
// number to (i, j, k); an integer division by a value known only at run time costs as
// much as the cell's own arithmetic).
__device__ __forceinline__ int tail_divmod(int a, int d, float rd, int& r) {
    int q = __float2int_rz((float)a * rd);
    r = a - q * d;
    if (r < 0) { --q; r += d; }
    else if (r >= d) { ++q; r -= d; }
    return q;
}

// Interior cell number c (x fastest) -> (i, j, k) of level L.
template <int DIM, class T>
__device__ __forceinline__ void tail_ijk(const TailLevel<T>& L, int c, int& i, int& j, int& k) {
    int ri;
    const int r = tail_divmod(c, L.g.nx, L.rnx, ri);
    i = 1 + ri;
    if (DIM == 3) {
        int rj;
        k = 1 + tail_divmod(r, L.g.ny, L.rny, rj);
        j = 1 + rj;
    } else {
        j = 1 + r;
        k = 0;
    }
}

// Value after the forward sweep's first colour: (b + 0)/d on an active odd cell
// (0 when d < 1e-30), 0 on every other cell.  Every load is issued before the
// tests; a discarded quotient divides by 1.
template <int DIM, class T>
__device__ __forceinline__ T tail_pre(const TailView<DIM, T>& V, int id, int sd) {
    const uint32_t c = __ldg(V.L.code + id);
    const T d = __ldg(V.L.dg + id);
    const T b = V.b[sd];
    const bool on = (c & (kActive | kOdd)) == (kActive | kOdd) && !(d < T(1e-30));
    const T v = (b + T(0)) / (on ? d : T(1));
    return on ? v : T(0);
}

// Forward sweep from x = 0; writes x on every interior cell.
template <int DIM, class T>
__device__ void tail_fwd(const TailView<DIM, T>& V) {
    const Geom& g = V.L.g;
    const int n = tail_ncell<DIM>(g), gx = g.sx, gxy = g.sxy, sx = V.L.csx, sxy = V.L.csxy;
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        int i, j, k;
        tail_ijk<DIM>(V.L, c, i, j, k);
        const int id = V.gid(i, j, k), sd = V.sid(i, j, k);
        const uint32_t code = __ldg(V.L.code + id);
        const T d = __ldg(V.L.dg + id);
        T cc[6];
        tail_coup<DIM>(V.L, id, cc);
        const T nb = tail_nb<DIM, T>(cc, tail_pre(V, id + 1, sd + 1), tail_pre(V, id - 1, sd - 1),
                                     tail_pre(V, id + gx, sd + sx), tail_pre(V, id - gx, sd - sx),
                                     DIM == 3 ? tail_pre(V, id + gxy, sd + sxy) : T(0),
                                     DIM == 3 ? tail_pre(V, id - gxy, sd - sxy) : T(0));
        const bool on = (code & kActive) && !(d < T(1e-30));
        // odd cells see x = 0 everywhere: (b + 0)/d
        const T v = (V.b[sd] + ((code & kOdd) ? T(0) : nb)) / (on ? d : T(1));
        V.x[sd] = on ? v : T(0);
    }
}

// b - A x of one cell (0 on an inactive cell): the reference's expression in FP64,
// the sum of couplings times differences in FP32 (fp32_ax).
template <int DIM, class T>
__device__ __forceinline__ T tail_r(const TailView<DIM, T>& V, int id, int sd) {
    const int sx = V.L.csx, sxy = V.L.csxy;
    const uint32_t code = __ldg(V.L.code + id);
    const T d = __ldg(V.L.dg + id);
    T cc[6];
    tail_coup<DIM>(V.L, id, cc);
    const T* x = V.x;
    const T xc = x[sd], xr = x[sd + 1], xl = x[sd - 1], xt = x[sd + sx], xb = x[sd - sx];
    const T xk = DIM == 3 ? x[sd + sxy] : T(0);
    const T xf = DIM == 3 ? x[sd - sxy] : T(0);
    T ax;
    if constexpr (sizeof(T) == 8) {
        ax = d * xc - cc[0] * xr - cc[1] * xl - cc[2] * xt - cc[3] * xb;
        if (DIM == 3) ax = ax - cc[4] * xk - cc[5] * xf;
    } else {
        const MLevel<T> none{};  // coarse levels: fp32_ax reads only the couplings
        ax = fp32_ax<DIM, T, false>(none, code, d, cc, xc, xr, xl, xt, xb, xk, xf);
    }
    return (code & kActive) ? V.b[sd] - ax : T(0);
}

// Coarse b = sum of the children's residuals in the order (di, dj, dk); 0 on an
// inactive coarse cell.
template <int DIM, class T>
__device__ void tail_res(const TailView<DIM, T>& F, const TailView<DIM, T>& C) {
    const Geom& cg = C.L.g;
    const int n = tail_ncell<DIM>(cg);
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        int ic, jc, kc;
        tail_ijk<DIM>(C.L, c, ic, jc, kc);
        const int i0 = 2 * ic - 1, j0 = 2 * jc - 1, k0 = DIM == 3 ? 2 * kc - 1 : 0;
        T r[8];
#pragma unroll
        for (int q = 0; q < (DIM == 3 ? 8 : 4); ++q) {
            const int di = DIM == 3 ? q >> 2 : q >> 1, dj = DIM == 3 ? (q >> 1) & 1 : q & 1;
            const int dk = DIM == 3 ? q & 1 : 0;
            r[q] = tail_r(F, F.gid(i0 + di, j0 + dj, k0 + dk), F.sid(i0 + di, j0 + dj, k0 + dk));
        }
        T s = T(0);
#pragma unroll
        for (int q = 0; q < (DIM == 3 ? 8 : 4); ++q) s += r[q];
        C.b[C.sid(ic, jc, kc)] = (__ldg(C.L.code + C.gid(ic, jc, kc)) & kActive) ? s : T(0);
    }
}

// 2 x_c of the parent of fine cell (i, j, k); the coarse x is 0 at solid and ghost
// cells, so every fine cell may add it.
template <int DIM, class T>
__device__ __forceinline__ T tail_prol(const TailView<DIM, T>& C, int i, int j, int k) {
    return T(2) * C.x[C.sid((i + 1) >> 1, (j + 1) >> 1, DIM == 3 ? (k + 1) >> 1 : 0)];
}

// Odd cell after the prolongation: its forward value plus 2 x_c (0 unless active
// and odd).
template <int DIM, class T>
__device__ __forceinline__ T tail_odd(const TailView<DIM, T>& V, const TailView<DIM, T>& C, int i,
                                      int j, int k) {
    const int id = V.gid(i, j, k);
    const uint32_t c = __ldg(V.L.code + id);
    const T d = __ldg(V.L.dg + id);
    const T b = V.b[V.sid(i, j, k)];
    const T pc = tail_prol(C, i, j, k);
    const bool on = (c & (kActive | kOdd)) == (kActive | kOdd);
    const bool small = d < T(1e-30);
    const T q = (b + T(0)) / (on && !small ? d : T(1));
    return on ? (small ? T(0) : q) + pc : T(0);
}

// Prolongation and the reverse sweep's even colour; writes x on every interior cell.
template <int DIM, class T>
__device__ void tail_up_even(const TailView<DIM, T>& V, const TailView<DIM, T>& C) {
    const Geom& g = V.L.g;
    const int n = tail_ncell<DIM>(g);
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        int i, j, k;
        tail_ijk<DIM>(V.L, c, i, j, k);
        const int id = V.gid(i, j, k), sd = V.sid(i, j, k);
        const uint32_t code = __ldg(V.L.code + id);
        const T d = __ldg(V.L.dg + id);
        const T pc = tail_prol(C, i, j, k);
        T cc[6];
        tail_coup<DIM>(V.L, id, cc);
        const T nb = tail_nb<DIM, T>(cc, tail_odd(V, C, i + 1, j, k), tail_odd(V, C, i - 1, j, k),
                                     tail_odd(V, C, i, j + 1, k), tail_odd(V, C, i, j - 1, k),
                                     DIM == 3 ? tail_odd(V, C, i, j, k + 1) : T(0),
                                     DIM == 3 ? tail_odd(V, C, i, j, k - 1) : T(0));
        const bool act = code & kActive, odd = code & kOdd, small = d < T(1e-30);
        // odd: pre-smoothed (b + 0)/d plus 2 x_c; even: (b + sum c_n x_n)/d, or 0 + 2 x_c
        // when skipped
        const T q = (V.b[sd] + (odd ? T(0) : nb)) / (act && !small ? d : T(1));
        T x;
        if (!act) x = T(0);
        else if (odd) x = (small ? T(0) : q) + pc;
        else x = small ? T(0) + pc : q;
        V.x[sd] = x;
    }
}

// The reverse sweep's odd colour, in place (odd cells read only even neighbours).
template <int DIM, class T>
__device__ void tail_up_odd(const TailView<DIM, T>& V) {
    const Geom& g = V.L.g;
    const int n = tail_ncell<DIM>(g), sx = V.L.csx, sxy = V.L.csxy;
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
        int i, j, k;
        tail_ijk<DIM>(V.L, c, i, j, k);
        const int id = V.gid(i, j, k), sd = V.sid(i, j, k);
        const uint32_t code = __ldg(V.L.code + id);
        const T d = __ldg(V.L.dg + id);
        T cc[6];
        tail_coup<DIM>(V.L, id, cc);
        const T* x = V.x;
        const T nb = tail_nb<DIM, T>(cc, x[sd + 1], x[sd - 1], x[sd + sx], x[sd - sx],
                                     DIM == 3 ? x[sd + sxy] : T(0), DIM == 3 ? x[sd - sxy] : T(0));
        if ((code & (kActive | kOdd)) == (kActive | kOdd) && !(d < T(1e-30)))
            V.x[sd] = (V.b[sd] + nb) / d;
    }
}

// Barrier of the first nw warps (named barrier 1; a warp barrier for one warp).
__device__ __forceinline__ void tail_warps_sync(int nw) {
    if (nw == 1) __syncwarp();
    else asm volatile("bar.sync 1, %0;" ::"r"(nw * 32) : "memory");
}

// Coarsest level: 10 x (forward + reverse) sweeps from x = 0 (x zeroed by the
// caller) by the first ceil(n / 64) warps, two cells a thread held in registers.
template <int DIM, class T>
__device__ void tail_coarsest(const TailView<DIM, T>& V) {
    const Geom& g = V.L.g;
    const int n = tail_ncell<DIM>(g), sx = V.L.csx, sxy = V.L.csxy;
    const int nw = (n + 63) / 64;
    if ((int)threadIdx.x >= nw * 32) return;
    const int nthr = nw * 32;
    int sd2[2] = {-1, -1}, par2[2] = {0, 0};
    T d2[2] = {T(1), T(1)}, c2[2][6];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int c = threadIdx.x + s * nthr;
#pragma unroll
        for (int q = 0; q < 6; ++q) c2[s][q] = T(0);
        if (c < n) {
            int i, j, k;
            tail_ijk<DIM>(V.L, c, i, j, k);
            const int id = V.gid(i, j, k);
            const uint32_t code = __ldg(V.L.code + id);
            const T d = __ldg(V.L.dg + id);
            if ((code & kActive) && !(d < T(1e-30))) {
                sd2[s] = V.sid(i, j, k);
                par2[s] = (i + j + k) & 1;
                d2[s] = d;
                tail_coup<DIM>(V.L, id, c2[s]);
            }
        }
    }
    T* x = V.x;
    for (int it = 0; it < 10; ++it)
        for (int h = 0; h < 4; ++h) {
            const int parity = (h == 0 || h == 3) ? 1 : 0;  // forward 1, 0; reverse 0, 1
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const int sd = sd2[s];
                if (sd >= 0 && par2[s] == parity) {
                    const T nb = tail_nb<DIM, T>(c2[s], x[sd + 1], x[sd - 1], x[sd + sx], x[sd - sx],
                                                 DIM == 3 ? x[sd + sxy] : T(0),
                                                 DIM == 3 ? x[sd - sxy] : T(0));
                    x[sd] = (V.b[sd] + nb) / d2[s];
                }
            }
            tail_warps_sync(nw);
        }
}

// One block.  Levels lv[0 .. nlev-2] go down (forward sweep, restriction),
// lv[nlev-1] is solved, then back up (prolongation + even colour, odd colour).
template <int DIM, class T>
__global__ void __launch_bounds__(tail_threads<T>()) k_tail(const __grid_constant__ TailArgs<T> A,
                                                            const int* __restrict__ done) {
    pdl_entry();
    if (done && *done) return;
    extern __shared__ __align__(16) unsigned char tail_smem[];
    T* sm = reinterpret_cast<T*>(tail_smem);
    for (int q = threadIdx.x; q < A.smem_elems; q += blockDim.x) sm[q] = T(0);
    __syncthreads();
    const int top = A.nlev - 1;
    {  // the first level's b
        const TailLevel<T>& L = A.lv[0];
        const int n = tail_ncell<DIM>(L.g);
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
            int i, j, k;
            tail_ijk<DIM>(L, c, i, j, k);
            sm[L.bs + i + j * L.csx + k * L.csxy] = __ldg(L.b + cidx(L.g, i, j, k));
        }
    }
    __syncthreads();
    auto view = [&](int q) { return TailView<DIM, T>{A.lv[q], sm + A.lv[q].xs, sm + A.lv[q].bs}; };
    for (int q = 0; q < top; ++q) {
        tail_fwd(view(q));
        __syncthreads();
        tail_res(view(q), view(q + 1));
        __syncthreads();
    }
    tail_coarsest(view(top));
    __syncthreads();
    for (int q = top - 1; q >= 0; --q) {
        tail_up_even(view(q), view(q + 1));
        __syncthreads();
        tail_up_odd(view(q));
        __syncthreads();
    }
    {  // the first level's x out
        const TailLevel<T>& L = A.lv[0];
        const int n = tail_ncell<DIM>(L.g);
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
            int i, j, k;
            tail_ijk<DIM>(L, c, i, j, k);
            L.x[cidx(L.g, i, j, k)] = sm[L.xs + i + j * L.csx + k * L.csxy];
        }
    }
}

}  // namespace
}  // namespace uaamg
