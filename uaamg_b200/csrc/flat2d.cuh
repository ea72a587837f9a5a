// The V-cycle levels of a 2D problem as flat walks over the level (no TMA ring): the
// four z marches of march.cuh -- forward sweep from x = 0, residual + restriction,
// prolongation + even colour, odd colour (+ the CG's z sums on the finest level) --
// for a level that is a single plane, where a march has nothing to pipeline.  Each
// kernel walks items (vertical cell pairs (i, j), (i, j+1) with j odd, or coarse
// cells) grid-stride, a warp over 32 consecutive columns, and issues every load of an
// item before using any.  The per-item arithmetic is the march's, operand for
// operand and in its order (march.cuh presmooth, mcoup, nbsum, mdiag, fp32_ax, the
// restriction's (di, dj) sum): on the finest level the couplings are 1/h^2 and the
// diagonal comes from the cell code's neighbour bits; a coarse level reads its
// diagonal dg and its +x / +y couplings (FP16 face counts times the finest 1/h^2 in
// the mixed form).  It is written as __host__ __device__ functions so that a host
// build of the same code can be checked against the oracle stage by stage; the FP64
// instantiation compiled with -fmad=false reproduces the reference bit for bit.
//
// Bounds: an item's reads stay in the padded level -- rows j-1 .. j+2 (the row above
// the pair is clamped to j+1 when j = ny, whose row j+1 is the ghost row), columns
// i-1 .. i+1, and for the prolongation the parents ((i+1)/2, (j+1)/2) of those
// cells, at most (nx+2)/2 = cnx+1 and cny+1 (the coarse ghost ring).
#pragma once
#include <cuda_fp16.h>

#include <cstdint>
#include <type_traits>

#include "march.cuh"

namespace uaamg {
namespace {

// A level's operator as the flat walks read it: unused on the finest level; on a
// coarse level the diagonal and the couplings towards +x and +y (the -x / -y ones are
// the neighbours' +x / +y), as the marches read them.
template <class T, class CS>
struct F2Op {
    const T* dg;
    const CS* cx;
    const CS* cy;
};

// num / d as the march's mdiv: the fast reciprocal in the mixed form (couplings
// stored in FP16), IEEE division otherwise.  The host copy divides exactly and is
// used for the FP64 and FP32 forms only.
template <class T, class CS>
__host__ __device__ __forceinline__ T f2_div(T num, T d) {
#ifdef __CUDA_ARCH__
    if constexpr (!std::is_same<CS, T>::value) return __fdividef(num, d);
    else return num / d;
#else
    return num / d;
#endif
}

// A stored coupling as T (march.cuh coupling): FP16 values are face counts times cs.
template <class T, class CS>
__host__ __device__ __forceinline__ T f2_coupling(CS v, T cs) {
    if constexpr (std::is_same<CS, T>::value) return v;
    else return (T)__half2float(v) * cs;
}

// Diagonal of cell id with code c at (i, j): on the finest level the march's table
// entry (summed in the reference's order +x, -x, +y, -y) plus the Dirichlet wall
// share; on a coarse level the stored diagonal.
template <class T, class CS, bool FINE>
__host__ __device__ __forceinline__ T f2_diag(const MLevel<T>& L, const F2Op<T, CS>& op, uint32_t c,
                                              int id, int i, int j) {
    if constexpr (FINE) {
        T d = ((c & 1u) ? L.idx2 : T(0)) + ((c & 2u) ? L.idx2 : T(0)) + ((c & 4u) ? L.idy2 : T(0)) +
              ((c & 8u) ? L.idy2 : T(0));
        if (L.dirichlet) {
            T w = T(0);
            if (i == 1) w += T(2) * L.idx2;
            if (i == L.g.nx) w += T(2) * L.idx2;
            if (j == 1) w += T(2) * L.idy2;
            if (j == L.g.ny) w += T(2) * L.idy2;
            d = d + w;
        }
        return d;
    } else {
        return op.dg[id];
    }
}

// Couplings of cell id in the reference's order +x, -x, +y, -y (march.cuh mcoup).
template <class T, class CS, bool FINE>
__host__ __device__ __forceinline__ void f2_coup(const MLevel<T>& L, const F2Op<T, CS>& op, int id,
                                                 T (&k)[4]) {
    if constexpr (FINE) {
        k[0] = k[1] = L.idx2;
        k[2] = k[3] = L.idy2;
    } else {
        k[0] = f2_coupling<T, CS>(op.cx[id], L.csx);
        k[1] = f2_coupling<T, CS>(op.cx[id - 1], L.csx);
        k[2] = f2_coupling<T, CS>(op.cy[id], L.csy);
        k[3] = f2_coupling<T, CS>(op.cy[id - L.g.sx], L.csy);
    }
}

// sum c_n v_n in the reference's order (march.cuh nbsum).
template <class T>
__host__ __device__ __forceinline__ T f2_nb(const T (&k)[4], T vr, T vl, T vt, T vb) {
    return k[0] * vr + k[1] * vl + k[2] * vt + k[3] * vb;
}

// Pre-smoothed value of cell id from x = 0: (b + 0)/d for an active odd cell (0 when
// d < 1e-30), 0 for every other cell.
template <class T, class CS, bool FINE>
__host__ __device__ __forceinline__ T f2_pre(const MLevel<T>& L, const F2Op<T, CS>& op, uint32_t c,
                                             T b, int id, int i, int j) {
    if ((c & (kActive | kOdd)) != (kActive | kOdd)) return T(0);
    const T d = f2_diag<T, CS, FINE>(L, op, c, id, i, j);
    if (d < T(1e-30)) return T(0);
    return f2_div<T, CS>(b + T(0), d);
}

// A x of an active cell: the reference's expression in FP64; in FP32 the sum of
// couplings times differences (march.cuh fp32_ax; on the finest level a term exists
// where the code bit says the coupling does).
template <class T, bool FINE>
__host__ __device__ __forceinline__ T f2_ax(const MLevel<T>& L, uint32_t c, T d, const T (&k)[4],
                                            T x, T xr, T xl, T xt, T xb) {
    if constexpr (sizeof(T) == 8) {
        return d * x - k[0] * xr - k[1] * xl - k[2] * xt - k[3] * xb;
    } else if constexpr (FINE) {
        const T tx = ((c & 1u) ? x - xr : T(0)) + ((c & 2u) ? x - xl : T(0));
        const T ty = ((c & 4u) ? x - xt : T(0)) + ((c & 8u) ? x - xb : T(0));
        const T ax = tx * L.idx2 + ty * L.idy2;
        const T sum = ((c & 1u) ? L.idx2 : T(0)) + ((c & 2u) ? L.idx2 : T(0)) +
                      ((c & 4u) ? L.idy2 : T(0)) + ((c & 8u) ? L.idy2 : T(0));
        return ax + (d - sum) * x;
    } else {
        const T ax = k[0] * (x - xr) + k[1] * (x - xl) + k[2] * (x - xt) + k[3] * (x - xb);
        const T sum = k[0] + k[1] + k[2] + k[3];
        return ax + (d - sum) * x;
    }
}

// The eight cells an item of a pair reads: 0 below A, 1 A = (i, j), 2 B = (i, j+1),
// 3 above B (B again when j = ny), 4 / 5 left / right of A, 6 / 7 left / right of B.
struct F2Pair {
    int id;          // A's index
    bool hb;         // B is an interior cell
    int off[8];      // index offsets from A
    int di[8], dj[8];
};

__host__ __device__ __forceinline__ F2Pair f2_pair(const Geom& g, int i, int j) {
    F2Pair p;
    const int sx = g.sx;
    p.id = i + j * sx;
    p.hb = j < g.ny;
    const int s2 = p.hb ? 2 * sx : sx;
    const int off[8] = {-sx, 0, sx, s2, -1, 1, sx - 1, sx + 1};
    const int di[8] = {0, 0, 0, 0, -1, 1, -1, 1};
    const int dj[8] = {-1, 0, 1, p.hb ? 2 : 1, 0, 0, 1, 1};
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        p.off[e] = off[e];
        p.di[e] = di[e];
        p.dj[e] = dj[e];
    }
    return p;
}

// Every thread owns one cell of each colour (A and B have opposite colours), so a
// warp never splits on the red-black parity: the even cell of the pair is B when A
// is odd ((i + j) odd), else A, and its four neighbours are odd.  Their slots among
// the eight, selected by ao = "A is odd": +x 7 / 5, -x 6 / 4, +y 3 / 2, -y 1 / 0; the
// pair's odd cell is the even cell's -y neighbour (A) or its +y neighbour (B).
template <class V>
__host__ __device__ __forceinline__ void f2_pick(bool ao, const V (&v)[8], V& r, V& l, V& t,
                                                 V& b) {
    r = ao ? v[7] : v[5];
    l = ao ? v[6] : v[4];
    t = ao ? v[3] : v[2];
    b = ao ? v[1] : v[0];
}

// Forward sweep from x = 0 of one pair (k_fwd_smooth): the odd cell gets its
// pre-smoothed value, the even cell (b + sum c_n x_n)/d from its odd neighbours'
// pre-smoothed values (0 when inactive or d < 1e-30); x written on both cells.
template <class T, class CS, bool FINE>
__host__ __device__ __forceinline__ void f2_fwd_pair(const MLevel<T>& L, const F2Op<T, CS>& op,
                                                     const uint8_t* code, const T* b, T* x, int i,
                                                     int j) {
    const F2Pair p = f2_pair(L.g, i, j);
    const bool ao = ((i + j) & 1) != 0;
    uint32_t cc[8];
    T bb[8];
    int id[8], ci[8], cj[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        id[e] = p.id + p.off[e];
        ci[e] = i + p.di[e];
        cj[e] = j + p.dj[e];
        cc[e] = code[id[e]];
        bb[e] = b[id[e]];
    }
    uint32_t cr, cl, ct, cb;
    T br, bl, bt, bbm;
    int dr, dl, dt, db, ir, il, it, ib, jr, jl, jt, jb;
    f2_pick(ao, cc, cr, cl, ct, cb);
    f2_pick(ao, bb, br, bl, bt, bbm);
    f2_pick(ao, id, dr, dl, dt, db);
    f2_pick(ao, ci, ir, il, it, ib);
    f2_pick(ao, cj, jr, jl, jt, jb);
    const int ie = ao ? id[2] : id[1];  // the even cell
    T k[4];
    f2_coup<T, CS, FINE>(L, op, ie, k);
    const T pr = f2_pre<T, CS, FINE>(L, op, cr, br, dr, ir, jr);
    const T pl = f2_pre<T, CS, FINE>(L, op, cl, bl, dl, il, jl);
    const T pt = f2_pre<T, CS, FINE>(L, op, ct, bt, dt, it, jt);
    const T pb = f2_pre<T, CS, FINE>(L, op, cb, bbm, db, ib, jb);
    const T vo = ao ? pb : pt;  // the pair's odd cell
    const uint32_t ce = ao ? cc[2] : cc[1];
    T ve = T(0);
    if (ce & kActive) {
        const T d = f2_diag<T, CS, FINE>(L, op, ce, ie, i, ao ? j + 1 : j);
        if (!(d < T(1e-30))) ve = f2_div<T, CS>((ao ? bb[2] : bb[1]) + f2_nb(k, pr, pl, pt, pb), d);
    }
    x[p.id] = ao ? vo : ve;
    if (p.hb) x[p.id + L.g.sx] = ao ? ve : vo;
}

// Residual b - A x of the four children of coarse cell (ic, jc) and their sum in the
// reference's (di, dj) order (k_restrict_res); 0 for an inactive coarse cell.
template <class T, class CS, bool FINE>
__host__ __device__ __forceinline__ void f2_res_cell(const MLevel<T>& L, const F2Op<T, CS>& op,
                                                     const uint8_t* code, const T* b, const T* x,
                                                     const uint8_t* ccode, T* cb, int ic, int jc) {
    const int sx = L.g.sx;
    const int i0 = 2 * ic - 1, j0 = 2 * jc - 1;
    const int id0 = i0 + j0 * sx;
    // x on rows j0-1 .. j0+2 and columns i0-1 .. i0+2 (the corners unused)
    T xv[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q)
            xv[r][q] = ((r == 0 || r == 3) && (q == 0 || q == 3)) ? T(0)
                                                                  : x[id0 + (r - 1) * sx + (q - 1)];
    uint32_t c[2][2];
    T bv[2][2], k[2][2][4], dv[2][2];
#pragma unroll
    for (int di = 0; di < 2; ++di)
#pragma unroll
        for (int dj = 0; dj < 2; ++dj) {
            const int id = id0 + di + dj * sx;
            c[di][dj] = code[id];
            bv[di][dj] = b[id];
            f2_coup<T, CS, FINE>(L, op, id, k[di][dj]);
            dv[di][dj] = f2_diag<T, CS, FINE>(L, op, c[di][dj], id, i0 + di, j0 + dj);
        }
    const uint32_t cc = ccode[ic + jc * L.cg.sx];
    T rv[2][2];
#pragma unroll
    for (int di = 0; di < 2; ++di)
#pragma unroll
        for (int dj = 0; dj < 2; ++dj) {
            rv[di][dj] = T(0);
            if (c[di][dj] & kActive) {
                const int r = 1 + dj, q = 1 + di;
                rv[di][dj] = bv[di][dj] - f2_ax<T, FINE>(L, c[di][dj], dv[di][dj], k[di][dj], xv[r][q],
                                                         xv[r][q + 1], xv[r][q - 1], xv[r + 1][q],
                                                         xv[r - 1][q]);
            }
        }
    T s = T(0);
    s += rv[0][0];
    s += rv[0][1];
    s += rv[1][0];
    s += rv[1][1];
    cb[ic + jc * L.cg.sx] = (cc & kActive) ? s : T(0);
}

// Prolongation and the even colour of the reverse sweep for one pair (k_up_even):
// an active odd cell holds its pre-smoothed value plus 2 x_parent, the even cell
// (b + sum c_n x_n)/d from those (0 + 2 x_parent when d < 1e-30); inactive cells 0.
template <class T, class CS, bool FINE>
__host__ __device__ __forceinline__ void f2_upe_pair(const MLevel<T>& L, const F2Op<T, CS>& op,
                                                     const uint8_t* code, const T* b, const T* xc,
                                                     T* x, int i, int j) {
    const F2Pair p = f2_pair(L.g, i, j);
    const int csx = L.cg.sx;
    const bool ao = ((i + j) & 1) != 0;
    uint32_t cc[8];
    T bb[8], xp[8];
    int id[8], ci[8], cj[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        id[e] = p.id + p.off[e];
        ci[e] = i + p.di[e];
        cj[e] = j + p.dj[e];
        cc[e] = code[id[e]];
        bb[e] = b[id[e]];
        xp[e] = xc[((ci[e] + 1) >> 1) + ((cj[e] + 1) >> 1) * csx];
    }
    // odd value of a cell: pre-smoothed + prolongation when active and odd, else 0
    auto oddval = [&](uint32_t c, T bv, T xpv, int cid, int ii, int jj) -> T {
        if ((c & (kActive | kOdd)) != (kActive | kOdd)) return T(0);
        const T d = f2_diag<T, CS, FINE>(L, op, c, cid, ii, jj);
        const T pre = d < T(1e-30) ? T(0) : f2_div<T, CS>(bv + T(0), d);
        return pre + T(2) * xpv;
    };
    uint32_t cr, cl, ct, cb;
    T br, bl, bt, bbm, xr, xl, xt, xbm;
    int dr, dl, dt, db, ir, il, it, ib, jr, jl, jt, jb;
    f2_pick(ao, cc, cr, cl, ct, cb);
    f2_pick(ao, bb, br, bl, bt, bbm);
    f2_pick(ao, xp, xr, xl, xt, xbm);
    f2_pick(ao, id, dr, dl, dt, db);
    f2_pick(ao, ci, ir, il, it, ib);
    f2_pick(ao, cj, jr, jl, jt, jb);
    const int ie = ao ? id[2] : id[1];  // the even cell
    T k[4];
    f2_coup<T, CS, FINE>(L, op, ie, k);
    const T orr = oddval(cr, br, xr, dr, ir, jr), ol = oddval(cl, bl, xl, dl, il, jl);
    const T ot = oddval(ct, bt, xt, dt, it, jt), ob = oddval(cb, bbm, xbm, db, ib, jb);
    const T vo = ao ? ob : ot;  // the pair's odd cell
    const uint32_t ce = ao ? cc[2] : cc[1];
    T ve = T(0);
    if (ce & kActive) {
        const T d = f2_diag<T, CS, FINE>(L, op, ce, ie, i, ao ? j + 1 : j);
        if (d < T(1e-30))
            ve = T(0) + T(2) * (ao ? xp[2] : xp[1]);
        else
            ve = f2_div<T, CS>((ao ? bb[2] : bb[1]) + f2_nb(k, orr, ol, ot, ob), d);
    }
    x[p.id] = ao ? vo : ve;
    if (p.hb) x[p.id + L.g.sx] = ao ? ve : vo;
}

// The odd colour of the reverse sweep for one pair, in place (k_up_odd): the odd cell
// reads only even neighbours, which nothing writes here.  With zdot (finest level),
// the fluid sums of z (the cells' new x), r z and r (r = b) are added to acc.
template <class T, class CS, bool FINE, bool ZDOT>
__host__ __device__ __forceinline__ void f2_upo_pair(const MLevel<T>& L, const F2Op<T, CS>& op,
                                                     const uint8_t* code, const T* b, T* x, int i,
                                                     int j, double (&acc)[3]) {
    const F2Pair p = f2_pair(L.g, i, j);
    T xx[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) xx[e] = x[p.id + p.off[e]];
    const uint32_t ca = code[p.id], cb = code[p.id + L.g.sx];
    const T ba = b[p.id], bb = b[p.id + L.g.sx];
    // the odd cell (A when i + j is odd) and its neighbours, selected without
    // run-time indexing so that everything stays in registers
    const bool ao = ((i + j) & 1) != 0;
    const int io = ao ? p.id : p.id + L.g.sx;
    const uint32_t co = ao ? ca : cb;
    const T bo = ao ? ba : bb;
    const T vr = ao ? xx[5] : xx[7], vl = ao ? xx[4] : xx[6];
    const T vt = ao ? xx[2] : xx[3], vb = ao ? xx[0] : xx[1];
    T za = xx[1], zb = xx[2];
    if ((ao || p.hb) && (co & kActive)) {
        T k[4];
        f2_coup<T, CS, FINE>(L, op, io, k);
        const T d = f2_diag<T, CS, FINE>(L, op, co, io, i, ao ? j : j + 1);
        if (!(d < T(1e-30))) {
            const T v = f2_div<T, CS>(bo + f2_nb(k, vr, vl, vt, vb), d);
            x[io] = v;
            if (ao) za = v;
            else zb = v;
        }
    }
    if (ZDOT) {
        if (ca & kActive) {
            const double zv = (double)za, rv = (double)ba;
            acc[0] += zv;
            acc[1] += rv * zv;
            acc[2] += rv;
        }
        if ((cb & kActive) && p.hb) {
            const double zv = (double)zb, rv = (double)bb;
            acc[0] += zv;
            acc[1] += rv * zv;
            acc[2] += rv;
        }
    }
}

// ---- kernels: grid-stride walks over the items, (32, 8) blocks -------------------

// Item `it` of a walk over rows of 32 items: (row, column).
__device__ __forceinline__ void f2_item(long long it, int ncol, int& row, int& col) {
    row = (int)(it / ncol);
    col = (int)(it - (long long)row * ncol);
}

template <class T, class CS, bool FINE>
__global__ void __launch_bounds__(256, 2) k_fwd_flat2d(MLevel<T> L, F2Op<T, CS> op,
                                                    const uint8_t* __restrict__ code,
                                                    const T* __restrict__ b, T* __restrict__ x,
                                                    const int* __restrict__ done) {
    pdl_entry();
    if (done && *done) return;
    const int nxc = (L.g.nx + 31) >> 5;
    const long long n = (long long)((L.g.ny + 1) >> 1) * nxc;
    for (long long it = (long long)blockIdx.x * blockDim.y + threadIdx.y; it < n;
         it += (long long)gridDim.x * blockDim.y) {
        int pr, ch;
        f2_item(it, nxc, pr, ch);
        const int i = 1 + (ch << 5) + (int)threadIdx.x;
        if (i <= L.g.nx) f2_fwd_pair<T, CS, FINE>(L, op, code, b, x, i, 1 + 2 * pr);
    }
}

template <class T, class CS, bool FINE>
__global__ void __launch_bounds__(256) k_res_flat2d(MLevel<T> L, F2Op<T, CS> op,
                                                    const uint8_t* __restrict__ code,
                                                    const T* __restrict__ b,
                                                    const T* __restrict__ x,
                                                    const uint8_t* __restrict__ ccode,
                                                    T* __restrict__ cb, const int* __restrict__ done) {
    pdl_entry();
    if (done && *done) return;
    const int ncx = (L.cg.nx + 31) >> 5;
    const long long n = (long long)L.cg.ny * ncx;
    for (long long it = (long long)blockIdx.x * blockDim.y + threadIdx.y; it < n;
         it += (long long)gridDim.x * blockDim.y) {
        int row, ch;
        f2_item(it, ncx, row, ch);
        const int ic = 1 + (ch << 5) + (int)threadIdx.x;
        if (ic <= L.cg.nx) f2_res_cell<T, CS, FINE>(L, op, code, b, x, ccode, cb, ic, 1 + row);
    }
}

template <class T, class CS, bool FINE>
__global__ void __launch_bounds__(256, 2) k_upe_flat2d(MLevel<T> L, F2Op<T, CS> op,
                                                    const uint8_t* __restrict__ code,
                                                    const T* __restrict__ b,
                                                    const T* __restrict__ xc, T* __restrict__ x,
                                                    const int* __restrict__ done) {
    pdl_entry();
    if (done && *done) return;
    const int nxc = (L.g.nx + 31) >> 5;
    const long long n = (long long)((L.g.ny + 1) >> 1) * nxc;
    for (long long it = (long long)blockIdx.x * blockDim.y + threadIdx.y; it < n;
         it += (long long)gridDim.x * blockDim.y) {
        int pr, ch;
        f2_item(it, nxc, pr, ch);
        const int i = 1 + (ch << 5) + (int)threadIdx.x;
        if (i <= L.g.nx) f2_upe_pair<T, CS, FINE>(L, op, code, b, xc, x, i, 1 + 2 * pr);
    }
}

// x is read and written in place (odd cells from even neighbours): not restrict.
template <class T, class CS, bool FINE, bool ZDOT>
__global__ void __launch_bounds__(256) k_upo_flat2d(MLevel<T> L, F2Op<T, CS> op,
                                                    const uint8_t* __restrict__ code,
                                                    const T* __restrict__ b, T* x,
                                                    const int* __restrict__ done, double* partials,
                                                    CGState* cg) {
    pdl_entry();
    if (done && *done) return;
    double acc[3] = {0.0, 0.0, 0.0};
    const int nxc = (L.g.nx + 31) >> 5;
    const long long n = (long long)((L.g.ny + 1) >> 1) * nxc;
    for (long long it = (long long)blockIdx.x * blockDim.y + threadIdx.y; it < n;
         it += (long long)gridDim.x * blockDim.y) {
        int pr, ch;
        f2_item(it, nxc, pr, ch);
        const int i = 1 + (ch << 5) + (int)threadIdx.x;
        if (i <= L.g.nx) f2_upo_pair<T, CS, FINE, ZDOT>(L, op, code, b, x, i, 1 + 2 * pr, acc);
    }
    if (ZDOT) {
        double tot[3];
        if (reduce_last<3>(acc, partials, &cg->counter[2], tot)) finish_zdot(cg, tot);
    }
}

}  // namespace
}  // namespace uaamg
