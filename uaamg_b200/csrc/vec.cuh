// CG vector kernels over whole padded arrays, layout conversions between the
// caller's layout and the pitched one, and the per-level set-up of cell codes and
// coarse diagonals.
#pragma once
#include "march.cuh"

namespace uaamg {
namespace {

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

// Mixed mode: x_hi += x_lo, x_lo = 0 on one vector of x_lo (its N cells).
template <class T>
__device__ __forceinline__ void vfold(typename Vec16<T>::V& x, double* xhi, long long t);
template <>
__device__ __forceinline__ void vfold<float>(float4& x, double* xhi, long long t) {
    double2* h = reinterpret_cast<double2*>(xhi) + 2 * t;
    double2 a = h[0], b = h[1];
    a.x += (double)x.x; a.y += (double)x.y; b.x += (double)x.z; b.y += (double)x.w;
    h[0] = a;
    h[1] = b;
    x = make_float4(0.f, 0.f, 0.f, 0.f);
}
template <>
__device__ __forceinline__ void vfold<double>(double2& x, double* xhi, long long t) {
    double2* h = reinterpret_cast<double2*>(xhi) + t;
    double2 a = *h;
    a.x += x.x; a.y += x.y;
    *h = a;
    x = make_double2(0.0, 0.0);
}

// In mixed mode (xhi given) a residual replacement in the previous iteration left
// cg->fold set: x_lo is first folded into the FP64 x_hi (the value x_hi + x_lo the
// replacement's residual was computed from) and restarts at 0.  Mixed mode also
// stops at max_iter here unless a convergence candidate awaits its confirmation
// (the residual replacement that follows stops it otherwise).
template <class T>
__global__ void __launch_bounds__(256) k_update_flat(long long nvec, T* x, T* r,
                                                     const T* __restrict__ p,
                                                     const T* __restrict__ ap, double* xhi,
                                                     double* partials, CGState* cg, double* hist) {
    pdl_entry();
    if (cg->done) return;
    using V = typename Vec16<T>::V;
    const T alpha = (T)cg->alpha;
    const bool fold = xhi && cg->fold;
    V* xv = reinterpret_cast<V*>(x);
    V* rv = reinterpret_cast<V*>(r);
    const V* pv = reinterpret_cast<const V*>(p);
    const V* av = reinterpret_cast<const V*>(ap);
    double acc[1] = {0.0};
    const long long stride = (long long)gridDim.x * blockDim.x;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (fold) {  // after a replacement (one iteration in replace_every): one vector a trip
        for (; t < nvec; t += stride) {
            V xx = xv[t], rr_ = rv[t];
            const V pp = __ldg(&pv[t]), aa = __ldg(&av[t]);
            vfold<T>(xx, xhi, t);
            vaxpy_rr<T>(xx, rr_, pp, aa, alpha, acc[0]);
            xv[t] = xx;
            rv[t] = rr_;
        }
    } else {  // two vectors a thread per trip, their loads issued together
        for (; t + stride < nvec; t += 2 * stride) {
            const long long t2 = t + stride;
            V xx = xv[t], rr_ = rv[t], x2 = xv[t2], r2 = rv[t2];
            const V pp = __ldg(&pv[t]), aa = __ldg(&av[t]), p2 = __ldg(&pv[t2]), a2 = __ldg(&av[t2]);
            vaxpy_rr<T>(xx, rr_, pp, aa, alpha, acc[0]);
            vaxpy_rr<T>(x2, r2, p2, a2, alpha, acc[0]);
            xv[t] = xx;
            rv[t] = rr_;
            xv[t2] = x2;
            rv[t2] = r2;
        }
        if (t < nvec) {
            V xx = xv[t], rr_ = rv[t];
            const V pp = __ldg(&pv[t]), aa = __ldg(&av[t]);
            vaxpy_rr<T>(xx, rr_, pp, aa, alpha, acc[0]);
            xv[t] = xx;
            rv[t] = rr_;
        }
    }
    double tot[1];
    if (reduce_last<1>(acc, partials, &cg->counter[1], tot)) {
        if (fold) cg->fold = 0;  // every other block has finished its loop
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
        if (cg->replace_every > 0 && !cg->done && cg->iter >= cg->max_iter && !cg->cand) {
            cg->status = CG_MAXITER;
            cg->done = 1;
        }
    }
}

// Layout conversions between the reference's layout (gr) and the pitched one (g).
template <int DIM, class T>
__global__ void k_import(Geom g, Geom gr, const double* __restrict__ src, T* dst) {
    pdl_entry();
    for_cells<DIM>(g, [&](int i, int j, int k, int id) { dst[id] = (T)src[cidx(gr, i, j, k)]; });
}
template <int DIM>
__global__ void k_import_mask(Geom g, Geom gr, const uint8_t* __restrict__ src, uint8_t* dst) {
    pdl_entry();
    for_cells<DIM>(g, [&](int i, int j, int k, int id) {
        dst[id] = src[cidx(gr, i, j, k)] ? 1 : 0;
    });
}
// The solution x = x_hi + x_lo (either part may be absent) into the reference
// layout: dst = x (overwrite) or dst += x (accumulate), interior cells.
template <int DIM, class T>
__global__ void k_export_x(Geom g, Geom gr, const double* __restrict__ xhi, const T* __restrict__ xlo,
                           double* dst, int accumulate) {
    pdl_entry();
    for_cells<DIM>(g, [&](int i, int j, int k, int id) {
        const double x = xhi && xlo ? xhi[id] + (double)xlo[id] : (xhi ? xhi[id] : (double)xlo[id]);
        const int rid = cidx(gr, i, j, k);
        dst[rid] = accumulate ? dst[rid] + x : x;
    });
}
// dst (reference layout) = src on interior cells (overwrite) or += src (accumulate).
template <int DIM, class T>
__global__ void k_export(Geom g, Geom gr, const T* __restrict__ src, double* dst, int accumulate) {
    pdl_entry();
    for_cells<DIM>(g, [&](int i, int j, int k, int id) {
        const int rid = cidx(gr, i, j, k);
        dst[rid] = accumulate ? dst[rid] + (double)src[id] : (double)src[id];
    });
}

// Cell codes of a level, one byte per cell: bit 6 the cell is an interior fluid
// cell, bit 7 its colour ((i+j+k) odd), and on the finest level (fine = 1) bits
// 0-5 whether its +x,-x,+y,-y,+z,-z neighbour is an interior fluid cell --
// exactly when the reference's coupling exists (uaamg_preconditioner_3d.cpp:50-66).
template <int DIM>
__global__ void k_codes(Geom g, const uint8_t* __restrict__ s, uint8_t* code, int fine) {
    pdl_entry();
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

// Diagonal of every fluid cell of a coarse level, in the reference's summation
// order (uaamg_preconditioner_3d.cpp:113-119), plus the Dirichlet wall channel.
template <int DIM, class T>
__global__ void k_diag(Geom g, const uint8_t* __restrict__ s, const T* __restrict__ cx,
                       const T* __restrict__ cy, const T* __restrict__ cz,
                       const T* __restrict__ wd, T* dg) {
    pdl_entry();
    for_cells<DIM>(g, [&](int, int, int, int id) {
        if (s[id]) return;
        T d = cx[id] + cx[id - 1] + cy[id] + cy[id - g.sx];
        if (DIM == 3) d = d + cz[id] + cz[id - g.sxy];
        if (wd) d = d + wd[id];
        dg[id] = d;
    });
}

// Couplings of a coarse level stored in FP16 as face counts: h = half(rint(c/cs))
// with cs the finest level's 1/h^2 along the axis, exact up to 2048 faces; the T
// coupling is replaced by its decoded value h * cs, so the diagonal (k_diag), the
// step-by-step V-cycle and the marches all use the same values.
__global__ void k_coupling_half(long long n, float* c, __half* h, float cs) {
    pdl_entry();
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const __half v = __float2half_rn(rintf(c[t] / cs));
        h[t] = v;
        c[t] = __half2float(v) * cs;
    }
}

}  // namespace
}  // namespace uaamg
