// Host build of the per-item functions of uaamg_b200/csrc/flat2d.cuh (the flat 2D
// V-cycle steps), for tests/test_flat2d_host.py: each step walks every item on the
// CPU, so its arithmetic can be compared with the oracle's V-cycle stages without a
// GPU.  Arrays are padded in the reference layout (row pitch nx + 2); the next level
// has cnx x cny cells.  fine != 0: the finest level (couplings from the cell codes);
// fine == 0: a coarse level with diagonal dg and +x / +y couplings cx, cy.
#include <cstdint>

#include "flat2d.cuh"

namespace {

using uaamg::F2Op;
using uaamg::MLevel;

template <class T>
MLevel<T> level(int nx, int ny, int cnx, int cny, double dx, double dy, int dirichlet) {
    MLevel<T> L{};
    L.g.nx = nx;
    L.g.ny = ny;
    L.g.nz = 0;
    L.g.sx = nx + 2;
    L.g.sxy = (nx + 2) * (ny + 2);
    L.g.n = L.g.sxy;
    L.cg.nx = cnx;
    L.cg.ny = cny;
    L.cg.nz = 0;
    L.cg.sx = cnx + 2;
    L.cg.sxy = (cnx + 2) * (cny + 2);
    L.cg.n = L.cg.sxy;
    L.idx2 = (T)(1.0 / (dx * dx));
    L.idy2 = (T)(1.0 / (dy * dy));
    L.idz2 = T(0);
    L.csx = L.csy = L.csz = T(1);
    L.dirichlet = dirichlet;
    L.zc = 2;
    return L;
}

template <class T, class CS, bool FINE>
void run(int step, const MLevel<T>& L, const F2Op<T, CS>& op, const uint8_t* code, const T* b,
         T* x, const uint8_t* ccode, T* cb, const T* xc, double* sums) {
    if (step == 0) {
        for (int j = 1; j <= L.g.ny; j += 2)
            for (int i = 1; i <= L.g.nx; ++i)
                uaamg::f2_fwd_pair<T, CS, FINE>(L, op, code, b, x, i, j);
    } else if (step == 1) {
        for (int jc = 1; jc <= L.cg.ny; ++jc)
            for (int ic = 1; ic <= L.cg.nx; ++ic)
                uaamg::f2_res_cell<T, CS, FINE>(L, op, code, b, x, ccode, cb, ic, jc);
    } else {
        for (int j = 1; j <= L.g.ny; j += 2)
            for (int i = 1; i <= L.g.nx; ++i)
                uaamg::f2_upe_pair<T, CS, FINE>(L, op, code, b, xc, x, i, j);
        double acc[3] = {0.0, 0.0, 0.0};
        for (int j = 1; j <= L.g.ny; j += 2)
            for (int i = 1; i <= L.g.nx; ++i)
                uaamg::f2_upo_pair<T, CS, FINE, true>(L, op, code, b, x, i, j, acc);
        for (int q = 0; q < 3; ++q) sums[q] = acc[q];
    }
}

template <class T>
void step_t(int step, int fine, int nx, int ny, int cnx, int cny, double dx, double dy, int dir,
            const T* dg, const T* cx, const T* cy, const uint8_t* code, const T* b, T* x,
            const uint8_t* ccode, T* cb, const T* xc, double* sums) {
    const MLevel<T> L = level<T>(nx, ny, cnx, cny, dx, dy, dir);
    F2Op<T, T> op;
    op.dg = dg;
    op.cx = cx;
    op.cy = cy;
    if (fine) run<T, T, true>(step, L, op, code, b, x, ccode, cb, xc, sums);
    else run<T, T, false>(step, L, op, code, b, x, ccode, cb, xc, sums);
}

}  // namespace

extern "C" {

// step 0: forward sweep from x = 0 (k_fwd_flat2d), x out;
// step 1: residual + restriction (k_res_flat2d), the next level's b out;
// step 2: prolongation + even colour, then odd colour with the z sums (k_upe_flat2d,
//         k_upo_flat2d): x out from the next level's xc; sums = (sum z, sum r z, sum r).
void f2h_step_f64(int step, int fine, int nx, int ny, int cnx, int cny, double dx, double dy,
                  int dir, const double* dg, const double* cx, const double* cy,
                  const uint8_t* code, const double* b, double* x, const uint8_t* ccode,
                  double* cb, const double* xc, double* sums) {
    step_t<double>(step, fine, nx, ny, cnx, cny, dx, dy, dir, dg, cx, cy, code, b, x, ccode, cb,
                   xc, sums);
}
void f2h_step_f32(int step, int fine, int nx, int ny, int cnx, int cny, double dx, double dy,
                  int dir, const float* dg, const float* cx, const float* cy, const uint8_t* code,
                  const float* b, float* x, const uint8_t* ccode, float* cb, const float* xc,
                  double* sums) {
    step_t<float>(step, fine, nx, ny, cnx, cny, dx, dy, dir, dg, cx, cy, code, b, x, ccode, cb, xc,
                  sums);
}

// The mixed form's coarse level: FP32 values, couplings stored as FP16 face counts
// (hcx, hcy) decoded as count * cs (csx, csy: the finest level's 1/h^2 per axis).
void f2h_step_mixed(int step, int nx, int ny, int cnx, int cny, double csx, double csy,
                    const float* dg, const uint16_t* hcx, const uint16_t* hcy, const uint8_t* code,
                    const float* b, float* x, const uint8_t* ccode, float* cb, const float* xc,
                    double* sums) {
    MLevel<float> L = level<float>(nx, ny, cnx, cny, 1.0, 1.0, 0);
    L.csx = (float)csx;
    L.csy = (float)csy;
    F2Op<float, __half> op;
    op.dg = dg;
    op.cx = reinterpret_cast<const __half*>(hcx);
    op.cy = reinterpret_cast<const __half*>(hcy);
    run<float, __half, false>(step, L, op, code, b, x, ccode, cb, xc, sums);
}

}  // extern "C"
