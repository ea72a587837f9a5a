// Host build of the per-item functions of uaamg_b200/csrc/flat2d.cuh (the flat 2D
// finest-level V-cycle steps), for tests/test_flat2d_host.py: each step walks every
// item on the CPU, so its arithmetic can be compared with the oracle's V-cycle stages
// without a GPU.  Arrays are padded in the reference layout (row pitch nx + 2);
// level 1 has cnx x cny cells.
#include <cstdint>

#include "flat2d.cuh"

namespace {

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

template <class T>
void fwd(const MLevel<T>& L, const uint8_t* code, const T* b, T* x) {
    for (int j = 1; j <= L.g.ny; j += 2)
        for (int i = 1; i <= L.g.nx; ++i) uaamg::f2_fwd_pair<T, T>(L, code, b, x, i, j);
}

template <class T>
void res(const MLevel<T>& L, const uint8_t* code, const T* b, const T* x, const uint8_t* ccode,
         T* cb) {
    for (int jc = 1; jc <= L.cg.ny; ++jc)
        for (int ic = 1; ic <= L.cg.nx; ++ic) uaamg::f2_res_cell<T>(L, code, b, x, ccode, cb, ic, jc);
}

template <class T>
void up(const MLevel<T>& L, const uint8_t* code, const T* b, const T* xc, T* x, double* sums) {
    for (int j = 1; j <= L.g.ny; j += 2)
        for (int i = 1; i <= L.g.nx; ++i) uaamg::f2_upe_pair<T, T>(L, code, b, xc, x, i, j);
    double acc[3] = {0.0, 0.0, 0.0};
    for (int j = 1; j <= L.g.ny; j += 2)
        for (int i = 1; i <= L.g.nx; ++i) uaamg::f2_upo_pair<T, T, true>(L, code, b, x, i, j, acc);
    for (int q = 0; q < 3; ++q) sums[q] = acc[q];
}

}  // namespace

extern "C" {

// Forward sweep from x = 0 (k_fwd_flat2d).
void f2h_fwd_f64(int nx, int ny, double dx, double dy, int dir, const uint8_t* code,
                 const double* b, double* x) {
    fwd<double>(level<double>(nx, ny, 1, 1, dx, dy, dir), code, b, x);
}
void f2h_fwd_f32(int nx, int ny, double dx, double dy, int dir, const uint8_t* code, const float* b,
                 float* x) {
    fwd<float>(level<float>(nx, ny, 1, 1, dx, dy, dir), code, b, x);
}

// Residual and restriction (k_res_flat2d) into the coarse b.
void f2h_res_f64(int nx, int ny, int cnx, int cny, double dx, double dy, int dir,
                 const uint8_t* code, const double* b, const double* x, const uint8_t* ccode,
                 double* cb) {
    res<double>(level<double>(nx, ny, cnx, cny, dx, dy, dir), code, b, x, ccode, cb);
}
void f2h_res_f32(int nx, int ny, int cnx, int cny, double dx, double dy, int dir,
                 const uint8_t* code, const float* b, const float* x, const uint8_t* ccode,
                 float* cb) {
    res<float>(level<float>(nx, ny, cnx, cny, dx, dy, dir), code, b, x, ccode, cb);
}

// Prolongation + even colour, then odd colour with the z sums (k_upe_flat2d,
// k_upo_flat2d): x from the coarse solution xc; sums = (sum z, sum r z, sum r).
void f2h_up_f64(int nx, int ny, int cnx, int cny, double dx, double dy, int dir,
                const uint8_t* code, const double* b, const double* xc, double* x, double* sums) {
    up<double>(level<double>(nx, ny, cnx, cny, dx, dy, dir), code, b, xc, x, sums);
}
void f2h_up_f32(int nx, int ny, int cnx, int cny, double dx, double dy, int dir,
                const uint8_t* code, const float* b, const float* xc, float* x, double* sums) {
    up<float>(level<float>(nx, ny, cnx, cny, dx, dy, dir), code, b, xc, x, sums);
}

}  // extern "C"
