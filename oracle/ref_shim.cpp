// Test infrastructure only: a C-ABI shim around the reference's own CPU solver
// classes, compiled together with the reference's unmodified source files by
// oracle/Makefile into oracle/_ref/libuaamg_ref.so.  Nothing in the product links
// this; tests, smoke() and the bench's CPU-baseline leg load it as the oracle.
//
// Reference classes driven here:
//   PCG / PCG3D                    src/solver/pcg.cpp:18-126, src/solver/pcg_3d.cpp:18-125
//   UAAMGPreconditioner[3D]        src/solver/preconditioner/uaamg_preconditioner.cpp:177-199,
//                                  src/solver/preconditioner/uaamg_preconditioner_3d.cpp:198-229
//   IdentityPreconditioner[3D]     include/solver/preconditioner/identity_preconditioner*.h
//   PressureProjection[3D]         src/pressure/pressure.cpp:5-33, src/pressure/pressure_3d.cpp:5-40
//   Grid / Grid3D                  include/core/grid.h:16-48, include/core/grid_3d.h:14-38
//   Grid::init_variable_lap        src/core/grid.cpp:12-17 (PCG::solve's lap_* branch)
//   SmoothCylinder                 src/geometry/cylinder_model.cpp:40-71
#include "core/grid.h"
#include "core/grid_3d.h"
#include "solver/pcg.h"
#include "solver/pcg_3d.h"
#include "solver/preconditioner/uaamg_preconditioner.h"
#include "solver/preconditioner/uaamg_preconditioner_3d.h"
#include "solver/preconditioner/identity_preconditioner.h"
#include "solver/preconditioner/identity_preconditioner_3d.h"
#include "pressure/pressure.h"
#include "pressure/pressure_3d.h"
#include "geometry/cylinder_model.h"

#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

namespace {

// Counts preconditioner applications so the caller can learn how many PCG
// iterations the reference ran (PCG::solve returns void).
template <class Base, class GridT>
class Counting : public Base {
public:
    Counting(std::unique_ptr<Base> inner, int* counter) : inner_(std::move(inner)), counter_(counter) {}
    void apply(const GridT& g, const std::vector<double>& r, std::vector<double>& z) override {
        if (counter_) ++*counter_;
        inner_->apply(g, r, z);
    }
    std::string name() const override { return inner_->name(); }
private:
    std::unique_ptr<Base> inner_;
    int* counter_;
};

Grid make2(int nx, int ny, double dx, double dy, const uint8_t* solid) {
    Grid g(nx, ny, nx * dx, ny * dy);
    g.dx = dx; g.dy = dy;  // exact spacing, no Lx/nx round trip
    const int n = g.p_size();
    if (solid) for (int c = 0; c < n; ++c) g.solid[c] = solid[c] != 0;
    return g;
}

Grid3D make3(int nx, int ny, int nz, double dx, double dy, double dz, const uint8_t* solid) {
    Grid3D g(nx, ny, nz, nx * dx, ny * dy, nz * dz);
    g.dx = dx; g.dy = dy; g.dz = dz;
    const int n = g.p_size();
    if (solid) for (int c = 0; c < n; ++c) g.solid[c] = solid[c] != 0;
    return g;
}

// Records the right-hand side a caller hands to solve() and leaves p untouched.
class CapturingSolver : public Solver {
public:
    explicit CapturingSolver(double* out) : out_(out) {}
    void solve(Grid&, const std::vector<double>& rhs, int, double) override {
        std::memcpy(out_, rhs.data(), sizeof(double) * rhs.size());
    }
    std::string name() const override { return "capture"; }
private:
    double* out_;
};

}  // namespace

extern "C" {

// One UAAMG V-cycle z = M^{-1} r on padded (nx+2)(ny+2) arrays.
void ref_vcycle_2d(int nx, int ny, double dx, double dy, const uint8_t* solid,
                   const double* r, double* z) {
    Grid g = make2(nx, ny, dx, dy, solid);
    const int n = g.p_size();
    std::vector<double> rv(r, r + n), zv(n, 0.0);
    UAAMGPreconditioner pc;
    pc.apply(g, rv, zv);
    std::memcpy(z, zv.data(), sizeof(double) * n);
}

void ref_vcycle_3d(int nx, int ny, int nz, double dx, double dy, double dz,
                   const uint8_t* solid, const double* r, double* z) {
    Grid3D g = make3(nx, ny, nz, dx, dy, dz, solid);
    const int n = g.p_size();
    std::vector<double> rv(r, r + n), zv(n, 0.0);
    UAAMGPreconditioner3D pc;
    pc.apply(g, rv, zv);
    std::memcpy(z, zv.data(), sizeof(double) * n);
}

// PCG(UAAMG) (precond=1) or PCG(Identity) (precond=0); p is in/out exactly like
// Grid::p in Solver::solve (callers zero it first).  Returns the number of
// preconditioner applications.
int ref_pcg_2d(int nx, int ny, double dx, double dy, const uint8_t* solid,
               const double* rhs, double* p, int max_iter, double tol, int precond) {
    Grid g = make2(nx, ny, dx, dy, solid);
    const int n = g.p_size();
    std::memcpy(g.p.data(), p, sizeof(double) * n);
    int applies = 0;
    std::unique_ptr<Preconditioner> inner;
    if (precond) inner = std::make_unique<UAAMGPreconditioner>();
    else         inner = std::make_unique<IdentityPreconditioner>();
    PCG solver(std::make_unique<Counting<Preconditioner, Grid>>(std::move(inner), &applies));
    std::vector<double> rv(rhs, rhs + n);
    solver.solve(g, rv, max_iter, tol);
    std::memcpy(p, g.p.data(), sizeof(double) * n);
    return applies;
}

// PCG(UAAMG) or PCG(Identity) on a grid whose variable-coefficient Laplacian is set
// (Grid::init_variable_lap, then the caller's padded lap_diag / lap_off_x / lap_off_y),
// so that PCG::solve takes its pcg.cpp:35-46 branch.
int ref_pcg_var_2d(int nx, int ny, double dx, double dy, const uint8_t* solid,
                   const double* lap_diag, const double* lap_off_x, const double* lap_off_y,
                   const double* rhs, double* p, int max_iter, double tol, int precond) {
    Grid g = make2(nx, ny, dx, dy, solid);
    const int n = g.p_size();
    g.init_variable_lap();
    std::memcpy(g.lap_diag.data(), lap_diag, sizeof(double) * n);
    std::memcpy(g.lap_off_x.data(), lap_off_x, sizeof(double) * n);
    std::memcpy(g.lap_off_y.data(), lap_off_y, sizeof(double) * n);
    std::memcpy(g.p.data(), p, sizeof(double) * n);
    int applies = 0;
    std::unique_ptr<Preconditioner> inner;
    if (precond) inner = std::make_unique<UAAMGPreconditioner>();
    else         inner = std::make_unique<IdentityPreconditioner>();
    PCG solver(std::make_unique<Counting<Preconditioner, Grid>>(std::move(inner), &applies));
    std::vector<double> rv(rhs, rhs + n);
    solver.solve(g, rv, max_iter, tol);
    std::memcpy(p, g.p.data(), sizeof(double) * n);
    return applies;
}

// SmoothCylinder(cx, cy, R, dx, dy, tw)::applyToLaplacian on a grid with the given
// mask: solid (in/out, OR-ed by the model) and the three padded coefficient arrays
// (out; zero where the model leaves them).
void ref_smooth_cylinder_2d(int nx, int ny, double dx, double dy, double cx, double cy, double R,
                            double tw, uint8_t* solid, double* diag, double* ox, double* oy) {
    Grid g = make2(nx, ny, dx, dy, solid);
    const int n = g.p_size();
    g.init_variable_lap();
    SmoothCylinder cyl(cx, cy, R, dx, dy, tw);
    cyl.applyToLaplacian(g, g.lap_diag, g.lap_off_x, g.lap_off_y);
    for (int c = 0; c < n; ++c) solid[c] = g.solid[c] ? 1 : 0;
    std::memcpy(diag, g.lap_diag.data(), sizeof(double) * n);
    std::memcpy(ox, g.lap_off_x.data(), sizeof(double) * n);
    std::memcpy(oy, g.lap_off_y.data(), sizeof(double) * n);
}

int ref_pcg_3d(int nx, int ny, int nz, double dx, double dy, double dz, const uint8_t* solid,
               const double* rhs, double* p, int max_iter, double tol, int precond) {
    Grid3D g = make3(nx, ny, nz, dx, dy, dz, solid);
    const int n = g.p_size();
    std::memcpy(g.p.data(), p, sizeof(double) * n);
    int applies = 0;
    std::unique_ptr<Preconditioner3D> inner;
    if (precond) inner = std::make_unique<UAAMGPreconditioner3D>();
    else         inner = std::make_unique<IdentityPreconditioner3D>();
    PCG3D solver(std::make_unique<Counting<Preconditioner3D, Grid3D>>(std::move(inner), &applies));
    std::vector<double> rv(rhs, rhs + n);
    solver.solve(g, rv, max_iter, tol);
    std::memcpy(p, g.p.data(), sizeof(double) * n);
    return applies;
}

// PressureProjection::project with PCG(UAAMG): u (nx+1)(ny+2), v (nx+2)(ny+1)
// are corrected in place; p (padded) receives the pressure.
int ref_project_2d(int nx, int ny, double dx, double dy, const uint8_t* solid,
                   double* u, double* v, double dt, int max_iter, double tol, double* p) {
    Grid g = make2(nx, ny, dx, dy, solid);
    std::memcpy(g.u.data(), u, sizeof(double) * g.u_size());
    std::memcpy(g.v.data(), v, sizeof(double) * g.v_size());
    int applies = 0;
    PCG solver(std::make_unique<Counting<Preconditioner, Grid>>(
        std::make_unique<UAAMGPreconditioner>(), &applies));
    PressureProjection::project(g, dt, solver, max_iter, tol);
    std::memcpy(u, g.u.data(), sizeof(double) * g.u_size());
    std::memcpy(v, g.v.data(), sizeof(double) * g.v_size());
    std::memcpy(p, g.p.data(), sizeof(double) * g.p_size());
    return applies;
}

// The right-hand side PressureProjection::recoverStaticPressure (pressure.cpp:35-66)
// builds for u (nx+1)(ny+2), v (nx+2)(ny+1); rhs is padded (nx+2)(ny+2).
void ref_static_rhs_2d(int nx, int ny, double dx, double dy, const uint8_t* solid,
                       const double* u, const double* v, double* rhs) {
    Grid g = make2(nx, ny, dx, dy, solid);
    std::memcpy(g.u.data(), u, sizeof(double) * g.u_size());
    std::memcpy(g.v.data(), v, sizeof(double) * g.v_size());
    CapturingSolver cap(rhs);
    PressureProjection::recoverStaticPressure(g, cap, 1, 1e-6);
}

int ref_project_3d(int nx, int ny, int nz, double dx, double dy, double dz, const uint8_t* solid,
                   double* u, double* v, double* w, double dt, int max_iter, double tol, double* p) {
    Grid3D g = make3(nx, ny, nz, dx, dy, dz, solid);
    std::memcpy(g.u.data(), u, sizeof(double) * g.u_size());
    std::memcpy(g.v.data(), v, sizeof(double) * g.v_size());
    std::memcpy(g.w.data(), w, sizeof(double) * g.w_size());
    int applies = 0;
    PCG3D solver(std::make_unique<Counting<Preconditioner3D, Grid3D>>(
        std::make_unique<UAAMGPreconditioner3D>(), &applies));
    PressureProjection3D::project(g, dt, solver, max_iter, tol);
    std::memcpy(u, g.u.data(), sizeof(double) * g.u_size());
    std::memcpy(v, g.v.data(), sizeof(double) * g.v_size());
    std::memcpy(w, g.w.data(), sizeof(double) * g.w_size());
    std::memcpy(p, g.p.data(), sizeof(double) * g.p_size());
    return applies;
}

}  // extern "C"
