// Test infrastructure only: runs the reference's OWN pressure projection
// (PressureProjection::project, src/pressure/pressure.cpp:5-33, and
// PressureProjection3D::project, src/pressure/pressure_3d.cpp:5-40) with the
// drop-in GPU solver a maintainer adds to the reference -- the GpuUAAMGPCG[3D]
// subclass, factory lines and SolverKind mirror of INTEGRATION.md section 2,
// extracted verbatim into gpu_uaamg_pcg.h, factory2d_lines.inc, factory3d_lines.inc
// and solver_kind.h by oracle/build_integration.py -- and with the reference's own
// PCG(UAAMGPreconditioner) / PCG3D(UAAMGPreconditioner3D), on identical grids.
//
// Two projection steps per grid, on the same solver objects, with the obstacle
// moved between them (the subclass must re-send the changed mask).  Prints one
// line per step with the largest differences of p and of the projected face
// velocities, relative to max(1, max |reference|), and exits 1 when one exceeds
// 1e-10 (the reference's own GPU-vs-CPU PCG bar, test_cuda_uaamg_3d.cu:94).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "core/grid.h"
#include "core/grid_3d.h"
#include "pressure/pressure.h"
#include "pressure/pressure_3d.h"
#include "solver/pcg.h"
#include "solver/pcg_3d.h"
#include "solver/preconditioner/uaamg_preconditioner.h"
#include "solver/preconditioner/uaamg_preconditioner_3d.h"

#include "gpu_uaamg_pcg.h"
#include "solver_kind.h"

namespace {

std::unique_ptr<Solver> create_2d(const std::string& name) {
#include "factory2d_lines.inc"
    return nullptr;
}

std::unique_ptr<Solver3D> create_3d(const std::string& name) {
#include "factory3d_lines.inc"
    return nullptr;
}

double max_rel(const std::vector<double>& a, const std::vector<double>& b) {
    double d = 0.0, m = 1.0;
    for (size_t c = 0; c < a.size(); ++c) {
        d = std::max(d, std::fabs(a[c] - b[c]));
        m = std::max(m, std::fabs(b[c]));
    }
    return d / m;
}

// ||b|| of PCG::solve's normalised right-hand side b = -(rhs - mean over fluid),
// rhs = div(u)/dt as PressureProjection::project forms it (for a tolerance that
// both solvers reach well inside their convergence)
double rhs_norm_2d(const Grid& g, double dt) {
    double s = 0.0, n = 0.0;
    std::vector<double> r(g.p.size(), 0.0);
    for (int i = 1; i <= g.nx; ++i)
        for (int j = 1; j <= g.ny; ++j)
            if (!g.is_solid(i, j)) {
                r[g.ip(i, j)] = g.divergence(i, j) / dt;
                s += r[g.ip(i, j)];
                n += 1.0;
            }
    const double m = n > 0 ? s / n : 0.0;
    double q = 0.0;
    for (int i = 1; i <= g.nx; ++i)
        for (int j = 1; j <= g.ny; ++j)
            if (!g.is_solid(i, j)) q += (r[g.ip(i, j)] - m) * (r[g.ip(i, j)] - m);
    return std::sqrt(q);
}

double rhs_norm_3d(const Grid3D& g, double dt) {
    double s = 0.0, n = 0.0;
    std::vector<double> r(g.p.size(), 0.0);
    for (int i = 1; i <= g.nx; ++i)
        for (int j = 1; j <= g.ny; ++j)
            for (int k = 1; k <= g.nz; ++k)
                if (!g.is_solid(i, j, k)) {
                    r[g.ip(i, j, k)] = g.divergence(i, j, k) / dt;
                    s += r[g.ip(i, j, k)];
                    n += 1.0;
                }
    const double m = n > 0 ? s / n : 0.0;
    double q = 0.0;
    for (int i = 1; i <= g.nx; ++i)
        for (int j = 1; j <= g.ny; ++j)
            for (int k = 1; k <= g.nz; ++k)
                if (!g.is_solid(i, j, k)) q += (r[g.ip(i, j, k)] - m) * (r[g.ip(i, j, k)] - m);
    return std::sqrt(q);
}

// 2D: 96 x 64 cells, dx = 1e-2, dy = 1.5e-2, disk of radius 8 cells; u = 1 + noise,
// v = noise (seeded); the disk moves 3 cells in x for the second step
void init_2d(Grid& g, int step) {
    std::mt19937_64 rng(11 + step);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::fill(g.solid.begin(), g.solid.end(), false);
    const double ci = 24.5 + 3 * step, cj = 32.5, r = 8.0;
    for (int i = 1; i <= g.nx; ++i)
        for (int j = 1; j <= g.ny; ++j)
            if ((i - ci) * (i - ci) + (j - cj) * (j - cj) < r * r) g.set_solid(i, j);
    for (auto& x : g.u) x = 1.0 + 0.3 * nd(rng);
    for (auto& x : g.v) x = 0.3 * nd(rng);
    std::fill(g.p.begin(), g.p.end(), 0.0);
}

// 3D: 28 x 24 x 20 cells, h = 1/24, sphere of radius 5 cells; the sphere moves 2
// cells in x for the second step
void init_3d(Grid3D& g, int step) {
    std::mt19937_64 rng(23 + step);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::fill(g.solid.begin(), g.solid.end(), false);
    const double ci = 10.5 + 2 * step, cj = 12.5, ck = 10.5, r = 5.0;
    for (int i = 1; i <= g.nx; ++i)
        for (int j = 1; j <= g.ny; ++j)
            for (int k = 1; k <= g.nz; ++k)
                if ((i - ci) * (i - ci) + (j - cj) * (j - cj) + (k - ck) * (k - ck) < r * r)
                    g.solid[g.ip(i, j, k)] = true;
    for (auto& x : g.u) x = 1.0 + 0.3 * nd(rng);
    for (auto& x : g.v) x = 0.3 * nd(rng);
    for (auto& x : g.w) x = 0.3 * nd(rng);
    std::fill(g.p.begin(), g.p.end(), 0.0);
}

}  // namespace

int main() {
    const double bar = 1e-10, dt = 1e-3;
    bool ok = true;
    const std::string key = solver_key(SolverKind::PCG_UAAMG_GPU);
    if (solver_kind(key) != SolverKind::PCG_UAAMG_GPU) {
        std::printf("SolverKind round trip failed for %s\n", key.c_str());
        return 1;
    }
    {
        auto gpu = create_2d(key);
        PCG ref(std::make_unique<UAAMGPreconditioner>());
        if (!gpu) { std::printf("2D factory returned no solver for %s\n", key.c_str()); return 1; }
        for (int step = 0; step < 2; ++step) {
            Grid ga(96, 64, 96 * 1e-2, 64 * 1.5e-2), gb(96, 64, 96 * 1e-2, 64 * 1.5e-2);
            ga.dx = gb.dx = 1e-2;
            ga.dy = gb.dy = 1.5e-2;
            init_2d(ga, step);
            init_2d(gb, step);
            const double tol = 1e-12 * rhs_norm_2d(gb, dt);
            PressureProjection::project(ga, dt, *gpu, 1000, tol);
            PressureProjection::project(gb, dt, ref, 1000, tol);
            const double dp = max_rel(ga.p, gb.p), du = max_rel(ga.u, gb.u), dv = max_rel(ga.v, gb.v);
            std::printf("2d step %d solver %s: dp %.3e du %.3e dv %.3e\n", step, gpu->name().c_str(),
                        dp, du, dv);
            ok = ok && dp <= bar && du <= bar && dv <= bar;
        }
    }
    {
        auto gpu = create_3d(key);
        auto ref = create_3d(solver_key(SolverKind::PCG_UAAMG));
        if (!gpu || !ref) { std::printf("3D factory returned no solver\n"); return 1; }
        for (int step = 0; step < 2; ++step) {
            const double h = 1.0 / 24;
            Grid3D ga(28, 24, 20, 28 * h, 24 * h, 20 * h), gb(28, 24, 20, 28 * h, 24 * h, 20 * h);
            ga.dx = gb.dx = ga.dy = gb.dy = ga.dz = gb.dz = h;
            init_3d(ga, step);
            init_3d(gb, step);
            const double tol = 1e-12 * rhs_norm_3d(gb, dt);
            PressureProjection3D::project(ga, dt, *gpu, 1000, tol);
            PressureProjection3D::project(gb, dt, *ref, 1000, tol);
            const double dp = max_rel(ga.p, gb.p), du = max_rel(ga.u, gb.u), dv = max_rel(ga.v, gb.v),
                         dw = max_rel(ga.w, gb.w);
            std::printf("3d step %d solvers %s / %s: dp %.3e du %.3e dv %.3e dw %.3e\n", step,
                        gpu->name().c_str(), ref->name().c_str(), dp, du, dv, dw);
            ok = ok && dp <= bar && du <= bar && dv <= bar && dw <= bar;
        }
    }
    std::printf(ok ? "integration ok\n" : "integration FAILED\n");
    return ok ? 0 : 1;
}
