// Seeded synthetic pressure-solve workloads (host code, C-ABI), shared by the
// bench, the tests and the examples so every consumer sees identical inputs.
// Arrays are the reference's ghost-padded, i-fastest layout.
//
// Generators (std::mt19937_64 + std::normal_distribution<double> /
// std::uniform_real_distribution<double>, libstdc++):
//   wl_spheres_3d        3D grid with random solid spheres and a smoothed
//                        Gaussian-noise RHS (the 256^3 mixed-precision workload)
//   wl_boxes             2D/3D grid with random solid boxes up to a target
//                        coverage and the same smoothed RHS (the batch workload)
//   wl_obstacle_flow_2d  2D disk obstacle, uniform inflow + random Fourier modes;
//                        RHS = div(u)/dt at fluid cells (the 2D projection workload)
//   wl_obstacle_flow_3d  3D sphere obstacle, same velocity model
//   wl_layered_lap_2d    variable-coefficient Laplacian of a layered medium
//                        (lap_diag / lap_off_x / lap_off_y of a 2D grid)
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#define WL_API extern "C" __attribute__((visibility("default")))

namespace {

inline size_t pid(int nx, int ny, int i, int j, int k) {
    return (size_t)i + (size_t)j * (nx + 2) + (size_t)k * (nx + 2) * (ny + 2);
}

// Separable Gaussian blur (sigma cells, kernel truncated at +-trunc, mirror
// "half-sample" reflection at the walls: index -1 -> 0, n -> n-1) of the
// interior of a padded field, FP64, in place.  dim 2 ignores z.
void blur(std::vector<double>& f, int dim, int nx, int ny, int nz, double sigma, int trunc) {
    if (sigma <= 0) return;
    std::vector<double> w(2 * trunc + 1);
    double s = 0;
    for (int t = -trunc; t <= trunc; ++t) s += (w[t + trunc] = std::exp(-0.5 * t * t / (sigma * sigma)));
    for (double& x : w) x /= s;
    auto refl = [](int q, int n) {
        while (q < 0 || q >= n) q = q < 0 ? -q - 1 : 2 * n - q - 1;
        return q;
    };
    const int kz = dim == 3 ? nz : 1, k0 = dim == 3 ? 1 : 0;
    std::vector<double> line, out;
    const int naxes = dim;
    for (int ax = 0; ax < naxes; ++ax) {
        const int n = ax == 0 ? nx : ax == 1 ? ny : nz;
        line.resize(n);
        out.resize(n);
        const int A = ax == 0 ? ny : nx, B = ax == 2 ? ny : kz;
        for (int b = 0; b < B; ++b)
            for (int a = 0; a < A; ++a) {
                auto at = [&](int q) -> double& {
                    if (ax == 0) return f[pid(nx, ny, q + 1, a + 1, b + k0)];
                    if (ax == 1) return f[pid(nx, ny, a + 1, q + 1, b + k0)];
                    return f[pid(nx, ny, a + 1, b + 1, q + 1)];
                };
                for (int q = 0; q < n; ++q) line[q] = at(q);
                for (int q = 0; q < n; ++q) {
                    double acc = 0;
                    for (int t = -trunc; t <= trunc; ++t) acc += w[t + trunc] * line[refl(q + t, n)];
                    out[q] = acc;
                }
                for (int q = 0; q < n; ++q) at(q) = out[q];
            }
    }
}

// Zero at solids and ghosts, subtract the fluid mean.
void finish_rhs(std::vector<double>& f, const uint8_t* solid, int dim, int nx, int ny, int nz) {
    const int k0 = dim == 3 ? 1 : 0, k1 = dim == 3 ? nz : 0;
    std::vector<double> g(f.size(), 0.0);
    double sum = 0;
    long cnt = 0;
    for (int k = k0; k <= k1; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const size_t c = pid(nx, ny, i, j, k);
                if (solid[c]) continue;
                g[c] = f[c];
                sum += f[c];
                ++cnt;
            }
    const double mean = cnt ? sum / (double)cnt : 0.0;
    for (int k = k0; k <= k1; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const size_t c = pid(nx, ny, i, j, k);
                if (!solid[c]) g[c] -= mean;
            }
    f.swap(g);
}

// Keeps the largest 6-connected (4-connected in 2D) component of fluid interior
// cells and turns every other fluid cell solid, so the Neumann problem has a
// single null-space constant and a zero-mean RHS is compatible.  Returns the
// number of cells filled.
long fill_pockets(uint8_t* solid, int dim, int nx, int ny, int nz) {
    const int kz = dim == 3 ? nz : 1, k0 = dim == 3 ? 1 : 0;
    const size_t n = (size_t)(nx + 2) * (ny + 2) * (dim == 3 ? (size_t)(nz + 2) : 1);
    std::vector<int> label(n, -1);
    std::vector<size_t> stack, sizes;
    int nlab = 0;
    for (int k = k0; k < k0 + kz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const size_t c0 = pid(nx, ny, i, j, k);
                if (solid[c0] || label[c0] >= 0) continue;
                size_t count = 0;
                label[c0] = nlab;
                stack.assign(1, c0);
                while (!stack.empty()) {
                    const size_t c = stack.back();
                    stack.pop_back();
                    ++count;
                    const int ci = (int)(c % (nx + 2)), cj = (int)((c / (nx + 2)) % (ny + 2));
                    const int ck = dim == 3 ? (int)(c / ((size_t)(nx + 2) * (ny + 2))) : 0;
                    const int nbi[6] = {ci - 1, ci + 1, ci, ci, ci, ci};
                    const int nbj[6] = {cj, cj, cj - 1, cj + 1, cj, cj};
                    const int nbk[6] = {ck, ck, ck, ck, ck - 1, ck + 1};
                    for (int q = 0; q < (dim == 3 ? 6 : 4); ++q) {
                        if (nbi[q] < 1 || nbi[q] > nx || nbj[q] < 1 || nbj[q] > ny) continue;
                        if (dim == 3 && (nbk[q] < 1 || nbk[q] > nz)) continue;
                        const size_t cn = pid(nx, ny, nbi[q], nbj[q], nbk[q]);
                        if (solid[cn] || label[cn] >= 0) continue;
                        label[cn] = nlab;
                        stack.push_back(cn);
                    }
                }
                sizes.push_back(count);
                ++nlab;
            }
    if (nlab <= 1) return 0;
    int best = 0;
    for (int q = 1; q < nlab; ++q)
        if (sizes[q] > sizes[best]) best = q;
    long filled = 0;
    for (size_t c = 0; c < n; ++c)
        if (label[c] >= 0 && label[c] != best) { solid[c] = 1; ++filled; }
    return filled;
}

void noise_rhs(std::mt19937_64& eng, std::vector<double>& f, int dim, int nx, int ny, int nz) {
    std::normal_distribution<double> nd(0.0, 1.0);
    const int k0 = dim == 3 ? 1 : 0, k1 = dim == 3 ? nz : 0;
    for (int k = k0; k <= k1; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) f[pid(nx, ny, i, j, k)] = nd(eng);
}

// Fourier velocity model: value(x, y[, z]) = base + sum_k A cos(th) + B sin(th),
// th = 2 pi (k.x / L), over integer k != 0 with |k|^2 <= kmax^2.  Coefficients
// (u_cos, u_sin, v_cos, v_sin[, w_cos, w_sin]) ~ N(0,1)/|k|^2 in k-major order.
struct Modes {
    std::vector<int> kx, ky, kz;
    std::vector<double> c;  // ncomp*2 per mode
    int ncomp;
};

Modes draw_modes(std::mt19937_64& eng, int dim, int kmax) {
    Modes m;
    m.ncomp = dim;
    std::normal_distribution<double> nd(0.0, 1.0);
    const int kzmax = dim == 3 ? kmax : 0;
    for (int a = -kmax; a <= kmax; ++a)
        for (int b = -kmax; b <= kmax; ++b)
            for (int q = -kzmax; q <= kzmax; ++q) {
                const int k2 = a * a + b * b + q * q;
                if (k2 == 0 || k2 > kmax * kmax) continue;
                m.kx.push_back(a); m.ky.push_back(b); m.kz.push_back(q);
                for (int t = 0; t < 2 * dim; ++t) m.c.push_back(nd(eng) / (double)k2);
            }
    return m;
}

// Evaluates component `comp` of the modes on a face array of nxf x nyf [x nzf]
// points at x = (i + ox)*dx etc. (i, j, k = array indices).
void eval_modes(const Modes& m, int comp, double base, int dim, int nxf, int nyf, int nzf,
                double ox, double oy, double oz, double dx, double dy, double dz, double lx,
                double ly, double lz, double* out) {
    const size_t nm = m.kx.size();
    const double tp = 2.0 * M_PI;
    const int kz1 = dim == 3 ? nzf : 1;
    std::vector<double> cx(nxf), sx(nxf);
    // group over kx: per (kx) accumulate C(j,k), S(j,k) over modes with that kx
    for (size_t c = 0; c < (size_t)nxf * nyf * kz1; ++c) out[c] = base;
    std::vector<double> C((size_t)nyf * kz1), S((size_t)nyf * kz1);
    int kxmin = 0, kxmax = 0;
    for (size_t q = 0; q < nm; ++q) { kxmin = std::min(kxmin, m.kx[q]); kxmax = std::max(kxmax, m.kx[q]); }
    for (int kx = kxmin; kx <= kxmax; ++kx) {
        std::fill(C.begin(), C.end(), 0.0);
        std::fill(S.begin(), S.end(), 0.0);
        bool any = false;
        for (size_t q = 0; q < nm; ++q) {
            if (m.kx[q] != kx) continue;
            any = true;
            const double A = m.c[q * 2 * m.ncomp + 2 * comp], B = m.c[q * 2 * m.ncomp + 2 * comp + 1];
            for (int k = 0; k < kz1; ++k) {
                const double phz = dim == 3 ? tp * m.kz[q] * (k + oz) * dz / lz : 0.0;
                for (int j = 0; j < nyf; ++j) {
                    const double ph = tp * m.ky[q] * (j + oy) * dy / ly + phz;
                    const double cy = std::cos(ph), sy = std::sin(ph);
                    C[(size_t)k * nyf + j] += A * cy + B * sy;
                    S[(size_t)k * nyf + j] += B * cy - A * sy;
                }
            }
        }
        if (!any) continue;
        for (int i = 0; i < nxf; ++i) {
            const double ph = tp * kx * (i + ox) * dx / lx;
            cx[i] = std::cos(ph);
            sx[i] = std::sin(ph);
        }
        for (int k = 0; k < kz1; ++k)
            for (int j = 0; j < nyf; ++j) {
                const double cc = C[(size_t)k * nyf + j], ss = S[(size_t)k * nyf + j];
                double* row = out + ((size_t)k * nyf + j) * nxf;
                for (int i = 0; i < nxf; ++i) row[i] += cx[i] * cc + sx[i] * ss;
            }
    }
}

}  // namespace

// 3D spheres workload.  Draw order: for each sphere (cx, cy, cz ~ U[0, n_axis),
// r ~ U[rmin, rmax]) in cell units, then one N(0,1) per interior cell
// (i fastest).  A cell is solid when its centre (i-0.5, j-0.5, k-0.5) lies
// strictly inside a sphere.  Fluid pockets cut off from the largest fluid region
// are filled (made solid).  RHS: the noise blurred (sigma, +-trunc), 0 at solids,
// fluid mean removed.  Returns the solid cell count.
WL_API long wl_spheres_3d(int nx, int ny, int nz, int nspheres, double rmin, double rmax,
                          uint64_t seed, double sigma, int trunc, uint8_t* solid, double* rhs) {
    std::mt19937_64 eng(seed);
    std::uniform_real_distribution<double> ux(0.0, nx), uy(0.0, ny), uz(0.0, nz), ur(rmin, rmax);
    const size_t n = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    std::memset(solid, 0, n);
    long nsolid = 0;
    for (int s = 0; s < nspheres; ++s) {
        const double cx = ux(eng), cy = uy(eng), cz = uz(eng), r = ur(eng);
        const int i0 = std::max(1, (int)std::floor(cx - r)), i1 = std::min(nx, (int)std::ceil(cx + r) + 1);
        const int j0 = std::max(1, (int)std::floor(cy - r)), j1 = std::min(ny, (int)std::ceil(cy + r) + 1);
        const int k0 = std::max(1, (int)std::floor(cz - r)), k1 = std::min(nz, (int)std::ceil(cz + r) + 1);
        for (int k = k0; k <= k1; ++k)
            for (int j = j0; j <= j1; ++j)
                for (int i = i0; i <= i1; ++i) {
                    const double ddx = i - 0.5 - cx, ddy = j - 0.5 - cy, ddz = k - 0.5 - cz;
                    if (ddx * ddx + ddy * ddy + ddz * ddz < r * r) {
                        uint8_t& c = solid[pid(nx, ny, i, j, k)];
                        if (!c) { c = 1; ++nsolid; }
                    }
                }
    }
    nsolid += fill_pockets(solid, 3, nx, ny, nz);
    std::vector<double> f(n, 0.0);
    noise_rhs(eng, f, 3, nx, ny, nz);
    blur(f, 3, nx, ny, nz, sigma, trunc);
    finish_rhs(f, solid, 3, nx, ny, nz);
    std::memcpy(rhs, f.data(), n * sizeof(double));
    return nsolid;
}

// Random axis-aligned solid boxes until the solid fraction reaches `coverage`;
// box sides ~ U[n/16, n/4] cells per axis, corner uniform; enclosed fluid
// pockets are filled.  Then the smoothed noise RHS as in wl_spheres_3d.  dim 2 ignores nz.  Returns the solid count.
WL_API long wl_boxes(int dim, int nx, int ny, int nz, double coverage, uint64_t seed, double sigma,
                     int trunc, uint8_t* solid, double* rhs) {
    std::mt19937_64 eng(seed);
    const int kz = dim == 3 ? nz : 1;
    const size_t n = (size_t)(nx + 2) * (ny + 2) * (dim == 3 ? (size_t)(nz + 2) : 1);
    std::memset(solid, 0, n);
    const double total = (double)nx * ny * kz;
    long nsolid = 0;
    int guard = 0;
    while ((double)nsolid < coverage * total && guard++ < 100000) {
        int lo[3], hi[3];
        const int dims[3] = {nx, ny, kz};
        for (int a = 0; a < dim; ++a) {
            const int N = dims[a];
            std::uniform_int_distribution<int> side(std::max(1, N / 16), std::max(1, N / 4));
            const int sd = side(eng);
            std::uniform_int_distribution<int> corner(1, std::max(1, N - sd + 1));
            lo[a] = corner(eng);
            hi[a] = std::min(N, lo[a] + sd - 1);
        }
        if (dim == 2) { lo[2] = 0; hi[2] = 0; }
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i) {
                    uint8_t& c = solid[pid(nx, ny, i, j, k)];
                    if (!c) { c = 1; ++nsolid; }
                }
    }
    nsolid += fill_pockets(solid, dim, nx, ny, nz);
    std::vector<double> f(n, 0.0);
    noise_rhs(eng, f, dim, nx, ny, nz);
    blur(f, dim, nx, ny, nz, sigma, trunc);
    finish_rhs(f, solid, dim, nx, ny, nz);
    std::memcpy(rhs, f.data(), n * sizeof(double));
    return nsolid;
}

// 2D obstacle flow: disk of radius 0.05*Ly at (0.25*Lx, 0.5*Ly) (cell centres
// strictly inside are solid); u = 1 + modes, v = modes with |k| <= kmax, phases
// advanced by omega_k * t (omega_k ~ N(0,1)*|k|, drawn after the amplitudes) when
// t != 0; u faces at (i*dx, (j-0.5)*dy), v faces at ((i-0.5)*dx, j*dy).
// rhs = div(u)/dt at fluid interior cells, 0 elsewhere.
WL_API long wl_obstacle_flow_2d(int nx, int ny, double dx, double dy, double dt, int kmax,
                                uint64_t seed, double t, uint8_t* solid, double* u, double* v,
                                double* rhs) {
    std::mt19937_64 eng(seed);
    const double lx = nx * dx, ly = ny * dy;
    const double cx = 0.25 * lx, cy = 0.5 * ly, r = 0.05 * ly;
    std::memset(solid, 0, (size_t)(nx + 2) * (ny + 2));
    long nsolid = 0;
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            const double x = (i - 0.5) * dx - cx, y = (j - 0.5) * dy - cy;
            if (x * x + y * y < r * r) { solid[pid(nx, ny, i, j, 0)] = 1; ++nsolid; }
        }
    Modes m = draw_modes(eng, 2, kmax);
    if (t != 0.0) {
        std::normal_distribution<double> nd(0.0, 1.0);
        for (size_t q = 0; q < m.kx.size(); ++q) {
            const double kk = std::sqrt((double)(m.kx[q] * m.kx[q] + m.ky[q] * m.ky[q]));
            const double ph = nd(eng) * kk * t;
            for (int comp = 0; comp < 2; ++comp) {
                double& A = m.c[q * 4 + 2 * comp];
                double& B = m.c[q * 4 + 2 * comp + 1];
                const double a = A * std::cos(ph) + B * std::sin(ph), b = B * std::cos(ph) - A * std::sin(ph);
                A = a; B = b;
            }
        }
    }
    eval_modes(m, 0, 1.0, 2, nx + 1, ny + 2, 1, 0.0, -0.5, 0.0, dx, dy, 1.0, lx, ly, 1.0, u);
    eval_modes(m, 1, 0.0, 2, nx + 2, ny + 1, 1, -0.5, 0.0, 0.0, dx, dy, 1.0, lx, ly, 1.0, v);
    std::memset(rhs, 0, sizeof(double) * (size_t)(nx + 2) * (ny + 2));
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            if (solid[pid(nx, ny, i, j, 0)]) continue;
            const double div = (u[i + (size_t)j * (nx + 1)] - u[i - 1 + (size_t)j * (nx + 1)]) / dx
                             + (v[i + (size_t)j * (nx + 2)] - v[i + (size_t)(j - 1) * (nx + 2)]) / dy;
            rhs[pid(nx, ny, i, j, 0)] = div / dt;
        }
    return nsolid;
}

// 3D obstacle flow: sphere of radius 0.05*Ly at (0.25*Lx, 0.5*Ly, 0.5*Lz);
// u = 1 + modes, v, w = modes; faces at the MAC positions; rhs = div/dt.
WL_API long wl_obstacle_flow_3d(int nx, int ny, int nz, double dx, double dy, double dz, double dt,
                                int kmax, uint64_t seed, double t, uint8_t* solid, double* u,
                                double* v, double* w, double* rhs) {
    std::mt19937_64 eng(seed);
    const double lx = nx * dx, ly = ny * dy, lz = nz * dz;
    const double cx = 0.25 * lx, cy = 0.5 * ly, cz = 0.5 * lz, r = 0.05 * ly;
    const size_t n = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    std::memset(solid, 0, n);
    long nsolid = 0;
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double x = (i - 0.5) * dx - cx, y = (j - 0.5) * dy - cy, z = (k - 0.5) * dz - cz;
                if (x * x + y * y + z * z < r * r) { solid[pid(nx, ny, i, j, k)] = 1; ++nsolid; }
            }
    Modes m = draw_modes(eng, 3, kmax);
    if (t != 0.0) {
        std::normal_distribution<double> nd(0.0, 1.0);
        for (size_t q = 0; q < m.kx.size(); ++q) {
            const double kk = std::sqrt((double)(m.kx[q] * m.kx[q] + m.ky[q] * m.ky[q] + m.kz[q] * m.kz[q]));
            const double ph = nd(eng) * kk * t;
            for (int comp = 0; comp < 3; ++comp) {
                double& A = m.c[q * 6 + 2 * comp];
                double& B = m.c[q * 6 + 2 * comp + 1];
                const double a = A * std::cos(ph) + B * std::sin(ph), b = B * std::cos(ph) - A * std::sin(ph);
                A = a; B = b;
            }
        }
    }
    eval_modes(m, 0, 1.0, 3, nx + 1, ny + 2, nz + 2, 0.0, -0.5, -0.5, dx, dy, dz, lx, ly, lz, u);
    eval_modes(m, 1, 0.0, 3, nx + 2, ny + 1, nz + 2, -0.5, 0.0, -0.5, dx, dy, dz, lx, ly, lz, v);
    eval_modes(m, 2, 0.0, 3, nx + 2, ny + 2, nz + 1, -0.5, -0.5, 0.0, dx, dy, dz, lx, ly, lz, w);
    std::memset(rhs, 0, sizeof(double) * n);
    const size_t su = nx + 1, suv = (size_t)(nx + 1) * (ny + 2);
    const size_t sv = nx + 2, svv = (size_t)(nx + 2) * (ny + 1);
    const size_t sw = nx + 2, sww = (size_t)(nx + 2) * (ny + 2);
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                if (solid[pid(nx, ny, i, j, k)]) continue;
                const double div = (u[i + j * su + k * suv] - u[(i - 1) + j * su + k * suv]) / dx
                                 + (v[i + j * sv + k * svv] - v[i + (j - 1) * sv + k * svv]) / dy
                                 + (w[i + j * sw + k * sww] - w[i + j * sw + (k - 1) * sww]) / dz;
                rhs[pid(nx, ny, i, j, k)] = div / dt;
            }
    return nsolid;
}

// Serving workload, one simulation id: an n x n (2D) or n^3 (3D) box, h = 1/n, with
// a disk / sphere of radius 0.05 n cells at (0.25 n, 0.5 n[, 0.5 n]) (cell centres
// strictly inside are solid), and two right-hand sides rhs0, rhs1 = div(u)/dt of
// two seeded velocity fields u = sum over 0 < |k| <= kmax of modes with N(0,1)/|k|^2
// cosine and sine amplitudes per component (dt = 1e-3), evaluated in closed form
// at cell centres: with phi = 2 pi k.x / L,
//   div u = sum_k (2 pi / L) [ -(k.A_k) sin phi + (k.B_k) cos phi ].
// A request at step t of the id uses rhs0 + (t / 20) rhs1 (an evolving field).
// Both are zero at solids with zero fluid mean.  Separable evaluation: the
// per-axis cosine/sine tables combine per row, so a cell costs 6 flops per mode.
// Coefficients of the 2D operator A v = d v_C + ox (v_L + v_R) + oy (v_B + v_T)
// (the lap_* form PCG::solve takes, pcg.cpp:35-46) for a layered medium: the x
// conductivity varies with the row, kx(j) = 1 + amp sin(2 pi (j - 1/2) / ny), the y
// conductivity with the column, ky(i) = 1 + amp cos(2 pi (i - 1/2) / nx), so the
// coupling between two cells is the same from either side (A symmetric) and every
// row sums to zero (the constant is A's null vector, as for the uniform operator).
// ox = -kx/dx^2, oy = -ky/dy^2, d = 2 kx/dx^2 + 2 ky/dy^2 on fluid cells; solid
// cells get d = 1e15 and no couplings (never read: solid rows are 0); ghosts 0.
// Returns the number of fluid cells.
WL_API long wl_layered_lap_2d(int nx, int ny, double dx, double dy, double amp,
                              const uint8_t* solid, double* diag, double* ox, double* oy) {
    const double pi = 3.14159265358979323846;
    const size_t n = (size_t)(nx + 2) * (ny + 2);
    std::memset(diag, 0, n * sizeof(double));
    std::memset(ox, 0, n * sizeof(double));
    std::memset(oy, 0, n * sizeof(double));
    const double ix = 1.0 / (dx * dx), iy = 1.0 / (dy * dy);
    long fluid = 0;
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            const size_t c = pid(nx, ny, i, j, 0);
            if (solid[c]) {
                diag[c] = 1e15;
                continue;
            }
            const double kx = 1.0 + amp * std::sin(2.0 * pi * (j - 0.5) / ny);
            const double ky = 1.0 + amp * std::cos(2.0 * pi * (i - 0.5) / nx);
            ox[c] = -kx * ix;
            oy[c] = -ky * iy;
            diag[c] = 2.0 * kx * ix + 2.0 * ky * iy;
            ++fluid;
        }
    return fluid;
}

WL_API long wl_serve_fields(int dim, int n, int kmax, uint64_t seed, uint8_t* solid, double* rhs0,
                            double* rhs1) {
    const int nz = dim == 3 ? n : 0;
    const size_t N = (size_t)(n + 2) * (n + 2) * (dim == 3 ? (size_t)(n + 2) : 1);
    std::memset(solid, 0, N);
    long nsolid = 0;
    const double c0 = 0.25 * n, c1 = 0.5 * n, rad = 0.05 * n;
    for (int k = dim == 3 ? 1 : 0; k <= nz; ++k)
        for (int j = 1; j <= n; ++j)
            for (int i = 1; i <= n; ++i) {
                const double x = i - 0.5 - c0, y = j - 0.5 - c1, z = dim == 3 ? k - 0.5 - c1 : 0.0;
                if (x * x + y * y + z * z < rad * rad) { solid[pid(n, n, i, j, k)] = 1; ++nsolid; }
            }
    std::mt19937_64 eng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<int> kx, ky, kz;
    const int kzr = dim == 3 ? kmax : 0;
    for (int a = -kmax; a <= kmax; ++a)
        for (int b = -kmax; b <= kmax; ++b)
            for (int c = -kzr; c <= kzr; ++c) {
                const int kk = a * a + b * b + c * c;
                if (kk == 0 || kk > kmax * kmax) continue;
                kx.push_back(a); ky.push_back(b); kz.push_back(c);
            }
    const size_t M = kx.size();
    const double two_pi_l = 2.0 * M_PI / n, dt = 1e-3;
    for (int field = 0; field < 2; ++field) {
        std::vector<double> P(M), Q(M);  // div u = sum P sin(phi) + Q cos(phi)
        for (size_t q = 0; q < M; ++q) {
            const double kk = (double)(kx[q] * kx[q] + ky[q] * ky[q] + kz[q] * kz[q]);
            const int kc[3] = {kx[q], ky[q], kz[q]};
            double ka = 0, kb = 0;
            for (int comp = 0; comp < dim; ++comp) {
                const double A = nd(eng) / kk, B = nd(eng) / kk;
                ka += kc[comp] * A;
                kb += kc[comp] * B;
            }
            P[q] = -two_pi_l * ka / dt;
            Q[q] = two_pi_l * kb / dt;
        }
        // per-axis tables of cos / sin (2 pi k x / L) at cell centres x = i - 0.5
        auto table = [&](const std::vector<int>& kv, std::vector<double>& ct, std::vector<double>& st) {
            ct.assign(M * (n + 2), 1.0);
            st.assign(M * (n + 2), 0.0);
            for (size_t q = 0; q < M; ++q)
                for (int i = 1; i <= n; ++i) {
                    const double ph = two_pi_l * kv[q] * (i - 0.5);
                    ct[q * (n + 2) + i] = std::cos(ph);
                    st[q * (n + 2) + i] = std::sin(ph);
                }
        };
        std::vector<double> cxt, sxt, cyt, syt, czt, szt;
        table(kx, cxt, sxt);
        table(ky, cyt, syt);
        if (dim == 3) table(kz, czt, szt);
        std::vector<double> f(N, 0.0), cr(M), sr(M);
        for (int k = dim == 3 ? 1 : 0; k <= nz; ++k)
            for (int j = 1; j <= n; ++j) {
                for (size_t q = 0; q < M; ++q) {  // phase of the row: phi_y + phi_z
                    const double cy = cyt[q * (n + 2) + j], sy = syt[q * (n + 2) + j];
                    const double cz = dim == 3 ? czt[q * (n + 2) + k] : 1.0;
                    const double sz = dim == 3 ? szt[q * (n + 2) + k] : 0.0;
                    cr[q] = cy * cz - sy * sz;
                    sr[q] = sy * cz + cy * sz;
                }
                double* row = &f[pid(n, n, 0, j, k)];
                for (int i = 1; i <= n; ++i) {
                    double acc = 0.0;
                    for (size_t q = 0; q < M; ++q) {
                        const double cx = cxt[q * (n + 2) + i], sx = sxt[q * (n + 2) + i];
                        acc += P[q] * (sx * cr[q] + cx * sr[q]) + Q[q] * (cx * cr[q] - sx * sr[q]);
                    }
                    row[i] = acc;
                }
            }
        finish_rhs(f, solid, dim, n, n, nz);
        std::memcpy(field == 0 ? rhs0 : rhs1, f.data(), N * sizeof(double));
    }
    return nsolid;
}
