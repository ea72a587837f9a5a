/* Test infrastructure only: plain-C restatement of the reference's CPU UAAMG-PCG
 * path (the oracle).  Only tests, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load this; the product never does.
 *
 * Layout (the reference's, include/core/mesh.h:30-35, include/core/mesh_3d.h:38):
 * ghost-padded, column-major, i fastest: id = i + j*(nx+2) [+ k*(nx+2)*(ny+2)].
 * dim == 2 ignores nz/dz. */
#ifndef UAAMG_ORACLE_H
#define UAAMG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oh_hier oh_hier;

/* Hierarchy set-up from a padded level-0 solid mask (1 = solid).
 * dirichlet != 0 turns every domain wall into a cell-centred Dirichlet p = 0 wall
 * (ghost = -interior); 0 keeps the reference's Neumann walls. */
oh_hier* oh_create(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                   const uint8_t* solid, int dirichlet);
void     oh_destroy(oh_hier* h);
int      oh_nlevels(const oh_hier* h);
void     oh_level_dims(const oh_hier* h, int l, int* nx, int* ny, int* nz);
/* Copies of level l's padded arrays. */
void     oh_level_solid(const oh_hier* h, int l, uint8_t* out);
void     oh_level_coeffs(const oh_hier* h, int l, double* cx, double* cy, double* cz,
                         double* diag);
/* z = M^{-1} r: one V(1,1) cycle (UAAMGPreconditioner[3D]::apply). */
void     oh_vcycle(oh_hier* h, const double* r, double* z);

/* PCG with the reference's semantics (PCG::solve / PCG3D::solve).
 *   precond    1 = UAAMG V-cycle, 0 = identity (plain CG)
 *   tol_mode   0 = stop when sqrt(r.r) < tol (the reference); 1 = when
 *              sqrt(r.r) < tol * ||b||, b the normalised RHS (so a warm start is
 *              measured against the same target as a cold one)
 *   warm       0 = p is accumulated from its incoming value with r0 = b (the
 *              reference); 1 = r0 = b - A p (true warm start)
 *   hist       optional, max_iter+1 entries: ||r_k|| after each update (hist[0] = ||r0||)
 * Returns the number of x updates performed; *status: 0 converged, 1 max_iter,
 * 2 breakdown (pAp < 1e-15 in the absolute mode, pAp < 1e-300 in the relative one). */
int oracle_pcg(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
               const uint8_t* solid, const double* rhs, double* p, int max_iter,
               double tol, int precond, int tol_mode, int warm, int dirichlet,
               double* hist, int* status);

/* The PCG's normalised right-hand side b = -(rhs - mean_fluid(rhs)) re-projected
 * to zero mean, as PCG::solve forms r before its loop, written to b (padded). */
void oracle_pcg_rhs(int dim, int nx, int ny, int nz, const uint8_t* solid,
                    const double* rhs, double* b, int dirichlet);

/* ||b - A x||_2 over fluid interior cells, A the PCG operator (-Laplacian with
 * Neumann solids/walls, pcg_3d.cpp:38-55), b from oracle_pcg_rhs.  Also returns
 * ||b||_2 in *bnorm. */
double oracle_true_residual(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                            const uint8_t* solid, const double* rhs, const double* x,
                            int dirichlet, double* bnorm);

/* A x with the PCG operator (solid rows 0). */
void oracle_matvec(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                   const uint8_t* solid, const double* x, double* ax, int dirichlet);

/* Face-velocity correction of PressureProjection::project (pressure.cpp:21-32,
 * pressure_3d.cpp:21-39): u -= dt*dp/dx on interior faces between fluid cells.
 * u: (nx+1)(ny+2)[(nz+2)], v: (nx+2)(ny+1)[(nz+2)], w: (nx+2)(ny+2)(nz+1). */
void oracle_correct_velocity(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                             const uint8_t* solid, const double* p, double dt,
                             double* u, double* v, double* w);

/* rhs = div(u)/dt at fluid interior cells, 0 elsewhere (pressure.cpp:10-14). */
void oracle_divergence_rhs(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                           const uint8_t* solid, const double* u, const double* v,
                           const double* w, double dt, double* rhs);

/* Variable-coefficient Laplacian of PCG::solve (pcg.cpp:35-46; Grid::lap_diag,
 * lap_off_x, lap_off_y, grid.h:23-31), 2D, padded arrays: the PCG of oracle_pcg
 * with that operator (Neumann walls), A x, and ||b - A x|| (with ||b|| in *bnorm). */
int oracle_pcg_var_2d(int nx, int ny, double dx, double dy, const uint8_t* solid,
                      const double* lap_diag, const double* lap_off_x, const double* lap_off_y,
                      const double* rhs, double* x, int max_iter, double tol, int precond,
                      int tol_mode, int warm, double* hist, int* status);
void oracle_matvec_var_2d(int nx, int ny, const uint8_t* solid, const double* lap_diag,
                          const double* lap_off_x, const double* lap_off_y, const double* x,
                          double* ax);
double oracle_true_residual_var_2d(int nx, int ny, const uint8_t* solid, const double* lap_diag,
                                   const double* lap_off_x, const double* lap_off_y,
                                   const double* rhs, const double* x, double* bnorm);
/* SmoothCylinder::applyToLaplacian (cylinder_model.cpp:50-71) on padded arrays;
 * inside != 0: solid fraction 1 inside the disk instead of outside. */
void oracle_smooth_cylinder_2d(int nx, int ny, double dx, double dy, double cx, double cy,
                               double R, double tw, int inside, uint8_t* solid, double* diag,
                               double* ox, double* oy);

/* RHS of PressureProjection::recoverStaticPressure (pressure.cpp:35-66), 2D. */
void oracle_static_rhs_2d(int nx, int ny, double dx, double dy, const uint8_t* solid,
                          const double* u, const double* v, double* rhs);

#ifdef __cplusplus
}
#endif
#endif
