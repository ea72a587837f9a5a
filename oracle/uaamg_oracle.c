/* Test infrastructure only — the oracle.  A plain-C restatement of the reference's
 * CPU UAAMG-preconditioned CG (A-006/UAAMGPCG), used by tests/, smoke() and the
 * bench's CPU-baseline leg as the oracle.  The product never links it.
 *
 * Every function follows a reference function line by line in ARITHMETIC ORDER
 * (loop nesting i→j→k for reductions, the same left-to-right sums), so that with
 * -ffp-contract=off it reproduces the reference bit for bit; the cited file:line
 * is given on each.  2D and 3D share one body: in 2D the k index is fixed at 0
 * (no z ghosts), there are no z couplings and a coarse cell has 4 children.
 *
 * Extension beyond the reference (config "plain method, CPU-runnable"): with
 * dirichlet != 0 every domain wall is a cell-centred Dirichlet p = 0 wall
 * (ghost = -interior).  In the PCG operator the outside neighbour then reads -p_C;
 * in the hierarchy a wall adds 2*h^-2 to a per-cell wall-diagonal channel that
 * Galerkin coarsening sums over children, and the null-space projections are
 * skipped (the operator is nonsingular). */
#include "uaamg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int nx, ny, nz;         /* nz == 0 marks 2D */
    double dx, dy, dz;
    long sx, sxy, n;        /* strides and padded size */
    uint8_t* solid;
    double *p, *b, *cx, *cy, *cz, *wd, *diag;
} olevel;

struct oh_hier {
    int dim, nl, dirichlet;
    olevel* L;
};

static inline long cid(const olevel* L, int i, int j, int k) {
    return (long)i + (long)j * L->sx + (long)k * L->sxy;
}

static void level_alloc(olevel* L, int dim, int nx, int ny, int nz, double dx, double dy,
                        double dz) {
    L->nx = nx; L->ny = ny; L->nz = dim == 3 ? nz : 0;
    L->dx = dx; L->dy = dy; L->dz = dz;
    L->sx = nx + 2;
    L->sxy = (long)(nx + 2) * (ny + 2);
    L->n = dim == 3 ? L->sxy * (nz + 2) : L->sxy;
    L->solid = (uint8_t*)calloc((size_t)L->n, 1);
    L->p = (double*)calloc((size_t)L->n, sizeof(double));
    L->b = (double*)calloc((size_t)L->n, sizeof(double));
    L->cx = (double*)calloc((size_t)L->n, sizeof(double));
    L->cy = (double*)calloc((size_t)L->n, sizeof(double));
    L->cz = (double*)calloc((size_t)L->n, sizeof(double));
    L->wd = (double*)calloc((size_t)L->n, sizeof(double));
    L->diag = (double*)calloc((size_t)L->n, sizeof(double));
}

static void level_free(olevel* L) {
    free(L->solid); free(L->p); free(L->b); free(L->cx); free(L->cy); free(L->cz);
    free(L->wd); free(L->diag);
}

/* Interior k range: 1..nz in 3D, the single plane 0 in 2D. */
#define KLO(L) ((L)->nz ? 1 : 0)
#define KHI(L) ((L)->nz ? (L)->nz : 0)
#define KCH(L) ((L)->nz ? 2 : 1)

/* uaamg_preconditioner_3d.cpp:11-32 / uaamg_preconditioner.cpp:23-41 */
static void build_hierarchy(oh_hier* h, int nx, int ny, int nz, double dx, double dy, double dz) {
    int cap = 32;
    h->L = (olevel*)calloc((size_t)cap, sizeof(olevel));
    h->nl = 0;
    const int d3 = h->dim == 3;
    while (nx >= 2 && ny >= 2 && (!d3 || nz >= 2)) {
        level_alloc(&h->L[h->nl++], h->dim, nx, ny, nz, dx, dy, dz);
        if (nx <= 4 || ny <= 4 || (d3 && nz <= 4)) break;
        nx /= 2; ny /= 2; nz /= 2;
        dx *= 2.0; dy *= 2.0; dz *= 2.0;
    }
}

/* uaamg_preconditioner_3d.cpp:34-45 (>= 4 of 8) / uaamg_preconditioner.cpp:43-53 (>= 2 of 4) */
static void restrict_solid(const olevel* f, olevel* c) {
    const int nch = c->nz ? 8 : 4;
    for (int ic = 1; ic <= c->nx; ic++)
        for (int jc = 1; jc <= c->ny; jc++)
            for (int kc = KLO(c); kc <= KHI(c); kc++) {
                int i_f = 2 * ic - 1, j_f = 2 * jc - 1, k_f = c->nz ? 2 * kc - 1 : 0, sc = 0;
                for (int di = 0; di < 2; di++)
                    for (int dj = 0; dj < 2; dj++)
                        for (int dk = 0; dk < KCH(c); dk++)
                            if (f->solid[cid(f, i_f + di, j_f + dj, k_f + dk)]) sc++;
                c->solid[cid(c, ic, jc, kc)] = (uint8_t)(2 * sc >= nch);
            }
}

/* Diagonal = sum of the 2*dim couplings in the reference's order
 * (uaamg_preconditioner_3d.cpp:72-74, 112-114; uaamg_preconditioner.cpp:73, 99-100),
 * plus the Dirichlet wall channel (0 for the reference's Neumann walls). */
static void set_diag(olevel* L) {
    memset(L->diag, 0, sizeof(double) * (size_t)L->n);
    for (int i = 1; i <= L->nx; i++)
        for (int j = 1; j <= L->ny; j++)
            for (int k = KLO(L); k <= KHI(L); k++) {
                long id = cid(L, i, j, k);
                if (L->solid[id]) continue;
                double d = L->cx[id] + L->cx[cid(L, i - 1, j, k)]
                         + L->cy[id] + L->cy[cid(L, i, j - 1, k)];
                if (L->nz) d = d + L->cz[id] + L->cz[cid(L, i, j, k - 1)];
                L->diag[id] = d + L->wd[id];
            }
}

/* uaamg_preconditioner_3d.cpp:50-76 / uaamg_preconditioner.cpp:56-75 */
static void setup_fine_coeffs(olevel* L, int dirichlet) {
    const double idx2 = 1.0 / (L->dx * L->dx), idy2 = 1.0 / (L->dy * L->dy);
    const double idz2 = L->nz ? 1.0 / (L->dz * L->dz) : 0.0;
    memset(L->cx, 0, sizeof(double) * (size_t)L->n);
    memset(L->cy, 0, sizeof(double) * (size_t)L->n);
    memset(L->cz, 0, sizeof(double) * (size_t)L->n);
    memset(L->wd, 0, sizeof(double) * (size_t)L->n);
    for (int i = 1; i <= L->nx; i++)
        for (int j = 1; j <= L->ny; j++)
            for (int k = KLO(L); k <= KHI(L); k++) {
                long id = cid(L, i, j, k);
                if (L->solid[id]) continue;
                if (i < L->nx && !L->solid[cid(L, i + 1, j, k)]) L->cx[id] = idx2;
                if (j < L->ny && !L->solid[cid(L, i, j + 1, k)]) L->cy[id] = idy2;
                if (L->nz && k < L->nz && !L->solid[cid(L, i, j, k + 1)]) L->cz[id] = idz2;
                if (dirichlet) {
                    double w = 0.0;
                    if (i == 1) w += 2.0 * idx2;
                    if (i == L->nx) w += 2.0 * idx2;
                    if (j == 1) w += 2.0 * idy2;
                    if (j == L->ny) w += 2.0 * idy2;
                    if (L->nz && k == 1) w += 2.0 * idz2;
                    if (L->nz && k == L->nz) w += 2.0 * idz2;
                    L->wd[id] = w;
                }
            }
    set_diag(L);
}

/* uaamg_preconditioner_3d.cpp:81-116 / uaamg_preconditioner.cpp:79-102 */
static void galerkin_coarsen(const olevel* f, olevel* c) {
    memset(c->cx, 0, sizeof(double) * (size_t)c->n);
    memset(c->cy, 0, sizeof(double) * (size_t)c->n);
    memset(c->cz, 0, sizeof(double) * (size_t)c->n);
    memset(c->wd, 0, sizeof(double) * (size_t)c->n);
    for (int ic = 1; ic <= c->nx; ic++)
        for (int jc = 1; jc <= c->ny; jc++)
            for (int kc = KLO(c); kc <= KHI(c); kc++) {
                long id = cid(c, ic, jc, kc);
                if (c->solid[id]) continue;
                int i_f = 2 * ic - 1, j_f = 2 * jc - 1, k_f = c->nz ? 2 * kc - 1 : 0;
                double sx = 0, sy = 0, sz = 0, sw = 0;
                for (int dj = 0; dj < 2; dj++)
                    for (int dk = 0; dk < KCH(c); dk++)
                        sx += f->cx[cid(f, i_f + 1, j_f + dj, k_f + dk)];
                for (int di = 0; di < 2; di++)
                    for (int dk = 0; dk < KCH(c); dk++)
                        sy += f->cy[cid(f, i_f + di, j_f + 1, k_f + dk)];
                if (c->nz)
                    for (int di = 0; di < 2; di++)
                        for (int dj = 0; dj < 2; dj++)
                            sz += f->cz[cid(f, i_f + di, j_f + dj, k_f + 1)];
                for (int di = 0; di < 2; di++)
                    for (int dj = 0; dj < 2; dj++)
                        for (int dk = 0; dk < KCH(c); dk++)
                            sw += f->wd[cid(f, i_f + di, j_f + dj, k_f + dk)];
                c->cx[id] = sx;
                c->cy[id] = sy;
                c->cz[id] = sz;
                c->wd[id] = sw;
            }
    set_diag(c);
}

/* uaamg_preconditioner_3d.cpp:123-141 / uaamg_preconditioner.cpp:105-121 */
static void sweep(olevel* L, int parity) {
    for (int i = 1; i <= L->nx; i++)
        for (int j = 1; j <= L->ny; j++)
            for (int k = KLO(L); k <= KHI(L); k++) {
                if (((i + j + k) & 1) != parity) continue;
                long id = cid(L, i, j, k);
                if (L->solid[id] || L->diag[id] < 1e-30) continue;
                long im = cid(L, i - 1, j, k), jm = cid(L, i, j - 1, k);
                double nb = L->cx[id] * L->p[cid(L, i + 1, j, k)] + L->cx[im] * L->p[im]
                          + L->cy[id] * L->p[cid(L, i, j + 1, k)] + L->cy[jm] * L->p[jm];
                if (L->nz) {
                    long km = cid(L, i, j, k - 1);
                    nb = nb + L->cz[id] * L->p[cid(L, i, j, k + 1)] + L->cz[km] * L->p[km];
                }
                L->p[id] = (L->b[id] + nb) / L->diag[id];
            }
}

static void smooth(olevel* L, int reverse) {
    int p0 = reverse ? 0 : 1;
    sweep(L, p0);
    sweep(L, 1 - p0);
}

/* uaamg_preconditioner_3d.cpp:144-165 / uaamg_preconditioner.cpp:124-144 */
static void restrict_residual(const olevel* f, olevel* c) {
    for (int ic = 1; ic <= c->nx; ic++)
        for (int jc = 1; jc <= c->ny; jc++)
            for (int kc = KLO(c); kc <= KHI(c); kc++) {
                long id = cid(c, ic, jc, kc);
                if (c->solid[id]) continue;
                int i_f = 2 * ic - 1, j_f = 2 * jc - 1, k_f = c->nz ? 2 * kc - 1 : 0;
                double sum = 0;
                for (int di = 0; di < 2; di++)
                    for (int dj = 0; dj < 2; dj++)
                        for (int dk = 0; dk < KCH(c); dk++) {
                            int fi = i_f + di, fj = j_f + dj, fk = k_f + dk;
                            long fid = cid(f, fi, fj, fk);
                            if (f->solid[fid]) continue;
                            long im = cid(f, fi - 1, fj, fk), jm = cid(f, fi, fj - 1, fk);
                            double ax = f->diag[fid] * f->p[fid]
                                      - f->cx[fid] * f->p[cid(f, fi + 1, fj, fk)] - f->cx[im] * f->p[im]
                                      - f->cy[fid] * f->p[cid(f, fi, fj + 1, fk)] - f->cy[jm] * f->p[jm];
                            if (f->nz) {
                                long km = cid(f, fi, fj, fk - 1);
                                ax = ax - f->cz[fid] * f->p[cid(f, fi, fj, fk + 1)] - f->cz[km] * f->p[km];
                            }
                            sum += f->b[fid] - ax;
                        }
                c->b[id] = sum;
            }
}

/* uaamg_preconditioner_3d.cpp:168-181 / uaamg_preconditioner.cpp:147-160 */
static void prolongate_add(const olevel* c, olevel* f) {
    for (int ic = 1; ic <= c->nx; ic++)
        for (int jc = 1; jc <= c->ny; jc++)
            for (int kc = KLO(c); kc <= KHI(c); kc++) {
                long id = cid(c, ic, jc, kc);
                if (c->solid[id]) continue;
                double val = 2.0 * c->p[id];
                int i_f = 2 * ic - 1, j_f = 2 * jc - 1, k_f = c->nz ? 2 * kc - 1 : 0;
                for (int di = 0; di < 2; di++)
                    for (int dj = 0; dj < 2; dj++)
                        for (int dk = 0; dk < KCH(c); dk++) {
                            long fid = cid(f, i_f + di, j_f + dj, k_f + dk);
                            if (!f->solid[fid]) f->p[fid] += val;
                        }
            }
}

/* uaamg_preconditioner_3d.cpp:183-196 / uaamg_preconditioner.cpp:162-175 */
static void vcycle(oh_hier* h, int l) {
    olevel* L = &h->L[l];
    if (l == h->nl - 1) {
        for (int s = 0; s < 10; s++) { smooth(L, 0); smooth(L, 1); }
        return;
    }
    smooth(L, 0);
    olevel* C = &h->L[l + 1];
    restrict_residual(L, C);
    memset(C->p, 0, sizeof(double) * (size_t)C->n);
    vcycle(h, l + 1);
    prolongate_add(C, L);
    smooth(L, 1);
}

oh_hier* oh_create(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                   const uint8_t* solid, int dirichlet) {
    oh_hier* h = (oh_hier*)calloc(1, sizeof(oh_hier));
    h->dim = dim;
    h->dirichlet = dirichlet;
    build_hierarchy(h, nx, ny, nz, dx, dy, dz);
    /* uaamg_preconditioner_3d.cpp:205-214: masks (ghosts included), then coefficients */
    memcpy(h->L[0].solid, solid, (size_t)h->L[0].n);
    for (int l = 1; l < h->nl; l++) restrict_solid(&h->L[l - 1], &h->L[l]);
    setup_fine_coeffs(&h->L[0], dirichlet);
    for (int l = 1; l < h->nl; l++) galerkin_coarsen(&h->L[l - 1], &h->L[l]);
    return h;
}

void oh_destroy(oh_hier* h) {
    if (!h) return;
    for (int l = 0; l < h->nl; l++) level_free(&h->L[l]);
    free(h->L);
    free(h);
}

int oh_nlevels(const oh_hier* h) { return h->nl; }

void oh_level_dims(const oh_hier* h, int l, int* nx, int* ny, int* nz) {
    *nx = h->L[l].nx; *ny = h->L[l].ny; *nz = h->L[l].nz;
}

void oh_level_solid(const oh_hier* h, int l, uint8_t* out) {
    memcpy(out, h->L[l].solid, (size_t)h->L[l].n);
}

void oh_level_coeffs(const oh_hier* h, int l, double* cx, double* cy, double* cz, double* diag) {
    const olevel* L = &h->L[l];
    size_t bytes = sizeof(double) * (size_t)L->n;
    if (cx) memcpy(cx, L->cx, bytes);
    if (cy) memcpy(cy, L->cy, bytes);
    if (cz) memcpy(cz, L->cz, bytes);
    if (diag) memcpy(diag, L->diag, bytes);
}

/* uaamg_preconditioner_3d.cpp:216-228 / uaamg_preconditioner.cpp:191-198 */
void oh_vcycle(oh_hier* h, const double* r, double* z) {
    olevel* L0 = &h->L[0];
    for (int i = 1; i <= L0->nx; i++)
        for (int j = 1; j <= L0->ny; j++)
            for (int k = KLO(L0); k <= KHI(L0); k++) {
                long id = cid(L0, i, j, k);
                L0->b[id] = r[id];
            }
    for (int l = 0; l < h->nl; l++) memset(h->L[l].p, 0, sizeof(double) * (size_t)h->L[l].n);
    vcycle(h, 0);
    for (int i = 1; i <= L0->nx; i++)
        for (int j = 1; j <= L0->ny; j++)
            for (int k = KLO(L0); k <= KHI(L0); k++) {
                long id = cid(L0, i, j, k);
                z[id] = L0->p[id];
            }
}

/* ------------------------------------------------------------------------- */
/* PCG (pcg_3d.cpp:18-125, pcg.cpp:18-126)                                    */

typedef struct {
    olevel g;               /* geometry + mask only (p/b/coeff arrays unused) */
    int dirichlet;
    /* 2D variable-coefficient operator (Grid::lap_*, grid.h:23-31), or NULL */
    const double *ld, *lox, *loy;
} ogrid;

static void grid_init(ogrid* G, int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                      const uint8_t* solid, int dirichlet) {
    memset(G, 0, sizeof(*G));
    G->g.nx = nx; G->g.ny = ny; G->g.nz = dim == 3 ? nz : 0;
    G->g.dx = dx; G->g.dy = dy; G->g.dz = dz;
    G->g.sx = nx + 2;
    G->g.sxy = (long)(nx + 2) * (ny + 2);
    G->g.n = dim == 3 ? G->g.sxy * (nz + 2) : G->g.sxy;
    G->g.solid = (uint8_t*)solid;
    G->dirichlet = dirichlet;
}

/* pcg_3d.cpp:38-55 / pcg.cpp:47-59 (uniform-coefficient branch); pcg.cpp:35-46
 * (variable-coefficient branch, 2D: d v_C + ox (v_L + v_R) + oy (v_B + v_T)) */
static void pcg_matvec(const ogrid* G, const double* v, double* av) {
    const olevel* L = &G->g;
    const double idx2 = 1.0 / (L->dx * L->dx), idy2 = 1.0 / (L->dy * L->dy);
    const double idz2 = L->nz ? 1.0 / (L->dz * L->dz) : 0.0;
    const double diag = L->nz ? 2.0 * (idx2 + idy2 + idz2) : 2.0 * (idx2 + idy2);
    const int nx = L->nx, ny = L->ny, nz = L->nz;
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++)
            for (int k = KLO(L); k <= KHI(L); k++) {
                long id = cid(L, i, j, k);
                if (L->solid[id]) { av[id] = 0.0; continue; }
                double vc = v[id];
                double wall = G->dirichlet ? -vc : vc;
                double vL = i > 1 ? (!L->solid[cid(L, i - 1, j, k)] ? v[cid(L, i - 1, j, k)] : vc) : wall;
                double vR = i < nx ? (!L->solid[cid(L, i + 1, j, k)] ? v[cid(L, i + 1, j, k)] : vc) : wall;
                double vB = j > 1 ? (!L->solid[cid(L, i, j - 1, k)] ? v[cid(L, i, j - 1, k)] : vc) : wall;
                double vT = j < ny ? (!L->solid[cid(L, i, j + 1, k)] ? v[cid(L, i, j + 1, k)] : vc) : wall;
                if (nz) {
                    double vF = k > 1 ? (!L->solid[cid(L, i, j, k - 1)] ? v[cid(L, i, j, k - 1)] : vc) : wall;
                    double vK = k < nz ? (!L->solid[cid(L, i, j, k + 1)] ? v[cid(L, i, j, k + 1)] : vc) : wall;
                    av[id] = diag * vc - (vL + vR) * idx2 - (vB + vT) * idy2 - (vF + vK) * idz2;
                } else if (G->ld) {
                    av[id] = G->ld[id] * vc + G->lox[id] * (vL + vR) + G->loy[id] * (vB + vT);
                } else {
                    av[id] = diag * vc - (vL + vR) * idx2 - (vB + vT) * idy2;
                }
            }
}

/* pcg_3d.cpp:57-64 */
static double pcg_dot(const ogrid* G, const double* a, const double* b) {
    const olevel* L = &G->g;
    double s = 0;
    for (int i = 1; i <= L->nx; i++)
        for (int j = 1; j <= L->ny; j++)
            for (int k = KLO(L); k <= KHI(L); k++) {
                long id = cid(L, i, j, k);
                if (!L->solid[id]) s += a[id] * b[id];
            }
    return s;
}

/* pcg_3d.cpp:66-77 */
static void pcg_subtract_mean(const ogrid* G, double* v) {
    if (G->dirichlet) return;
    const olevel* L = &G->g;
    double sum = 0; int count = 0;
    for (int i = 1; i <= L->nx; i++)
        for (int j = 1; j <= L->ny; j++)
            for (int k = KLO(L); k <= KHI(L); k++) {
                long id = cid(L, i, j, k);
                if (!L->solid[id]) { sum += v[id]; count++; }
            }
    double mean = (count > 0) ? sum / count : 0.0;
    for (int i = 1; i <= L->nx; i++)
        for (int j = 1; j <= L->ny; j++)
            for (int k = KLO(L); k <= KHI(L); k++) {
                long id = cid(L, i, j, k);
                if (!L->solid[id]) v[id] -= mean;
            }
}

/* pcg_3d.cpp:22-36 then :80-81 (r = rhs; subtract_mean(r)) */
static void pcg_prepare_rhs(const ogrid* G, const double* rhs_in, double* r) {
    const olevel* L = &G->g;
    memcpy(r, rhs_in, sizeof(double) * (size_t)L->n);
    double sum = 0; int count = 0;
    for (int i = 1; i <= L->nx; i++)
        for (int j = 1; j <= L->ny; j++)
            for (int k = KLO(L); k <= KHI(L); k++) {
                long id = cid(L, i, j, k);
                if (!L->solid[id]) { sum += r[id]; count++; }
            }
    double mean = (count > 0) ? sum / count : 0.0;
    if (G->dirichlet) mean = 0.0;
    for (int i = 1; i <= L->nx; i++)
        for (int j = 1; j <= L->ny; j++)
            for (int k = KLO(L); k <= KHI(L); k++) {
                long id = cid(L, i, j, k);
                if (!L->solid[id]) r[id] = -(r[id] - mean);
            }
    pcg_subtract_mean(G, r);
}

void oracle_pcg_rhs(int dim, int nx, int ny, int nz, const uint8_t* solid,
                    const double* rhs, double* b, int dirichlet) {
    ogrid G;
    grid_init(&G, dim, nx, ny, nz, 1.0, 1.0, 1.0, solid, dirichlet);
    pcg_prepare_rhs(&G, rhs, b);
}

void oracle_matvec(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                   const uint8_t* solid, const double* x, double* ax, int dirichlet) {
    ogrid G;
    grid_init(&G, dim, nx, ny, nz, dx, dy, dz, solid, dirichlet);
    memset(ax, 0, sizeof(double) * (size_t)G.g.n);
    pcg_matvec(&G, x, ax);
}

double oracle_true_residual(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                            const uint8_t* solid, const double* rhs, const double* x,
                            int dirichlet, double* bnorm) {
    ogrid G;
    grid_init(&G, dim, nx, ny, nz, dx, dy, dz, solid, dirichlet);
    size_t n = (size_t)G.g.n;
    double* b = (double*)calloc(n, sizeof(double));
    double* ax = (double*)calloc(n, sizeof(double));
    pcg_prepare_rhs(&G, rhs, b);
    pcg_matvec(&G, x, ax);
    for (size_t c = 0; c < n; c++) ax[c] = b[c] - ax[c];
    double rr = pcg_dot(&G, ax, ax);
    if (bnorm) *bnorm = sqrt(pcg_dot(&G, b, b));
    free(b); free(ax);
    return sqrt(rr);
}

static int pcg_impl(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                    const uint8_t* solid, const double* ld, const double* lox,
                    const double* loy, const double* rhs_in, double* x, int max_iter,
                    double tol, int precond, int tol_mode, int warm, int dirichlet,
                    double* hist, int* status) {
    ogrid G;
    grid_init(&G, dim, nx, ny, nz, dx, dy, dz, solid, dirichlet);
    G.ld = ld; G.lox = lox; G.loy = loy;
    const size_t n = (size_t)G.g.n;
    double* r = (double*)calloc(n, sizeof(double));
    double* z = (double*)calloc(n, sizeof(double));
    double* p = (double*)calloc(n, sizeof(double));
    double* ap = (double*)calloc(n, sizeof(double));
    oh_hier* h = precond ? oh_create(dim, nx, ny, nz, dx, dy, dz, solid, dirichlet) : NULL;
    const olevel* L = &G.g;
    int updates = 0, st = 1;

    pcg_prepare_rhs(&G, rhs_in, r);
    const double bnorm = sqrt(pcg_dot(&G, r, r));
    if (warm) {                      /* r0 = b - A x0 (not in the reference) */
        pcg_matvec(&G, x, ap);
        for (int i = 1; i <= L->nx; i++)
            for (int j = 1; j <= L->ny; j++)
                for (int k = KLO(L); k <= KHI(L); k++) {
                    long id = cid(L, i, j, k);
                    if (!L->solid[id]) r[id] -= ap[id];
                }
        pcg_subtract_mean(&G, r);
    }
    double r0 = sqrt(pcg_dot(&G, r, r));
    double tol_abs = tol_mode ? tol * bnorm : tol;
    if (hist) hist[0] = r0;

    if (precond) oh_vcycle(h, r, z); else memcpy(z, r, sizeof(double) * n);
    pcg_subtract_mean(&G, z);
    memcpy(p, z, sizeof(double) * n);
    double rsold = pcg_dot(&G, r, z);

    for (int it = 0; it < max_iter; it++) {
        pcg_matvec(&G, p, ap);
        double pap = pcg_dot(&G, p, ap);
        /* pcg_3d.cpp:97 (absolute 1e-15); the relative mode only stops on a
         * non-positive p.Ap, since 1e-15 is scale-dependent */
        if (pap < (tol_mode ? 1e-300 : 1e-15)) { st = 2; break; }
        double alpha = rsold / pap;
        for (int i = 1; i <= L->nx; i++)
            for (int j = 1; j <= L->ny; j++)
                for (int k = KLO(L); k <= KHI(L); k++) {
                    long id = cid(L, i, j, k);
                    if (!L->solid[id]) {
                        x[id] += alpha * p[id];
                        r[id] -= alpha * ap[id];
                    }
                }
        updates++;
        double rsnew = pcg_dot(&G, r, r);
        if (hist) hist[updates] = sqrt(rsnew);
        if (sqrt(rsnew) < tol_abs) { st = 0; break; }
        if (precond) oh_vcycle(h, r, z); else memcpy(z, r, sizeof(double) * n);
        pcg_subtract_mean(&G, z);
        double beta = pcg_dot(&G, r, z) / rsold;
        for (int i = 1; i <= L->nx; i++)
            for (int j = 1; j <= L->ny; j++)
                for (int k = KLO(L); k <= KHI(L); k++) {
                    long id = cid(L, i, j, k);
                    if (!L->solid[id]) p[id] = z[id] + beta * p[id];
                }
        rsold = pcg_dot(&G, r, z);
    }
    if (status) *status = st;
    oh_destroy(h);
    free(r); free(z); free(p); free(ap);
    return updates;
}

int oracle_pcg(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
               const uint8_t* solid, const double* rhs_in, double* x, int max_iter,
               double tol, int precond, int tol_mode, int warm, int dirichlet,
               double* hist, int* status) {
    return pcg_impl(dim, nx, ny, nz, dx, dy, dz, solid, NULL, NULL, NULL, rhs_in, x, max_iter,
                    tol, precond, tol_mode, warm, dirichlet, hist, status);
}

/* ------------------------------------------------------------------------- */
/* Variable-coefficient Laplacian (Grid::lap_*, pcg.cpp:35-46), 2D            */

int oracle_pcg_var_2d(int nx, int ny, double dx, double dy, const uint8_t* solid,
                      const double* lap_diag, const double* lap_off_x, const double* lap_off_y,
                      const double* rhs_in, double* x, int max_iter, double tol, int precond,
                      int tol_mode, int warm, double* hist, int* status) {
    return pcg_impl(2, nx, ny, 0, dx, dy, 1.0, solid, lap_diag, lap_off_x, lap_off_y, rhs_in, x,
                    max_iter, tol, precond, tol_mode, warm, 0, hist, status);
}

void oracle_matvec_var_2d(int nx, int ny, const uint8_t* solid, const double* lap_diag,
                          const double* lap_off_x, const double* lap_off_y, const double* x,
                          double* ax) {
    ogrid G;
    grid_init(&G, 2, nx, ny, 0, 1.0, 1.0, 1.0, solid, 0);
    G.ld = lap_diag; G.lox = lap_off_x; G.loy = lap_off_y;
    memset(ax, 0, sizeof(double) * (size_t)G.g.n);
    pcg_matvec(&G, x, ax);
}

double oracle_true_residual_var_2d(int nx, int ny, const uint8_t* solid, const double* lap_diag,
                                   const double* lap_off_x, const double* lap_off_y,
                                   const double* rhs, const double* x, double* bnorm) {
    ogrid G;
    grid_init(&G, 2, nx, ny, 0, 1.0, 1.0, 1.0, solid, 0);
    G.ld = lap_diag; G.lox = lap_off_x; G.loy = lap_off_y;
    size_t n = (size_t)G.g.n;
    double* b = (double*)calloc(n, sizeof(double));
    double* ax = (double*)calloc(n, sizeof(double));
    pcg_prepare_rhs(&G, rhs, b);
    pcg_matvec(&G, x, ax);
    for (size_t c = 0; c < n; c++) ax[c] = b[c] - ax[c];
    double rr = pcg_dot(&G, ax, ax);
    if (bnorm) *bnorm = sqrt(pcg_dot(&G, b, b));
    free(b); free(ax);
    return sqrt(rr);
}

/* SmoothCylinder::applyToLaplacian (cylinder_model.cpp:5-10, 40-48, 50-71): solid
 * fraction phi = smoothstep((r - R) / tw) of the cell centre; phi > 0.9 marks the
 * cell solid (diag 1e15, no couplings); otherwise face permeabilities
 * c = 1 - (phi + phi_nb)/2 + 0.1 give diag = (cL + cR)/dx^2 + (cB + cT)/dy^2 and
 * off_x = -(cL + cR)/(2 dx^2), off_y = -(cB + cT)/(2 dy^2).  inside != 0 flips the
 * fraction to smoothstep((R - r) / tw), solid inside the disk.  Interior cells
 * only; solid is OR-ed, the ghost coefficients are left as they are. */
static double oc_smoothstep(double t) {
    if (t <= -1.0) return 0.0;
    if (t >= 1.0) return 1.0;
    double s = (t + 1.0) * 0.5;
    return s * s * (3.0 - 2.0 * s);
}

static double oc_frac(double cx, double cy, double R, double tw, int inside, double x, double y) {
    double r = sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy));
    return oc_smoothstep(inside ? (R - r) / tw : (r - R) / tw);
}

void oracle_smooth_cylinder_2d(int nx, int ny, double dx, double dy, double cx, double cy,
                               double R, double tw, int inside, uint8_t* solid, double* diag,
                               double* ox, double* oy) {
    const double eps = 0.1, large = 1e15;
    if (!(tw > 0)) tw = dx;
    for (int j = 1; j <= ny; j++)
        for (int i = 1; i <= nx; i++) {
            long idx = i + (long)j * (nx + 2);
            double xc = (i - 0.5) * dx, yc = (j - 0.5) * dy;
            double phi = oc_frac(cx, cy, R, tw, inside, xc, yc);
            if (phi > 0.9) {
                solid[idx] = 1;
                diag[idx] = large; ox[idx] = 0; oy[idx] = 0;
            } else {
                double pL = oc_frac(cx, cy, R, tw, inside, xc - dx, yc);
                double pR = oc_frac(cx, cy, R, tw, inside, xc + dx, yc);
                double pB = oc_frac(cx, cy, R, tw, inside, xc, yc - dy);
                double pT = oc_frac(cx, cy, R, tw, inside, xc, yc + dy);
                double cL = 1.0 - 0.5 * (phi + pL) + eps, cR = 1.0 - 0.5 * (phi + pR) + eps;
                double cB = 1.0 - 0.5 * (phi + pB) + eps, cT = 1.0 - 0.5 * (phi + pT) + eps;
                double ix = 1.0 / (dx * dx), iy = 1.0 / (dy * dy);
                diag[idx] = (cL + cR) * ix + (cB + cT) * iy;
                ox[idx] = -0.5 * (cL + cR) * ix;
                oy[idx] = -0.5 * (cB + cT) * iy;
            }
        }
}

/* ------------------------------------------------------------------------- */
/* Pressure projection pieces (pressure.cpp:10-14, 21-32; pressure_3d.cpp:10-15, 21-39) */

void oracle_divergence_rhs(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                           const uint8_t* solid, const double* u, const double* v,
                           const double* w, double dt, double* rhs) {
    ogrid G;
    grid_init(&G, dim, nx, ny, nz, dx, dy, dz, solid, 0);
    const olevel* L = &G.g;
    memset(rhs, 0, sizeof(double) * (size_t)L->n);
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++)
            for (int k = KLO(L); k <= KHI(L); k++) {
                long id = cid(L, i, j, k);
                if (L->solid[id]) continue;
                if (dim == 3) {
                    /* operators_3d.h:17-21; u index iu = i + j(nx+1) + k(nx+1)(ny+2) */
                    long su = nx + 1, suv = (long)(nx + 1) * (ny + 2);
                    long sv = nx + 2, svv = (long)(nx + 2) * (ny + 1);
                    long sw = nx + 2, sww = (long)(nx + 2) * (ny + 2);
                    double div = (u[i + j * su + k * suv] - u[(i - 1) + j * su + k * suv]) / dx
                               + (v[i + j * sv + k * svv] - v[i + (j - 1) * sv + k * svv]) / dy
                               + (w[i + j * sw + k * sww] - w[i + j * sw + (k - 1) * sww]) / dz;
                    rhs[id] = div / dt;
                } else {
                    /* operators.h:18-21 */
                    long su = nx + 1, sv = nx + 2;
                    double div = (u[i + j * su] - u[(i - 1) + j * su]) / dx
                               + (v[i + j * sv] - v[i + (j - 1) * sv]) / dy;
                    rhs[id] = div / dt;
                }
            }
}

void oracle_correct_velocity(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                             const uint8_t* solid, const double* p, double dt,
                             double* u, double* v, double* w) {
    ogrid G;
    grid_init(&G, dim, nx, ny, nz, dx, dy, dz, solid, 0);
    const olevel* L = &G.g;
    if (dim == 2) {
        long su = nx + 1, sv = nx + 2;
        for (int i = 1; i < nx; i++)
            for (int j = 1; j <= ny; j++) {
                if (L->solid[cid(L, i, j, 0)] || L->solid[cid(L, i + 1, j, 0)]) continue;
                u[i + j * su] -= dt * (p[cid(L, i + 1, j, 0)] - p[cid(L, i, j, 0)]) / dx;
            }
        for (int i = 1; i <= nx; i++)
            for (int j = 1; j < ny; j++) {
                if (L->solid[cid(L, i, j, 0)] || L->solid[cid(L, i, j + 1, 0)]) continue;
                v[i + j * sv] -= dt * (p[cid(L, i, j + 1, 0)] - p[cid(L, i, j, 0)]) / dy;
            }
        return;
    }
    long su = nx + 1, suv = (long)(nx + 1) * (ny + 2);
    long sv = nx + 2, svv = (long)(nx + 2) * (ny + 1);
    long sw = nx + 2, sww = (long)(nx + 2) * (ny + 2);
    for (int k = 1; k <= nz; k++)
        for (int j = 1; j <= ny; j++)
            for (int i = 1; i < nx; i++) {
                if (L->solid[cid(L, i, j, k)] || L->solid[cid(L, i + 1, j, k)]) continue;
                u[i + j * su + k * suv] -= dt * (p[cid(L, i + 1, j, k)] - p[cid(L, i, j, k)]) / dx;
            }
    for (int k = 1; k <= nz; k++)
        for (int j = 1; j < ny; j++)
            for (int i = 1; i <= nx; i++) {
                if (L->solid[cid(L, i, j, k)] || L->solid[cid(L, i, j + 1, k)]) continue;
                v[i + j * sv + k * svv] -= dt * (p[cid(L, i, j + 1, k)] - p[cid(L, i, j, k)]) / dy;
            }
    for (int k = 1; k < nz; k++)
        for (int j = 1; j <= ny; j++)
            for (int i = 1; i <= nx; i++) {
                if (L->solid[cid(L, i, j, k)] || L->solid[cid(L, i, j, k + 1)]) continue;
                w[i + j * sw + k * sww] -= dt * (p[cid(L, i, j, k + 1)] - p[cid(L, i, j, k)]) / dz;
            }
}

/* RHS of PressureProjection::recoverStaticPressure (pressure.cpp:35-66), 2D:
 * rhs = -(du/dx^2 + 2 du/dy dv/dx + dv/dy^2) on fluid cells, with cell-centre
 * velocities uc, vc at indices clamped to the interior and the cross derivatives
 * dropped next to a solid (up/down for du/dy, left/right for dv/dx). */
static double os_uc(const double* u, int nx, int ny, int i, int j) {
    i = i < 1 ? 1 : (i > nx ? nx : i);
    j = j < 1 ? 1 : (j > ny ? ny : j);
    const long su = nx + 1;
    return 0.5 * (u[i + j * su] + u[(i - 1) + j * su]);
}
static double os_vc(const double* v, int nx, int ny, int i, int j) {
    i = i < 1 ? 1 : (i > nx ? nx : i);
    j = j < 1 ? 1 : (j > ny ? ny : j);
    const long sv = nx + 2;
    return 0.5 * (v[i + j * sv] + v[i + (j - 1) * sv]);
}

void oracle_static_rhs_2d(int nx, int ny, double dx, double dy, const uint8_t* solid,
                          const double* u, const double* v, double* rhs) {
    const long sp = nx + 2, su = nx + 1, sv = nx + 2;
    memset(rhs, 0, sizeof(double) * (size_t)(nx + 2) * (ny + 2));
    for (int i = 1; i <= nx; i++)
        for (int j = 1; j <= ny; j++) {
            if (solid[i + j * sp]) continue;
            double du_dx = (u[i + j * su] - u[(i - 1) + j * su]) / dx;
            double dv_dy = (v[i + j * sv] - v[i + (j - 1) * sv]) / dy;
            int sL = solid[(i - 1) + j * sp] != 0, sR = solid[(i + 1) + j * sp] != 0;
            int sB = solid[i + (j - 1) * sp] != 0, sT = solid[i + (j + 1) * sp] != 0;
            double du_dy = (sB || sT) ? 0.0
                                      : (os_uc(u, nx, ny, i, j + 1) - os_uc(u, nx, ny, i, j - 1)) / (2 * dy);
            double dv_dx = (sL || sR) ? 0.0
                                      : (os_vc(v, nx, ny, i + 1, j) - os_vc(v, nx, ny, i - 1, j)) / (2 * dx);
            rhs[i + j * sp] = -(du_dx * du_dx + 2.0 * du_dy * dv_dx + dv_dy * dv_dy);
        }
}
