/* ORACLE / TEST INFRASTRUCTURE — CPU restatement of QUILL's per-timestep
 * particle-in-cell loop (QUILL-PIC/Quill, n_sr = 1, QED off for whole steps;
 * the QED rate functions and the random stream are restated for unit tests).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * this file, and only as the checker.  It is pinned bit-for-bit against the
 * reference's own sources (oracle/_ref, built by `make -C oracle ref`) in
 * tests/test_oracle_vs_ref.py and against tests/golden/*.npz.
 *
 * Data layout of the restatement (not the reference's): one structure-of-
 * arrays particle store holding every species, kept in the reference's
 * traversal order — cells lexicographic (i, j, k; k fastest) and, inside a
 * cell, the order of the cell's linked list from its head.  The reference's
 * relinking (plist.cpp:7-39, head insertion of movers, advance.cpp:377-386
 * start = head) is restated as an array rule:
 *   new list of cell c = [particles that arrived in c, in DESCENDING
 *                         traversal order] ++ [particles that stayed in c,
 *                         in ASCENDING traversal order]
 * Arithmetic follows the reference expression by expression (same operand
 * association; the library is built with -ffp-contract=off), so sums of the
 * current J are formed in the same order and results are bit-identical.
 */
#include "qp_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI_ 3.141592653589793

struct qor_region {
    int nx, ny, nz;
    long nc;
    double dx, dy, dz, dt, dtdx, dtdy, dtdz, lam, e_s;
    int solver, pusher, qed;
    int n_ion;
    double icmr[16];
    /* fields: planes E(0..2) B(3..5) J(6..8) Bbar(9..11) */
    double* f[12];
    /* particles */
    long n, cap;
    double *x, *y, *z, *ux, *uy, *uz, *g, *q, *cmr, *chi;
    long* cell;
    /* lagged Fibonacci stream, mc.cpp:12-23 */
    double rnd[55];
    int n_random;
    /* solver coefficients */
    double fp_ax, fp_ay, fp_az, fp_bx, fp_by, fp_bz;   /* five-point, maxwell.cpp:24-33 */
    double nd_ax, nd_bx, nd_ay, nd_by, nd_az, nd_bz;   /* NDFX, maxwell.cpp:238-249 */
    /* diagnostics: cells with i in [dlo, dhi) (compute_N's n1, n2) */
    double diag[10 + 32];
    int dlo, dhi;
};

#define IDX(r, i, j, k) ((((long)(i)) * (r)->ny + (j)) * (r)->nz + (k))
#define EX(r) ((r)->f[0])
#define EY(r) ((r)->f[1])
#define EZ(r) ((r)->f[2])
#define BX(r) ((r)->f[3])
#define BY(r) ((r)->f[4])
#define BZ(r) ((r)->f[5])
#define JX(r) ((r)->f[6])
#define JY(r) ((r)->f[7])
#define JZ(r) ((r)->f[8])
#define BEX(r) ((r)->f[9])
#define BEY(r) ((r)->f[10])
#define BEZ(r) ((r)->f[11])

static void grow(qor_region* r, long need) {
    if (need <= r->cap) return;
    long c = r->cap ? r->cap : 1024;
    while (c < need) c *= 2;
    double** arrs[10] = {&r->x, &r->y, &r->z, &r->ux, &r->uy, &r->uz, &r->g, &r->q, &r->cmr, &r->chi};
    for (int a = 0; a < 10; a++) *arrs[a] = (double*)realloc(*arrs[a], sizeof(double) * c);
    r->cell = (long*)realloc(r->cell, sizeof(long) * c);
    r->cap = c;
}

qor_region* qor_create(int nx, int ny, int nz, double dx, double dy, double dz, double dt,
                       double lambda_cm, int solver, int pusher, int qed, int n_ion,
                       const double* icmr, int seed) {
    qor_region* r = (qor_region*)calloc(1, sizeof(qor_region));
    r->nx = nx; r->ny = ny; r->nz = nz;
    r->nc = (long)nx * ny * nz;
    r->dlo = 0; r->dhi = nx;
    r->dx = dx; r->dy = dy; r->dz = dz; r->dt = dt;
    /* maxwell.cpp:6-8 */
    r->dtdx = dt / dx; r->dtdy = dt / dy; r->dtdz = dt / dz;
    r->lam = lambda_cm;
    r->e_s = lambda_cm / 2.4263086e-10; /* main.cpp:2276 */
    r->solver = solver; r->pusher = pusher; r->qed = qed;
    r->n_ion = n_ion;
    for (int i = 0; i < n_ion && i < 16; i++) r->icmr[i] = icmr[i];
    for (int a = 0; a < 12; a++) r->f[a] = (double*)calloc(r->nc, sizeof(double));
    /* five-point coefficients, maxwell.cpp:24-33 */
    r->fp_ax = 0.25 * (1 - dx / dt * sin(0.5 * PI_ * fmin(1.0, dt / dx)));
    r->fp_ay = 0.25 * (1 - dy / dt * sin(0.5 * PI_ * fmin(1.0, dt / dy)));
    r->fp_az = 0.25 * (1 - dz / dt * sin(0.5 * PI_ * fmin(1.0, dt / dz)));
    r->fp_bx = 1 - 2 * r->fp_ax;
    r->fp_by = 1 - 2 * r->fp_ay;
    r->fp_bz = 1 - 2 * r->fp_az;
    /* NDFX coefficients, maxwell.cpp:238-249 */
    {
        double kappa = 1.25 * (sqrt(3) - 1) * 0.5 / sqrt(3);
        r->nd_bx = (1 - kappa);
        r->nd_ax = 0.5 * (1 - r->nd_bx);
        r->nd_by = 1 - kappa * dx * dx / (dy * dy);
        r->nd_bz = 1 - kappa * dx * dx / (dz * dz);
        r->nd_ay = 0.5 * (1 - r->nd_by);
        r->nd_az = 0.5 * (1 - r->nd_bz);
    }
    /* random stream initialisation, low-level.cpp:131-137 */
    srand(seed);
    for (int i = 0; i < 55; i++) r->rnd[i] = (double)rand() / (double)RAND_MAX;
    r->n_random = 0;
    return r;
}

void qor_destroy(qor_region* r) {
    if (!r) return;
    for (int a = 0; a < 12; a++) free(r->f[a]);
    free(r->x); free(r->y); free(r->z); free(r->ux); free(r->uy); free(r->uz);
    free(r->g); free(r->q); free(r->cmr); free(r->chi); free(r->cell);
    free(r);
}

void qor_set_fields(qor_region* r, const double* ex, const double* ey, const double* ez,
                    const double* bx, const double* by, const double* bz) {
    size_t s = sizeof(double) * r->nc;
    memcpy(EX(r), ex, s); memcpy(EY(r), ey, s); memcpy(EZ(r), ez, s);
    memcpy(BX(r), bx, s); memcpy(BY(r), by, s); memcpy(BZ(r), bz, s);
}

void qor_get_fields(qor_region* r, double* out) {
    for (int a = 0; a < 12; a++) memcpy(out + a * r->nc, r->f[a], sizeof(double) * r->nc);
}

/* ------------------------------------------------------------------------ */
/* B at E positions, advance.cpp:20-83                                       */
/* ------------------------------------------------------------------------ */
static double bex8(qor_region* r, int i, int j, int k) {
    const double* b = BX(r);
    return 0.125 * (b[IDX(r, i, j, k)] + b[IDX(r, i + 1, j, k)] + b[IDX(r, i, j, k - 1)] +
                    b[IDX(r, i + 1, j, k - 1)] + b[IDX(r, i, j - 1, k)] + b[IDX(r, i + 1, j - 1, k)] +
                    b[IDX(r, i, j - 1, k - 1)] + b[IDX(r, i + 1, j - 1, k - 1)]);
}
static double bey8(qor_region* r, int i, int j, int k) {
    const double* b = BY(r);
    return 0.125 * (b[IDX(r, i, j, k)] + b[IDX(r, i - 1, j, k)] + b[IDX(r, i, j, k - 1)] +
                    b[IDX(r, i - 1, j, k - 1)] + b[IDX(r, i, j + 1, k)] + b[IDX(r, i - 1, j + 1, k)] +
                    b[IDX(r, i, j + 1, k - 1)] + b[IDX(r, i - 1, j + 1, k - 1)]);
}
static double bez8(qor_region* r, int i, int j, int k) {
    const double* b = BZ(r);
    return 0.125 * (b[IDX(r, i, j, k)] + b[IDX(r, i - 1, j, k)] + b[IDX(r, i, j, k + 1)] +
                    b[IDX(r, i - 1, j, k + 1)] + b[IDX(r, i, j - 1, k)] + b[IDX(r, i - 1, j - 1, k)] +
                    b[IDX(r, i, j - 1, k + 1)] + b[IDX(r, i - 1, j - 1, k + 1)]);
}

static void interpolate_be(qor_region* r) {
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    const double *bx = BX(r), *by = BY(r), *bz = BZ(r);
    double *ex = BEX(r), *ey = BEY(r), *ez = BEZ(r);
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++)
            for (int k = 1; k < nz - 1; k++) {
                long c = IDX(r, i, j, k);
                ex[c] = bex8(r, i, j, k);
                ey[c] = bey8(r, i, j, k);
                ez[c] = bez8(r, i, j, k);
            }
    /* x faces */
    for (int j = 1; j < ny - 1; j++)
        for (int k = 1; k < nz - 1; k++) {
            int i = 0;
            long c = IDX(r, i, j, k);
            ex[c] = bex8(r, i, j, k);
            ey[c] = 0.25 * (by[IDX(r, i, j, k)] + by[IDX(r, i, j, k - 1)] + by[IDX(r, i, j + 1, k)] + by[IDX(r, i, j + 1, k - 1)]);
            ez[c] = 0.25 * (bz[IDX(r, i, j, k)] + bz[IDX(r, i, j, k + 1)] + bz[IDX(r, i, j - 1, k)] + bz[IDX(r, i, j - 1, k + 1)]);
            i = nx - 1;
            c = IDX(r, i, j, k);
            ex[c] = 0.25 * (bx[IDX(r, i, j, k)] + bx[IDX(r, i, j, k - 1)] + bx[IDX(r, i, j - 1, k)] + bx[IDX(r, i, j - 1, k - 1)]);
            ey[c] = bey8(r, i, j, k);
            ez[c] = bez8(r, i, j, k);
        }
    /* y faces */
    for (int i = 1; i < nx - 1; i++)
        for (int k = 1; k < nz - 1; k++) {
            int j = 0;
            long c = IDX(r, i, j, k);
            ex[c] = 0.25 * (bx[IDX(r, i, j, k)] + bx[IDX(r, i + 1, j, k)] + bx[IDX(r, i, j, k - 1)] + bx[IDX(r, i + 1, j, k - 1)]);
            ey[c] = bey8(r, i, j, k);
            ez[c] = 0.25 * (bz[IDX(r, i, j, k)] + bz[IDX(r, i - 1, j, k)] + bz[IDX(r, i, j, k + 1)] + bz[IDX(r, i - 1, j, k + 1)]);
            j = ny - 1;
            c = IDX(r, i, j, k);
            ex[c] = bex8(r, i, j, k);
            ey[c] = 0.25 * (by[IDX(r, i, j, k)] + by[IDX(r, i - 1, j, k)] + by[IDX(r, i, j, k - 1)] + by[IDX(r, i - 1, j, k - 1)]);
            ez[c] = bez8(r, i, j, k);
        }
    /* z faces */
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++) {
            int k = 0;
            long c = IDX(r, i, j, k);
            ex[c] = 0.25 * (bx[IDX(r, i, j, k)] + bx[IDX(r, i + 1, j, k)] + bx[IDX(r, i, j - 1, k)] + bx[IDX(r, i + 1, j - 1, k)]);
            ey[c] = 0.25 * (by[IDX(r, i, j, k)] + by[IDX(r, i - 1, j, k)] + by[IDX(r, i, j + 1, k)] + by[IDX(r, i - 1, j + 1, k)]);
            ez[c] = bez8(r, i, j, k);
            k = nz - 1;
            c = IDX(r, i, j, k);
            ex[c] = bex8(r, i, j, k);
            ey[c] = bey8(r, i, j, k);
            ez[c] = 0.25 * (bz[IDX(r, i, j, k)] + bz[IDX(r, i - 1, j, k)] + bz[IDX(r, i, j - 1, k)] + bz[IDX(r, i - 1, j - 1, k)]);
        }
}

/* ------------------------------------------------------------------------ */
/* Maxwell solvers, maxwell.cpp:10-597                                       */
/* ------------------------------------------------------------------------ */
#define E_(a, i, j, k) r->f[a][IDX(r, i, j, k)]
#define B_(a, i, j, k) r->f[3 + (a)][IDX(r, i, j, k)]
#define J_(a, i, j, k) r->f[6 + (a)][IDX(r, i, j, k)]

/* FDTD, maxwell.cpp:445-522: 2-point curl, update ranges [1, n-1) plus the
 * low faces for the components tangential to them. */
static void fdtd_bx(qor_region* r, int i, int j, int k) {
    B_(0, i, j, k) += 0.5 * (-r->dtdy * (E_(2, i, j + 1, k) - E_(2, i, j, k)) + r->dtdz * (E_(1, i, j, k + 1) - E_(1, i, j, k)));
}
static void fdtd_by(qor_region* r, int i, int j, int k) {
    B_(1, i, j, k) += 0.5 * (r->dtdx * (E_(2, i + 1, j, k) - E_(2, i, j, k)) - r->dtdz * (E_(0, i, j, k + 1) - E_(0, i, j, k)));
}
static void fdtd_bz(qor_region* r, int i, int j, int k) {
    B_(2, i, j, k) += 0.5 * (r->dtdy * (E_(0, i, j + 1, k) - E_(0, i, j, k)) - r->dtdx * (E_(1, i + 1, j, k) - E_(1, i, j, k)));
}
static void fdtd_ex(qor_region* r, int i, int j, int k) {
    E_(0, i, j, k) += r->dtdy * (B_(2, i, j, k) - B_(2, i, j - 1, k)) - r->dtdz * (B_(1, i, j, k) - B_(1, i, j, k - 1)) - J_(0, i, j, k) * r->dx;
}
static void fdtd_ey(qor_region* r, int i, int j, int k) {
    E_(1, i, j, k) += -r->dtdx * (B_(2, i, j, k) - B_(2, i - 1, j, k)) + r->dtdz * (B_(0, i, j, k) - B_(0, i, j, k - 1)) - J_(1, i, j, k) * r->dy;
}
static void fdtd_ez(qor_region* r, int i, int j, int k) {
    E_(2, i, j, k) += r->dtdx * (B_(1, i, j, k) - B_(1, i - 1, j, k)) - r->dtdy * (B_(0, i, j, k) - B_(0, i, j - 1, k)) - J_(2, i, j, k) * r->dz;
}
static void fdtd_advance_b(qor_region* r) {
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++)
            for (int k = 1; k < nz - 1; k++) { fdtd_bx(r, i, j, k); fdtd_by(r, i, j, k); fdtd_bz(r, i, j, k); }
    for (int j = 1; j < ny - 1; j++)
        for (int k = 1; k < nz - 1; k++) { fdtd_by(r, 0, j, k); fdtd_bz(r, 0, j, k); }
    for (int i = 1; i < nx - 1; i++)
        for (int k = 1; k < nz - 1; k++) { fdtd_bx(r, i, 0, k); fdtd_bz(r, i, 0, k); }
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++) { fdtd_bx(r, i, j, 0); fdtd_by(r, i, j, 0); }
}
static void fdtd_advance_e(qor_region* r) {
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++)
            for (int k = 1; k < nz - 1; k++) { fdtd_ex(r, i, j, k); fdtd_ey(r, i, j, k); fdtd_ez(r, i, j, k); }
    for (int j = 1; j < ny - 1; j++)
        for (int k = 1; k < nz - 1; k++) fdtd_ex(r, 0, j, k);
    for (int i = 1; i < nx - 1; i++)
        for (int k = 1; k < nz - 1; k++) fdtd_ey(r, i, 0, k);
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++) fdtd_ez(r, i, j, 0);
}

/* NDFX, maxwell.cpp:251-328: curl smoothed transversely (coefficients
 * kappa, a, b); update ranges [2, n-1) plus the i/j/k = 1 planes. */
static void ndfx_bx(qor_region* r, int i, int j, int k) {
    B_(0, i, j, k) += 0.5 * (-r->dtdy * (r->nd_bz * (E_(2, i, j + 1, k) - E_(2, i, j, k)) + r->nd_az * (E_(2, i, j + 1, k + 1) - E_(2, i, j, k + 1) + E_(2, i, j + 1, k - 1) - E_(2, i, j, k - 1))) +
                             r->dtdz * (r->nd_by * (E_(1, i, j, k + 1) - E_(1, i, j, k)) + r->nd_ay * (E_(1, i, j + 1, k + 1) - E_(1, i, j + 1, k) + E_(1, i, j - 1, k + 1) - E_(1, i, j - 1, k))));
}
static void ndfx_by(qor_region* r, int i, int j, int k) {
    B_(1, i, j, k) += 0.5 * (r->dtdx * (r->nd_bz * (E_(2, i + 1, j, k) - E_(2, i, j, k)) + r->nd_az * (E_(2, i + 1, j, k + 1) - E_(2, i, j, k + 1) + E_(2, i + 1, j, k - 1) - E_(2, i, j, k - 1))) -
                             r->dtdz * (r->nd_bx * (E_(0, i, j, k + 1) - E_(0, i, j, k)) + r->nd_ax * (E_(0, i + 1, j, k + 1) - E_(0, i + 1, j, k) + E_(0, i - 1, j, k + 1) - E_(0, i - 1, j, k))));
}
static void ndfx_bz(qor_region* r, int i, int j, int k) {
    B_(2, i, j, k) += 0.5 * (r->dtdy * (r->nd_bx * (E_(0, i, j + 1, k) - E_(0, i, j, k)) + r->nd_ax * (E_(0, i + 1, j + 1, k) - E_(0, i + 1, j, k) + E_(0, i - 1, j + 1, k) - E_(0, i - 1, j, k))) -
                             r->dtdx * (r->nd_by * (E_(1, i + 1, j, k) - E_(1, i, j, k)) + r->nd_ay * (E_(1, i + 1, j + 1, k) - E_(1, i, j + 1, k) + E_(1, i + 1, j - 1, k) - E_(1, i, j - 1, k))));
}
static void ndfx_ex(qor_region* r, int i, int j, int k) {
    E_(0, i, j, k) = E_(0, i, j, k) + r->dtdy * (r->nd_bz * (B_(2, i, j, k) - B_(2, i, j - 1, k)) + r->nd_az * (B_(2, i, j, k + 1) - B_(2, i, j - 1, k + 1) + B_(2, i, j, k - 1) - B_(2, i, j - 1, k - 1))) -
                     r->dtdz * (r->nd_by * (B_(1, i, j, k) - B_(1, i, j, k - 1)) + r->nd_ay * (B_(1, i, j + 1, k) - B_(1, i, j + 1, k - 1) + B_(1, i, j - 1, k) - B_(1, i, j - 1, k - 1))) -
                     J_(0, i, j, k) * r->dx;
}
static void ndfx_ey(qor_region* r, int i, int j, int k) {
    E_(1, i, j, k) = E_(1, i, j, k) - r->dtdx * (r->nd_bz * (B_(2, i, j, k) - B_(2, i - 1, j, k)) + r->nd_az * (B_(2, i, j, k + 1) - B_(2, i - 1, j, k + 1) + B_(2, i, j, k - 1) - B_(2, i - 1, j, k - 1))) +
                     r->dtdz * (r->nd_bx * (B_(0, i, j, k) - B_(0, i, j, k - 1)) + r->nd_ax * (B_(0, i + 1, j, k) - B_(0, i + 1, j, k - 1) + B_(0, i - 1, j, k) - B_(0, i - 1, j, k - 1))) -
                     J_(1, i, j, k) * r->dy;
}
static void ndfx_ez(qor_region* r, int i, int j, int k) {
    E_(2, i, j, k) = E_(2, i, j, k) + r->dtdx * (r->nd_by * (B_(1, i, j, k) - B_(1, i - 1, j, k)) + r->nd_ay * (B_(1, i, j + 1, k) - B_(1, i - 1, j + 1, k) + B_(1, i, j - 1, k) - B_(1, i - 1, j - 1, k))) -
                     r->dtdy * (r->nd_bx * (B_(0, i, j, k) - B_(0, i, j - 1, k)) + r->nd_ax * (B_(0, i + 1, j, k) - B_(0, i + 1, j - 1, k) + B_(0, i - 1, j, k) - B_(0, i - 1, j - 1, k))) -
                     J_(2, i, j, k) * r->dz;
}
static void ndfx_advance_b(qor_region* r) {
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    for (int i = 2; i < nx - 1; i++)
        for (int j = 2; j < ny - 1; j++)
            for (int k = 2; k < nz - 1; k++) { ndfx_bx(r, i, j, k); ndfx_by(r, i, j, k); ndfx_bz(r, i, j, k); }
    for (int j = 2; j < ny - 1; j++)
        for (int k = 2; k < nz - 1; k++) { ndfx_by(r, 1, j, k); ndfx_bz(r, 1, j, k); }
    for (int i = 2; i < nx - 1; i++)
        for (int k = 2; k < nz - 1; k++) { ndfx_bx(r, i, 1, k); ndfx_bz(r, i, 1, k); }
    for (int i = 2; i < nx - 1; i++)
        for (int j = 2; j < ny - 1; j++) { ndfx_bx(r, i, j, 1); ndfx_by(r, i, j, 1); }
}
static void ndfx_advance_e(qor_region* r) {
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    for (int i = 2; i < nx - 1; i++)
        for (int j = 2; j < ny - 1; j++)
            for (int k = 2; k < nz - 1; k++) { ndfx_ex(r, i, j, k); ndfx_ey(r, i, j, k); ndfx_ez(r, i, j, k); }
    for (int j = 2; j < ny - 1; j++)
        for (int k = 2; k < nz - 1; k++) ndfx_ex(r, 1, j, k);
    for (int i = 2; i < nx - 1; i++)
        for (int k = 2; k < nz - 1; k++) ndfx_ey(r, i, 1, k);
    for (int i = 2; i < nx - 1; i++)
        for (int j = 2; j < ny - 1; j++) ndfx_ez(r, i, j, 1);
}

/* Five-point, maxwell.cpp:35-125: 4-point derivative along each axis with
 * coefficients a, b; B ranges [1, n-2) plus the high faces (with a truncated
 * stencil for the derivative normal to the face), E ranges [2, n-2) plus the
 * i/j/k = 1 planes. */
/* d/dy of ez at (i,j,k) seen from B, full and high-face (j = ny-1) forms */
#define FP_D4(F, a, bb, p2, p1, p0, m1) (bb * ((p1) - (p0)) + a * ((p2) - (p1) + (p0) - (m1)))
static void fp_bx(qor_region* r, int i, int j, int k, int yface, int zface) {
    double dy_, dz_;
    if (yface) dy_ = r->fp_by * (-E_(2, i, j, k)) + r->fp_ay * (E_(2, i, j, k) - E_(2, i, j - 1, k));
    else dy_ = r->fp_by * (E_(2, i, j + 1, k) - E_(2, i, j, k)) + r->fp_ay * (E_(2, i, j + 2, k) - E_(2, i, j + 1, k) + E_(2, i, j, k) - E_(2, i, j - 1, k));
    if (zface) dz_ = r->fp_bz * (-E_(1, i, j, k)) + r->fp_az * (E_(1, i, j, k) - E_(1, i, j, k - 1));
    else dz_ = r->fp_bz * (E_(1, i, j, k + 1) - E_(1, i, j, k)) + r->fp_az * (E_(1, i, j, k + 2) - E_(1, i, j, k + 1) + E_(1, i, j, k) - E_(1, i, j, k - 1));
    B_(0, i, j, k) += 0.5 * (-r->dtdy * dy_ + r->dtdz * dz_);
}
static void fp_by(qor_region* r, int i, int j, int k, int xface, int zface) {
    double dx_, dz_;
    if (xface) dx_ = r->fp_bx * (-E_(2, i, j, k)) + r->fp_ax * (E_(2, i, j, k) - E_(2, i - 1, j, k));
    else dx_ = r->fp_bx * (E_(2, i + 1, j, k) - E_(2, i, j, k)) + r->fp_ax * (E_(2, i + 2, j, k) - E_(2, i + 1, j, k) + E_(2, i, j, k) - E_(2, i - 1, j, k));
    if (zface) dz_ = r->fp_bz * (-E_(0, i, j, k)) + r->fp_az * (E_(0, i, j, k) - E_(0, i, j, k - 1));
    else dz_ = r->fp_bz * (E_(0, i, j, k + 1) - E_(0, i, j, k)) + r->fp_az * (E_(0, i, j, k + 2) - E_(0, i, j, k + 1) + E_(0, i, j, k) - E_(0, i, j, k - 1));
    B_(1, i, j, k) += 0.5 * (r->dtdx * dx_ - r->dtdz * dz_);
}
static void fp_bz(qor_region* r, int i, int j, int k, int xface, int yface) {
    double dy_, dx_;
    if (yface) dy_ = r->fp_by * (-E_(0, i, j, k)) + r->fp_ay * (E_(0, i, j, k) - E_(0, i, j - 1, k));
    else dy_ = r->fp_by * (E_(0, i, j + 1, k) - E_(0, i, j, k)) + r->fp_ay * (E_(0, i, j + 2, k) - E_(0, i, j + 1, k) + E_(0, i, j, k) - E_(0, i, j - 1, k));
    if (xface) dx_ = r->fp_bx * (-E_(1, i, j, k)) + r->fp_ax * (E_(1, i, j, k) - E_(1, i - 1, j, k));
    else dx_ = r->fp_bx * (E_(1, i + 1, j, k) - E_(1, i, j, k)) + r->fp_ax * (E_(1, i + 2, j, k) - E_(1, i + 1, j, k) + E_(1, i, j, k) - E_(1, i - 1, j, k));
    B_(2, i, j, k) += 0.5 * (r->dtdy * dy_ - r->dtdx * dx_);
}
static void fp_ex(qor_region* r, int i, int j, int k) {
    E_(0, i, j, k) = E_(0, i, j, k) + r->dtdy * (r->fp_by * (B_(2, i, j, k) - B_(2, i, j - 1, k)) + r->fp_ay * (B_(2, i, j + 1, k) - B_(2, i, j, k) + B_(2, i, j - 1, k) - B_(2, i, j - 2, k))) -
                     r->dtdz * (r->fp_bz * (B_(1, i, j, k) - B_(1, i, j, k - 1)) + r->fp_az * (B_(1, i, j, k + 1) - B_(1, i, j, k) + B_(1, i, j, k - 1) - B_(1, i, j, k - 2))) -
                     J_(0, i, j, k) * r->dx;
}
static void fp_ey(qor_region* r, int i, int j, int k) {
    E_(1, i, j, k) = E_(1, i, j, k) - r->dtdx * (r->fp_bx * (B_(2, i, j, k) - B_(2, i - 1, j, k)) + r->fp_ax * (B_(2, i + 1, j, k) - B_(2, i, j, k) + B_(2, i - 1, j, k) - B_(2, i - 2, j, k))) +
                     r->dtdz * (r->fp_bz * (B_(0, i, j, k) - B_(0, i, j, k - 1)) + r->fp_az * (B_(0, i, j, k + 1) - B_(0, i, j, k) + B_(0, i, j, k - 1) - B_(0, i, j, k - 2))) -
                     J_(1, i, j, k) * r->dy;
}
static void fp_ez(qor_region* r, int i, int j, int k) {
    E_(2, i, j, k) = E_(2, i, j, k) + r->dtdx * (r->fp_bx * (B_(1, i, j, k) - B_(1, i - 1, j, k)) + r->fp_ax * (B_(1, i + 1, j, k) - B_(1, i, j, k) + B_(1, i - 1, j, k) - B_(1, i - 2, j, k))) -
                     r->dtdy * (r->fp_by * (B_(0, i, j, k) - B_(0, i, j - 1, k)) + r->fp_ay * (B_(0, i, j + 1, k) - B_(0, i, j, k) + B_(0, i, j - 1, k) - B_(0, i, j - 2, k))) -
                     J_(2, i, j, k) * r->dz;
}
static void fp_advance_b(qor_region* r) {
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    for (int i = 1; i < nx - 2; i++)
        for (int j = 1; j < ny - 2; j++)
            for (int k = 1; k < nz - 2; k++) { fp_bx(r, i, j, k, 0, 0); fp_by(r, i, j, k, 0, 0); fp_bz(r, i, j, k, 0, 0); }
    for (int j = 1; j < ny - 2; j++)
        for (int k = 1; k < nz - 2; k++) { int i = nx - 1; fp_bx(r, i, j, k, 0, 0); fp_by(r, i, j, k, 1, 0); fp_bz(r, i, j, k, 1, 0); }
    for (int i = 1; i < nx - 2; i++)
        for (int k = 1; k < nz - 2; k++) { int j = ny - 1; fp_bx(r, i, j, k, 1, 0); fp_by(r, i, j, k, 0, 0); fp_bz(r, i, j, k, 0, 1); }
    for (int i = 1; i < nx - 2; i++)
        for (int j = 1; j < ny - 2; j++) { int k = nz - 1; fp_bx(r, i, j, k, 0, 1); fp_by(r, i, j, k, 0, 1); fp_bz(r, i, j, k, 0, 0); }
}
static void fp_advance_e(qor_region* r) {
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    for (int i = 2; i < nx - 2; i++)
        for (int j = 2; j < ny - 2; j++)
            for (int k = 2; k < nz - 2; k++) { fp_ex(r, i, j, k); fp_ey(r, i, j, k); fp_ez(r, i, j, k); }
    for (int j = 2; j < ny - 2; j++)
        for (int k = 2; k < nz - 2; k++) fp_ex(r, 1, j, k);
    for (int i = 2; i < nx - 2; i++)
        for (int k = 2; k < nz - 2; k++) fp_ey(r, i, 1, k);
    for (int i = 2; i < nx - 2; i++)
        for (int j = 2; j < ny - 2; j++) fp_ez(r, i, j, 1);
}

static void zero_faces(qor_region* r, int axis, int plane, int lo, const int* comps, int ncomp) {
    /* zero components on one plane over [0, n-1) of the two other axes */
    (void)lo;
    const int n[3] = {r->nx, r->ny, r->nz};
    int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
    if (a1 > a2) { int t = a1; a1 = a2; a2 = t; }
    for (int u = 0; u < n[a1] - 1; u++)
        for (int v = 0; v < n[a2] - 1; v++) {
            int ijk[3];
            ijk[axis] = plane; ijk[a1] = u; ijk[a2] = v;
            long c = IDX(r, ijk[0], ijk[1], ijk[2]);
            for (int m = 0; m < ncomp; m++) r->f[comps[m]][c] = 0;
        }
}

/* init_boundaries of each solver, maxwell.cpp:135-236, 338-438, 532-597:
 * components zeroed once on the box faces (plane index, components). */
void qor_init_boundaries(qor_region* r) {
    static const int all6[6] = {0, 1, 2, 3, 4, 5};
    const int nx = r->nx, ny = r->ny, nz = r->nz;
    if (r->solver == 0) { /* FDTD */
        const int x0[3] = {1, 2, 3}, y0[3] = {0, 2, 4}, z0[3] = {1, 0, 5};
        zero_faces(r, 0, 0, 0, x0, 3); zero_faces(r, 0, nx - 1, 0, all6, 6);
        zero_faces(r, 1, 0, 0, y0, 3); zero_faces(r, 1, ny - 1, 0, all6, 6);
        zero_faces(r, 2, 0, 0, z0, 3); zero_faces(r, 2, nz - 1, 0, all6, 6);
    } else if (r->solver == 1) { /* NDFX */
        const int x1[3] = {1, 2, 3}, y1[3] = {0, 2, 4}, z1[3] = {1, 0, 5};
        zero_faces(r, 0, 0, 0, all6, 6); zero_faces(r, 0, 1, 0, x1, 3); zero_faces(r, 0, nx - 1, 0, all6, 6);
        zero_faces(r, 1, 0, 0, all6, 6); zero_faces(r, 1, 1, 0, y1, 3); zero_faces(r, 1, ny - 1, 0, all6, 6);
        zero_faces(r, 2, 0, 0, all6, 6); zero_faces(r, 2, 1, 0, z1, 3); zero_faces(r, 2, nz - 1, 0, all6, 6);
    } else { /* five-point */
        zero_faces(r, 0, 0, 0, all6, 6); zero_faces(r, 1, 0, 0, all6, 6); zero_faces(r, 2, 0, 0, all6, 6);
        zero_faces(r, 0, nx - 1, 0, all6, 6); zero_faces(r, 1, ny - 1, 0, all6, 6); zero_faces(r, 2, nz - 1, 0, all6, 6);
        const int xa[2] = {4, 5}, xb[2] = {2, 1};
        const int ya[2] = {3, 5}, yb[2] = {0, 2};
        const int za[2] = {3, 4}, zb[2] = {0, 1};
        zero_faces(r, 0, nx - 2, 0, xa, 2); zero_faces(r, 0, 1, 0, xb, 2);
        zero_faces(r, 1, ny - 2, 0, ya, 2); zero_faces(r, 1, 1, 0, yb, 2);
        zero_faces(r, 2, nz - 2, 0, za, 2); zero_faces(r, 2, 1, 0, zb, 2);
    }
    interpolate_be(r);
}

/* maxwell_solver::advance (maxwell.cpp:10-22) then interpolate_be
 * (advance.cpp:13-18). */
void qor_fadvance(qor_region* r) {
    if (r->solver == 0) { fdtd_advance_b(r); fdtd_advance_e(r); fdtd_advance_b(r); }
    else if (r->solver == 1) { ndfx_advance_b(r); ndfx_advance_e(r); ndfx_advance_b(r); }
    else { fp_advance_b(r); fp_advance_e(r); fp_advance_b(r); }
    interpolate_be(r);
}

/* ------------------------------------------------------------------------ */
/* Particles                                                                 */
/* ------------------------------------------------------------------------ */
void qor_add_particles(qor_region* r, long n, const double* x, const double* y, const double* z,
                       const double* ux, const double* uy, const double* uz, const double* g,
                       const double* q, const double* cmr, const double* chi) {
    /* Inside a cell the given order becomes the list order; particles of a
     * later call go before those already present, as head insertion
     * (plist.cpp:22-39) would put them.  Realised as a stable sort by cell of
     * [new particles, old particles]. */
    long n0 = r->n, nt = n0 + n;
    grow(r, nt);
    double* arrs[10] = {r->x, r->y, r->z, r->ux, r->uy, r->uz, r->g, r->q, r->cmr, r->chi};
    const double* src[10] = {x, y, z, ux, uy, uz, g, q, cmr, chi};
    double* tmp = (double*)malloc(sizeof(double) * (nt ? nt : 1));
    long* cl = (long*)malloc(sizeof(long) * (nt ? nt : 1));
    for (long p = 0; p < n; p++) cl[p] = IDX(r, (int)x[p], (int)y[p], (int)z[p]);
    for (long p = 0; p < n0; p++) cl[n + p] = r->cell[p];
    long* cnt = (long*)calloc(r->nc + 1, sizeof(long));
    for (long p = 0; p < nt; p++) cnt[cl[p] + 1]++;
    for (long c = 0; c < r->nc; c++) cnt[c + 1] += cnt[c];
    long* perm = (long*)malloc(sizeof(long) * (nt ? nt : 1));
    for (long p = 0; p < nt; p++) perm[cnt[cl[p]]++] = p;
    free(cnt);
    for (int a = 0; a < 10; a++) {
        for (long p = 0; p < nt; p++) {
            long s = perm[p];
            tmp[p] = s < n ? (src[a] ? src[a][s] : 0.0) : arrs[a][s - n];
        }
        memcpy(arrs[a], tmp, sizeof(double) * nt);
    }
    for (long p = 0; p < nt; p++) r->cell[p] = cl[perm[p]];
    free(cl); free(tmp); free(perm);
    r->n = nt;
}

long qor_count_particles(qor_region* r) { return r->n; }

long qor_get_particles(qor_region* r, long cap, double* out, long* cell) {
    double* arrs[10] = {r->x, r->y, r->z, r->ux, r->uy, r->uz, r->g, r->q, r->cmr, r->chi};
    long n = r->n < cap ? r->n : cap;
    for (int a = 0; a < 10; a++) memcpy(out + a * cap, arrs[a], sizeof(double) * n);
    if (cell) memcpy(cell, r->cell, sizeof(long) * n);
    return r->n;
}

/* pusher.cpp:5-42 — Vay (2008): half-step field terms, gamma from the
 * quadratic invariant, then rotation with the stored gamma. */
static void push_vay(double cmr, double* ux, double* uy, double* uz, double* g,
                     const double* E, const double* B, double dt) {
    double ex, ey, ez, bx, by, bz, t, wx, wy, wz, bw;
    t = dt * cmr;
    ex = E[0] * t; ey = E[1] * t; ez = E[2] * t;
    t = 0.5 * t;
    bx = B[0] * t; by = B[1] * t; bz = B[2] * t;
    wx = *ux + ex + (*uy * bz - *uz * by) / *g;
    wy = *uy + ey + (*uz * bx - *ux * bz) / *g;
    wz = *uz + ez + (*ux * by - *uy * bx) / *g;
    t = bx * bx + by * by + bz * bz;
    bw = bx * wx + by * wy + bz * wz;
    double gg = 1 + wx * wx + wy * wy + wz * wz - t;
    gg = sqrt(0.5 * (gg + sqrt(gg * gg + 4 * (t + bw * bw))));
    t = 1 / (1 + t / (gg * gg));
    bw = bw / (gg * gg);
    *ux = (wx + (wy * bz - wz * by) / gg + bx * bw) * t;
    *uy = (wy + (wz * bx - wx * bz) / gg + by * bw) * t;
    *uz = (wz + (wx * by - wy * bx) / gg + bz * bw) * t;
    *g = gg;
}

/* pusher.cpp:44-97 — Boris: half electric kick, magnetic rotation with
 * t = qB dt/(2 m gamma), second half kick, gamma from u. */
static void push_boris(double cmr, double* ux, double* uy, double* uz, double* g,
                       const double* E, const double* B, double dt) {
    double t = 0.5 * dt * cmr;
    double ex = E[0] * t, ey = E[1] * t, ez = E[2] * t;
    double u1x = *ux + ex, u1y = *uy + ey, u1z = *uz + ez;
    double gg = sqrt(1 + u1x * u1x + u1y * u1y + u1z * u1z);
    t /= gg;
    double bx = B[0] * t, by = B[1] * t, bz = B[2] * t;
    double wx = u1x + (u1y * bz - u1z * by);
    double wy = u1y + (u1z * bx - u1x * bz);
    double wz = u1z + (u1x * by - u1y * bx);
    t = 2 / (1 + bx * bx + by * by + bz * bz);
    u1x += (wy * bz - wz * by) * t;
    u1y += (wz * bx - wx * bz) * t;
    u1z += (wx * by - wy * bx) * t;
    *ux = u1x + ex; *uy = u1y + ey; *uz = u1z + ez;
    *g = sqrt(1 + *ux * *ux + *uy * *uy + *uz * *uz);
}

void qor_push(int pusher, double cmr, double* s, const double* e, const double* b, double dt) {
    if (pusher == 0) push_vay(cmr, &s[0], &s[1], &s[2], &s[3], e, b, dt);
    else push_boris(cmr, &s[0], &s[1], &s[2], &s[3], e, b, dt);
}

/* deposition.cpp:431-471: Ex is interpolated in (y, z) at the particle's i,
 * Ey in (x, z), Ez in (x, y); B uses the same weights on Bbar. */
static void gather(qor_region* r, double x, double y, double z, double* e, double* b) {
    int i = (int)floor(x), j = (int)floor(y), k = (int)floor(z);
    double xa = x - i, xb = 1 - xa, ya = y - j, yb = 1 - ya, za = z - k, zb = 1 - za;
    const double *ex = EX(r), *ey = EY(r), *ez = EZ(r);
    const double *bx = BEX(r), *by = BEY(r), *bz = BEZ(r);
    e[0] = ex[IDX(r, i, j, k)] * yb * zb + ex[IDX(r, i, j + 1, k)] * ya * zb + ex[IDX(r, i, j, k + 1)] * yb * za + ex[IDX(r, i, j + 1, k + 1)] * ya * za;
    e[1] = ey[IDX(r, i, j, k)] * xb * zb + ey[IDX(r, i + 1, j, k)] * xa * zb + ey[IDX(r, i, j, k + 1)] * xb * za + ey[IDX(r, i + 1, j, k + 1)] * xa * za;
    e[2] = ez[IDX(r, i, j, k)] * xb * yb + ez[IDX(r, i + 1, j, k)] * xa * yb + ez[IDX(r, i, j + 1, k)] * xb * ya + ez[IDX(r, i + 1, j + 1, k)] * xa * ya;
    b[0] = bx[IDX(r, i, j, k)] * yb * zb + bx[IDX(r, i, j + 1, k)] * ya * zb + bx[IDX(r, i, j, k + 1)] * yb * za + bx[IDX(r, i, j + 1, k + 1)] * ya * za;
    b[1] = by[IDX(r, i, j, k)] * xb * zb + by[IDX(r, i + 1, j, k)] * xa * zb + by[IDX(r, i, j, k + 1)] * xb * za + by[IDX(r, i + 1, j, k + 1)] * xa * za;
    b[2] = bz[IDX(r, i, j, k)] * xb * yb + bz[IDX(r, i + 1, j, k)] * xa * yb + bz[IDX(r, i, j + 1, k)] * xb * ya + bz[IDX(r, i + 1, j + 1, k)] * xa * ya;
}

void qor_gather(qor_region* r, double x, double y, double z, double* e, double* b) { gather(r, x, y, z, e, b); }

/* deposition.cpp:13-39: charge-conserving current of a straight segment d
 * starting at p inside the cell with lower corner w (12 contributions). */
static void seg_dep(qor_region* r, const double* p, const double* d, double q, int wi, int wj, int wk) {
    double xa = p[0] - wi, xb = 1 - xa, ya = p[1] - wj, yb = 1 - ya, za = p[2] - wk, zb = 1 - za;
    double* jx = JX(r); double* jy = JY(r); double* jz = JZ(r);
    const double dx = d[0], dy = d[1], dz = d[2];
    jx[IDX(r, wi, wj + 1, wk + 1)] = jx[IDX(r, wi, wj + 1, wk + 1)] + dx * q * (ya * za + 0.5 * (dz * ya + dy * za) + dy * dz / 3);
    jx[IDX(r, wi, wj, wk + 1)] = jx[IDX(r, wi, wj, wk + 1)] + dx * q * (yb * za + 0.5 * (dz * yb - dy * za) - dy * dz / 3);
    jx[IDX(r, wi, wj + 1, wk)] = jx[IDX(r, wi, wj + 1, wk)] + dx * q * (ya * zb + 0.5 * (-dz * ya + dy * zb) - dy * dz / 3);
    jx[IDX(r, wi, wj, wk)] = jx[IDX(r, wi, wj, wk)] + dx * q * (yb * zb - 0.5 * (dz * yb + dy * zb) + dy * dz / 3);
    jy[IDX(r, wi + 1, wj, wk + 1)] = jy[IDX(r, wi + 1, wj, wk + 1)] + dy * q * (xa * za + 0.5 * (dx * za + dz * xa) + dx * dz / 3);
    jy[IDX(r, wi, wj, wk + 1)] = jy[IDX(r, wi, wj, wk + 1)] + dy * q * (xb * za + 0.5 * (-dx * za + dz * xb) - dx * dz / 3);
    jy[IDX(r, wi + 1, wj, wk)] = jy[IDX(r, wi + 1, wj, wk)] + dy * q * (xa * zb + 0.5 * (dx * zb - dz * xa) - dx * dz / 3);
    jy[IDX(r, wi, wj, wk)] = jy[IDX(r, wi, wj, wk)] + dy * q * (xb * zb - 0.5 * (dx * zb + dz * xb) + dx * dz / 3);
    jz[IDX(r, wi + 1, wj + 1, wk)] = jz[IDX(r, wi + 1, wj + 1, wk)] + dz * q * (xa * ya + 0.5 * (dx * ya + dy * xa) + dx * dy / 3);
    jz[IDX(r, wi, wj + 1, wk)] = jz[IDX(r, wi, wj + 1, wk)] + dz * q * (xb * ya + 0.5 * (-dx * ya + dy * xb) - dx * dy / 3);
    jz[IDX(r, wi + 1, wj, wk)] = jz[IDX(r, wi + 1, wj, wk)] + dz * q * (xa * yb + 0.5 * (dx * yb - dy * xa) - dx * dy / 3);
    jz[IDX(r, wi, wj, wk)] = jz[IDX(r, wi, wj, wk)] + dz * q * (xb * yb - 0.5 * (dx * yb + dy * xb) + dx * dy / 3);
}

static void advance_seg(double* p, const double* d) { p[0] = p[0] + d[0]; p[1] = p[1] + d[1]; p[2] = p[2] + d[2]; }

/* Three ratios sorted descending (low-level.cpp:316-366, `regulate`), with
 * the reference's tie handling. */
static void sort3_desc(double a, double b, double c, double* vx, double* vy, double* vz) {
    if (a > b) {
        if (b > c) { *vx = a; *vy = b; *vz = c; }
        else { *vz = b; if (a > c) { *vx = a; *vy = c; } else { *vx = c; *vy = a; } }
    } else {
        if (c > b) { *vx = c; *vy = b; *vz = a; }
        else { *vx = b; if (a > c) { *vy = a; *vz = c; } else { *vy = c; *vz = a; } }
    }
}

static int imax(int a, int b) { return a > b ? a : b; }

/* deposition.cpp:41-356: the straight path p -> p + d is split where it
 * crosses cell faces (0..3 crossings -> 1..4 segments); each segment is
 * deposited in the cell it lies in, and p is advanced segment by segment. */
static void jdeposition(qor_region* r, double* p, const double* d, double q) {
    int c1[3], c2[3];
    for (int a = 0; a < 3; a++) { c1[a] = (int)floor(p[a]); c2[a] = (int)floor(p[a] + d[a]); }
    int cx = c1[0] != c2[0], cy = c1[1] != c2[1], cz = c1[2] != c2[2];
    int ncross = cx + cy + cz;
    double s[3];
    int w[3] = {c1[0], c1[1], c1[2]};
    if (ncross == 0) {
        seg_dep(r, p, d, q, w[0], w[1], w[2]);
        advance_seg(p, d);
    } else if (ncross == 1) {
        int a = cx ? 0 : (cy ? 1 : 2);
        /* first part up to the face of axis a, other axes in proportion */
        s[a] = imax(c1[a], c2[a]) - p[a];
        for (int o = 0; o < 3; o++) if (o != a) s[o] = d[o] * s[a] / d[a];
        seg_dep(r, p, s, q, w[0], w[1], w[2]);
        advance_seg(p, s);
        for (int o = 0; o < 3; o++) s[o] = d[o] - s[o];
        w[a] = c2[a];
        seg_dep(r, p, s, q, w[0], w[1], w[2]);
        advance_seg(p, s);
    } else if (ncross == 2) {
        /* axis A carries the reference's path1, axis B its path2; path1 is
         * y for (y,z) and (x,y), x for (x,z).  B goes first only if
         * path1 > path2. */
        int A, B;
        if (!cx) { A = 1; B = 2; }
        else if (!cy) { A = 0; B = 2; }
        else { A = 1; B = 0; }
        double pa = (imax(c1[A], c2[A]) - p[A]) / d[A];
        double pb = (imax(c1[B], c2[B]) - p[B]) / d[B];
        int first = A, second = B;
        double p1 = pa, p2 = pb;
        if (pa > pb) { first = B; second = A; p1 = pb; p2 = pa; }
        for (int o = 0; o < 3; o++) s[o] = d[o] * p1;
        seg_dep(r, p, s, q, w[0], w[1], w[2]);
        advance_seg(p, s);
        for (int o = 0; o < 3; o++) s[o] = d[o] * (p2 - p1);
        w[first] = c2[first];
        seg_dep(r, p, s, q, w[0], w[1], w[2]);
        advance_seg(p, s);
        for (int o = 0; o < 3; o++) s[o] = d[o] * (1 - p2);
        w[second] = c2[second];
        seg_dep(r, p, s, q, w[0], w[1], w[2]);
        advance_seg(p, s);
    } else {
        double path[3];
        for (int a = 0; a < 3; a++) path[a] = (imax(c1[a], c2[a]) - p[a]) / d[a];
        double vx, vy, vz;
        sort3_desc(path[0], path[1], path[2], &vx, &vy, &vz);
        const double fr[4] = {vz, vy - vz, vx - vy, 1 - vx};
        for (int sgi = 0; sgi < 4; sgi++) {
            for (int o = 0; o < 3; o++) s[o] = d[o] * fr[sgi];
            if (sgi > 0)
                for (int o = 0; o < 3; o++) w[o] = (int)floor(p[o] + 0.5 * s[o]);
            seg_dep(r, p, s, q, w[0], w[1], w[2]);
            advance_seg(p, s);
        }
    }
}

void qor_jdeposition(qor_region* r, double* pos, const double* d, double q) { jdeposition(r, pos, d, q); }

void qor_zero_j(qor_region* r) {
    memset(JX(r), 0, sizeof(double) * r->nc);
    memset(JY(r), 0, sizeof(double) * r->nc);
    memset(JZ(r), 0, sizeof(double) * r->nc);
}

/* plist.cpp:42-48 */
static int is_inside(qor_region* r, int i, int j, int k) {
    return i > 0 && i < r->nx - 2 && j > 0 && j < r->ny - 2 && k > 0 && k < r->nz - 2;
}
/* plist.cpp:73-102: layers {0, n-2, n-1} of every axis are emptied */
static int in_kill_layer(qor_region* r, long c) {
    int k = (int)(c % r->nz), j = (int)((c / r->nz) % r->ny), i = (int)(c / ((long)r->nz * r->ny));
    return i == 0 || i >= r->nx - 2 || j == 0 || j >= r->ny - 2 || k == 0 || k >= r->nz - 2;
}

/* advance.cpp:90-387 with QED off */
void qor_padvance(qor_region* r, double external_bz) {
    const long n = r->n;
    long* newc = (long*)malloc(sizeof(long) * (n ? n : 1));
    qor_zero_j(r);
    for (long p = 0; p < n; p++) {
        if (in_kill_layer(r, r->cell[p])) { newc[p] = -1; continue; }
        double e[3], b[3];
        gather(r, r->x[p], r->y[p], r->z[p], e, b);
        b[2] += external_bz;
        double pos[3] = {r->x[p], r->y[p], r->z[p]};
        double cm = r->cmr[p];
        if (cm == 0) {
            /* photon with QED off: straight flight, no current */
            double a = r->dt / r->g[p];
            double dsp[3] = {r->ux[p] * a, r->uy[p] * a, r->uz[p] * a};
            dsp[0] = dsp[0] / r->dx; dsp[1] = dsp[1] / r->dy; dsp[2] = dsp[2] / r->dz;
            advance_seg(pos, dsp);
        } else {
            if (r->pusher == 0) push_vay(cm, &r->ux[p], &r->uy[p], &r->uz[p], &r->g[p], e, b, r->dt);
            else push_boris(cm, &r->ux[p], &r->uy[p], &r->uz[p], &r->g[p], e, b, r->dt);
            double a = r->dt / r->g[p];
            double dsp[3] = {r->ux[p] * a, r->uy[p] * a, r->uz[p] * a};
            dsp[0] = dsp[0] / r->dx; dsp[1] = dsp[1] / r->dy; dsp[2] = dsp[2] / r->dz;
            jdeposition(r, pos, dsp, r->q[p]);
        }
        r->x[p] = pos[0]; r->y[p] = pos[1]; r->z[p] = pos[2];
        int ni = (int)pos[0], nj = (int)pos[1], nk = (int)pos[2];
        long nc = IDX(r, ni, nj, nk);
        if (nc != r->cell[p] && !is_inside(r, ni, nj, nk)) newc[p] = -1;
        else newc[p] = nc;
    }
    /* rebin: arrivals descending, then stayers ascending (see header) */
    long* arr = (long*)calloc(r->nc, sizeof(long));
    long* tot = (long*)calloc(r->nc + 1, sizeof(long));
    for (long p = 0; p < n; p++) {
        if (newc[p] < 0) continue;
        tot[newc[p] + 1]++;
        if (newc[p] != r->cell[p]) arr[newc[p]]++;
    }
    for (long c = 0; c < r->nc; c++) tot[c + 1] += tot[c];
    long nn = tot[r->nc];
    long* dst = (long*)malloc(sizeof(long) * (n ? n : 1));
    long* fill = (long*)calloc(r->nc, sizeof(long));
    for (long p = n - 1; p >= 0; p--)
        if (newc[p] >= 0 && newc[p] != r->cell[p]) dst[p] = tot[newc[p]] + fill[newc[p]]++;
    for (long p = 0; p < n; p++)
        if (newc[p] >= 0 && newc[p] == r->cell[p]) dst[p] = tot[newc[p]] + arr[newc[p]] + (fill[newc[p]]++ - arr[newc[p]]);
    double* arrs[10] = {r->x, r->y, r->z, r->ux, r->uy, r->uz, r->g, r->q, r->cmr, r->chi};
    double* tmp = (double*)malloc(sizeof(double) * (nn ? nn : 1));
    for (int a = 0; a < 10; a++) {
        for (long p = 0; p < n; p++) if (newc[p] >= 0) tmp[dst[p]] = arrs[a][p];
        memcpy(arrs[a], tmp, sizeof(double) * nn);
    }
    for (long p = 0; p < n; p++) if (newc[p] >= 0) r->cell[dst[p]] = newc[p];
    r->n = nn;
    free(tmp); free(fill); free(dst); free(tot); free(arr); free(newc);
}

/* fout.cpp:41-138: cells with i in [n1, nx - n2) = [dlo, dhi) */
void qor_compute_diag(qor_region* r, double* d) {
    const double dx = r->dx, dy = r->dy, dz = r->dz, lam = r->lam;
    const double aN = dx * dy * dz * 1.11485e13 * lam / (8 * PI_ * PI_ * PI_);
    const double aE = 0.5 * dx * dy * dz * 3.691e4 * lam / 1e7;
    const double bE = 8.2e-14 * dx * dy * dz * 1.11485e13 * lam / (8 * PI_ * PI_ * PI_);
    double Ne = 0, Np = 0, Nph = 0, ef = 0, ee = 0, ep = 0, eph = 0;
    int nqe = 0, nqp = 0, nqg = 0;
    int nqi[16] = {0};
    double ie[16] = {0};
    const long ynz = (long)r->ny * r->nz;
    long p = 0;
    while (p < r->n && r->cell[p] < r->dlo * ynz) p++;
    for (long c = r->dlo * ynz; c < r->dhi * ynz; c++) {
        ef += EX(r)[c] * EX(r)[c] + EY(r)[c] * EY(r)[c] + EZ(r)[c] * EZ(r)[c] + BX(r)[c] * BX(r)[c] + BY(r)[c] * BY(r)[c] + BZ(r)[c] * BZ(r)[c];
        for (; p < r->n && r->cell[p] == c; p++) {
            double cm = r->cmr[p], q = r->q[p], g = r->g[p];
            if (cm == -1) { Ne -= q; nqe++; ee -= (g - 1) * q; }
            else if (cm == 1) { Np += q; nqp++; ep += (g - 1) * q; }
            else if (cm == 0) { Nph += q; nqg++; eph += g * q; }
            else {
                for (int m = 0; m < r->n_ion; m++)
                    if (cm == r->icmr[m]) { ie[m] += (g - 1) * q / r->icmr[m]; break; }
            }
            for (int m = 0; m < r->n_ion; m++) if (cm == r->icmr[m]) nqi[m]++;
        }
    }
    d[0] = Ne * aN; d[1] = Np * aN; d[2] = Nph * aN;
    d[3] = nqe; d[4] = nqp; d[5] = nqg;
    d[6] = ef * aE; d[7] = ee * bE; d[8] = ep * bE; d[9] = eph * bE;
    for (int m = 0; m < r->n_ion; m++) { d[10 + 2 * m] = nqi[m]; d[11 + 2 * m] = ie[m] * bE; }
}

int qor_diag_len(qor_region* r) { return 10 + 2 * r->n_ion; }

/* main.cpp:2321-2331 with QED off */
void qor_step(qor_region* r, int nsteps, double external_bz, double* diag) {
    for (int l = 0; l < nsteps; l++) {
        qor_padvance(r, external_bz);
        double d[42];
        qor_compute_diag(r, d);
        qor_fadvance(r);
        if (diag) memcpy(diag + (long)l * qor_diag_len(r), d, sizeof(double) * qor_diag_len(r));
    }
}

/* ------------------------------------------------------------------------ */
/* QED rate functions and the random stream (mc.cpp:12-116)                   */
/* ------------------------------------------------------------------------ */
double qor_get_rand(qor_region* r) {
    double a = r->rnd[r->n_random % 55] - r->rnd[(r->n_random + 31) % 55];
    if (a < 0) a = a + 1;
    r->rnd[r->n_random % 55] = a;
    r->n_random = r->n_random < 55 ? r->n_random + 1 : 0;
    return a;
}

/* ------------------------------------------------------------------------ */
/* Moving window (advance.cpp:389-454)                                          */
/* ------------------------------------------------------------------------ */
/* The particles of the layer i = 0 are erased, E, B and Bbar move one cell
 * towards -x (the layer nx-1 becomes zero; J is left as it is), the cell
 * lists move with them and every particle's x decreases by 1.  The list
 * order inside a cell is kept. */
void qor_moving_window(qor_region* r) {
    const long ynz = (long)r->ny * r->nz;
    long m = 0;
    for (long t = 0; t < r->n; t++) {
        if (r->cell[t] < ynz) continue;
        r->x[m] = r->x[t] - 1; r->y[m] = r->y[t]; r->z[m] = r->z[t];
        r->ux[m] = r->ux[t]; r->uy[m] = r->uy[t]; r->uz[m] = r->uz[t];
        r->g[m] = r->g[t]; r->q[m] = r->q[t]; r->cmr[m] = r->cmr[t]; r->chi[m] = r->chi[t];
        r->cell[m] = r->cell[t] - ynz;
        m++;
    }
    r->n = m;
    const int planes[9] = {0, 1, 2, 3, 4, 5, 9, 10, 11};
    for (int a = 0; a < 9; a++) {
        double* f = r->f[planes[a]];
        memmove(f, f + ynz, sizeof(double) * (size_t)(r->nc - ynz));
        memset(f + (r->nc - ynz), 0, sizeof(double) * (size_t)ynz);
    }
}

/* ------------------------------------------------------------------------ */
/* Particle merging (mc.cpp:198-462)                                           */
/* ------------------------------------------------------------------------ */
/* class index of a particle: 0 electrons, 1 positrons, 2 photons, 3+ii ions;
 * -1 for an ion cmr not in the table (the reference skips those) */
static int merge_class(const qor_region* r, double cmr) {
    if (cmr == -1) return 0;
    if (cmr == 1) return 1;
    if (cmr == 0) return 2;
    for (int ii = 0; ii < r->n_ion; ii++)
        if (cmr == r->icmr[ii]) return 3 + ii;
    return -1;
}

/* _ppd (mc.cpp:198-200) */
static double merge_ppd(double q, double q0) { return 1 / (1 + pow(2 * q / q0, 4)); }

static void merge_erase(qor_region* r, const char* keep) {
    long m = 0;
    for (long t = 0; t < r->n; t++) {
        if (!keep[t]) continue;
        r->x[m] = r->x[t]; r->y[m] = r->y[t]; r->z[m] = r->z[t];
        r->ux[m] = r->ux[t]; r->uy[m] = r->uy[t]; r->uz[m] = r->uz[t];
        r->g[m] = r->g[t]; r->q[m] = r->q[t]; r->cmr[m] = r->cmr[t]; r->chi[m] = r->chi[t];
        r->cell[m] = r->cell[t];
        m++;
    }
    r->n = m;
}

/* spatial_region::pmerging: particles are deleted with probability ppd
 * ("ti": ppd[0] for all; "nl": ppd of the class times _ppd of the weight
 * relative to the class's mean weight), drawing one random number per
 * particle in traversal order; the weights are then rescaled so that the
 * total charge of each class is kept. */
void qor_pmerging(qor_region* r, int mode, const double* ppd) {
    const int nk = 3 + r->n_ion;
    double qs[19], a[19];
    for (int i = 0; i < nk; i++) { qs[i] = 0; a[i] = 0; }
    for (long t = 0; t < r->n; t++) {
        const int c = merge_class(r, r->cmr[t]);
        if (c == 0) a[0] -= r->q[t];
        else if (c > 0) a[c] += r->q[t];
    }
    char* keep = (char*)malloc(r->n > 0 ? (size_t)r->n : 1);
    if (mode == 1) {
        for (long t = 0; t < r->n; t++) {
            keep[t] = 1;
            if (qor_get_rand(r) < ppd[0]) {
                const int c = merge_class(r, r->cmr[t]);
                if (c == 0) qs[0] -= r->q[t];
                else if (c > 0) qs[c] += r->q[t];
                keep[t] = 0;
            }
        }
        merge_erase(r, keep);
        for (int i = 0; i < nk; i++)
            if (a[i] - qs[i] != 0) a[i] = a[i] / (a[i] - qs[i]);
        for (long t = 0; t < r->n; t++) {
            const int c = merge_class(r, r->cmr[t]);
            if (c >= 0) r->q[t] = a[c] * r->q[t];
        }
    } else {
        double av_q[19];
        for (int i = 0; i < nk; i++) av_q[i] = 0;
        for (long t = 0; t < r->n; t++) {
            const int c = merge_class(r, r->cmr[t]);
            if (c >= 0) av_q[c] += 1;
        }
        for (int i = 0; i < nk; i++) av_q[i] = a[i] / av_q[i];
        for (long t = 0; t < r->n; t++) {
            keep[t] = 1;
            const int c = merge_class(r, r->cmr[t]);
            if (c < 0) continue;
            const double qq = c == 0 ? -r->q[t] : r->q[t];
            if (qor_get_rand(r) < ppd[c] * merge_ppd(qq, av_q[c])) keep[t] = 0;
        }
        merge_erase(r, keep);
        for (long t = 0; t < r->n; t++) {
            const int c = merge_class(r, r->cmr[t]);
            if (c < 0) continue;
            if (c == 0) {
                r->q[t] = r->q[t] / (1 - ppd[0] * merge_ppd(-r->q[t], av_q[0]));
                qs[0] -= r->q[t];
            } else {
                r->q[t] = r->q[t] / (1 - ppd[c] * merge_ppd(r->q[t], av_q[c]));
                qs[c] += r->q[t];
            }
        }
        for (int i = 0; i < nk; i++) a[i] = qs[i] != 0 ? a[i] / qs[i] : 0;
        for (long t = 0; t < r->n; t++) {
            const int c = merge_class(r, r->cmr[t]);
            if (c >= 0) r->q[t] = a[c] * r->q[t];
        }
    }
    free(keep);
}

/* quantum parameter chi = |gamma E + u x B|^2 - (u.E)^2, square-rooted and
 * divided by the Sauter field (mc.cpp:26-38) */
double qor_chi(qor_region* r, const double* e, const double* b, const double* u, double g) {
    double a1, a2;
    a1 = g * e[0] + u[1] * b[2] - u[2] * b[1];
    a2 = a1 * a1;
    a1 = g * e[1] - u[0] * b[2] + u[2] * b[0];
    a2 += a1 * a1;
    a1 = g * e[2] + u[0] * b[1] - u[1] * b[0];
    a2 += a1 * a1;
    a1 = u[0] * e[0] + u[1] * e[1] + u[2] * e[2];
    a2 -= a1 * a1;
    return sqrt(a2) / r->e_s;
}

/* emission spectrum with Airy-function fits (mc.cpp:40-74); for chi <= 0.133
 * r is mapped onto [0, r_max] in place and the rate carries a factor r_max */
double qor_w(qor_region* r, double g, double* rr, double chi) {
    double rv = *rr;
    if ((1 - rv) * g < 1 || rv == 0 || chi == 0) return 0;
    const double es = r->e_s;
    if (chi > 0.133) {
        double d = rv / ((1 - rv) * chi);
        double a = pow(d, (double)1 / 3);
        double kappa = a * a;
        return -0.0020591 * es / (g * g) * exp(-2 * d / 3) *
               (1 / sqrt(sqrt((kappa + 0.80049) * (kappa + 0.80049) * (kappa + 0.80049))) -
                (2 * (1 - rv) + rv * rv) * chi * a / rv * sqrt(sqrt(kappa + 0.70861 * (1 - 0.65 * kappa / (1 + kappa * kappa)))));
    }
    double r_max = 1 / (1 + 2 / (3 * 5 * chi));
    rv = r_max * rv;
    *rr = rv;
    double d = rv / ((1 - rv) * chi);
    double a = pow(d, (double)1 / 3);
    double kappa = a * a;
    return -r_max * 0.0020591 * es / (g * g) * exp(-2 * d / 3) *
           (1 / sqrt(sqrt((kappa + 0.80049) * (kappa + 0.80049) * (kappa + 0.80049))) -
            (2 * (1 - rv) + rv * rv) * chi * a / rv * sqrt(sqrt(kappa + 0.70861 * (1 - 0.65 * kappa / (1 + kappa * kappa)))));
}

/* pair-creation spectrum (mc.cpp:76-97) */
double qor_tilde_w(qor_region* r, double g, double rr, double chi) {
    if (chi == 0 || rr * g < 1 || (1 - rr) * g < 1) return 0;
    double d = 1 / (rr * (1 - rr) * chi);
    double a = pow(d, (double)1 / 3);
    double kappa = a * a;
    return 0.0020591 * r->e_s / (g * g) * exp(-2 * d / 3) *
           (1 / sqrt(sqrt((kappa + 0.80049) * (kappa + 0.80049) * (kappa + 0.80049))) -
            (2 * rr * (1 - rr) - 1) * chi * a * sqrt(sqrt(kappa + 0.70861 * (1 - 0.65 * kappa / (1 + kappa * kappa)))));
}

/* Schwinger pair-creation rate per unit volume and time (mc.cpp:99-116) */
double qor_mathcal_W(qor_region* r, const double* e, const double* b) {
    double f = 0.5 * (e[0] * e[0] + e[1] * e[1] + e[2] * e[2] - b[0] * b[0] - b[1] * b[1] - b[2] * b[2]);
    double gg = e[0] * b[0] + e[1] * b[1] + e[2] * b[2];
    double a = sqrt(f * f + gg * gg);
    double xi = sqrt(a + f), theta = sqrt(a - f);
    const double es = r->e_s;
    if (xi != 0) {
        if (theta != 0) return es * es / (4 * PI_) * xi * theta / tanh(PI_ * theta / xi) * exp(-PI_ * es / xi);
        return es * es / (4 * PI_) * xi * xi / PI_ * exp(-PI_ * es / xi);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* x-slabs of a region (main.cpp:1286-1423)                                   */
/* ------------------------------------------------------------------------ */
void qor_set_diag_range(qor_region* r, int lo, int hi) { r->dlo = lo; r->dhi = hi; }

/* send_field_slice / receive_field_slice: ce, cb, cj, cbe of the cells with
 * i in [i0, i0 + w); 12 blocks of w*ny*nz */
void qor_get_field_slab(qor_region* r, int i0, int w, double* out12) {
    const long m = (long)w * r->ny * r->nz, off = (long)i0 * r->ny * r->nz;
    for (int a = 0; a < 12; a++) memcpy(out12 + a * m, r->f[a] + off, sizeof(double) * (size_t)m);
}

void qor_set_field_slab(qor_region* r, int i0, int w, const double* in12) {
    const long m = (long)w * r->ny * r->nz, off = (long)i0 * r->ny * r->nz;
    for (int a = 0; a < 12; a++) memcpy(r->f[a] + off, in12 + a * m, sizeof(double) * (size_t)m);
}

/* traversal range [*a, *b) of the slab's cells */
static void slab_range(qor_region* r, int i0, int w, long* a, long* b) {
    const long c0 = (long)i0 * r->ny * r->nz, c1 = (long)(i0 + w) * r->ny * r->nz;
    long p = 0;
    while (p < r->n && r->cell[p] < c0) p++;
    *a = p;
    while (p < r->n && r->cell[p] < c1) p++;
    *b = p;
}

/* pack_particle_slice (main.cpp:1330-1394): the slab's cell lists in order;
 * out10 as qor_get_particles.  Returns the count. */
long qor_get_particle_slab(qor_region* r, int i0, int w, long cap, double* out10, long* cell) {
    long a, b;
    slab_range(r, i0, w, &a, &b);
    const double* arrs[10] = {r->x, r->y, r->z, r->ux, r->uy, r->uz, r->g, r->q, r->cmr, r->chi};
    const long m = b - a < cap ? b - a : cap;
    if (out10)
        for (int k = 0; k < 10; k++) memcpy(out10 + k * cap, arrs[k] + a, sizeof(double) * (size_t)m);
    if (cell) memcpy(cell, r->cell + a, sizeof(long) * (size_t)m);
    return b - a;
}

/* unpack_particle_slice (main.cpp:1360-1423): the slab's lists are erased
 * and rebuilt from the given particles in the given order (cells from the
 * positions). */
void qor_replace_particle_slab(qor_region* r, int i0, int w, long n, const double* x, const double* y,
                               const double* z, const double* ux, const double* uy, const double* uz,
                               const double* g, const double* q, const double* cmr, const double* chi) {
    long a, b;
    slab_range(r, i0, w, &a, &b);
    double* arrs[10] = {r->x, r->y, r->z, r->ux, r->uy, r->uz, r->g, r->q, r->cmr, r->chi};
    const long tail = r->n - b;
    for (int k = 0; k < 10; k++) memmove(arrs[k] + a, arrs[k] + b, sizeof(double) * (size_t)tail);
    memmove(r->cell + a, r->cell + b, sizeof(long) * (size_t)tail);
    r->n -= b - a;
    if (n > 0) qor_add_particles(r, n, x, y, z, ux, uy, uz, g, q, cmr, chi);
}

/* particles per x-layer (calculate_layer_weights, balancing.cpp:25-40) */
void qor_layer_counts(qor_region* r, long* counts) {
    const long ynz = (long)r->ny * r->nz;
    for (int i = 0; i < r->nx; i++) counts[i] = 0;
    for (long p = 0; p < r->n; p++) counts[r->cell[p] / ynz]++;
}
