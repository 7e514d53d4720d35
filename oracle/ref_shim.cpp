// ORACLE / TEST INFRASTRUCTURE — not part of the product.
//
// C-ABI shim around the reference's own CPU implementation of the per-timestep
// PIC loop (QUILL `spatial_region`).  It is compiled together with the
// reference sources src/*.cpp minus src/main.cpp (see oracle/Makefile) into
// oracle/_ref/libquill_ref.so.  Tests and the CPU-baseline leg of bench.py
// load it to (1) pin the C restatement in oracle/qp_oracle.c and (2) check
// the CUDA path against the reference itself.
//
// The reference needs seven globals that normally live in src/main.cpp
// (advance.cpp:9-11, low-level.cpp:12-14, plist.cpp:4-5, mc.cpp:9); they are
// defined here with the values of a one-region (n_sr = 1) run.
//
// Step order is the time loop of src/main.cpp:2321-2331:
//   birth_from_vacuum(q) ; padvance(external_bz) ; compute_N ; compute_energy ;
//   fadvance()
// with the n_sr = 1 arguments n1 = n2 = 0 and the normalisations of
// src/main.cpp:2324-2327.

#include <cmath>
#include <cstring>
#include <vector>
#include "main.h"
#include "pusher.h"
#include "containers.h"
#include "balancing.h"

bool catching_enabled = false;
bool dump_photons = false;
double lambda = 1e-4;
int mpi_rank = 0;
int n_sr = 1;
int nm = 4;
bool qed_enabled = false;

namespace {
const double PI_ = 3.141592653589793;

struct RefRegion {
    spatial_region sr;
    int nx, ny, nz;
    double dx, dy, dz, dt;
    double lam;
    int qed;
    std::vector<double> icmr;
    int n1 = 0, n2 = 0;  // compute_N / compute_energy range [n1, nx - n2)
};

inline long lin(const RefRegion* r, int i, int j, int k) {
    return ((long)i * r->ny + j) * r->nz + k;
}
}  // namespace

extern "C" {

// solver: 0 FDTD, 1 NDFX, 2 FIVE_POINT ; pusher: 0 VAY, 1 BORIS
void* qref_create(int nx, int ny, int nz, double dx, double dy, double dz, double dt,
                  double lambda_cm, int solver, int pusher, int qed,
                  int n_ion, const double* icmr, int seed) {
    RefRegion* r = new RefRegion();
    r->nx = nx; r->ny = ny; r->nz = nz;
    r->dx = dx; r->dy = dy; r->dz = dz; r->dt = dt;
    r->lam = lambda_cm;
    r->qed = qed;
    lambda = lambda_cm;
    qed_enabled = qed != 0;
    r->icmr.assign(icmr, icmr + n_ion);
    maxwell_solver_enum se = solver == 0 ? maxwell_solver_enum::FDTD
                           : solver == 1 ? maxwell_solver_enum::NDFX
                                         : maxwell_solver_enum::FIVE_POINT;
    pusher_enum pe = pusher == 0 ? pusher_enum::VAY : pusher_enum::BORIS;
    // e_s = lambda / 2.4263086e-10, as src/main.cpp:2276
    r->sr.init(0, dx, dy, dz, dt, lambda_cm / 2.4263086e-10, 1, 1, 1, n_ion,
               r->icmr.empty() ? nullptr : r->icmr.data(), "results", se, pe);
    r->sr.create_arrays(nx, ny, nz, seed);
    return r;
}

void qref_destroy(void* h) { delete (RefRegion*)h; }

// Planes are (i, j, k) with k fastest, one double per cell per component.
void qref_set_fields(void* h, const double* ex, const double* ey, const double* ez,
                     const double* bx, const double* by, const double* bz) {
    RefRegion* r = (RefRegion*)h;
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                long c = lin(r, i, j, k);
                r->sr.ce[i][j][k].ex = ex[c];
                r->sr.ce[i][j][k].ey = ey[c];
                r->sr.ce[i][j][k].ez = ez[c];
                r->sr.cb[i][j][k].bx = bx[c];
                r->sr.cb[i][j][k].by = by[c];
                r->sr.cb[i][j][k].bz = bz[c];
            }
}

// out: 12 planes E(3) B(3) J(3) Bbar(3)
void qref_get_fields(void* h, double* out) {
    RefRegion* r = (RefRegion*)h;
    long nc = (long)r->nx * r->ny * r->nz;
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                long c = lin(r, i, j, k);
                out[0 * nc + c] = r->sr.ce[i][j][k].ex;
                out[1 * nc + c] = r->sr.ce[i][j][k].ey;
                out[2 * nc + c] = r->sr.ce[i][j][k].ez;
                out[3 * nc + c] = r->sr.cb[i][j][k].bx;
                out[4 * nc + c] = r->sr.cb[i][j][k].by;
                out[5 * nc + c] = r->sr.cb[i][j][k].bz;
                out[6 * nc + c] = r->sr.cj[i][j][k].jx;
                out[7 * nc + c] = r->sr.cj[i][j][k].jy;
                out[8 * nc + c] = r->sr.cj[i][j][k].jz;
                out[9 * nc + c] = r->sr.cbe[i][j][k].bex;
                out[10 * nc + c] = r->sr.cbe[i][j][k].bey;
                out[11 * nc + c] = r->sr.cbe[i][j][k].bez;
            }
}

// The initial pulses: f_init_cos (init.cpp:6-210) and f_init_focused
// (init.cpp:212-385) on the region's E and B, with the reference's argument
// order.
void qref_f_init_cos(void* h, double a0y, double a0z, double xsigma, double ysigma, double zsigma, double x0,
                     int sscos, int b_sign, double x1, double phase, double y0, double z0, int append, double phi,
                     double xtarget, double ytarget, double ztarget) {
    ((RefRegion*)h)->sr.f_init_cos(a0y, a0z, xsigma, ysigma, zsigma, x0, sscos, b_sign != 0, x1, phase, y0, z0,
                                   append != 0, phi, xtarget, ytarget, ztarget);
}

void qref_f_init_focused(void* h, double a0y, double a0z, double xsigma, double sigma0, double x0, double x1,
                         int b_sign, double phase, double y0, double z0, int append, double phi, int sscos, double K,
                         double xtarget, double ytarget, double ztarget) {
    ((RefRegion*)h)->sr.f_init_focused(a0y, a0z, xsigma, sigma0, x0, x1, b_sign != 0, phase, y0, z0, append != 0,
                                       phi, sscos, K, xtarget, ytarget, ztarget);
}

// f_init_boundaries + interpolate_be, as src/main.cpp:2288-2289
void qref_init_boundaries(void* h) {
    RefRegion* r = (RefRegion*)h;
    r->sr.f_init_boundaries();
    r->sr.interpolate_be();
}

// Particles are given in traversal order: within each cell the first one
// given becomes the list head.  Head insertion (plist.cpp:22-39) reverses, so
// they are placed from last to first.  start = head afterwards, as
// fill_cell_by_particles does (init.cpp:477).
void qref_add_particles(void* h, long n, const double* x, const double* y, const double* z,
                        const double* ux, const double* uy, const double* uz, const double* g,
                        const double* q, const double* cmr, const double* chi) {
    RefRegion* r = (RefRegion*)h;
    for (long p = n - 1; p >= 0; p--) {
        particle* a = r->sr.new_particle();
        a->x = x[p]; a->y = y[p]; a->z = z[p];
        a->ux = ux[p]; a->uy = uy[p]; a->uz = uz[p];
        a->g = g[p]; a->q = q[p]; a->cmr = cmr[p];
#ifndef QUILL_NOQED
        a->chi = chi ? chi[p] : 0.0;
#endif
        a->trn = 0;
        a->next = nullptr;
        a->previous = nullptr;
        int i = (int)a->x, j = (int)a->y, k = (int)a->z;
        // place() without its is_inside filter: loaded particles in the
        // boundary layers stay until p_boundary erases them in padvance.
        a->next = r->sr.cp[i][j][k].pl.head;
        if (a->next) a->next->previous = a;
        r->sr.cp[i][j][k].pl.head = a;
    }
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++)
                r->sr.cp[i][j][k].pl.start = r->sr.cp[i][j][k].pl.head;
}

long qref_count_particles(void* h) {
    RefRegion* r = (RefRegion*)h;
    long n = 0;
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++)
                for (particle* p = r->sr.cp[i][j][k].pl.head; p; p = p->next) n++;
    return n;
}

// Dump in traversal order (cells lexicographic, list from head).
// out: 10 arrays of n: x y z ux uy uz g q cmr chi ; cell: linear cell index
long qref_get_particles(void* h, long cap, double* out, long* cell) {
    RefRegion* r = (RefRegion*)h;
    long n = 0;
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++)
                for (particle* p = r->sr.cp[i][j][k].pl.head; p; p = p->next) {
                    if (n < cap) {
                        out[0 * cap + n] = p->x;
                        out[1 * cap + n] = p->y;
                        out[2 * cap + n] = p->z;
                        out[3 * cap + n] = p->ux;
                        out[4 * cap + n] = p->uy;
                        out[5 * cap + n] = p->uz;
                        out[6 * cap + n] = p->g;
                        out[7 * cap + n] = p->q;
                        out[8 * cap + n] = p->cmr;
#ifndef QUILL_NOQED
                        out[9 * cap + n] = p->chi;
#else
                        out[9 * cap + n] = 0.0;
#endif
                        if (cell) cell[n] = lin(r, i, j, k);
                    }
                    n++;
                }
    return n;
}

// diag[0..]: N_e N_p N_ph N_qp_e N_qp_p N_qp_g energy_f energy_e energy_p
//            energy_ph  then per ion population: N_qp_i, ienergy
static void fill_diag(RefRegion* r, double* d) {
    spatial_region& s = r->sr;
    d[0] = s.N_e; d[1] = s.N_p; d[2] = s.N_ph;
    d[3] = s.N_qp_e; d[4] = s.N_qp_p; d[5] = s.N_qp_g;
    d[6] = s.energy_f; d[7] = s.energy_e; d[8] = s.energy_p; d[9] = s.energy_ph;
    for (size_t n = 0; n < r->icmr.size(); n++) {
        d[10 + 2 * n] = s.N_qp_i[n];
        d[11 + 2 * n] = s.ienergy[n];
    }
}

int qref_diag_len(void* h) { return 10 + 2 * (int)((RefRegion*)h)->icmr.size(); }

// One or more full timesteps in the order of src/main.cpp:2321-2331.
// diag (nullable) receives qref_diag_len() doubles per step.
void qref_step(void* h, int nsteps, double external_bz, double* diag) {
    RefRegion* r = (RefRegion*)h;
    lambda = r->lam;
    qed_enabled = r->qed != 0;
    const double dx = r->dx, dy = r->dy, dz = r->dz;
    for (int l = 0; l < nsteps; l++) {
        r->sr.birth_from_vacuum(8 * PI_ * PI_ / (dx * dy * dz) * 2.818e-13 / lambda);
        r->sr.padvance(external_bz);
        r->sr.compute_N(r->n1, r->n2, dx * dy * dz * 1.11485e13 * lambda / (8 * PI_ * PI_ * PI_));
        r->sr.compute_energy(r->n1, r->n2, 0.5 * dx * dy * dz * 3.691e4 * lambda / 1e7,
                             8.2e-14 * dx * dy * dz * 1.11485e13 * lambda / (8 * PI_ * PI_ * PI_));
        r->sr.fadvance();
        if (diag) fill_diag(r, diag + (long)l * qref_diag_len(h));
    }
}

// Particle half of a step only (padvance), for kernel-level tests.
void qref_padvance(void* h, double external_bz) {
    RefRegion* r = (RefRegion*)h;
    qed_enabled = r->qed != 0;
    r->sr.padvance(external_bz);
}

// Field half of a step only (solver advance + interpolate_be).
void qref_fadvance(void* h) { ((RefRegion*)h)->sr.fadvance(); }

void qref_compute_diag(void* h, double* diag) {
    RefRegion* r = (RefRegion*)h;
    const double dx = r->dx, dy = r->dy, dz = r->dz;
    lambda = r->lam;
    r->sr.compute_N(r->n1, r->n2, dx * dy * dz * 1.11485e13 * lambda / (8 * PI_ * PI_ * PI_));
    r->sr.compute_energy(r->n1, r->n2, 0.5 * dx * dy * dz * 3.691e4 * lambda / 1e7,
                         8.2e-14 * dx * dy * dz * 1.11485e13 * lambda / (8 * PI_ * PI_ * PI_));
    fill_diag(r, diag);
}

// --- single-particle kernels -------------------------------------------------

// state[0..6] = ux uy uz g (in/out) ; pusher 0 VAY, 1 BORIS (pusher.cpp:5-97)
void qref_push(int pusher, double cmr, double* state, const double* e, const double* b, double dt) {
    particle p;
    p.ux = state[0]; p.uy = state[1]; p.uz = state[2]; p.g = state[3]; p.cmr = cmr;
    vector3d ev, bv;
    ev.x = e[0]; ev.y = e[1]; ev.z = e[2];
    bv.x = b[0]; bv.y = b[1]; bv.z = b[2];
    if (pusher == 0) push_vay(p, ev, bv, dt); else push_boris(p, ev, bv, dt);
    state[0] = p.ux; state[1] = p.uy; state[2] = p.uz; state[3] = p.g;
}

// Current deposition of one particle moving by d (cell units) into the
// region's J (deposition.cpp:41-356).  pos[3] in/out.
void qref_jdeposition(void* h, double* pos, const double* d, double q) {
    RefRegion* r = (RefRegion*)h;
    particle p;
    p.x = pos[0]; p.y = pos[1]; p.z = pos[2]; p.q = q;
    vector3d dv;
    dv.x = d[0]; dv.y = d[1]; dv.z = d[2];
    r->sr.jdeposition(p, dv);
    pos[0] = p.x; pos[1] = p.y; pos[2] = p.z;
}

void qref_zero_j(void* h) {
    RefRegion* r = (RefRegion*)h;
    for (int i = 0; i < r->nx; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                r->sr.cj[i][j][k].jx = 0;
                r->sr.cj[i][j][k].jy = 0;
                r->sr.cj[i][j][k].jz = 0;
            }
}

// Field gather at (x, y, z) in cell units (deposition.cpp:431-471).
void qref_gather(void* h, double x, double y, double z, double* e, double* b) {
    RefRegion* r = (RefRegion*)h;
    vector3d ev = r->sr.e_to_particle(x, y, z);
    vector3d bv = r->sr.b_to_particle(x, y, z);
    e[0] = ev.x; e[1] = ev.y; e[2] = ev.z;
    b[0] = bv.x; b[1] = bv.y; b[2] = bv.z;
}

#ifndef QUILL_NOQED
// QED rates (mc.cpp:26-116).  w may rescale r (returned through *r).
double qref_chi(void* h, const double* e, const double* b, const double* u, double g) {
    vector3d ev, bv, uv;
    ev.x = e[0]; ev.y = e[1]; ev.z = e[2];
    bv.x = b[0]; bv.y = b[1]; bv.z = b[2];
    uv.x = u[0]; uv.y = u[1]; uv.z = u[2];
    return ((RefRegion*)h)->sr.chi(ev, bv, uv, g);
}
double qref_w(void* h, double g, double* r, double chi) {
    return ((RefRegion*)h)->sr.w(g, *r, chi);
}
double qref_tilde_w(void* h, double g, double r, double chi) {
    return ((RefRegion*)h)->sr.tilde_w(g, r, chi);
}
double qref_mathcal_W(void* h, const double* e, const double* b) {
    vector3d ev, bv;
    ev.x = e[0]; ev.y = e[1]; ev.z = e[2];
    bv.x = b[0]; bv.y = b[1]; bv.z = b[2];
    return ((RefRegion*)h)->sr.mathcal_W(ev, bv);
}
#endif

// Lagged-Fibonacci stream (mc.cpp:12-23) seeded by create_arrays(seed).
double qref_get_rand(void* h) { return ((RefRegion*)h)->sr.get_rand(); }

// spatial_region::moving_window (advance.cpp:389-454).
void qref_moving_window(void* h) { ((RefRegion*)h)->sr.moving_window(); }

// spatial_region::pmerging (mc.cpp:202-462).  mode 1 = "ti", 2 = "nl";
// ppd has 3 + n_ion entries (electrons, positrons, photons, ion populations).
void qref_pmerging(void* h, int mode, const double* ppd) {
    RefRegion* r = (RefRegion*)h;
    std::vector<double> p(ppd, ppd + 3 + r->icmr.size());
    r->sr.pmerging(p.data(), mode == 1 ? "ti" : "nl");
}

// --- x-slabs (the n_sr > 1 exchange of src/main.cpp:1286-1514) -------------

void qref_set_diag_range(void* h, int lo, int hi) {
    RefRegion* r = (RefRegion*)h;
    r->n1 = lo;
    r->n2 = r->nx - hi;
}

// ce cb cj cbe of the cells with i in [i0, i0 + w): 12 blocks of w*ny*nz
void qref_get_field_slab(void* h, int i0, int w, double* out) {
    RefRegion* r = (RefRegion*)h;
    const long m = (long)w * r->ny * r->nz;
    for (int i = i0; i < i0 + w; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                const long c = lin(r, i - i0, j, k);
                const celle& e = r->sr.ce[i][j][k];
                const cellb& b = r->sr.cb[i][j][k];
                const cellj& jj = r->sr.cj[i][j][k];
                const cellbe& be = r->sr.cbe[i][j][k];
                const double v[12] = {e.ex, e.ey, e.ez, b.bx, b.by, b.bz, jj.jx, jj.jy, jj.jz, be.bex, be.bey, be.bez};
                for (int a = 0; a < 12; a++) out[a * m + c] = v[a];
            }
}

void qref_set_field_slab(void* h, int i0, int w, const double* in) {
    RefRegion* r = (RefRegion*)h;
    const long m = (long)w * r->ny * r->nz;
    for (int i = i0; i < i0 + w; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) {
                const long c = lin(r, i - i0, j, k);
                celle& e = r->sr.ce[i][j][k];
                cellb& b = r->sr.cb[i][j][k];
                cellj& jj = r->sr.cj[i][j][k];
                cellbe& be = r->sr.cbe[i][j][k];
                e.ex = in[c]; e.ey = in[m + c]; e.ez = in[2 * m + c];
                b.bx = in[3 * m + c]; b.by = in[4 * m + c]; b.bz = in[5 * m + c];
                jj.jx = in[6 * m + c]; jj.jy = in[7 * m + c]; jj.jz = in[8 * m + c];
                be.bex = in[9 * m + c]; be.bey = in[10 * m + c]; be.bez = in[11 * m + c];
            }
}

// The slab's cell lists, each from its head (the order pack_cell sends).
long qref_get_particle_slab(void* h, int i0, int w, long cap, double* out, long* cell) {
    RefRegion* r = (RefRegion*)h;
    long n = 0;
    for (int i = i0; i < i0 + w; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++)
                for (particle* p = r->sr.cp[i][j][k].pl.head; p; p = p->next) {
                    if (out && n < cap) {
#ifndef QUILL_NOQED
                        const double chi = p->chi;
#else
                        const double chi = 0.0;
#endif
                        const double v[10] = {p->x, p->y, p->z, p->ux, p->uy, p->uz, p->g, p->q, p->cmr, chi};
                        for (int a = 0; a < 10; a++) out[a * cap + n] = v[a];
                    }
                    if (cell && n < cap) cell[n] = lin(r, i, j, k);
                    n++;
                }
    return n;
}

// The slab's lists are erased (spatial_region::erase) and rebuilt with the
// given particles, in the given order inside each cell (as unpack_cell
// leaves them); a particle's cell follows from its position.
void qref_replace_particle_slab(void* h, int i0, int w, long n, const double* x, const double* y, const double* z,
                                const double* ux, const double* uy, const double* uz, const double* g,
                                const double* q, const double* cmr, const double* chi) {
    RefRegion* r = (RefRegion*)h;
    for (int i = i0; i < i0 + w; i++)
        for (int j = 0; j < r->ny; j++)
            for (int k = 0; k < r->nz; k++) r->sr.erase(r->sr.cp[i][j][k].pl);
    qref_add_particles(h, n, x, y, z, ux, uy, uz, g, q, cmr, chi);
}

// particles per x-layer: spatial_region::calculate_layer_weights with
// particle weight 1, minus the ny*nz it starts each layer from
void qref_layer_counts(void* h, long* counts) {
    RefRegion* r = (RefRegion*)h;
    std::vector<double> wts = r->sr.calculate_layer_weights(1.0);
    for (int i = 0; i < r->nx; i++) counts[i] = (long)(wts[i] - (double)r->ny * r->nz);
}

// calculate_optimal_partition / normalize_new_partition /
// calculate_partition_imbalance (balancing.cpp:54-175)
void qref_optimal_partition(const double* weights, int n, int regions, int overlap, int* out) {
    std::vector<double> wv(weights, weights + n);
    std::vector<int> p = calculate_optimal_partition(wv, regions, overlap);
    for (int i = 0; i < regions; i++) out[i] = p[i];
}

void qref_normalize_partition(const int* old_p, const int* new_p, int regions, int overlap, int* out) {
    std::vector<int> a(old_p, old_p + regions), b(new_p, new_p + regions);
    std::vector<int> p = normalize_new_partition(a, b, overlap);
    for (int i = 0; i < regions; i++) out[i] = p[i];
}

double qref_partition_imbalance(const double* weights, int n, const int* part, int regions, int overlap) {
    std::vector<double> wv(weights, weights + n);
    std::vector<int> p(part, part + regions);
    return calculate_partition_imbalance(wv, p, overlap);
}

// Catching (catching_enabled, main.cpp:3531-3534): particles erased outside
// the region are recorded by delete_particle and their energy summed by
// update_energy_deleted (low-level.cpp:247-313).  The flag is the process's.
void qref_set_catching(void* h, int on) {
    (void)h;
    catching_enabled = on != 0;
}

// energy_e_deleted, energy_p_deleted, energy_ph_deleted, then
// ienergy_deleted per ion population (Joules); the record list is dropped.
void qref_energy_deleted(void* h, double* out) {
    RefRegion* r = (RefRegion*)h;
    out[0] = r->sr.energy_e_deleted;
    out[1] = r->sr.energy_p_deleted;
    out[2] = r->sr.energy_ph_deleted;
    for (size_t m = 0; m < r->icmr.size(); m++) out[3 + m] = r->sr.ienergy_deleted[m];
    r->sr.deleted_particles.clear();
}

}  // extern "C"
