/* ORACLE / TEST INFRASTRUCTURE — a CPU restatement of QUILL's per-timestep
 * PIC loop used only as a checker by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py.  Never linked into the product.
 *
 * Parity: pinned bit-for-bit against the reference's own sources compiled by
 * oracle/Makefile (`make ref`), see tests/test_oracle_vs_ref.py, and against
 * the committed golden vectors in tests/golden/.
 */
#ifndef QP_ORACLE_H
#define QP_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct qor_region qor_region;

/* solver: 0 FDTD, 1 NDFX, 2 FIVE_POINT ; pusher: 0 VAY, 1 BORIS */
qor_region* qor_create(int nx, int ny, int nz, double dx, double dy, double dz, double dt,
                       double lambda_cm, int solver, int pusher, int qed, int n_ion,
                       const double* icmr, int seed);
void qor_destroy(qor_region* r);
void qor_set_fields(qor_region* r, const double* ex, const double* ey, const double* ez,
                    const double* bx, const double* by, const double* bz);
void qor_get_fields(qor_region* r, double* out12);
void qor_init_boundaries(qor_region* r);
void qor_add_particles(qor_region* r, long n, const double* x, const double* y, const double* z,
                       const double* ux, const double* uy, const double* uz, const double* g,
                       const double* q, const double* cmr, const double* chi);
long qor_count_particles(qor_region* r);
long qor_get_particles(qor_region* r, long cap, double* out10, long* cell);
int qor_diag_len(qor_region* r);
void qor_step(qor_region* r, int nsteps, double external_bz, double* diag);
void qor_padvance(qor_region* r, double external_bz);
void qor_fadvance(qor_region* r);
void qor_compute_diag(qor_region* r, double* diag);
void qor_push(int pusher, double cmr, double* state, const double* e, const double* b, double dt);
void qor_jdeposition(qor_region* r, double* pos, const double* d, double q);
void qor_zero_j(qor_region* r);
void qor_gather(qor_region* r, double x, double y, double z, double* e, double* b);
double qor_chi(qor_region* r, const double* e, const double* b, const double* u, double g);
double qor_w(qor_region* r, double g, double* rr, double chi);
double qor_tilde_w(qor_region* r, double g, double rr, double chi);
double qor_mathcal_W(qor_region* r, const double* e, const double* b);
double qor_get_rand(qor_region* r);
/* spatial_region::moving_window: shift by one cell towards -x */
void qor_moving_window(qor_region* r);
/* particle merging, mode 1 "ti", 2 "nl"; ppd[3 + n_ion] */
void qor_pmerging(qor_region* r, int mode, const double* ppd);
/* x-slabs: diagnostics over i in [lo, hi); field planes and cell lists of
 * the cells with i in [i0, i0 + w) */
void qor_set_diag_range(qor_region* r, int lo, int hi);
void qor_get_field_slab(qor_region* r, int i0, int w, double* out12);
void qor_set_field_slab(qor_region* r, int i0, int w, const double* in12);
long qor_get_particle_slab(qor_region* r, int i0, int w, long cap, double* out10, long* cell);
void qor_replace_particle_slab(qor_region* r, int i0, int w, long n, const double* x, const double* y,
                               const double* z, const double* ux, const double* uy, const double* uz,
                               const double* g, const double* q, const double* cmr, const double* chi);
void qor_layer_counts(qor_region* r, long* counts);

#ifdef __cplusplus
}
#endif
#endif
