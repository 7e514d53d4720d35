/*
 * quill_b200 — B200-native per-timestep particle-in-cell loop of QUILL
 * (QUILL-PIC/Quill), one GPU, one spatial region (n_sr = 1).
 *
 * C ABI of libquill_b200.so.  Plain pointers and sizes only; every call
 * returns a qp_status and leaves a message for qp_last_error().  One handle
 * owns one region on one GPU; a handle is not thread-safe.
 *
 * The reference has no plugin or FFI: its seam is the C++ object
 * `spatial_region` (include/main.h:17-170) driven by main() in
 * src/main.cpp:2319-2432.  Each entry point below cites the member function
 * or code it replaces.
 *
 * Units are the reference's: time in 1/omega, lengths in c/omega, particle
 * positions in cell units (x = i at node i), momenta u = p/(mc), fields in
 * m c omega / e.  Field planes are indexed (i, j, k) with k fastest, as
 * field3d (src/containers.cpp:4-22).
 */
#ifndef QUILL_B200_H
#define QUILL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QP_MAX_SPECIES 8

typedef enum {
    QP_OK = 0,
    QP_ERR_CONFIG = 1,   /* bad parameters or input data */
    QP_ERR_CAPACITY = 2, /* a particle store is full (device append overflow) */
    QP_ERR_NAN = 3,      /* non-finite particle state detected */
    QP_ERR_TIMEOUT = 4,  /* a bounded device wait gave up */
    QP_ERR_CUDA = 5,     /* CUDA runtime error */
    QP_ERR_STATE = 6,    /* call not valid in the handle's current state */
    QP_ERR_ARG = 7       /* null pointer or out-of-range argument */
} qp_status;

/* maxwell_solver_enum, include/containers.h:82-84 */
typedef enum { QP_SOLVER_FDTD = 0, QP_SOLVER_NDFX = 1, QP_SOLVER_FIVE_POINT = 2 } qp_solver;
/* pusher_enum, include/containers.h:86-88 */
typedef enum { QP_PUSHER_VAY = 0, QP_PUSHER_BORIS = 1 } qp_pusher;
/* FP64: the reference arithmetic.  MIXED: positions as int cell + f32
 * offset, FP32 push, gather, deposition and stencils; FP64 diagnostics. */
typedef enum { QP_PREC_FP64 = 0, QP_PREC_MIXED = 1 } qp_precision;

typedef struct {
    int nx, ny, nz;              /* cells per axis (spatial_region::create_arrays) */
    double dx, dy, dz, dt;       /* c/omega and 1/omega (spatial_region::init) */
    double lambda_cm;            /* wavelength in cm: e_s = lambda/2.4263086e-10 (main.cpp:2276)
                                    and the N / energy normalisations (main.cpp:2324-2327) */
    int solver;                  /* qp_solver */
    int pusher;                  /* qp_pusher */
    int qed;                     /* 0/1: photon emission, Breit-Wheeler pairs, vacuum pairs */
    int precision;               /* qp_precision */
    uint64_t seed;               /* counter-based random stream seed (QED) */
    int n_species;
    double cmr[QP_MAX_SPECIES];  /* charge/mass: -1 electrons, +1 positrons, 0 photons,
                                    anything else an ion population (icmr, main.cpp:3251-3330),
                                    ion populations numbered in table order */
    int64_t capacity[QP_MAX_SPECIES]; /* particle slots per species (0 = grow on load only) */
    int device;                  /* CUDA device ordinal */
} qp_params;

/* Per-step diagnostics: spatial_region::compute_N and compute_energy
 * (fout.cpp:41-138) with the normalisations of main.cpp:2326-2327. */
typedef struct {
    double N_e, N_p, N_ph;               /* weighted counts */
    int64_t N_qp_e, N_qp_p, N_qp_g;      /* macro-particle counts */
    double energy_f, energy_e, energy_p, energy_ph; /* Joules */
    int n_ion;
    int64_t N_qp_i[QP_MAX_SPECIES];
    double ienergy[QP_MAX_SPECIES];
    int64_t n_macro[QP_MAX_SPECIES];     /* live particles per species (table order) */
    int32_t status;                      /* qp_status raised on the device in this step */
    int32_t pad_;
    double energy_erased;                /* Joules carried off by the particles erased in this step
                                            (p_boundary and place), with the normalisation and
                                            species signs of the energy terms; 0 unless enabled by
                                            qp_set_erased_tracking.  No reference counterpart. */
    double energy_erased_sp[QP_MAX_SPECIES]; /* the same per species (table order), as
                                            update_energy_deleted (low-level.cpp:288-313) */
} qp_diag;

typedef struct qp_handle qp_handle;

/* Library version string. */
const char* qp_version(void);

/* Message of the last failing call on h (or of the last failed qp_create
 * when h is NULL). */
const char* qp_last_error(const qp_handle* h);

/* spatial_region::init + create_arrays (low-level.cpp:61-150): allocate the
 * fields and particle stores of one region on params->device. */
int qp_create(const qp_params* params, qp_handle** out);

/* ~spatial_region (low-level.cpp:152-184). */
int qp_destroy(qp_handle* h);

/* Copy E and B from planes of nx*ny*nz doubles each (k fastest), in host
 * or device memory; the device copy is converted to the handle's precision.  Replaces the field
 * initialisers writing spatial_region::ce/cb (init.cpp:6-400). */
int qp_load_fields(qp_handle* h, const double* ex, const double* ey, const double* ez,
                   const double* bx, const double* by, const double* bz);

/* f_init_boundaries + interpolate_be, called once after loading
 * (main.cpp:2288-2289, advance.cpp:85-88, maxwell.cpp:135/338/532). */
int qp_init_boundaries(qp_handle* h);

/* Append n particles of one species from host or device arrays (cell
 * units; chi may be NULL).  Within a cell the given order becomes the traversal order;
 * particles of a later call precede those already in the cell, as head
 * insertion by spatial_region::place (plist.cpp:22-39) would put them.
 * Positions must lie in [0, n) per axis.  Replaces new_particle + place
 * in fill_cell_by_particles (init.cpp:402-478). */
int qp_load_particles(qp_handle* h, int species, int64_t n, const double* x, const double* y,
                      const double* z, const double* ux, const double* uy, const double* uz,
                      const double* g, const double* q, const double* chi);

/* nsteps timesteps, each in the order of main.cpp:2321-2331:
 *   birth_from_vacuum -> padvance(external_bz) -> compute_N/compute_energy
 *   -> fadvance.
 * diag (nullable) receives one record per step. */
int qp_step(qp_handle* h, int nsteps, double external_bz, qp_diag* diag);

/* Diagnostics of the last completed step. */
int qp_get_diag(qp_handle* h, qp_diag* out);

/* Copy fields out (host or device memory): 12 planes E(3) B(3) J(3)
 * Bbar(3), FP64. */
int qp_dump_fields(qp_handle* h, double* out12);

/* Live particle count of one species. */
int qp_count_particles(qp_handle* h, int species, int64_t* n);

/* Copy one species to host in traversal order (cells lexicographic, list
 * order inside a cell).  Each pointer may be NULL; cell receives the linear
 * cell index (i*ny + j)*nz + k.  cap is the capacity of every array. */
int qp_dump_particles(qp_handle* h, int species, int64_t cap, double* x, double* y, double* z,
                      double* ux, double* uy, double* uz, double* g, double* q, double* chi,
                      int64_t* cell);

/* Device-resident snapshot of the full state (fields, particles, random
 * counters, step) into slot 0..3 / restore from it.  No reference
 * counterpart (the reference has no checkpointing). */
int qp_checkpoint(qp_handle* h, int slot);
int qp_restore(qp_handle* h, int slot);

/* Wait for all work of the handle's stream. */
int qp_synchronize(qp_handle* h);

/* Run all work of h on the given cudaStream_t.  NULL keeps the handle's own
 * stream, which is created non-blocking: it is not ordered with the legacy
 * default stream, so a caller that works on the default stream orders the
 * two itself (qp_synchronize before reusing memory the handle reads or
 * writes, or hand the handle a stream of its own here). */
int qp_set_stream(qp_handle* h, void* cuda_stream);

/* Number of this library's kernel launches issued since the handle was
 * created (for launch accounting). */
int qp_launch_count(qp_handle* h, int64_t* out);

/* Device evaluation of the QED rate functions of mc.cpp:26-116 for n
 * samples (host or device arrays).  in: 12 doubles per sample
 * (e[3] b[3] u[3] g r chi); out: 5 per sample (chi(e,b,u,g), w(g,r,chi),
 * r after w (w rescales r for chi <= 0.133), tilde_w(g,r,chi),
 * mathcal_W(e,b)).  e_s = lambda_cm / 2.4263086e-10 (main.cpp:2276). */
int qp_eval_qed_rates(int device, double lambda_cm, int64_t n, const double* in, double* out);

/* Same results as qp_eval_qed_rates, for callers that cannot allocate GPU
 * memory (their device memory is owned by another allocator, or they cannot
 * afford the device-wide synchronisation of cudaFree).  No counterpart in
 * the reference.  Allocates nothing: inputs and outputs are staged in a
 * fixed array inside the library (at most 16384 samples per call; larger n
 * is rejected with QP_ERR_ARG).  All calls share that array: calls that
 * overlap on the GPU race.  The first call on a device looks the array up
 * and should come before any stream capture; the address it finds is kept,
 * so the call must not be used after cudaDeviceReset.  The caller's current
 * device is left as it was.  Errors: qp_last_error(NULL). */
int qp_eval_qed_rates_noalloc(int device, double lambda_cm, int64_t n, const double* in, double* out);

/* Per-phase CUDA-event timing of qp_step on the handle's stream: enable
 * (resets the totals) or disable.  No reference counterpart (the reference
 * logs coarse times() wall clocks only, main.cpp:2228-2230). */
int qp_set_timing(qp_handle* h, int enable);

/* Accumulated milliseconds since qp_set_timing(h, 1): [0] particle push and
 * current deposition, [1] rebin, [2] Maxwell solver + Bbar, [3] J reset and
 * diagnostics; *steps = timed steps (nullable). */
int qp_get_timing(qp_handle* h, double* ms4, int64_t* steps);

/* QED steps since qp_set_timing(h, 1), in milliseconds, each part of [0] of
 * qp_get_timing: [0] preparation (room for the particles a push can create,
 * the vacuum-pair kernel, the merge of its pairs into the cell lists, and
 * the host synchronisation that reads their count), [1] the push kernels,
 * [2] the read-back of the born-particle counts after them; *steps = timed
 * QED steps (nullable). */
int qp_get_qed_timing(qp_handle* h, double* ms3, int64_t* steps);

/* Reference-order current deposition (parity switch; FP64, QED off): each
 * step sums every J element's terms from zero in the order the reference's
 * padvance adds them (cells lexicographic, each cell's list of all species
 * from its head, then segment and term; advance.cpp:90-387,
 * deposition.cpp:13-39), instead of with atomics, so that the region stays
 * bit-identical to the reference over any number of steps.  Several times
 * slower than the default deposition and 1.3 kB of scratch per particle;
 * for parity runs.  With several species the cross-species list order
 * starts, after a load, as species 0's particles of each cell first, then
 * species 1's, and so on.  enable = 0 releases the scratch.  QP_ERR_CONFIG
 * for mixed precision or QED. */
int qp_set_ordered_current(qp_handle* h, int enable);

/* Sum the energy of the particles each step erases (p_boundary before the
 * push, place() after it) into qp_diag.energy_erased, so that
 * energy_f + energy_e + energy_p + energy_ph + ienergy plus the erased energy
 * accumulated over the steps is the closed energy balance of the region.
 * QED-off steps only.  No reference counterpart (the reference drops erased
 * particles' energy unless it catches them, main.cpp:1516-1689). */
int qp_set_erased_tracking(qp_handle* h, int enable);

/* spatial_region::moving_window (advance.cpp:389-454), called by the time
 * loop after a step when check_moving_window (main.cpp:1953-1979) says so:
 * the particles of the layer i = 0 are erased, E, B and Bbar move one cell
 * towards -x (the last layer becomes zero; J is left as it is) and every
 * particle moves one cell towards -x with them.  New plasma for the front
 * layer is the caller's (qp_load_particles), as add_moving_window_particles
 * (main.cpp:1750-1883). */
int qp_moving_window(qp_handle* h);

/* Catching (catching = on: delete_particle, low-level.cpp:247-259): record
 * every particle the steps erase (p_boundary before the push, place() after
 * it) into a device buffer of `capacity` records; enable = 0 frees it.
 * Records beyond the capacity are dropped and counted.  Use with
 * qp_set_erased_tracking for the energy_deleted output.  Photons or pairs
 * born outside the region (QED) are not recorded. */
int qp_set_catching(qp_handle* h, int enable, int64_t capacity);

/* dump_photons (advance.cpp:302-306): photons emitted by leptons are
 * deleted as they are born and recorded in the capture buffer that
 * qp_get_caught reads (allocated with `capacity` records if catching has
 * none), their energy counted in qp_diag.energy_erased_sp of the photon
 * species.  Needs QED. */
int qp_set_dump_photons(qp_handle* h, int enable, int64_t capacity);

/* The recorded particles (species index, position in cell units, u, g, q,
 * chi), ordered by species, then as the reference deletes them: by step,
 * the p_boundary erasures before the moves out of the region, each in
 * traversal order.  With every array pointer NULL only *n_out (and
 * *dropped) are set and the buffer is kept; otherwise cap must be at least
 * *n_out, the records are copied (host or device arrays, each nullable) and
 * the buffer is emptied, as write_deleted_particles clears its list
 * (main.cpp:189-330). */
int qp_get_caught(qp_handle* h, int64_t cap, int32_t* species, double* x, double* y, double* z, double* ux,
                  double* uy, double* uz, double* g, double* q, double* chi, int64_t* n_out, int64_t* dropped);

/* Particle tracks (start_tracking, main.cpp:1516-1612; fout_tracks,
 * fout.cpp:706-734): enable = 1 gives every particle a track number, 0 =
 * untracked, carried by the steps; enable = 0 drops them.  Particles that
 * join later (loads, QED births) are untracked. */
int qp_set_tracking(qp_handle* h, int enable);

/* Traversal position of the first particle of `species` in each of the n
 * cells (linear index (i*ny + j)*nz + k), -1 for an empty cell: the head of
 * the reference's cell list restricted to that species. */
int qp_first_in_cells(qp_handle* h, int species, int64_t n, const int64_t* cells, int64_t* first);

/* Give the particles at the n traversal positions the track numbers given. */
int qp_set_track_numbers(qp_handle* h, int species, int64_t n, const int64_t* positions, const int64_t* numbers);

/* The tracked particles of a species in traversal order (at most 65536):
 * track number, position in cell units, u, g, q, chi (arrays host or
 * device, nullable; all NULL: count only into *n_out). */
int qp_get_tracked(qp_handle* h, int species, int64_t cap, int64_t* trn, double* x, double* y, double* z,
                   double* ux, double* uy, double* uz, double* g, double* q, double* chi, int64_t* n_out);

/* x-slabs, for a decomposition into overlapping x-slab regions (the
 * reference's n_sr > 1 layout and synchronize_regions, main.cpp:1286-1514).
 *
 * The diagnostics of qp_step count only the cells with i in [i_lo, i_hi)
 * (compute_N / compute_energy's n1 and n2, main.cpp:2325-2327); the
 * default is the whole region. */
int qp_set_diag_range(qp_handle* h, int i_lo, int i_hi);

/* Copy the 12 field planes (E B J Bbar) of the slab i in [i0, i0 + width)
 * out / in: 12 blocks of width*ny*nz doubles, k fastest (send_field_slice /
 * receive_field_slice, main.cpp:1286-1302).  Host or device memory. */
int qp_get_field_slab(qp_handle* h, int i0, int width, double* out12);
int qp_set_field_slab(qp_handle* h, int i0, int width, const double* in12);

/* The particles of one species in the slab, in traversal order (cell
 * lists in order, pack_particle_slice, main.cpp:1330-1394): positions in
 * cell units of this region, host or device arrays.  All arrays NULL: count
 * only. */
int qp_get_particle_slab(qp_handle* h, int species, int i0, int width, int64_t cap, double* x, double* y, double* z,
                         double* ux, double* uy, double* uz, double* g, double* q, double* chi, int64_t* n_out);

/* Replace the particles of one species in the slab by the n given
 * (unpack_particle_slice, main.cpp:1360-1423): the slab's cell lists become
 * exactly these, in the given order inside each cell; a particle's cell
 * follows from its position.  Host or device arrays. */
int qp_replace_particle_slab(qp_handle* h, int species, int i0, int width, int64_t n, const double* x,
                             const double* y, const double* z, const double* ux, const double* uy, const double* uz,
                             const double* g, const double* q, const double* chi);

/* The field slices the reference's output writers use (fout.cpp:180-235),
 * for the 12 planes E B J Bbar in turn: for each i the nz/2 line along y
 * (ny values) and the ny/2 line along z (nz values), then the plane i = ix
 * (ny*nz values, k fastest).  out: 12 * (nx*(ny+nz) + ny*nz) doubles, host
 * or device. */
int qp_dump_field_slices(qp_handle* h, int ix, double* out);

/* max over the cells with i in [i0, i1) of Ex^2+Ey^2+Ez^2+Bx^2+By^2+Bz^2
 * (spatial_region::get_max_w, low-level.cpp:512-532), for the moving
 * window's AUTO mode (check_moving_window, main.cpp:1961-1975). */
int qp_max_w(qp_handle* h, int i0, int i1, double* out);

/* Quasiparticles per x-layer, all species: counts[nx] (the particle term
 * of spatial_region::calculate_layer_weights, balancing.cpp:25-40). */
int qp_layer_counts(qp_handle* h, int64_t* counts);

/* Particle merging modes (the reference's `pmerging` parameter, main.cpp:3397). */
enum { QP_MERGE_TI = 1, QP_MERGE_NL = 2 };

/* spatial_region::pmerging (mc.cpp:198-462), called by the time loop before
 * a step when evaluate_merging_condition (main.cpp:1691-1748) found too many
 * macro-particles.  ppd holds one deletion probability per species in table
 * order ([0, 1)); QP_MERGE_TI deletes every particle with ppd[0],
 * QP_MERGE_NL each species' particles with ppd[s] / (1 + (2|q|/<|q|>)^4)
 * and rescales the survivors by 1 / (1 - that probability).  The weights
 * of each species are then renormalised to keep its total charge.  The
 * survivors keep their traversal order.  The random numbers are the
 * counter-based stream of the handle's seed, so the deletions match the
 * reference in distribution, not particle for particle. */
int qp_pmerging(qp_handle* h, int mode, const double* ppd);

/* Discrete adjoint (no reference counterpart): runs nsteps steps from the
 * handle's current state and returns the loss L = energy_e after the last
 * step (compute_energy's electron kinetic energy, fout.cpp:87-138) with its
 * exact gradients with respect to the six field planes as loaded by
 * qp_load_fields (grad_fields: 6*nx*ny*nz doubles, Ex Ey Ez Bx By Bz, the
 * zeroing of qp_init_boundaries applied) and to every electron's weight q
 * (grad_q: one double per particle, in the traversal order qp_dump_particles
 * returns at the start).  Covers FP64, FDTD, Boris, QED off, one species of
 * cmr -1; qp_init_boundaries must have run.  The state is saved every
 * `every` steps and each segment is re-run forward once for the backward
 * sweep (memory: about (nsteps/every) states + every step records).  The
 * handle is left in its state at entry.  Pointers may be host or device
 * memory; each of loss, grad_fields and grad_q is nullable. */
int qp_adjoint_energy(qp_handle* h, int nsteps, int every, double external_bz, double* grad_fields,
                      double* grad_q, double* loss);

#ifdef __cplusplus
}
#endif
#endif /* QUILL_B200_H */
