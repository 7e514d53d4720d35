// FP64 path: the reference arithmetic on the GPU.  Built with --fmad=false so
// that every multiply and add rounds separately, as the reference CPU build
// does with -ffp-contract=off.
#include "qp_kernels.cuh"
#include "qp_qed.cuh"

namespace qp {

// One thread per particle of a chunk, in traversal order (advance.cpp:90-387 with QED
// off: photons fly straight without current, :155-252; leptons and ions are
// pushed and deposit, :253-371).  The particle is read through perm from the
// previous layout and written at its traversal position into the other
// buffer.  The current goes through the warp's segment-slot run reduction
// (deposit_runs).  newcell (-1 = erased, place(), plist.cpp:7-39) and the
// particles-per-new-cell histogram (count) feed the rebin.
template <int PUSHER, int KIND, int BS, int MINB, bool PF>
__global__ void __launch_bounds__(BS, MINB) k_push64(Fields<double> f, Grid g, PStore64 src, PStore64 dst,
                                                   const int32_t* __restrict__ perm, int32_t* __restrict__ newcell,
                                                   int32_t* __restrict__ count, PushArgs a) {
    // the grid (a few waves) strides over the particles in block-sized
    // chunks; the diagnostics are summed per thread over its chunks and
    // block-reduced once.  Against one thread per particle this measured
    // 10 % (FP64) and 17 % (mixed) faster.
    double dq = 0.0, de = 0.0, er = 0.0;
    unsigned long long dc = 0;
    const ChunkRange cr = chunk_range(a.n, a.resident);
    // software pipeline over the thread's chunks: the slot and position of
    // the next chunk's particle are loaded during this chunk, so that the
    // loads of a particle's momenta and of its fields issue together
    int p_nx = 0;
    double x_nx = 0.0, y_nx = 0.0, z_nx = 0.0;
    if (PF) {
        const int s0 = cr.first * blockDim.x + threadIdx.x;
        if (cr.first < cr.end && s0 < a.n) {
            p_nx = perm[s0];
            x_nx = src.x[p_nx]; y_nx = src.y[p_nx]; z_nx = src.z[p_nx];
        }
    }
    for (int ch = cr.first; ch < cr.end; ch += cr.step) {
    const int s = ch * blockDim.x + threadIdx.x;
    const int s_nx = (ch + cr.step) * blockDim.x + threadIdx.x;
    const bool has_nx = PF && ch + cr.step < cr.end && s_nx < a.n;
    int nc = -1, p = p_nx, i0 = 0, j0 = 0, k0 = 0;
    bool nc_owned = true;
    bool live = false, active = false;
    double pos[3] = {x_nx, y_nx, z_nx}, d[3] = {0.0, 0.0, 0.0};
    double ux = 0.0, uy = 0.0, uz = 0.0, gm = 1.0, q = 0.0;
    if (!PF && s < a.n) {
        p = perm[s];
        pos[0] = src.x[p]; pos[1] = src.y[p]; pos[2] = src.z[p];
    }
    if (has_nx) p_nx = perm[s_nx];
    if (s < a.n) {
        ux = src.ux[p]; uy = src.uy[p]; uz = src.uz[p]; gm = src.g[p];
        q = src.q[p];
        i0 = (int)pos[0]; j0 = (int)pos[1]; k0 = (int)pos[2];
        live = !kill_layer(g, i0, j0, k0);  // p_boundary, plist.cpp:73-102
        if (live) {
            double E[3], B[3];
            gather(f, g, i0, j0, k0, pos[0] - i0, pos[1] - j0, pos[2] - k0, E, B);
            B[2] += a.ext_bz;
            if (KIND != KIND_PHOTON) push<PUSHER>(a.cmr, ux, uy, uz, gm, E, B, a.dt);
            // particle::get_displacement (containers.cpp:58-67), then per-axis
            // division by the cell size (advance.cpp:281-284)
            const double t = a.dt / gm;
            d[0] = ux * t; d[1] = uy * t; d[2] = uz * t;
            d[0] = div_fixed(d[0], a.dx, a.rdx);
            d[1] = div_fixed(d[1], a.dy, a.rdy);
            d[2] = div_fixed(d[2], a.dz, a.rdz);
            if (KIND == KIND_PHOTON) {
                pos[0] = pos[0] + d[0]; pos[1] = pos[1] + d[1]; pos[2] = pos[2] + d[2];
            } else {
                active = true;
            }
            if (!isfinite(gm)) atomicOr(a.status, (unsigned int)ST_NAN);
        }
    }
    if (has_nx) {
        x_nx = src.x[p_nx]; y_nx = src.y[p_nx]; z_nx = src.z[p_nx];
    }
    deposit_runs(f, g, pos, d, q, 0, 0, 0, active, a.status);
    if (s < a.n) {
        if (live) {
            const int i1 = (int)pos[0], j1 = (int)pos[1], k1 = (int)pos[2];
            const bool moved = (i1 != i0) || (j1 != j0) || (k1 != k0);
            if (!moved || inside(g, i1, j1, k1)) nc = cidx(g, i1, j1, k1);
        }
        newcell[s] = nc;
        // an erasure in the exchange area of an x-slab is not one of the whole box (delete_particle,
        // low-level.cpp:247-259): only erasures inside [dlo, dhi) are caught and counted
        if (nc < 0 && !((int)pos[0] >= a.dlo && (int)pos[0] < a.dhi)) nc_owned = false;
        if (nc < 0 && a.cat && nc_owned)
            catch_particle(*a.cat, a.sp, a.step, live ? 1 : 0, s, pos[0], pos[1], pos[2], ux, uy, uz, gm, q,
                           src.chi ? src.chi[p] : 0.0);
        if (nc >= 0) {
            dst.x[s] = pos[0]; dst.y[s] = pos[1]; dst.z[s] = pos[2];
            dst.ux[s] = ux; dst.uy[s] = uy; dst.uz[s] = uz;
            dst.g[s] = gm; dst.q[s] = q;
            if (dst.chi) dst.chi[s] = src.chi[p];
            if (a.trn_dst) a.trn_dst[s] = a.trn_src[p];
            const int ii = (int)pos[0];
            if (ii >= a.dlo && ii < a.dhi) {
                dq += q;
                de += KIND == KIND_PHOTON ? gm * q : (gm - 1) * q;
                dc += 1;
            }
        }
        // energy of the particles erased in this push
        if (a.track && nc < 0 && nc_owned) er += KIND == KIND_PHOTON ? gm * q : (gm - 1) * q;
    }
    warp_count_runs(count, nc);
    }
    block_diag(a.diag, a.sp, dq, de, dc);
    if (a.track) block_sum(&a.diag->sum_erased[a.sp], er);  // (uniform)
}

// Particle born during a push: appended to the target species' output
// buffer with its final cell, erased (not stored) if the cell is not inside
// (place(p), plist.cpp:22-39).  Counted in the target's diagnostics.
__device__ __forceinline__ void append64(const AppendTarget<PStore64>& t, const Grid& g, int dlo, int dhi,
                                         const double pos[3],
                                         const double u[3], double gm, double q, double chi, bool photon,
                                         unsigned int* status, DiagAccum* diag) {
    const int i = (int)pos[0], j = (int)pos[1], k = (int)pos[2];
    if (!(pos[0] >= 0.0 && pos[1] >= 0.0 && pos[2] >= 0.0) || !inside(g, i, j, k)) return;
    const int slot = t.base + atomicAdd(t.counter, 1);
    if (slot >= t.cap) {
        atomicOr(status, (unsigned int)ST_CAPACITY);
        return;
    }
    t.dst.x[slot] = pos[0]; t.dst.y[slot] = pos[1]; t.dst.z[slot] = pos[2];
    t.dst.ux[slot] = u[0]; t.dst.uy[slot] = u[1]; t.dst.uz[slot] = u[2];
    t.dst.g[slot] = gm; t.dst.q[slot] = q;
    if (t.dst.chi) t.dst.chi[slot] = chi;
    t.newcell[slot] = cidx(g, i, j, k);
    if (i < dlo || i >= dhi) return;
    atomicAdd(&diag->sum_q[t.sp], q);
    atomicAdd(&diag->sum_e[t.sp], photon ? gm * q : (gm - 1) * q);
    atomicAdd(&diag->cnt[t.sp], 1ull);
}

// bear_particle (mc.cpp:118-139): momentum along `dir` with gamma g.
__device__ __forceinline__ void bear_u(const double dir[3], double gm, bool photon, double u[3]) {
    const double d2 = dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2];
    const double a = photon ? gm / sqrt(d2) : sqrt((gm * gm - 1) / d2);
    u[0] = a * dir[0]; u[1] = a * dir[1]; u[2] = a * dir[2];
}

// A lepton born from a photon: pushed from t_n, chi at t_{n+1/2}, moved with
// current deposition (advance.cpp:172-236), then appended.
template <int PUSHER>
__device__ __forceinline__ void born_lepton64(const Fields<double>& f, const Grid& g, const PushArgs& a,
                                              const QedArgs& qa, const double pos0[3], const double dir[3],
                                              double gm, double chi, double q, double cmr, const double E[3],
                                              const double B[3], const AppendTarget<PStore64>& t) {
    double u[3];
    bear_u(dir, gm, false, u);
    const double up[3] = {u[0], u[1], u[2]};
    const double gp = gm;
    push<PUSHER>(cmr, u[0], u[1], u[2], gm, E, B, a.dt);
    const double ui[3] = {0.5 * (u[0] + up[0]), 0.5 * (u[1] + up[1]), 0.5 * (u[2] + up[2])};
    const double gi = 0.5 * (gm + gp);
    chi = qed_chi(E, B, ui, gi, qa.e_s);
    const double tt = a.dt / gm;
    double d[3] = {u[0] * tt, u[1] * tt, u[2] * tt};
    d[0] = d[0] / a.dx; d[1] = d[1] / a.dy; d[2] = d[2] / a.dz;
    double pos[3] = {pos0[0], pos0[1], pos0[2]};
    jdeposition(f, g, pos, d, q, 0, 0, 0, a.status);
    append64(t, g, a.dlo, a.dhi, pos, u, gm, q, chi, false, a.status, a.diag);
}

// advance.cpp:90-387 with QED on.  Photons: chi, pair creation with
// probability tilde_w g dt (pairs pushed and deposited here, the photon is
// erased), else straight flight.  Leptons: push, chi at t_{n+1/2}, photon
// emission with probability w g dt (photon placed with the reference's time
// shifts, lepton recoils by (1 - r), is re-gathered, re-pushed and deposits).
// Random numbers: Philox4x32-10 keyed by the seed, counter (traversal
// position, species, tag, step) -> (r, acceptance draw).
// t0: photons (lepton kernel) or electrons (photon kernel); t1: positrons.
template <int PUSHER, int KIND>
__global__ void __launch_bounds__(256, 2) k_push64_qed(Fields<double> f, Grid g, PStore64 src, PStore64 dst,
                                                    const int32_t* __restrict__ perm,
                                                    int32_t* __restrict__ newcell, PushArgs a, QedArgs qa,
                                                    AppendTarget<PStore64> t0, AppendTarget<PStore64> t1) {
    double dq = 0.0, de = 0.0;
    unsigned long long dc = 0;
    // block-sized chunks with the grid striding over them, diagnostics
    // reduced once per block (as in the pushes without QED)
    const ChunkRange cr = chunk_range(a.n, a.resident);
    // the next chunk's slot loaded a chunk ahead, its position once the
    // slot has arrived (as in k_push64)
    int p_nx = 0;
    {
        const int s0 = cr.first * blockDim.x + threadIdx.x;
        if (cr.first < cr.end && s0 < a.n) p_nx = perm[s0];
    }
    for (int ch = cr.first; ch < cr.end; ch += cr.step) {
    const int s = ch * blockDim.x + threadIdx.x;
    const int s_nx = (ch + cr.step) * blockDim.x + threadIdx.x;
    const int p = p_nx;
    if (ch + cr.step < cr.end && s_nx < a.n) p_nx = perm[s_nx];
    // the lepton's own move without emission (the common case) deposits its
    // current after the branches, through the warp's run sums (deposit_runs:
    // every lane of the warp takes part); the rare moves after an emission
    // deposit directly
    double pos[3] = {0.0, 0.0, 0.0}, dmove[3] = {0.0, 0.0, 0.0};
    double ux = 0.0, uy = 0.0, uz = 0.0, gm = 1.0, q = 0.0, chi = 0.0;
    int i0 = 0, j0 = 0, k0 = 0, nc = -1;
    bool converted = false;  // a photon that became a pair is not an erasure
    bool deferred = false;   // the move's current and cell wait for deposit_runs
    if (s < a.n) {
        pos[0] = src.x[p]; pos[1] = src.y[p]; pos[2] = src.z[p];
        ux = src.ux[p]; uy = src.uy[p]; uz = src.uz[p]; gm = src.g[p];
        q = src.q[p];
        chi = src.chi[p];
        i0 = (int)pos[0]; j0 = (int)pos[1]; k0 = (int)pos[2];
        if (!kill_layer(g, i0, j0, k0)) {
            double E[3], B[3];
            gather(f, g, i0, j0, k0, pos[0] - i0, pos[1] - j0, pos[2] - k0, E, B);
            B[2] += a.ext_bz;
            double r, r2;
            uniform2(philox4x32_10((uint32_t)s, (uint32_t)a.sp, RNG_PUSH, qa.step, qa.key0, qa.key1), r, r2);
            if (KIND == KIND_PHOTON) {
                const double ui[3] = {ux, uy, uz};
                const double g_prev = gm, chi_prev = chi;
                chi = qed_chi(E, B, ui, gm, qa.e_s);
                const double am = 0.5 * (chi + chi_prev);
                const bool pair = !(r2 >= qed_tilde_w(g_prev, r, am, qa.e_s) * g_prev * a.dt);
                if (!pair) {
                    const double t = a.dt / gm;
                    double d[3] = {ux * t, uy * t, uz * t};
                    d[0] = d[0] / a.dx; d[1] = d[1] / a.dy; d[2] = d[2] / a.dz;
                    pos[0] = pos[0] + d[0]; pos[1] = pos[1] + d[1]; pos[2] = pos[2] + d[2];
                    const int i1 = (int)pos[0], j1 = (int)pos[1], k1 = (int)pos[2];
                    const bool moved = (i1 != i0) || (j1 != j0) || (k1 != k0);
                    if (!moved || inside(g, i1, j1, k1)) nc = cidx(g, i1, j1, k1);
                } else {
                    converted = true;
                    // electron with r of the photon energy, positron with 1 - r
                    born_lepton64<PUSHER>(f, g, a, qa, pos, ui, r * g_prev, r * chi, -q, -1.0, E, B, t0);
                    born_lepton64<PUSHER>(f, g, a, qa, pos, ui, (1 - r) * gm, (1 - r) * chi, q, 1.0, E, B, t1);
                }
            } else {
                const double up[3] = {ux, uy, uz};
                const double g_prev = gm, chi_prev = chi;
                push<PUSHER>(a.cmr, ux, uy, uz, gm, E, B, a.dt);
                const double ui[3] = {0.5 * (ux + up[0]), 0.5 * (uy + up[1]), 0.5 * (uz + up[2])};
                const double gi = 0.5 * (gm + g_prev);
                chi = qed_chi(E, B, ui, gi, qa.e_s);
                const double am = 0.5 * (chi + chi_prev);
                const bool emit = !(r2 >= qed_w(g_prev, r, am, qa.e_s) * g_prev * a.dt);
                if (!emit) {
                    const double t = a.dt / gm;
                    dmove[0] = ux * t; dmove[1] = uy * t; dmove[2] = uz * t;
                    dmove[0] = dmove[0] / a.dx; dmove[1] = dmove[1] / a.dy; dmove[2] = dmove[2] / a.dz;
                    deferred = true;
                } else {
                    // photon born at the lepton's t_n position, then moved
                    // to t_{n+3/2} (advance.cpp:294-306)
                    double am2 = 0.5 * a.dt / g_prev;
                    double ph[3] = {pos[0] - am2 * up[0] / a.dx, pos[1] - am2 * up[1] / a.dy,
                                    pos[2] - am2 * up[2] / a.dz};
                    const double gph = r * g_prev;
                    double uph[3];
                    bear_u(up, gph, true, uph);
                    const double a3 = 3 * am2 * g_prev / gph;
                    ph[0] += a3 * uph[0] / a.dx;
                    ph[1] += a3 * uph[1] / a.dy;
                    ph[2] += a3 * uph[2] / a.dz;
                    if (a.dcat) {
                        // dump_photons: the photon is deleted as it is born (advance.cpp:302-306),
                        // recorded with its energy unless it sits in an exchange area
                        const int pi = (int)ph[0];
                        if (pi >= a.dlo && pi < a.dhi) {
                            catch_particle(*a.dcat, t0.sp, a.step, 2, s, ph[0], ph[1], ph[2], uph[0], uph[1], uph[2],
                                           gph, fabs(q), r * chi);
                            atomicAdd(&a.diag->sum_erased[t0.sp], gph * fabs(q));
                        }
                    } else {
                        append64(t0, g, a.dlo, a.dhi, ph, uph, gph, fabs(q), r * chi, true, a.status, a.diag);
                    }
                    // recoil (advance.cpp:308-322)
                    chi = (1 - r) * chi;
                    gm = (1 - r) * g_prev;
                    const double sc = sqrt((gm * gm - 1) / (up[0] * up[0] + up[1] * up[1] + up[2] * up[2]));
                    ux = up[0] * sc; uy = up[1] * sc; uz = up[2] * sc;
                    pos[0] -= am2 * up[0] / a.dx;
                    pos[1] -= am2 * up[1] / a.dy;
                    pos[2] -= am2 * up[2] / a.dz;
                    am2 = am2 * g_prev / gm;
                    pos[0] += am2 * ux / a.dx;
                    pos[1] += am2 * uy / a.dy;
                    pos[2] += am2 * uz / a.dz;
                    const int i1 = (int)pos[0], j1 = (int)pos[1], k1 = (int)pos[2];
                    if (pos[0] >= 0.0 && pos[1] >= 0.0 && pos[2] >= 0.0 && inside(g, i1, j1, k1)) {
                        gather(f, g, i1, j1, k1, pos[0] - i1, pos[1] - j1, pos[2] - k1, E, B);
                        B[2] += a.ext_bz;
                        push<PUSHER>(a.cmr, ux, uy, uz, gm, E, B, a.dt);
                        const double t = a.dt / gm;
                        double d[3] = {ux * t, uy * t, uz * t};
                        d[0] = d[0] / a.dx; d[1] = d[1] / a.dy; d[2] = d[2] / a.dz;
                        jdeposition(f, g, pos, d, q, 0, 0, 0, a.status);
                        const int i2 = (int)pos[0], j2 = (int)pos[1], k2 = (int)pos[2];
                        const bool moved = (i2 != i1) || (j2 != j1) || (k2 != k1);
                        if (!moved || inside(g, i2, j2, k2)) nc = cidx(g, i2, j2, k2);
                    }
                }
            }
            if (!isfinite(gm)) atomicOr(a.status, (unsigned int)ST_NAN);
        }
    }
    if (KIND != KIND_PHOTON) deposit_runs(f, g, pos, dmove, q, 0, 0, 0, deferred, a.status);
    if (s < a.n) {
        if (deferred) {
            const int i1 = (int)pos[0], j1 = (int)pos[1], k1 = (int)pos[2];
            const bool moved = (i1 != i0) || (j1 != j0) || (k1 != k0);
            if (!moved || inside(g, i1, j1, k1)) nc = cidx(g, i1, j1, k1);
        }
        newcell[s] = nc;
        const bool erased = nc < 0 && !converted && (int)pos[0] >= a.dlo && (int)pos[0] < a.dhi;
        if (erased && a.cat)
            catch_particle(*a.cat, a.sp, a.step, kill_layer(g, i0, j0, k0) ? 0 : 1, s, pos[0], pos[1], pos[2], ux, uy,
                           uz, gm, q, chi);
        if (erased && a.track)  // erasures are few: one atomic each
            atomicAdd(&a.diag->sum_erased[a.sp], KIND == KIND_PHOTON ? gm * q : (gm - 1) * q);
        if (nc >= 0) {
            dst.x[s] = pos[0]; dst.y[s] = pos[1]; dst.z[s] = pos[2];
            dst.ux[s] = ux; dst.uy[s] = uy; dst.uz[s] = uz;
            dst.g[s] = gm; dst.q[s] = q; dst.chi[s] = chi;
            if (a.trn_dst) a.trn_dst[s] = a.trn_src[p];
            const int ii = (int)pos[0];
            if (ii >= a.dlo && ii < a.dhi) {
                dq += q;
                de += KIND == KIND_PHOTON ? gm * q : (gm - 1) * q;
                dc += 1;
            }
        }
    }
    }
    block_diag(a.diag, a.sp, dq, de, dc);
}

// birth_from_vacuum (mc.cpp:142-196): per cell of [2, n-2)^3, fields at the
// cell centre, pair with probability W dt dx dy dz; the pair starts at rest
// and is pushed back by half a step.  Pairs go to the free slots of the
// current buffers of the electron (t0) and positron (t1) stores; the host
// then merges them at the head of their cells.
template <int PUSHER>
__global__ void __launch_bounds__(256) k_vacuum64(Fields<double> f, Grid g, QedArgs qa, double dt, double dV,
                                                  double qv, AppendTarget<PStore64> t0,
                                                  AppendTarget<PStore64> t1, unsigned int* status) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nc) return;
    const int k = c % g.nz, j = (c / g.nz) % g.ny, i = c / g.nynz;
    if (i < 2 || i >= g.nx - 2 || j < 2 || j >= g.ny - 2 || k < 2 || k >= g.nz - 2) return;
    double E[3], B[3];
    gather(f, g, i, j, k, 0.5, 0.5, 0.5, E, B);
    double r, r2;
    uniform2(philox4x32_10((uint32_t)c, 0u, RNG_VACUUM, qa.step, qa.key0, qa.key1), r, r2);
    if (!(r < qed_vacuum_W(E, B, qa.e_s) * dt * dV)) return;
    const double pos[3] = {i + 0.5, j + 0.5, k + 0.5};
    for (int e = 0; e < 2; e++) {
        const AppendTarget<PStore64>& t = e == 0 ? t0 : t1;
        double ux = 0, uy = 0, uz = 0, gm = 1;
        push<PUSHER>(e == 0 ? -1.0 : 1.0, ux, uy, uz, gm, E, B, -0.5 * dt);
        const int slot = t.base + atomicAdd(t.counter, 1);
        if (slot >= t.cap) {
            atomicOr(status, (unsigned int)ST_CAPACITY);
            continue;
        }
        t.dst.x[slot] = pos[0]; t.dst.y[slot] = pos[1]; t.dst.z[slot] = pos[2];
        t.dst.ux[slot] = ux; t.dst.uy[slot] = uy; t.dst.uz[slot] = uz;
        t.dst.g[slot] = gm; t.dst.q[slot] = e == 0 ? -qv : qv;
        t.dst.chi[slot] = 0.0;
        t.newcell[slot] = c;
    }
}

// Element-wise evaluation of the QED rate functions on the device.
// in: 12 doubles per sample (e[3] b[3] u[3] g r chi); out: 5 per sample
// (chi(e,b,u,g), w(g, r, chi), r after w, tilde_w(g, r, chi), vacuum W(e,b)).
__global__ void k_qed_rates(int n, const double* __restrict__ in, double* __restrict__ out, double e_s) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double* v = in + 12 * (size_t)t;
    const double e[3] = {v[0], v[1], v[2]}, b[3] = {v[3], v[4], v[5]}, u[3] = {v[6], v[7], v[8]};
    double r = v[10];
    double* o = out + 5 * (size_t)t;
    o[0] = qed_chi(e, b, u, v[9], e_s);
    o[1] = qed_w(v[9], r, v[11], e_s);
    o[2] = r;
    o[3] = qed_tilde_w(v[9], v[10], v[11], e_s);
    o[4] = qed_vacuum_W(e, b, e_s);
}

cudaError_t launch_qed_rates(int n, const double* d_in, double* d_out, double e_s, cudaStream_t st) {
    if (n > 0) k_qed_rates<<<(n + 255) / 256, 256, 0, st>>>(n, d_in, d_out, e_s);
    return cudaGetLastError();
}


SolverCoef solver_coef(const qp_params& p);

void launch_fields_fp64(State& s, int phase) {
    Fields<double> f = fields_of<double>(s);
    Coef<double> c(solver_coef(s.prm));
    dim3 blk(32, 8, 1);
    dim3 grd((s.grid.nz + 31) / 32, (s.grid.ny + 7) / 8, s.grid.nx);
    const int sol = s.prm.solver;
#define QP_LF(SOL, PH) k_field<double, SOL, PH><<<grd, blk, 0, s.stream>>>(f, s.grid, c, s.d_diag, s.diag_lo, s.diag_hi)
    if (phase == 4) {
        if (sol == QP_SOLVER_FDTD) QP_LF(QP_SOLVER_FDTD, 4);
        else if (sol == QP_SOLVER_NDFX) QP_LF(QP_SOLVER_NDFX, 4);
        else QP_LF(QP_SOLVER_FIVE_POINT, 4);
    } else if (phase == 0 || phase == 2) {
        if (sol == QP_SOLVER_FDTD) QP_LF(QP_SOLVER_FDTD, 0);
        else if (sol == QP_SOLVER_NDFX) QP_LF(QP_SOLVER_NDFX, 0);
        else QP_LF(QP_SOLVER_FIVE_POINT, 0);
    } else if (phase == 1) {
        if (sol == QP_SOLVER_FDTD) QP_LF(QP_SOLVER_FDTD, 1);
        else if (sol == QP_SOLVER_NDFX) QP_LF(QP_SOLVER_NDFX, 1);
        else QP_LF(QP_SOLVER_FIVE_POINT, 1);
    } else {
        QP_LF(QP_SOLVER_FDTD, 3);
    }
#undef QP_LF
    s.launches++;
}

void zero_planes_fp64(State& s, const ZeroPlane* zp, int n) {
    Fields<double> f = fields_of<double>(s);
    for (int a = 0; a < n; a++) {
        int nu = zp[a].axis == 2 ? s.grid.ny : s.grid.nz;
        int nv = zp[a].axis == 0 ? s.grid.ny : s.grid.nx;
        dim3 grd((nu + 127) / 128, nv);
        k_zero_plane<double><<<grd, 128, 0, s.stream>>>(f, s.grid, zp[a].axis, zp[a].plane, zp[a].comps);
        s.launches++;
    }
}

static PStore64 store64(Species& sp, int b) {
    PStore64 st;
    double** ps[9] = {&st.x, &st.y, &st.z, &st.ux, &st.uy, &st.uz, &st.g, &st.q, &st.chi};
    for (int a = 0; a < 9; a++) *ps[a] = (double*)sp.buf[b][a];
    return st;
}

static AppendTarget<PStore64> target64(State& s, int si, bool output) {
    Species& sp = s.sp[si];
    AppendTarget<PStore64> t;
    t.dst = store64(sp, output ? 1 - sp.cur : sp.cur);
    t.newcell = sp.newcell;
    t.counter = sp.d_counter;
    t.base = (int)(output ? sp.n : sp.slots);
    t.cap = (int)sp.cap;
    t.sp = si;
    return t;
}

static QedArgs qed_args(State& s) {
    QedArgs q;
    q.e_s = s.prm.lambda_cm / 2.4263086e-10;  // main.cpp:2276
    q.key0 = (uint32_t)(s.prm.seed & 0xffffffffu);
    q.key1 = (uint32_t)(s.prm.seed >> 32);
    q.step = (uint32_t)s.step_index;
    return q;
}

int launch_push_fp64_qed(State& s, int si, double external_bz) {
    Species& sp = s.sp[si];
    if (sp.n == 0) return QP_OK;
    if (sp.kind == KIND_ION) {
        launch_push_fp64(s, si, external_bz);
        return QP_OK;
    }
    PStore64 src = store64(sp, sp.cur), dst = store64(sp, 1 - sp.cur);
    PushArgs a{};
    a.cmr = sp.cmr; a.dt = s.prm.dt; a.dx = s.prm.dx; a.dy = s.prm.dy; a.dz = s.prm.dz;
    a.ext_bz = external_bz; a.n = (int)sp.n; a.sp = si; a.kind = sp.kind;
    a.status = s.d_status; a.diag = s.d_diag;
    a.track = s.track_erased ? 1 : 0;
    a.step = (uint32_t)s.step_index;
    a.cat = s.catch_erasures ? s.d_cat : nullptr;
    a.dcat = s.dump_photons ? s.d_cat : nullptr;
    a.trn_src = sp.trn[sp.cur];
    a.trn_dst = sp.trn[1 - sp.cur];
    a.dlo = s.diag_lo; a.dhi = s.diag_hi;
    QedArgs qa = qed_args(s);
    AppendTarget<PStore64> t0, t1;
    if (sp.kind == KIND_PHOTON) {
        t0 = target64(s, s.sp_e, true);
        t1 = target64(s, s.sp_p, true);
    } else {
        t0 = target64(s, s.sp_ph, true);
        t1 = t0;
    }
    const int nb = push_blocks(s, sp.n, PushShape{256, 2}, s.push_waves_qed, &a.resident);  // chunked grid (2 resident blocks per SM assumed)
    Fields<double> f = fields_of<double>(s);
    const bool vay = s.prm.pusher == QP_PUSHER_VAY;
#define QP_LQ(P, K) k_push64_qed<P, K><<<nb, 256, 0, s.stream>>>(f, s.grid, src, dst, sp.perm, sp.newcell, a, qa, t0, t1)
    if (sp.kind == KIND_PHOTON) {
        if (vay) QP_LQ(QP_PUSHER_VAY, KIND_PHOTON);
        else QP_LQ(QP_PUSHER_BORIS, KIND_PHOTON);
    } else {
        if (vay) QP_LQ(QP_PUSHER_VAY, KIND_LEPTON);
        else QP_LQ(QP_PUSHER_BORIS, KIND_LEPTON);
    }
#undef QP_LQ
    s.launches++;
    return QP_OK;
}

int launch_vacuum_fp64(State& s) {
    const double PI = 3.141592653589793;
    const qp_params& p = s.prm;
    const double dV = p.dx * p.dy * p.dz;
    const double qv = 8 * PI * PI / dV * 2.818e-13 / p.lambda_cm;  // main.cpp:2324
    QedArgs qa = qed_args(s);
    AppendTarget<PStore64> t0 = target64(s, s.sp_e, false), t1 = target64(s, s.sp_p, false);
    Fields<double> f = fields_of<double>(s);
    const int nb = (s.grid.nc + 255) / 256;
    if (p.pusher == QP_PUSHER_VAY)
        k_vacuum64<QP_PUSHER_VAY><<<nb, 256, 0, s.stream>>>(f, s.grid, qa, p.dt, dV, qv, t0, t1, s.d_status);
    else
        k_vacuum64<QP_PUSHER_BORIS><<<nb, 256, 0, s.stream>>>(f, s.grid, qa, p.dt, dV, qv, t0, t1, s.d_status);
    s.launches++;
    return QP_OK;
}

// Push of one species; also leaves the particles-per-new-cell histogram in
// sp.count (zeroed here), so the rebin skips its counting pass.
void launch_push_fp64(State& s, int si, double external_bz) {
    Species& sp = s.sp[si];
    cudaMemsetAsync(sp.count, 0, (size_t)s.grid.nc * sizeof(int32_t), s.stream);
    if (sp.n == 0) return;
    PStore64 src = store64(sp, sp.cur), dst = store64(sp, 1 - sp.cur);
    PushArgs a{};
    a.cmr = sp.cmr; a.dt = s.prm.dt; a.dx = s.prm.dx; a.dy = s.prm.dy; a.dz = s.prm.dz;
    a.rdx = 1.0 / s.prm.dx; a.rdy = 1.0 / s.prm.dy; a.rdz = 1.0 / s.prm.dz;
    a.ext_bz = external_bz; a.n = (int)sp.n; a.sp = si; a.kind = sp.kind;
    a.status = s.d_status; a.diag = s.d_diag;
    a.track = s.track_erased ? 1 : 0;
    a.step = (uint32_t)s.step_index;
    a.cat = s.catch_erasures ? s.d_cat : nullptr;
    a.dcat = s.dump_photons ? s.d_cat : nullptr;
    a.trn_src = sp.trn[sp.cur];
    a.trn_dst = sp.trn[1 - sp.cur];
    a.dlo = s.diag_lo; a.dhi = s.diag_hi;
    const PushShape sh = push_shapes64[s.push_shape];
    const int nb = push_blocks(s, sp.n, sh, s.push_waves, &a.resident);
    Fields<double> f = fields_of<double>(s);
    const bool vay = s.prm.pusher == QP_PUSHER_VAY;
#define QP_LS(P, K, BS, MB) \
    do { if (s.prefetch) k_push64<P, K, BS, MB, true><<<nb, BS, 0, s.stream>>>(f, s.grid, src, dst, sp.perm, sp.newcell, sp.count, a); \
         else k_push64<P, K, BS, MB, false><<<nb, BS, 0, s.stream>>>(f, s.grid, src, dst, sp.perm, sp.newcell, sp.count, a); } while (0)
#define QP_LP(P, K)                              \
    do { switch (s.push_shape) {                 \
        case 1: QP_LS(P, K, 256, 3); break;      \
        case 2: QP_LS(P, K, 192, 3); break;      \
        case 3: QP_LS(P, K, 128, 5); break;      \
        case 4: QP_LS(P, K, 128, 4); break;      \
        case 5: QP_LS(P, K, 64, 8); break;       \
        default: QP_LS(P, K, 256, 2); break;     \
    } } while (0)
    if (sp.kind == KIND_PHOTON) QP_LP(QP_PUSHER_BORIS, KIND_PHOTON);
    else if (vay) QP_LP(QP_PUSHER_VAY, KIND_LEPTON);
    else QP_LP(QP_PUSHER_BORIS, KIND_LEPTON);
#undef QP_LP
#undef QP_LS
    s.launches++;
}


}  // namespace qp
