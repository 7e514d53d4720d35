// Mixed-precision path: positions as a linear cell index plus an FP32 offset
// in [0, 1), FP32 push, gather, current deposition and Maxwell stencils.
// Diagnostics are accumulated in FP64.  The algorithms are the reference's;
// the deposition runs in the particle's cell frame (offsets), which is the
// reference's absolute-coordinate algorithm shifted by an integer.
#include "qp_kernels.cuh"
#include "qp_qed.cuh"

namespace qp {

struct PushArgs32 {
    float cmr, dt, idx, idy, idz, ext_bz;
    int n, sp, kind;
    int track;  // sum the energy of erased particles into diag->sum_erased
    unsigned int* status;
    DiagAccum* diag;
    uint32_t step;
    const CatchBuf* cat;  // device copy; nullptr: erasures are not recorded
    const CatchBuf* dcat;  // dump_photons: emitted photons recorded here instead of kept; nullptr: kept
    const int32_t* trn_src;  // track numbers in, by slot / out, by traversal position; nullptr: off
    int32_t* trn_dst;
    int dlo, dhi;  // the diagnostics count particles whose new cell has i in [dlo, dhi)
    int resident;  // blocks per group of the chunk order (chunk_range)
};

__device__ __forceinline__ float wrap_offset(float o, int& shift) {
    const float fl = floorf(o);
    shift = (int)fl;
    float r = o - fl;
    // keep the offset in [0, 1) after rounding
    if (r >= 1.0f) r = 0.99999994f;
    if (r < 0.0f) r = 0.0f;
    return r;
}

// The particles in traversal order as k_push64 takes them (a grid of a few
// waves striding over block-sized chunks, diagnostics reduced once).  The
// move runs in the particle's cell frame (offsets in [0, 1)), the current
// through the warp's segment-slot run reduction (deposit_runs).
template <int PUSHER, int KIND, int BS, int MINB, bool PF>
__global__ void __launch_bounds__(BS, MINB) k_push32(Fields<float> f, Grid g, PStore32 src, PStore32 dst,
                                                   const int32_t* __restrict__ perm, int32_t* __restrict__ newcell,
                                                   int32_t* __restrict__ count, PushArgs32 a) {
    double dq = 0.0, de = 0.0, er = 0.0;
    unsigned long long dc = 0;
    const ChunkRange cr = chunk_range(a.n, a.resident);
    // software pipeline over the thread's chunks: the slot and cell of the
    // next chunk's particle are loaded during this chunk, so that the loads
    // of a particle's state and of its fields issue together at the top
    int p_nx = 0, c_nx = 0;
    if (PF) {
        const int s0 = cr.first * blockDim.x + threadIdx.x;
        if (cr.first < cr.end && s0 < a.n) {
            p_nx = perm[s0];
            c_nx = src.cell[p_nx];
        }
    }
    for (int ch = cr.first; ch < cr.end; ch += cr.step) {
        const int s = ch * blockDim.x + threadIdx.x;
        const int s_nx = (ch + cr.step) * blockDim.x + threadIdx.x;
        const bool has_nx = PF && ch + cr.step < cr.end && s_nx < a.n;
        int nc = -1, p = p_nx, i0 = 0, j0 = 0, k0 = 0;
        int c0 = c_nx;
        if (!PF && s < a.n) {
            p = perm[s];
            c0 = src.cell[p];
        }
        if (has_nx) p_nx = perm[s_nx];
        bool nc_owned = true;
        bool live = false, active = false;
        float o[3] = {0.f, 0.f, 0.f}, d[3] = {0.f, 0.f, 0.f};
        float ux = 0.f, uy = 0.f, uz = 0.f, gm = 1.f, q = 0.f;
        if (s < a.n) {
            i0 = g.div_nynz.div(c0);
            const int r0 = c0 - i0 * g.nynz;
            j0 = g.div_nz.div(r0);
            k0 = r0 - j0 * g.nz;
            o[0] = src.ox[p]; o[1] = src.oy[p]; o[2] = src.oz[p];
            ux = src.ux[p]; uy = src.uy[p]; uz = src.uz[p]; gm = src.g[p];
            q = src.q[p];
            live = !kill_layer(g, i0, j0, k0);
            if (live) {
                float E[3], B[3];
                gather(f, g, i0, j0, k0, o[0], o[1], o[2], E, B);
                B[2] += a.ext_bz;
                if (KIND != KIND_PHOTON) push<PUSHER>(a.cmr, ux, uy, uz, gm, E, B, a.dt);
                const float t = a.dt / gm;
                d[0] = ux * t * a.idx; d[1] = uy * t * a.idy; d[2] = uz * t * a.idz;
                if (KIND == KIND_PHOTON) {
                    o[0] += d[0]; o[1] += d[1]; o[2] += d[2];
                } else {
                    active = true;
                }
                if (!isfinite(gm)) atomicOr(a.status, (unsigned int)ST_NAN);
            }
        }
        if (has_nx) c_nx = src.cell[p_nx];
        deposit_runs(f, g, o, d, q, i0, j0, k0, active, a.status);
        if (s < a.n) {
            int i1 = i0, j1 = j0, k1 = k0;
            if (live) {
                int si, sj, sk;
                o[0] = wrap_offset(o[0], si);
                o[1] = wrap_offset(o[1], sj);
                o[2] = wrap_offset(o[2], sk);
                i1 = i0 + si; j1 = j0 + sj; k1 = k0 + sk;
                const bool moved = si | sj | sk;
                if (!moved || inside(g, i1, j1, k1)) nc = cidx(g, i1, j1, k1);
            }
            newcell[s] = nc;
            // an erasure in the exchange area of an x-slab is not one of the whole box (delete_particle,
            // low-level.cpp:247-259): only erasures inside [dlo, dhi) are caught and counted
            if (nc < 0 && !(i1 >= a.dlo && i1 < a.dhi)) nc_owned = false;
            if (nc < 0 && a.cat && nc_owned)
                catch_particle(*a.cat, a.sp, a.step, live ? 1 : 0, s, (double)i1 + (double)o[0], (double)j1 + (double)o[1],
                               (double)k1 + (double)o[2], ux, uy, uz, gm, q, src.chi ? (double)src.chi[p] : 0.0);
            if (nc >= 0) {
                dst.cell[s] = nc;
                dst.ox[s] = o[0]; dst.oy[s] = o[1]; dst.oz[s] = o[2];
                dst.ux[s] = ux; dst.uy[s] = uy; dst.uz[s] = uz;
                dst.g[s] = gm; dst.q[s] = q;
                if (dst.chi) dst.chi[s] = src.chi[p];
                if (a.trn_dst) a.trn_dst[s] = a.trn_src[p];
                if (i1 >= a.dlo && i1 < a.dhi) {
                    dq += (double)q;
                    de += KIND == KIND_PHOTON ? (double)gm * (double)q : ((double)gm - 1.0) * (double)q;
                    dc += 1;
                }
            }
            // energy of the particles erased in this push
            if (a.track && nc < 0 && nc_owned)
                er += KIND == KIND_PHOTON ? (double)gm * (double)q : ((double)gm - 1.0) * (double)q;
        }
        warp_count_runs(count, nc);
    }
    block_diag(a.diag, a.sp, dq, de, dc);
    if (a.track) block_sum(&a.diag->sum_erased[a.sp], er);  // (uniform)
}

// ----------------------------------------------------------------------------
// QED in mixed precision: advance.cpp:90-387 with QED on, as k_push64_qed, in
// FP32 and in the particle's cell frame.  The reference decides emission and
// pair creation per step by rejection (draw r, accept with probability
// rate(r) g dt), so there is no optical depth to carry between steps; the
// rates are evaluated in FP32 and compared with the FP64 draw.  The random
// streams are the FP64 path's (same Philox counters).
// ----------------------------------------------------------------------------

// bear_particle (mc.cpp:118-139): momentum along `dir` with gamma g.
__device__ __forceinline__ void bear_u32(const float dir[3], float gm, bool photon, float u[3]) {
    const float d2 = dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2];
    const float a = photon ? gm / sqrtf(d2) : sqrtf(fmaxf(gm * gm - 1.f, 0.f) / d2);
    u[0] = a * dir[0]; u[1] = a * dir[1]; u[2] = a * dir[2];
}

// Particle born during a push at offset o of cell (ci, cj, ck) (o may leave
// [0, 1)): appended to the target's output buffer, erased if its cell is not
// inside (place(p), plist.cpp:22-39).  Counted in the target's diagnostics.
__device__ __forceinline__ void append32(const AppendTarget<PStore32>& t, const Grid& g, int dlo, int dhi, int ci,
                                         int cj, int ck, const float o[3], const float u[3], float gm, float q,
                                         float chi, bool photon, unsigned int* status, DiagAccum* diag) {
    int si, sj, sk;
    const float ox = wrap_offset(o[0], si), oy = wrap_offset(o[1], sj), oz = wrap_offset(o[2], sk);
    const int i = ci + si, j = cj + sj, k = ck + sk;
    if (!inside(g, i, j, k)) return;
    const int slot = t.base + atomicAdd(t.counter, 1);
    if (slot >= t.cap) {
        atomicOr(status, (unsigned int)ST_CAPACITY);
        return;
    }
    const int c = cidx(g, i, j, k);
    t.dst.cell[slot] = c;
    t.dst.ox[slot] = ox; t.dst.oy[slot] = oy; t.dst.oz[slot] = oz;
    t.dst.ux[slot] = u[0]; t.dst.uy[slot] = u[1]; t.dst.uz[slot] = u[2];
    t.dst.g[slot] = gm; t.dst.q[slot] = q;
    if (t.dst.chi) t.dst.chi[slot] = chi;
    t.newcell[slot] = c;
    if (i < dlo || i >= dhi) return;
    atomicAdd(&diag->sum_q[t.sp], (double)q);
    atomicAdd(&diag->sum_e[t.sp], photon ? (double)gm * (double)q : ((double)gm - 1.0) * (double)q);
    atomicAdd(&diag->cnt[t.sp], 1ull);
}

// A lepton born from a photon at offset o of cell (ci, cj, ck): pushed from
// t_n, chi at t_{n+1/2}, moved with current deposition (advance.cpp:172-236).
template <int PUSHER>
__device__ __forceinline__ void born_lepton32(const Fields<float>& f, const Grid& g, const PushArgs32& a,
                                              float e_s, int ci, int cj, int ck, const float o0[3],
                                              const float dir[3], float gm, float chi, float q, float cmr,
                                              const float E[3], const float B[3], const AppendTarget<PStore32>& t) {
    float u[3];
    bear_u32(dir, gm, false, u);
    const float up[3] = {u[0], u[1], u[2]};
    const float gp = gm;
    push<PUSHER>(cmr, u[0], u[1], u[2], gm, E, B, a.dt);
    const float ui[3] = {0.5f * (u[0] + up[0]), 0.5f * (u[1] + up[1]), 0.5f * (u[2] + up[2])};
    chi = qed_chi(E, B, ui, 0.5f * (gm + gp), e_s);
    const float tt = a.dt / gm;
    const float d[3] = {u[0] * tt * a.idx, u[1] * tt * a.idy, u[2] * tt * a.idz};
    float o[3] = {o0[0], o0[1], o0[2]};
    jdeposition(f, g, o, d, q, ci, cj, ck, a.status);
    append32(t, g, a.dlo, a.dhi, ci, cj, ck, o, u, gm, q, chi, false, a.status, a.diag);
}

template <int PUSHER, int KIND>
__global__ void __launch_bounds__(256, 2) k_push32_qed(Fields<float> f, Grid g, PStore32 src, PStore32 dst,
                                                    const int32_t* __restrict__ perm,
                                                    int32_t* __restrict__ newcell, PushArgs32 a, QedArgs qa,
                                                    AppendTarget<PStore32> t0, AppendTarget<PStore32> t1) {
    double dq = 0.0, de = 0.0;
    unsigned long long dc = 0;
    // block-sized chunks with the grid striding over them, diagnostics
    // reduced once per block (as in the pushes without QED)
    const ChunkRange cr = chunk_range(a.n, a.resident);
    // the next chunk's slot loaded a chunk ahead (as in k_push32)
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
    float o[3] = {0.f, 0.f, 0.f}, dmove[3] = {0.f, 0.f, 0.f};
    float ux = 0.f, uy = 0.f, uz = 0.f, gm = 1.f, q = 0.f, chi = 0.f;
    int i0 = 0, j0 = 0, k0 = 0, nc = -1, i1 = 0, j1 = 0, k1 = 0;
    bool converted = false;  // a photon that became a pair is not an erasure
    bool live = false;
    bool deferred = false;   // the move's current and cell wait for deposit_runs
    if (s < a.n) {
        const int c0 = src.cell[p];
        i0 = g.div_nynz.div(c0);
        const int r0 = c0 - i0 * g.nynz;
        j0 = g.div_nz.div(r0);
        k0 = r0 - j0 * g.nz;
        o[0] = src.ox[p]; o[1] = src.oy[p]; o[2] = src.oz[p];
        ux = src.ux[p]; uy = src.uy[p]; uz = src.uz[p]; gm = src.g[p];
        q = src.q[p];
        chi = src.chi[p];
        const float e_s = (float)qa.e_s;
        i1 = i0; j1 = j0; k1 = k0;
        live = !kill_layer(g, i0, j0, k0);
        if (live) {
            float E[3], B[3];
            gather(f, g, i0, j0, k0, o[0], o[1], o[2], E, B);
            B[2] += a.ext_bz;
            double rd, r2;
            uniform2(philox4x32_10((uint32_t)s, (uint32_t)a.sp, RNG_PUSH, qa.step, qa.key0, qa.key1), rd, r2);
            float r = (float)rd;
            if (KIND == KIND_PHOTON) {
                const float ui[3] = {ux, uy, uz};
                const float g_prev = gm, chi_prev = chi;
                chi = qed_chi(E, B, ui, gm, e_s);
                const float am = 0.5f * (chi + chi_prev);
                // tilde_w's range check (r g >= 1 and (1 - r) g >= 1, mc.cpp:76-97)
                // on the FP64 draw: in FP32, 1 - r rounds to 1 for draws below
                // 2^-24 and the check would let them through
                const bool room = rd * (double)g_prev >= 1.0 && (1.0 - rd) * (double)g_prev >= 1.0;
                const bool pair = room && !(r2 >= (double)(qed_tilde_w(g_prev, r, am, e_s) * g_prev * a.dt));
                if (!pair) {
                    const float tt = a.dt / gm;
                    o[0] += ux * tt * a.idx; o[1] += uy * tt * a.idy; o[2] += uz * tt * a.idz;
                    int si, sj, sk;
                    o[0] = wrap_offset(o[0], si); o[1] = wrap_offset(o[1], sj); o[2] = wrap_offset(o[2], sk);
                    i1 = i0 + si; j1 = j0 + sj; k1 = k0 + sk;
                    if (!(si | sj | sk) || inside(g, i1, j1, k1)) nc = cidx(g, i1, j1, k1);
                } else {
                    converted = true;
                    // electron with r of the photon energy, positron with 1 - r
                    born_lepton32<PUSHER>(f, g, a, e_s, i0, j0, k0, o, ui, r * g_prev, r * chi, -q, -1.f, E, B, t0);
                    born_lepton32<PUSHER>(f, g, a, e_s, i0, j0, k0, o, ui, (1.f - r) * gm, (1.f - r) * chi, q, 1.f,
                                          E, B, t1);
                }
            } else {
                const float up[3] = {ux, uy, uz};
                const float g_prev = gm, chi_prev = chi;
                push<PUSHER>(a.cmr, ux, uy, uz, gm, E, B, a.dt);
                const float ui[3] = {0.5f * (ux + up[0]), 0.5f * (uy + up[1]), 0.5f * (uz + up[2])};
                chi = qed_chi(E, B, ui, 0.5f * (gm + g_prev), e_s);
                const float am = 0.5f * (chi + chi_prev);
                // w's range check ((1 - r) g >= 1, r > 0, mc.cpp:40-74) on the
                // FP64 draw, as for tilde_w: a resting lepton cannot emit
                const bool room = rd > 0.0 && (1.0 - rd) * (double)g_prev >= 1.0;
                const bool emit = room && !(r2 >= (double)(qed_w(g_prev, r, am, e_s) * g_prev * a.dt));
                if (!emit) {
                    const float tt = a.dt / gm;
                    dmove[0] = ux * tt * a.idx; dmove[1] = uy * tt * a.idy; dmove[2] = uz * tt * a.idz;
                    deferred = true;
                } else {
                    // photon born at the lepton's t_n position, then moved to
                    // t_{n+3/2} (advance.cpp:294-306)
                    float am2 = 0.5f * a.dt / g_prev;
                    float ph[3] = {o[0] - am2 * up[0] * a.idx, o[1] - am2 * up[1] * a.idy,
                                   o[2] - am2 * up[2] * a.idz};
                    const float gph = r * g_prev;
                    float uph[3];
                    bear_u32(up, gph, true, uph);
                    const float a3 = 3.f * am2 * g_prev / gph;
                    ph[0] += a3 * uph[0] * a.idx;
                    ph[1] += a3 * uph[1] * a.idy;
                    ph[2] += a3 * uph[2] * a.idz;
                    if (a.dcat) {
                        // dump_photons: the photon is deleted as it is born (advance.cpp:302-306)
                        const double px = (double)i0 + (double)ph[0];
                        if ((int)floor(px) >= a.dlo && (int)floor(px) < a.dhi) {
                            catch_particle(*a.dcat, t0.sp, a.step, 2, s, px, (double)j0 + (double)ph[1],
                                           (double)k0 + (double)ph[2], uph[0], uph[1], uph[2], gph, fabsf(q), r * chi);
                            atomicAdd(&a.diag->sum_erased[t0.sp], (double)gph * (double)fabsf(q));
                        }
                    } else {
                        append32(t0, g, a.dlo, a.dhi, i0, j0, k0, ph, uph, gph, fabsf(q), r * chi, true, a.status,
                                 a.diag);
                    }
                    // recoil (advance.cpp:308-322)
                    chi = (1.f - r) * chi;
                    gm = (1.f - r) * g_prev;
                    const float sc =
                        sqrtf(fmaxf(gm * gm - 1.f, 0.f) / (up[0] * up[0] + up[1] * up[1] + up[2] * up[2]));
                    ux = up[0] * sc; uy = up[1] * sc; uz = up[2] * sc;
                    o[0] -= am2 * up[0] * a.idx;
                    o[1] -= am2 * up[1] * a.idy;
                    o[2] -= am2 * up[2] * a.idz;
                    am2 = am2 * g_prev / gm;
                    o[0] += am2 * ux * a.idx;
                    o[1] += am2 * uy * a.idy;
                    o[2] += am2 * uz * a.idz;
                    int si, sj, sk;
                    o[0] = wrap_offset(o[0], si); o[1] = wrap_offset(o[1], sj); o[2] = wrap_offset(o[2], sk);
                    i1 = i0 + si; j1 = j0 + sj; k1 = k0 + sk;
                    if (inside(g, i1, j1, k1)) {
                        gather(f, g, i1, j1, k1, o[0], o[1], o[2], E, B);
                        B[2] += a.ext_bz;
                        push<PUSHER>(a.cmr, ux, uy, uz, gm, E, B, a.dt);
                        const float tt = a.dt / gm;
                        const float d[3] = {ux * tt * a.idx, uy * tt * a.idy, uz * tt * a.idz};
                        jdeposition(f, g, o, d, q, i1, j1, k1, a.status);
                        int ti, tj, tk;
                        o[0] = wrap_offset(o[0], ti); o[1] = wrap_offset(o[1], tj); o[2] = wrap_offset(o[2], tk);
                        const int i2 = i1 + ti, j2 = j1 + tj, k2 = k1 + tk;
                        if (!(ti | tj | tk) || inside(g, i2, j2, k2)) nc = cidx(g, i2, j2, k2);
                        i1 = i2; j1 = j2; k1 = k2;
                    }
                }
            }
            if (!isfinite(gm)) atomicOr(a.status, (unsigned int)ST_NAN);
        }
    }
    if (KIND != KIND_PHOTON) deposit_runs(f, g, o, dmove, q, i0, j0, k0, deferred, a.status);
    if (s < a.n) {
        if (deferred) {
            int si, sj, sk;
            o[0] = wrap_offset(o[0], si); o[1] = wrap_offset(o[1], sj); o[2] = wrap_offset(o[2], sk);
            i1 = i0 + si; j1 = j0 + sj; k1 = k0 + sk;
            if (!(si | sj | sk) || inside(g, i1, j1, k1)) nc = cidx(g, i1, j1, k1);
        }
        newcell[s] = nc;
        const bool erased = nc < 0 && !converted && i1 >= a.dlo && i1 < a.dhi;
        if (erased && a.cat)
            catch_particle(*a.cat, a.sp, a.step, live ? 1 : 0, s, (double)i1 + (double)o[0],
                           (double)j1 + (double)o[1], (double)k1 + (double)o[2], ux, uy, uz, gm, q, chi);
        if (erased && a.track)  // erasures are few: one atomic each
            atomicAdd(&a.diag->sum_erased[a.sp],
                      KIND == KIND_PHOTON ? (double)gm * (double)q : ((double)gm - 1.0) * (double)q);
        if (nc >= 0) {
            dst.cell[s] = nc;
            dst.ox[s] = o[0]; dst.oy[s] = o[1]; dst.oz[s] = o[2];
            dst.ux[s] = ux; dst.uy[s] = uy; dst.uz[s] = uz;
            dst.g[s] = gm; dst.q[s] = q; dst.chi[s] = chi;
            if (a.trn_dst) a.trn_dst[s] = a.trn_src[p];
            if (i1 >= a.dlo && i1 < a.dhi) {
                dq += (double)q;
                de += KIND == KIND_PHOTON ? (double)gm * (double)q : ((double)gm - 1.0) * (double)q;
                dc += 1;
            }
        }
    }
    }
    block_diag(a.diag, a.sp, dq, de, dc);
}

// birth_from_vacuum (mc.cpp:142-196) for the mixed stores: the rate in FP64
// from the FP32 fields at the cell centre (it underflows in FP32 long before
// FP64); the pair starts at rest at offsets (1/2, 1/2, 1/2) and is pushed
// back half a step in FP32.
template <int PUSHER>
__global__ void __launch_bounds__(256) k_vacuum32(Fields<float> f, Grid g, QedArgs qa, float dt, double dtdV,
                                                  float qv, AppendTarget<PStore32> t0,
                                                  AppendTarget<PStore32> t1, unsigned int* status) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nc) return;
    const int k = c % g.nz, j = (c / g.nz) % g.ny, i = c / g.nynz;
    if (i < 2 || i >= g.nx - 2 || j < 2 || j >= g.ny - 2 || k < 2 || k >= g.nz - 2) return;
    float E[3], B[3];
    gather(f, g, i, j, k, 0.5f, 0.5f, 0.5f, E, B);
    double r, r2;
    uniform2(philox4x32_10((uint32_t)c, 0u, RNG_VACUUM, qa.step, qa.key0, qa.key1), r, r2);
    const double Ed[3] = {E[0], E[1], E[2]}, Bd[3] = {B[0], B[1], B[2]};
    if (!(r < qed_vacuum_W(Ed, Bd, qa.e_s) * dtdV)) return;
    for (int e = 0; e < 2; e++) {
        const AppendTarget<PStore32>& t = e == 0 ? t0 : t1;
        float ux = 0.f, uy = 0.f, uz = 0.f, gm = 1.f;
        push<PUSHER>(e == 0 ? -1.f : 1.f, ux, uy, uz, gm, E, B, -0.5f * dt);
        const int slot = t.base + atomicAdd(t.counter, 1);
        if (slot >= t.cap) {
            atomicOr(status, (unsigned int)ST_CAPACITY);
            continue;
        }
        t.dst.cell[slot] = c;
        t.dst.ox[slot] = 0.5f; t.dst.oy[slot] = 0.5f; t.dst.oz[slot] = 0.5f;
        t.dst.ux[slot] = ux; t.dst.uy[slot] = uy; t.dst.uz[slot] = uz;
        t.dst.g[slot] = gm; t.dst.q[slot] = e == 0 ? -qv : qv;
        t.dst.chi[slot] = 0.f;
        t.newcell[slot] = c;
    }
}


SolverCoef solver_coef(const qp_params& p);

void launch_fields_mixed(State& s, int phase) {
    Fields<float> f = fields_of<float>(s);
    Coef<float> c(solver_coef(s.prm));
    dim3 blk(32, 8, 1);
    constexpr int CPT = FieldCells<float>::value;
    dim3 grd((s.grid.nz + 31) / 32, (s.grid.ny + 7) / 8, (s.grid.nx + CPT - 1) / CPT);
    const int sol = s.prm.solver;
#define QP_LF(SOL, PH) k_field<float, SOL, PH><<<grd, blk, 0, s.stream>>>(f, s.grid, c, s.d_diag, s.diag_lo, s.diag_hi)
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

void zero_planes_mixed(State& s, const ZeroPlane* zp, int n) {
    Fields<float> f = fields_of<float>(s);
    for (int a = 0; a < n; a++) {
        int nu = zp[a].axis == 2 ? s.grid.ny : s.grid.nz;
        int nv = zp[a].axis == 0 ? s.grid.ny : s.grid.nx;
        dim3 grd((nu + 127) / 128, nv);
        k_zero_plane<float><<<grd, 128, 0, s.stream>>>(f, s.grid, zp[a].axis, zp[a].plane, zp[a].comps);
        s.launches++;
    }
}

// Push of one species; also leaves the particles-per-new-cell histogram in
// sp.count (zeroed here).
void launch_push_mixed(State& s, int si, double external_bz) {
    Species& sp = s.sp[si];
    cudaMemsetAsync(sp.count, 0, (size_t)s.grid.nc * sizeof(int32_t), s.stream);
    if (sp.n == 0) return;
    PStore32 src, dst;
    src.cell = (int32_t*)sp.buf[sp.cur][0];
    dst.cell = (int32_t*)sp.buf[1 - sp.cur][0];
    float** ps[9] = {&src.ox, &src.oy, &src.oz, &src.ux, &src.uy, &src.uz, &src.g, &src.q, &src.chi};
    float** pd[9] = {&dst.ox, &dst.oy, &dst.oz, &dst.ux, &dst.uy, &dst.uz, &dst.g, &dst.q, &dst.chi};
    for (int a = 0; a < 9; a++) {
        *ps[a] = (float*)sp.buf[sp.cur][1 + a];
        *pd[a] = (float*)sp.buf[1 - sp.cur][1 + a];
    }
    PushArgs32 a{};
    a.cmr = (float)sp.cmr; a.dt = (float)s.prm.dt;
    a.idx = (float)(1.0 / s.prm.dx); a.idy = (float)(1.0 / s.prm.dy); a.idz = (float)(1.0 / s.prm.dz);
    a.ext_bz = (float)external_bz; a.n = (int)sp.n; a.sp = si; a.kind = sp.kind;
    a.status = s.d_status; a.diag = s.d_diag;
    a.track = s.track_erased ? 1 : 0;
    a.step = (uint32_t)s.step_index;
    a.cat = s.catch_erasures ? s.d_cat : nullptr;
    a.dcat = s.dump_photons ? s.d_cat : nullptr;
    a.trn_src = sp.trn[sp.cur];
    a.trn_dst = sp.trn[1 - sp.cur];
    a.dlo = s.diag_lo; a.dhi = s.diag_hi;
    const PushShape sh = push_shapes32[s.push_shape_mixed];
    const int nb = push_blocks(s, sp.n, sh, s.push_waves_mixed, &a.resident);
    Fields<float> f = fields_of<float>(s);
    const bool vay = s.prm.pusher == QP_PUSHER_VAY;
#define QP_LS(P, K, BS, MB) \
    do { if (s.prefetch) k_push32<P, K, BS, MB, true><<<nb, BS, 0, s.stream>>>(f, s.grid, src, dst, sp.perm, sp.newcell, sp.count, a); \
         else k_push32<P, K, BS, MB, false><<<nb, BS, 0, s.stream>>>(f, s.grid, src, dst, sp.perm, sp.newcell, sp.count, a); } while (0)
#define QP_LP(P, K)                              \
    do { switch (s.push_shape_mixed) {                 \
        case 0: QP_LS(P, K, 256, 3); break;      \
        case 2: QP_LS(P, K, 128, 7); break;      \
        case 3: QP_LS(P, K, 128, 6); break;      \
        case 4: QP_LS(P, K, 128, 8); break;      \
        case 5: QP_LS(P, K, 64, 14); break;      \
        default: QP_LS(P, K, 256, 4); break;     \
    } } while (0)
    if (sp.kind == KIND_PHOTON) QP_LP(QP_PUSHER_BORIS, KIND_PHOTON);
    else if (vay) QP_LP(QP_PUSHER_VAY, KIND_LEPTON);
    else QP_LP(QP_PUSHER_BORIS, KIND_LEPTON);
#undef QP_LP
#undef QP_LS
    s.launches++;
}

static PStore32 store32(Species& sp, int b) {
    PStore32 st;
    st.cell = (int32_t*)sp.buf[b][0];
    float** ps[9] = {&st.ox, &st.oy, &st.oz, &st.ux, &st.uy, &st.uz, &st.g, &st.q, &st.chi};
    for (int a = 0; a < 9; a++) *ps[a] = (float*)sp.buf[b][1 + a];
    return st;
}

static AppendTarget<PStore32> target32(State& s, int si, bool output) {
    Species& sp = s.sp[si];
    AppendTarget<PStore32> t;
    t.dst = store32(sp, output ? 1 - sp.cur : sp.cur);
    t.newcell = sp.newcell;
    t.counter = sp.d_counter;
    t.base = (int)(output ? sp.n : sp.slots);
    t.cap = (int)sp.cap;
    t.sp = si;
    return t;
}

static QedArgs qed_args32(State& s) {
    QedArgs q;
    q.e_s = s.prm.lambda_cm / 2.4263086e-10;  // main.cpp:2276
    q.key0 = (uint32_t)(s.prm.seed & 0xffffffffu);
    q.key1 = (uint32_t)(s.prm.seed >> 32);
    q.step = (uint32_t)s.step_index;
    return q;
}

int launch_push_mixed_qed(State& s, int si, double external_bz) {
    Species& sp = s.sp[si];
    if (sp.n == 0) return QP_OK;
    if (sp.kind == KIND_ION) {
        launch_push_mixed(s, si, external_bz);
        return QP_OK;
    }
    PStore32 src = store32(sp, sp.cur), dst = store32(sp, 1 - sp.cur);
    PushArgs32 a{};
    a.cmr = (float)sp.cmr; a.dt = (float)s.prm.dt;
    a.idx = (float)(1.0 / s.prm.dx); a.idy = (float)(1.0 / s.prm.dy); a.idz = (float)(1.0 / s.prm.dz);
    a.ext_bz = (float)external_bz; a.n = (int)sp.n; a.sp = si; a.kind = sp.kind;
    a.status = s.d_status; a.diag = s.d_diag;
    a.track = s.track_erased ? 1 : 0;
    a.step = (uint32_t)s.step_index;
    a.cat = s.catch_erasures ? s.d_cat : nullptr;
    a.dcat = s.dump_photons ? s.d_cat : nullptr;
    a.trn_src = sp.trn[sp.cur];
    a.trn_dst = sp.trn[1 - sp.cur];
    a.dlo = s.diag_lo; a.dhi = s.diag_hi;
    QedArgs qa = qed_args32(s);
    AppendTarget<PStore32> t0, t1;
    if (sp.kind == KIND_PHOTON) {
        t0 = target32(s, s.sp_e, true);
        t1 = target32(s, s.sp_p, true);
    } else {
        t0 = target32(s, s.sp_ph, true);
        t1 = t0;
    }
    // chunked grid in groups of two blocks per SM (three, as the 80 registers
    // would allow, measured the same in the cascade)
    const int nb = push_blocks(s, sp.n, PushShape{256, 2}, s.push_waves_qed, &a.resident);
    Fields<float> f = fields_of<float>(s);
    const bool vay = s.prm.pusher == QP_PUSHER_VAY;
#define QP_LQ(P, K) k_push32_qed<P, K><<<nb, 256, 0, s.stream>>>(f, s.grid, src, dst, sp.perm, sp.newcell, a, qa, t0, t1)
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

int launch_vacuum_mixed(State& s) {
    const double PI = 3.141592653589793;
    const qp_params& p = s.prm;
    const double dV = p.dx * p.dy * p.dz;
    const double qv = 8 * PI * PI / dV * 2.818e-13 / p.lambda_cm;  // main.cpp:2324
    QedArgs qa = qed_args32(s);
    AppendTarget<PStore32> t0 = target32(s, s.sp_e, false), t1 = target32(s, s.sp_p, false);
    Fields<float> f = fields_of<float>(s);
    const int nb = (s.grid.nc + 255) / 256;
    if (p.pusher == QP_PUSHER_VAY)
        k_vacuum32<QP_PUSHER_VAY><<<nb, 256, 0, s.stream>>>(f, s.grid, qa, (float)p.dt, p.dt * dV, (float)qv, t0, t1,
                                                             s.d_status);
    else
        k_vacuum32<QP_PUSHER_BORIS><<<nb, 256, 0, s.stream>>>(f, s.grid, qa, (float)p.dt, p.dt * dV, (float)qv, t0,
                                                               t1, s.d_status);
    s.launches++;
    return QP_OK;
}


}  // namespace qp
