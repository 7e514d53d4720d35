// Mixed-precision path: positions as a linear cell index plus an FP32 offset
// in [0, 1), FP32 push, gather, current deposition and Maxwell stencils.
// Diagnostics are accumulated in FP64.  The algorithms are the reference's;
// the deposition runs in the particle's cell frame (offsets), which is the
// reference's absolute-coordinate algorithm shifted by an integer.
#include "qp_kernels.cuh"

namespace qp {

struct PushArgs32 {
    float cmr, dt, idx, idy, idz, ext_bz;
    int n, sp, kind;
    int track;  // sum the energy of erased particles into diag->sum_erased
    unsigned int* status;
    DiagAccum* diag;
    uint32_t step;
    const CatchBuf* cat;  // device copy; nullptr: catching off
    const int32_t* trn_src;  // track numbers in, by slot / out, by traversal position; nullptr: off
    int32_t* trn_dst;
    int dlo, dhi;  // the diagnostics count particles whose new cell has i in [dlo, dhi)
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

// One thread per particle in traversal order (see k_push64): the move runs in
// the particle's cell frame (offsets in [0, 1)), the current through the
// warp's segment-slot run reduction (deposit_runs).
template <int PUSHER, int KIND, int MINB>
__global__ void __launch_bounds__(256, MINB) k_push32(Fields<float> f, Grid g, PStore32 src, PStore32 dst,
                                                   const int32_t* __restrict__ perm, int32_t* __restrict__ newcell,
                                                   int32_t* __restrict__ count, PushArgs32 a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double dq = 0.0, de = 0.0;
    unsigned long long dc = 0;
    int nc = -1, p = 0, i0 = 0, j0 = 0, k0 = 0;
    bool nc_owned = true;
    bool live = false, active = false;
    float o[3] = {0.f, 0.f, 0.f}, d[3] = {0.f, 0.f, 0.f};
    float ux = 0.f, uy = 0.f, uz = 0.f, gm = 1.f, q = 0.f;
    if (s < a.n) {
        p = perm[s];
        const int c0 = src.cell[p];
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
                dq = (double)q;
                de = KIND == KIND_PHOTON ? (double)gm * (double)q : ((double)gm - 1.0) * (double)q;
                dc = 1;
            }
        }
    }
    warp_count_runs(count, nc);
    block_diag(a.diag, a.sp, dq, de, dc);
    if (a.track) {  // uniform: energy of the particles erased in this push
        const double er = (s < a.n && nc < 0 && nc_owned)
                              ? (KIND == KIND_PHOTON ? (double)gm * (double)q : ((double)gm - 1.0) * (double)q)
                              : 0.0;
        block_sum(&a.diag->sum_erased[a.sp], er);
    }
}

static Fields<float> fields32(State& s) {
    float* b = (float*)s.fields;
    const size_t nc = (size_t)s.grid.nc;
    Fields<float> f;
    float** p[12] = {&f.ex, &f.ey, &f.ez, &f.bx, &f.by, &f.bz, &f.jx, &f.jy, &f.jz, &f.bex, &f.bey, &f.bez};
    for (int a = 0; a < 12; a++) *p[a] = b + a * nc;
    return f;
}

SolverCoef solver_coef(const qp_params& p);

void launch_fields_mixed(State& s, int phase) {
    Fields<float> f = fields32(s);
    Coef<float> c(solver_coef(s.prm));
    dim3 blk(32, 8, 1);
    dim3 grd((s.grid.nz + 31) / 32, (s.grid.ny + 7) / 8, s.grid.nx);
    const int sol = s.prm.solver;
#define QP_LF(SOL, PH) k_field<float, SOL, PH><<<grd, blk, 0, s.stream>>>(f, s.grid, c)
    if (phase == 0 || phase == 2) {
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
    Fields<float> f = fields32(s);
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
    PushArgs32 a;
    a.cmr = (float)sp.cmr; a.dt = (float)s.prm.dt;
    a.idx = (float)(1.0 / s.prm.dx); a.idy = (float)(1.0 / s.prm.dy); a.idz = (float)(1.0 / s.prm.dz);
    a.ext_bz = (float)external_bz; a.n = (int)sp.n; a.sp = si; a.kind = sp.kind;
    a.status = s.d_status; a.diag = s.d_diag;
    a.track = s.track_erased ? 1 : 0;
    a.step = (uint32_t)s.step_index;
    a.cat = s.d_cat;
    a.trn_src = sp.trn[sp.cur];
    a.trn_dst = sp.trn[1 - sp.cur];
    a.dlo = s.diag_lo; a.dhi = s.diag_hi;
    const int nb = (int)((sp.n + 255) / 256);
    Fields<float> f = fields32(s);
    const bool vay = s.prm.pusher == QP_PUSHER_VAY;
#define QP_LP(P, K)                                                                                          \
    if (s.push_minblocks_mixed == 4)                                                                          \
        k_push32<P, K, 4><<<nb, 256, 0, s.stream>>>(f, s.grid, src, dst, sp.perm, sp.newcell, sp.count, a);   \
    else                                                                                                      \
        k_push32<P, K, 3><<<nb, 256, 0, s.stream>>>(f, s.grid, src, dst, sp.perm, sp.newcell, sp.count, a)
    if (sp.kind == KIND_PHOTON) QP_LP(QP_PUSHER_BORIS, KIND_PHOTON);
    else if (vay) QP_LP(QP_PUSHER_VAY, KIND_LEPTON);
    else QP_LP(QP_PUSHER_BORIS, KIND_LEPTON);
#undef QP_LP
    s.launches++;
}

void launch_field_energy_mixed(State& s) {
    Fields<float> f = fields32(s);
    const size_t off = (size_t)s.diag_lo * s.grid.nynz;
    Fields<float> fo = f;
    fo.ex += off; fo.ey += off; fo.ez += off; fo.bx += off; fo.by += off; fo.bz += off;
    k_field_energy<float><<<148 * 4, 256, 0, s.stream>>>(fo, (s.diag_hi - s.diag_lo) * s.grid.nynz, s.d_diag);
    s.launches++;
}

}  // namespace qp
