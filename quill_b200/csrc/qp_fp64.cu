// FP64 path: the reference arithmetic on the GPU.  Built with --fmad=false so
// that every multiply and add rounds separately, as the reference CPU build
// does with -ffp-contract=off.
#include "qp_kernels.cuh"

namespace qp {

// One thread per particle in traversal order: gather -> push -> current
// deposition (moving the particle segment by segment) -> new cell.  The
// particle is read through perm from the previous layout and written at its
// traversal position into the other buffer.  Erased particles (outside
// is_inside after a move, or in a p_boundary layer on entry) get newcell -1.
// advance.cpp:90-387 with QED off: photons fly straight without current
// (:155-252), leptons and ions are pushed and deposit (:253-371).
template <int PUSHER, int KIND>
__global__ void __launch_bounds__(256) k_push64(Fields<double> f, Grid g, PStore64 src, PStore64 dst,
                                                const int32_t* __restrict__ perm,
                                                int32_t* __restrict__ newcell, PushArgs a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double dq = 0.0, de = 0.0;
    unsigned long long dc = 0;
    if (s < a.n) {
        const int p = perm[s];
        double pos[3] = {src.x[p], src.y[p], src.z[p]};
        double ux = src.ux[p], uy = src.uy[p], uz = src.uz[p], gm = src.g[p];
        const double q = src.q[p];
        const int i0 = (int)pos[0], j0 = (int)pos[1], k0 = (int)pos[2];
        int nc = -1;
        if (!kill_layer(g, i0, j0, k0)) {
            double E[3], B[3];
            {
                const int i = (int)floor(pos[0]), j = (int)floor(pos[1]), k = (int)floor(pos[2]);
                gather(f, g, i, j, k, pos[0] - i, pos[1] - j, pos[2] - k, E, B);
            }
            B[2] += a.ext_bz;
            if (KIND != KIND_PHOTON) push<PUSHER>(a.cmr, ux, uy, uz, gm, E, B, a.dt);
            // particle::get_displacement (containers.cpp:58-67), then per-axis
            // division by the cell size (advance.cpp:281-284)
            const double t = a.dt / gm;
            double d[3] = {ux * t, uy * t, uz * t};
            d[0] = d[0] / a.dx;
            d[1] = d[1] / a.dy;
            d[2] = d[2] / a.dz;
            if (KIND == KIND_PHOTON) {
                pos[0] = pos[0] + d[0];
                pos[1] = pos[1] + d[1];
                pos[2] = pos[2] + d[2];
            } else {
                jdeposition(f, g, pos, d, q, 0, 0, 0, a.status);
            }
            if (!isfinite(gm)) atomicOr(a.status, (unsigned int)ST_NAN);
            // place(p, i, j, k) (plist.cpp:7-39): relink only if the cell
            // changed, erase if the new cell is not inside
            const int i1 = (int)pos[0], j1 = (int)pos[1], k1 = (int)pos[2];
            const bool moved = (i1 != i0) || (j1 != j0) || (k1 != k0);
            if (!moved || inside(g, i1, j1, k1)) nc = cidx(g, i1, j1, k1);
        }
        newcell[s] = nc;
        if (nc >= 0) {
            dst.x[s] = pos[0]; dst.y[s] = pos[1]; dst.z[s] = pos[2];
            dst.ux[s] = ux; dst.uy[s] = uy; dst.uz[s] = uz;
            dst.g[s] = gm; dst.q[s] = q;
            if (dst.chi) dst.chi[s] = src.chi[p];
            dq = q;
            de = KIND == KIND_PHOTON ? gm * q : (gm - 1) * q;
            dc = 1;
        }
    }
    block_diag(a.diag, a.sp, dq, de, dc);
}

static Fields<double> fields64(State& s) {
    double* b = (double*)s.fields;
    const size_t nc = (size_t)s.grid.nc;
    Fields<double> f;
    double** p[12] = {&f.ex, &f.ey, &f.ez, &f.bx, &f.by, &f.bz, &f.jx, &f.jy, &f.jz, &f.bex, &f.bey, &f.bez};
    for (int a = 0; a < 12; a++) *p[a] = b + a * nc;
    return f;
}

SolverCoef solver_coef(const qp_params& p);

void launch_fields_fp64(State& s, int phase) {
    Fields<double> f = fields64(s);
    Coef<double> c(solver_coef(s.prm));
    dim3 blk(32, 8, 1);
    dim3 grd((s.grid.nz + 31) / 32, (s.grid.ny + 7) / 8, s.grid.nx);
    const int sol = s.prm.solver;
#define QP_LF(SOL, PH) k_field<double, SOL, PH><<<grd, blk, 0, s.stream>>>(f, s.grid, c)
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

void zero_planes_fp64(State& s, const ZeroPlane* zp, int n) {
    Fields<double> f = fields64(s);
    for (int a = 0; a < n; a++) {
        int nu = zp[a].axis == 2 ? s.grid.ny : s.grid.nz;
        int nv = zp[a].axis == 0 ? s.grid.ny : s.grid.nx;
        dim3 grd((nu + 127) / 128, nv);
        k_zero_plane<double><<<grd, 128, 0, s.stream>>>(f, s.grid, zp[a].axis, zp[a].plane, zp[a].comps);
        s.launches++;
    }
}

void launch_push_fp64(State& s, int si, double external_bz) {
    Species& sp = s.sp[si];
    if (sp.n == 0) return;
    PStore64 src, dst;
    double** ps[9] = {&src.x, &src.y, &src.z, &src.ux, &src.uy, &src.uz, &src.g, &src.q, &src.chi};
    double** pd[9] = {&dst.x, &dst.y, &dst.z, &dst.ux, &dst.uy, &dst.uz, &dst.g, &dst.q, &dst.chi};
    for (int a = 0; a < 9; a++) {
        *ps[a] = (double*)sp.buf[sp.cur][a];
        *pd[a] = (double*)sp.buf[1 - sp.cur][a];
    }
    PushArgs a;
    a.cmr = sp.cmr; a.dt = s.prm.dt; a.dx = s.prm.dx; a.dy = s.prm.dy; a.dz = s.prm.dz;
    a.ext_bz = external_bz; a.n = (int)sp.n; a.sp = si; a.kind = sp.kind;
    a.status = s.d_status; a.diag = s.d_diag;
    const int nb = (int)((sp.n + 255) / 256);
    Fields<double> f = fields64(s);
    const bool vay = s.prm.pusher == QP_PUSHER_VAY;
#define QP_LP(P, K) k_push64<P, K><<<nb, 256, 0, s.stream>>>(f, s.grid, src, dst, sp.perm, sp.newcell, a)
    if (sp.kind == KIND_PHOTON) QP_LP(QP_PUSHER_BORIS, KIND_PHOTON);
    else if (vay) QP_LP(QP_PUSHER_VAY, KIND_LEPTON);
    else QP_LP(QP_PUSHER_BORIS, KIND_LEPTON);
#undef QP_LP
    s.launches++;
}

void launch_field_energy_fp64(State& s) {
    Fields<double> f = fields64(s);
    k_field_energy<double><<<148 * 4, 256, 0, s.stream>>>(f, s.grid.nc, s.d_diag);
    s.launches++;
}

}  // namespace qp
