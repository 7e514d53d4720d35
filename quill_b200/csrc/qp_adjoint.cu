// Hand-written discrete adjoint of the QED-off FP64 step (FDTD solver, Boris
// pusher): gradients of the final electron kinetic energy (compute_energy's
// energy_e, fout.cpp:87-138) with respect to the loaded E and B planes and to
// every electron's weight q.  No reference counterpart.
//
// Forward step n (qp_step): particles  (x, u, q) -> gather E, Bbar at x ->
// Boris -> d = u' dt / (g' dx) -> segment-split deposition J(x, d, q),
// x' = x + d -> rebin;  fields  B1 = B + 1/2 Cb E,  E' = E + Ce B1 - dx J,
// B' = B1 + 1/2 Cb E',  Bbar' = Avg B'.  Its adjoint, in reverse:
//   lE* = lE' + 1/2 Cb^T lB'        lB1 = lB' + Ce^T lE*     lJ = -dx lE*
//   lE  = lE* + 1/2 Cb^T lB1        lB  = lB1 (+ Avg^T lBbar from the gather)
// and per particle the transposed Jacobians of deposition, displacement,
// push and gather (evaluated with dual numbers on the branch the forward
// step took), the gather's field adjoints scattered onto the grid.  The
// rebin is a permutation: adjoints follow particles through it.
//
// Checkpointing: the state is saved every `every` steps; each segment is
// re-run forward from its checkpoint while the particle inputs, E, Bbar and
// the rebin permutation of every step are recorded, then swept in reverse.
//
// Built with --fmad=false: the values recomputed inside the backward kernels
// equal the FP64 forward step's, so branch decisions (cell floors, crossing
// order) match it.
//
// Mixed precision: the forward and its re-runs are the FP32 step; each
// step's recorded inputs (cell + offset widened to absolute FP64 positions,
// FP32 momenta, weights, E and Bbar) are the linearisation points of the same
// FP64 adjoint.  The gradient is that of the FP64 step map along the FP32
// trajectory: it agrees with the FP64 adjoint to the FP32 trajectory's
// distance from the FP64 one.
#include <cmath>
#include <string>
#include <vector>

#include "qp_dual.cuh"
#include "qp_kernels.cuh"

namespace qp {

namespace {

struct Lam7 {  // particle adjoints: x y z ux uy uz q
    double* a[7];
};

__device__ __forceinline__ bool in_r(int v, int lo, int hi) { return v >= lo && v < hi; }

// FDTD update masks (maxwell.cpp:445-522): which cells update which component
__device__ __forceinline__ void fdtd_masks(const Grid& g, int i, int j, int k, bool mb[3], bool me[3]) {
    const bool ii = in_r(i, 1, g.nx - 1), jj = in_r(j, 1, g.ny - 1), kk = in_r(k, 1, g.nz - 1);
    mb[0] = ii && ((jj && kk) || (j == 0 && kk) || (k == 0 && jj));
    mb[1] = jj && ((ii && kk) || (i == 0 && kk) || (k == 0 && ii));
    mb[2] = kk && ((ii && jj) || (i == 0 && jj) || (j == 0 && ii));
    me[0] = jj && kk && (ii || i == 0);
    me[1] = ii && kk && (jj || j == 0);
    me[2] = ii && jj && (kk || k == 0);
}

// lE += 1/2 Cb^T lB : transpose of B += 1/2 (curl terms of E)
__global__ void k_cbT(Grid g, double dtdx, double dtdy, double dtdz, const double* __restrict__ lbx,
                      const double* __restrict__ lby, const double* __restrict__ lbz, double* lex, double* ley,
                      double* lez) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= g.nc) return;
    const int k = y % g.nz, j = (y / g.nz) % g.ny, i = y / g.nynz;
    bool mb[3], me[3];
    fdtd_masks(g, i, j, k, mb, me);
    const int I = g.nynz, J = g.nz;
    if (mb[0]) {  // bx += 0.5*(-dtdy*(ez[y+J]-ez[y]) + dtdz*(ey[y+1]-ey[y]))
        const double a = 0.5 * lbx[y];
        atomicAdd(lez + y + J, -dtdy * a); atomicAdd(lez + y, dtdy * a);
        atomicAdd(ley + y + 1, dtdz * a); atomicAdd(ley + y, -dtdz * a);
    }
    if (mb[1]) {  // by += 0.5*(dtdx*(ez[y+I]-ez[y]) - dtdz*(ex[y+1]-ex[y]))
        const double a = 0.5 * lby[y];
        atomicAdd(lez + y + I, dtdx * a); atomicAdd(lez + y, -dtdx * a);
        atomicAdd(lex + y + 1, -dtdz * a); atomicAdd(lex + y, dtdz * a);
    }
    if (mb[2]) {  // bz += 0.5*(dtdy*(ex[y+J]-ex[y]) - dtdx*(ey[y+I]-ey[y]))
        const double a = 0.5 * lbz[y];
        atomicAdd(lex + y + J, dtdy * a); atomicAdd(lex + y, -dtdy * a);
        atomicAdd(ley + y + I, -dtdx * a); atomicAdd(ley + y, dtdx * a);
    }
}

// lB += Ce^T lE and lJ = -dx * lE on updated cells: transpose of
// E += curl terms of B - J dx
__global__ void k_ceT(Grid g, double dtdx, double dtdy, double dtdz, double dx, double dy, double dz,
                      const double* __restrict__ lex, const double* __restrict__ ley, const double* __restrict__ lez,
                      double* lbx, double* lby, double* lbz, double* ljx, double* ljy, double* ljz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= g.nc) return;
    const int k = x % g.nz, j = (x / g.nz) % g.ny, i = x / g.nynz;
    bool mb[3], me[3];
    fdtd_masks(g, i, j, k, mb, me);
    const int I = g.nynz, J = g.nz;
    ljx[x] = 0.0; ljy[x] = 0.0; ljz[x] = 0.0;
    if (me[0]) {  // ex += dtdy*(bz[x]-bz[x-J]) - dtdz*(by[x]-by[x-1]) - jx*dx
        const double a = lex[x];
        atomicAdd(lbz + x, dtdy * a); atomicAdd(lbz + x - J, -dtdy * a);
        atomicAdd(lby + x, -dtdz * a); atomicAdd(lby + x - 1, dtdz * a);
        ljx[x] = -dx * a;
    }
    if (me[1]) {  // ey += -dtdx*(bz[x]-bz[x-I]) + dtdz*(bx[x]-bx[x-1]) - jy*dy
        const double a = ley[x];
        atomicAdd(lbz + x, -dtdx * a); atomicAdd(lbz + x - I, dtdx * a);
        atomicAdd(lbx + x, dtdz * a); atomicAdd(lbx + x - 1, -dtdz * a);
        ljy[x] = -dy * a;
    }
    if (me[2]) {  // ez += dtdx*(by[x]-by[x-I]) - dtdy*(bx[x]-bx[x-J]) - jz*dz
        const double a = lez[x];
        atomicAdd(lby + x, dtdx * a); atomicAdd(lby + x - I, -dtdx * a);
        atomicAdd(lbx + x, -dtdy * a); atomicAdd(lbx + x - J, dtdy * a);
        ljz[x] = -dz * a;
    }
}

// lB += Avg^T lBbar : transpose of interpolate_be (advance.cpp:20-83)
__global__ void k_avgT(Grid g, const double* __restrict__ lbbx, const double* __restrict__ lbby,
                       const double* __restrict__ lbbz, double* lbx, double* lby, double* lbz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= g.nc) return;
    const int k = x % g.nz, j = (x / g.nz) % g.ny, i = x / g.nynz;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool in_i = in_r(i, 1, nx - 1), in_j = in_r(j, 1, ny - 1), in_k = in_r(k, 1, nz - 1);
    const bool main_ = in_i && in_j && in_k;
    const bool i0 = i == 0 && in_j && in_k, i1 = i == nx - 1 && in_j && in_k;
    const bool j0 = j == 0 && in_i && in_k, j1 = j == ny - 1 && in_i && in_k;
    const bool k0 = k == 0 && in_i && in_j, k1 = k == nz - 1 && in_i && in_j;
    if (!(main_ || i0 || i1 || j0 || j1 || k0 || k1)) return;
    const int I = g.nynz, J = nz;
    {
        const double a = lbbx[x];
        if (i1) { const double c = 0.25 * a; atomicAdd(lbx + x, c); atomicAdd(lbx + x - 1, c); atomicAdd(lbx + x - J, c); atomicAdd(lbx + x - J - 1, c); }
        else if (j0) { const double c = 0.25 * a; atomicAdd(lbx + x, c); atomicAdd(lbx + x + I, c); atomicAdd(lbx + x - 1, c); atomicAdd(lbx + x + I - 1, c); }
        else if (k0) { const double c = 0.25 * a; atomicAdd(lbx + x, c); atomicAdd(lbx + x + I, c); atomicAdd(lbx + x - J, c); atomicAdd(lbx + x + I - J, c); }
        else {
            const double c = 0.125 * a;
            const int o[8] = {0, I, -1, I - 1, -J, I - J, -J - 1, I - J - 1};
            for (int t = 0; t < 8; t++) atomicAdd(lbx + x + o[t], c);
        }
    }
    {
        const double a = lbby[x];
        if (i0) { const double c = 0.25 * a; atomicAdd(lby + x, c); atomicAdd(lby + x - 1, c); atomicAdd(lby + x + J, c); atomicAdd(lby + x + J - 1, c); }
        else if (j1) { const double c = 0.25 * a; atomicAdd(lby + x, c); atomicAdd(lby + x - I, c); atomicAdd(lby + x - 1, c); atomicAdd(lby + x - I - 1, c); }
        else if (k0) { const double c = 0.25 * a; atomicAdd(lby + x, c); atomicAdd(lby + x - I, c); atomicAdd(lby + x + J, c); atomicAdd(lby + x - I + J, c); }
        else {
            const double c = 0.125 * a;
            const int o[8] = {0, -I, -1, -I - 1, J, -I + J, J - 1, -I + J - 1};
            for (int t = 0; t < 8; t++) atomicAdd(lby + x + o[t], c);
        }
    }
    {
        const double a = lbbz[x];
        if (i0) { const double c = 0.25 * a; atomicAdd(lbz + x, c); atomicAdd(lbz + x + 1, c); atomicAdd(lbz + x - J, c); atomicAdd(lbz + x - J + 1, c); }
        else if (j0) { const double c = 0.25 * a; atomicAdd(lbz + x, c); atomicAdd(lbz + x - I, c); atomicAdd(lbz + x + 1, c); atomicAdd(lbz + x - I + 1, c); }
        else if (k1) { const double c = 0.25 * a; atomicAdd(lbz + x, c); atomicAdd(lbz + x - I, c); atomicAdd(lbz + x - J, c); atomicAdd(lbz + x - I - J, c); }
        else {
            const double c = 0.125 * a;
            const int o[8] = {0, -I, 1, -I + 1, -J, -I - J, -J + 1, -I - J + 1};
            for (int t = 0; t < 8; t++) atomicAdd(lbz + x + o[t], c);
        }
    }
}

// Inputs of one step in traversal order (x y z ux uy uz q), read through perm.
__global__ void k_record(PStore64 src, const int32_t* __restrict__ perm, int n, Lam7 rec, double* g_out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = perm[s];
    rec.a[0][s] = src.x[p]; rec.a[1][s] = src.y[p]; rec.a[2][s] = src.z[p];
    rec.a[3][s] = src.ux[p]; rec.a[4][s] = src.uy[p]; rec.a[5][s] = src.uz[p];
    rec.a[6][s] = src.q[p];
    if (g_out) g_out[s] = src.g[p];
}

// The same from the mixed store: absolute positions cell + offset, FP32
// values widened to FP64.
__global__ void k_record32(Grid g, PStore32 src, const int32_t* __restrict__ perm, int n, Lam7 rec,
                           double* g_out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = perm[s];
    const int c = src.cell[p];
    const int i = c / g.nynz, j = (c / g.nz) % g.ny, k = c % g.nz;
    rec.a[0][s] = i + (double)src.ox[p]; rec.a[1][s] = j + (double)src.oy[p]; rec.a[2][s] = k + (double)src.oz[p];
    rec.a[3][s] = src.ux[p]; rec.a[4][s] = src.uy[p]; rec.a[5][s] = src.uz[p];
    rec.a[6][s] = src.q[p];
    if (g_out) g_out[s] = src.g[p];
}

__global__ void k_widen(const float* __restrict__ a, double* __restrict__ b, size_t n) {
    const size_t x = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) b[x] = a[x];
}

// Adjoints through the rebin: out[perm[t]] = in[t] (erased particles keep 0).
__global__ void k_map(const int32_t* __restrict__ perm, int n_next, Lam7 in, Lam7 out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_next) return;
    const int s = perm[t];
#pragma unroll
    for (int a = 0; a < 7; a++) out.a[a][s] = in.a[a][t];
}

// Final-state adjoint of energy_e = -b sum (g - 1) q:
// dL/du = -b q u / g, dL/dq = -b (g - 1).
__global__ void k_loss_seed(Lam7 rec, const double* __restrict__ gam, int n, double b, Lam7 lam) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double q = rec.a[6][s], g = gam[s];
    lam.a[0][s] = 0.0; lam.a[1][s] = 0.0; lam.a[2][s] = 0.0;
    lam.a[3][s] = -b * q * rec.a[3][s] / g;
    lam.a[4][s] = -b * q * rec.a[4][s] / g;
    lam.a[5][s] = -b * q * rec.a[5][s] / g;
    lam.a[6][s] = -b * (g - 1);
}

// Sink that contracts deposition contributions with lJ instead of adding
// them to J: grad += lJ[target] * d(contribution)/d(inputs).
template <int N>
struct AdjSink {
    const double* lj[3];
    double* grad;
    __device__ __forceinline__ void add(int comp, int, int, int, int c, const Dual<N>& v) const {
        const double l = __ldg(lj[comp] + c);
#pragma unroll
        for (int a = 0; a < N; a++) grad[a] += l * v.d[a];
    }
};

// Dual gather: fields are constants, the weights depend on x.
template <int N>
__device__ __forceinline__ void gather_dual(const Fields<double>& f, const Grid& g, int i, int j, int k, Dual<N> xa,
                                            Dual<N> ya, Dual<N> za, Dual<N> E[3], Dual<N> B[3]) {
    const Dual<N> xb = 1.0 - xa, yb = 1.0 - ya, zb = 1.0 - za;
    const int c = cidx(g, i, j, k);
    const int cj1 = c + g.nz, ck1 = c + 1, ci1 = c + g.nynz;
    E[0] = f.ex[c] * yb * zb + f.ex[cj1] * ya * zb + f.ex[ck1] * yb * za + f.ex[cj1 + 1] * ya * za;
    E[1] = f.ey[c] * xb * zb + f.ey[ci1] * xa * zb + f.ey[ck1] * xb * za + f.ey[ci1 + 1] * xa * za;
    E[2] = f.ez[c] * xb * yb + f.ez[ci1] * xa * yb + f.ez[cj1] * xb * ya + f.ez[ci1 + g.nz] * xa * ya;
    B[0] = f.bex[c] * yb * zb + f.bex[cj1] * ya * zb + f.bex[ck1] * yb * za + f.bex[cj1 + 1] * ya * za;
    B[1] = f.bey[c] * xb * zb + f.bey[ci1] * xa * zb + f.bey[ck1] * xb * za + f.bey[ci1 + 1] * xa * za;
    B[2] = f.bez[c] * xb * yb + f.bez[ci1] * xa * yb + f.bez[cj1] * xb * ya + f.bez[ci1 + g.nz] * xa * ya;
}

// Per-particle adjoint of one step.  f holds E and Bbar of step n (read) and
// lE / lBbar accumulators (jx.. = lJ, read; ex.. / bex.. of `lf` written).
__global__ void __launch_bounds__(128) k_adj_particles(Fields<double> f, Grid g, Lam7 rec, int n, PushArgs a,
                                                       const double* __restrict__ ljx, const double* __restrict__ ljy,
                                                       const double* __restrict__ ljz, Lam7 lam,
                                                       double* lex, double* ley, double* lez,
                                                       double* lbbx, double* lbby, double* lbbz) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double x0 = rec.a[0][s], y0 = rec.a[1][s], z0 = rec.a[2][s];
    const int i0 = (int)x0, j0 = (int)y0, k0 = (int)z0;
    if (kill_layer(g, i0, j0, k0)) {  // erased by p_boundary before the push
#pragma unroll
        for (int t = 0; t < 7; t++) lam.a[t][s] = 0.0;
        return;
    }
    const double u0[3] = {rec.a[3][s], rec.a[4][s], rec.a[5][s]};
    const double q = rec.a[6][s];
    // forward values, as the forward step computed them
    double E[3], B[3];
    gather(f, g, i0, j0, k0, x0 - i0, y0 - j0, z0 - k0, E, B);
    B[2] += a.ext_bz;
    double ux = u0[0], uy = u0[1], uz = u0[2], gm = 1.0;
    push_boris(a.cmr, ux, uy, uz, gm, E, B, a.dt);
    const double t = a.dt / gm;
    double d[3] = {ux * t, uy * t, uz * t};
    d[0] = d[0] / a.dx; d[1] = d[1] / a.dy; d[2] = d[2] / a.dz;
    // adjoints of the step's outputs (mapped through the rebin)
    const double lxo[3] = {lam.a[0][s], lam.a[1][s], lam.a[2][s]};
    const double luo[3] = {lam.a[3][s], lam.a[4][s], lam.a[5][s]};
    const double lqo = lam.a[6][s];
    // A: deposition and x' = x + d over (x, d, q)
    double gA[7] = {0, 0, 0, 0, 0, 0, 0};
    {
        Dual<7> p[3] = {Dual<7>::seed(x0, 0), Dual<7>::seed(y0, 1), Dual<7>::seed(z0, 2)};
        const Dual<7> dd[3] = {Dual<7>::seed(d[0], 3), Dual<7>::seed(d[1], 4), Dual<7>::seed(d[2], 5)};
        const Dual<7> qq = Dual<7>::seed(q, 6);
        AdjSink<7> sink;
        sink.lj[0] = ljx; sink.lj[1] = ljy; sink.lj[2] = ljz;
        sink.grad = gA;
        jdeposition_to(sink, g, p, dd, qq, 0, 0, 0, a.status);
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int k = 0; k < 7; k++) gA[k] += lxo[c] * p[c].d[k];
    }
    // B: d = u' (dt / g') / dx over u'
    double lu1[3] = {luo[0], luo[1], luo[2]};
    {
        Dual<3> u1[3] = {Dual<3>::seed(ux, 0), Dual<3>::seed(uy, 1), Dual<3>::seed(uz, 2)};
        const Dual<3> g1 = sqrt(1.0 + u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
        const Dual<3> tt = a.dt / g1;
        const double dxs[3] = {a.dx, a.dy, a.dz};
        for (int c = 0; c < 3; c++) {
            const Dual<3> dc = (u1[c] * tt) / dxs[c];
#pragma unroll
            for (int k = 0; k < 3; k++) lu1[k] += gA[3 + c] * dc.d[k];
        }
    }
    // C: u' = Boris(u, Ep, Bp) over (u, Ep, Bp)
    double gC[9];
    {
        Dual<9> cu[3] = {Dual<9>::seed(u0[0], 0), Dual<9>::seed(u0[1], 1), Dual<9>::seed(u0[2], 2)};
        const Dual<9> cE[3] = {Dual<9>::seed(E[0], 3), Dual<9>::seed(E[1], 4), Dual<9>::seed(E[2], 5)};
        const Dual<9> cB[3] = {Dual<9>::seed(B[0], 6), Dual<9>::seed(B[1], 7), Dual<9>::seed(B[2], 8)};
        Dual<9> cg(1.0);
        push_boris(Dual<9>(a.cmr), cu[0], cu[1], cu[2], cg, cE, cB, Dual<9>(a.dt));
#pragma unroll
        for (int k = 0; k < 9; k++) gC[k] = lu1[0] * cu[0].d[k] + lu1[1] * cu[1].d[k] + lu1[2] * cu[2].d[k];
    }
    // D: Ep, Bp = gather(x) over x; scatter the field adjoints
    double gD[3] = {0, 0, 0};
    {
        const Dual<3> xa = Dual<3>::seed(x0 - i0, 0), ya = Dual<3>::seed(y0 - j0, 1), za = Dual<3>::seed(z0 - k0, 2);
        Dual<3> dE[3], dB[3];
        gather_dual(f, g, i0, j0, k0, xa, ya, za, dE, dB);
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int k = 0; k < 3; k++) gD[k] += gC[3 + c] * dE[c].d[k] + gC[6 + c] * dB[c].d[k];
        const double xa_ = x0 - i0, ya_ = y0 - j0, za_ = z0 - k0;
        const double xb_ = 1 - xa_, yb_ = 1 - ya_, zb_ = 1 - za_;
        const int c = cidx(g, i0, j0, k0);
        const int cj1 = c + g.nz, ck1 = c + 1, ci1 = c + g.nynz;
        const double le0 = gC[3], le1 = gC[4], le2 = gC[5], lb0 = gC[6], lb1 = gC[7], lb2 = gC[8];
        atomicAdd(lex + c, le0 * yb_ * zb_); atomicAdd(lex + cj1, le0 * ya_ * zb_);
        atomicAdd(lex + ck1, le0 * yb_ * za_); atomicAdd(lex + cj1 + 1, le0 * ya_ * za_);
        atomicAdd(ley + c, le1 * xb_ * zb_); atomicAdd(ley + ci1, le1 * xa_ * zb_);
        atomicAdd(ley + ck1, le1 * xb_ * za_); atomicAdd(ley + ci1 + 1, le1 * xa_ * za_);
        atomicAdd(lez + c, le2 * xb_ * yb_); atomicAdd(lez + ci1, le2 * xa_ * yb_);
        atomicAdd(lez + cj1, le2 * xb_ * ya_); atomicAdd(lez + ci1 + g.nz, le2 * xa_ * ya_);
        atomicAdd(lbbx + c, lb0 * yb_ * zb_); atomicAdd(lbbx + cj1, lb0 * ya_ * zb_);
        atomicAdd(lbbx + ck1, lb0 * yb_ * za_); atomicAdd(lbbx + cj1 + 1, lb0 * ya_ * za_);
        atomicAdd(lbby + c, lb1 * xb_ * zb_); atomicAdd(lbby + ci1, lb1 * xa_ * zb_);
        atomicAdd(lbby + ck1, lb1 * xb_ * za_); atomicAdd(lbby + ci1 + 1, lb1 * xa_ * za_);
        atomicAdd(lbbz + c, lb2 * xb_ * yb_); atomicAdd(lbbz + ci1, lb2 * xa_ * yb_);
        atomicAdd(lbbz + cj1, lb2 * xb_ * ya_); atomicAdd(lbbz + ci1 + g.nz, lb2 * xa_ * ya_);
    }
    lam.a[0][s] = gA[0] + gD[0];
    lam.a[1][s] = gA[1] + gD[1];
    lam.a[2][s] = gA[2] + gD[2];
    lam.a[3][s] = gC[0];
    lam.a[4][s] = gC[1];
    lam.a[5][s] = gC[2];
    lam.a[6][s] = gA[6] + lqo;
}

// Zero the adjoint of components that init_boundaries set to zero
// (FDTD, maxwell.cpp:532-597).
__global__ void k_zero_mask(Grid g, double* l6) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= g.nc) return;
    const int k = x % g.nz, j = (x / g.nz) % g.ny, i = x / g.nynz;
    const size_t nc = (size_t)g.nc;
    auto z = [&](int comp) { l6[comp * nc + x] = 0.0; };
    const bool jin = j < g.ny - 1, kin = k < g.nz - 1, iin = i < g.nx - 1;
    if (i == 0 && jin && kin) { z(1); z(2); z(3); }
    if (i == g.nx - 1 && jin && kin) for (int c = 0; c < 6; c++) z(c);
    if (j == 0 && iin && kin) { z(0); z(2); z(4); }
    if (j == g.ny - 1 && iin && kin) for (int c = 0; c < 6; c++) z(c);
    if (k == 0 && iin && jin) { z(1); z(0); z(5); }
    if (k == g.nz - 1 && iin && jin) for (int c = 0; c < 6; c++) z(c);
}

// Device memory of one adjoint run, released on every return path.
struct Workspace {
    std::vector<void*> owned;
    std::vector<State::Snap> ck;
    ~Workspace() {
        for (void* p : owned) cudaFree(p);
        for (auto& c : ck) snapshot_free(c);
    }
    template <typename T>
    cudaError_t alloc(T** p, size_t count) {
        void* v = nullptr;
        const cudaError_t e = cudaMalloc(&v, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) owned.push_back(v);
        *p = (T*)v;
        return e;
    }
    void release(void* p) {
        for (auto& q : owned)
            if (q == p) { cudaFree(q); q = nullptr; }
    }
};

// Per-step record of a checkpoint segment's forward re-run.
struct StepRec {
    int n = 0, n_next = 0;
    Lam7 in;                   // particle inputs in traversal order
    double* fields = nullptr;  // E (3 planes) and Bbar (3 planes) at the step's start
    int32_t* perm = nullptr;   // traversal order after the step's rebin
};

PStore64 cur_store(Species& sp) {
    PStore64 st;
    double** ps[9] = {&st.x, &st.y, &st.z, &st.ux, &st.uy, &st.uz, &st.g, &st.q, &st.chi};
    for (int a = 0; a < 9; a++) *ps[a] = (double*)sp.buf[sp.cur][a];
    return st;
}

PStore32 cur_store32(Species& sp) {
    PStore32 st;
    st.cell = (int32_t*)sp.buf[sp.cur][0];
    float** ps[9] = {&st.ox, &st.oy, &st.oz, &st.ux, &st.uy, &st.uz, &st.g, &st.q, &st.chi};
    for (int a = 0; a < 9; a++) *ps[a] = (float*)sp.buf[sp.cur][1 + a];
    return st;
}

inline int nblk(size_t n, int b) { return (int)((n + b - 1) / b); }

// The step's particle inputs in traversal order, FP64, from either store.
void record_inputs(State& s, Species& sp, int n, Lam7 rec, double* g_out) {
    if (n <= 0) return;
    if (s.fp64) k_record<<<nblk(n, 256), 256, 0, s.stream>>>(cur_store(sp), sp.perm, n, rec, g_out);
    else k_record32<<<nblk(n, 256), 256, 0, s.stream>>>(s.grid, cur_store32(sp), sp.perm, n, rec, g_out);
}

// E (planes 0..2) and Bbar (9..11) at the step's start, FP64.
cudaError_t record_fields(State& s, double* out) {
    const size_t nc = (size_t)s.grid.nc;
    const int src[6] = {0, 1, 2, 9, 10, 11};
    for (int a = 0; a < 6; a++) {
        if (s.fp64) {
            const cudaError_t e = cudaMemcpyAsync(out + a * nc, s.plane[src[a]], nc * 8, cudaMemcpyDeviceToDevice,
                                                  s.stream);
            if (e != cudaSuccess) return e;
        } else {
            k_widen<<<nblk(nc, 256), 256, 0, s.stream>>>((const float*)s.plane[src[a]], out + a * nc, nc);
        }
    }
    return cudaGetLastError();
}

}  // namespace

int adjoint_energy(State& s, qp_handle* h, int nsteps, int every, double ext_bz, double* grad6, double* grad_q,
                   double* loss_out) {
    const qp_params& P = s.prm;
    if (P.solver != QP_SOLVER_FDTD || P.pusher != QP_PUSHER_BORIS || P.qed || s.sp.size() != 1 || s.sp[0].cmr != -1) {
        s.err = "the adjoint covers FDTD, Boris, QED off and one electron species";
        return QP_ERR_CONFIG;
    }
    if (!s.boundaries_done) { s.err = "qp_init_boundaries has not run"; return QP_ERR_STATE; }
    if (s.diag_lo != 0 || s.diag_hi != s.grid.nx) { s.err = "the adjoint needs the full diagnostic range"; return QP_ERR_STATE; }
    if (nsteps < 1 || every < 1) { s.err = "nsteps and the checkpoint interval must be positive"; return QP_ERR_ARG; }
    const Grid g = s.grid;
    const size_t nc = (size_t)g.nc;
    const double PI = 3.141592653589793;
    // compute_energy's electron normalisation (main.cpp:2326-2327)
    const double bE = 8.2e-14 * P.dx * P.dy * P.dz * 1.11485e13 * P.lambda_cm / (8 * PI * PI * PI);
    Species& sp = s.sp[0];
    const int n0 = (int)sp.n;
    Workspace w;
    int r;
    // forward pass, state saved at the start of every segment
    w.ck.resize((nsteps + every - 1) / every);
    qp_diag last{};
    for (int l = 0; l < nsteps; l++) {
        if (l % every == 0 && (r = snapshot_take(s, w.ck[l / every])) != QP_OK) return r;
        if ((r = qp_step(h, 1, ext_bz, &last)) != QP_OK) return r;
    }
    if (loss_out) *loss_out = last.energy_e;
    double *lE6, *lEt, *lB1, *lJ, *lBb;
    QP_CUDA_CHECK(s, w.alloc(&lE6, 6 * nc));  // lE (planes 0..2), lB (3..5)
    QP_CUDA_CHECK(s, w.alloc(&lEt, 3 * nc));
    QP_CUDA_CHECK(s, w.alloc(&lB1, 3 * nc));
    QP_CUDA_CHECK(s, w.alloc(&lJ, 3 * nc));
    QP_CUDA_CHECK(s, w.alloc(&lBb, 3 * nc));
    QP_CUDA_CHECK(s, cudaMemsetAsync(lE6, 0, 6 * nc * 8, s.stream));
    const size_t cap = (size_t)sp.cap;
    Lam7 la, lb;
    for (int a = 0; a < 7; a++) {
        QP_CUDA_CHECK(s, w.alloc(&la.a[a], cap));
        QP_CUDA_CHECK(s, w.alloc(&lb.a[a], cap));
    }
    // seed: adjoint of the final particles
    {
        const int n = (int)sp.n;
        Lam7 rec;
        double* gam;
        for (int a = 0; a < 7; a++) QP_CUDA_CHECK(s, w.alloc(&rec.a[a], n));
        QP_CUDA_CHECK(s, w.alloc(&gam, n));
        if (n > 0) {
            record_inputs(s, sp, n, rec, gam);
            k_loss_seed<<<nblk(n, 256), 256, 0, s.stream>>>(rec, gam, n, bE, la);
        }
        QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
        for (int a = 0; a < 7; a++) w.release(rec.a[a]);
        w.release(gam);
    }
    const SolverCoef C = solver_coef(P);
    PushArgs pa{};
    pa.cmr = -1.0; pa.dt = P.dt; pa.dx = P.dx; pa.dy = P.dy; pa.dz = P.dz; pa.ext_bz = ext_bz;
    pa.n = 0; pa.sp = 0; pa.kind = KIND_LEPTON; pa.status = s.d_status; pa.diag = s.d_diag;
    pa.track = 0;
    pa.step = 0;
    pa.cat = nullptr;
    pa.dcat = nullptr;
    pa.trn_src = nullptr;
    pa.trn_dst = nullptr;
    pa.dlo = 0; pa.dhi = s.grid.nx;
    const int nbc = nblk(nc, 256);
    double* lE = lE6;
    double* lB = lE6 + 3 * nc;
    for (int seg = (int)w.ck.size() - 1; seg >= 0; seg--) {
        // re-run the segment from its checkpoint, recording every step
        if ((r = snapshot_restore(s, w.ck[seg])) != QP_OK) return r;
        const int l0 = seg * every, l1 = std::min(nsteps, l0 + every);
        std::vector<StepRec> recs(l1 - l0);
        for (int l = l0; l < l1; l++) {
            StepRec& R = recs[l - l0];
            R.n = (int)sp.n;
            for (int a = 0; a < 7; a++) QP_CUDA_CHECK(s, w.alloc(&R.in.a[a], R.n));
            record_inputs(s, sp, R.n, R.in, nullptr);
            QP_CUDA_CHECK(s, w.alloc(&R.fields, 6 * nc));
            QP_CUDA_CHECK(s, record_fields(s, R.fields));
            if ((r = qp_step(h, 1, ext_bz, nullptr)) != QP_OK) return r;
            R.n_next = (int)sp.n;
            QP_CUDA_CHECK(s, w.alloc(&R.perm, R.n_next));
            if (R.n_next > 0)
                QP_CUDA_CHECK(s, cudaMemcpyAsync(R.perm, sp.perm, (size_t)R.n_next * 4, cudaMemcpyDeviceToDevice, s.stream));
        }
        // sweep the segment backwards
        for (int l = l1 - 1; l >= l0; l--) {
            StepRec& R = recs[l - l0];
            // fields: B' = B1 + 1/2 Cb E',  E' = E + Ce B1 - dx J,  B1 = B + 1/2 Cb E
            QP_CUDA_CHECK(s, cudaMemcpyAsync(lEt, lE, 3 * nc * 8, cudaMemcpyDeviceToDevice, s.stream));
            k_cbT<<<nbc, 256, 0, s.stream>>>(g, C.dtdx, C.dtdy, C.dtdz, lB, lB + nc, lB + 2 * nc, lEt, lEt + nc,
                                            lEt + 2 * nc);
            QP_CUDA_CHECK(s, cudaMemcpyAsync(lB1, lB, 3 * nc * 8, cudaMemcpyDeviceToDevice, s.stream));
            k_ceT<<<nbc, 256, 0, s.stream>>>(g, C.dtdx, C.dtdy, C.dtdz, P.dx, P.dy, P.dz, lEt, lEt + nc, lEt + 2 * nc,
                                            lB1, lB1 + nc, lB1 + 2 * nc, lJ, lJ + nc, lJ + 2 * nc);
            QP_CUDA_CHECK(s, cudaMemcpyAsync(lE, lEt, 3 * nc * 8, cudaMemcpyDeviceToDevice, s.stream));
            k_cbT<<<nbc, 256, 0, s.stream>>>(g, C.dtdx, C.dtdy, C.dtdz, lB1, lB1 + nc, lB1 + 2 * nc, lE, lE + nc,
                                            lE + 2 * nc);
            QP_CUDA_CHECK(s, cudaMemcpyAsync(lB, lB1, 3 * nc * 8, cudaMemcpyDeviceToDevice, s.stream));
            // particles: adjoints through the rebin, then through the push
            for (int a = 0; a < 7; a++)
                QP_CUDA_CHECK(s, cudaMemsetAsync(lb.a[a], 0, std::max<size_t>(R.n, 1) * 8, s.stream));
            if (R.n_next > 0) k_map<<<nblk(R.n_next, 256), 256, 0, s.stream>>>(R.perm, R.n_next, la, lb);
            QP_CUDA_CHECK(s, cudaMemsetAsync(lBb, 0, 3 * nc * 8, s.stream));
            Fields<double> f;
            f.ex = R.fields; f.ey = R.fields + nc; f.ez = R.fields + 2 * nc;
            f.bex = R.fields + 3 * nc; f.bey = R.fields + 4 * nc; f.bez = R.fields + 5 * nc;
            f.bx = f.by = f.bz = nullptr;
            f.jx = f.jy = f.jz = nullptr;
            if (R.n > 0)
                k_adj_particles<<<nblk(R.n, 128), 128, 0, s.stream>>>(f, g, R.in, R.n, pa, lJ, lJ + nc, lJ + 2 * nc, lb,
                                                                    lE, lE + nc, lE + 2 * nc, lBb, lBb + nc,
                                                                    lBb + 2 * nc);
            k_avgT<<<nbc, 256, 0, s.stream>>>(g, lBb, lBb + nc, lBb + 2 * nc, lB, lB + nc, lB + 2 * nc);
            std::swap(la, lb);
            QP_CUDA_CHECK(s, cudaGetLastError());
            QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
            for (int a = 0; a < 7; a++) w.release(R.in.a[a]);
            w.release(R.fields);
            w.release(R.perm);
        }
    }
    // the loaded planes went through init_boundaries' zeroing
    k_zero_mask<<<nbc, 256, 0, s.stream>>>(g, lE6);
    QP_CUDA_CHECK(s, cudaGetLastError());
    if (grad6) QP_CUDA_CHECK(s, cudaMemcpyAsync(grad6, lE6, 6 * nc * 8, cudaMemcpyDefault, s.stream));
    if (grad_q && n0 > 0)
        QP_CUDA_CHECK(s, cudaMemcpyAsync(grad_q, la.a[6], (size_t)n0 * 8, cudaMemcpyDefault, s.stream));
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    unsigned int st = 0;
    QP_CUDA_CHECK(s, cudaMemcpy(&st, s.d_status, sizeof st, cudaMemcpyDeviceToHost));
    // leave the region in its initial state
    if ((r = snapshot_restore(s, w.ck[0])) != QP_OK) return r;
    if (st & ST_BOUNDS) { s.err = "a deposition target left the grid in the adjoint"; return QP_ERR_CONFIG; }
    return QP_OK;
}

}  // namespace qp

extern "C" int qp_adjoint_energy(qp_handle* h, int nsteps, int every, double external_bz, double* grad_fields,
                                 double* grad_q, double* loss) {
    if (!h) return QP_ERR_ARG;
    qp::State& s = *qp::state_of(h);
    const cudaError_t e = cudaSetDevice(s.prm.device);
    if (e != cudaSuccess) { s.err = cudaGetErrorString(e); return QP_ERR_CUDA; }
    return qp::adjoint_energy(s, h, nsteps, every, external_bz, grad_fields, grad_q, loss);
}
