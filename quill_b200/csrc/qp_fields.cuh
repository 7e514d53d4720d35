// Maxwell stencils and the B -> E-position average, per cell, templated on the
// real type.  Each function updates the components of one cell that the
// reference updates in the given sub-step, with the reference's update ranges
// and face special cases (maxwell.cpp, advance.cpp:20-83).  All reads of a
// sub-step are of the other field (B reads E, E reads B and J), so in-place
// per-cell updates reproduce the reference's sequential sweeps exactly.
#pragma once

#include "qp_physics.cuh"

namespace qp {

struct SolverCoef {
    double dtdx, dtdy, dtdz, dx, dy, dz;
    // five-point a, b per axis (maxwell.cpp:24-33)
    double fax, fay, faz, fbx, fby, fbz;
    // NDFX a, b per axis (maxwell.cpp:238-249)
    double nax, nay, naz, nbx, nby, nbz;
};

// Coefficients of the three solvers for a parameter set (qp_api.cu).
SolverCoef solver_coef(const qp_params& p);

template <typename T>
struct Coef {
    T dtdx, dtdy, dtdz, dx, dy, dz;
    T fax, fay, faz, fbx, fby, fbz;
    T nax, nay, naz, nbx, nby, nbz;
    __host__ __device__ Coef() {}
    __host__ Coef(const SolverCoef& c)
        : dtdx(T(c.dtdx)), dtdy(T(c.dtdy)), dtdz(T(c.dtdz)), dx(T(c.dx)), dy(T(c.dy)), dz(T(c.dz)),
          fax(T(c.fax)), fay(T(c.fay)), faz(T(c.faz)), fbx(T(c.fbx)), fby(T(c.fby)), fbz(T(c.fbz)),
          nax(T(c.nax)), nay(T(c.nay)), naz(T(c.naz)), nbx(T(c.nbx)), nby(T(c.nby)), nbz(T(c.nbz)) {}
};

#define QP_IN(v, lo, hi) ((v) >= (lo) && (v) < (hi))

// ---------------------------------------------------------------- FDTD ----
// maxwell.cpp:445-522.  B: [1, n-1)^3 plus the i/j/k = 0 faces for the
// components tangential to them; E: same ranges.
template <typename T>
__device__ __forceinline__ void fdtd_b(const Fields<T>& f, const Grid& g, const Coef<T>& c, int i, int j, int k) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool in_i = QP_IN(i, 1, nx - 1), in_j = QP_IN(j, 1, ny - 1), in_k = QP_IN(k, 1, nz - 1);
    const int x = cidx(g, i, j, k);
    const int xi = x + g.nynz, xj = x + nz, xk = x + 1;
    // bx: main, j = 0 face, k = 0 face
    if (in_i && ((in_j && in_k) || (j == 0 && in_k) || (k == 0 && in_j)))
        f.bx[x] += T(0.5) * (-c.dtdy * (f.ez[xj] - f.ez[x]) + c.dtdz * (f.ey[xk] - f.ey[x]));
    // by: main, i = 0 face, k = 0 face
    if (in_j && ((in_i && in_k) || (i == 0 && in_k) || (k == 0 && in_i)))
        f.by[x] += T(0.5) * (c.dtdx * (f.ez[xi] - f.ez[x]) - c.dtdz * (f.ex[xk] - f.ex[x]));
    // bz: main, i = 0 face, j = 0 face
    if (in_k && ((in_i && in_j) || (i == 0 && in_j) || (j == 0 && in_i)))
        f.bz[x] += T(0.5) * (c.dtdy * (f.ex[xj] - f.ex[x]) - c.dtdx * (f.ey[xi] - f.ey[x]));
}

template <typename T>
__device__ __forceinline__ void fdtd_e(const Fields<T>& f, const Grid& g, const Coef<T>& c, int i, int j, int k) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool in_i = QP_IN(i, 1, nx - 1), in_j = QP_IN(j, 1, ny - 1), in_k = QP_IN(k, 1, nz - 1);
    const int x = cidx(g, i, j, k);
    const int xi = x - g.nynz, xj = x - nz, xk = x - 1;
    if (in_j && in_k && (in_i || i == 0))
        f.ex[x] += c.dtdy * (f.bz[x] - f.bz[xj]) - c.dtdz * (f.by[x] - f.by[xk]) - f.jx[x] * c.dx;
    if (in_i && in_k && (in_j || j == 0))
        f.ey[x] += -c.dtdx * (f.bz[x] - f.bz[xi]) + c.dtdz * (f.bx[x] - f.bx[xk]) - f.jy[x] * c.dy;
    if (in_i && in_j && (in_k || k == 0))
        f.ez[x] += c.dtdx * (f.by[x] - f.by[xi]) - c.dtdy * (f.bx[x] - f.bx[xj]) - f.jz[x] * c.dz;
}

// fdtd_b / fdtd_e for CPT consecutive interior cells (i0 .. i0+CPT-1, j, k
// all in the main region): the E (B) values the i-difference reads are
// loaded once per plane and shared by neighbouring cells; each update is the
// main-region formula in the same operation order.  es (PHASE 4 of k_field)
// receives E^2 + B^2 of the cells with i in [dlo, dhi) before the update.
template <typename T, int CPT, bool ENERGY>
__device__ __forceinline__ void fdtd_b_run(const Fields<T>& f, const Grid& g, const Coef<T>& c, int i0, int j, int k,
                                           int dlo, int dhi, double& es) {
    const int I = g.nynz, J = g.nz;
    const int x0 = cidx(g, i0, j, k);
    T ey_[CPT + 1], ez_[CPT + 1];
#pragma unroll
    for (int p = 0; p <= CPT; p++) {
        ey_[p] = f.ey[x0 + p * I];
        ez_[p] = f.ez[x0 + p * I];
    }
#pragma unroll
    for (int u = 0; u < CPT; u++) {
        const int x = x0 + u * I;
        const T ex = f.ex[x], exj = f.ex[x + J], exk = f.ex[x + 1], eyk = f.ey[x + 1], ezj = f.ez[x + J];
        const T bx = f.bx[x], by = f.by[x], bz = f.bz[x];
        if (ENERGY && i0 + u >= dlo && i0 + u < dhi) {
            const double a = ex, b = ey_[u], d = ez_[u], e = bx, h = by, m = bz;
            es += a * a + b * b + d * d + e * e + h * h + m * m;
        }
        f.bx[x] = bx + T(0.5) * (-c.dtdy * (ezj - ez_[u]) + c.dtdz * (eyk - ey_[u]));
        f.by[x] = by + T(0.5) * (c.dtdx * (ez_[u + 1] - ez_[u]) - c.dtdz * (exk - ex));
        f.bz[x] = bz + T(0.5) * (c.dtdy * (exj - ex) - c.dtdx * (ey_[u + 1] - ey_[u]));
    }
}

template <typename T, int CPT>
__device__ __forceinline__ void fdtd_e_run(const Fields<T>& f, const Grid& g, const Coef<T>& c, int i0, int j, int k) {
    const int I = g.nynz, J = g.nz;
    const int x0 = cidx(g, i0, j, k);
    T by_[CPT + 1], bz_[CPT + 1];  // planes i0-1 .. i0+CPT-1
#pragma unroll
    for (int p = 0; p <= CPT; p++) {
        by_[p] = f.by[x0 + (p - 1) * I];
        bz_[p] = f.bz[x0 + (p - 1) * I];
    }
#pragma unroll
    for (int u = 0; u < CPT; u++) {
        const int x = x0 + u * I;
        const T bx = f.bx[x], bxj = f.bx[x - J], bxk = f.bx[x - 1], byk = f.by[x - 1], bzj = f.bz[x - J];
        f.ex[x] = f.ex[x] + (c.dtdy * (bz_[u + 1] - bzj) - c.dtdz * (by_[u + 1] - byk) - f.jx[x] * c.dx);
        f.ey[x] = f.ey[x] + (-c.dtdx * (bz_[u + 1] - bz_[u]) + c.dtdz * (bx - bxk) - f.jy[x] * c.dy);
        f.ez[x] = f.ez[x] + (c.dtdx * (by_[u + 1] - by_[u]) - c.dtdy * (bx - bxj) - f.jz[x] * c.dz);
    }
}

// ---------------------------------------------------------------- NDFX ----
// maxwell.cpp:251-328.  B and E: [2, n-1)^3 plus the i/j/k = 1 planes for the
// components tangential to them.
template <typename T>
__device__ __forceinline__ void ndfx_b(const Fields<T>& f, const Grid& g, const Coef<T>& c, int i, int j, int k) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool in_i = QP_IN(i, 2, nx - 1), in_j = QP_IN(j, 2, ny - 1), in_k = QP_IN(k, 2, nz - 1);
    const int x = cidx(g, i, j, k);
    const int I = g.nynz, J = nz;
    if (in_i && ((in_j && in_k) || (j == 1 && in_k) || (k == 1 && in_j)))
        f.bx[x] += T(0.5) * (-c.dtdy * (c.nbz * (f.ez[x + J] - f.ez[x]) + c.naz * (f.ez[x + J + 1] - f.ez[x + 1] + f.ez[x + J - 1] - f.ez[x - 1])) +
                             c.dtdz * (c.nby * (f.ey[x + 1] - f.ey[x]) + c.nay * (f.ey[x + J + 1] - f.ey[x + J] + f.ey[x - J + 1] - f.ey[x - J])));
    if (in_j && ((in_i && in_k) || (i == 1 && in_k) || (k == 1 && in_i)))
        f.by[x] += T(0.5) * (c.dtdx * (c.nbz * (f.ez[x + I] - f.ez[x]) + c.naz * (f.ez[x + I + 1] - f.ez[x + 1] + f.ez[x + I - 1] - f.ez[x - 1])) -
                             c.dtdz * (c.nbx * (f.ex[x + 1] - f.ex[x]) + c.nax * (f.ex[x + I + 1] - f.ex[x + I] + f.ex[x - I + 1] - f.ex[x - I])));
    if (in_k && ((in_i && in_j) || (i == 1 && in_j) || (j == 1 && in_i)))
        f.bz[x] += T(0.5) * (c.dtdy * (c.nbx * (f.ex[x + J] - f.ex[x]) + c.nax * (f.ex[x + I + J] - f.ex[x + I] + f.ex[x - I + J] - f.ex[x - I])) -
                             c.dtdx * (c.nby * (f.ey[x + I] - f.ey[x]) + c.nay * (f.ey[x + I + J] - f.ey[x + J] + f.ey[x + I - J] - f.ey[x - J])));
}

template <typename T>
__device__ __forceinline__ void ndfx_e(const Fields<T>& f, const Grid& g, const Coef<T>& c, int i, int j, int k) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool in_i = QP_IN(i, 2, nx - 1), in_j = QP_IN(j, 2, ny - 1), in_k = QP_IN(k, 2, nz - 1);
    const int x = cidx(g, i, j, k);
    const int I = g.nynz, J = nz;
    if (in_j && in_k && (in_i || i == 1))
        f.ex[x] = f.ex[x] + c.dtdy * (c.nbz * (f.bz[x] - f.bz[x - J]) + c.naz * (f.bz[x + 1] - f.bz[x - J + 1] + f.bz[x - 1] - f.bz[x - J - 1])) -
                  c.dtdz * (c.nby * (f.by[x] - f.by[x - 1]) + c.nay * (f.by[x + J] - f.by[x + J - 1] + f.by[x - J] - f.by[x - J - 1])) -
                  f.jx[x] * c.dx;
    if (in_i && in_k && (in_j || j == 1))
        f.ey[x] = f.ey[x] - c.dtdx * (c.nbz * (f.bz[x] - f.bz[x - I]) + c.naz * (f.bz[x + 1] - f.bz[x - I + 1] + f.bz[x - 1] - f.bz[x - I - 1])) +
                  c.dtdz * (c.nbx * (f.bx[x] - f.bx[x - 1]) + c.nax * (f.bx[x + I] - f.bx[x + I - 1] + f.bx[x - I] - f.bx[x - I - 1])) -
                  f.jy[x] * c.dy;
    if (in_i && in_j && (in_k || k == 1))
        f.ez[x] = f.ez[x] + c.dtdx * (c.nby * (f.by[x] - f.by[x - I]) + c.nay * (f.by[x + J] - f.by[x - I + J] + f.by[x - J] - f.by[x - I - J])) -
                  c.dtdy * (c.nbx * (f.bx[x] - f.bx[x - J]) + c.nax * (f.bx[x + I] - f.bx[x + I - J] + f.bx[x - I] - f.bx[x - I - J])) -
                  f.jz[x] * c.dz;
}

// ---------------------------------------------------------- five-point ----
// maxwell.cpp:35-125.  B: [1, n-2)^3 plus the high faces (i = nx-1, ...)
// where the derivative normal to the face uses a truncated stencil; E:
// [2, n-2)^3 plus the i/j/k = 1 planes.
template <typename T>
__device__ __forceinline__ T fp_d(T b, T a, T p2, T p1, T p0, T m1) {
    return b * (p1 - p0) + a * (p2 - p1 + p0 - m1);
}
template <typename T>
__device__ __forceinline__ T fp_dface(T b, T a, T p0, T m1) {
    return b * (-p0) + a * (p0 - m1);
}

template <typename T>
__device__ __forceinline__ void fp_b(const Fields<T>& f, const Grid& g, const Coef<T>& c, int i, int j, int k) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool in_i = QP_IN(i, 1, nx - 2), in_j = QP_IN(j, 1, ny - 2), in_k = QP_IN(k, 1, nz - 2);
    const bool fi = (i == nx - 1), fj = (j == ny - 1), fk = (k == nz - 1);
    // regions: main, i-face (j,k inner), j-face (i,k inner), k-face (i,j inner)
    const bool main_ = in_i && in_j && in_k;
    const bool face_i = fi && in_j && in_k;
    const bool face_j = fj && in_i && in_k;
    const bool face_k = fk && in_i && in_j;
    if (!(main_ || face_i || face_j || face_k)) return;
    const int x = cidx(g, i, j, k);
    const int I = g.nynz, J = nz;
    {   // bx: y-derivative of ez truncated on the j-face, z-derivative of ey on the k-face
        T dy_ = face_j ? fp_dface(c.fby, c.fay, f.ez[x], f.ez[x - J])
                       : fp_d(c.fby, c.fay, f.ez[x + 2 * J], f.ez[x + J], f.ez[x], f.ez[x - J]);
        T dz_ = face_k ? fp_dface(c.fbz, c.faz, f.ey[x], f.ey[x - 1])
                       : fp_d(c.fbz, c.faz, f.ey[x + 2], f.ey[x + 1], f.ey[x], f.ey[x - 1]);
        f.bx[x] += T(0.5) * (-c.dtdy * dy_ + c.dtdz * dz_);
    }
    {   // by
        T dx_ = face_i ? fp_dface(c.fbx, c.fax, f.ez[x], f.ez[x - I])
                       : fp_d(c.fbx, c.fax, f.ez[x + 2 * I], f.ez[x + I], f.ez[x], f.ez[x - I]);
        T dz_ = face_k ? fp_dface(c.fbz, c.faz, f.ex[x], f.ex[x - 1])
                       : fp_d(c.fbz, c.faz, f.ex[x + 2], f.ex[x + 1], f.ex[x], f.ex[x - 1]);
        f.by[x] += T(0.5) * (c.dtdx * dx_ - c.dtdz * dz_);
    }
    {   // bz
        T dy_ = face_j ? fp_dface(c.fby, c.fay, f.ex[x], f.ex[x - J])
                       : fp_d(c.fby, c.fay, f.ex[x + 2 * J], f.ex[x + J], f.ex[x], f.ex[x - J]);
        T dx_ = face_i ? fp_dface(c.fbx, c.fax, f.ey[x], f.ey[x - I])
                       : fp_d(c.fbx, c.fax, f.ey[x + 2 * I], f.ey[x + I], f.ey[x], f.ey[x - I]);
        f.bz[x] += T(0.5) * (c.dtdy * dy_ - c.dtdx * dx_);
    }
}

template <typename T>
__device__ __forceinline__ void fp_e(const Fields<T>& f, const Grid& g, const Coef<T>& c, int i, int j, int k) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool in_i = QP_IN(i, 2, nx - 2), in_j = QP_IN(j, 2, ny - 2), in_k = QP_IN(k, 2, nz - 2);
    const int x = cidx(g, i, j, k);
    const int I = g.nynz, J = nz;
    if (in_j && in_k && (in_i || i == 1))
        f.ex[x] = f.ex[x] + c.dtdy * (c.fby * (f.bz[x] - f.bz[x - J]) + c.fay * (f.bz[x + J] - f.bz[x] + f.bz[x - J] - f.bz[x - 2 * J])) -
                  c.dtdz * (c.fbz * (f.by[x] - f.by[x - 1]) + c.faz * (f.by[x + 1] - f.by[x] + f.by[x - 1] - f.by[x - 2])) -
                  f.jx[x] * c.dx;
    if (in_i && in_k && (in_j || j == 1))
        f.ey[x] = f.ey[x] - c.dtdx * (c.fbx * (f.bz[x] - f.bz[x - I]) + c.fax * (f.bz[x + I] - f.bz[x] + f.bz[x - I] - f.bz[x - 2 * I])) +
                  c.dtdz * (c.fbz * (f.bx[x] - f.bx[x - 1]) + c.faz * (f.bx[x + 1] - f.bx[x] + f.bx[x - 1] - f.bx[x - 2])) -
                  f.jy[x] * c.dy;
    if (in_i && in_j && (in_k || k == 1))
        f.ez[x] = f.ez[x] + c.dtdx * (c.fbx * (f.by[x] - f.by[x - I]) + c.fax * (f.by[x + I] - f.by[x] + f.by[x - I] - f.by[x - 2 * I])) -
                  c.dtdy * (c.fby * (f.bx[x] - f.bx[x - J]) + c.fay * (f.bx[x + J] - f.bx[x] + f.bx[x - J] - f.bx[x - 2 * J])) -
                  f.jz[x] * c.dz;
}

// ------------------------------------------------------- B at E points ----
// advance.cpp:20-83: 8-point average inside, 4-point on the six faces for
// the components whose stencil leaves the box there; edges keep their value.
template <typename T>
__device__ __forceinline__ void bbar(const Fields<T>& f, const Grid& g, int i, int j, int k) {
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const bool in_i = QP_IN(i, 1, nx - 1), in_j = QP_IN(j, 1, ny - 1), in_k = QP_IN(k, 1, nz - 1);
    const bool main_ = in_i && in_j && in_k;
    const bool i0 = i == 0 && in_j && in_k, i1 = i == nx - 1 && in_j && in_k;
    const bool j0 = j == 0 && in_i && in_k, j1 = j == ny - 1 && in_i && in_k;
    const bool k0 = k == 0 && in_i && in_j, k1 = k == nz - 1 && in_i && in_j;
    if (!(main_ || i0 || i1 || j0 || j1 || k0 || k1)) return;
    const int x = cidx(g, i, j, k);
    const int I = g.nynz, J = nz;
    const T* bx = f.bx;
    const T* by = f.by;
    const T* bz = f.bz;
    // bex: 4-point on i = nx-1, j = 0, k = 0
    if (i1) f.bex[x] = T(0.25) * (bx[x] + bx[x - 1] + bx[x - J] + bx[x - J - 1]);
    else if (j0) f.bex[x] = T(0.25) * (bx[x] + bx[x + I] + bx[x - 1] + bx[x + I - 1]);
    else if (k0) f.bex[x] = T(0.25) * (bx[x] + bx[x + I] + bx[x - J] + bx[x + I - J]);
    else f.bex[x] = T(0.125) * (bx[x] + bx[x + I] + bx[x - 1] + bx[x + I - 1] + bx[x - J] + bx[x + I - J] + bx[x - J - 1] + bx[x + I - J - 1]);
    // bey: 4-point on i = 0, j = ny-1, k = 0
    if (i0) f.bey[x] = T(0.25) * (by[x] + by[x - 1] + by[x + J] + by[x + J - 1]);
    else if (j1) f.bey[x] = T(0.25) * (by[x] + by[x - I] + by[x - 1] + by[x - I - 1]);
    else if (k0) f.bey[x] = T(0.25) * (by[x] + by[x - I] + by[x + J] + by[x - I + J]);
    else f.bey[x] = T(0.125) * (by[x] + by[x - I] + by[x - 1] + by[x - I - 1] + by[x + J] + by[x - I + J] + by[x + J - 1] + by[x - I + J - 1]);
    // bez: 4-point on i = 0, j = 0, k = nz-1
    if (i0) f.bez[x] = T(0.25) * (bz[x] + bz[x + 1] + bz[x - J] + bz[x - J + 1]);
    else if (j0) f.bez[x] = T(0.25) * (bz[x] + bz[x - I] + bz[x + 1] + bz[x - I + 1]);
    else if (k1) f.bez[x] = T(0.25) * (bz[x] + bz[x - I] + bz[x - J] + bz[x - I - J]);
    else f.bez[x] = T(0.125) * (bz[x] + bz[x - I] + bz[x + 1] + bz[x - I + 1] + bz[x - J] + bz[x - I - J] + bz[x - J + 1] + bz[x - I - J + 1]);
}

// bbar for CPT consecutive interior cells (i0 .. i0+CPT-1, j, k all in the
// main region): the B values of the CPT+1 planes each component's stencil
// spans are loaded once into registers and shared by neighbouring cells; the
// sums are bbar's 8-point sums in bbar's order.
template <typename T, int CPT>
__device__ __forceinline__ void bbar_run(const Fields<T>& f, const Grid& g, int i0, int j, int k) {
    const int I = g.nynz, J = g.nz;
    const int x0 = cidx(g, i0, j, k);
    T ax[CPT + 1][4], ay[CPT + 1][4], az[CPT + 1][4];
#pragma unroll
    for (int p = 0; p <= CPT; p++) {
        const int bx0 = x0 + p * I;        // bx: planes i0 .. i0+CPT
        ax[p][0] = f.bx[bx0]; ax[p][1] = f.bx[bx0 - 1]; ax[p][2] = f.bx[bx0 - J]; ax[p][3] = f.bx[bx0 - J - 1];
        const int b0 = x0 + (p - 1) * I;   // by, bz: planes i0-1 .. i0+CPT-1
        ay[p][0] = f.by[b0]; ay[p][1] = f.by[b0 - 1]; ay[p][2] = f.by[b0 + J]; ay[p][3] = f.by[b0 + J - 1];
        az[p][0] = f.bz[b0]; az[p][1] = f.bz[b0 + 1]; az[p][2] = f.bz[b0 - J]; az[p][3] = f.bz[b0 - J + 1];
    }
#pragma unroll
    for (int u = 0; u < CPT; u++) {
        const int x = x0 + u * I;
        f.bex[x] = T(0.125) * (ax[u][0] + ax[u + 1][0] + ax[u][1] + ax[u + 1][1] + ax[u][2] + ax[u + 1][2] +
                               ax[u][3] + ax[u + 1][3]);
        f.bey[x] = T(0.125) * (ay[u + 1][0] + ay[u][0] + ay[u + 1][1] + ay[u][1] + ay[u + 1][2] + ay[u][2] +
                               ay[u + 1][3] + ay[u][3]);
        f.bez[x] = T(0.125) * (az[u + 1][0] + az[u][0] + az[u + 1][1] + az[u][1] + az[u + 1][2] + az[u][2] +
                               az[u + 1][3] + az[u][3]);
    }
}

// init_boundaries (maxwell.cpp:135-236, 338-438, 532-597): components set to
// zero once on given planes over [0, n-1) of the two other axes.  comps is a
// bit mask over (ex ey ez bx by bz).
struct ZeroPlane {
    int axis, plane, comps;
};

}  // namespace qp
