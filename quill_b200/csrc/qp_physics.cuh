// Device arithmetic of QUILL's per-timestep loop, templated on the real type
// T (double for the FP64 path, float for the mixed path).
//
// Expression trees follow the reference operation by operation (same operand
// association) so that the FP64 instantiation, compiled with --fmad=false,
// performs the same IEEE operation sequence as the reference CPU build with
// -ffp-contract=off.  Citations are to the reference's source files.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "qp_internal.h"

namespace qp {

template <typename T>
__device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

__device__ __forceinline__ int cidx(const Grid& g, int i, int j, int k) {
    return (i * g.ny + j) * g.nz + k;
}

// ----------------------------------------------------------------------------
// Pushers (pusher.cpp)
// ----------------------------------------------------------------------------

// Vay (2008), pusher.cpp:5-42.  Uses the stored gamma g for the first
// rotation, so g must be consistent with u on entry.
template <typename T>
__device__ __forceinline__ void push_vay(T cmr, T& ux, T& uy, T& uz, T& g, const T E[3],
                                         const T B[3], T dt) {
    T t = dt * cmr;
    T ex = E[0] * t, ey = E[1] * t, ez = E[2] * t;
    t = T(0.5) * t;
    T bx = B[0] * t, by = B[1] * t, bz = B[2] * t;
    T wx = ux + ex + (uy * bz - uz * by) / g;
    T wy = uy + ey + (uz * bx - ux * bz) / g;
    T wz = uz + ez + (ux * by - uy * bx) / g;
    t = bx * bx + by * by + bz * bz;
    T bw = bx * wx + by * wy + bz * wz;
    T gg = T(1) + wx * wx + wy * wy + wz * wz - t;
    gg = sqrt(T(0.5) * (gg + sqrt(gg * gg + T(4) * (t + bw * bw))));
    t = T(1) / (T(1) + t / (gg * gg));
    bw = bw / (gg * gg);
    ux = (wx + (wy * bz - wz * by) / gg + bx * bw) * t;
    uy = (wy + (wz * bx - wx * bz) / gg + by * bw) * t;
    uz = (wz + (wx * by - wy * bx) / gg + bz * bw) * t;
    g = gg;
}

// Boris, pusher.cpp:44-97.
template <typename T>
__device__ __forceinline__ void push_boris(T cmr, T& ux, T& uy, T& uz, T& g, const T E[3],
                                           const T B[3], T dt) {
    T t = T(0.5) * dt * cmr;
    T ex = E[0] * t, ey = E[1] * t, ez = E[2] * t;
    T u1x = ux + ex, u1y = uy + ey, u1z = uz + ez;
    T gg = sqrt(T(1) + u1x * u1x + u1y * u1y + u1z * u1z);
    t /= gg;
    T bx = B[0] * t, by = B[1] * t, bz = B[2] * t;
    T wx = u1x + (u1y * bz - u1z * by);
    T wy = u1y + (u1z * bx - u1x * bz);
    T wz = u1z + (u1x * by - u1y * bx);
    t = T(2) / (T(1) + bx * bx + by * by + bz * bz);
    u1x += (wy * bz - wz * by) * t;
    u1y += (wz * bx - wx * bz) * t;
    u1z += (wx * by - wy * bx) * t;
    ux = u1x + ex;
    uy = u1y + ey;
    uz = u1z + ez;
    g = sqrt(T(1) + ux * ux + uy * uy + uz * uz);
}

template <int PUSHER, typename T>
__device__ __forceinline__ void push(T cmr, T& ux, T& uy, T& uz, T& g, const T E[3], const T B[3],
                                     T dt) {
    if (PUSHER == QP_PUSHER_VAY) push_vay(cmr, ux, uy, uz, g, E, B, dt);
    else push_boris(cmr, ux, uy, uz, g, E, B, dt);
}

// ----------------------------------------------------------------------------
// Field gather (deposition.cpp:431-471): Ex is interpolated in (y, z) at the
// particle's i, Ey in (x, z), Ez in (x, y); B the same on Bbar.
// (i, j, k) is the particle's cell, (xa, ya, za) its offset in the cell.
// ----------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void gather(const Fields<T>& f, const Grid& gr, int i, int j, int k, T xa,
                                       T ya, T za, T E[3], T B[3]) {
    const T xb = T(1) - xa, yb = T(1) - ya, zb = T(1) - za;
    const int c = cidx(gr, i, j, k);
    const int cj1 = c + gr.nz, ck1 = c + 1, ci1 = c + gr.nynz;
    E[0] = ld(f.ex + c) * yb * zb + ld(f.ex + cj1) * ya * zb + ld(f.ex + ck1) * yb * za + ld(f.ex + cj1 + 1) * ya * za;
    E[1] = ld(f.ey + c) * xb * zb + ld(f.ey + ci1) * xa * zb + ld(f.ey + ck1) * xb * za + ld(f.ey + ci1 + 1) * xa * za;
    E[2] = ld(f.ez + c) * xb * yb + ld(f.ez + ci1) * xa * yb + ld(f.ez + cj1) * xb * ya + ld(f.ez + ci1 + gr.nz) * xa * ya;
    B[0] = ld(f.bex + c) * yb * zb + ld(f.bex + cj1) * ya * zb + ld(f.bex + ck1) * yb * za + ld(f.bex + cj1 + 1) * ya * za;
    B[1] = ld(f.bey + c) * xb * zb + ld(f.bey + ci1) * xa * zb + ld(f.bey + ck1) * xb * za + ld(f.bey + ci1 + 1) * xa * za;
    B[2] = ld(f.bez + c) * xb * yb + ld(f.bez + ci1) * xa * yb + ld(f.bez + cj1) * xb * ya + ld(f.bez + ci1 + gr.nz) * xa * ya;
}

// ----------------------------------------------------------------------------
// Current deposition (deposition.cpp:13-356)
// ----------------------------------------------------------------------------

// Destination of the current contributions: J in HBM through atomics.
template <typename T>
struct GlobalSink {
    Fields<T> f;
    __device__ __forceinline__ void add(int comp, int, int, int, int c, T v) const {
        T* base = comp == 0 ? f.jx : (comp == 1 ? f.jy : f.jz);
        atomicAdd(base + c, v);
    }
};

// x / 3.  In FP64 by Markstein's correction of a reciprocal product
// (P. W. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Develop. 34(1), 1990): r = RN(1/3) is
// a third of an ulp from 1/3, so q = RN(x r) lies within one ulp of x / 3;
// the residual x - 3 q is exact in one FMA, and RN(q + r (x - 3 q)) is the
// correctly rounded quotient, i.e. what IEEE division returns (for results
// above the subnormal range; the sign of a zero is copied from x).  Three
// dependent operations instead of a full division.
__device__ __forceinline__ double div3(double x) {
    const double r = 0x1.5555555555555p-2;  // RN(1/3)
    const double q = x * r;
    return copysign(fma(fma(-q, 3.0, x), r, q), x);
}
template <typename T>
__device__ __forceinline__ T div3(T x) { return x / T(3); }

// x / y in FP64 for a divisor y > 0 fixed over a launch, given r = RN(1/y)
// (an IEEE division on the host): q0 = RN(x r) is within about 1.5 ulp of
// x / y, one FMA correction makes it faithful, and a second one gives the
// correctly rounded quotient (Markstein's theorem, as div3), i.e. the value
// of IEEE division, for results above the subnormal range.
__device__ __forceinline__ double div_fixed(double x, double y, double r) {
    const double q0 = x * r;
    const double q1 = fma(fma(-q0, y, x), r, q0);
    return copysign(fma(fma(-q1, y, x), r, q1), x);
}

// The 12 contributions of one segment from its start offsets in the cell
// (xa, ya, za) = p - w, its displacement d and charge q, with seg_dep's
// arithmetic and order; targets relative to the corner cell c: jx at
// c+nz+1, c+1, c+nz, c; jy at c+I+1, c+1, c+I, c; jz at c+I+nz, c+nz, c+I,
// c (I = ny*nz).
template <typename T>
__device__ __forceinline__ void seg_values_at(T xa, T ya, T za, const T d[3], T q, T v[12]) {
    const T xb = T(1) - xa, yb = T(1) - ya, zb = T(1) - za;
    const T dx = d[0], dy = d[1], dz = d[2];
    v[0] = dx * q * (ya * za + T(0.5) * (dz * ya + dy * za) + div3(dy * dz));
    v[1] = dx * q * (yb * za + T(0.5) * (dz * yb - dy * za) - div3(dy * dz));
    v[2] = dx * q * (ya * zb + T(0.5) * (-dz * ya + dy * zb) - div3(dy * dz));
    v[3] = dx * q * (yb * zb - T(0.5) * (dz * yb + dy * zb) + div3(dy * dz));
    v[4] = dy * q * (xa * za + T(0.5) * (dx * za + dz * xa) + div3(dx * dz));
    v[5] = dy * q * (xb * za + T(0.5) * (-dx * za + dz * xb) - div3(dx * dz));
    v[6] = dy * q * (xa * zb + T(0.5) * (dx * zb - dz * xa) - div3(dx * dz));
    v[7] = dy * q * (xb * zb - T(0.5) * (dx * zb + dz * xb) + div3(dx * dz));
    v[8] = dz * q * (xa * ya + T(0.5) * (dx * ya + dy * xa) + div3(dx * dy));
    v[9] = dz * q * (xb * ya + T(0.5) * (-dx * ya + dy * xb) - div3(dx * dy));
    v[10] = dz * q * (xa * yb + T(0.5) * (dx * yb - dy * xa) - div3(dx * dy));
    v[11] = dz * q * (xb * yb - T(0.5) * (dx * yb + dy * xb) + div3(dx * dy));
}

// The same in FP32 (mixed precision), factored: with A = ya + dy/2,
// B = za + dz/2 and c = dy dz / 12 the four jx terms are dx q (A B + c),
// dx q ((1 - A) B - c), dx q (A (1 - B) - c) and dx q ((1 - A)(1 - B) + c),
// equal to the expanded ones in exact arithmetic (likewise jy with x, z and
// jz with x, y), in about half the operations.  Their sum is dx q, as the
// expanded terms' is.
__device__ __forceinline__ void seg_values_at(float xa, float ya, float za, const float d[3], float q, float v[12]) {
    const float dx = d[0], dy = d[1], dz = d[2];
    const float ax = fmaf(0.5f, dx, xa), ay = fmaf(0.5f, dy, ya), az = fmaf(0.5f, dz, za);
    const float k12 = 1.0f / 12.0f;
    const float cx = dy * dz * k12, cy = dx * dz * k12, cz = dx * dy * k12;
    const float wx = dx * q, wy = dy * q, wz = dz * q;
    float ab = ay * az;
    v[0] = wx * (ab + cx);
    v[1] = wx * (az - ab - cx);
    v[2] = wx * (ay - ab - cx);
    v[3] = wx * (1.0f - ay - az + ab + cx);
    ab = ax * az;
    v[4] = wy * (ab + cy);
    v[5] = wy * (az - ab - cy);
    v[6] = wy * (ax - ab - cy);
    v[7] = wy * (1.0f - ax - az + ab + cy);
    ab = ax * ay;
    v[8] = wz * (ab + cz);
    v[9] = wz * (ay - ab - cz);
    v[10] = wz * (ax - ab - cz);
    v[11] = wz * (1.0f - ax - ay + ab + cz);
}

// 12 contributions of one straight segment d starting at p, lying in the cell
// with lower corner w (deposition.cpp:13-39).  p and w are in the particle's
// frame; the global cell of the corner is base + w.  Out-of-grid targets are
// skipped and flagged (cannot happen for dt < dx, dy, dz).
template <typename T, typename Sink>
__device__ __forceinline__ void seg_dep(const Sink& sink, const Grid& gr, const T p[3], const T d[3], T q,
                                        const int w[3], int bi, int bj, int bk, unsigned int* status) {
    const int wi = bi + w[0], wj = bj + w[1], wk = bk + w[2];
    if (wi < 0 || wj < 0 || wk < 0 || wi + 1 >= gr.nx || wj + 1 >= gr.ny || wk + 1 >= gr.nz) {
        atomicOr(status, (unsigned int)ST_BOUNDS);
        return;
    }
    T v[12];
    seg_values_at(p[0] - T(w[0]), p[1] - T(w[1]), p[2] - T(w[2]), d, q, v);
    const int c = cidx(gr, wi, wj, wk);
    const int cj1 = c + gr.nz, ck1 = c + 1, ci1 = c + gr.nynz;
    sink.add(0, wi, wj + 1, wk + 1, cj1 + 1, v[0]);
    sink.add(0, wi, wj, wk + 1, ck1, v[1]);
    sink.add(0, wi, wj + 1, wk, cj1, v[2]);
    sink.add(0, wi, wj, wk, c, v[3]);
    sink.add(1, wi + 1, wj, wk + 1, ci1 + 1, v[4]);
    sink.add(1, wi, wj, wk + 1, ck1, v[5]);
    sink.add(1, wi + 1, wj, wk, ci1, v[6]);
    sink.add(1, wi, wj, wk, c, v[7]);
    sink.add(2, wi + 1, wj + 1, wk, ci1 + gr.nz, v[8]);
    sink.add(2, wi, wj + 1, wk, cj1, v[9]);
    sink.add(2, wi + 1, wj, wk, ci1, v[10]);
    sink.add(2, wi, wj, wk, c, v[11]);
}

// The same from the start point p and the cell's lower corner w.
template <typename T>
__device__ __forceinline__ void seg_values(const T p[3], const T d[3], T q, const int w[3], T v[12]) {
    seg_values_at(p[0] - T(w[0]), p[1] - T(w[1]), p[2] - T(w[2]), d, q, v);
}

// Three ratios sorted descending with the reference's tie handling
// (`regulate`, low-level.cpp:316-366).
template <typename T>
__device__ __forceinline__ void sort3_desc(T a, T b, T c, T& vx, T& vy, T& vz) {
    if (a > b) {
        if (b > c) { vx = a; vy = b; vz = c; }
        else { vz = b; if (a > c) { vx = a; vy = c; } else { vx = c; vy = a; } }
    } else {
        if (c > b) { vx = c; vy = b; vz = a; }
        else { vx = b; if (a > c) { vy = a; vz = c; } else { vy = c; vz = a; } }
    }
}

template <typename T>
__device__ __forceinline__ int ifloor(T v) { return (int)floor(v); }

// Split the straight path p -> p + d at the cell faces it crosses (1..4
// segments), deposit each segment in its cell and advance p segment by
// segment (deposition.cpp:41-356).  p is in a frame whose integer lattice is
// the cell lattice shifted by base (base = 0 for absolute FP64 positions).
// Written with per-axis selects instead of run-time array indices so that
// everything stays in registers; the arithmetic is the reference's.
template <typename T, typename Sink>
__device__ __forceinline__ void jdeposition_to(const Sink& f, const Grid& gr, T p[3], const T d[3], T q,
                                               int bi, int bj, int bk, unsigned int* status) {
    const int c1x = ifloor(p[0]), c1y = ifloor(p[1]), c1z = ifloor(p[2]);
    const int c2x = ifloor(p[0] + d[0]), c2y = ifloor(p[1] + d[1]), c2z = ifloor(p[2] + d[2]);
    const bool cx = c1x != c2x, cy = c1y != c2y, cz = c1z != c2z;
    const int ncross = (int)cx + (int)cy + (int)cz;
    int w[3] = {c1x, c1y, c1z};
    T s[3];
    if (ncross == 0) {
        seg_dep(f, gr, p, d, q, w, bi, bj, bk, status);
        p[0] = p[0] + d[0]; p[1] = p[1] + d[1]; p[2] = p[2] + d[2];
    } else if (ncross == 1) {
        // the crossing axis a: up to its face, the other axes in proportion
        const T pa = cx ? p[0] : (cy ? p[1] : p[2]);
        const T da = cx ? d[0] : (cy ? d[1] : d[2]);
        const int ma = cx ? max(c1x, c2x) : (cy ? max(c1y, c2y) : max(c1z, c2z));
        const T sa = T(ma) - pa;
        s[0] = cx ? sa : d[0] * sa / da;
        s[1] = cy ? sa : d[1] * sa / da;
        s[2] = cz ? sa : d[2] * sa / da;
        seg_dep(f, gr, p, s, q, w, bi, bj, bk, status);
        p[0] = p[0] + s[0]; p[1] = p[1] + s[1]; p[2] = p[2] + s[2];
        s[0] = d[0] - s[0]; s[1] = d[1] - s[1]; s[2] = d[2] - s[2];
        if (cx) w[0] = c2x;
        if (cy) w[1] = c2y;
        if (cz) w[2] = c2z;
        seg_dep(f, gr, p, s, q, w, bi, bj, bk, status);
        p[0] = p[0] + s[0]; p[1] = p[1] + s[1]; p[2] = p[2] + s[2];
    } else if (ncross == 2) {
        // axis A carries the reference's path1 (y for (y,z) and (x,y), x for
        // (x,z)), axis B its path2 (z, z, x); B goes first only if
        // path1 > path2
        const bool A0 = cx && !cy;   // A = x (x,z case); else A = y
        const bool B0 = cx && cy;    // B = x (x,y case); else B = z
        const T pA = A0 ? p[0] : p[1], dA = A0 ? d[0] : d[1];
        const int mA = A0 ? max(c1x, c2x) : max(c1y, c2y);
        const T pB = B0 ? p[0] : p[2], dB = B0 ? d[0] : d[2];
        const int mB = B0 ? max(c1x, c2x) : max(c1z, c2z);
        const T pa = (T(mA) - pA) / dA;
        const T pb = (T(mB) - pB) / dB;
        const bool bfirst = pa > pb;
        const T p1 = bfirst ? pb : pa, p2 = bfirst ? pa : pb;
        // axis indices of the first and second crossing
        const int fa = bfirst ? (B0 ? 0 : 2) : (A0 ? 0 : 1);
        const int sa2 = bfirst ? (A0 ? 0 : 1) : (B0 ? 0 : 2);
        s[0] = d[0] * p1; s[1] = d[1] * p1; s[2] = d[2] * p1;
        seg_dep(f, gr, p, s, q, w, bi, bj, bk, status);
        p[0] = p[0] + s[0]; p[1] = p[1] + s[1]; p[2] = p[2] + s[2];
        const T pm = p2 - p1;
        s[0] = d[0] * pm; s[1] = d[1] * pm; s[2] = d[2] * pm;
        if (fa == 0) w[0] = c2x;
        if (fa == 1) w[1] = c2y;
        if (fa == 2) w[2] = c2z;
        seg_dep(f, gr, p, s, q, w, bi, bj, bk, status);
        p[0] = p[0] + s[0]; p[1] = p[1] + s[1]; p[2] = p[2] + s[2];
        const T pr = T(1) - p2;
        s[0] = d[0] * pr; s[1] = d[1] * pr; s[2] = d[2] * pr;
        if (sa2 == 0) w[0] = c2x;
        if (sa2 == 1) w[1] = c2y;
        if (sa2 == 2) w[2] = c2z;
        seg_dep(f, gr, p, s, q, w, bi, bj, bk, status);
        p[0] = p[0] + s[0]; p[1] = p[1] + s[1]; p[2] = p[2] + s[2];
    } else {
        const T path0 = (T(max(c1x, c2x)) - p[0]) / d[0];
        const T path1 = (T(max(c1y, c2y)) - p[1]) / d[1];
        const T path2 = (T(max(c1z, c2z)) - p[2]) / d[2];
        T vx, vy, vz;
        sort3_desc(path0, path1, path2, vx, vy, vz);
        const T fr[4] = {vz, vy - vz, vx - vy, T(1) - vx};
#pragma unroll
        for (int sg = 0; sg < 4; sg++) {
            s[0] = d[0] * fr[sg]; s[1] = d[1] * fr[sg]; s[2] = d[2] * fr[sg];
            if (sg > 0) {
                w[0] = ifloor(p[0] + T(0.5) * s[0]);
                w[1] = ifloor(p[1] + T(0.5) * s[1]);
                w[2] = ifloor(p[2] + T(0.5) * s[2]);
            }
            seg_dep(f, gr, p, s, q, w, bi, bj, bk, status);
            p[0] = p[0] + s[0]; p[1] = p[1] + s[1]; p[2] = p[2] + s[2];
        }
    }
}

// jdeposition straight into J in HBM (atomics per contribution).
template <typename T>
__device__ __forceinline__ void jdeposition(const Fields<T>& f, const Grid& gr, T p[3], const T d[3], T q,
                                            int bi, int bj, int bk, unsigned int* status) {
    GlobalSink<T> sink{f};
    jdeposition_to(sink, gr, p, d, q, bi, bj, bk, status);
}

}  // namespace qp
