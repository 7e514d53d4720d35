// Kernel bodies shared by the FP64 translation unit (qp_fp64.cu, built with
// --fmad=false) and the mixed-precision one (qp_mixed.cu, FMA allowed).
#pragma once

#include "qp_fields.cuh"

namespace qp {

// (k, j, i) = (x, y, z) launch axes; each thread updates the cells (i, j, k)
// for FieldCells<T> consecutive i (two in FP32, where one cell's bytes are
// too few to keep enough loads in flight), every cell independently.
template <typename T>
struct FieldCells { static constexpr int value = 1; };
template <>
struct FieldCells<float> { static constexpr int value = 2; };

template <typename V>
__device__ __forceinline__ V warp_sum(V v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// PHASE 0 half B, 1 E, 3 B at E points; 4 half B that first sums E^2 + B^2
// of its cells with i in [dlo, dhi) in FP64 (compute_energy's field term,
// fout.cpp:101-102, on the fields before fadvance): the values are loaded by
// the stencil anyway, and one atomic per block goes to slot blockIdx %
// FIELD_SLOTS of acc->field.
template <typename T, int SOLVER, int PHASE>
__global__ void __launch_bounds__(256) k_field(Fields<T> f, Grid g, Coef<T> c, DiagAccum* acc, int dlo, int dhi) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    constexpr int CPT = FieldCells<T>::value;
    double es = 0.0;
    const int ib = blockIdx.z * CPT;
    // a thread whose cells are all interior takes the fast path: no face
    // cases, the loads along i shared between its cells
    const bool interior = k >= 1 && k < g.nz - 1 && j >= 1 && j < g.ny - 1 && ib >= 1 && ib + CPT <= g.nx - 1;
    if (interior && PHASE == 3) {
        bbar_run<T, CPT>(f, g, ib, j, k);
    } else if (interior && SOLVER == QP_SOLVER_FDTD && (PHASE == 0 || PHASE == 4)) {
        fdtd_b_run<T, CPT, PHASE == 4>(f, g, c, ib, j, k, dlo, dhi, es);
    } else if (interior && SOLVER == QP_SOLVER_FDTD && PHASE == 1) {
        fdtd_e_run<T, CPT>(f, g, c, ib, j, k);
    } else if (k < g.nz && j < g.ny) {
#pragma unroll
        for (int u = 0; u < CPT; u++) {
            const int i = blockIdx.z * CPT + u;
            if (i >= g.nx) break;
            if (PHASE == 4 && i >= dlo && i < dhi) {
                const int x = cidx(g, i, j, k);
                const double ex = f.ex[x], ey = f.ey[x], ez = f.ez[x], bx = f.bx[x], by = f.by[x], bz = f.bz[x];
                es += ex * ex + ey * ey + ez * ez + bx * bx + by * by + bz * bz;
            }
            if (PHASE == 0 || PHASE == 4) {
                if (SOLVER == QP_SOLVER_FDTD) fdtd_b(f, g, c, i, j, k);
                else if (SOLVER == QP_SOLVER_NDFX) ndfx_b(f, g, c, i, j, k);
                else fp_b(f, g, c, i, j, k);
            } else if (PHASE == 1) {
                if (SOLVER == QP_SOLVER_FDTD) fdtd_e(f, g, c, i, j, k);
                else if (SOLVER == QP_SOLVER_NDFX) ndfx_e(f, g, c, i, j, k);
                else fp_e(f, g, c, i, j, k);
            } else {
                bbar(f, g, i, j, k);
            }
        }
    }
    if (PHASE == 4) {
        __shared__ double sh[8];
        const int t = threadIdx.y * blockDim.x + threadIdx.x;
        es = warp_sum(es);
        if ((t & 31) == 0) sh[t >> 5] = es;
        __syncthreads();
        if (t < 32) {
            es = t < (int)((blockDim.x * blockDim.y) >> 5) ? sh[t] : 0.0;
            es = warp_sum(es);
            if (t == 0 && es != 0.0) {
                const unsigned b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
                atomicAdd(&acc->field[b % FIELD_SLOTS], es);
            }
        }
    }
}

// Zero the components in mask `comps` (bits ex ey ez bx by bz) on plane
// `plane` of axis `axis`, over [0, n-1) of the two other axes.
template <typename T>
__global__ void k_zero_plane(Fields<T> f, Grid g, int axis, int plane, int comps) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y;
    int i, j, k;
    int nu, nv;
    if (axis == 0) { nu = g.nz; nv = g.ny; i = plane; j = v; k = u; }
    else if (axis == 1) { nu = g.nz; nv = g.nx; i = v; j = plane; k = u; }
    else { nu = g.ny; nv = g.nx; i = v; j = u; k = plane; }
    if (u >= nu - 1 || v >= nv - 1) return;
    const int x = cidx(g, i, j, k);
    if (comps & 1) f.ex[x] = T(0);
    if (comps & 2) f.ey[x] = T(0);
    if (comps & 4) f.ez[x] = T(0);
    if (comps & 8) f.bx[x] = T(0);
    if (comps & 16) f.by[x] = T(0);
    if (comps & 32) f.bz[x] = T(0);
}

// Block-wide sums of three values, one atomic per block into the species'
// diagnostic accumulators.
__device__ __forceinline__ void block_diag(DiagAccum* acc, int sp, double dq, double de,
                                           unsigned long long dc) {
    // the block's values through shared memory, summed by its first warp
    // (blocks of at most 256 threads); the counts with one warp reduction
    __shared__ double s_q[256], s_e[256];
    __shared__ unsigned s_c[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    s_q[threadIdx.x] = dq;
    s_e[threadIdx.x] = de;
    const unsigned c = __reduce_add_sync(0xffffffffu, (unsigned)dc);
    if (lane == 0) s_c[wid] = c;
    __syncthreads();
    if (wid == 0) {
        double q = 0.0, e = 0.0;
        for (int u = lane; u < (int)blockDim.x; u += 32) {
            q += s_q[u];
            e += s_e[u];
        }
        q = warp_sum(q);
        e = warp_sum(e);
        const int nw = (blockDim.x + 31) >> 5;
        const unsigned cc = __reduce_add_sync(0xffffffffu, lane < nw ? s_c[lane] : 0u);
        if (lane == 0 && cc) {
            atomicAdd(&acc->sum_q[sp], q);
            atomicAdd(&acc->sum_e[sp], e);
            atomicAdd(&acc->cnt[sp], (unsigned long long)cc);
        }
    }
}

// Block-wide sum of one value, one atomic per block.
__device__ __forceinline__ void block_sum(double* acc, double v) {
    __shared__ double s_v[32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s_v[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < (int)((blockDim.x + 31) >> 5) ? s_v[lane] : 0.0;
        v = warp_sum(v);
        if (lane == 0 && v != 0.0) atomicAdd(acc, v);
    }
}

// Erased by p_boundary (plist.cpp:73-102): layers {0, n-2, n-1} of each axis.
__device__ __forceinline__ bool kill_layer(const Grid& g, int i, int j, int k) {
    return i <= 0 || i >= g.nx - 2 || j <= 0 || j >= g.ny - 2 || k <= 0 || k >= g.nz - 2;
}
// is_inside (plist.cpp:42-48)
__device__ __forceinline__ bool inside(const Grid& g, int i, int j, int k) {
    return i > 0 && i < g.nx - 2 && j > 0 && j < g.ny - 2 && k > 0 && k < g.nz - 2;
}

// Warp-level segmented reduction over runs of equal keys in consecutive lanes
// (particles are sorted by cell, so a cell's particles sit in neighbouring
// lanes).  Lanes with key < 0 take no part.  On return the first lane of
// each run holds the run's sum in v[] and `head` is true for it.  Every lane
// of the warp must call this.
template <typename T, int NV>
__device__ __forceinline__ bool warp_run_sum(int key, T v[NV]) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int ukey = key >= 0 ? key : -1 - lane;  // non-members form runs of one
    const int prev = __shfl_up_sync(full, ukey, 1);
    const bool head = lane == 0 || prev != ukey;
    const unsigned heads = __ballot_sync(full, head);
    // lanes (lane, lane + d] belong to this run iff no head among them; once
    // no run is longer than d, longer strides cannot join anything
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long span = ((1ull << d) - 1ull) << (lane + 1);
        const bool same = lane + d < 32 && ((unsigned long long)heads & span) == 0ull;
        if (!__any_sync(full, same)) break;
#pragma unroll
        for (int a = 0; a < NV; a++) {
            const T o = __shfl_down_sync(full, v[a], d);
            if (same) v[a] += o;
        }
    }
    return head && key >= 0;
}

// The 12 J contributions of single-segment moves, summed per run of equal
// corner cell in the warp and added to J by the run's first lane.
template <typename T>
__device__ __forceinline__ void warp_deposit_runs(const Fields<T>& f, const Grid& g, int corner, T v[12]) {
    if (warp_run_sum<T, 12>(corner, v)) {
        const int c = corner, I = g.nynz, J = g.nz;
        atomicAdd(f.jx + c + J + 1, v[0]);
        atomicAdd(f.jx + c + 1, v[1]);
        atomicAdd(f.jx + c + J, v[2]);
        atomicAdd(f.jx + c, v[3]);
        atomicAdd(f.jy + c + I + 1, v[4]);
        atomicAdd(f.jy + c + 1, v[5]);
        atomicAdd(f.jy + c + I, v[6]);
        atomicAdd(f.jy + c, v[7]);
        atomicAdd(f.jz + c + I + J, v[8]);
        atomicAdd(f.jz + c + J, v[9]);
        atomicAdd(f.jz + c + I, v[10]);
        atomicAdd(f.jz + c, v[11]);
    }
}

// Current deposition of the whole warp's moves (deposition.cpp:41-356).
// Every move's first segment starts in the particle's own cell, so the first
// segments of a cell's particles share their 12 targets: they are summed over
// runs of equal cells in the warp and added to J once per run.  Moves that
// cross faces then deposit their further segments directly.  The segment
// arithmetic per crossing case is the reference's (see jdeposition_to); p is
// advanced segment by segment.  Every lane of the warp must call this; lanes
// with active == false take no part.
template <typename T>
__device__ __forceinline__ void deposit_runs(const Fields<T>& f, const Grid& g, T p[3], const T d[3], T q, int bi,
                                             int bj, int bk, bool active, unsigned int* status) {
    int c1x = 0, c1y = 0, c1z = 0, c2x = 0, c2y = 0, c2z = 0;
    int nx_ = 0;
    bool cx = false, cy = false, cz = false;
    // case data: 1 crossing: u = first segment; 2: u0 = p1, u1 = p2 - p1,
    // u2 = 1 - p2, fa / sa2 = axes of the first / second crossing; 3: u =
    // (vx, vy, vz), the crossing fractions sorted descending
    T u0 = T(0), u1 = T(0), u2 = T(0);
    int fa = 0, sa2 = 0;
    T v[12];
    int corner = -1;
    if (active) {
        c1x = ifloor(p[0]); c1y = ifloor(p[1]); c1z = ifloor(p[2]);
        c2x = ifloor(p[0] + d[0]); c2y = ifloor(p[1] + d[1]); c2z = ifloor(p[2] + d[2]);
        cx = c1x != c2x; cy = c1y != c2y; cz = c1z != c2z;
        nx_ = (int)cx + (int)cy + (int)cz;
        T s[3];
        if (nx_ == 0) {
            s[0] = d[0]; s[1] = d[1]; s[2] = d[2];
        } else if (nx_ == 1) {
            const T pa = cx ? p[0] : (cy ? p[1] : p[2]);
            const T da = cx ? d[0] : (cy ? d[1] : d[2]);
            const int ma = cx ? max(c1x, c2x) : (cy ? max(c1y, c2y) : max(c1z, c2z));
            const T sa = T(ma) - pa;
            u0 = cx ? sa : d[0] * sa / da;
            u1 = cy ? sa : d[1] * sa / da;
            u2 = cz ? sa : d[2] * sa / da;
            s[0] = u0; s[1] = u1; s[2] = u2;
        } else if (nx_ == 2) {
            const bool A0 = cx && !cy, B0 = cx && cy;
            const T pA = A0 ? p[0] : p[1], dA = A0 ? d[0] : d[1];
            const int mA = A0 ? max(c1x, c2x) : max(c1y, c2y);
            const T pB = B0 ? p[0] : p[2], dB = B0 ? d[0] : d[2];
            const int mB = B0 ? max(c1x, c2x) : max(c1z, c2z);
            const T pa = (T(mA) - pA) / dA;
            const T pb = (T(mB) - pB) / dB;
            const bool bfirst = pa > pb;
            const T p1 = bfirst ? pb : pa, p2 = bfirst ? pa : pb;
            fa = bfirst ? (B0 ? 0 : 2) : (A0 ? 0 : 1);
            sa2 = bfirst ? (A0 ? 0 : 1) : (B0 ? 0 : 2);
            u0 = p1;
            u1 = p2 - p1;
            u2 = T(1) - p2;
            s[0] = d[0] * u0; s[1] = d[1] * u0; s[2] = d[2] * u0;
        } else {
            const T path0 = (T(max(c1x, c2x)) - p[0]) / d[0];
            const T path1 = (T(max(c1y, c2y)) - p[1]) / d[1];
            const T path2 = (T(max(c1z, c2z)) - p[2]) / d[2];
            sort3_desc(path0, path1, path2, u0, u1, u2);
            s[0] = d[0] * u2; s[1] = d[1] * u2; s[2] = d[2] * u2;
        }
        const int w0[3] = {c1x, c1y, c1z};
        const int wi = bi + c1x, wj = bj + c1y, wk = bk + c1z;
        if (wi < 0 || wj < 0 || wk < 0 || wi + 1 >= g.nx || wj + 1 >= g.ny || wk + 1 >= g.nz) {
            atomicOr(status, (unsigned int)ST_BOUNDS);
        } else {
            seg_values(p, s, q, w0, v);
            corner = cidx(g, wi, wj, wk);
        }
        p[0] = p[0] + s[0]; p[1] = p[1] + s[1]; p[2] = p[2] + s[2];
    }
    if (corner < 0) {
#pragma unroll
        for (int k = 0; k < 12; k++) v[k] = T(0);
    }
    warp_deposit_runs(f, g, corner, v);
    if (nx_ > 0) {
        GlobalSink<T> sink{f};
        int w[3] = {c1x, c1y, c1z};
        for (int sg = 1; sg <= nx_; sg++) {
            T s[3];
            if (nx_ == 1) {
                s[0] = d[0] - u0; s[1] = d[1] - u1; s[2] = d[2] - u2;
                if (cx) w[0] = c2x;
                if (cy) w[1] = c2y;
                if (cz) w[2] = c2z;
            } else if (nx_ == 2) {
                const T fr = sg == 1 ? u1 : u2;
                s[0] = d[0] * fr; s[1] = d[1] * fr; s[2] = d[2] * fr;
                const int ax = sg == 1 ? fa : sa2;
                if (ax == 0) w[0] = c2x;
                if (ax == 1) w[1] = c2y;
                if (ax == 2) w[2] = c2z;
            } else {
                const T fr = sg == 1 ? u1 - u2 : (sg == 2 ? u0 - u1 : T(1) - u0);
                s[0] = d[0] * fr; s[1] = d[1] * fr; s[2] = d[2] * fr;
                w[0] = ifloor(p[0] + T(0.5) * s[0]);
                w[1] = ifloor(p[1] + T(0.5) * s[1]);
                w[2] = ifloor(p[2] + T(0.5) * s[2]);
            }
            seg_dep(sink, g, p, s, q, w, bi, bj, bk, status);
            p[0] = p[0] + s[0]; p[1] = p[1] + s[1]; p[2] = p[2] + s[2];
        }
    }
}

// Particles per new cell for the rebin, one atomic per run of equal cells.
__device__ __forceinline__ void warp_count_runs(int32_t* count, int cell) {
    // lanes with the same cell, wherever they sit in the warp: one atomic each
    const unsigned m = __match_any_sync(0xffffffffu, cell);
    if (cell >= 0 && (threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(count + cell, __popc(m));
}

__device__ __forceinline__ void catch_particle(const CatchBuf& c, int sp, uint32_t step, int phase, int s,
                                               double x, double y, double z, double ux, double uy, double uz,
                                               double g, double q, double chi) {
    const int slot = atomicAdd(c.counter, 1);
    if (slot >= c.cap) return;
    c.x[slot] = x; c.y[slot] = y; c.z[slot] = z;
    c.ux[slot] = ux; c.uy[slot] = uy; c.uz[slot] = uz;
    c.g[slot] = g; c.q[slot] = q; c.chi[slot] = chi;
    c.sp[slot] = sp;
    c.key[slot] = ((int64_t)step << 33) | ((int64_t)phase << 32) | (int64_t)(uint32_t)s;
}

// Chunk order of the push grids.  The grid is `waves` groups of `resident`
// blocks; group w takes the w-th contiguous part of the block-sized chunks
// of the traversal, its blocks striding over that part by `resident`.  The
// chunks in flight at any time are then neighbours in memory (the field and
// J tiles they share stay in L2), and the later groups take over as blocks
// finish, which balances the load.
struct ChunkRange {
    int first, end, step;
};
__device__ __forceinline__ ChunkRange chunk_range(int n, int resident) {
    const int nch = (int)(((long long)n + blockDim.x - 1) / blockDim.x);
    const int waves = gridDim.x / resident;
    const int per = (nch + waves - 1) / waves;
    const int w = blockIdx.x / resident, r = blockIdx.x % resident;
    return ChunkRange{w * per + r, min(nch, (w + 1) * per), resident};
}

struct PushArgs {
    double cmr, dt, dx, dy, dz, ext_bz;
    double rdx, rdy, rdz;  // RN(1 / dx) ... for div_fixed
    int resident;          // blocks per group of the chunk order (chunk_range)
    int n, sp, kind;
    int track;  // sum the energy of erased particles into diag->sum_erased
    uint32_t step;
    const CatchBuf* cat;  // device copy; nullptr: erasures are not recorded
    const CatchBuf* dcat;  // dump_photons: emitted photons recorded here instead of kept; nullptr: kept
    const int32_t* trn_src;  // track numbers in, by slot / out, by traversal position; nullptr: off
    int32_t* trn_dst;
    int dlo, dhi;  // the diagnostics count particles whose new cell has i in [dlo, dhi)
    unsigned int* status;
    DiagAccum* diag;
};

// Destination of particles born during a push (QED): slots
// [base, cap) of the target species' output buffer, claimed with *counter.
template <typename Store>
struct AppendTarget {
    Store dst;
    int32_t* newcell;
    int* counter;
    int base;
    int cap;
    int sp;  // species index (diagnostics)
};

struct QedArgs {
    double e_s;
    uint32_t key0, key1;  // random stream key (seed)
    uint32_t step;        // step counter
};

}  // namespace qp
