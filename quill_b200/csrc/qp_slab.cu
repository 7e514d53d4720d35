// Slabs of a region along x, for a decomposition into x-slab regions that
// overlap (the reference's n_sr > 1 layout, main.cpp:1286-1514): the
// neighbours' owned cells overwrite a region's halo cells after every step,
// fields (ce, cb, cj, cbe) and particle lists alike, and the diagnostics of
// each region count its owned cells only (compute_N / compute_energy with
// n1, n2 = nm at inner faces, main.cpp:2325-2327).
//
// An x-slab [i0, i0 + w) is contiguous in every field plane (k fastest) and
// in the traversal order of every species ([cell_start[i0 ny nz],
// cell_start[(i0 + w) ny nz])).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "qp_internal.h"

static double __longlong_as_double_host(unsigned long long v) {
    double d;
    memcpy(&d, &v, sizeof d);
    return d;
}

namespace qp {

namespace {

struct SlabArrays { const void* a[10]; };
struct SlabOut { double* o[9]; };

// Particles at traversal positions [a, a + m): state in doubles, absolute
// cell-unit positions (x y z ux uy uz g q chi), into the non-null outputs.
template <bool FP64>
__global__ void k_slab_gather(Grid g, const int32_t* __restrict__ perm, int a, int m, SlabArrays arr, SlabOut out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const int p = perm[a + t];
    double v[9];
    if (FP64) {
        for (int c = 0; c < 8; c++) v[c] = ((const double*)arr.a[c])[p];
        v[8] = arr.a[8] ? ((const double*)arr.a[8])[p] : 0.0;
    } else {
        const int cell = ((const int32_t*)arr.a[0])[p];
        const int i = cell / g.nynz, j = (cell / g.nz) % g.ny, k = cell % g.nz;
        v[0] = i + (double)((const float*)arr.a[1])[p];
        v[1] = j + (double)((const float*)arr.a[2])[p];
        v[2] = k + (double)((const float*)arr.a[3])[p];
        for (int c = 3; c < 8; c++) v[c] = (double)((const float*)arr.a[c + 1])[p];
        v[8] = arr.a[9] ? (double)((const float*)arr.a[9])[p] : 0.0;
    }
    for (int c = 0; c < 9; c++)
        if (out.o[c]) out.o[c][t] = v[c];
}

// Drop the traversal range [a, b): the permutation closes the gap, cells of
// the slab [c0, c1) become empty and later cells move back by b - a.
__global__ void k_slab_drop_perm(const int32_t* __restrict__ perm, int a, int b, int n, int32_t* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    if (s < a) out[s] = perm[s];
    else if (s >= b) out[s - (b - a)] = perm[s];
}

__global__ void k_slab_drop_starts(int nc, int c0, int c1, int a, int b, const int32_t* __restrict__ cs,
                                   int32_t* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > nc) return;
    out[c] = c <= c0 ? cs[c] : (c < c1 ? a : cs[c] - (b - a));
}

// A slab at the low or high x end of the region holds the head or the tail
// of every traversal.  Replacing its particles is then a concatenation: the
// new particles (in cell order, all inside the slab) become the head / tail,
// and the starts of the other cells shift by a constant.
enum { EDGE_OUTSIDE = 4 };

__global__ void k_edge_count(const int32_t* __restrict__ cells, int n, int c0, int c1, int32_t* __restrict__ count,
                             unsigned int* flags) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int c = cells[p];
    if (c < c0 || c >= c1) atomicOr(flags, (unsigned int)EDGE_OUTSIDE);
    else atomicAdd(count + (c - c0), 1);
}

// low end, cells [0, c1): new particles at positions [0, n_new), the kept
// particles (old positions [b, n)) after them
__global__ void k_edge_low_perm(const int32_t* __restrict__ perm, int b, int n_keep, int n_new, int slot0,
                                int32_t* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n_new) out[t] = slot0 + t;
    else if (t < n_new + n_keep) out[t] = perm[b + t - n_new];
}

__global__ void k_edge_low_starts(int nc, int c1, int b, int n_new, const int32_t* __restrict__ cs,
                                  const int32_t* __restrict__ starts_new, int32_t* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > nc) return;
    out[c] = c <= c1 ? starts_new[c] : cs[c] - b + n_new;
}

// high end, cells [c0, nc): new particles at positions [a, a + n_new), in place
__global__ void k_edge_high_perm(int32_t* __restrict__ perm, int a, int n_new, int slot0) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n_new) perm[a + t] = slot0 + t;
}

__global__ void k_edge_high_starts(int nc, int c0, int a, const int32_t* __restrict__ starts_new,
                                   int32_t* __restrict__ cs) {
    const int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (c > nc) return;
    cs[c] = a + starts_new[c - c0];
}

}  // namespace

}  // namespace qp

#define QP_SLAB_ENTRY(h, s)                                                           \
    if (!(h)) return QP_ERR_ARG;                                                      \
    qp::State& s = *qp::state_of(h);                                                  \
    {                                                                                 \
        const cudaError_t e0 = cudaSetDevice(s.prm.device);                           \
        if (e0 != cudaSuccess) { s.err = cudaGetErrorString(e0); return QP_ERR_CUDA; } \
    }

static bool slab_ok(qp::State& s, int i0, int width) {
    if (i0 < 0 || width < 0 || i0 + width > s.grid.nx) {
        s.err = "slab outside the region";
        return false;
    }
    return true;
}

// A pointer to device memory of this region's GPU: slab data can be read or
// written there directly, without a staging buffer.
static bool on_region_device(qp::State& s, const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice && at.device == s.prm.device;
}

extern "C" int qp_set_diag_range(qp_handle* h, int i_lo, int i_hi) {
    QP_SLAB_ENTRY(h, s);
    if (i_lo < 0 || i_hi > s.grid.nx || i_lo > i_hi) { s.err = "diagnostic range outside the region"; return QP_ERR_ARG; }
    s.diag_lo = i_lo;
    s.diag_hi = i_hi;
    return QP_OK;
}

// 12 planes of the slab <-> 12 consecutive blocks of m doubles (device).
template <typename T>
__global__ void k_field_slab_out(qp::Planes<T> f, size_t off, size_t m, double* __restrict__ out) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 12 * m) return;
    const size_t a = t / m, c = t - a * m;
    out[t] = (double)f.p[a][off + c];
}

template <typename T>
__global__ void k_field_slab_in(const double* __restrict__ in, size_t off, size_t m, qp::Planes<T> f) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 12 * m) return;
    const size_t a = t / m, c = t - a * m;
    f.p[a][off + c] = (T)in[t];
}

// Host or device buffers (the copies are cudaMemcpyDefault).
extern "C" int qp_get_field_slab(qp_handle* h, int i0, int width, double* out12) {
    QP_SLAB_ENTRY(h, s);
    if (!slab_ok(s, i0, width) || !out12) return QP_ERR_ARG;
    const size_t m = (size_t)width * s.grid.nynz, off = (size_t)i0 * s.grid.nynz;
    if (m == 0) return QP_OK;
    const bool direct = on_region_device(s, out12);
    double* d = out12;
    if (!direct) QP_CUDA_CHECK(s, qp::scratch_alloc(s, (void**)&d, 12 * m * sizeof(double)));
    const unsigned nb = (unsigned)((12 * m + 255) / 256);
    if (s.fp64) k_field_slab_out<double><<<nb, 256, 0, s.stream>>>(qp::planes_of<double>(s), off, m, d);
    else k_field_slab_out<float><<<nb, 256, 0, s.stream>>>(qp::planes_of<float>(s), off, m, d);
    s.launches++;
    const cudaError_t e = cudaGetLastError();
    if (!direct) {
        if (e == cudaSuccess) cudaMemcpyAsync(out12, d, 12 * m * sizeof(double), cudaMemcpyDefault, s.stream);
        qp::scratch_free(s, d);
    }
    const cudaError_t e2 = cudaStreamSynchronize(s.stream);
    if (e != cudaSuccess || e2 != cudaSuccess) { s.err = cudaGetErrorString(e != cudaSuccess ? e : e2); return QP_ERR_CUDA; }
    return QP_OK;
}

extern "C" int qp_set_field_slab(qp_handle* h, int i0, int width, const double* in12) {
    QP_SLAB_ENTRY(h, s);
    if (!slab_ok(s, i0, width) || !in12) return QP_ERR_ARG;
    const size_t m = (size_t)width * s.grid.nynz, off = (size_t)i0 * s.grid.nynz;
    if (m == 0) return QP_OK;
    const bool direct = on_region_device(s, in12);
    const double* d = in12;
    cudaError_t e = cudaSuccess;
    double* stage = nullptr;
    if (!direct) {
        QP_CUDA_CHECK(s, qp::scratch_alloc(s, (void**)&stage, 12 * m * sizeof(double)));
        e = cudaMemcpyAsync(stage, in12, 12 * m * sizeof(double), cudaMemcpyDefault, s.stream);
        d = stage;
    }
    const unsigned nb = (unsigned)((12 * m + 255) / 256);
    if (e == cudaSuccess) {
        if (s.fp64) k_field_slab_in<double><<<nb, 256, 0, s.stream>>>(d, off, m, qp::planes_of<double>(s));
        else k_field_slab_in<float><<<nb, 256, 0, s.stream>>>(d, off, m, qp::planes_of<float>(s));
        s.launches++;
        e = cudaGetLastError();
    }
    if (stage) qp::scratch_free(s, stage);
    const cudaError_t e2 = cudaStreamSynchronize(s.stream);
    if (e != cudaSuccess || e2 != cudaSuccess) { s.err = cudaGetErrorString(e != cudaSuccess ? e : e2); return QP_ERR_CUDA; }
    return QP_OK;
}

// max of E^2 + B^2 over the cells with i in [i0, i1) (get_max_w,
// low-level.cpp:512-532).  w >= 0, so the bit patterns of the doubles order
// like the values and an unsigned 64-bit atomicMax takes the maximum.
template <typename T>
__global__ void k_max_w(qp::Fields<T> f, size_t off, size_t m, unsigned long long* out) {
    double w = 0.0;
    for (size_t x = off + (size_t)blockIdx.x * blockDim.x + threadIdx.x; x < off + m; x += (size_t)gridDim.x * blockDim.x) {
        const double ex = f.ex[x], ey = f.ey[x], ez = f.ez[x], bx = f.bx[x], by = f.by[x], bz = f.bz[x];
        const double v = ex * ex + ey * ey + ez * ez + bx * bx + by * by + bz * bz;
        if (v > w) w = v;
    }
    for (int o = 16; o > 0; o >>= 1) w = fmax(w, __shfl_down_sync(0xffffffffu, w, o));
    if ((threadIdx.x & 31) == 0 && w > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(w));
}

extern "C" int qp_max_w(qp_handle* h, int i0, int i1, double* out) {
    QP_SLAB_ENTRY(h, s);
    if (!out) return QP_ERR_ARG;
    i0 = std::max(i0, 0);
    i1 = std::min(i1, s.grid.nx);
    *out = 0.0;
    if (i1 <= i0) return QP_OK;
    const size_t off = (size_t)i0 * s.grid.nynz, m = (size_t)(i1 - i0) * s.grid.nynz;
    unsigned long long* d = nullptr;
    QP_CUDA_CHECK(s, cudaMalloc(&d, sizeof(unsigned long long)));
    QP_CUDA_CHECK(s, cudaMemsetAsync(d, 0, sizeof(unsigned long long), s.stream));
    if (s.fp64) k_max_w<double><<<148 * 4, 256, 0, s.stream>>>(qp::fields_of<double>(s), off, m, d);
    else k_max_w<float><<<148 * 4, 256, 0, s.stream>>>(qp::fields_of<float>(s), off, m, d);
    s.launches++;
    unsigned long long v = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&v, d, sizeof(v), cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
    cudaFree(d);
    if (e != cudaSuccess) { s.err = cudaGetErrorString(e); return QP_ERR_CUDA; }
    *out = __longlong_as_double_host(v);
    return QP_OK;
}

// The field output slices of the reference's writers (fout.cpp:180-235):
// per component, for each i the line along y at k = nz/2 and the line along
// z at j = ny/2, then the plane i = ix.
template <typename T>
__global__ void k_field_slices(qp::Planes<T> f, int nx, int ny, int nz, int ix, size_t per,
                               double* __restrict__ out) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 12 * per) return;
    const int a = (int)(t / per);
    const size_t r = t - (size_t)a * per;
    const size_t lines = (size_t)nx * (ny + nz);
    long cell;
    if (r < lines) {
        const int i = (int)(r / (ny + nz)), u = (int)(r - (size_t)i * (ny + nz));
        cell = u < ny ? ((long)i * ny + u) * nz + nz / 2 : ((long)i * ny + ny / 2) * nz + (u - ny);
    } else {
        const size_t v = r - lines;
        const int j = (int)(v / nz), k = (int)(v - (size_t)j * nz);
        cell = ((long)ix * ny + j) * nz + k;
    }
    out[t] = (double)f.p[a][cell];
}

extern "C" int qp_dump_field_slices(qp_handle* h, int ix, double* out) {
    QP_SLAB_ENTRY(h, s);
    if (!out || ix < 0 || ix >= s.grid.nx) { s.err = "qp_dump_field_slices: bad argument"; return QP_ERR_ARG; }
    const int nx = s.grid.nx, ny = s.grid.ny, nz = s.grid.nz;
    const size_t per = (size_t)nx * (ny + nz) + (size_t)ny * nz;
    double* d = nullptr;
    QP_CUDA_CHECK(s, cudaMalloc(&d, 12 * per * sizeof(double)));
    const unsigned nb = (unsigned)((12 * per + 255) / 256);
    if (s.fp64) k_field_slices<double><<<nb, 256, 0, s.stream>>>(qp::planes_of<double>(s), nx, ny, nz, ix, per, d);
    else k_field_slices<float><<<nb, 256, 0, s.stream>>>(qp::planes_of<float>(s), nx, ny, nz, ix, per, d);
    s.launches++;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, 12 * per * sizeof(double), cudaMemcpyDefault, s.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
    cudaFree(d);
    if (e != cudaSuccess) { s.err = cudaGetErrorString(e); return QP_ERR_CUDA; }
    return QP_OK;
}

// Quasiparticles per x-layer, all species (the particle part of
// spatial_region::calculate_layer_weights, balancing.cpp:25-40).
extern "C" int qp_layer_counts(qp_handle* h, int64_t* counts) {
    QP_SLAB_ENTRY(h, s);
    if (!counts) return QP_ERR_ARG;
    const int nx = s.grid.nx, ynz = s.grid.nynz;
    for (int i = 0; i < nx; i++) counts[i] = 0;
    std::vector<int32_t> cs(nx + 1);
    for (auto& sp : s.sp) {
        if (sp.n == 0) continue;
        QP_CUDA_CHECK(s, cudaMemcpy2DAsync(cs.data(), sizeof(int32_t), sp.cell_start, (size_t)ynz * sizeof(int32_t),
                                           sizeof(int32_t), nx + 1, cudaMemcpyDeviceToHost, s.stream));
        QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
        for (int i = 0; i < nx; i++) counts[i] += cs[i + 1] - cs[i];
    }
    return QP_OK;
}

// traversal range of the slab's cells
static int slab_range(qp::State& s, qp::Species& sp, int i0, int width, int32_t& a, int32_t& b) {
    const size_t c0 = (size_t)i0 * s.grid.nynz, c1 = (size_t)(i0 + width) * s.grid.nynz;
    QP_CUDA_CHECK(s, cudaMemcpyAsync(&a, sp.cell_start + c0, sizeof(int32_t), cudaMemcpyDeviceToHost, s.stream));
    QP_CUDA_CHECK(s, cudaMemcpyAsync(&b, sp.cell_start + c1, sizeof(int32_t), cudaMemcpyDeviceToHost, s.stream));
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    return QP_OK;
}

extern "C" int qp_get_particle_slab(qp_handle* h, int species, int i0, int width, int64_t cap, double* x, double* y,
                                    double* z, double* ux, double* uy, double* uz, double* g, double* q, double* chi,
                                    int64_t* n_out) {
    QP_SLAB_ENTRY(h, s);
    if (!n_out || species < 0 || species >= (int)s.sp.size() || !slab_ok(s, i0, width)) return QP_ERR_ARG;
    qp::Species& sp = s.sp[species];
    *n_out = 0;
    if (sp.n == 0 || width == 0) return QP_OK;
    int32_t a = 0, b = 0;
    int r = slab_range(s, sp, i0, width, a, b);
    if (r != QP_OK) return r;
    const int m = b - a;
    *n_out = m;
    double* out[9] = {x, y, z, ux, uy, uz, g, q, chi};
    bool any = false;
    for (double* p : out) any = any || p;
    if (!any || m == 0) return QP_OK;
    if (cap < m) { s.err = "output arrays shorter than the slab's particles"; return QP_ERR_ARG; }
    qp::SlabArrays arr;
    for (int c = 0; c < 10; c++) arr.a[c] = sp.buf[sp.cur][c];
    bool direct = true;
    for (double* p : out)
        if (p && !on_region_device(s, p)) direct = false;
    qp::SlabOut o;
    double* d9 = nullptr;
    if (direct) {
        for (int c = 0; c < 9; c++) o.o[c] = out[c];
    } else {
        QP_CUDA_CHECK(s, qp::scratch_alloc(s, (void**)&d9, (size_t)9 * m * sizeof(double)));
        for (int c = 0; c < 9; c++) o.o[c] = out[c] ? d9 + (size_t)c * m : nullptr;
    }
    if (s.fp64) qp::k_slab_gather<true><<<(m + 255) / 256, 256, 0, s.stream>>>(s.grid, sp.perm, a, m, arr, o);
    else qp::k_slab_gather<false><<<(m + 255) / 256, 256, 0, s.stream>>>(s.grid, sp.perm, a, m, arr, o);
    s.launches++;
    cudaError_t e = cudaGetLastError();
    if (!direct) {
        for (int c = 0; c < 9 && e == cudaSuccess; c++)
            if (out[c]) e = cudaMemcpyAsync(out[c], o.o[c], m * sizeof(double), cudaMemcpyDefault, s.stream);
        qp::scratch_free(s, d9);
    }
    const cudaError_t e2 = cudaStreamSynchronize(s.stream);
    if (e != cudaSuccess || e2 != cudaSuccess) { s.err = cudaGetErrorString(e != cudaSuccess ? e : e2); return QP_ERR_CUDA; }
    return QP_OK;
}

// Replace the particles of an end slab (i0 == 0 or i0 + width == nx) by n
// particles in cell order inside the slab: stage them in free slots, check,
// then concatenate (see k_edge_*).  Returns QP_OK, an error, or 1 when the
// input does not qualify (unsorted or outside the slab; nothing changed).
static int replace_edge_slab(qp::State& s, int si, int i0, int width, int64_t n, const double* const* src) {
    qp::Species& sp = s.sp[si];
    const int nc = s.grid.nc;
    const int c0 = i0 * s.grid.nynz, c1 = (i0 + width) * s.grid.nynz, mc = c1 - c0;
    const bool low = i0 == 0;
    const int64_t slot0 = sp.slots;
    if (slot0 + n >= (int64_t)INT32_MAX) { s.err = "particle count exceeds 2^31-1"; return QP_ERR_CAPACITY; }
    int r = qp::ensure_capacity(s, si, slot0 + n);
    if (r != QP_OK) return r;
    // scratch: cells (n), per-slab-cell counts and starts (mc + 1 each),
    // flags + first bad index
    char* scratch = nullptr;
    const size_t cells_b = (size_t)n * 4, cnt_b = (size_t)(mc + 1) * 4;
    QP_CUDA_CHECK(s, qp::scratch_alloc(s, (void**)&scratch, cells_b + 2 * cnt_b + 16));
    int32_t* cells = (int32_t*)scratch;
    int32_t* count = (int32_t*)(scratch + cells_b);
    int32_t* starts = (int32_t*)(scratch + cells_b + cnt_b);
    unsigned int* flags = (unsigned int*)(scratch + cells_b + 2 * cnt_b);
    int* first_bad = (int*)(flags + 1);
    auto fail = [&](cudaError_t e) {
        qp::scratch_free(s, scratch);
        s.err = cudaGetErrorString(e);
        return QP_ERR_CUDA;
    };
    cudaError_t e = cudaMemsetAsync(flags, 0, 4, s.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(first_bad, 0x7f, 4, s.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(count, 0, cnt_b, s.stream);
    if (e != cudaSuccess) return fail(e);
    if ((r = qp::stage_particles(s, si, n, src, cells, flags, first_bad)) != QP_OK) {
        qp::scratch_free(s, scratch);
        return r;
    }
    qp::launch_check_sorted(s, cells, (int)n, flags);
    qp::k_edge_count<<<(unsigned)((n + 255) / 256), 256, 0, s.stream>>>(cells, (int)n, c0, c1, count, flags);
    s.launches++;
    // flags and the slab's traversal range [a, b) in one synchronisation
    int32_t hv[3] = {0, 0, 0};
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hv[0], flags, 4, cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess && sp.n > 0) e = cudaMemcpyAsync(&hv[1], sp.cell_start + c0, 4, cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess && sp.n > 0) e = cudaMemcpyAsync(&hv[2], sp.cell_start + c1, 4, cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
    if (e != cudaSuccess) return fail(e);
    if (hv[0] != 0) {  // the general path decides (and reports invalid input)
        qp::scratch_free(s, scratch);
        return 1;
    }
    const int a = sp.n > 0 ? hv[1] : 0, b = sp.n > 0 ? hv[2] : 0;
    const int n_old = (int)sp.n, nn = (int)n;
    qp::exclusive_scan_i32(s, count, starts, mc);
    if (low) {
        const int n_keep = n_old - b;
        if (nn + n_keep > 0)
            qp::k_edge_low_perm<<<(nn + n_keep + 255) / 256, 256, 0, s.stream>>>(sp.perm, b, n_keep, nn, (int)slot0,
                                                                                sp.newcell);
        qp::k_edge_low_starts<<<(nc + 1 + 255) / 256, 256, 0, s.stream>>>(nc, c1, b, nn, sp.cell_start, starts,
                                                                          sp.cell_next);
        s.launches += 2;
    } else {
        if (nn > 0) qp::k_edge_high_perm<<<(nn + 255) / 256, 256, 0, s.stream>>>(sp.perm, a, nn, (int)slot0);
        qp::k_edge_high_starts<<<(mc + 1 + 255) / 256, 256, 0, s.stream>>>(nc, c0, a, starts, sp.cell_start);
        s.launches += 2;
    }
    if (sp.trn[sp.cur]) cudaMemsetAsync(sp.trn[sp.cur] + slot0, 0, n * sizeof(int32_t), s.stream);
    qp::scratch_free(s, scratch);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
    if (e != cudaSuccess) { s.err = cudaGetErrorString(e); return QP_ERR_CUDA; }
    if (low) {
        std::swap(sp.perm, sp.newcell);
        std::swap(sp.cell_start, sp.cell_next);
        sp.n = (int64_t)nn + (n_old - b);
    } else {
        sp.n = (int64_t)a + nn;
    }
    sp.slots = slot0 + n;
    s.layout_epoch++;
    return QP_OK;
}

extern "C" int qp_replace_particle_slab(qp_handle* h, int species, int i0, int width, int64_t n, const double* x,
                                        const double* y, const double* z, const double* ux, const double* uy,
                                        const double* uz, const double* g, const double* q, const double* chi) {
    QP_SLAB_ENTRY(h, s);
    if (species < 0 || species >= (int)s.sp.size() || !slab_ok(s, i0, width) || n < 0) return QP_ERR_ARG;
    qp::Species& sp = s.sp[species];
    const bool edge = width > 0 && (i0 == 0 || i0 + width == s.grid.nx);
    if (edge && n > 0 && x && y && z && ux && uy && uz && g && q) {
        const double* src[9] = {x, y, z, ux, uy, uz, g, q, chi};
        const int r = replace_edge_slab(s, species, i0, width, n, src);
        if (r != 1) return r;
    }
    if (sp.n > 0 && width > 0) {
        int32_t a = 0, b = 0;
        int r = slab_range(s, sp, i0, width, a, b);
        if (r != QP_OK) return r;
        if (b > a) {
            const int nn = (int)sp.n;
            const int c0 = i0 * s.grid.nynz, c1 = (i0 + width) * s.grid.nynz;
            qp::k_slab_drop_perm<<<(nn + 255) / 256, 256, 0, s.stream>>>(sp.perm, a, b, nn, sp.newcell);
            qp::k_slab_drop_starts<<<(s.grid.nc + 1 + 255) / 256, 256, 0, s.stream>>>(s.grid.nc, c0, c1, a, b,
                                                                                      sp.cell_start, sp.cell_next);
            s.launches += 2;
            QP_CUDA_CHECK(s, cudaGetLastError());
            QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
            std::swap(sp.perm, sp.newcell);
            std::swap(sp.cell_start, sp.cell_next);
            sp.n = nn - (b - a);
            s.layout_epoch++;
        }
    }
    if (n == 0) return QP_OK;
    return qp_load_particles(h, species, n, x, y, z, ux, uy, uz, g, q, chi);
}
