// Device side of loading particles and fields: validation, cell indices,
// order check, conversion to the mixed representation, per-cell counts.
#include "qp_kernels.cuh"

namespace qp {

enum LoadFlags { LD_INVALID = 1, LD_UNSORTED = 2 };

// Validate positions (inside [0, n) per axis) and finiteness, write the
// linear cell of each particle, flag input that is not in cell order.
__global__ void k_load_cells(Grid g, const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, const double* __restrict__ ux,
                             const double* __restrict__ uy, const double* __restrict__ uz,
                             const double* __restrict__ gm, const double* __restrict__ q, int n,
                             int32_t* __restrict__ cells, unsigned int* flags, int* first_bad, int base) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double px = x[p], py = y[p], pz = z[p];
    const bool ok = px >= 0.0 && px < (double)g.nx && py >= 0.0 && py < (double)g.ny && pz >= 0.0 &&
                    pz < (double)g.nz && isfinite(ux[p]) && isfinite(uy[p]) && isfinite(uz[p]) &&
                    isfinite(gm[p]) && isfinite(q[p]);
    int c = 0;
    if (ok) c = cidx(g, (int)px, (int)py, (int)pz);
    else {
        atomicOr(flags, (unsigned int)LD_INVALID);
        atomicMin(first_bad, base + p);
    }
    cells[base + p] = c;
}

__global__ void k_check_sorted(const int32_t* __restrict__ cells, int n, unsigned int* flags) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0 || p >= n) return;
    if (cells[p - 1] > cells[p]) atomicOr(flags, (unsigned int)LD_UNSORTED);
}

__global__ void k_histogram(const int32_t* __restrict__ cells, int n, int32_t* __restrict__ count) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) atomicAdd(count + cells[p], 1);
}

// FP64 input -> (cell, FP32 offset) store at slot offset `at`.
__global__ void k_to_mixed(Grid g, const double* __restrict__ x, const double* __restrict__ y,
                           const double* __restrict__ z, const double* __restrict__ ux,
                           const double* __restrict__ uy, const double* __restrict__ uz,
                           const double* __restrict__ gm, const double* __restrict__ q,
                           const double* __restrict__ chi, int n, PStore32 dst, int at) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const double px = x[p], py = y[p], pz = z[p];
    const int i = (int)px, j = (int)py, k = (int)pz;
    const int s = at + p;
    dst.cell[s] = cidx(g, i, j, k);
    float o[3] = {(float)(px - i), (float)(py - j), (float)(pz - k)};
    for (int a = 0; a < 3; a++)
        if (o[a] >= 1.0f) o[a] = 0.99999994f;
    dst.ox[s] = o[0]; dst.oy[s] = o[1]; dst.oz[s] = o[2];
    dst.ux[s] = (float)ux[p]; dst.uy[s] = (float)uy[p]; dst.uz[s] = (float)uz[p];
    dst.g[s] = (float)gm[p]; dst.q[s] = (float)q[p];
    if (dst.chi) dst.chi[s] = chi ? (float)chi[p] : 0.0f;
}

__global__ void k_f64_to_f32(const double* __restrict__ a, float* __restrict__ b, size_t n) {
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < n; x += (size_t)gridDim.x * blockDim.x)
        b[x] = (float)a[x];
}

__global__ void k_f32_to_f64(const float* __restrict__ a, double* __restrict__ b, size_t n) {
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < n; x += (size_t)gridDim.x * blockDim.x)
        b[x] = (double)a[x];
}

void launch_f32_to_f64(State& s, const float* a, double* b, size_t n) {
    k_f32_to_f64<<<148 * 8, 256, 0, s.stream>>>(a, b, n);
    s.launches++;
}

void launch_load_cells(State& s, const double* const* a, int n, int32_t* cells, unsigned int* flags,
                       int* first_bad, int base) {
    if (n <= 0) return;
    k_load_cells<<<(n + 255) / 256, 256, 0, s.stream>>>(s.grid, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], n,
                                                         cells, flags, first_bad, base);
    s.launches++;
}

void launch_check_sorted(State& s, const int32_t* cells, int n, unsigned int* flags) {
    k_check_sorted<<<(n + 255) / 256, 256, 0, s.stream>>>(cells, n, flags);
    s.launches++;
}

void launch_histogram(State& s, const int32_t* cells, int n, int32_t* count) {
    cudaMemsetAsync(count, 0, (size_t)s.grid.nc * sizeof(int32_t), s.stream);
    if (n > 0) {
        k_histogram<<<(n + 255) / 256, 256, 0, s.stream>>>(cells, n, count);
        s.launches++;
    }
}

void launch_to_mixed(State& s, const double* const* a, int n, PStore32 dst, int at) {
    if (n <= 0) return;
    k_to_mixed<<<(n + 255) / 256, 256, 0, s.stream>>>(s.grid, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8],
                                                       n, dst, at);
    s.launches++;
}

void launch_f64_to_f32(State& s, const double* a, float* b, size_t n) {
    k_f64_to_f32<<<148 * 8, 256, 0, s.stream>>>(a, b, n);
    s.launches++;
}

}  // namespace qp
