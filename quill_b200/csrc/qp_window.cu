// Moving window: spatial_region::moving_window (advance.cpp:389-454).
//
// The particles of the layer i = 0 are erased; E, B and Bbar move one cell
// towards -x and the layer nx-1 becomes zero (J is left as it is, as the
// reference leaves cj); every particle moves with its cell: x - 1 (FP64) or
// cell - ny*nz (mixed).  In the traversal order the erased particles are the
// first cell_start[ny*nz] positions, so the permutation and the cell ranges
// shift by that many positions and by one layer of cells; the order inside
// each cell is kept.
#include <algorithm>
#include <string>
#include <utility>

#include "qp_internal.h"

namespace qp {

namespace {

template <typename T>
__global__ void k_window_fields(const T* __restrict__ scratch, T* __restrict__ plane, size_t keep, size_t nc) {
    const size_t x = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x < keep) plane[x] = scratch[x];
    else if (x < nc) plane[x] = T(0);
}

// Particles at traversal positions [n0, n): position shifted by one cell,
// moved to position s - n0 of the new permutation.
__global__ void k_window_particles64(const int32_t* __restrict__ perm, int n0, int n, double* __restrict__ x,
                                     int32_t* __restrict__ perm_new) {
    const int s = n0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = perm[s];
    x[p] = x[p] - 1;
    perm_new[s - n0] = p;
}

__global__ void k_window_particles32(const int32_t* __restrict__ perm, int n0, int n, int ynz,
                                     int32_t* __restrict__ cell, int32_t* __restrict__ perm_new) {
    const int s = n0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = perm[s];
    cell[p] = cell[p] - ynz;
    perm_new[s - n0] = p;
}

__global__ void k_window_starts(int nc, int ynz, int n0, int n, const int32_t* __restrict__ cs,
                                int32_t* __restrict__ cs_new) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > nc) return;
    cs_new[c] = c + ynz <= nc ? cs[c + ynz] - n0 : n - n0;
}

}  // namespace

int moving_window(State& s) {
    const size_t nc = (size_t)s.grid.nc, ynz = (size_t)s.grid.nynz, keep = nc - ynz;
    const size_t elem = s.field_elem;
    if (!s.window_scratch) QP_CUDA_CHECK(s, cudaMalloc(&s.window_scratch, nc * elem));
    // E (planes 0..2), B (3..5), Bbar (9..11)
    const int planes[9] = {0, 1, 2, 3, 4, 5, 9, 10, 11};
    const int nb = (int)((nc + 255) / 256);
    for (int a = 0; a < 9; a++) {
        char* plane = (char*)s.plane[planes[a]];
        QP_CUDA_CHECK(s, cudaMemcpyAsync(s.window_scratch, plane + ynz * elem, keep * elem, cudaMemcpyDeviceToDevice,
                                         s.stream));
        if (s.fp64)
            k_window_fields<double><<<nb, 256, 0, s.stream>>>((const double*)s.window_scratch, (double*)plane, keep, nc);
        else
            k_window_fields<float><<<nb, 256, 0, s.stream>>>((const float*)s.window_scratch, (float*)plane, keep, nc);
        s.launches++;
    }
    for (auto& sp : s.sp) {
        if (sp.n == 0) continue;
        int32_t n0 = 0;
        QP_CUDA_CHECK(s, cudaMemcpyAsync(&n0, sp.cell_start + ynz, sizeof(int32_t), cudaMemcpyDeviceToHost, s.stream));
        QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
        const int n = (int)sp.n;
        const int m = n - n0;
        if (m > 0) {
            if (s.fp64)
                k_window_particles64<<<(m + 255) / 256, 256, 0, s.stream>>>(sp.perm, n0, n, (double*)sp.buf[sp.cur][0],
                                                                            sp.newcell);
            else
                k_window_particles32<<<(m + 255) / 256, 256, 0, s.stream>>>(sp.perm, n0, n, (int)ynz,
                                                                            (int32_t*)sp.buf[sp.cur][0], sp.newcell);
            s.launches++;
        }
        k_window_starts<<<(int)((nc + 1 + 255) / 256), 256, 0, s.stream>>>((int)nc, (int)ynz, n0, n, sp.cell_start,
                                                                            sp.cell_next);
        s.launches++;
        QP_CUDA_CHECK(s, cudaGetLastError());
        std::swap(sp.perm, sp.newcell);
        std::swap(sp.cell_start, sp.cell_next);
        sp.n = m;
    }
    QP_CUDA_CHECK(s, cudaGetLastError());
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    return QP_OK;
}

}  // namespace qp

extern "C" int qp_moving_window(qp_handle* h) {
    if (!h) return QP_ERR_ARG;
    qp::State& s = *qp::state_of(h);
    const cudaError_t e = cudaSetDevice(s.prm.device);
    if (e != cudaSuccess) { s.err = cudaGetErrorString(e); return QP_ERR_CUDA; }
    return qp::moving_window(s);
}
