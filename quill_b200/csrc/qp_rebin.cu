// Counting-sort rebin of the particle stores and the device-wide exclusive
// scan it uses.
//
// The reference keeps one doubly linked list per cell and relinks a particle
// whose cell changed by head insertion into the new cell (plist.cpp:7-39,
// advance.cpp:377-386).  After a step the list of cell c is therefore
//     [arrivals in c, in DESCENDING traversal order]
//  ++ [particles that stayed in c, in ASCENDING traversal order]
// where traversal order is cells lexicographic and list order inside a cell.
// This file rebuilds exactly that order as a permutation, deterministically:
// a particle moves at most one cell per axis and step (dt < dx, dy, dz), so
// the arrivals of c come from its 26 neighbours, whose particles occupy
// known contiguous ranges of the traversal order at the start of the step.
#include "qp_internal.h"
#include "qp_kernels.cuh"

namespace qp {

// For a destination cell c = (i, j, k) inside the grid, the particles that
// can arrive come from the 3x3 neighbouring lines (i-di, j-dj); on each line
// the source cells k+1, k, k-1 form one contiguous traversal range
// [cs[(i-di, j-dj, k-1)], cs[(i-di, j-dj, k+2)]).

// Number of particles whose new cell is c (one thread per destination cell).
__global__ void __launch_bounds__(256) k_rebin_count(Grid g, const int32_t* __restrict__ cs,
                                                     const int32_t* __restrict__ newcell,
                                                     int32_t* __restrict__ count) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nc) return;
    const int k = c % g.nz, j = (c / g.nz) % g.ny, i = c / g.nynz;
    int n = 0;
    if (inside(g, i, j, k)) {
        for (int di = -1; di <= 1; di++)
            for (int dj = -1; dj <= 1; dj++) {
                const int l = c - di * g.nynz - dj * g.nz;
                const int e = __ldg(cs + l + 2);
                for (int p = __ldg(cs + l - 1); p < e; p++) n += (__ldg(newcell + p) == c);
            }
    }
    count[c] = n;
}

// Fill perm for destination cell c from start[c] (after the particles born
// in c, if any): arrivals from the source cells in descending linear index
// ((i+1, j+1, k+1) first), each scanned from its last particle down, then
// the stayers in ascending order.
__global__ void __launch_bounds__(256) k_rebin_assign(Grid g, const int32_t* __restrict__ cs,
                                                      const int32_t* __restrict__ newcell,
                                                      const int32_t* __restrict__ start,
                                                      const int32_t* __restrict__ born,
                                                      int32_t* __restrict__ perm) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nc) return;
    const int k = c % g.nz, j = (c / g.nz) % g.ny, i = c / g.nynz;
    if (!inside(g, i, j, k)) return;
    int pos = start[c] + (born ? born[c] : 0);
    const int end = start[c + 1];
    if (pos == end) return;
    const int own_b = __ldg(cs + c), own_e = __ldg(cs + c + 1);
    for (int di = -1; di <= 1; di++)
        for (int dj = -1; dj <= 1; dj++) {
            const int l = c - di * g.nynz - dj * g.nz;
            const int b = __ldg(cs + l - 1);
            for (int p = __ldg(cs + l + 2) - 1; p >= b; p--) {
                if (di == 0 && dj == 0 && p >= own_b && p < own_e) continue;  // the cell's own particles
                if (__ldg(newcell + p) == c) perm[pos++] = p;
            }
        }
    for (int p = own_b; p < own_e; p++)
        if (__ldg(newcell + p) == c) perm[pos++] = p;
}

// Particles born during this step's pushes (QED) sit at slots [n, n + A) of
// the output buffer with their cell in newcell.  They go first in their cell
// (they were head-inserted when born, plist.cpp:22-39); among themselves in
// claim order.
__global__ void k_born_hist(const int32_t* __restrict__ newcell, int n, int A, int32_t* __restrict__ born) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A) return;
    const int c = newcell[n + t];
    if (c >= 0) atomicAdd(born + c, 1);
}

__global__ void k_add_i32_inplace(int32_t* __restrict__ a, const int32_t* __restrict__ b, int n) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) a[x] += b[x];
}

__global__ void k_born_place(const int32_t* __restrict__ newcell, int n, int A, const int32_t* __restrict__ start,
                             int32_t* __restrict__ fill, int32_t* __restrict__ perm) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A) return;
    const int c = newcell[n + t];
    if (c < 0) return;
    perm[start[c] + atomicAdd(fill + c, 1)] = n + t;
}

// ---------------------------------------------------------------- scan ----
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ int block_excl_scan(int v, int* sh, int& total) {
    // warp inclusive scan
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int w = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
        int z = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += y;
        }
        sh[lane] = z - w;  // exclusive warp offsets
        if (lane == 31) sh[32] = z;
    }
    __syncthreads();
    total = sh[32];
    const int r = sh[wid] + x - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(const int32_t* in, int32_t* out, int n,
                                                             int32_t* tile_sums) {
    __shared__ int sh[33];
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int sum = 0;
#pragma unroll
    for (int t = 0; t < SCAN_ITEMS; t++) {
        v[t] = (base + t < n) ? in[base + t] : 0;
        sum += v[t];
    }
    int total;
    int off = block_excl_scan(sum, sh, total);
#pragma unroll
    for (int t = 0; t < SCAN_ITEMS; t++) {
        if (base + t < n) out[base + t] = off;
        off += v[t];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Exclusive scan of the tile sums in one block; writes the grand total to
// tile_sums[nt] (nt tiles).
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_sums(int32_t* tile_sums, int nt) {
    __shared__ int sh[33];
    int carry = 0;
    for (int b = 0; b < nt; b += SCAN_THREADS) {
        const int idx = b + threadIdx.x;
        const int v = idx < nt ? tile_sums[idx] : 0;
        int total;
        const int off = block_excl_scan(v, sh, total);
        if (idx < nt) tile_sums[idx] = carry + off;
        carry += total;
    }
    if (threadIdx.x == 0) tile_sums[nt] = carry;
}

__global__ void __launch_bounds__(256) k_scan_add(int32_t* out, int n, const int32_t* tile_sums, int nt) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) out[x] += tile_sums[x / SCAN_TILE];
    if (x == 0) out[n] = tile_sums[nt];
}

// out[0..n] = exclusive scan of in[0..n), out[n] = total.
void exclusive_scan_i32(State& s, const int32_t* in, int32_t* out, int n) {
    const int nt = (n + SCAN_TILE - 1) / SCAN_TILE;
    int32_t* sums = (int32_t*)s.scan_tmp;
    k_scan_tiles<<<nt, SCAN_THREADS, 0, s.stream>>>(in, out, n, sums);
    k_scan_sums<<<1, SCAN_THREADS, 0, s.stream>>>(sums, nt);
    k_scan_add<<<(n + 255) / 256, 256, 0, s.stream>>>(out, n, sums, nt);
    s.launches += 3;
}

int64_t rebin(State& s, int si, int64_t born, bool counted) {
    Species& sp = s.sp[si];
    const Grid g = s.grid;
    const int nb = (g.nc + 255) / 256;
    const int n = (int)sp.n, A = (int)born;
    if (!counted) {
        k_rebin_count<<<nb, 256, 0, s.stream>>>(g, sp.cell_start, sp.newcell, sp.count);
        s.launches++;
    }
    if (A > 0) {
        cudaMemsetAsync(sp.born, 0, (size_t)g.nc * sizeof(int32_t), s.stream);
        cudaMemsetAsync(sp.born_fill, 0, (size_t)g.nc * sizeof(int32_t), s.stream);
        k_born_hist<<<(A + 255) / 256, 256, 0, s.stream>>>(sp.newcell, n, A, sp.born);
        k_add_i32_inplace<<<nb, 256, 0, s.stream>>>(sp.count, sp.born, g.nc);
        s.launches += 2;
    }
    exclusive_scan_i32(s, sp.count, sp.cell_next, g.nc);
    k_rebin_assign<<<nb, 256, 0, s.stream>>>(g, sp.cell_start, sp.newcell, sp.cell_next, A > 0 ? sp.born : nullptr,
                                             sp.perm);
    s.launches++;
    if (A > 0) {
        k_born_place<<<(A + 255) / 256, 256, 0, s.stream>>>(sp.newcell, n, A, sp.cell_next, sp.born_fill, sp.perm);
        s.launches++;
    }
    std::swap(sp.cell_start, sp.cell_next);
    sp.cur = 1 - sp.cur;
    sp.slots = (int64_t)n + A;  // the push wrote traversal positions [0, n), births after them
    int32_t total = 0;
    cudaMemcpyAsync(&total, sp.cell_start + g.nc, sizeof(int32_t), cudaMemcpyDeviceToHost, s.stream);
    cudaStreamSynchronize(s.stream);
    sp.n = total;
    return total;
}

// Merge freshly uploaded particles (slots [slot0, slot0 + n_new) of the
// current buffer, already sorted by cell with given order inside a cell,
// per-cell counts in new_count) in front of the old particles of each cell.
__global__ void __launch_bounds__(256) k_load_merge(Grid g, const int32_t* __restrict__ old_start,
                                                    const int32_t* __restrict__ new_start,
                                                    const int32_t* __restrict__ merged_start,
                                                    const int32_t* __restrict__ old_perm,
                                                    int32_t* __restrict__ perm, int slot0) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nc) return;
    int pos = merged_start[c];
    for (int p = new_start[c]; p < new_start[c + 1]; p++) perm[pos++] = slot0 + p;
    for (int p = old_start[c]; p < old_start[c + 1]; p++) perm[pos++] = old_perm[p];
}

__global__ void k_add_i32(const int32_t* a, const int32_t* b, int32_t* out, int n) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) out[x] = (a[x + 1] - a[x]) + (b[x + 1] - b[x]);
}

// new_start: exclusive scan of the new particles' per-cell counts (device,
// nc+1); scratch: nc+1 ints.  perm_out receives the merged permutation.
int load_merge(State& s, int si, int64_t slot0, const int32_t* d_new_start, int32_t* d_perm_out) {
    Species& sp = s.sp[si];
    const Grid g = s.grid;
    const int nb = (g.nc + 255) / 256;
    k_add_i32<<<nb, 256, 0, s.stream>>>(sp.cell_start, d_new_start, sp.count, g.nc);
    exclusive_scan_i32(s, sp.count, sp.cell_next, g.nc);
    k_load_merge<<<nb, 256, 0, s.stream>>>(g, sp.cell_start, d_new_start, sp.cell_next, sp.perm, d_perm_out,
                                           (int)slot0);
    s.launches += 2;
    std::swap(sp.cell_start, sp.cell_next);
    return QP_OK;
}

}  // namespace qp
