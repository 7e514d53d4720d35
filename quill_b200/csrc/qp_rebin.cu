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

// The rebin runs in two passes over the new cells computed by the push:
//  1. scatter (thread per old traversal position t): a particle that stays
//     in its cell c (t in c's old range [cs[c], cs[c+1])) takes, from the end
//     of c's new range, the slot given by the number of c's stayers after it
//     (a warp ballot plus, for ranges continuing past the warp, a short
//     scan), so the stayers land in ascending order with no atomics; an
//     arrival or a born particle (t >= n) claims the next slot from the front
//     of the range (one atomic per run of equal cells in the warp);
//  2. front order (thread per cell): the claimed front part is put in list
//     order, born ascending then arrivals DESCENDING by old position; it is
//     short (the arrivals of one step), long parts go to a block each.

// Sort key of a front entry: born (x >= n_old) ascending first, then
// arrivals (x < n_old) by DESCENDING old position; both fit 32 bits.
__device__ __forceinline__ unsigned front_key(int x, int n_old) {
    if (x >= n_old) return (unsigned)(x - n_old);               // born: [0, 2^31)
    return 0x80000000u + (unsigned)(n_old - 1 - x);             // arrival: [2^31, 2^32)
}

// Particles per new cell (entries < 0 skipped), one atomic per run.
__global__ void __launch_bounds__(256) k_rebin_count(const int32_t* __restrict__ newcell, int total,
                                                     int32_t* __restrict__ count) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    warp_count_runs(count, t < total ? __ldg(newcell + t) : -1);
}

// Positions per warp of the scatter: REBIN_CHUNKS chunks of 32, whose loads
// and claims are issued together (the kernel waits on memory and atomics).
constexpr int REBIN_CHUNKS = 4;

__global__ void __launch_bounds__(256) k_rebin_scatter(const int32_t* __restrict__ newcell, int total,
                                                       const int32_t* __restrict__ cs,
                                                       const int32_t* __restrict__ start,
                                                       int32_t* __restrict__ cursor, int32_t* __restrict__ perm,
                                                       unsigned int* status) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int w0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32 * REBIN_CHUNKS;
    int key[REBIN_CHUNKS], e[REBIN_CHUNKS], end[REBIN_CHUNKS], b[REBIN_CHUNKS];
#pragma unroll
    for (int h = 0; h < REBIN_CHUNKS; h++) {
        const int t = w0 + 32 * h + lane;
        key[h] = t < total ? __ldg(newcell + t) : -1;
    }
#pragma unroll
    for (int h = 0; h < REBIN_CHUNKS; h++) {
        // independent loads, issued together: the old range of the new cell
        // and the end of its new range (used if the particle stayed)
        b[h] = 0; e[h] = 0; end[h] = 0;
        if (key[h] >= 0) {
            b[h] = __ldg(cs + key[h]);
            e[h] = __ldg(cs + key[h] + 1);
            end[h] = __ldg(start + key[h] + 1);
        }
    }
    int base[REBIN_CHUNKS], hl[REBIN_CHUNKS], akey[REBIN_CHUNKS];
#pragma unroll
    for (int h = 0; h < REBIN_CHUNKS; h++) {
        const int wb = w0 + 32 * h;  // first position of this chunk
        const int t = wb + lane;
        const bool stay = key[h] >= 0 && t >= b[h] && t < e[h];
        // stayers: slot counted from the end of the new range
        const unsigned smask = __ballot_sync(full, stay);
        if (stay) {
            const int hi = min(e[h] - wb, 32);
            const unsigned below_hi = hi >= 32 ? full : ((1u << hi) - 1u);
            const unsigned above_me = lane == 31 ? 0u : ~((2u << lane) - 1u);
            int after = __popc(smask & below_hi & above_me);
            for (int u = wb + 32; u < e[h]; u++) after += __ldg(newcell + u) == key[h];
            const int pos = end[h] - 1 - after;
            if (pos >= 0 && pos < total) perm[pos] = t;
            else atomicOr(status, (unsigned int)ST_BOUNDS);  // counts inconsistent with the cells
        }
        // arrivals and born: claimed from the front, one atomic per run
        akey[h] = (key[h] >= 0 && !stay) ? key[h] : -1;
        const int ukey = akey[h] >= 0 ? akey[h] : -1 - lane;
        const int prev = __shfl_up_sync(full, ukey, 1);
        const bool head = lane == 0 || prev != ukey;
        const unsigned heads = __ballot_sync(full, head);
        const unsigned upto = lane == 31 ? full : ((2u << lane) - 1u);
        hl[h] = 31 - __clz(heads & upto);                 // first lane of this lane's run
        const unsigned above = heads & ~upto;
        const int next = above ? __ffs(above) - 1 : 32;   // first lane of the next run
        base[h] = 0;
        if (head && akey[h] >= 0) base[h] = atomicAdd(cursor + akey[h], next - lane);
    }
#pragma unroll
    for (int h = 0; h < REBIN_CHUNKS; h++) {
        const int bb = __shfl_sync(full, base[h], hl[h]);
        if (akey[h] >= 0) {
            const int pos = bb + lane - hl[h];
            if (pos >= 0 && pos < total) perm[pos] = w0 + 32 * h + lane;
            else atomicOr(status, (unsigned int)ST_BOUNDS);
        }
    }
}

// Front part [start[c], cursor[c]) of each cell into list order, in place.
// The part holds one step's arrivals: up to 8 entries are sorted in
// registers, up to REBIN_LONG_SEG by insertion sort in place, longer parts
// are queued for k_rebin_front_long.
__global__ void __launch_bounds__(256) k_rebin_front(int ncell, const int32_t* __restrict__ start,
                                                     const int32_t* __restrict__ cursor, int n_old, int total,
                                                     int32_t* __restrict__ perm, int32_t* __restrict__ long_list,
                                                     int* __restrict__ n_long, unsigned int* status) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    int b = 0, f = 0;
    if (c < ncell) {
        b = __ldg(start + c);
        f = __ldg(cursor + c) - b;
        if (f >= 2 && (b < 0 || b + f > total)) {  // counts inconsistent with the cells
            atomicOr(status, (unsigned int)ST_BOUNDS);
            f = 0;
        }
        if (f > REBIN_LONG_SEG) {
            long_list[atomicAdd(n_long, 1)] = c;
            f = 0;
        }
    }
    // the sorting network is chosen for the longest part in the warp (most
    // parts are 0 or 1 long, a few 2, rarely more than 4)
    const int fmax = __reduce_max_sync(0xffffffffu, f);
    if (fmax < 2) return;
    if (fmax == 2) {
        if (f == 2) {
            const int x0 = perm[b], x1 = perm[b + 1];
            if (front_key(x0, n_old) > front_key(x1, n_old)) {
                perm[b] = x1;
                perm[b + 1] = x0;
            }
        }
        return;
    }
    if (fmax <= 4) {
        if (f < 2) return;
        int x[4];
        unsigned k[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            x[u] = u < f ? perm[b + u] : 0;
            k[u] = u < f ? front_key(x[u], n_old) : 0xffffffffu;
        }
        // optimal 4-input network: (0,1) (2,3) (0,2) (1,3) (1,2)
        auto cx = [&](int i, int j) {
            if (k[i] > k[j]) {
                const unsigned tk = k[i]; k[i] = k[j]; k[j] = tk;
                const int tx = x[i]; x[i] = x[j]; x[j] = tx;
            }
        };
        cx(0, 1); cx(2, 3); cx(0, 2); cx(1, 3); cx(1, 2);
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (u < f) perm[b + u] = x[u];
        return;
    }
    if (f < 2) return;
    if (f <= 8) {
        // in registers: all loads issued together, odd-even transposition sort
        int x[8];
        unsigned k[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            x[u] = u < f ? perm[b + u] : 0;
            k[u] = u < f ? front_key(x[u], n_old) : 0xffffffffu;
        }
#pragma unroll
        for (int r = 0; r < 8; r++) {
#pragma unroll
            for (int u = r & 1; u + 1 < 8; u += 2) {
                if (k[u] > k[u + 1]) {
                    const unsigned tk = k[u]; k[u] = k[u + 1]; k[u + 1] = tk;
                    const int tx = x[u]; x[u] = x[u + 1]; x[u + 1] = tx;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (u < f) perm[b + u] = x[u];
        return;
    }
    for (int u = b + 1; u < b + f; u++) {
        const int x = perm[u];
        const unsigned kx = front_key(x, n_old);
        int v = u - 1;
        while (v >= b && front_key(perm[v], n_old) > kx) {
            perm[v + 1] = perm[v];
            v--;
        }
        perm[v + 1] = x;
    }
}

// A long front part per block: copied to scratch, each entry ranked by
// counting the entries with a smaller key, written back.
__global__ void __launch_bounds__(256) k_rebin_front_long(const int32_t* __restrict__ start,
                                                          const int32_t* __restrict__ cursor, int n_old,
                                                          int32_t* __restrict__ perm, int32_t* __restrict__ scratch,
                                                          const int32_t* __restrict__ long_list,
                                                          const int* __restrict__ n_long) {
    const int nl = *n_long;
    for (int li = blockIdx.x; li < nl; li += gridDim.x) {
        const int c = long_list[li];
        const int b = start[c], e = cursor[c];
        for (int u = b + (int)threadIdx.x; u < e; u += blockDim.x) scratch[u] = perm[u];
        __syncthreads();
        for (int u = b + (int)threadIdx.x; u < e; u += blockDim.x) {
            const int x = scratch[u];
            const unsigned kx = front_key(x, n_old);
            int r = 0;
            for (int v = b; v < e; v++) r += front_key(scratch[v], n_old) < kx;
            perm[b + r] = x;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- scan ----
// Reduce-then-scan over tiles of SCAN_TILE items: k_scan_reduce sums each
// tile, k_scan_sums scans the tile sums in one block, k_scan_down scans each
// tile from its offset and writes the result (and the copy).  The input is
// read twice and the output written once: 3 (4 with the copy) passes of
// 4 bytes per item.  Items are loaded and stored four at a time when the
// arrays are 16-byte aligned.
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
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

// The SCAN_ITEMS items of this thread (consecutive), zero past n.
template <bool VEC>
__device__ __forceinline__ void scan_load(const int32_t* in, int n, int base, int v[SCAN_ITEMS]) {
    if (VEC && base + SCAN_ITEMS <= n) {
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS / 4; q++) {
            const int4 w = *reinterpret_cast<const int4*>(in + base + 4 * q);
            v[4 * q] = w.x; v[4 * q + 1] = w.y; v[4 * q + 2] = w.z; v[4 * q + 3] = w.w;
        }
    } else {
#pragma unroll
        for (int t = 0; t < SCAN_ITEMS; t++) v[t] = base + t < n ? in[base + t] : 0;
    }
}

template <bool VEC>
__device__ __forceinline__ void scan_store(int32_t* out, int n, int base, const int v[SCAN_ITEMS]) {
    if (VEC && base + SCAN_ITEMS <= n) {
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS / 4; q++)
            *reinterpret_cast<int4*>(out + base + 4 * q) = make_int4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else {
#pragma unroll
        for (int t = 0; t < SCAN_ITEMS; t++)
            if (base + t < n) out[base + t] = v[t];
    }
}

template <bool VEC>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const int32_t* __restrict__ in, int n,
                                                              int32_t* __restrict__ tile_sums) {
    __shared__ int sh[33];
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    scan_load<VEC>(in, n, base, v);
    int sum = 0;
#pragma unroll
    for (int t = 0; t < SCAN_ITEMS; t++) sum += v[t];
    int total;
    block_excl_scan(sum, sh, total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Exclusive scan of the tile sums in one block; writes the grand total to
// tile_sums[nt] (nt tiles).
__global__ void __launch_bounds__(1024) k_scan_sums(int32_t* tile_sums, int nt) {
    __shared__ int sh[33];
    int carry = 0;
    for (int b = 0; b < nt; b += blockDim.x) {
        const int idx = b + threadIdx.x;
        const int v = idx < nt ? tile_sums[idx] : 0;
        int total;
        const int off = block_excl_scan(v, sh, total);
        if (idx < nt) tile_sums[idx] = carry + off;
        carry += total;
    }
    if (threadIdx.x == 0) tile_sums[nt] = carry;
}

// in may alias out or copy: every thread reads its items before writing them.
template <bool VEC>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_down(const int32_t* in, int32_t* out, int n,
                                                            const int32_t* __restrict__ tile_sums, int nt,
                                                            int32_t* copy) {
    __shared__ int sh[33];
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    scan_load<VEC>(in, n, base, v);
    int sum = 0;
#pragma unroll
    for (int t = 0; t < SCAN_ITEMS; t++) sum += v[t];
    int total;
    int off = block_excl_scan(sum, sh, total) + tile_sums[blockIdx.x];
#pragma unroll
    for (int t = 0; t < SCAN_ITEMS; t++) {
        const int x = v[t];
        v[t] = off;
        off += x;
    }
    scan_store<VEC>(out, n, base, v);
    if (copy) scan_store<VEC>(copy, n, base, v);
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = tile_sums[nt];
}

// out[0..n] = exclusive scan of in[0..n), out[n] = total; copy[0..n) (if
// given, may alias in) receives out[0..n) as well.  in may alias out.
void exclusive_scan_i32(State& s, const int32_t* in, int32_t* out, int n, int32_t* copy) {
    const int nt = (n + SCAN_TILE - 1) / SCAN_TILE;
    int32_t* sums = (int32_t*)s.scan_tmp;
    const bool vec = ((uintptr_t)in % 16 == 0) && ((uintptr_t)out % 16 == 0) && ((uintptr_t)copy % 16 == 0);
    if (nt > 0) {
        if (vec) k_scan_reduce<true><<<nt, SCAN_THREADS, 0, s.stream>>>(in, n, sums);
        else k_scan_reduce<false><<<nt, SCAN_THREADS, 0, s.stream>>>(in, n, sums);
    }
    k_scan_sums<<<1, 1024, 0, s.stream>>>(sums, nt);
    if (nt > 0) {
        if (vec) k_scan_down<true><<<nt, SCAN_THREADS, 0, s.stream>>>(in, out, n, sums, nt, copy);
        else k_scan_down<false><<<nt, SCAN_THREADS, 0, s.stream>>>(in, out, n, sums, nt, copy);
    } else {
        cudaMemcpyAsync(out, sums, sizeof(int32_t), cudaMemcpyDeviceToDevice, s.stream);  // out[0] = 0
    }
    s.launches += 3;
}

void rebin(State& s, int si, int64_t born, bool counted) {
    Species& sp = s.sp[si];
    const Grid g = s.grid;
    const int n = (int)sp.n, A = (int)born;
    const int total = n + A;
    if (!counted) {
        cudaMemsetAsync(sp.count, 0, (size_t)g.nc * sizeof(int32_t), s.stream);
        if (total > 0) {
            k_rebin_count<<<(total + 255) / 256, 256, 0, s.stream>>>(sp.newcell, total, sp.count);
            s.launches++;
        }
    }
    // cell_next = exclusive scan of the counts; count becomes the claim cursor
    exclusive_scan_i32(s, sp.count, sp.cell_next, g.nc, sp.count);
    if (total > 0) {
        const int per_block = 256 * REBIN_CHUNKS;
        k_rebin_scatter<<<(total + per_block - 1) / per_block, 256, 0, s.stream>>>(
            sp.newcell, total, sp.cell_start, sp.cell_next, sp.count, sp.perm, s.d_status);
        s.launches++;
    }
    int* n_long = (int*)s.long_list;  // entry 0: count; cells from entry 1
    cudaMemsetAsync(n_long, 0, sizeof(int), s.stream);
    k_rebin_front<<<(g.nc + 255) / 256, 256, 0, s.stream>>>(g.nc, sp.cell_next, sp.count, n, total, sp.perm,
                                                             s.long_list + 1, n_long, s.d_status);
    k_rebin_front_long<<<2 * 148, 256, 0, s.stream>>>(sp.cell_next, sp.count, n, sp.perm, sp.newcell,
                                                      s.long_list + 1, n_long);
    s.launches += 2;
    std::swap(sp.cell_start, sp.cell_next);
    sp.cur = 1 - sp.cur;
    sp.slots = (int64_t)total;  // the push wrote traversal positions [0, n), births after them
    // the new count, read back with the step's diagnostics (qp_step sets
    // sp.n after its end-of-step synchronisation)
    cudaMemcpyAsync(s.h_count + si, sp.cell_start + g.nc, sizeof(int32_t), cudaMemcpyDeviceToHost, s.stream);
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
    exclusive_scan_i32(s, sp.count, sp.cell_next, g.nc, nullptr);
    k_load_merge<<<nb, 256, 0, s.stream>>>(g, sp.cell_start, d_new_start, sp.cell_next, sp.perm, d_perm_out,
                                           (int)slot0);
    s.launches += 2;
    std::swap(sp.cell_start, sp.cell_next);
    return QP_OK;
}

}  // namespace qp
