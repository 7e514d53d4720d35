// Particle tracks (start_tracking, main.cpp:1516-1612; fout_tracks,
// fout.cpp:706-734).  A track number (0 = untracked) per particle lives in
// an optional array per species, double-buffered like the particle store:
// the pushes carry it from slot to traversal position, and the passes that
// only rewrite the permutation (rebin, merging, moving window) leave it with
// its particle.  Particles that join the region (loads, births) start
// untracked.
#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "qp_internal.h"

namespace qp {

namespace {

// First traversal position of each requested cell (-1 if it is empty).
__global__ void k_first_in_cells(const int32_t* __restrict__ cs, int ncell, const int64_t* __restrict__ cells, int n,
                                 int64_t* __restrict__ first) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int64_t c = cells[r];
    if (c < 0 || c >= ncell) { first[r] = -1; return; }
    first[r] = cs[c] < cs[c + 1] ? cs[c] : -1;
}

__global__ void k_set_track(const int32_t* __restrict__ perm, int np, const int64_t* __restrict__ pos,
                            const int64_t* __restrict__ num, int n, int32_t* __restrict__ trn) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int64_t s = pos[r];
    if (s >= 0 && s < np) trn[perm[s]] = (int32_t)num[r];
}

// Tracked particles: traversal position, track number and state, appended
// in any order (the host sorts them by traversal position).
template <bool FP64>
__global__ void k_collect_tracked(Grid g, const int32_t* __restrict__ perm, int n, const int32_t* __restrict__ trn,
                                  void* const* arrays, int cap, int* counter, int64_t* out_s, int32_t* out_trn,
                                  double* out9) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int p = perm[s];
    const int32_t t = trn[p];
    if (t == 0) return;
    const int slot = atomicAdd(counter, 1);
    if (slot >= cap) return;
    out_s[slot] = s;
    out_trn[slot] = t;
    double v[9];
    if (FP64) {
        for (int a = 0; a < 8; a++) v[a] = ((const double*)arrays[a])[p];
        v[8] = arrays[8] ? ((const double*)arrays[8])[p] : 0.0;
    } else {
        const int c = ((const int32_t*)arrays[0])[p];
        const int i = c / g.nynz, j = (c / g.nz) % g.ny, k = c % g.nz;
        v[0] = i + (double)((const float*)arrays[1])[p];
        v[1] = j + (double)((const float*)arrays[2])[p];
        v[2] = k + (double)((const float*)arrays[3])[p];
        for (int a = 3; a < 8; a++) v[a] = (double)((const float*)arrays[a + 1])[p];
        v[8] = arrays[9] ? (double)((const float*)arrays[9])[p] : 0.0;
    }
    for (int a = 0; a < 9; a++) out9[(size_t)a * cap + slot] = v[a];
}

}  // namespace

int tracking_set(State& s, bool enable) {
    for (auto& sp : s.sp)
        for (int b = 0; b < 2; b++) {
            cudaFree(sp.trn[b]);
            sp.trn[b] = nullptr;
        }
    s.tracking = enable;
    if (!enable) return QP_OK;
    for (auto& sp : s.sp) {
        if (sp.cap == 0) continue;
        for (int b = 0; b < 2; b++) {
            QP_CUDA_CHECK(s, cudaMalloc(&sp.trn[b], sp.cap * sizeof(int32_t)));
            QP_CUDA_CHECK(s, cudaMemsetAsync(sp.trn[b], 0, sp.cap * sizeof(int32_t), s.stream));
        }
    }
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    return QP_OK;
}

}  // namespace qp

#define QP_TRACK_ENTRY(h, s)                                                          \
    if (!(h)) return QP_ERR_ARG;                                                      \
    qp::State& s = *qp::state_of(h);                                                  \
    {                                                                                 \
        const cudaError_t e0 = cudaSetDevice(s.prm.device);                           \
        if (e0 != cudaSuccess) { s.err = cudaGetErrorString(e0); return QP_ERR_CUDA; } \
    }

extern "C" int qp_set_tracking(qp_handle* h, int enable) {
    QP_TRACK_ENTRY(h, s);
    return qp::tracking_set(s, enable != 0);
}

extern "C" int qp_first_in_cells(qp_handle* h, int species, int64_t n, const int64_t* cells, int64_t* first) {
    QP_TRACK_ENTRY(h, s);
    if (species < 0 || species >= (int)s.sp.size() || n < 0 || (n > 0 && (!cells || !first))) {
        s.err = "qp_first_in_cells: bad argument";
        return QP_ERR_ARG;
    }
    if (n == 0) return QP_OK;
    int64_t *dc = nullptr, *df = nullptr;
    QP_CUDA_CHECK(s, cudaMalloc(&dc, n * sizeof(int64_t)));
    QP_CUDA_CHECK(s, cudaMalloc(&df, n * sizeof(int64_t)));
    QP_CUDA_CHECK(s, cudaMemcpy(dc, cells, n * sizeof(int64_t), cudaMemcpyDefault));
    qp::k_first_in_cells<<<(int)((n + 255) / 256), 256, 0, s.stream>>>(s.sp[species].cell_start, s.grid.nc, dc, (int)n, df);
    QP_CUDA_CHECK(s, cudaGetLastError());
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    QP_CUDA_CHECK(s, cudaMemcpy(first, df, n * sizeof(int64_t), cudaMemcpyDefault));
    cudaFree(dc);
    cudaFree(df);
    return QP_OK;
}

extern "C" int qp_set_track_numbers(qp_handle* h, int species, int64_t n, const int64_t* positions,
                                    const int64_t* numbers) {
    QP_TRACK_ENTRY(h, s);
    if (!s.tracking) { s.err = "tracking is off"; return QP_ERR_STATE; }
    if (species < 0 || species >= (int)s.sp.size() || n < 0 || (n > 0 && (!positions || !numbers))) {
        s.err = "qp_set_track_numbers: bad argument";
        return QP_ERR_ARG;
    }
    qp::Species& sp = s.sp[species];
    if (n == 0 || sp.n == 0) return QP_OK;
    int64_t *dp = nullptr, *dn = nullptr;
    QP_CUDA_CHECK(s, cudaMalloc(&dp, n * sizeof(int64_t)));
    QP_CUDA_CHECK(s, cudaMalloc(&dn, n * sizeof(int64_t)));
    QP_CUDA_CHECK(s, cudaMemcpy(dp, positions, n * sizeof(int64_t), cudaMemcpyDefault));
    QP_CUDA_CHECK(s, cudaMemcpy(dn, numbers, n * sizeof(int64_t), cudaMemcpyDefault));
    qp::k_set_track<<<(int)((n + 255) / 256), 256, 0, s.stream>>>(sp.perm, (int)sp.n, dp, dn, (int)n, sp.trn[sp.cur]);
    QP_CUDA_CHECK(s, cudaGetLastError());
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    cudaFree(dp);
    cudaFree(dn);
    return QP_OK;
}

extern "C" int qp_get_tracked(qp_handle* h, int species, int64_t cap, int64_t* trn, double* x, double* y,
                              double* z, double* ux, double* uy, double* uz, double* g, double* q, double* chi,
                              int64_t* n_out) {
    QP_TRACK_ENTRY(h, s);
    if (!n_out || species < 0 || species >= (int)s.sp.size()) { s.err = "qp_get_tracked: bad argument"; return QP_ERR_ARG; }
    if (!s.tracking) { s.err = "tracking is off"; return QP_ERR_STATE; }
    qp::Species& sp = s.sp[species];
    *n_out = 0;
    if (sp.n == 0) return QP_OK;
    // the tracked particles are few; collect up to `room` of them
    const int room = (int)std::min<int64_t>(sp.n, 1 << 16);
    int* counter = nullptr;
    int64_t* ds = nullptr;
    int32_t* dt = nullptr;
    double* d9 = nullptr;
    void** darr = nullptr;
    QP_CUDA_CHECK(s, cudaMalloc(&counter, sizeof(int)));
    QP_CUDA_CHECK(s, cudaMemset(counter, 0, sizeof(int)));
    QP_CUDA_CHECK(s, cudaMalloc(&ds, room * sizeof(int64_t)));
    QP_CUDA_CHECK(s, cudaMalloc(&dt, room * sizeof(int32_t)));
    QP_CUDA_CHECK(s, cudaMalloc(&d9, (size_t)9 * room * sizeof(double)));
    QP_CUDA_CHECK(s, cudaMalloc(&darr, 10 * sizeof(void*)));
    QP_CUDA_CHECK(s, cudaMemcpy(darr, sp.buf[sp.cur], 10 * sizeof(void*), cudaMemcpyHostToDevice));
    const int nb = (int)((sp.n + 255) / 256);
    if (s.fp64)
        qp::k_collect_tracked<true><<<nb, 256, 0, s.stream>>>(s.grid, sp.perm, (int)sp.n, sp.trn[sp.cur], darr, room,
                                                             counter, ds, dt, d9);
    else
        qp::k_collect_tracked<false><<<nb, 256, 0, s.stream>>>(s.grid, sp.perm, (int)sp.n, sp.trn[sp.cur], darr, room,
                                                              counter, ds, dt, d9);
    QP_CUDA_CHECK(s, cudaGetLastError());
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    int cnt = 0;
    QP_CUDA_CHECK(s, cudaMemcpy(&cnt, counter, sizeof(int), cudaMemcpyDeviceToHost));
    const int64_t m = std::min(cnt, room);
    if (cnt > room) {
        cudaFree(counter); cudaFree(ds); cudaFree(dt); cudaFree(d9); cudaFree(darr);
        s.err = "more than 65536 tracked particles in one species";
        return QP_ERR_CAPACITY;
    }
    double* out[9] = {x, y, z, ux, uy, uz, g, q, chi};
    bool any = trn != nullptr;
    for (double* p : out) any = any || p != nullptr;
    int r = QP_OK;
    if (any && cap < m) {
        s.err = "output arrays shorter than the tracked particles";
        r = QP_ERR_ARG;
    } else if (any && m > 0) {
        std::vector<int64_t> hs(m);
        std::vector<int32_t> ht(m);
        std::vector<double> col(m), tmp(m);
        cudaMemcpy(hs.data(), ds, m * sizeof(int64_t), cudaMemcpyDeviceToHost);
        cudaMemcpy(ht.data(), dt, m * sizeof(int32_t), cudaMemcpyDeviceToHost);
        std::vector<int64_t> order(m);
        std::iota(order.begin(), order.end(), 0);
        std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return hs[a] < hs[b]; });
        if (trn) {
            std::vector<int64_t> tv(m);
            for (int64_t i = 0; i < m; i++) tv[i] = ht[order[i]];
            cudaMemcpy(trn, tv.data(), m * sizeof(int64_t), cudaMemcpyDefault);
        }
        for (int a = 0; a < 9; a++) {
            if (!out[a]) continue;
            cudaMemcpy(col.data(), d9 + (size_t)a * room, m * sizeof(double), cudaMemcpyDeviceToHost);
            for (int64_t i = 0; i < m; i++) tmp[i] = col[order[i]];
            cudaMemcpy(out[a], tmp.data(), m * sizeof(double), cudaMemcpyDefault);
        }
    }
    *n_out = m;
    cudaFree(counter);
    cudaFree(ds);
    cudaFree(dt);
    cudaFree(d9);
    cudaFree(darr);
    return r;
}
