// Particle merging: spatial_region::pmerging (mc.cpp:198-462), run between
// steps when the macro-particle count exceeds its limit (the trigger is
// main.cpp:1691-1748, evaluated by the caller from qp_diag's counts).
//
// Per species (a class of the reference: electrons, positrons, photons, one
// ion population):
//   a  = sum of the weights, signed so that it is positive for electrons
//        (a[0] -= q) and the others (a[c] += q);
//   "ti": every particle is deleted with probability ppd[0]; the survivors'
//        weights are multiplied by a / (a - deleted charge);
//   "nl": a particle of weight q is deleted with probability
//        ppd * _ppd(|q|, a / N), _ppd(q, q0) = 1 / (1 + (2 q / q0)^4); a
//        survivor's weight becomes q / (1 - that probability), and then all
//        are multiplied by a / (sum of the new weights).
// The reference draws one number of its sequential lagged-Fibonacci stream
// per particle in traversal order; here each particle draws from the
// counter-based Philox stream keyed by (seed, step, traversal position), so
// the deletions are the same in distribution, not particle for particle.
//
// Deletion keeps the traversal order of the survivors: an exclusive scan of
// the keep flags gives each survivor its new position and each cell its new
// first position (the scan at the cell's old first position).
#include <algorithm>
#include <cmath>
#include <string>
#include <utility>
#include <vector>

#include "qp_kernels.cuh"
#include "qp_qed.cuh"

namespace qp {

namespace {

constexpr uint32_t RNG_MERGE = 0x4Du;

// _ppd(q, q0) = 1 / (1 + (2 q / q0)^4); the fourth power as two squarings
// (within two ulps of pow(., 4), which costs several times more)
__device__ __forceinline__ double merge_ppd(double q, double q0) {
    const double x = 2.0 * q / q0, x2 = x * x;
    return 1.0 / (1.0 + x2 * x2);
}

template <typename QT>
__global__ void __launch_bounds__(256) k_merge_sum(const int32_t* __restrict__ perm, int n, const QT* __restrict__ q,
                                                   double sgn, double* acc) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const double v = s < n ? sgn * (double)q[perm[s]] : 0.0;
    block_sum(acc, v);
}

// Draw, decide, (nl) rescale the survivors, flag, and sum: the deleted
// signed charge (ti) or the survivors' new signed charge (nl) into acc[1].
// acc[0] holds the species' signed charge a (k_merge_sum); the mean weight
// a / n is taken here, so the host does not wait for it.
template <typename QT>
__global__ void __launch_bounds__(256) k_merge_mark(const int32_t* __restrict__ perm, int n, QT* __restrict__ q,
                                                    int mode, double ppd, double sgn, uint32_t sp,
                                                    uint32_t step, uint32_t key0, uint32_t key1,
                                                    int32_t* __restrict__ keep, double* acc) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (s < n) {
        const int p = perm[s];
        const double qq = (double)q[p];
        const double av_q = acc[0] / n;
        const double pdel = mode == QP_MERGE_TI ? ppd : ppd * merge_ppd(sgn * qq, av_q);
        double r, r2;
        uniform2(philox4x32_10((uint32_t)s, sp, RNG_MERGE, step, key0, key1), r, r2);
        const bool k = !(r < pdel);
        keep[s] = k ? 1 : 0;
        if (mode == QP_MERGE_TI) {
            if (!k) v = sgn * qq;
        } else if (k) {
            const double qn = qq / (1.0 - pdel);
            q[p] = (QT)qn;
            v = sgn * (double)(QT)qn;
        }
    }
    block_sum(acc + 1, v);
}

// Survivors: weight times f, moved to their new traversal position.
// keep was scanned in place: survivor flag = scan[s+1] - scan[s].
// f restores the species' charge a = acc[0]: a / (a - deleted) for ti
// (mc.cpp:280-283), a / (new sum) for nl (mc.cpp:431-436).
template <typename QT>
__global__ void __launch_bounds__(256) k_merge_compact(const int32_t* __restrict__ perm, int n,
                                                       const int32_t* __restrict__ scan, QT* __restrict__ q, int mode,
                                                       const double* __restrict__ acc, int32_t* __restrict__ perm_new) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int pos = scan[s];
    if (scan[s + 1] == pos) return;  // deleted
    const double a = acc[0], h = acc[1];
    double f;
    if (mode == QP_MERGE_TI) f = (a - h != 0) ? a / (a - h) : a;
    else f = h != 0 ? a / h : 0.0;
    const int p = perm[s];
    q[p] = (QT)(f * (double)q[p]);
    perm_new[pos] = p;
}

__global__ void k_merge_starts(int ncell, const int32_t* __restrict__ cs, const int32_t* __restrict__ scan,
                               int32_t* __restrict__ cs_new) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c <= ncell) cs_new[c] = scan[cs[c]];
}

// Stream-ordered; the species' new count goes to s.h_count[si] (pinned),
// read by the caller after its synchronisation.  acc: two doubles of
// device scratch.
template <typename QT>
int merge_species(State& s, int si, int mode, double ppd, int32_t* scratch, double* acc) {
    Species& sp = s.sp[si];
    const int n = (int)sp.n;
    const double sgn = sp.cmr == -1 ? -1.0 : 1.0;
    QT* q = (QT*)sp.buf[sp.cur][s.fp64 ? 7 : 8];
    const int nb = (n + 255) / 256;
    QP_CUDA_CHECK(s, cudaMemsetAsync(acc, 0, 2 * sizeof(double), s.stream));
    k_merge_sum<QT><<<nb, 256, 0, s.stream>>>(sp.perm, n, q, sgn, acc);
    const uint32_t key0 = (uint32_t)(s.prm.seed & 0xffffffffu), key1 = (uint32_t)(s.prm.seed >> 32);
    k_merge_mark<QT><<<nb, 256, 0, s.stream>>>(sp.perm, n, q, mode, ppd, sgn, (uint32_t)si, (uint32_t)s.step_index,
                                               key0, key1, scratch, acc);
    exclusive_scan_i32(s, scratch, scratch, n);
    k_merge_compact<QT><<<nb, 256, 0, s.stream>>>(sp.perm, n, scratch, q, mode, acc, sp.newcell);
    k_merge_starts<<<(s.grid.nc + 1 + 255) / 256, 256, 0, s.stream>>>(s.grid.nc, sp.cell_start, scratch, sp.cell_next);
    s.launches += 4;
    QP_CUDA_CHECK(s, cudaGetLastError());
    QP_CUDA_CHECK(s, cudaMemcpyAsync(s.h_count + si, scratch + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s.stream));
    std::swap(sp.perm, sp.newcell);
    std::swap(sp.cell_start, sp.cell_next);
    return QP_OK;
}

}  // namespace

}  // namespace qp

extern "C" int qp_pmerging(qp_handle* h, int mode, const double* ppd) {
    if (!h) return QP_ERR_ARG;
    qp::State& s = *qp::state_of(h);
    cudaError_t e = cudaSetDevice(s.prm.device);
    if (e != cudaSuccess) { s.err = cudaGetErrorString(e); return QP_ERR_CUDA; }
    if (mode != QP_MERGE_TI && mode != QP_MERGE_NL) { s.err = "merging mode must be QP_MERGE_TI or QP_MERGE_NL"; return QP_ERR_ARG; }
    if (!ppd) { s.err = "null ppd"; return QP_ERR_ARG; }
    const int ns = (int)s.sp.size();
    for (int i = 0; i < (mode == QP_MERGE_TI ? 1 : ns); i++)
        if (!(ppd[i] >= 0.0 && ppd[i] < 1.0)) { s.err = "ppd must lie in [0, 1)"; return QP_ERR_ARG; }
    int64_t nmax = 0;
    for (auto& sp : s.sp) nmax = std::max(nmax, sp.n);
    if (nmax == 0) return QP_OK;
    // the scan's tile sums are sized for the cells; particles can outnumber them
    const size_t tiles = (size_t)((nmax + 4095) / 4096 + 2) * sizeof(int32_t);
    if (tiles > s.scan_tmp_bytes) {
        void* t = nullptr;
        e = cudaMalloc(&t, tiles);
        if (e != cudaSuccess) { s.err = std::string("qp_pmerging: ") + cudaGetErrorString(e); return QP_ERR_CUDA; }
        cudaFree(s.scan_tmp);
        s.scan_tmp = t;
        s.scan_tmp_bytes = tiles;
    }
    // keep flags, scanned in place (n + 1), then two doubles of sums
    const size_t keep_b = ((size_t)(nmax + 1) * sizeof(int32_t) + 15) / 16 * 16;
    char* scratch = nullptr;
    e = qp::scratch_alloc(s, (void**)&scratch, keep_b + 2 * sizeof(double));
    if (e != cudaSuccess) { s.err = std::string("qp_pmerging: ") + cudaGetErrorString(e); return QP_ERR_CUDA; }
    std::vector<char> merged(ns, 0);
    int r = QP_OK;
    for (int i = 0; i < ns && r == QP_OK; i++) {
        const double p = mode == QP_MERGE_TI ? ppd[0] : ppd[i];
        if (s.sp[i].n == 0 || p <= 0.0) continue;
        merged[i] = 1;
        r = s.fp64 ? qp::merge_species<double>(s, i, mode, p, (int32_t*)scratch, (double*)(scratch + keep_b))
                   : qp::merge_species<float>(s, i, mode, p, (int32_t*)scratch, (double*)(scratch + keep_b));
    }
    qp::scratch_free(s, scratch);
    e = cudaStreamSynchronize(s.stream);
    if (r == QP_OK && e != cudaSuccess) { s.err = std::string("qp_pmerging: ") + cudaGetErrorString(e); r = QP_ERR_CUDA; }
    if (r != QP_OK) return r;
    for (int i = 0; i < ns; i++)
        if (merged[i]) s.sp[i].n = s.h_count[i];
    return QP_OK;
}
