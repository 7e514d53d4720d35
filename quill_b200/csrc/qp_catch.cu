// Catching (delete_particle with catching_enabled, low-level.cpp:247-259):
// the push kernels record every particle they erase into a device buffer;
// qp_get_caught hands the records out in the reference's deletion order and
// empties the buffer, as write_deleted_particles clears its list
// (main.cpp:189-330).
#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "qp_internal.h"

namespace qp {

static void catch_free(CatchBuf& c) {
    double* d[9] = {c.x, c.y, c.z, c.ux, c.uy, c.uz, c.g, c.q, c.chi};
    for (double* p : d) cudaFree(p);
    cudaFree(c.sp);
    cudaFree(c.key);
    cudaFree(c.counter);
    c = CatchBuf{};
}

void catch_release(State& s) {
    catch_free(s.cat);
    cudaFree(s.d_cat);
    s.d_cat = nullptr;
}

}  // namespace qp

namespace qp {
static int catch_alloc(State& s, int64_t capacity) {
    if (capacity <= 0 || capacity >= INT32_MAX) { s.err = "catching capacity must lie in [1, 2^31-1)"; return QP_ERR_ARG; }
    cudaError_t e = cudaSuccess;
    CatchBuf c{};
    double** d[9] = {&c.x, &c.y, &c.z, &c.ux, &c.uy, &c.uz, &c.g, &c.q, &c.chi};
    for (double** p : d)
        if (e == cudaSuccess) e = cudaMalloc(p, (size_t)capacity * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&c.sp, (size_t)capacity * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&c.key, (size_t)capacity * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&c.counter, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c.counter, 0, sizeof(int));
    c.cap = (int)capacity;
    CatchBuf* dc = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&dc, sizeof(CatchBuf));
    if (e == cudaSuccess) e = cudaMemcpy(dc, &c, sizeof(CatchBuf), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) cudaFree(dc);
    if (e != cudaSuccess) {
        catch_free(c);
        s.err = std::string("capture buffer: ") + cudaGetErrorString(e);
        return QP_ERR_CUDA;
    }
    s.cat = c;
    s.d_cat = dc;
    return QP_OK;
}
}  // namespace qp

// Erasures recorded (catching_enabled) or not.  The buffer is shared with
// dump_photons; enabling allocates it anew with `capacity` records.
extern "C" int qp_set_catching(qp_handle* h, int enable, int64_t capacity) {
    if (!h) return QP_ERR_ARG;
    qp::State& s = *qp::state_of(h);
    cudaError_t e = cudaSetDevice(s.prm.device);
    if (e != cudaSuccess) { s.err = cudaGetErrorString(e); return QP_ERR_CUDA; }
    cudaStreamSynchronize(s.stream);
    if (!enable) {
        s.catch_erasures = false;
        if (!s.dump_photons) qp::catch_release(s);
        return QP_OK;
    }
    qp::catch_release(s);
    const int r = qp::catch_alloc(s, capacity);
    s.catch_erasures = r == QP_OK;
    return r;
}

// dump_photons (advance.cpp:302-306): photons emitted by leptons are deleted
// as they are born, into the capture buffer (allocated with `capacity`
// records if there is none), with their energy in qp_diag's erased energy.
extern "C" int qp_set_dump_photons(qp_handle* h, int enable, int64_t capacity) {
    if (!h) return QP_ERR_ARG;
    qp::State& s = *qp::state_of(h);
    cudaError_t e = cudaSetDevice(s.prm.device);
    if (e != cudaSuccess) { s.err = cudaGetErrorString(e); return QP_ERR_CUDA; }
    cudaStreamSynchronize(s.stream);
    if (!enable) {
        s.dump_photons = false;
        if (!s.catch_erasures) qp::catch_release(s);
        return QP_OK;
    }
    if (!s.prm.qed) { s.err = "dump_photons needs QED"; return QP_ERR_STATE; }
    if (!s.cat.counter) {
        const int r = qp::catch_alloc(s, capacity);
        if (r != QP_OK) return r;
    }
    s.dump_photons = true;
    return QP_OK;
}

extern "C" int qp_get_caught(qp_handle* h, int64_t cap, int32_t* species, double* x, double* y, double* z,
                             double* ux, double* uy, double* uz, double* g, double* q, double* chi, int64_t* n_out,
                             int64_t* dropped) {
    if (!h || !n_out) return QP_ERR_ARG;
    qp::State& s = *qp::state_of(h);
    cudaError_t e = cudaSetDevice(s.prm.device);
    if (e != cudaSuccess) { s.err = cudaGetErrorString(e); return QP_ERR_CUDA; }
    if (!s.cat.counter) { s.err = "catching is off"; return QP_ERR_STATE; }
    int cnt = 0;
    QP_CUDA_CHECK(s, cudaMemcpyAsync(&cnt, s.cat.counter, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    const int64_t m = std::min<int64_t>(cnt, s.cat.cap);
    *n_out = m;
    if (dropped) *dropped = cnt - m;
    double* out[9] = {x, y, z, ux, uy, uz, g, q, chi};
    bool any = species != nullptr;
    for (double* p : out) any = any || p != nullptr;
    if (!any) return QP_OK;  // count only; the buffer is kept
    if (cap < m) { s.err = "output arrays shorter than the caught records"; return QP_ERR_ARG; }
    // host copies, ordered by species, then step, phase and traversal position
    std::vector<int64_t> key(m);
    std::vector<int32_t> sp(m);
    if (m > 0) {
        QP_CUDA_CHECK(s, cudaMemcpy(key.data(), s.cat.key, m * sizeof(int64_t), cudaMemcpyDeviceToHost));
        QP_CUDA_CHECK(s, cudaMemcpy(sp.data(), s.cat.sp, m * sizeof(int32_t), cudaMemcpyDeviceToHost));
    }
    std::vector<int64_t> order(m);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
        return sp[a] != sp[b] ? sp[a] < sp[b] : key[a] < key[b];
    });
    if (species) {
        std::vector<int32_t> t(m);
        for (int64_t i = 0; i < m; i++) t[i] = sp[order[i]];
        if (m > 0) QP_CUDA_CHECK(s, cudaMemcpy(species, t.data(), m * sizeof(int32_t), cudaMemcpyDefault));
    }
    const double* src[9] = {s.cat.x, s.cat.y, s.cat.z, s.cat.ux, s.cat.uy, s.cat.uz, s.cat.g, s.cat.q, s.cat.chi};
    std::vector<double> a(m), t(m);
    for (int k = 0; k < 9; k++) {
        if (!out[k] || m == 0) continue;
        QP_CUDA_CHECK(s, cudaMemcpy(a.data(), src[k], m * sizeof(double), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < m; i++) t[i] = a[order[i]];
        QP_CUDA_CHECK(s, cudaMemcpy(out[k], t.data(), m * sizeof(double), cudaMemcpyDefault));
    }
    QP_CUDA_CHECK(s, cudaMemset(s.cat.counter, 0, sizeof(int)));
    return QP_OK;
}
