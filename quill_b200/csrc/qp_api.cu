// C ABI of libquill_b200 (include/quill_b200.h): host-side orchestration of
// one region on one GPU.  Each call maps onto the spatial_region member or
// main() code it replaces (cited per function).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "qp_internal.h"
#include "qp_fields.cuh"

#define QP_VERSION_STRING "quill_b200 0.1 (sm_100a)"

namespace qp {

SolverCoef solver_coef(const qp_params& p) {
    const double PI = 3.141592653589793;
    SolverCoef c;
    // maxwell.cpp:6-8
    c.dtdx = p.dt / p.dx;
    c.dtdy = p.dt / p.dy;
    c.dtdz = p.dt / p.dz;
    c.dx = p.dx; c.dy = p.dy; c.dz = p.dz;
    // five-point, maxwell.cpp:24-33
    c.fax = 0.25 * (1 - p.dx / p.dt * std::sin(0.5 * PI * std::min(1.0, p.dt / p.dx)));
    c.fay = 0.25 * (1 - p.dy / p.dt * std::sin(0.5 * PI * std::min(1.0, p.dt / p.dy)));
    c.faz = 0.25 * (1 - p.dz / p.dt * std::sin(0.5 * PI * std::min(1.0, p.dt / p.dz)));
    c.fbx = 1 - 2 * c.fax;
    c.fby = 1 - 2 * c.fay;
    c.fbz = 1 - 2 * c.faz;
    // NDFX, maxwell.cpp:238-249
    const double kappa = 1.25 * (std::sqrt(3.0) - 1) * 0.5 / std::sqrt(3.0);
    c.nbx = (1 - kappa);
    c.nax = 0.5 * (1 - c.nbx);
    c.nby = 1 - kappa * p.dx * p.dx / (p.dy * p.dy);
    c.nbz = 1 - kappa * p.dx * p.dx / (p.dz * p.dz);
    c.nay = 0.5 * (1 - c.nby);
    c.naz = 0.5 * (1 - c.nbz);
    return c;
}

void zero_planes_fp64(State& s, const ZeroPlane* zp, int n);
void zero_planes_mixed(State& s, const ZeroPlane* zp, int n);
int load_merge(State& s, int si, int64_t slot0, const int32_t* d_new_start, int32_t* d_perm_out);

static int n_arrays(const State& s) { return s.fp64 ? 9 : 10; }

// New particles at slots [slot0, slot0 + n_new) of the current buffer, sorted
// by cell (cells in d_cells, device): per-cell counts -> starts -> merged in
// front of the particles already in each cell (head insertion order).
static int merge_sorted_slots(State& s, int si, int64_t slot0, int64_t n_new, const int32_t* d_cells) {
    Species& sp = s.sp[si];
    const Grid gr = s.grid;
    // the merged permutation goes to sp.newcell (free between steps; d_cells
    // is never a part of it), which then becomes sp.perm
    int32_t* nstart = nullptr;
    QP_CUDA_CHECK(s, scratch_alloc(s, (void**)&nstart, (size_t)(gr.nc + 1) * sizeof(int32_t)));
    launch_histogram(s, d_cells, (int)n_new, sp.count);
    exclusive_scan_i32(s, sp.count, nstart, gr.nc);
    if (sp.trn[sp.cur]) QP_CUDA_CHECK(s, cudaMemsetAsync(sp.trn[sp.cur] + slot0, 0, n_new * sizeof(int32_t), s.stream));
    load_merge(s, si, slot0, nstart, sp.newcell);
    scratch_free(s, nstart);
    QP_CUDA_CHECK(s, cudaGetLastError());
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    std::swap(sp.perm, sp.newcell);
    sp.n += n_new;
    sp.slots = slot0 + n_new;
    s.layout_epoch++;
    return QP_OK;
}
static size_t arr_elem(const State& s, int a) { return s.fp64 ? 8 : 4; }

// Allocate (or grow, keeping contents) the particle arrays of a species.
cudaError_t scratch_alloc(State& s, void** p, size_t bytes) {
    if (!s.pool) {
        cudaMemPoolProps pr = {};
        pr.allocType = cudaMemAllocationTypePinned;
        pr.location.type = cudaMemLocationTypeDevice;
        pr.location.id = s.prm.device;
        cudaError_t e = cudaMemPoolCreate(&s.pool, &pr);
        if (e != cudaSuccess) {
            s.pool = nullptr;
            return e;
        }
        unsigned long long keep = ~0ull;
        e = cudaMemPoolSetAttribute(s.pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
    }
    return cudaMallocFromPoolAsync(p, bytes, s.pool, s.stream);
}

void scratch_free(State& s, void* p) {
    if (p) cudaFreeAsync(p, s.stream);
}

int ensure_capacity(State& s, int si, int64_t need) {
    Species& sp = s.sp[si];
    if (need <= sp.cap) return QP_OK;
    if (need >= (int64_t)INT32_MAX) {
        s.err = "particle count exceeds 2^31-1 per species";
        return QP_ERR_CAPACITY;
    }
    int64_t cap = std::max<int64_t>(need, sp.cap + sp.cap / 2);
    cap = std::min<int64_t>(cap, (int64_t)INT32_MAX - 1);
    const int na = n_arrays(s);
    // Every caller runs between steps: the live particles are slots
    // [0, sp.slots) of buf[cur] (perm: positions [0, n)); buf[1 - cur] is
    // the next push's output and holds nothing to keep.
    for (int b = 0; b < 2; b++)
        for (int a = 0; a < na; a++) {
            if (s.fp64 && a == 8 && !s.prm.qed) continue;   // chi only with QED
            if (!s.fp64 && a == 9 && !s.prm.qed) continue;
            void* p = nullptr;
            QP_CUDA_CHECK(s, cudaMalloc(&p, cap * arr_elem(s, a)));
            if (sp.buf[b][a]) {
                if (b == sp.cur && sp.slots > 0)
                    QP_CUDA_CHECK(s, cudaMemcpyAsync(p, sp.buf[b][a], sp.slots * arr_elem(s, a), cudaMemcpyDeviceToDevice, s.stream));
                QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
                cudaFree(sp.buf[b][a]);
            }
            sp.buf[b][a] = p;
        }
    int32_t* np = nullptr;
    QP_CUDA_CHECK(s, cudaMalloc(&np, cap * sizeof(int32_t)));
    if (sp.perm) {
        if (sp.n > 0)
            QP_CUDA_CHECK(s, cudaMemcpyAsync(np, sp.perm, sp.n * sizeof(int32_t), cudaMemcpyDeviceToDevice, s.stream));
        QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
        cudaFree(sp.perm);
    }
    sp.perm = np;
    if (sp.newcell) cudaFree(sp.newcell);
    QP_CUDA_CHECK(s, cudaMalloc(&sp.newcell, cap * sizeof(int32_t)));
    if (s.tracking)
        for (int b = 0; b < 2; b++) {
            int32_t* t = nullptr;
            QP_CUDA_CHECK(s, cudaMalloc(&t, cap * sizeof(int32_t)));
            QP_CUDA_CHECK(s, cudaMemsetAsync(t, 0, cap * sizeof(int32_t), s.stream));
            if (sp.trn[b]) {
                if (b == sp.cur && sp.slots > 0)
                    QP_CUDA_CHECK(s, cudaMemcpyAsync(t, sp.trn[b], sp.slots * sizeof(int32_t), cudaMemcpyDeviceToDevice, s.stream));
                QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
                cudaFree(sp.trn[b]);
            }
            sp.trn[b] = t;
        }
    sp.cap = cap;
    // the rebin's list of long cells: at most cap / (REBIN_LONG_SEG + 1)
    const int64_t need_long = cap / (REBIN_LONG_SEG + 1) + 2;
    if (s.long_cap < need_long) {
        cudaFree(s.long_list);
        s.long_list = nullptr;
        s.long_cap = 0;
        QP_CUDA_CHECK(s, cudaMalloc(&s.long_list, need_long * sizeof(int32_t)));
        s.long_cap = need_long;
    }
    return QP_OK;
}

// Release every device and pinned allocation of a region.
static void free_state(State* s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    cudaFree(s->fields);
    for (auto& sp : s->sp) {
        for (int b = 0; b < 2; b++)
            for (int a = 0; a < 10; a++) cudaFree(sp.buf[b][a]);
        cudaFree(sp.perm);
        cudaFree(sp.newcell);
        cudaFree(sp.trn[0]);
        cudaFree(sp.trn[1]);
        cudaFree(sp.cell_start);
        cudaFree(sp.cell_next);
        cudaFree(sp.count);
        cudaFree(sp.d_counter);
    }
    for (auto& sn : s->snap) {
        cudaFree(sn.fields);
        for (auto& v : sn.arrays)
            for (void* p : v) cudaFree(p);
        for (auto* p : sn.cell_start) cudaFree(p);
    }
    cudaFree(s->d_diag);
    cudaFreeHost(s->h_diag);
    cudaFreeHost(s->h_count);
    cudaFree(s->d_status);
    cudaFree(s->long_list);
    cudaFree(s->window_scratch);
    catch_release(*s);
    ordered_release(*s);
    s->window_scratch = nullptr;
    s->long_list = nullptr;
    cudaFree(s->scan_tmp);
    for (auto& e : s->ev)
        if (e) cudaEventDestroy(e);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    s->stream = nullptr;
    if (s->pool) cudaMemPoolDestroy(s->pool);
    s->pool = nullptr;
}

int snapshot_take(State& s, State::Snap& sn) {
    const size_t nc = (size_t)s.grid.nc;
    if (!sn.fields) QP_CUDA_CHECK(s, cudaMalloc(&sn.fields, 12 * nc * s.field_elem));
    for (int a = 0; a < 12; a++)
        QP_CUDA_CHECK(s, cudaMemcpyAsync((char*)sn.fields + a * nc * s.field_elem, s.plane[a], nc * s.field_elem,
                                         cudaMemcpyDeviceToDevice, s.stream));
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    for (auto& v : sn.arrays)
        for (void* p : v) cudaFree(p);
    sn.arrays.assign(s.sp.size(), std::vector<void*>(12, nullptr));
    sn.n.assign(s.sp.size(), 0);
    sn.cap.assign(s.sp.size(), 0);
    sn.slots.assign(s.sp.size(), 0);
    sn.cell_start.resize(s.sp.size(), nullptr);
    for (size_t i = 0; i < s.sp.size(); i++) {
        Species& sp = s.sp[i];
        const int64_t cap = sp.cap;
        sn.cap[i] = cap;
        sn.n[i] = sp.n;
        sn.slots[i] = sp.slots;
        if (cap > 0) {
            for (int a = 0; a < 10; a++) {
                if (!sp.buf[sp.cur][a]) continue;
                QP_CUDA_CHECK(s, cudaMalloc(&sn.arrays[i][a], cap * arr_elem(s, a)));
                QP_CUDA_CHECK(s, cudaMemcpyAsync(sn.arrays[i][a], sp.buf[sp.cur][a], cap * arr_elem(s, a), cudaMemcpyDeviceToDevice, s.stream));
            }
            QP_CUDA_CHECK(s, cudaMalloc(&sn.arrays[i][10], cap * 4));
            QP_CUDA_CHECK(s, cudaMemcpyAsync(sn.arrays[i][10], sp.perm, cap * 4, cudaMemcpyDeviceToDevice, s.stream));
            if (sp.trn[sp.cur]) {
                QP_CUDA_CHECK(s, cudaMalloc(&sn.arrays[i][11], cap * 4));
                QP_CUDA_CHECK(s, cudaMemcpyAsync(sn.arrays[i][11], sp.trn[sp.cur], cap * 4, cudaMemcpyDeviceToDevice, s.stream));
            }
        }
        if (!sn.cell_start[i]) QP_CUDA_CHECK(s, cudaMalloc(&sn.cell_start[i], (nc + 1) * 4));
        QP_CUDA_CHECK(s, cudaMemcpyAsync(sn.cell_start[i], sp.cell_start, (nc + 1) * 4, cudaMemcpyDeviceToDevice, s.stream));
    }
    sn.step_index = s.step_index;
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    sn.valid = true;
    return QP_OK;
}

int snapshot_restore(State& s, State::Snap& sn) {
    if (!sn.valid) { s.err = "checkpoint slot is empty"; return QP_ERR_STATE; }
    const size_t nc = (size_t)s.grid.nc;
    for (int a = 0; a < 12; a++)
        QP_CUDA_CHECK(s, cudaMemcpyAsync(s.plane[a], (char*)sn.fields + a * nc * s.field_elem, nc * s.field_elem,
                                         cudaMemcpyDeviceToDevice, s.stream));
    for (size_t i = 0; i < s.sp.size(); i++) {
        Species& sp = s.sp[i];
        const int64_t cap = sn.cap[i];
        int r = ensure_capacity(s, (int)i, cap);
        if (r != QP_OK) return r;
        if (cap > 0) {
            for (int a = 0; a < 10; a++) {
                if (!sp.buf[sp.cur][a] || !sn.arrays[i][a]) continue;
                QP_CUDA_CHECK(s, cudaMemcpyAsync(sp.buf[sp.cur][a], sn.arrays[i][a], cap * arr_elem(s, a), cudaMemcpyDeviceToDevice, s.stream));
            }
            QP_CUDA_CHECK(s, cudaMemcpyAsync(sp.perm, sn.arrays[i][10], cap * 4, cudaMemcpyDeviceToDevice, s.stream));
            if (sp.trn[sp.cur] && sn.arrays[i].size() > 11 && sn.arrays[i][11])
                QP_CUDA_CHECK(s, cudaMemcpyAsync(sp.trn[sp.cur], sn.arrays[i][11], cap * 4, cudaMemcpyDeviceToDevice, s.stream));
        }
        QP_CUDA_CHECK(s, cudaMemcpyAsync(sp.cell_start, sn.cell_start[i], (nc + 1) * 4, cudaMemcpyDeviceToDevice, s.stream));
        sp.n = sn.n[i];
        sp.slots = sn.slots[i];
    }
    s.layout_epoch++;
    s.step_index = sn.step_index;
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    return QP_OK;
}

void snapshot_free(State::Snap& sn) {
    cudaFree(sn.fields);
    sn.fields = nullptr;
    for (auto& v : sn.arrays)
        for (void* p : v) cudaFree(p);
    sn.arrays.clear();
    for (auto* p : sn.cell_start) cudaFree(p);
    sn.cell_start.clear();
    sn.valid = false;
}

}  // namespace qp

struct qp_handle {
    qp::State st;
};

qp::State* qp::state_of(qp_handle* h) { return &h->st; }

using namespace qp;

static thread_local std::string g_create_error;

namespace qp {
cudaError_t launch_qed_rates(int n, const double* d_in, double* d_out, double e_s, cudaStream_t st);
// Message for qp_last_error(NULL) from entry points without a handle.
void set_global_error(const std::string& msg) { g_create_error = msg; }
}

#define QP_H_CHECK(h)                              \
    do {                                           \
        if (!(h)) return QP_ERR_ARG;               \
        cudaError_t e0 = cudaSetDevice((h)->st.prm.device); \
        if (e0 != cudaSuccess) {                   \
            (h)->st.err = cudaGetErrorString(e0);  \
            return QP_ERR_CUDA;                    \
        }                                          \
    } while (0)

extern "C" {

const char* qp_version(void) { return QP_VERSION_STRING; }

const char* qp_last_error(const qp_handle* h) {
    if (!h) return g_create_error.c_str();
    return h->st.err.c_str();
}

int qp_create(const qp_params* prm, qp_handle** out) {
    if (!prm || !out) { g_create_error = "null argument"; return QP_ERR_ARG; }
    *out = nullptr;
    const qp_params& p = *prm;
    auto bad = [&](const char* m) { g_create_error = m; return QP_ERR_CONFIG; };
    if (p.nx < 5 || p.ny < 5 || p.nz < 5) return bad("grid must have at least 5 cells per axis");
    if ((int64_t)p.nx * p.ny * p.nz >= (int64_t)INT32_MAX - 1) return bad("grid exceeds 2^31 cells");
    if (!(p.dx > 0 && p.dy > 0 && p.dz > 0 && p.dt > 0)) return bad("dx, dy, dz, dt must be positive");
    // a particle must not move more than one cell per axis and step
    if (!(p.dt < p.dx && p.dt < p.dy && p.dt < p.dz)) return bad("dt must be smaller than dx, dy and dz");
    if (p.solver < 0 || p.solver > 2) return bad("unknown solver");
    if (p.pusher < 0 || p.pusher > 1) return bad("unknown pusher");
    if (p.precision < 0 || p.precision > 1) return bad("unknown precision");
    if (p.n_species < 0 || p.n_species > QP_MAX_SPECIES) return bad("n_species out of range");
    if (!(p.lambda_cm > 0)) return bad("lambda_cm must be positive");
    if (p.qed) {
        bool has_e = false, has_p = false, has_ph = false;
        for (int i = 0; i < p.n_species; i++) {
            has_e |= p.cmr[i] == -1;
            has_p |= p.cmr[i] == 1;
            has_ph |= p.cmr[i] == 0;
        }
        if (!(has_e && has_p && has_ph)) return bad("QED needs species with cmr -1, +1 and 0");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_create_error = "no CUDA device";
        return QP_ERR_CUDA;
    }
    if (p.device < 0 || p.device >= ndev) return bad("device ordinal out of range");
    qp_handle* h = new qp_handle();
    State& s = h->st;
    s.prm = p;
    s.fp64 = p.precision == QP_PREC_FP64;
    s.grid.nx = p.nx; s.grid.ny = p.ny; s.grid.nz = p.nz;
    s.grid.nynz = p.ny * p.nz;
    s.grid.nc = p.nx * p.ny * p.nz;
    s.grid.div_nz.init((uint32_t)p.nz);
    s.diag_lo = 0;
    s.diag_hi = p.nx;
    s.grid.div_nynz.init((uint32_t)(p.ny * p.nz));
    s.field_elem = s.fp64 ? 8 : 4;
    if (const char* v = getenv("QP_PREFETCH")) s.prefetch = atoi(v) != 0;
    if (const char* v = getenv("QP_PUSH_SHAPE")) {
        const int i = atoi(v);
        if (i >= 0 && i < n_push_shapes64) s.push_shape = i;
    }
    if (const char* v = getenv("QP_PUSH_SHAPE_MIXED")) {
        const int i = atoi(v);
        if (i >= 0 && i < n_push_shapes32) s.push_shape_mixed = i;
    }
    if (const char* w = getenv("QP_PUSH_WAVES"))
        s.push_waves = s.push_waves_mixed = s.push_waves_qed = atoi(w) > 0 ? atoi(w) : 0;
    {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p.device) == cudaSuccess && sms > 0)
            s.sm_count = sms;
    }
    cudaError_t e = cudaSetDevice(p.device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
    s.own_stream = true;
    const size_t nc = (size_t)s.grid.nc;
    if (e == cudaSuccess) e = cudaMalloc(&s.fields, 12 * nc * s.field_elem);
    if (e == cudaSuccess) e = cudaMemsetAsync(s.fields, 0, 12 * nc * s.field_elem, s.stream);
    if (e == cudaSuccess)
        for (int a = 0; a < 12; a++) s.plane[a] = (char*)s.fields + a * nc * s.field_elem;
    if (e == cudaSuccess) e = cudaMalloc(&s.d_diag, sizeof(DiagAccum));
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&s.h_diag, sizeof(DiagAccum), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&s.h_count, QP_MAX_SPECIES * sizeof(int32_t), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMalloc(&s.d_status, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemsetAsync(s.d_status, 0, sizeof(unsigned int), s.stream);
    s.scan_tmp_bytes = ((nc + 4095) / 4096 + 2) * sizeof(int32_t);
    if (e == cudaSuccess) e = cudaMalloc(&s.scan_tmp, s.scan_tmp_bytes);
    int ion = 0;
    s.sp.resize(p.n_species);
    for (int i = 0; i < p.n_species && e == cudaSuccess; i++) {
        Species& sp = s.sp[i];
        sp.cmr = p.cmr[i];
        sp.kind = p.cmr[i] == 0 ? KIND_PHOTON : (std::fabs(p.cmr[i]) == 1 ? KIND_LEPTON : KIND_ION);
        sp.ion_index = sp.kind == KIND_ION ? ion++ : -1;
        if (sp.cmr == -1 && s.sp_e < 0) s.sp_e = i;
        if (sp.cmr == 1 && s.sp_p < 0) s.sp_p = i;
        if (sp.cmr == 0 && s.sp_ph < 0) s.sp_ph = i;
        if (p.qed) {
            if (e == cudaSuccess) e = cudaMalloc(&sp.d_counter, sizeof(int));
            if (e == cudaSuccess) e = cudaMemsetAsync(sp.d_counter, 0, sizeof(int), s.stream);
        }
        e = cudaMalloc(&sp.cell_start, (nc + 1) * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMemsetAsync(sp.cell_start, 0, (nc + 1) * sizeof(int32_t), s.stream);
        if (e == cudaSuccess) e = cudaMalloc(&sp.cell_next, (nc + 1) * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMalloc(&sp.count, nc * sizeof(int32_t));
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
    if (e != cudaSuccess) {
        g_create_error = std::string("qp_create: ") + cudaGetErrorString(e);
        free_state(&h->st);
        delete h;
        return QP_ERR_CUDA;
    }
    for (int i = 0; i < p.n_species; i++) {
        int64_t c = p.capacity[i];
        if (c > 0) {
            int r = ensure_capacity(s, i, c);
            if (r != QP_OK) {
                g_create_error = s.err;
                free_state(&h->st);
                delete h;
                return r;
            }
        }
    }
    *out = h;
    return QP_OK;
}

int qp_destroy(qp_handle* h) {
    if (!h) return QP_OK;
    cudaSetDevice(h->st.prm.device);
    free_state(&h->st);
    delete h;
    return QP_OK;
}

int qp_set_stream(qp_handle* h, void* stream) {
    QP_H_CHECK(h);
    State& s = h->st;
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    if (stream) {
        if (s.own_stream) cudaStreamDestroy(s.stream);
        s.stream = (cudaStream_t)stream;
        s.own_stream = false;
    }
    return QP_OK;
}

int qp_synchronize(qp_handle* h) {
    QP_H_CHECK(h);
    QP_CUDA_CHECK(h->st, cudaStreamSynchronize(h->st.stream));
    return QP_OK;
}

int qp_eval_qed_rates(int device, double lambda_cm, int64_t n, const double* in, double* out) {
    if (n < 0 || (n > 0 && (!in || !out)) || n > (int64_t)INT32_MAX / 12) return QP_ERR_ARG;
    if (n == 0) return QP_OK;
    if (cudaSetDevice(device) != cudaSuccess) return QP_ERR_CUDA;
    double *din = nullptr, *dout = nullptr;
    cudaError_t e = cudaMalloc(&din, n * 12 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dout, n * 5 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(din, in, n * 12 * sizeof(double), cudaMemcpyDefault);
    if (e == cudaSuccess) e = launch_qed_rates((int)n, din, dout, lambda_cm / 2.4263086e-10, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, n * 5 * sizeof(double), cudaMemcpyDefault);
    cudaFree(din);
    cudaFree(dout);
    if (e != cudaSuccess) {
        g_create_error = cudaGetErrorString(e);
        return QP_ERR_CUDA;
    }
    return QP_OK;
}

int qp_set_erased_tracking(qp_handle* h, int enable) {
    QP_H_CHECK(h);
    h->st.track_erased = enable != 0;
    return QP_OK;
}

int qp_set_timing(qp_handle* h, int enable) {
    QP_H_CHECK(h);
    State& s = h->st;
    if (enable && !s.ev[0])
        for (auto& e : s.ev) QP_CUDA_CHECK(s, cudaEventCreate(&e));
    s.timing = enable != 0;
    for (double& v : s.phase_ms) v = 0;
    s.phase_steps = 0;
    for (double& v : s.qed_ms) v = 0;
    s.qed_steps = 0;
    return QP_OK;
}

int qp_get_qed_timing(qp_handle* h, double* ms3, int64_t* steps) {
    if (!h || !ms3) return QP_ERR_ARG;
    for (int i = 0; i < 3; i++) ms3[i] = h->st.qed_ms[i];
    if (steps) *steps = h->st.qed_steps;
    return QP_OK;
}

int qp_get_timing(qp_handle* h, double* ms4, int64_t* steps) {
    if (!h || !ms4) return QP_ERR_ARG;
    for (int i = 0; i < 4; i++) ms4[i] = h->st.phase_ms[i];
    if (steps) *steps = h->st.phase_steps;
    return QP_OK;
}

int qp_launch_count(qp_handle* h, int64_t* out) {
    if (!h || !out) return QP_ERR_ARG;
    *out = h->st.launches;
    return QP_OK;
}

int qp_load_fields(qp_handle* h, const double* ex, const double* ey, const double* ez, const double* bx,
                   const double* by, const double* bz) {
    QP_H_CHECK(h);
    State& s = h->st;
    if (!ex || !ey || !ez || !bx || !by || !bz) { s.err = "null field plane"; return QP_ERR_ARG; }
    const size_t nc = (size_t)s.grid.nc;
    const double* src[6] = {ex, ey, ez, bx, by, bz};
    // host or device planes (unified addressing decides the copy direction)
    if (s.fp64) {
        for (int a = 0; a < 6; a++)
            QP_CUDA_CHECK(s, cudaMemcpyAsync(s.plane[a], src[a], nc * 8, cudaMemcpyDefault, s.stream));
    } else {
        double* stage = nullptr;
        QP_CUDA_CHECK(s, cudaMalloc(&stage, nc * 8));
        for (int a = 0; a < 6; a++) {
            QP_CUDA_CHECK(s, cudaMemcpyAsync(stage, src[a], nc * 8, cudaMemcpyDefault, s.stream));
            launch_f64_to_f32(s, stage, (float*)s.plane[a], nc);
        }
        QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
        cudaFree(stage);
    }
    QP_CUDA_CHECK(s, cudaGetLastError());
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    s.boundaries_done = false;
    return QP_OK;
}

int qp_init_boundaries(qp_handle* h) {
    QP_H_CHECK(h);
    State& s = h->st;
    const int nx = s.grid.nx, ny = s.grid.ny, nz = s.grid.nz;
    const int ALL = 63, EX = 1, EY = 2, EZ = 4, BX = 8, BY = 16, BZ = 32;
    std::vector<ZeroPlane> zp;
    if (s.prm.solver == QP_SOLVER_FDTD) {  // maxwell.cpp:532-597
        zp = {{0, 0, EY | EZ | BX}, {0, nx - 1, ALL}, {1, 0, EX | EZ | BY}, {1, ny - 1, ALL},
              {2, 0, EY | EX | BZ}, {2, nz - 1, ALL}};
    } else if (s.prm.solver == QP_SOLVER_NDFX) {  // maxwell.cpp:338-438
        zp = {{0, 0, ALL}, {0, 1, EY | EZ | BX}, {0, nx - 1, ALL}, {1, 0, ALL}, {1, 1, EX | EZ | BY},
              {1, ny - 1, ALL}, {2, 0, ALL}, {2, 1, EY | EX | BZ}, {2, nz - 1, ALL}};
    } else {  // maxwell.cpp:135-236
        zp = {{0, 0, ALL}, {1, 0, ALL}, {2, 0, ALL}, {0, nx - 1, ALL}, {1, ny - 1, ALL}, {2, nz - 1, ALL},
              {0, nx - 2, BY | BZ}, {0, 1, EZ | EY}, {1, ny - 2, BX | BZ}, {1, 1, EX | EZ},
              {2, nz - 2, BX | BY}, {2, 1, EX | EY}};
    }
    if (s.fp64) {
        zero_planes_fp64(s, zp.data(), (int)zp.size());
        launch_fields_fp64(s, 3);
    } else {
        zero_planes_mixed(s, zp.data(), (int)zp.size());
        launch_fields_mixed(s, 3);
    }
    QP_CUDA_CHECK(s, cudaGetLastError());
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    s.boundaries_done = true;
    return QP_OK;
}

// Host fallback for input that is not in cell order: gather to the host,
// stable counting sort by cell (the given order is kept inside a cell) and
// load again in sorted order.
static int load_unsorted(qp_handle* h, int si, int64_t n, const double* const* src);

}  // extern "C"

// Copy n particles into slots [sp.slots, sp.slots + n) of the current
// buffer (FP64 straight into the slots, mixed precision through an FP64
// stage), write their cells into `cells` and flag invalid ones (LD_INVALID
// into *flags, the first bad index into *first_bad).  Stream-ordered; the
// caller synchronises before reading the flags.
int qp::stage_particles(State& s, int si, int64_t n, const double* const* src, int32_t* cells,
                        unsigned int* flags, int* first_bad) {
    Species& sp = s.sp[si];
    const int64_t slot0 = sp.slots;
    const int cur = sp.cur;
    if (s.fp64) {
        for (int a = 0; a < 9; a++) {
            if (!sp.buf[cur][a]) continue;
            double* dst = (double*)sp.buf[cur][a] + slot0;
            if (src[a]) QP_CUDA_CHECK(s, cudaMemcpyAsync(dst, src[a], n * 8, cudaMemcpyDefault, s.stream));
            else QP_CUDA_CHECK(s, cudaMemsetAsync(dst, 0, n * 8, s.stream));
        }
        const double* st[8];
        for (int a = 0; a < 8; a++) st[a] = (const double*)sp.buf[cur][a] + slot0;
        launch_load_cells(s, st, (int)n, cells, flags, first_bad, 0);
        return QP_OK;
    }
    const int64_t CH = std::min<int64_t>(n, 1 << 24);
    double* stage = nullptr;
    QP_CUDA_CHECK(s, scratch_alloc(s, (void**)&stage, CH * 9 * sizeof(double)));
    PStore32 dst;
    dst.cell = (int32_t*)sp.buf[cur][0];
    float** pd[9] = {&dst.ox, &dst.oy, &dst.oz, &dst.ux, &dst.uy, &dst.uz, &dst.g, &dst.q, &dst.chi};
    for (int a = 0; a < 9; a++) *pd[a] = (float*)sp.buf[cur][1 + a];
    for (int64_t c0 = 0; c0 < n; c0 += CH) {
        const int64_t m = std::min<int64_t>(CH, n - c0);
        const double* st[9];
        for (int a = 0; a < 9; a++) {
            double* d = stage + a * CH;
            cudaError_t e = src[a] ? cudaMemcpyAsync(d, src[a] + c0, m * 8, cudaMemcpyDefault, s.stream)
                                   : cudaMemsetAsync(d, 0, m * 8, s.stream);
            if (e != cudaSuccess) {
                scratch_free(s, stage);
                s.err = cudaGetErrorString(e);
                return QP_ERR_CUDA;
            }
            st[a] = d;
        }
        launch_load_cells(s, st, (int)m, cells, flags, first_bad, (int)c0);
        launch_to_mixed(s, st, (int)m, dst, (int)(slot0 + c0));
    }
    scratch_free(s, stage);
    return QP_OK;
}

extern "C" {

int qp_load_particles(qp_handle* h, int si, int64_t n, const double* x, const double* y, const double* z,
                      const double* ux, const double* uy, const double* uz, const double* g, const double* q,
                      const double* chi) {
    QP_H_CHECK(h);
    State& s = h->st;
    if (si < 0 || si >= (int)s.sp.size()) { s.err = "species index out of range"; return QP_ERR_ARG; }
    if (n < 0) { s.err = "negative particle count"; return QP_ERR_ARG; }
    if (n == 0) return QP_OK;
    if (!x || !y || !z || !ux || !uy || !uz || !g || !q) { s.err = "null particle array"; return QP_ERR_ARG; }
    Species& sp = s.sp[si];
    const int64_t slot0 = sp.slots;
    if (slot0 + n >= (int64_t)INT32_MAX) { s.err = "particle count exceeds 2^31-1"; return QP_ERR_CAPACITY; }
    int r = ensure_capacity(s, si, slot0 + n);
    if (r != QP_OK) return r;
    const double* src[9] = {x, y, z, ux, uy, uz, g, q, chi};
    // scratch: cells (n), flags, first bad index, per-cell counts and starts
    int32_t* cells = nullptr;
    unsigned int* flags = nullptr;
    int* first_bad = nullptr;
    QP_CUDA_CHECK(s, scratch_alloc(s, (void**)&cells, n * sizeof(int32_t)));
    if (cudaError_t e = scratch_alloc(s, (void**)&flags, sizeof(unsigned int) + sizeof(int)); e != cudaSuccess) {
        scratch_free(s, cells);
        s.err = cudaGetErrorString(e);
        return QP_ERR_CUDA;
    }
    first_bad = (int*)(flags + 1);
    QP_CUDA_CHECK(s, cudaMemsetAsync(flags, 0, sizeof(unsigned int), s.stream));
    QP_CUDA_CHECK(s, cudaMemsetAsync(first_bad, 0x7f, sizeof(int), s.stream));
    if ((r = stage_particles(s, si, n, src, cells, flags, first_bad)) != QP_OK) {
        scratch_free(s, cells);
        scratch_free(s, flags);
        return r;
    }
    launch_check_sorted(s, cells, (int)n, flags);
    unsigned int hf[2] = {0, 0};
    QP_CUDA_CHECK(s, cudaMemcpyAsync(hf, flags, 2 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s.stream));
    QP_CUDA_CHECK(s, cudaGetLastError());
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    auto release = [&]() { scratch_free(s, cells); scratch_free(s, flags); };
    if (hf[0] & 1) {
        release();
        char b[160];
        snprintf(b, sizeof b, "particle %d outside the grid [0, n) or not finite", (int)hf[1]);
        s.err = b;
        return QP_ERR_CONFIG;
    }
    if (hf[0] & 2) {
        release();
        return load_unsorted(h, si, n, src);
    }
    int rm = merge_sorted_slots(s, si, slot0, n, cells);
    release();
    return rm;
}

static int load_unsorted(qp_handle* h, int si, int64_t n, const double* const* src) {
    State& s = h->st;
    const Grid gr = s.grid;
    std::vector<std::vector<double>> a(9);
    for (int k = 0; k < 9; k++) {
        if (!src[k]) continue;
        a[k].resize(n);
        QP_CUDA_CHECK(s, cudaMemcpy(a[k].data(), src[k], n * 8, cudaMemcpyDefault));
    }
    std::vector<int32_t> cell(n);
    for (int64_t p = 0; p < n; p++) cell[p] = ((int)a[0][p] * gr.ny + (int)a[1][p]) * gr.nz + (int)a[2][p];
    std::vector<int64_t> start(gr.nc + 1, 0);
    for (int64_t p = 0; p < n; p++) start[cell[p] + 1]++;
    for (int c = 0; c < gr.nc; c++) start[c + 1] += start[c];
    std::vector<int64_t> order(n);
    for (int64_t p = 0; p < n; p++) order[start[cell[p]]++] = p;
    std::vector<std::vector<double>> b(9);
    const double* ptr[9] = {nullptr};
    for (int k = 0; k < 9; k++) {
        if (a[k].empty()) continue;
        b[k].resize(n);
        for (int64_t t = 0; t < n; t++) b[k][t] = a[k][order[t]];
        ptr[k] = b[k].data();
    }
    return qp_load_particles(h, si, n, ptr[0], ptr[1], ptr[2], ptr[3], ptr[4], ptr[5], ptr[6], ptr[7], ptr[8]);
}

// Before a QED step: make room for every particle a push can create (a
// photon per lepton, a pair per photon), then birth_from_vacuum: pairs
// written to free slots of the current e-/e+ buffers, sorted by cell on the
// host (they are rare) and merged at the head of their cells.
static int qed_prepare(State& s) {
    const int e = s.sp_e, p = s.sp_p, ph = s.sp_ph;
    int64_t nlep = 0;
    for (auto& sp : s.sp)
        if (sp.kind == KIND_LEPTON) nlep += sp.n;
    const int64_t nph = s.sp[ph].n;
    int r;
    if ((r = ensure_capacity(s, ph, std::max(s.sp[ph].slots, nph + nlep) + 1)) != QP_OK) return r;
    if ((r = ensure_capacity(s, e, std::max(s.sp[e].slots, s.sp[e].n + nph) + 1024)) != QP_OK) return r;
    if ((r = ensure_capacity(s, p, std::max(s.sp[p].slots, s.sp[p].n + nph) + 1024)) != QP_OK) return r;
    for (auto& sp : s.sp)
        if (sp.d_counter) QP_CUDA_CHECK(s, cudaMemsetAsync(sp.d_counter, 0, sizeof(int), s.stream));
    if (s.fp64) launch_vacuum_fp64(s);
    else launch_vacuum_mixed(s);
    int kv[2] = {0, 0};
    QP_CUDA_CHECK(s, cudaMemcpyAsync(&kv[0], s.sp[e].d_counter, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
    QP_CUDA_CHECK(s, cudaMemcpyAsync(&kv[1], s.sp[p].d_counter, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    const int who[2] = {e, p};
    for (int w = 0; w < 2; w++) {
        Species& sp = s.sp[who[w]];
        const int64_t k = std::min<int64_t>(kv[w], sp.cap - sp.slots);
        if (k <= 0) continue;
        const int64_t slot0 = sp.slots;
        std::vector<int32_t> cells(k);
        QP_CUDA_CHECK(s, cudaMemcpy(cells.data(), sp.newcell + slot0, k * 4, cudaMemcpyDeviceToHost));
        std::vector<int64_t> order(k);
        for (int64_t t = 0; t < k; t++) order[t] = t;
        std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return cells[a] < cells[b]; });
        // every array of the store (8-byte elements in FP64, 4-byte cell
        // and offsets in mixed precision) in cell order
        const int na = n_arrays(s);
        const size_t el = arr_elem(s, 0);
        std::vector<char> tmp(k * el), srt(k * el);
        for (int a = 0; a < na; a++) {
            if (!sp.buf[sp.cur][a]) continue;
            char* d = (char*)sp.buf[sp.cur][a] + slot0 * el;
            QP_CUDA_CHECK(s, cudaMemcpy(tmp.data(), d, k * el, cudaMemcpyDeviceToHost));
            for (int64_t t = 0; t < k; t++) memcpy(&srt[t * el], &tmp[order[t] * el], el);
            QP_CUDA_CHECK(s, cudaMemcpy(d, srt.data(), k * el, cudaMemcpyHostToDevice));
        }
        std::vector<int32_t> sc(k);
        for (int64_t t = 0; t < k; t++) sc[t] = cells[order[t]];
        int32_t* dc = nullptr;
        QP_CUDA_CHECK(s, scratch_alloc(s, (void**)&dc, k * 4));
        QP_CUDA_CHECK(s, cudaMemcpyAsync(dc, sc.data(), k * 4, cudaMemcpyHostToDevice, s.stream));
        r = merge_sorted_slots(s, who[w], slot0, k, dc);
        scratch_free(s, dc);
        if (r != QP_OK) return r;
    }
    // room for a photon from every lepton, the vacuum pairs included
    nlep = 0;
    for (auto& sp : s.sp)
        if (sp.kind == KIND_LEPTON) nlep += sp.n;
    if ((r = ensure_capacity(s, ph, std::max(s.sp[ph].slots, nph + nlep) + 1)) != QP_OK) return r;
    for (auto& sp : s.sp)
        if (sp.d_counter) QP_CUDA_CHECK(s, cudaMemsetAsync(sp.d_counter, 0, sizeof(int), s.stream));
    return QP_OK;
}

static void fill_diag(State& s, qp_diag* d) {
    const qp_params& p = s.prm;
    const double PI = 3.141592653589793;
    const double dV = p.dx * p.dy * p.dz;
    // normalisations of main.cpp:2326-2327
    const double aN = dV * 1.11485e13 * p.lambda_cm / (8 * PI * PI * PI);
    const double aE = 0.5 * dV * 3.691e4 * p.lambda_cm / 1e7;
    const double bE = 8.2e-14 * dV * 1.11485e13 * p.lambda_cm / (8 * PI * PI * PI);
    memset(d, 0, sizeof(*d));
    const DiagAccum& a = *s.h_diag;
    double Ne = 0, Np = 0, Nph = 0, ee = 0, ep = 0, eph = 0, er = 0;
    for (size_t i = 0; i < s.sp.size(); i++) {
        const Species& sp = s.sp[i];
        d->n_macro[i] = (int64_t)a.cnt[i];
        // erased energy with each species' sign and scale (as energy_e/p/ph, ienergy)
        double ers = 0;
        if (sp.cmr == -1) ers = -a.sum_erased[i];
        else if (sp.cmr == 1 || sp.cmr == 0) ers = a.sum_erased[i];
        else if (sp.ion_index >= 0) ers = a.sum_erased[i] / sp.cmr;
        er += ers;
        d->energy_erased_sp[i] = ers * bE;
        // compute_N / compute_energy species tests (fout.cpp:62-77, 105-126)
        if (sp.cmr == -1) { Ne -= a.sum_q[i]; ee -= a.sum_e[i]; d->N_qp_e += a.cnt[i]; }
        else if (sp.cmr == 1) { Np += a.sum_q[i]; ep += a.sum_e[i]; d->N_qp_p += a.cnt[i]; }
        else if (sp.cmr == 0) { Nph += a.sum_q[i]; eph += a.sum_e[i]; d->N_qp_g += a.cnt[i]; }
        else if (sp.ion_index >= 0) {
            d->N_qp_i[sp.ion_index] += a.cnt[i];
            d->ienergy[sp.ion_index] += a.sum_e[i] / sp.cmr * bE;
        }
    }
    int nion = 0;
    for (const auto& sp : s.sp) nion += sp.kind == KIND_ION;
    d->n_ion = nion;
    d->N_e = Ne * aN; d->N_p = Np * aN; d->N_ph = Nph * aN;
    double wf = 0.0;
    for (int k = 0; k < FIELD_SLOTS; k++) wf += a.field[k];
    d->energy_f = wf * aE;
    d->energy_e = ee * bE; d->energy_p = ep * bE; d->energy_ph = eph * bE;
    d->energy_erased = er * bE;
}

int qp_step(qp_handle* h, int nsteps, double external_bz, qp_diag* diag) {
    QP_H_CHECK(h);
    State& s = h->st;
    if (nsteps < 0) { s.err = "negative step count"; return QP_ERR_ARG; }
    const size_t nc = (size_t)s.grid.nc;
    for (int l = 0; l < nsteps; l++) {
        if (s.timing) QP_CUDA_CHECK(s, cudaEventRecord(s.ev[0], s.stream));
        // padvance (advance.cpp:90-387): J = 0, push and deposit every species
        for (int a = 6; a < 9; a++) QP_CUDA_CHECK(s, cudaMemsetAsync(s.plane[a], 0, nc * s.field_elem, s.stream));
        QP_CUDA_CHECK(s, cudaMemsetAsync(s.d_diag, 0, sizeof(DiagAccum), s.stream));
        if (s.timing) QP_CUDA_CHECK(s, cudaEventRecord(s.ev[1], s.stream));
        std::vector<int> born(s.sp.size(), 0);
        if (s.prm.qed) {
            int r = qed_prepare(s);
            if (r != QP_OK) return r;
            if (s.timing) QP_CUDA_CHECK(s, cudaEventRecord(s.ev[5], s.stream));
            for (auto& sp : s.sp)  // particles born in this push: untracked
                if (sp.trn[1 - sp.cur] && sp.cap > sp.n)
                    QP_CUDA_CHECK(s, cudaMemsetAsync(sp.trn[1 - sp.cur] + sp.n, 0, (sp.cap - sp.n) * sizeof(int32_t), s.stream));
            for (size_t i = 0; i < s.sp.size(); i++) {
                if (s.fp64) launch_push_fp64_qed(s, (int)i, external_bz);
                else launch_push_mixed_qed(s, (int)i, external_bz);
            }
            QP_CUDA_CHECK(s, cudaGetLastError());
            if (s.timing) QP_CUDA_CHECK(s, cudaEventRecord(s.ev[6], s.stream));
            for (size_t i = 0; i < s.sp.size(); i++)
                QP_CUDA_CHECK(s, cudaMemcpyAsync(&born[i], s.sp[i].d_counter, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
            QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
            for (size_t i = 0; i < s.sp.size(); i++)
                born[i] = (int)std::min<int64_t>(born[i], s.sp[i].cap - s.sp[i].n);
        } else if (s.ord.on) {
            int r = ordered_push_all(s, external_bz);
            if (r != QP_OK) return r;
        } else {
            for (size_t i = 0; i < s.sp.size(); i++) {
                if (s.fp64) launch_push_fp64(s, (int)i, external_bz);
                else launch_push_mixed(s, (int)i, external_bz);
            }
        }
        const bool counted = !s.prm.qed;
        QP_CUDA_CHECK(s, cudaGetLastError());
        if (s.timing) QP_CUDA_CHECK(s, cudaEventRecord(s.ev[2], s.stream));
        std::vector<char> rebinned(s.sp.size(), 0);
        for (size_t i = 0; i < s.sp.size(); i++)
            if (s.sp[i].n > 0 || born[i] > 0) {
                rebin(s, (int)i, born[i], counted);
                rebinned[i] = 1;
            }
        if (s.ord.on) {
            int r = ordered_after_rebin(s);
            if (r != QP_OK) return r;
        }
        QP_CUDA_CHECK(s, cudaGetLastError());
        if (s.timing) QP_CUDA_CHECK(s, cudaEventRecord(s.ev[3], s.stream));
        if (s.timing) QP_CUDA_CHECK(s, cudaEventRecord(s.ev[4], s.stream));
        // fadvance: half B, E, half B, Bbar (maxwell.cpp:10-22, advance.cpp:13-18);
        // the first half B also sums compute_energy's field term on E, B
        // before the update (main.cpp:2327)
        for (int ph = 0; ph < 4; ph++) {
            const int kp = ph == 0 ? 4 : (ph == 2 ? 0 : ph);
            if (s.fp64) launch_fields_fp64(s, kp);
            else launch_fields_mixed(s, kp);
        }
        QP_CUDA_CHECK(s, cudaGetLastError());
        QP_CUDA_CHECK(s, cudaMemcpyAsync(s.h_diag, s.d_diag, sizeof(DiagAccum), cudaMemcpyDeviceToHost, s.stream));
        unsigned int st = 0;
        QP_CUDA_CHECK(s, cudaMemcpyAsync(&st, s.d_status, sizeof(unsigned int), cudaMemcpyDeviceToHost, s.stream));
        QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
        for (size_t i = 0; i < s.sp.size(); i++)
            if (rebinned[i]) s.sp[i].n = s.h_count[i];
        if (s.timing) {
            cudaEvent_t end = nullptr;
            QP_CUDA_CHECK(s, cudaEventCreate(&end));
            QP_CUDA_CHECK(s, cudaEventRecord(end, s.stream));
            QP_CUDA_CHECK(s, cudaEventSynchronize(end));
            float t01, t12, t23, t34, t4e;
            cudaEventElapsedTime(&t01, s.ev[0], s.ev[1]);
            cudaEventElapsedTime(&t12, s.ev[1], s.ev[2]);
            cudaEventElapsedTime(&t23, s.ev[2], s.ev[3]);
            cudaEventElapsedTime(&t34, s.ev[3], s.ev[4]);
            cudaEventElapsedTime(&t4e, s.ev[4], end);
            cudaEventDestroy(end);
            s.phase_ms[0] += t12;
            s.phase_ms[1] += t23;
            s.phase_ms[2] += t4e;
            s.phase_ms[3] += t01 + t34;
            s.phase_steps++;
            if (s.prm.qed) {
                float q0, q1, q2;
                cudaEventElapsedTime(&q0, s.ev[1], s.ev[5]);
                cudaEventElapsedTime(&q1, s.ev[5], s.ev[6]);
                cudaEventElapsedTime(&q2, s.ev[6], s.ev[2]);
                s.qed_ms[0] += q0;
                s.qed_ms[1] += q1;
                s.qed_ms[2] += q2;
                s.qed_steps++;
            }
        }
        fill_diag(s, &s.last_diag);
        s.last_diag.status = st ? (st & ST_NAN ? QP_ERR_NAN : (st & ST_CAPACITY ? QP_ERR_CAPACITY : QP_ERR_CONFIG)) : QP_OK;
        s.have_diag = true;
        s.step_index++;
        if (diag) diag[l] = s.last_diag;
        if (st) {
            s.err = st & ST_NAN ? "non-finite particle momentum" :
                    (st & ST_CAPACITY ? "particle store full" : "particle left the grid bounds");
            return s.last_diag.status;
        }
    }
    return QP_OK;
}

int qp_get_diag(qp_handle* h, qp_diag* out) {
    QP_H_CHECK(h);
    if (!out) return QP_ERR_ARG;
    if (!h->st.have_diag) { h->st.err = "no step has run"; return QP_ERR_STATE; }
    *out = h->st.last_diag;
    return QP_OK;
}

int qp_dump_fields(qp_handle* h, double* out) {
    QP_H_CHECK(h);
    State& s = h->st;
    if (!out) return QP_ERR_ARG;
    const size_t nc = (size_t)s.grid.nc;
    cudaPointerAttributes at{};
    const bool dev = cudaPointerGetAttributes(&at, out) == cudaSuccess && at.type == cudaMemoryTypeDevice;
    cudaGetLastError();
    for (int a = 0; a < 12; a++) {
        double* o = out + a * nc;
        if (s.fp64) {
            QP_CUDA_CHECK(s, cudaMemcpyAsync(o, s.plane[a], nc * 8, cudaMemcpyDefault, s.stream));
        } else if (dev) {
            launch_f32_to_f64(s, (const float*)s.plane[a], o, nc);
        } else {
            std::vector<float> tmp(nc);
            QP_CUDA_CHECK(s, cudaMemcpyAsync(tmp.data(), s.plane[a], nc * 4, cudaMemcpyDeviceToHost, s.stream));
            QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
            for (size_t c = 0; c < nc; c++) o[c] = tmp[c];
        }
    }
    QP_CUDA_CHECK(s, cudaGetLastError());
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    return QP_OK;
}

int qp_count_particles(qp_handle* h, int si, int64_t* n) {
    QP_H_CHECK(h);
    if (!n || si < 0 || si >= (int)h->st.sp.size()) return QP_ERR_ARG;
    *n = h->st.sp[si].n;
    return QP_OK;
}

int qp_dump_particles(qp_handle* h, int si, int64_t cap, double* x, double* y, double* z, double* ux,
                      double* uy, double* uz, double* g, double* q, double* chi, int64_t* cell) {
    QP_H_CHECK(h);
    State& s = h->st;
    if (si < 0 || si >= (int)s.sp.size()) return QP_ERR_ARG;
    Species& sp = s.sp[si];
    const int64_t n = sp.n;
    if (cap < n) { s.err = "dump capacity smaller than the particle count"; return QP_ERR_ARG; }
    if (n == 0) return QP_OK;
    std::vector<int32_t> perm(n), cs(s.grid.nc + 1);
    QP_CUDA_CHECK(s, cudaMemcpyAsync(perm.data(), sp.perm, n * 4, cudaMemcpyDeviceToHost, s.stream));
    QP_CUDA_CHECK(s, cudaMemcpyAsync(cs.data(), sp.cell_start, (s.grid.nc + 1) * 4, cudaMemcpyDeviceToHost, s.stream));
    QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
    // slots in use: [0, max perm]
    int32_t used = 0;
    for (int64_t t = 0; t < n; t++) used = std::max(used, perm[t] + 1);
    std::vector<int32_t> cl(n);
    for (int c = 0; c < s.grid.nc; c++)
        for (int t = cs[c]; t < cs[c + 1]; t++) cl[t] = c;
    if (cell)
        for (int64_t t = 0; t < n; t++) cell[t] = cl[t];
    const int cur = sp.cur;
    if (s.fp64) {
        double* dst[9] = {x, y, z, ux, uy, uz, g, q, chi};
        std::vector<double> tmp(used);
        for (int a = 0; a < 9; a++) {
            if (!dst[a]) continue;
            if (!sp.buf[cur][a]) { std::fill(dst[a], dst[a] + n, 0.0); continue; }
            QP_CUDA_CHECK(s, cudaMemcpyAsync(tmp.data(), sp.buf[cur][a], (size_t)used * 8, cudaMemcpyDeviceToHost, s.stream));
            QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
            for (int64_t t = 0; t < n; t++) dst[a][t] = tmp[perm[t]];
        }
    } else {
        std::vector<float> tmp(used);
        std::vector<int32_t> tci(used);
        QP_CUDA_CHECK(s, cudaMemcpyAsync(tci.data(), sp.buf[cur][0], (size_t)used * 4, cudaMemcpyDeviceToHost, s.stream));
        QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
        double* pos[3] = {x, y, z};
        for (int a = 0; a < 3; a++) {
            if (!pos[a]) continue;
            QP_CUDA_CHECK(s, cudaMemcpyAsync(tmp.data(), sp.buf[cur][1 + a], (size_t)used * 4, cudaMemcpyDeviceToHost, s.stream));
            QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
            for (int64_t t = 0; t < n; t++) {
                const int c = tci[perm[t]];
                const int ii = c / s.grid.nynz, jj = (c / s.grid.nz) % s.grid.ny, kk = c % s.grid.nz;
                const int base = a == 0 ? ii : (a == 1 ? jj : kk);
                pos[a][t] = (double)base + (double)tmp[perm[t]];
            }
        }
        double* dst[6] = {ux, uy, uz, g, q, chi};
        for (int a = 0; a < 6; a++) {
            if (!dst[a]) continue;
            if (!sp.buf[cur][4 + a]) { std::fill(dst[a], dst[a] + n, 0.0); continue; }
            QP_CUDA_CHECK(s, cudaMemcpyAsync(tmp.data(), sp.buf[cur][4 + a], (size_t)used * 4, cudaMemcpyDeviceToHost, s.stream));
            QP_CUDA_CHECK(s, cudaStreamSynchronize(s.stream));
            for (int64_t t = 0; t < n; t++) dst[a][t] = tmp[perm[t]];
        }
    }
    return QP_OK;
}

int qp_checkpoint(qp_handle* h, int slot) {
    QP_H_CHECK(h);
    if (slot < 0 || slot > 3) return QP_ERR_ARG;
    return snapshot_take(h->st, h->st.snap[slot]);
}

int qp_restore(qp_handle* h, int slot) {
    QP_H_CHECK(h);
    if (slot < 0 || slot > 3) return QP_ERR_ARG;
    return snapshot_restore(h->st, h->st.snap[slot]);
}

}  // extern "C"
