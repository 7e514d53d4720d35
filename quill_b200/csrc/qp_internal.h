// Internal declarations of libquill_b200: device state of one region and the
// kernel entry points shared between translation units.
#pragma once

#include <algorithm>

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "quill_b200.h"

namespace qp {

// Particle kinds, from the charge-to-mass test chain of padvance
// (advance.cpp:155 photon cmr == 0, :253 |cmr| == 1 lepton, :360 ion).
enum Kind { KIND_PHOTON = 0, KIND_LEPTON = 1, KIND_ION = 2 };

// Device error word bits, OR-ed by kernels into State::d_status.
enum StatusBits {
    ST_NAN = 1u << 0,       // non-finite gamma after a push
    ST_BOUNDS = 1u << 1,    // an access would have left the grid (skipped)
    ST_CAPACITY = 1u << 2,  // append beyond a store's capacity (dropped)
};

// Division of a non-negative int32 by a fixed divisor d >= 2 with one
// multiply-high and a shift (round-up reciprocal m = ceil(2^(31+l) / d),
// l = ceil(log2 d); exact for every n < 2^31).
struct FastDiv {
    uint32_t m = 0;
    int sh = 0;  // l - 1
    void init(uint32_t d) {
        int l = 0;
        while ((1ull << l) < d) l++;
        m = (uint32_t)(((1ull << (31 + l)) + d - 1) / d);
        sh = l - 1;
    }
#ifdef __CUDACC__
    __device__ __forceinline__ int div(int n) const { return (int)(__umulhi((uint32_t)n, m) >> sh); }
#endif
};

struct Grid {
    int nx, ny, nz;
    int nynz;
    int nc;  // nx*ny*nz < 2^31
    FastDiv div_nz, div_nynz;
};

// Fields: 12 planes of nc elements (E, B, J, Bbar), element type T.
template <typename T>
struct Fields {
    T* ex; T* ey; T* ez;
    T* bx; T* by; T* bz;
    T* jx; T* jy; T* jz;
    T* bex; T* bey; T* bez;
};

// FP64 particle store, structure of arrays, one slot per particle.
struct PStore64 {
    double *x, *y, *z, *ux, *uy, *uz, *g, *q, *chi;
};

// Mixed particle store: linear cell index plus FP32 offset in [0, 1).
struct PStore32 {
    int32_t* cell;
    float *ox, *oy, *oz, *ux, *uy, *uz, *g, *q, *chi;
};

struct Species {
    double cmr = -1;
    int kind = KIND_LEPTON;
    int ion_index = -1;
    int64_t n = 0;       // live particles
    int64_t slots = 0;   // slots of buf[cur] that perm may reference
    int64_t cap = 0;     // allocated slots
    // two buffers of each array; `cur` holds the particles in the layout of
    // the previous push, read through `perm` in traversal order
    void* buf[2][10] = {{nullptr}};
    int cur = 0;
    int32_t* perm = nullptr;       // traversal position -> slot in buf[cur]
    int32_t* newcell = nullptr;    // cell after this push (-1 = erased), by traversal position;
                                   // also the rebin's scratch (swapped with perm)
    int32_t* cell_start = nullptr; // nc+1, traversal order at the start of a step
    int32_t* cell_next = nullptr;  // nc+1, traversal order after the rebin
    int32_t* count = nullptr;      // nc, rebin histogram
    int* d_counter = nullptr;      // device append counter (QED)
    int32_t* trn[2] = {nullptr, nullptr};  // track numbers (0 = untracked), per buffer; tracking only
    // reference-order deposition with several species: order keys of the
    // merged list of all species, by slot, per buffer; gstep: this step's
    // key by traversal position (qp_ordered.cu)
    int32_t* grank[2] = {nullptr, nullptr};
    int32_t* gstep = nullptr;
    int64_t gcap = 0;
};

constexpr int FIELD_SLOTS = 64;

struct DiagAccum {
    // per species: live count, sum q, sum of (g-1)q (or g q for photons)
    double sum_q[QP_MAX_SPECIES];
    double sum_e[QP_MAX_SPECIES];
    unsigned long long cnt[QP_MAX_SPECIES];
    // sum over cells of E^2 + B^2, in FIELD_SLOTS partial sums (the blocks of
    // the first half-B kernel add into slot blockIdx % FIELD_SLOTS)
    double field[FIELD_SLOTS];
    double sum_erased[QP_MAX_SPECIES];  // sum of (g-1)q (g q for photons) of erased particles
};

// Erased particles recorded for catching (delete_particle with
// catching_enabled, low-level.cpp:247-259): one slot per particle claimed with
// *counter; slots beyond cap are dropped (the counter keeps counting).  key
// orders the records as the reference deletes them: step, then the
// p_boundary erasures before the push (phase 0) ahead of the moves out of the
// region (phase 1), each in traversal order.
struct CatchBuf {
    double *x, *y, *z, *ux, *uy, *uz, *g, *q, *chi;
    int32_t* sp;
    int64_t* key;
    int* counter;  // nullptr: catching off
    int cap;
};

struct State {
    qp_params prm;
    Grid grid;
    int fp64 = 1;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;  // scratch (scratch_alloc), created on first use
    bool own_stream = false;
    void* fields = nullptr;       // allocation of the 12 planes
    size_t field_elem = 8;
    // the device address of each plane (ex ey ez bx by bz jx jy jz bex bey bez)
    void* plane[12] = {nullptr};
    std::vector<Species> sp;
    DiagAccum* d_diag = nullptr;  // device accumulators
    DiagAccum* h_diag = nullptr;  // pinned host copy
    int32_t* h_count = nullptr;   // pinned: each species' count after the step's rebin
    unsigned int* d_status = nullptr;
    void* scan_tmp = nullptr;     // block sums for the exclusive scans
    size_t scan_tmp_bytes = 0;
    qp_diag last_diag{};
    bool have_diag = false;
    int64_t launches = 0;
    int64_t step_index = 0;
    bool boundaries_done = false;
    int sp_e = -1, sp_p = -1, sp_ph = -1;  // QED species (cmr -1, +1, 0)
    // launch shape of the non-QED pushes: threads per block and the CTAs per
    // SM its register budget targets (push_shapes64 / push_shapes32 below;
    // QP_PUSH_SHAPE and QP_PUSH_SHAPE_MIXED select by index)
    bool prefetch = true;  // pushes: next chunk's slot and cell (FP64: position) loaded a chunk ahead (QP_PREFETCH)
    int push_shape = 0;
    int push_shape_mixed = 3;
    // grid of the pushes: at most push_waves x (SMs x CTAs per SM) blocks
    // striding over the particles; per push (FP64 256 groups measured 1 %
    // faster than 128, mixed 128 1 % faster than 256); QP_PUSH_WAVES sets
    // all three (0: one thread per particle)
    int push_waves = 256, push_waves_mixed = 128, push_waves_qed = 128;
    int sm_count = 148;
    std::string err;
    // optional per-phase CUDA-event timing of qp_step (push, rebin, fields,
    // diagnostics + J reset)
    bool timing = false;
    bool track_erased = false;  // qp_set_erased_tracking
    bool tracking = false;      // qp_set_tracking: Species::trn allocated and carried by the pushes
    int diag_lo = 0, diag_hi = 0;  // qp_set_diag_range: cells i in [diag_lo, diag_hi) counted (create: [0, nx))
    void* window_scratch = nullptr;  // one field plane, for the moving window's shift
    CatchBuf cat{};                  // capture buffer (counter null = none)
    bool catch_erasures = false;     // qp_set_catching: erasures go to the buffer
    bool dump_photons = false;       // qp_set_dump_photons: emitted photons go to the buffer
    CatchBuf* d_cat = nullptr;       // its device copy, passed to the push kernels
    cudaEvent_t ev[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    double phase_ms[4] = {0, 0, 0, 0};
    int64_t phase_steps = 0;
    // QED steps: preparation (capacity, vacuum pairs and their merge), push
    // kernels, read-back of the born counts (qp_get_qed_timing)
    double qed_ms[3] = {0, 0, 0};
    int64_t qed_steps = 0;
    // cells whose new range is too long for the per-thread ordering of the
    // rebin: entry 0 counts them, entries 1.. list them
    int32_t* long_list = nullptr;
    int64_t long_cap = 0;
    // bumped by every change of the particle layout other than a step's
    // rebin, merging and the moving window (loads, restores, slab
    // replacements): the reference-order deposition then rebuilds its keys
    int64_t layout_epoch = 0;
    // reference-order deposition (qp_set_ordered_current, qp_ordered.cu)
    struct Ordered {
        bool on = false;
        int64_t epoch = -1;          // layout_epoch the order keys belong to
        int64_t cap_particles = 0;   // entry buffers sized for this many particles
        int32_t* tgt = nullptr;      // 48 entries per particle: target (component * nc + cell)
        int64_t* key = nullptr;      //   order key (rank * 48 + term index)
        double* val = nullptr;       //   term
        int32_t* nent = nullptr;     // entries used per particle
        int64_t* skey = nullptr;     // entries bucketed by target
        double* sval = nullptr;
        int32_t* jcount = nullptr;   // 3 nc + 1: entries per target, then claim cursors
        int32_t* jstart = nullptr;   // 3 nc + 1: bucket starts
        void* scan_tmp = nullptr;    // tile sums of the 3 nc scan
    } ord;
    // checkpoints (device-resident copies)
    struct Snap {
        bool valid = false;
        void* fields = nullptr;
        std::vector<std::vector<void*>> arrays;  // per species, 10 arrays + perm
        std::vector<int64_t> n, cap, slots;
        std::vector<int32_t*> cell_start;
        int64_t step_index = 0;
    } snap[4];
};

// The 12 field planes of the current step as typed device pointers.
template <typename T>
inline Fields<T> fields_of(const State& s) {
    Fields<T> f;
    T** p[12] = {&f.ex, &f.ey, &f.ez, &f.bx, &f.by, &f.bz, &f.jx, &f.jy, &f.jz, &f.bex, &f.bey, &f.bez};
    for (int a = 0; a < 12; a++) *p[a] = (T*)s.plane[a];
    return f;
}
// The same as an array (plane a = component a of ex .. bez).
template <typename T>
struct Planes {
    T* p[12];
};
template <typename T>
inline Planes<T> planes_of(const State& s) {
    Planes<T> q;
    for (int a = 0; a < 12; a++) q.p[a] = (T*)s.plane[a];
    return q;
}

// Blocks for a push over n particles in block-sized chunks (chunk_range): up
// to `waves` groups of `resident` blocks (the blocks resident at once: SMs x
// CTAs per SM); one chunk per block if waves is 0 or the chunks are fewer
// than the resident blocks.
// Launch shapes of the pushes: {threads per block, CTAs per SM}; a block
// takes chunks of `threads` particles.  FP64: 128 registers per thread run
// the loop without spills (256 x 2, the default); the smaller budgets trade
// spills for resident warps and measured 0-25 % slower at 512^3.  Mixed:
// 80 registers run without spills; on 128-thread blocks (128 x 6, the
// default) with the next chunk's slot and cell loaded a chunk ahead this
// measured fastest; 72 registers (128 x 7) spill under the prefetch.
struct PushShape {
    int threads, minb;
};
constexpr PushShape push_shapes64[] = {{256, 2}, {256, 3}, {192, 3}, {128, 5}, {128, 4}, {64, 8}};
constexpr PushShape push_shapes32[] = {{256, 3}, {256, 4}, {128, 7}, {128, 6}, {128, 8}, {64, 14}};
constexpr int n_push_shapes64 = 6, n_push_shapes32 = 6;

inline int push_blocks(const State& s, int64_t n, PushShape sh, int waves, int* resident) {
    const int64_t nch = (n + sh.threads - 1) / sh.threads;
    const int minb = sh.minb;
    const int64_t r = (int64_t)s.sm_count * minb;
    if (waves <= 0 || nch <= r) {
        *resident = (int)(nch > 0 ? nch : 1);
        return (int)nch;
    }
    const int64_t w = std::min<int64_t>(waves, (nch + r - 1) / r);
    *resident = (int)r;
    return (int)(r * w);
}

// Device copy of the full state into a snapshot / back (qp_checkpoint,
// qp_restore, the adjoint's checkpoints); snapshot_free releases one.
int snapshot_take(State& s, State::Snap& sn);
int snapshot_restore(State& s, State::Snap& sn);
void snapshot_free(State::Snap& sn);
State* state_of(qp_handle* h);
void catch_release(State& s);  // frees the catching buffer (qp_catch.cu)

// Adjoint of qp_step's FP64 FDTD/Boris path (qp_adjoint.cu).
int adjoint_energy(State& s, qp_handle* h, int nsteps, int every, double ext_bz, double* grad6, double* grad_q,
                   double* loss_out);

// Reference-order deposition (qp_ordered.cu): every species pushed with its
// current terms summed per J element in the reference's order; the order
// keys of several species rebuilt after the rebin; buffers released.
int ordered_push_all(State& s, double external_bz);
int ordered_after_rebin(State& s);
void ordered_release(State& s);

// ---- kernels / launchers (FP64, qp_fp64.cu) ----
// phase: 0 half B, 1 E, 2 half B, 3 Bbar, 4 half B summing E^2 + B^2 of the
// cells [diag_lo, diag_hi) before the update (compute_energy's field term)
void launch_fields_fp64(State& s, int phase);
void launch_init_boundaries_fp64(State& s);
void launch_push_fp64(State& s, int species, double external_bz);
int launch_push_fp64_qed(State& s, int species, double external_bz);
int launch_vacuum_fp64(State& s);

// ---- mixed precision (qp_mixed.cu) ----
void launch_fields_mixed(State& s, int phase);
void launch_init_boundaries_mixed(State& s);
void launch_push_mixed(State& s, int species, double external_bz);
int launch_push_mixed_qed(State& s, int species, double external_bz);
int launch_vacuum_mixed(State& s);

// ---- rebin and scans (qp_rebin.cu) ----
// Rebin after a push: count -> scan -> assign; leaves the new traversal
// order in sp.perm / sp.cell_start and swaps buffers.  The new particle
// count is copied to s.h_count[species] on the stream (the caller sets sp.n
// after synchronising).  counted: sp.count already holds the particles per
// new cell (tiled push).
void rebin(State& s, int species, int64_t born, bool counted);
// Cells with more particles than this are ordered by a block each.
constexpr int REBIN_LONG_SEG = 64;
// Loading (qp_load.cu)
void launch_load_cells(State& s, const double* const* a, int n, int32_t* cells, unsigned int* flags,
                       int* first_bad, int base);
void launch_check_sorted(State& s, const int32_t* cells, int n, unsigned int* flags);
void launch_histogram(State& s, const int32_t* cells, int n, int32_t* count);
void launch_to_mixed(State& s, const double* const* a, int n, PStore32 dst, int at);
void launch_f64_to_f32(State& s, const double* a, float* b, size_t n);
void launch_f32_to_f64(State& s, const float* a, double* b, size_t n);
void exclusive_scan_i32(State& s, const int32_t* in, int32_t* out, int n, int32_t* copy = nullptr);
// Particle store (qp_api.cu): grow the arrays of a species to `need` slots,
// keeping their contents; copy n particles (9 FP64 arrays, host or device,
// chi may be null) into slots [sp.slots, sp.slots + n) with their cells and
// validity flags (stream-ordered, nothing synchronised).
int ensure_capacity(State& s, int si, int64_t need);
// Per-call scratch, stream-ordered on s.stream, from a memory pool the region
// owns.  The pool keeps the memory it has mapped (unlimited release
// threshold), so repeated calls cost no mapping; it goes with the region.
cudaError_t scratch_alloc(State& s, void** p, size_t bytes);
void scratch_free(State& s, void* p);
int stage_particles(State& s, int si, int64_t n, const double* const* src, int32_t* cells, unsigned int* flags,
                    int* first_bad);

}  // namespace qp

#define QP_CUDA_CHECK(s, call)                                                  \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) {                                                 \
            (s).err = std::string(#call) + ": " + cudaGetErrorString(e_);        \
            return QP_ERR_CUDA;                                                  \
        }                                                                        \
    } while (0)
