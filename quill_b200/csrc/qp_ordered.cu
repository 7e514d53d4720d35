// Reference-order current deposition (qp_set_ordered_current): the FP64
// step with J summed in exactly the order of the reference's padvance, so
// that the GPU state stays bit-identical to the reference over any number of
// steps, not only to within the rounding of an atomic summation order.
//
// The reference walks the particles in traversal order (cells
// lexicographic, each cell's list from its head, all species in one list;
// advance.cpp:90-387) and adds every one of a segment's 12 terms straight
// into cj (deposition.cpp:13-39: cj = cj + term).  A J element therefore
// holds the terms that reach it, added one by one from zero in the order
// (particle's traversal rank, its segment, the term within the segment).
// Here each push thread writes its terms as entries (target, key, value)
// with key = rank * 48 + running term index (at most 4 segments x 12
// terms); the entries are bucketed by target (count, scan, scatter), each
// bucket is ordered by key and summed from zero in that order.
//
// With several species the rank is the position in the merged list of all
// species, which the per-species stores do not hold.  Each particle then
// carries an order key (State::Species::grank, indexed by slot like the
// payload).  After the rebin a per-cell pass rebuilds the keys with the
// reference's list rule (plist.cpp:22-39, advance.cpp:377-386): the cell's
// arrivals first, by descending old key, then its stayers by ascending old
// key.  Keys are first built (and rebuilt after a load, a checkpoint restore
// or a slab replacement) as one load of all species concatenated in species
// order would place them: within each cell species 0's particles, then
// species 1's, and so on.  Merging and the moving window keep the relative
// order and leave the keys valid.
//
// Built with --fmad=false like the other FP64 kernels.  FP64 only, QED off.
// This is a parity mode: it costs several times the atomic deposition and
// needs 48 entries (about 1.3 kB) per particle of scratch.
#include "qp_kernels.cuh"

namespace qp {

constexpr int ENT_PER_PARTICLE = 48;

// Terms of jdeposition_to recorded as entries instead of added to J.
struct EntrySink {
    int32_t* tgt;
    int64_t* key;
    double* val;
    int32_t* jcount;
    int nc;
    int64_t idx0;  // first entry of this particle
    int64_t key0;  // rank * 48
    mutable int k = 0;
    __device__ __forceinline__ void add(int comp, int, int, int, int c, double v) const {
        const int t = comp * nc + c;
        const int64_t e = idx0 + k;
        tgt[e] = t;
        key[e] = key0 + k;
        val[e] = v;
        atomicAdd(jcount + t, 1);
        k++;
    }
};

struct OrderedArgs {
    int32_t* tgt;
    int64_t* key;
    double* val;
    int32_t* nent;          // entries per particle (species offset + traversal position)
    int32_t* jcount;        // entries per target
    int64_t base;           // species offset in particles
    const int32_t* gsrc;    // order keys by slot (several species); nullptr: the traversal position is the rank
    int32_t* gstep;         // order key of traversal position s this step (several species)
};

// k_push64 with the deposition recorded as entries: one thread per particle
// in traversal order; everything else (p_boundary, gather, push,
// displacement, place, catching, tracks, diagnostics, the rebin histogram)
// as k_push64 does it.
template <int PUSHER, int KIND>
__global__ void __launch_bounds__(256) k_push64_ordered(Fields<double> f, Grid g, PStore64 src, PStore64 dst,
                                                        const int32_t* __restrict__ perm,
                                                        int32_t* __restrict__ newcell, int32_t* __restrict__ count,
                                                        PushArgs a, OrderedArgs o) {
    double dq = 0.0, de = 0.0, er = 0.0;
    unsigned long long dc = 0;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    int nc = -1;
    if (s < a.n) {
        const int p = perm[s];
        double pos[3] = {src.x[p], src.y[p], src.z[p]};
        double ux = src.ux[p], uy = src.uy[p], uz = src.uz[p], gm = src.g[p];
        const double q = src.q[p];
        const int i0 = (int)pos[0], j0 = (int)pos[1], k0 = (int)pos[2];
        const bool live = !kill_layer(g, i0, j0, k0);  // p_boundary, plist.cpp:73-102
        const int64_t rank = o.gsrc ? (int64_t)o.gsrc[p] : (int64_t)s;
        if (o.gstep) o.gstep[s] = (int32_t)rank;
        int nent = 0;
        if (live) {
            double E[3], B[3];
            gather(f, g, i0, j0, k0, pos[0] - i0, pos[1] - j0, pos[2] - k0, E, B);
            B[2] += a.ext_bz;
            if (KIND != KIND_PHOTON) push<PUSHER>(a.cmr, ux, uy, uz, gm, E, B, a.dt);
            const double t = a.dt / gm;
            double d[3] = {ux * t, uy * t, uz * t};
            d[0] = div_fixed(d[0], a.dx, a.rdx);
            d[1] = div_fixed(d[1], a.dy, a.rdy);
            d[2] = div_fixed(d[2], a.dz, a.rdz);
            if (KIND == KIND_PHOTON) {
                pos[0] = pos[0] + d[0]; pos[1] = pos[1] + d[1]; pos[2] = pos[2] + d[2];
            } else {
                EntrySink sink{o.tgt, o.key, o.val, o.jcount, g.nc,
                               (o.base + s) * (int64_t)ENT_PER_PARTICLE, rank * ENT_PER_PARTICLE};
                jdeposition_to(sink, g, pos, d, q, 0, 0, 0, a.status);
                nent = sink.k;
            }
            if (!isfinite(gm)) atomicOr(a.status, (unsigned int)ST_NAN);
        }
        o.nent[o.base + s] = nent;
        bool nc_owned = true;
        if (live) {
            const int i1 = (int)pos[0], j1 = (int)pos[1], k1 = (int)pos[2];
            const bool moved = (i1 != i0) || (j1 != j0) || (k1 != k0);
            if (!moved || inside(g, i1, j1, k1)) nc = cidx(g, i1, j1, k1);
        }
        newcell[s] = nc;
        if (nc < 0 && !((int)pos[0] >= a.dlo && (int)pos[0] < a.dhi)) nc_owned = false;
        if (nc < 0 && a.cat && nc_owned)
            catch_particle(*a.cat, a.sp, a.step, live ? 1 : 0, s, pos[0], pos[1], pos[2], ux, uy, uz, gm, q,
                           src.chi ? src.chi[p] : 0.0);
        if (nc >= 0) {
            dst.x[s] = pos[0]; dst.y[s] = pos[1]; dst.z[s] = pos[2];
            dst.ux[s] = ux; dst.uy[s] = uy; dst.uz[s] = uz;
            dst.g[s] = gm; dst.q[s] = q;
            if (dst.chi) dst.chi[s] = src.chi[p];
            if (a.trn_dst) a.trn_dst[s] = a.trn_src[p];
            const int ii = (int)pos[0];
            if (ii >= a.dlo && ii < a.dhi) {
                dq += q;
                de += KIND == KIND_PHOTON ? gm * q : (gm - 1) * q;
                dc += 1;
            }
        }
        if (a.track && nc < 0 && nc_owned) er += KIND == KIND_PHOTON ? gm * q : (gm - 1) * q;
    }
    warp_count_runs(count, nc);
    block_diag(a.diag, a.sp, dq, de, dc);
    if (a.track) block_sum(&a.diag->sum_erased[a.sp], er);
}

// Entries into their target's bucket (any order inside a bucket).
__global__ void __launch_bounds__(256) k_entries_scatter(int64_t n_particles, const int32_t* __restrict__ nent,
                                                         const int32_t* __restrict__ tgt,
                                                         const int64_t* __restrict__ key,
                                                         const double* __restrict__ val, int32_t* __restrict__ cur,
                                                         int64_t* __restrict__ skey, double* __restrict__ sval) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t pi = e / ENT_PER_PARTICLE;
    if (pi >= n_particles) return;
    if ((int)(e - pi * ENT_PER_PARTICLE) >= nent[pi]) return;
    const int pos = atomicAdd(cur + tgt[e], 1);
    skey[pos] = key[e];
    sval[pos] = val[e];
}

// Each target's bucket ordered by key (insertion sort: buckets hold the
// terms of the particles of the neighbouring cells, tens of entries) and
// summed from zero in that order, as cj = cj + term does.
__global__ void __launch_bounds__(256) k_entries_sum(int nc, const int32_t* __restrict__ start,
                                                     int64_t* __restrict__ skey, double* __restrict__ sval,
                                                     double* __restrict__ jx, double* __restrict__ jy,
                                                     double* __restrict__ jz) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 3 * nc) return;
    const int b = start[t], e = start[t + 1];
    for (int i = b + 1; i < e; i++) {
        const int64_t k = skey[i];
        const double v = sval[i];
        int j = i - 1;
        while (j >= b && skey[j] > k) {
            skey[j + 1] = skey[j];
            sval[j + 1] = sval[j];
            j--;
        }
        skey[j + 1] = k;
        sval[j + 1] = v;
    }
    double acc = 0.0;
    for (int i = b; i < e; i++) acc = acc + sval[i];
    const int comp = t / nc;
    (comp == 0 ? jx : (comp == 1 ? jy : jz))[t - comp * nc] = acc;
}

struct SpeciesOrder {
    int ns;
    const int32_t* start[QP_MAX_SPECIES];      // cell starts (the order being described)
    const int32_t* old_start[QP_MAX_SPECIES];  // cell starts before the rebin (merge only)
    const int32_t* perm[QP_MAX_SPECIES];
    const int32_t* gold[QP_MAX_SPECIES];       // old keys by slot (merge only)
    int32_t* gnew[QP_MAX_SPECIES];             // new keys by slot
};

// First keys: within each cell species by species (species 0 first), each
// in its traversal order.  One thread per (species si) traversal position.
__global__ void __launch_bounds__(256) k_grank_init(Grid g, PStore64 st, SpeciesOrder o, int si, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int slot = o.perm[si][t];
    const int c = cidx(g, (int)st.x[slot], (int)st.y[slot], (int)st.z[slot]);
    int r = t - o.start[si][c];
    for (int s2 = 0; s2 < o.ns; s2++) {
        r += o.start[s2][c];
        if (s2 < si) r += o.start[s2][c + 1] - o.start[s2][c];
    }
    o.gnew[si][slot] = r;
}

// New keys after the rebin, one thread per cell: the merged list of the
// cell is its arrivals (any species) by descending old key, then its
// stayers by ascending old key.  A particle stays if its old traversal
// position (its slot in the new buffer) lies in the cell's old range.
__global__ void __launch_bounds__(256) k_grank_merge(int nc, SpeciesOrder o) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    int base = 0, arrivals = 0;
    for (int s = 0; s < o.ns; s++) {
        base += o.start[s][c];
        const int lo = o.old_start[s][c], hi = o.old_start[s][c + 1];
        for (int t = o.start[s][c]; t < o.start[s][c + 1]; t++) {
            const int slot = o.perm[s][t];
            arrivals += !(slot >= lo && slot < hi);
        }
    }
    for (int s = 0; s < o.ns; s++) {
        const int lo = o.old_start[s][c], hi = o.old_start[s][c + 1];
        for (int t = o.start[s][c]; t < o.start[s][c + 1]; t++) {
            const int slot = o.perm[s][t];
            const bool stay = slot >= lo && slot < hi;
            const int key = o.gold[s][slot];
            int pos = stay ? arrivals : 0;
            for (int s2 = 0; s2 < o.ns; s2++) {
                const int lo2 = o.old_start[s2][c], hi2 = o.old_start[s2][c + 1];
                for (int t2 = o.start[s2][c]; t2 < o.start[s2][c + 1]; t2++) {
                    const int slot2 = o.perm[s2][t2];
                    const bool stay2 = slot2 >= lo2 && slot2 < hi2;
                    const int key2 = o.gold[s2][slot2];
                    if (stay) pos += (stay2 && key2 < key);
                    else pos += (!stay2 && key2 > key);
                }
            }
            o.gnew[s][slot] = base + pos;
        }
    }
}

static PStore64 store64_of(Species& sp, int b) {
    PStore64 st;
    double** ps[9] = {&st.x, &st.y, &st.z, &st.ux, &st.uy, &st.uz, &st.g, &st.q, &st.chi};
    for (int a = 0; a < 9; a++) *ps[a] = (double*)sp.buf[b][a];
    return st;
}


void ordered_release(State& s) {
    State::Ordered& o = s.ord;
    cudaFree(o.tgt); cudaFree(o.key); cudaFree(o.val); cudaFree(o.nent);
    cudaFree(o.skey); cudaFree(o.sval); cudaFree(o.jcount); cudaFree(o.jstart); cudaFree(o.scan_tmp);
    o.tgt = nullptr; o.key = nullptr; o.val = nullptr; o.nent = nullptr;
    o.skey = nullptr; o.sval = nullptr; o.jcount = nullptr; o.jstart = nullptr; o.scan_tmp = nullptr;
    o.cap_particles = 0;
    for (auto& sp : s.sp) {
        cudaFree(sp.grank[0]); cudaFree(sp.grank[1]); cudaFree(sp.gstep);
        sp.grank[0] = sp.grank[1] = sp.gstep = nullptr;
        sp.gcap = 0;
    }
    o.epoch = -1;
}

// Buffers for this step's entries and, with several species, valid order
// keys for the current layout.
static int ordered_prepare(State& s) {
    State::Ordered& o = s.ord;
    const int64_t nc3 = 3 * (int64_t)s.grid.nc;
    int64_t np = 0;
    for (auto& sp : s.sp) np += sp.n;
    if (np * ENT_PER_PARTICLE >= (int64_t)INT32_MAX) {
        s.err = "reference-order deposition: more than 44 million particles";
        return QP_ERR_CAPACITY;
    }
    if (!o.jcount) {
        QP_CUDA_CHECK(s, cudaMalloc(&o.jcount, (nc3 + 1) * sizeof(int32_t)));
        QP_CUDA_CHECK(s, cudaMalloc(&o.jstart, (nc3 + 1) * sizeof(int32_t)));
        QP_CUDA_CHECK(s, cudaMalloc(&o.scan_tmp, ((nc3 + 4095) / 4096 + 2) * sizeof(int32_t)));
    }
    if (np > o.cap_particles) {
        const int64_t cap = std::max<int64_t>(np, o.cap_particles + o.cap_particles / 2);
        const int64_t ne = cap * ENT_PER_PARTICLE;
        cudaFree(o.tgt); cudaFree(o.key); cudaFree(o.val); cudaFree(o.nent); cudaFree(o.skey); cudaFree(o.sval);
        o.tgt = nullptr; o.key = nullptr; o.val = nullptr; o.nent = nullptr; o.skey = nullptr; o.sval = nullptr;
        QP_CUDA_CHECK(s, cudaMalloc(&o.tgt, ne * sizeof(int32_t)));
        QP_CUDA_CHECK(s, cudaMalloc(&o.key, ne * sizeof(int64_t)));
        QP_CUDA_CHECK(s, cudaMalloc(&o.val, ne * sizeof(double)));
        QP_CUDA_CHECK(s, cudaMalloc(&o.skey, ne * sizeof(int64_t)));
        QP_CUDA_CHECK(s, cudaMalloc(&o.sval, ne * sizeof(double)));
        QP_CUDA_CHECK(s, cudaMalloc(&o.nent, cap * sizeof(int32_t)));
        o.cap_particles = cap;
    }
    QP_CUDA_CHECK(s, cudaMemsetAsync(o.jcount, 0, (nc3 + 1) * sizeof(int32_t), s.stream));
    const int ns = (int)s.sp.size();
    if (ns < 2 || o.epoch == s.layout_epoch) return QP_OK;
    // first keys for the current layout
    SpeciesOrder so{};
    so.ns = ns;
    for (int i = 0; i < ns; i++) {
        Species& sp = s.sp[i];
        if (sp.gcap < sp.cap) {
            cudaFree(sp.grank[0]); cudaFree(sp.grank[1]); cudaFree(sp.gstep);
            sp.grank[0] = sp.grank[1] = sp.gstep = nullptr;
            const int64_t cap = std::max<int64_t>(sp.cap, 1);
            QP_CUDA_CHECK(s, cudaMalloc(&sp.grank[0], cap * sizeof(int32_t)));
            QP_CUDA_CHECK(s, cudaMalloc(&sp.grank[1], cap * sizeof(int32_t)));
            QP_CUDA_CHECK(s, cudaMalloc(&sp.gstep, cap * sizeof(int32_t)));
            sp.gcap = cap;
        }
        so.start[i] = sp.cell_start;
        so.perm[i] = sp.perm;
        so.gnew[i] = sp.grank[sp.cur];
    }
    for (int i = 0; i < ns; i++) {
        Species& sp = s.sp[i];
        if (sp.n == 0) continue;
        k_grank_init<<<(int)((sp.n + 255) / 256), 256, 0, s.stream>>>(s.grid, store64_of(sp, sp.cur), so, i,
                                                                     (int)sp.n);
        s.launches++;
    }
    QP_CUDA_CHECK(s, cudaGetLastError());
    o.epoch = s.layout_epoch;
    return QP_OK;
}

// All species pushed with their terms recorded, then J summed per target in
// the reference's order.
int ordered_push_all(State& s, double external_bz) {
    int r = ordered_prepare(s);
    if (r != QP_OK) return r;
    State::Ordered& o = s.ord;
    const int ns = (int)s.sp.size();
    Fields<double> f = fields_of<double>(s);
    int64_t base = 0;
    for (int si = 0; si < ns; si++) {
        Species& sp = s.sp[si];
        QP_CUDA_CHECK(s, cudaMemsetAsync(sp.count, 0, (size_t)s.grid.nc * sizeof(int32_t), s.stream));
        if (sp.n == 0) continue;
        PStore64 src = store64_of(sp, sp.cur), dst = store64_of(sp, 1 - sp.cur);
        PushArgs a{};
        a.cmr = sp.cmr; a.dt = s.prm.dt; a.dx = s.prm.dx; a.dy = s.prm.dy; a.dz = s.prm.dz;
        a.rdx = 1.0 / s.prm.dx; a.rdy = 1.0 / s.prm.dy; a.rdz = 1.0 / s.prm.dz;
        a.ext_bz = external_bz; a.n = (int)sp.n; a.sp = si; a.kind = sp.kind;
        a.status = s.d_status; a.diag = s.d_diag;
        a.track = s.track_erased ? 1 : 0;
        a.step = (uint32_t)s.step_index;
        a.cat = s.catch_erasures ? s.d_cat : nullptr;
        a.dcat = nullptr;
        a.trn_src = sp.trn[sp.cur];
        a.trn_dst = sp.trn[1 - sp.cur];
        a.dlo = s.diag_lo; a.dhi = s.diag_hi;
        OrderedArgs oa{o.tgt, o.key, o.val, o.nent, o.jcount, base,
                       ns > 1 ? sp.grank[sp.cur] : nullptr, ns > 1 ? sp.gstep : nullptr};
        const int nb = (int)((sp.n + 255) / 256);
        const bool vay = s.prm.pusher == QP_PUSHER_VAY;
        if (sp.kind == KIND_PHOTON)
            k_push64_ordered<QP_PUSHER_BORIS, KIND_PHOTON><<<nb, 256, 0, s.stream>>>(
                f, s.grid, src, dst, sp.perm, sp.newcell, sp.count, a, oa);
        else if (vay)
            k_push64_ordered<QP_PUSHER_VAY, KIND_LEPTON><<<nb, 256, 0, s.stream>>>(
                f, s.grid, src, dst, sp.perm, sp.newcell, sp.count, a, oa);
        else
            k_push64_ordered<QP_PUSHER_BORIS, KIND_LEPTON><<<nb, 256, 0, s.stream>>>(
                f, s.grid, src, dst, sp.perm, sp.newcell, sp.count, a, oa);
        s.launches++;
        base += sp.n;
    }
    const int nc3 = 3 * s.grid.nc;
    // bucket starts (jstart) and claim cursors (jcount, overwritten)
    void* keep = s.scan_tmp;
    s.scan_tmp = o.scan_tmp;
    exclusive_scan_i32(s, o.jcount, o.jstart, nc3, o.jcount);
    s.scan_tmp = keep;
    if (base > 0) {
        const int64_t ne = base * ENT_PER_PARTICLE;
        k_entries_scatter<<<(int)((ne + 255) / 256), 256, 0, s.stream>>>(base, o.nent, o.tgt, o.key, o.val,
                                                                         o.jcount, o.skey, o.sval);
        k_entries_sum<<<(nc3 + 255) / 256, 256, 0, s.stream>>>(s.grid.nc, o.jstart, o.skey, o.sval, f.jx, f.jy, f.jz);
        s.launches += 2;
    }
    QP_CUDA_CHECK(s, cudaGetLastError());
    return QP_OK;
}

// After the rebin of every species: the order keys of the new layout.
int ordered_after_rebin(State& s) {
    const int ns = (int)s.sp.size();
    if (ns < 2) return QP_OK;
    SpeciesOrder so{};
    so.ns = ns;
    for (int i = 0; i < ns; i++) {
        Species& sp = s.sp[i];
        so.start[i] = sp.cell_start;
        so.old_start[i] = sp.cell_next;  // the rebin swapped them
        so.perm[i] = sp.perm;
        so.gold[i] = sp.gstep;            // by the new slot (old traversal position)
        so.gnew[i] = sp.grank[sp.cur];
    }
    k_grank_merge<<<(s.grid.nc + 255) / 256, 256, 0, s.stream>>>(s.grid.nc, so);
    s.launches++;
    QP_CUDA_CHECK(s, cudaGetLastError());
    s.ord.epoch = s.layout_epoch;
    return QP_OK;
}

}  // namespace qp

extern "C" int qp_set_ordered_current(qp_handle* h, int enable) {
    qp::State* sp = qp::state_of(h);
    if (!sp) return QP_ERR_ARG;
    qp::State& s = *sp;
    if (enable && (!s.fp64 || s.prm.qed)) {
        s.err = "reference-order deposition needs FP64 precision and QED off";
        return QP_ERR_CONFIG;
    }
    s.ord.on = enable != 0;
    if (!s.ord.on) qp::ordered_release(s);
    else s.ord.epoch = -1;
    return QP_OK;
}
