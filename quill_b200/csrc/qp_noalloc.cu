// qp_eval_qed_rates_noalloc: the QED rate evaluation of qp_eval_qed_rates
// without any device allocation.
//
// Who needs it: programs whose GPU memory belongs to another allocator (a
// framework's caching allocator, a host application that reserves the whole
// device up front) and that must not call cudaMalloc / cudaFree themselves;
// also loops where the implicit device-wide synchronisation of cudaFree is
// not acceptable.  qp_eval_qed_rates stages its inputs and outputs in device
// buffers it allocates and frees on every call; this variant stages them in
// a fixed array that lives in this library's device memory.
//
// The staging array is a file-scope __device__ array: every GPU that loads
// the library holds it (QP_NOALLOC_MAX_SAMPLES * 17 doubles, 2.2 MB) until
// the process exits.  All calls share it and it keeps the last call's
// contents; nothing in it needs to start at zero because the kernel writes
// every output element of a call.  Calls that overlap on the GPU (from
// several host threads, or on several devices sharing a host thread without
// waiting) race on the array.  The first call on a device looks up the
// array's device address (cudaGetSymbolAddress) with that device current;
// make that first call before any stream capture.  The address is kept for
// the life of the process: after cudaDeviceReset on that device the module
// is loaded again and the kept address is stale, so the entry point must not
// be used after a device reset.  The call leaves the caller's current device
// as it found it.
#include <cstdio>
#include <mutex>
#include <string>

#include "qp_internal.h"

#define QP_NOALLOC_MAX_SAMPLES 16384

namespace qp {
cudaError_t launch_qed_rates(int n, const double* d_in, double* d_out, double e_s, cudaStream_t st);
void set_global_error(const std::string& msg);
}  // namespace qp

// inputs (12 per sample) then outputs (5 per sample)
static __device__ __align__(256) double g_rate_staging[QP_NOALLOC_MAX_SAMPLES * 17];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_dev_ptr[kMaxDevices] = {nullptr};

// Device address of the staging array on `device` (current), looked up once.
cudaError_t staging_ptr(int device, double** out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_dev_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_rate_staging);
        if (e != cudaSuccess) return e;
        g_dev_ptr[device] = (double*)p;
    }
    *out = g_dev_ptr[device];
    return cudaSuccess;
}
}  // namespace

extern "C" int qp_eval_qed_rates_noalloc(int device, double lambda_cm, int64_t n, const double* in, double* out) {
    using qp::set_global_error;
    if (n < 0 || (n > 0 && (!in || !out))) {
        set_global_error("qp_eval_qed_rates_noalloc: null array or negative count");
        return QP_ERR_ARG;
    }
    if (n > QP_NOALLOC_MAX_SAMPLES) {
        char b[160];
        snprintf(b, sizeof b, "qp_eval_qed_rates_noalloc: %lld samples exceed the fixed staging size of %d",
                 (long long)n, QP_NOALLOC_MAX_SAMPLES);
        set_global_error(b);
        return QP_ERR_ARG;
    }
    if (device < 0 || device >= kMaxDevices) {
        set_global_error("qp_eval_qed_rates_noalloc: device ordinal out of range");
        return QP_ERR_ARG;
    }
    if (n == 0) return QP_OK;
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != device) e = cudaSetDevice(device);
    double* base = nullptr;
    if (e == cudaSuccess) e = staging_ptr(device, &base);
    if (e == cudaSuccess) {
        double* d_in = base;
        double* d_out = base + (size_t)QP_NOALLOC_MAX_SAMPLES * 12;
        e = cudaMemcpyAsync(d_in, in, (size_t)n * 12 * sizeof(double), cudaMemcpyDefault, 0);
        if (e == cudaSuccess) e = qp::launch_qed_rates((int)n, d_in, d_out, lambda_cm / 2.4263086e-10, 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, (size_t)n * 5 * sizeof(double), cudaMemcpyDefault, 0);
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    }
    // the caller's current device is restored whatever happened above
    if (prev >= 0 && prev != device) {
        const cudaError_t e2 = cudaSetDevice(prev);
        if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) {
        set_global_error(std::string("qp_eval_qed_rates_noalloc: ") + cudaGetErrorString(e));
        return QP_ERR_CUDA;
    }
    return QP_OK;
}
