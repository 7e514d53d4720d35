// Forward-mode dual numbers: a value and its derivatives along N input
// directions.  The adjoint kernels evaluate the particle update (gather,
// Boris push, displacement, segment-split deposition) on Dual<N> to get the
// local Jacobian-vector products they contract with the adjoint variables.
// Branches (cell floors, crossing order) are taken on the value part, so the
// derivative is that of the branch the forward step took.
// The type and its functions live in qp::ad so that they are found by
// argument-dependent lookup for Dual arguments only and do not hide the
// math library's sqrt / floor for double inside namespace qp.
#pragma once

#include <cuda_runtime.h>

namespace qp {
namespace ad {

template <int N>
struct Dual {
    double v;
    double d[N];
    __device__ __forceinline__ Dual() : v(0.0) {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = 0.0;
    }
    __device__ __forceinline__ Dual(double x) : v(x) {  // constant
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = 0.0;
    }
    __device__ __forceinline__ explicit Dual(int x) : Dual((double)x) {}
    __device__ __forceinline__ static Dual seed(double x, int dir) {
        Dual r(x);
        r.d[dir] = 1.0;
        return r;
    }
};

#define QP_DUAL_BIN(OP, VAL, DER)                                                                \
    template <int N>                                                                             \
    __device__ __forceinline__ Dual<N> operator OP(const Dual<N>& a, const Dual<N>& b) {        \
        Dual<N> r;                                                                               \
        r.v = VAL;                                                                               \
        _Pragma("unroll") for (int i = 0; i < N; i++) r.d[i] = DER;                              \
        return r;                                                                                \
    }

QP_DUAL_BIN(+, a.v + b.v, a.d[i] + b.d[i])
QP_DUAL_BIN(-, a.v - b.v, a.d[i] - b.d[i])
QP_DUAL_BIN(*, a.v * b.v, a.d[i] * b.v + a.v * b.d[i])
#undef QP_DUAL_BIN

template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> r;
    r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) { return a / Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }
template <int N> __device__ __forceinline__ Dual<N>& operator+=(Dual<N>& a, const Dual<N>& b) { a = a + b; return a; }
template <int N> __device__ __forceinline__ Dual<N>& operator-=(Dual<N>& a, const Dual<N>& b) { a = a - b; return a; }
template <int N> __device__ __forceinline__ Dual<N>& operator/=(Dual<N>& a, const Dual<N>& b) { a = a / b; return a; }

template <int N>
__device__ __forceinline__ Dual<N> sqrt(const Dual<N>& a) {
    Dual<N> r;
    r.v = ::sqrt(a.v);
    const double h = 0.5 / r.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * h;
    return r;
}
template <int N> __device__ __forceinline__ bool operator>(const Dual<N>& a, const Dual<N>& b) { return a.v > b.v; }
template <int N> __device__ __forceinline__ bool operator<(const Dual<N>& a, const Dual<N>& b) { return a.v < b.v; }
template <int N> __device__ __forceinline__ double floor(const Dual<N>& a) { return ::floor(a.v); }
template <int N> __device__ __forceinline__ bool isfinite(const Dual<N>& a) { return ::isfinite(a.v); }

}  // namespace ad
using ad::Dual;
}  // namespace qp
