// QED: the reference's photon-emission and Breit-Wheeler rates (mc.cpp:26-116)
// as device functions, and the counter-based random numbers that replace the
// reference's sequential lagged-Fibonacci stream (mc.cpp:12-23).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace qp {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplications with the
// published multipliers and Weyl key increments.  Counter = (a, b, c, d),
// key = (k0, k1).
struct Philox4 {
    uint32_t v[4];
};

__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                          uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t hi0 = mulhi32(M0, c0), lo0 = M0 * c0;
        const uint32_t hi1 = mulhi32(M1, c2), lo1 = M1 * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += W0; k1 += W1;
    }
    Philox4 o;
    o.v[0] = c0; o.v[1] = c1; o.v[2] = c2; o.v[3] = c3;
    return o;
}

// Two uniforms in [0, 1) with 53 random bits each.
__host__ __device__ __forceinline__ void uniform2(const Philox4& p, double& a, double& b) {
    const double s = 1.0 / 9007199254740992.0;  // 2^-53
    a = (double)(((uint64_t)(p.v[0] >> 5) << 26) | (p.v[1] >> 6)) * s;
    b = (double)(((uint64_t)(p.v[2] >> 5) << 26) | (p.v[3] >> 6)) * s;
}

// Random stream tags (third counter word).
enum RngTag : uint32_t { RNG_PUSH = 0x51u, RNG_VACUUM = 0x56u };

// ----------------------------------------------------------------------------
// Rates, mc.cpp:26-116.  e_s is the Sauter field in m c omega / e.
// ----------------------------------------------------------------------------

// The radicand of chi is >= 0 in exact arithmetic (|u| <= g); for a photon
// moving along E its two terms cancel, and FP32 rounding (with approximate
// division and square root) can leave it slightly negative, which would make
// chi, then every rate, NaN.  The FP32 path clamps it; the FP64 path keeps
// the reference's arithmetic as it is.
__device__ __forceinline__ double chi_radicand(double a2) { return a2; }
__device__ __forceinline__ float chi_radicand(float a2) { return a2 > 0.f ? a2 : 0.f; }

// chi = sqrt(|g E + u x B|^2 - (u.E)^2) / e_s  (mc.cpp:26-38)
template <typename T>
__device__ __forceinline__ T qed_chi(const T e[3], const T b[3], const T u[3], T g, T e_s) {
    T a1 = g * e[0] + u[1] * b[2] - u[2] * b[1];
    T a2 = a1 * a1;
    a1 = g * e[1] - u[0] * b[2] + u[2] * b[0];
    a2 += a1 * a1;
    a1 = g * e[2] + u[0] * b[1] - u[1] * b[0];
    a2 += a1 * a1;
    a1 = u[0] * e[0] + u[1] * e[1] + u[2] * e[2];
    a2 -= a1 * a1;
    return sqrt(chi_radicand(a2)) / e_s;
}

// Photon emission spectrum (mc.cpp:40-74) with the Airy-function fits
// Ai'(x) ~ exp(-2/3 x^1.5)/(2 sqrt(pi)) (x + 0.70861 (1 - 0.65 x/(1+x^2)))^1/4
// and int_x^inf Ai ~ exp(-2/3 x^1.5)/sqrt(2 pi)/(x + 0.80049)^3/4;
// 0.0020591 = 1/(137 * 2 sqrt(pi)).  For chi <= 0.133 the photon fraction r
// is mapped onto [0, r_max] (r is updated) and the rate carries r_max.
template <typename T>
__device__ __forceinline__ T qed_w(T g, T& r, T chi, T e_s) {
    if ((T(1) - r) * g < T(1) || r == T(0) || chi == T(0)) return T(0);
    T scale = T(1);
    if (!(chi > T(0.133))) {
        const T r_max = T(1) / (T(1) + T(2) / (T(3) * T(5) * chi));
        r = r_max * r;
        scale = r_max;
    }
    const T d = r / ((T(1) - r) * chi);
    // FP32 (denormals flushed): (1 - r) chi can underflow to 0 where FP64
    // keeps it; d is then infinite and the formula 0 * NaN.  The rate of
    // that limit is 0.
    if (sizeof(T) == 4 && !(d <= T(3.0e38))) return T(0);
    // d^(1/3): the reference's pow(d, 1./3) raises d to the rounded third,
    // cbrt to the exact one; for the d of these rates (up to ~1e30) the two
    // differ by about 1e-15 relative in FP64 (in FP32, where the third is
    // rounded to 24 bits, by up to ~1e-6, cbrt being the closer), and cbrt
    // costs a fraction of pow
    const T a = cbrt(d);
    const T kappa = a * a;
    const T k3 = (kappa + T(0.80049)) * (kappa + T(0.80049)) * (kappa + T(0.80049));
    const T inner = T(1) / sqrt(sqrt(k3)) -
                    (T(2) * (T(1) - r) + r * r) * chi * a / r *
                        sqrt(sqrt(kappa + T(0.70861) * (T(1) - T(0.65) * kappa / (T(1) + kappa * kappa))));
    return -scale * T(0.0020591) * e_s / (g * g) * exp(-T(2) * d / T(3)) * inner;
}

// Pair-creation spectrum (mc.cpp:76-97).
template <typename T>
__device__ __forceinline__ T qed_tilde_w(T g, T r, T chi, T e_s) {
    if (chi == T(0) || r * g < T(1) || (T(1) - r) * g < T(1)) return T(0);
    const T d = T(1) / (r * (T(1) - r) * chi);
    if (sizeof(T) == 4 && !(d <= T(3.0e38))) return T(0);  // as qed_w
    const T a = cbrt(d);  // as qed_w
    const T kappa = a * a;
    const T k3 = (kappa + T(0.80049)) * (kappa + T(0.80049)) * (kappa + T(0.80049));
    return T(0.0020591) * e_s / (g * g) * exp(-T(2) * d / T(3)) *
           (T(1) / sqrt(sqrt(k3)) - (T(2) * r * (T(1) - r) - T(1)) * chi * a *
                                        sqrt(sqrt(kappa + T(0.70861) * (T(1) - T(0.65) * kappa / (T(1) + kappa * kappa)))));
}

// Schwinger pair-creation probability per unit volume and time in
// omega^4/c^3 (mc.cpp:99-116).
template <typename T>
__device__ __forceinline__ T qed_vacuum_W(const T e[3], const T b[3], T e_s) {
    const T PI = T(3.141592653589793);
    const T f = T(0.5) * (e[0] * e[0] + e[1] * e[1] + e[2] * e[2] - b[0] * b[0] - b[1] * b[1] - b[2] * b[2]);
    const T g = e[0] * b[0] + e[1] * b[1] + e[2] * b[2];
    const T a = sqrt(f * f + g * g);
    const T xi = sqrt(a + f), theta = sqrt(a - f);
    if (xi == T(0)) return T(0);
    if (theta != T(0)) return e_s * e_s / (T(4) * PI) * xi * theta / tanh(PI * theta / xi) * exp(-PI * e_s / xi);
    return e_s * e_s / (T(4) * PI) * xi * xi / PI * exp(-PI * e_s / xi);
}

}  // namespace qp
