// ws_device.cuh -- per-point device arithmetic of the BF3W inviscid RHS.
//
// Steger-Warming flux-vector splitting with the entropy fix and the 7th-order
// WENO-SYMBO reconstruction, in FP64 (the drop-in) and FP32 (the mixed form).
// The formulas are those of the reference:
//   split : src/solver/OCFD_NS_Jacobian3d.cpp:55-129 (and its inlined copies in
//           src/kernels/OCFD_split.cpp:199-255), with tmp0 = rho*(0.5/gamma) as
//           the fused kernel forms it (OCFD_split.cpp:229, 0.5/Gamma passed at
//           OCFD_NS_Jacobian3d.cpp:251);
//   WENO  : src/kernels/OCFD_Schemes.cpp:306-368 (P) and :491-553 (M); the M
//           form equals the P form on the reversed stencil.
// The FP64 code keeps the reference's terms; it lets the compiler contract
// multiply-adds and reassociates two products (the leave-one-out weight
// products and the P+M face sum), which changes results at the 1e-16 level
// only.  Parity with the reference is 1e-12 relative (tests/test_gpu_parity.py).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ws {

// Constants derived from gamma, Ama and EPSL_SW (OCFD_init.cpp:379-407).
template <typename T>
struct SplitK {
    T eps2;   // epsl_sw^2
    T hrg;    // 0.5/gamma
    T c1;     // split_C1 = 2(gamma-1)
    T c3;     // split_C3 = (3-gamma)/(2(gamma-1))
    T gm1;    // gamma-1
};

__device__ __forceinline__ double ws_sqrt(double x) { return sqrt(x); }
// FP32 square root and quotient of the mixed form: the hardware approximations
// (sqrt.approx / div.full, relative error ~2^-22), far below the FP32
// rounding noise the mixed form already accepts.
__device__ __forceinline__ float ws_sqrt(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ double ws_div(double a, double b) { return a / b; }
__device__ __forceinline__ float ws_div(float a, float b) { return __fdividef(a, b); }

// ---------------------------------------------------------------------------
// Steger-Warming split, Cartesian metrics (gradient = unit vector of DIR,
// |grad| = 1): F+ in out[0..4], F- in out[5..9].
// ---------------------------------------------------------------------------
template <int DIR, typename T>
__device__ __forceinline__ void sw_split_cart(T d, T u, T v, T w, T c,
                                              const SplitK<T>& k, T out[10]) {
    const T un = DIR == 0 ? u : (DIR == 1 ? v : w);
    const T e1 = un, e2 = un - c, e3 = un + c;
    const T e1p = (e1 + ws_sqrt(e1 * e1 + k.eps2)) * T(0.5);
    const T e2p = (e2 + ws_sqrt(e2 * e2 + k.eps2)) * T(0.5);
    const T e3p = (e3 + ws_sqrt(e3 * e3 + k.eps2)) * T(0.5);
    const T e1m = e1 - e1p, e2m = e2 - e2p, e3m = e3 - e3p;
    const T t0 = d * k.hrg;
    // velocity -/+ c along DIR
    const T uc1 = DIR == 0 ? u - c : u, uc2 = DIR == 0 ? u + c : u;
    const T vc1 = DIR == 1 ? v - c : v, vc2 = DIR == 1 ? v + c : v;
    const T wc1 = DIR == 2 ? w - c : w, wc2 = DIR == 2 ? w + c : w;
    const T vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * T(0.5);
    const T vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * T(0.5);
    const T vv = k.gm1 * (u * u + v * v + w * w);
    const T w2 = k.c3 * c * c;
    const T a1p = k.c1 * e1p, a1m = k.c1 * e1m;
    out[0] = t0 * (a1p + e2p + e3p);
    out[1] = t0 * (a1p * u + e2p * uc1 + e3p * uc2);
    out[2] = t0 * (a1p * v + e2p * vc1 + e3p * vc2);
    out[3] = t0 * (a1p * w + e2p * wc1 + e3p * wc2);
    out[4] = t0 * (e1p * vv + e2p * vvc1 + e3p * vvc2 + w2 * (e2p + e3p));
    out[5] = t0 * (a1m + e2m + e3m);
    out[6] = t0 * (a1m * u + e2m * uc1 + e3m * uc2);
    out[7] = t0 * (a1m * v + e2m * vc1 + e3m * vc2);
    out[8] = t0 * (a1m * w + e2m * wc1 + e3m * wc2);
    out[9] = t0 * (e1m * vv + e2m * vvc1 + e3m * vvc2 + w2 * (e2m + e3m));
}

// ---------------------------------------------------------------------------
// Steger-Warming split, general metric gradient (a1,a2,a3).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void sw_split_gen(T d, T u, T v, T w, T c, T a1, T a2, T a3,
                                             const SplitK<T>& k, T out[10]) {
    const T ss = ws_sqrt(a1 * a1 + a2 * a2 + a3 * a3);
    const T rcp = ws_div(T(1), ss);
    const T k1 = a1 * rcp, k2 = a2 * rcp, k3 = a3 * rcp;
    const T vs = a1 * u + a2 * v + a3 * w;
    const T e1 = vs, e2 = vs - c * ss, e3 = vs + c * ss;
    const T e1p = (e1 + ws_sqrt(e1 * e1 + k.eps2)) * T(0.5);
    const T e2p = (e2 + ws_sqrt(e2 * e2 + k.eps2)) * T(0.5);
    const T e3p = (e3 + ws_sqrt(e3 * e3 + k.eps2)) * T(0.5);
    const T e1m = e1 - e1p, e2m = e2 - e2p, e3m = e3 - e3p;
    const T t0 = d * k.hrg;
    const T uc1 = u - c * k1, uc2 = u + c * k1;
    const T vc1 = v - c * k2, vc2 = v + c * k2;
    const T wc1 = w - c * k3, wc2 = w + c * k3;
    const T vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * T(0.5);
    const T vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * T(0.5);
    const T vv = k.gm1 * (u * u + v * v + w * w);
    const T w2 = k.c3 * c * c;
    const T a1p = k.c1 * e1p, a1m = k.c1 * e1m;
    out[0] = t0 * (a1p + e2p + e3p);
    out[1] = t0 * (a1p * u + e2p * uc1 + e3p * uc2);
    out[2] = t0 * (a1p * v + e2p * vc1 + e3p * vc2);
    out[3] = t0 * (a1p * w + e2p * wc1 + e3p * wc2);
    out[4] = t0 * (e1p * vv + e2p * vvc1 + e3p * vvc2 + w2 * (e2p + e3p));
    out[5] = t0 * (a1m + e2m + e3m);
    out[6] = t0 * (a1m * u + e2m * uc1 + e3m * uc2);
    out[7] = t0 * (a1m * v + e2m * vc1 + e3m * vc2);
    out[8] = t0 * (a1m * w + e2m * wc1 + e3m * wc2);
    out[9] = t0 * (e1m * vv + e2m * vvc1 + e3m * vvc2 + w2 * (e2m + e3m));
}

// ---------------------------------------------------------------------------
// WENO7-SYMBO face value from t[0..7] = points i-3..i+4 (P orientation),
// returned as numerator/denominator so that the caller can combine the P and
// M faces with one division.  FP64: the reference's product weights
// w_k = d_k * prod_{j != k}(eps + beta_j), formed with shared partial
// products.  FP32: the equivalent normalised weights d_k / (eps + beta_k),
// which cannot overflow the FP32 range the way a product of four indicators
// can.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void weno7_symbo_nd(const T t[8], T& num, T& den);

template <>
__device__ __forceinline__ void weno7_symbo_nd<double>(const double t[8], double& num,
                                                       double& den) {
    double q, b0, b1, b2, b3, b4;
    q = -2.0 * t[0] + 9.0 * t[1] - 18.0 * t[2] + 11.0 * t[3];   b0 = 720.0 * q * q;
    q = t[1] - 6.0 * t[2] + 3.0 * t[3] + 2.0 * t[4];             b1 = 720.0 * q * q;
    q = -2.0 * t[2] - 3.0 * t[3] + 6.0 * t[4] - t[5];            b2 = 720.0 * q * q;
    q = -11.0 * t[3] + 18.0 * t[4] - 9.0 * t[5] + 2.0 * t[6];    b3 = 720.0 * q * q;
    q = -26.0 * t[4] + 57.0 * t[5] - 42.0 * t[6] + 11.0 * t[7]; b4 = 720.0 * q * q;
    q = -6.0 * t[0] + 24.0 * t[1] - 30.0 * t[2] + 12.0 * t[3];  b0 += 780.0 * q * q;
    q = 6.0 * t[2] - 12.0 * t[3] + 6.0 * t[4];                   b1 += 780.0 * q * q;
    q = 6.0 * t[3] - 12.0 * t[4] + 6.0 * t[5];                   b2 += 780.0 * q * q;
    q = 12.0 * t[3] - 30.0 * t[4] + 24.0 * t[5] - 6.0 * t[6];    b3 += 780.0 * q * q;
    q = 18.0 * t[4] - 48.0 * t[5] + 42.0 * t[6] - 12.0 * t[7];   b4 += 780.0 * q * q;
    q = -6.0 * t[0] + 18.0 * (t[1] - t[2]) + 6.0 * t[3];         b0 += 781.0 * q * q;
    q = -6.0 * t[1] + 18.0 * (t[2] - t[3]) + 6.0 * t[4];         b1 += 781.0 * q * q;
    q = -6.0 * t[2] + 18.0 * (t[3] - t[4]) + 6.0 * t[5];         b2 += 781.0 * q * q;
    q = -6.0 * t[3] + 18.0 * (t[4] - t[5]) + 6.0 * t[6];         b3 += 781.0 * q * q;
    q = -6.0 * t[4] + 18.0 * (t[5] - t[6]) + 6.0 * t[7];         b4 += 781.0 * q * q;
    b4 = fmax(fmax(fmax(b0, b1), fmax(b2, b3)), b4);
    const double e = 2.592e-6;
    const double e0 = e + b0, e1 = e + b1, e2 = e + b2, e3 = e + b3, e4 = e + b4;
    // leave-one-out products from prefix / suffix partial products
    const double p01 = e0 * e1, p34 = e3 * e4;
    const double p012 = p01 * e2, p234 = e2 * p34;
    const double w0 = 0.0401954833730 * (e1 * p234);
    const double w1 = 0.2493800006710 * (e0 * p234);
    const double w2 = 0.4802686256260 * (p01 * p34);
    const double w3 = 0.2009775476730 * (p012 * e4);
    const double w4 = 0.0291783426580 * (p012 * e3);
    double acc;
    q = -3.0 * t[0] + 13.0 * t[1] - 23.0 * t[2] + 25.0 * t[3];  acc = w0 * q;
    q = t[1] - 5.0 * t[2] + 13.0 * t[3] + 3.0 * t[4];            acc += w1 * q;
    q = -t[2] + 7.0 * t[3] + 7.0 * t[4] - t[5];                  acc += w2 * q;
    q = 3.0 * t[3] + 13.0 * t[4] - 5.0 * t[5] + t[6];            acc += w3 * q;
    q = 25.0 * t[4] - 23.0 * t[5] + 13.0 * t[6] - 3.0 * t[7];    acc += w4 * q;
    num = acc;
    den = 12.0 * (w0 + w1 + w2 + w3 + w4);
}

template <>
__device__ __forceinline__ void weno7_symbo_nd<float>(const float t[8], float& num,
                                                      float& den) {
    float q, b0, b1, b2, b3, b4;
    q = -2.0f * t[0] + 9.0f * t[1] - 18.0f * t[2] + 11.0f * t[3];   b0 = 720.0f * q * q;
    q = t[1] - 6.0f * t[2] + 3.0f * t[3] + 2.0f * t[4];              b1 = 720.0f * q * q;
    q = -2.0f * t[2] - 3.0f * t[3] + 6.0f * t[4] - t[5];             b2 = 720.0f * q * q;
    q = -11.0f * t[3] + 18.0f * t[4] - 9.0f * t[5] + 2.0f * t[6];    b3 = 720.0f * q * q;
    q = -26.0f * t[4] + 57.0f * t[5] - 42.0f * t[6] + 11.0f * t[7]; b4 = 720.0f * q * q;
    q = -6.0f * t[0] + 24.0f * t[1] - 30.0f * t[2] + 12.0f * t[3];  b0 += 780.0f * q * q;
    q = 6.0f * t[2] - 12.0f * t[3] + 6.0f * t[4];                    b1 += 780.0f * q * q;
    q = 6.0f * t[3] - 12.0f * t[4] + 6.0f * t[5];                    b2 += 780.0f * q * q;
    q = 12.0f * t[3] - 30.0f * t[4] + 24.0f * t[5] - 6.0f * t[6];   b3 += 780.0f * q * q;
    q = 18.0f * t[4] - 48.0f * t[5] + 42.0f * t[6] - 12.0f * t[7];  b4 += 780.0f * q * q;
    q = -6.0f * t[0] + 18.0f * (t[1] - t[2]) + 6.0f * t[3];         b0 += 781.0f * q * q;
    q = -6.0f * t[1] + 18.0f * (t[2] - t[3]) + 6.0f * t[4];         b1 += 781.0f * q * q;
    q = -6.0f * t[2] + 18.0f * (t[3] - t[4]) + 6.0f * t[5];         b2 += 781.0f * q * q;
    q = -6.0f * t[3] + 18.0f * (t[4] - t[5]) + 6.0f * t[6];         b3 += 781.0f * q * q;
    q = -6.0f * t[4] + 18.0f * (t[5] - t[6]) + 6.0f * t[7];         b4 += 781.0f * q * q;
    b4 = fmaxf(fmaxf(fmaxf(b0, b1), fmaxf(b2, b3)), b4);
    const float e = 2.592e-6f;
    const float w0 = __fdividef(0.0401954833730f, e + b0);
    const float w1 = __fdividef(0.2493800006710f, e + b1);
    const float w2 = __fdividef(0.4802686256260f, e + b2);
    const float w3 = __fdividef(0.2009775476730f, e + b3);
    const float w4 = __fdividef(0.0291783426580f, e + b4);
    float acc;
    q = -3.0f * t[0] + 13.0f * t[1] - 23.0f * t[2] + 25.0f * t[3];  acc = w0 * q;
    q = t[1] - 5.0f * t[2] + 13.0f * t[3] + 3.0f * t[4];             acc += w1 * q;
    q = -t[2] + 7.0f * t[3] + 7.0f * t[4] - t[5];                    acc += w2 * q;
    q = 3.0f * t[3] + 13.0f * t[4] - 5.0f * t[5] + t[6];             acc += w3 * q;
    q = 25.0f * t[4] - 23.0f * t[5] + 13.0f * t[6] - 3.0f * t[7];    acc += w4 * q;
    num = acc;
    den = 12.0f * (w0 + w1 + w2 + w3 + w4);
}

// ---------------------------------------------------------------------------
// Small PTX helpers: 8-byte asynchronous global->shared copies (cp.async).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

}  // namespace ws
