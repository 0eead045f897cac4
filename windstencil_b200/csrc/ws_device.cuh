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
// The split keeps the reference's terms.  The WENO is an exact algebraic
// rewrite on stencil differences (below); with FMA contraction and the shared
// P/M division the results differ from the reference's evaluation order at
// the 1e-15 level only.  Parity with the reference is 1e-12 relative
// (tests/test_gpu_parity.py).
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
// evaluated on the first, second and third differences of the stencil:
//   D_j = t_{j+1}-t_j,  S_j = D_{j+1}-D_j,  T_j = S_{j+1}-S_j.
// In these variables the reference's three derivative rounds of candidate k
// are a 3-term first-difference form r_k, 6 x a 1-2 term second-difference
// form s_k, and 6 x T_k, so (all indicators divided by 720, eps likewise)
//   beta_k/720 = r_k^2 + 39 s_k^2 + 39.05 T_k^2
// and, because each candidate's coefficients sum to 12,
//   q_k = 12 t_3 + l_k(D),   face = t_3 + sum w_k l_k / (12 sum w_k).
// Both are exact algebraic rewrites of OCFD_Schemes.cpp:306-368; they remove
// about a fifth of the FP64 operations and agree with the reference form to
// ~1e-15 relative.  The result is returned as t_3 + num/den so that the P and
// M faces of one flux can share a single division.
// FP64: the reference's product weights w_k = d_k * prod_{j != k}(eps + beta_j)
// from shared partial products.  FP32 (mixed form): the equivalent normalised
// weights d_k / (eps + beta_k), which cannot overflow the FP32 range the way a
// product of four indicators can.
// ---------------------------------------------------------------------------
template <typename T>
struct WenoDiffs {
    T D0, D1, D2, D3, D4, D5, D6;
    T b0, b1, b2, b3, b4;
};

template <typename T>
__device__ __forceinline__ void weno7_indicators(const T t[8], WenoDiffs<T>& o) {
    o.D0 = t[1] - t[0]; o.D1 = t[2] - t[1]; o.D2 = t[3] - t[2]; o.D3 = t[4] - t[3];
    o.D4 = t[5] - t[4]; o.D5 = t[6] - t[5]; o.D6 = t[7] - t[6];
    const T S0 = o.D1 - o.D0, S1 = o.D2 - o.D1, S2 = o.D3 - o.D2, S3 = o.D4 - o.D3;
    const T S4 = o.D5 - o.D4, S5 = o.D6 - o.D5;
    const T T0 = S1 - S0, T1 = S2 - S1, T2 = S3 - S2, T3 = S4 - S3, T4 = S5 - S4;
    const T c2 = T(39.0), c3 = T(39.05);
    T r, s;
    r = T(2) * o.D0 - T(7) * o.D1 + T(11) * o.D2;    s = T(2) * S1 - S0;
    o.b0 = (c3 * T0) * T0 + ((c2 * s) * s + r * r);
    r = T(5) * o.D2 - o.D1 + T(2) * o.D3;            s = S2;
    o.b1 = (c3 * T1) * T1 + ((c2 * s) * s + r * r);
    r = T(2) * o.D2 + T(5) * o.D3 - o.D4;            s = S3;
    o.b2 = (c3 * T2) * T2 + ((c2 * s) * s + r * r);
    r = T(11) * o.D3 - T(7) * o.D4 + T(2) * o.D5;    s = T(2) * S3 - S4;
    o.b3 = (c3 * T3) * T3 + ((c2 * s) * s + r * r);
    r = T(26) * o.D4 - T(31) * o.D5 + T(11) * o.D6;  s = T(3) * S4 - T(2) * S5;
    o.b4 = (c3 * T4) * T4 + ((c2 * s) * s + r * r);
}

template <typename T>
__device__ __forceinline__ void weno7_candidates(const WenoDiffs<T>& o, T w0, T w1, T w2, T w3,
                                                 T w4, T& num, T& den) {
    const T l0 = T(3) * o.D0 - T(10) * o.D1 + T(13) * o.D2;
    const T l1 = T(4) * o.D2 - o.D1 + T(3) * o.D3;
    const T l2 = o.D2 + T(6) * o.D3 - o.D4;
    const T l3 = T(9) * o.D3 - T(4) * o.D4 + o.D5;
    const T l4 = T(12) * o.D3 - T(13) * o.D4 + T(10) * o.D5 - T(3) * o.D6;
    num = w0 * l0 + w1 * l1 + w2 * l2 + w3 * l3 + w4 * l4;
    den = T(12) * (w0 + w1 + w2 + w3 + w4);
}

// face value = t[3] + num/den
template <typename T>
__device__ __forceinline__ void weno7_symbo_nd(const T t[8], T& num, T& den);

template <>
__device__ __forceinline__ void weno7_symbo_nd<double>(const double t[8], double& num,
                                                       double& den) {
    WenoDiffs<double> o;
    weno7_indicators<double>(t, o);
    const double b4 = fmax(fmax(fmax(o.b0, o.b1), fmax(o.b2, o.b3)), o.b4);
    const double e = 2.592e-6 / 720.0;
    const double e0 = e + o.b0, e1 = e + o.b1, e2 = e + o.b2, e3 = e + o.b3, e4 = e + b4;
    const double p01 = e0 * e1, p34 = e3 * e4;
    const double p012 = p01 * e2, p234 = e2 * p34;
    weno7_candidates<double>(o, 0.0401954833730 * (e1 * p234), 0.2493800006710 * (e0 * p234),
                             0.4802686256260 * (p01 * p34), 0.2009775476730 * (p012 * e4),
                             0.0291783426580 * (p012 * e3), num, den);
}

// ---------------------------------------------------------------------------
// Mixed form: the P and M reconstructions of one face are the same arithmetic
// on two stencils, so they run as the two lanes of Blackwell's packed FP32x2
// instructions (FFMA2/FADD2/FMUL2): t[k] = (P stencil k, M stencil k).  The
// normalised weights d_k/(eps+beta_k) take their reciprocals in pairs,
// 1/a = b/(ab) and 1/b = a/(ab), from the approximate hardware reciprocal;
// ab stays inside the FP32 range for any indicator below ~1e19.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float c) { return make_float2(c, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(f2(-1.f), b, a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float2 rcp2(float2 x) {
    return make_float2(rcp_approx(x.x), rcp_approx(x.y));
}

// face value of lane L = t[3].L + num.L / den.L
__device__ __forceinline__ void weno7_symbo_pm_f32x2(const float2 t[8], float2& num,
                                                     float2& den) {
    const float2 D0 = sub2(t[1], t[0]), D1 = sub2(t[2], t[1]), D2 = sub2(t[3], t[2]);
    const float2 D3 = sub2(t[4], t[3]), D4 = sub2(t[5], t[4]), D5 = sub2(t[6], t[5]);
    const float2 D6 = sub2(t[7], t[6]);
    const float2 S0 = sub2(D1, D0), S1 = sub2(D2, D1), S2 = sub2(D3, D2), S3 = sub2(D4, D3);
    const float2 S4 = sub2(D5, D4), S5 = sub2(D6, D5);
    const float2 T0 = sub2(S1, S0), T1 = sub2(S2, S1), T2 = sub2(S3, S2), T3 = sub2(S4, S3);
    const float2 T4 = sub2(S5, S4);
    const float2 c2 = f2(39.0f), c3 = f2(39.05f);
    auto beta = [&](float2 r, float2 s, float2 T) {
        return fma2(mul2(c3, T), T, fma2(mul2(c2, s), s, mul2(r, r)));
    };
    float2 r, s;
    r = fma2(f2(11.f), D2, fma2(f2(-7.f), D1, mul2(f2(2.f), D0)));
    s = fma2(f2(2.f), S1, mul2(f2(-1.f), S0));
    const float2 b0 = beta(r, s, T0);
    r = fma2(f2(2.f), D3, fma2(f2(5.f), D2, mul2(f2(-1.f), D1)));
    const float2 b1 = beta(r, S2, T1);
    r = fma2(f2(-1.f), D4, fma2(f2(5.f), D3, mul2(f2(2.f), D2)));
    const float2 b2 = beta(r, S3, T2);
    r = fma2(f2(2.f), D5, fma2(f2(-7.f), D4, mul2(f2(11.f), D3)));
    s = fma2(f2(2.f), S3, mul2(f2(-1.f), S4));
    const float2 b3 = beta(r, s, T3);
    r = fma2(f2(11.f), D6, fma2(f2(-31.f), D5, mul2(f2(26.f), D4)));
    s = fma2(f2(3.f), S4, mul2(f2(-2.f), S5));
    float2 b4 = beta(r, s, T4);
    b4.x = fmaxf(fmaxf(fmaxf(b0.x, b1.x), fmaxf(b2.x, b3.x)), b4.x);
    b4.y = fmaxf(fmaxf(fmaxf(b0.y, b1.y), fmaxf(b2.y, b3.y)), b4.y);
    const float2 e = f2(2.592e-6f / 720.0f);
    const float2 e0 = add2(e, b0), e1 = add2(e, b1), e2 = add2(e, b2), e3 = add2(e, b3);
    const float2 e4 = add2(e, b4);
    const float2 r01 = rcp2(mul2(e0, e1)), r23 = rcp2(mul2(e2, e3)), r4 = rcp2(e4);
    const float2 w0 = mul2(mul2(f2(0.0401954833730f), e1), r01);
    const float2 w1 = mul2(mul2(f2(0.2493800006710f), e0), r01);
    const float2 w2 = mul2(mul2(f2(0.4802686256260f), e3), r23);
    const float2 w3 = mul2(mul2(f2(0.2009775476730f), e2), r23);
    const float2 w4 = mul2(f2(0.0291783426580f), r4);
    const float2 l0 = fma2(f2(13.f), D2, fma2(f2(-10.f), D1, mul2(f2(3.f), D0)));
    const float2 l1 = fma2(f2(3.f), D3, fma2(f2(4.f), D2, mul2(f2(-1.f), D1)));
    const float2 l2 = fma2(f2(-1.f), D4, fma2(f2(6.f), D3, D2));
    const float2 l3 = fma2(f2(-4.f), D4, fma2(f2(9.f), D3, D5));
    const float2 l4 =
        fma2(f2(-3.f), D6, fma2(f2(10.f), D5, fma2(f2(-13.f), D4, mul2(f2(12.f), D3))));
    num = fma2(w4, l4, fma2(w3, l3, fma2(w2, l2, fma2(w1, l1, mul2(w0, l0)))));
    den = mul2(f2(12.f), add2(add2(add2(w0, w1), add2(w2, w3)), w4));
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
