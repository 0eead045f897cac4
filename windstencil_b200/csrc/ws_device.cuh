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

// SSP-RK3 stage formulas, src/solver/OCFD_time.cpp:15-65 (ker1/ker2/ker3):
// stage 1 f = fn + dt*du; stage 2 f = 3/4 fn + 1/4 (f + dt*du);
// stage 3 f = 1/3 fn + 2/3 (f + dt*du).
__device__ __forceinline__ double ws_rk_stage(int krk, double fn, double f, double du,
                                              double dt) {
    if (krk == 1) return fn + dt * du;
    if (krk == 2) return (3.0 / 4.0) * fn + (1.0 / 4.0) * (f + dt * du);
    return (1.0 / 3.0) * fn + (2.0 / 3.0) * (f + dt * du);
}

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
// evaluated on the first differences of the stencil D_j = t_{j+1}-t_j, with
// S_j = D_{j+1}-D_j and T_j = S_{j+1}-S_j.  In these variables the
// reference's three derivative rounds of candidate k (OCFD_Schemes.cpp:
// 306-368) are a 3-term first-difference form r_k, 6 x a 1-2 term
// second-difference form s_k and 6 x T_k, so
//   beta_k / (720 * 39) = (r_k/sqrt 39)^2 + s_k^2 + (39.05/39) T_k^2,
// a positive-definite quadratic form in three consecutive D_j.  The common
// factor 720*39 is taken out of every indicator and of eps, which leaves the
// normalised weights unchanged, and each form is evaluated through its
// Cholesky factor (wk::UF below): e_k = eps' + beta'_k costs nine operations
// on the D_j and needs no S_j / T_j.  Each candidate's coefficients sum to
// 12, so q_k = 12 t_3 + l_k(D)
// and face = t_3 + sum d_k P_k l_k / (12 sum d_k P_k), P_k the product of the
// other four e_j (the reference's product weights); d_k is folded into the
// l_k coefficients.  All of this is an exact algebraic rewrite (agreement
// with the reference form ~1e-15 relative) that removes about a third of the
// FP64 operations.  The result is t_3 + num/den so that the P and M faces of
// one flux can share a single division.
// ---------------------------------------------------------------------------
namespace wk {
constexpr double R = 0.16012815380508713;     // 1/sqrt(39)
constexpr double C = 39.05 / 39.0;            // third-derivative weight / second's
constexpr double EPS = 2.592e-6 / (720.0 * 39.0);
constexpr double D0 = 0.0401954833730, D1 = 0.2493800006710, D2 = 0.4802686256260,
                 D3 = 0.2009775476730, D4 = 0.0291783426580;
}  // namespace wk


// The FP64 coefficients live in constant memory: a DFMA/DMUL takes a
// constant-bank operand directly, whereas a 64-bit literal that does not fit
// the instruction's immediate field is rebuilt in uniform registers (two
// moves) at every use -- about 30 extra issue slots per reconstruction.
// The array is never written; its values are the constexpr ones above.
namespace wk {
enum Coef {
    E0, E1 = E0 + 6, E2 = E1 + 6, E3 = E2 + 6, E4 = E3 + 6,     // indicator factors
    EPSC = E4 + 6,
    R11, RM7, R2, R5, RM1, RM31, R26, CC,                       // chain form

    L0A, L0B, L0C, L1A, L1B, L1C, L2A, L2B, L2C, L3A, L3B, L3C,   // d_k l_k
    L4A, L4B, L4C, L4D,
    Q0, Q1, Q2, Q3, Q4,                                       // 12 d_k
    NCOEF
};
// Cholesky factors of the five indicator forms.  In the variables above,
// e_k - eps' = r_k^2 + s_k^2 + (39.05/39) T_k^2 is a positive-definite
// quadratic form Q_k in three consecutive first differences; with those
// taken in the order (v0, v1, v2) below, Q_k = U^T U for an upper-triangular
// U, so e_k = eps' + y0^2 + y1^2 + y2^2 with
//   y0 = U00 v0 + U01 v1 + U02 v2,  y1 = U11 v1 + U12 v2,  y2 = U22 v2
// (nine operations, and no second / third difference chains).  The factors
// follow from the reference's derivative-round weights alone (rounded from a
// 40-digit evaluation); the identity holds to 1e-16 relative.
//   e0: (D2, D0, D1)  e1: (D3, D1, D2)  e2: (D2, D4, D3)
//   e3: (D3, D4, D5)  e4: (D4, D5, D6)
constexpr double UF[30] = {
    2.8467255143139729562, 1.2524511398998827387, -3.5047014637543644273,
    0.73158205008709597394, -1.3287246702332208323, 0.4616241568745027212,
    1.4504641167040823579, 0.65496277299069166801, -1.8932931980378698419,
    0.77327022632416193136, -1.1519034838986927736, 0.85715405628127057224,
    1.0506408300871206129, 0.90421005237462993517, -1.6619893270367691926,
    1.0996941657150618495, -1.4803950271616324632, 0.83209127295316749707,
    2.8467255143139729562, -3.5047014637543644273, 1.2524511398998827387,
    1.4066293440336288338, -0.69106415444385934995, 0.24008879701567067037,
    5.22825165658802088, -7.2049383318732343462, 2.7417607885329328577,
    1.3172006225543553721, -0.75306405648544262277, 0.13960107141105386569};
}  // namespace wk
static __constant__ double wkc[wk::NCOEF] = {
    wk::UF[0], wk::UF[1], wk::UF[2], wk::UF[3], wk::UF[4], wk::UF[5],
    wk::UF[6], wk::UF[7], wk::UF[8], wk::UF[9], wk::UF[10], wk::UF[11],
    wk::UF[12], wk::UF[13], wk::UF[14], wk::UF[15], wk::UF[16], wk::UF[17],
    wk::UF[18], wk::UF[19], wk::UF[20], wk::UF[21], wk::UF[22], wk::UF[23],
    wk::UF[24], wk::UF[25], wk::UF[26], wk::UF[27], wk::UF[28], wk::UF[29],
    wk::EPS,
    11 * wk::R, -7 * wk::R, 2 * wk::R, 5 * wk::R, -wk::R, -31 * wk::R, 26 * wk::R, wk::C,
    13 * wk::D0, -10 * wk::D0, 3 * wk::D0, 3 * wk::D1, 4 * wk::D1, -wk::D1,
    -wk::D2, 6 * wk::D2, wk::D2, wk::D3, -4 * wk::D3, 9 * wk::D3,
    -3 * wk::D4, 10 * wk::D4, -13 * wk::D4, 12 * wk::D4,
    12 * wk::D0, 12 * wk::D1, 12 * wk::D2, 12 * wk::D3, 12 * wk::D4};

// eps' + the Cholesky form of factor set `f` (wk::E0 .. wk::E4) on (v0, v1, v2)
__device__ __forceinline__ double weno_e(double v0, double v1, double v2, int f) {
    const double* k = wkc + f;
    const double y0 = fma(k[2], v2, fma(k[1], v1, k[0] * v0));
    const double y1 = fma(k[4], v2, k[3] * v1);
    const double y2 = k[5] * v2;
    return fma(y0, y0, fma(y1, y1, fma(y2, y2, wkc[wk::EPSC])));
}

// max of two indicators (both > 0): positive doubles order like their bit
// patterns read as signed integers, so the comparison runs on the integer
// pipe instead of the FP64 one (a NaN operand is selected and propagates to
// the face value, as it would through the products anyway)
__device__ __forceinline__ double pos_max(double a, double b) {
    const long long x = __double_as_longlong(a), y = __double_as_longlong(b);
    return __longlong_as_double(x > y ? x : y);
}

// face value = t[3] + num/den
// The same indicators in the difference-chain form: r_k from the D_j, s_k from
// the S_j and C T_k^2 from the T_j (ten operations per indicator counting the
// shared S_j / T_j chains, against nine for the Cholesky form).  It holds
// fewer values live at once, which is what the stage kernels (EPI), at the
// 80-register limit of 704 threads, need: with the Cholesky form they spill.
__device__ __forceinline__ double weno_e_chain(double r, double s, double t3) {
    return fma(r, r, fma(s, s, fma(wkc[wk::CC] * t3, t3, wkc[wk::EPSC])));
}

// face value = t[3] + num/den; CHOL selects the indicator form (identical
// values up to rounding)
template <bool CHOL>
__device__ __forceinline__ void weno7_symbo_nd(const double t[8], double& num, double& den) {
    using namespace wk;
    const double* k = wkc;
    const double D0 = t[1] - t[0], D1 = t[2] - t[1], D2 = t[3] - t[2], D3 = t[4] - t[3];
    const double D4 = t[5] - t[4], D5 = t[6] - t[5], D6 = t[7] - t[6];
    double e0, e1, e2, e3, e4;
    if (CHOL) {
        e0 = weno_e(D2, D0, D1, E0);
        e1 = weno_e(D3, D1, D2, E1);
        e2 = weno_e(D2, D4, D3, E2);
        e3 = weno_e(D3, D4, D5, E3);
        e4 = weno_e(D4, D5, D6, E4);
    } else {
        const double S0 = D1 - D0, S1 = D2 - D1, S2 = D3 - D2, S3 = D4 - D3;
        const double S4 = D5 - D4, S5 = D6 - D5;
        const double T0 = S1 - S0, T1 = S2 - S1, T2 = S3 - S2, T3 = S4 - S3, T4 = S5 - S4;
        e0 = weno_e_chain(fma(k[R11], D2, fma(k[RM7], D1, k[R2] * D0)), fma(2.0, S1, -S0), T0);
        e1 = weno_e_chain(fma(k[R2], D3, fma(k[R5], D2, k[RM1] * D1)), S2, T1);
        e2 = weno_e_chain(fma(k[RM1], D4, fma(k[R5], D3, k[R2] * D2)), S3, T2);
        e3 = weno_e_chain(fma(k[R2], D5, fma(k[RM7], D4, k[R11] * D3)), fma(2.0, S3, -S4), T3);
        e4 = weno_e_chain(fma(k[R11], D6, fma(k[RM31], D5, k[R26] * D4)),
                          fma(-2.0, S5, 3.0 * S4), T4);
    }
    e4 = pos_max(pos_max(pos_max(e0, e1), pos_max(e2, e3)), e4);   // SYMBO
    // leave-one-out products from prefix / suffix partial products
    const double p01 = e0 * e1, p34 = e3 * e4;
    const double p012 = p01 * e2, p234 = e2 * p34;
    const double P0 = e1 * p234, P1 = e0 * p234, P2 = p01 * p34, P3 = p012 * e4, P4 = p012 * e3;
    const double l0 = fma(k[L0A], D2, fma(k[L0B], D1, k[L0C] * D0));
    const double l1 = fma(k[L1A], D3, fma(k[L1B], D2, k[L1C] * D1));
    const double l2 = fma(k[L2A], D4, fma(k[L2B], D3, k[L2C] * D2));
    const double l3 = fma(k[L3A], D5, fma(k[L3B], D4, k[L3C] * D3));
    const double l4 = fma(k[L4A], D6, fma(k[L4B], D5, fma(k[L4C], D4, k[L4D] * D3)));
    num = fma(P4, l4, fma(P3, l3, fma(P2, l2, fma(P1, l1, P0 * l0))));
    den = fma(k[Q4], P4, fma(k[Q3], P3, fma(k[Q2], P2, fma(k[Q1], P1, k[Q0] * P0))));
}

// ---------------------------------------------------------------------------
// CLOSURE face mode: the boundary closures of the reference's ring kernel
// (split_Jac3d_Stager_Warming_ker_boundary, OCFD_NS_Jacobian3d.cpp:1063-1085
// for x, :1515-1584 for y).  WENO5 family on a 5-point stencil s[0..4]
// (OCFD_bound_Scheme.cpp:560-719; three-candidate forms OCFD_Schemes.cpp:
// 1110-1140 and :1170-1200, whose P form takes a0 and a1 from S1 and S2
// before they are accumulated -- kept), eps = 1e-6, no linear weights.
// These run only on the faces next to a CLOSURE face, in FP64.
// ---------------------------------------------------------------------------
namespace w5 {
constexpr double E12 = 12.0 * 1e-6;
__device__ __forceinline__ double s_lo(const double* s) {   // candidate on s[2..4]
    const double t0 = s[2] - 2.0 * s[3] + s[4], t1 = 3.0 * s[2] - 4.0 * s[3] + s[4];
    return 13 * t0 * t0 + 3 * t1 * t1;
}
__device__ __forceinline__ double s_mid(const double* s) {  // candidate on s[1..3]
    const double t0 = s[1] - 2.0 * s[2] + s[3], t1 = s[1] - s[3];
    return 13 * t0 * t0 + 3 * t1 * t1;
}
__device__ __forceinline__ double s_hi(const double* s) {   // candidate on s[0..2]
    const double t0 = s[0] - 2.0 * s[1] + s[2], t1 = s[0] - 4.0 * s[1] + 3.0 * s[2];
    return 13 * t0 * t0 + 3 * t1 * t1;
}
__device__ __forceinline__ double s_lo_m(const double* s) { // mirror of s_hi on s[2..4]
    const double t0 = s[4] - 2.0 * s[3] + s[2], t1 = s[4] - 4.0 * s[3] + 3.0 * s[2];
    return 13 * t0 * t0 + 3 * t1 * t1;
}
__device__ __forceinline__ double s_hi_m(const double* s) { // mirror of s_lo on s[0..2]
    const double t0 = s[2] - 2.0 * s[1] + s[0], t1 = 3.0 * s[2] - 4.0 * s[1] + s[0];
    return 13 * t0 * t0 + 3 * t1 * t1;
}
__device__ __forceinline__ double w(double S) { return 1.0 / ((E12 + S) * (E12 + S)); }
__device__ __forceinline__ double sq(double S) { return (E12 + S) * (E12 + S); }
// candidate values (times 6)
__device__ __forceinline__ double q_lo(const double* s) { return 2.0 * s[2] + 5.0 * s[3] - s[4]; }
__device__ __forceinline__ double q_mid(const double* s) { return -s[1] + 5.0 * s[2] + 2.0 * s[3]; }
__device__ __forceinline__ double q_hi(const double* s) { return 2.0 * s[0] - 7.0 * s[1] + 11.0 * s[2]; }
__device__ __forceinline__ double qm_lo(const double* s) { return 2.0 * s[4] - 7.0 * s[3] + 11.0 * s[2]; }
__device__ __forceinline__ double qm_mid(const double* s) { return -s[3] + 5.0 * s[2] + 2.0 * s[1]; }
__device__ __forceinline__ double qm_hi(const double* s) { return 2.0 * s[2] + 5.0 * s[1] - s[0]; }

__device__ __forceinline__ double p_lift(const double* s) {
    const double a0 = w(s_lo(s));
    return a0 * q_lo(s) / (6.0 * a0);
}
__device__ __forceinline__ double p_lift_plus(const double* s) {
    const double a0 = w(s_lo(s)), a1 = w(s_mid(s));
    return (a0 * q_lo(s) + a1 * q_mid(s)) / (6.0 * (a0 + a1));
}
__device__ __forceinline__ double p_right_plus(const double* s) {
    const double a1 = w(s_mid(s)), a2 = w(s_hi(s));
    return (a1 * q_mid(s) + a2 * q_hi(s)) / (6.0 * (a1 + a2));
}
__device__ __forceinline__ double p3(const double* s) {
    const double S0 = s_lo(s), S1 = s_mid(s);
    const double a0 = sq(0.0) * sq(0.0);     // from S1, S2 before they are accumulated
    const double a1 = sq(S0) * sq(0.0);
    const double a2 = sq(S0) * sq(S1);
    return (a0 * q_lo(s) + a1 * q_mid(s) + a2 * q_hi(s)) / (6.0 * (a0 + a1 + a2));
}
__device__ __forceinline__ double m_lift(const double* s) {
    const double a2 = w(s_lo_m(s));
    return a2 * qm_lo(s) / (6.0 * a2);
}
__device__ __forceinline__ double m_lift_plus(const double* s) {
    const double a1 = w(s_mid(s)), a2 = w(s_lo_m(s));
    return (a1 * qm_mid(s) + a2 * qm_lo(s)) / (6.0 * (a1 + a2));
}
__device__ __forceinline__ double m_right_plus(const double* s) {
    const double a0 = w(s_hi_m(s)), a1 = w(s_mid(s));
    return (a0 * qm_hi(s) + a1 * qm_mid(s)) / (6.0 * (a0 + a1));
}
__device__ __forceinline__ double m3(const double* s) {
    const double a0 = w(s_hi_m(s)), a1 = w(s_mid(s)), a2 = w(s_lo_m(s));
    return (a0 * qm_hi(s) + a1 * qm_mid(s) + a2 * qm_lo(s)) / (6.0 * (a0 + a1 + a2));
}
// OCFD_Schemes.cpp:822-835
__device__ __forceinline__ double minmod2(double x1, double x2) {
    const double s1 = x1 >= 0 ? 1.0 : -1.0, s2 = x2 >= 0 ? 1.0 : -1.0;
    return 0.5 * (s1 + s2) * fmin(fabs(x1), fabs(x2));
}
}  // namespace w5

// ---------------------------------------------------------------------------
// Mixed form: the P and M reconstructions of one face are the same arithmetic
// on two stencils, so they run as the two lanes of Blackwell's packed FP32x2
// instructions (FFMA2/FADD2/FMUL2): t[k] = (P stencil k, M stencil k).  Same
// rescaled indicators; the normalised weights d_k/e_k take their reciprocals
// in pairs, 1/a = b/(ab) and 1/b = a/(ab), from the approximate hardware
// reciprocal (ab stays inside the FP32 range for any indicator below ~1e17);
// d_k is folded into the l_k coefficients.
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
// eps' + the Cholesky form of factor set F (wk::E0 .. wk::E4) on (v0, v1, v2),
// both lanes
template <int F>
__device__ __forceinline__ float2 weno_e2(float2 v0, float2 v1, float2 v2) {
    constexpr float u0 = (float)wk::UF[F], u1 = (float)wk::UF[F + 1], u2 = (float)wk::UF[F + 2];
    constexpr float u3 = (float)wk::UF[F + 3], u4 = (float)wk::UF[F + 4];
    constexpr float u5 = (float)wk::UF[F + 5];
    const float2 y0 = fma2(f2(u2), v2, fma2(f2(u1), v1, mul2(f2(u0), v0)));
    const float2 y1 = fma2(f2(u4), v2, mul2(f2(u3), v1));
    const float2 y2 = mul2(f2(u5), v2);
    return fma2(y0, y0, fma2(y1, y1, fma2(y2, y2, f2((float)wk::EPS))));
}

// face value of lane L = t[3].L + num.L / den.L
__device__ __forceinline__ void weno7_symbo_pm_f32x2(const float2 t[8], float2& num,
                                                     float2& den) {
    const float2 D0 = sub2(t[1], t[0]), D1 = sub2(t[2], t[1]), D2 = sub2(t[3], t[2]);
    const float2 D3 = sub2(t[4], t[3]), D4 = sub2(t[5], t[4]), D5 = sub2(t[6], t[5]);
    const float2 D6 = sub2(t[7], t[6]);
    const float2 e0 = weno_e2<wk::E0>(D2, D0, D1), e1 = weno_e2<wk::E1>(D3, D1, D2);
    const float2 e2 = weno_e2<wk::E2>(D2, D4, D3), e3 = weno_e2<wk::E3>(D3, D4, D5);
    float2 e4 = weno_e2<wk::E4>(D4, D5, D6);
    e4.x = fmaxf(fmaxf(fmaxf(e0.x, e1.x), fmaxf(e2.x, e3.x)), e4.x);
    e4.y = fmaxf(fmaxf(fmaxf(e0.y, e1.y), fmaxf(e2.y, e3.y)), e4.y);
    const float2 r01 = rcp2(mul2(e0, e1)), r23 = rcp2(mul2(e2, e3)), r4 = rcp2(e4);
    const float2 i0 = mul2(e1, r01), i1 = mul2(e0, r01), i2 = mul2(e3, r23), i3 = mul2(e2, r23);
    constexpr float d0 = (float)wk::D0, d1 = (float)wk::D1, d2 = (float)wk::D2,
                    d3 = (float)wk::D3, d4 = (float)wk::D4;
    const float2 l0 = fma2(f2(13 * d0), D2, fma2(f2(-10 * d0), D1, mul2(f2(3 * d0), D0)));
    const float2 l1 = fma2(f2(3 * d1), D3, fma2(f2(4 * d1), D2, mul2(f2(-d1), D1)));
    const float2 l2 = fma2(f2(-d2), D4, fma2(f2(6 * d2), D3, mul2(f2(d2), D2)));
    const float2 l3 = fma2(f2(d3), D5, fma2(f2(-4 * d3), D4, mul2(f2(9 * d3), D3)));
    const float2 l4 =
        fma2(f2(-3 * d4), D6, fma2(f2(10 * d4), D5, fma2(f2(-13 * d4), D4, mul2(f2(12 * d4), D3))));
    num = fma2(r4, l4, fma2(i3, l3, fma2(i2, l2, fma2(i1, l1, mul2(i0, l0)))));
    den = fma2(f2(12 * d4), r4, fma2(f2(12 * d3), i3,
               fma2(f2(12 * d2), i2, fma2(f2(12 * d1), i1, mul2(f2(12 * d0), i0)))));
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

// ---------------------------------------------------------------------------
// TMA tile loads (cp.async.bulk.tensor, no multicast) completing on an
// mbarrier in shared memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}
// one arrival that also announces `bytes` of transactions to come
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// wait for the phase of parity `parity` to complete; false when it has not
// after a bounded number of polls (each poll may suspend for a while)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  int polls = 1 << 22) {
    for (int i = 0; i < polls; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// 3D tile of `map` at element coordinates (x, y, z) into shared memory; x
// times the element size must be a multiple of 16 bytes
__device__ __forceinline__ void tma_load_3d(void* dst, const void* map, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

}  // namespace ws
