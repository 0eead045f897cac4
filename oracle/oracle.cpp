// oracle.cpp -- CPU restatement of WindStencil's inviscid RHS (test infrastructure).
//
// This file is the checker for the CUDA product and the CPU baseline of
// bench.py; the product never links it.  Every function names the reference
// code it restates (paths relative to the WindStencil source tree).  The
// arithmetic keeps the reference's operation order so that, compiled with
// -ffp-contract=off, the scalar kernels agree bit-for-bit with the reference's
// own functions built for the host (oracle/build_ref.py).
//
// The whole-field RHS follows the reference's decomposed path, which the fused
// kernel OCFD_split.cpp:36-3918 replaces:
//   per direction: split (OCFD_NS_Jacobian3d.cpp:55-129) over the line with its
//   4 ghost points on each side, then P and M WENO7-SYMBO faces
//   (OCFD_Schemes.cpp:306-368, :491-553) and du += -J*(F(i+1/2)-F(i-1/2))/h,
//   first all P terms then all M terms (OCFD_Schemes.cpp:221-296; job shifts in
//   OCFD_Schemes_Choose.cpp:87-101 and :372-385), x then y then z.
#include "oracle.h"

#include <cmath>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ----------------------------------------------------------------------------
// Operation-counting scalar: used once, single-threaded, by or_op_counts() to
// freeze the algorithmic FLOP count of one cell-RHS.
// ----------------------------------------------------------------------------
struct OpTally { long add = 0, mul = 0, div = 0, sqrt = 0, max = 0; };
OpTally g_tally;

// A value built from the literal 0.0 (the reference's accumulator
// initialisers, `S0 = 0.0; S0 += ...`) is flagged so that adding to it is not
// counted: 0.0 + x == x here because every such x is a product >= +0 or the
// first weighted candidate, and a compiler may not drop it only because of -0.
struct Cnt {
    double v;
    bool zero_literal;
    Cnt() : v(0), zero_literal(true) {}
    Cnt(double x) : v(x), zero_literal(x == 0.0) {}
    static Cnt result(double x) { Cnt c(x); c.zero_literal = false; return c; }
};
inline Cnt operator+(Cnt a, Cnt b) {
    if (!a.zero_literal && !b.zero_literal) g_tally.add++;
    return Cnt::result(a.v + b.v);
}
inline Cnt operator-(Cnt a, Cnt b) { g_tally.add++; return Cnt::result(a.v - b.v); }
inline Cnt operator*(Cnt a, Cnt b) { g_tally.mul++; return Cnt::result(a.v * b.v); }
inline Cnt operator/(Cnt a, Cnt b) { g_tally.div++; return Cnt::result(a.v / b.v); }
inline Cnt operator-(Cnt a) { Cnt c = a; c.v = -a.v; return c; }
inline Cnt& operator+=(Cnt& a, Cnt b) { a = a + b; return a; }
inline Cnt& operator/=(Cnt& a, Cnt b) { a = a / b; return a; }
inline Cnt op_sqrt(Cnt a) { g_tally.sqrt++; return Cnt::result(std::sqrt(a.v)); }
inline Cnt op_max(Cnt a, Cnt b) { g_tally.max++; return Cnt::result(std::fmax(a.v, b.v)); }
inline double op_sqrt(double a) { return std::sqrt(a); }
inline double op_max(double a, double b) { return std::fmax(a, b); }

// ----------------------------------------------------------------------------
// WENO7-SYMBO (Martin et al., J. Comput. Phys. 220 (2006) 270-289), the "_opt"
// form the fused kernel calls: OCFD_Schemes.cpp:306-368 (P) and :491-553 (M).
// s[0..7] are the split-flux values at points i-3..i+4; the result is the face
// value at i+1/2.  The M form is the same formula on the reversed stencil
// (t[k] = s[7-k]); the reference writes it out with the same operation order,
// so the two agree bit-for-bit.
// Smoothness indicators: three derivative rounds weighted 720, 780, 781;
// beta_4 <- max(beta_0..beta_4); weights d_k * prod_{j!=k}(eps + beta_j) with
// eps = 2.592e-6 and the bandwidth-optimised linear weights d_k below.
// ----------------------------------------------------------------------------
template <typename R, typename S>
R weno7_symbo(const S& t) {
    R b0 = 0.0, b1 = 0.0, b2 = 0.0, b3 = 0.0, b4 = 0.0;
    R q;
    // first derivative round
    q = R(-2.0) * t(0) + R(9.0) * t(1) - R(18.0) * t(2) + R(11.0) * t(3);   b0 += R(720.0) * q * q;
    q = t(1) - R(6.0) * t(2) + R(3.0) * t(3) + R(2.0) * t(4);               b1 += R(720.0) * q * q;
    q = R(-2.0) * t(2) - R(3.0) * t(3) + R(6.0) * t(4) - t(5);              b2 += R(720.0) * q * q;
    q = R(-11.0) * t(3) + R(18.0) * t(4) - R(9.0) * t(5) + R(2.0) * t(6);   b3 += R(720.0) * q * q;
    q = R(-26.0) * t(4) + R(57.0) * t(5) - R(42.0) * t(6) + R(11.0) * t(7); b4 += R(720.0) * q * q;
    // second derivative round
    q = R(-6.0) * t(0) + R(24.0) * t(1) - R(30.0) * t(2) + R(12.0) * t(3);  b0 += R(780.0) * q * q;
    q = R(6.0) * t(2) - R(12.0) * t(3) + R(6.0) * t(4);                      b1 += R(780.0) * q * q;
    q = R(6.0) * t(3) - R(12.0) * t(4) + R(6.0) * t(5);                      b2 += R(780.0) * q * q;
    q = R(12.0) * t(3) - R(30.0) * t(4) + R(24.0) * t(5) - R(6.0) * t(6);   b3 += R(780.0) * q * q;
    q = R(18.0) * t(4) - R(48.0) * t(5) + R(42.0) * t(6) - R(12.0) * t(7);  b4 += R(780.0) * q * q;
    // third derivative round
    q = R(-6.0) * t(0) + R(18.0) * (t(1) - t(2)) + R(6.0) * t(3);           b0 += R(781.0) * q * q;
    q = R(-6.0) * t(1) + R(18.0) * (t(2) - t(3)) + R(6.0) * t(4);           b1 += R(781.0) * q * q;
    q = R(-6.0) * t(2) + R(18.0) * (t(3) - t(4)) + R(6.0) * t(5);           b2 += R(781.0) * q * q;
    q = R(-6.0) * t(3) + R(18.0) * (t(4) - t(5)) + R(6.0) * t(6);           b3 += R(781.0) * q * q;
    q = R(-6.0) * t(4) + R(18.0) * (t(5) - t(6)) + R(6.0) * t(7);           b4 += R(781.0) * q * q;
    // SYMBO: the downwind indicator takes the largest of the five
    b4 = op_max(op_max(op_max(b0, b1), op_max(b2, b3)), b4);
    const R e(2.592e-6);
    const R w0 = R(0.0401954833730) * (e + b1) * (e + b2) * (e + b3) * (e + b4);
    const R w1 = R(0.2493800006710) * (e + b0) * (e + b2) * (e + b3) * (e + b4);
    const R w2 = R(0.4802686256260) * (e + b0) * (e + b1) * (e + b3) * (e + b4);
    const R w3 = R(0.2009775476730) * (e + b0) * (e + b1) * (e + b2) * (e + b4);
    const R w4 = R(0.0291783426580) * (e + b0) * (e + b1) * (e + b2) * (e + b3);
    // candidate reconstructions (times 12) and the convex combination
    R acc = 0.0;
    q = R(-3.0) * t(0) + R(13.0) * t(1) - R(23.0) * t(2) + R(25.0) * t(3);  acc += w0 * q;
    q = t(1) - R(5.0) * t(2) + R(13.0) * t(3) + R(3.0) * t(4);              acc += w1 * q;
    q = -t(2) + R(7.0) * t(3) + R(7.0) * t(4) - t(5);                        acc += w2 * q;
    q = R(3.0) * t(3) + R(13.0) * t(4) - R(5.0) * t(5) + t(6);              acc += w3 * q;
    q = R(25.0) * t(4) - R(23.0) * t(5) + R(13.0) * t(6) - R(3.0) * t(7);   acc += w4 * q;
    acc /= (R(12.0) * (w0 + w1 + w2 + w3 + w4));
    return acc;
}

template <typename R>
struct Fwd { const R* s; R operator()(int k) const { return s[k]; } };
template <typename R>
struct Rev { const R* s; R operator()(int k) const { return s[7 - k]; } };

template <typename R> R weno_p(const R* s) { return weno7_symbo<R>(Fwd<R>{s}); }
template <typename R> R weno_m(const R* s) { return weno7_symbo<R>(Rev<R>{s}); }

// ----------------------------------------------------------------------------
// Steger-Warming flux-vector splitting with entropy fix, one point, one
// direction: OCFD_NS_Jacobian3d.cpp:55-129 (split_Jac3d_Stager_Warming_ker_origin).
// (a1,a2,a3) is the metric gradient of the direction; C1 = 2(g-1),
// C3 = (3-g)/(2(g-1)) (OCFD_init.cpp:385-386).
// ----------------------------------------------------------------------------
template <typename R>
void sw_split(R d, R u, R v, R w, R cc, R a1, R a2, R a3, double gamma,
              double epsl_sw, R* fp, R* fm) {
    const R g(gamma), eps(epsl_sw);
    const R c1(2.0 * (gamma - 1.0));
    const R c3((3.0 - gamma) / (2.0 * (gamma - 1.0)));
    R ss = op_sqrt(a1 * a1 + a2 * a2 + a3 * a3);
    R k1 = a1 / ss, k2 = a2 / ss, k3 = a3 / ss;
    R vs = a1 * u + a2 * v + a3 * w;
    R e1 = vs, e2 = vs - cc * ss, e3 = vs + cc * ss;
    R e1p = (e1 + op_sqrt(e1 * e1 + eps * eps)) * R(0.50);
    R e2p = (e2 + op_sqrt(e2 * e2 + eps * eps)) * R(0.50);
    R e3p = (e3 + op_sqrt(e3 * e3 + eps * eps)) * R(0.50);
    R e1m = e1 - e1p, e2m = e2 - e2p, e3m = e3 - e3p;
    R t0 = d / (R(2.0) * g);
    R uc1 = u - cc * k1, uc2 = u + cc * k1;
    R vc1 = v - cc * k2, vc2 = v + cc * k2;
    R wc1 = w - cc * k3, wc2 = w + cc * k3;
    R vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * R(0.50);
    R vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * R(0.50);
    R vv = (g - R(1.0)) * (u * u + v * v + w * w);
    R w2 = c3 * cc * cc;
    fp[0] = t0 * (c1 * e1p + e2p + e3p);
    fp[1] = t0 * (c1 * e1p * u + e2p * uc1 + e3p * uc2);
    fp[2] = t0 * (c1 * e1p * v + e2p * vc1 + e3p * vc2);
    fp[3] = t0 * (c1 * e1p * w + e2p * wc1 + e3p * wc2);
    fp[4] = t0 * (e1p * vv + e2p * vvc1 + e3p * vvc2 + w2 * (e2p + e3p));
    fm[0] = t0 * (c1 * e1m + e2m + e3m);
    fm[1] = t0 * (c1 * e1m * u + e2m * uc1 + e3m * uc2);
    fm[2] = t0 * (c1 * e1m * v + e2m * vc1 + e3m * vc2);
    fm[3] = t0 * (c1 * e1m * w + e2m * wc1 + e3m * wc2);
    fm[4] = t0 * (e1m * vv + e2m * vvc1 + e3m * vvc2 + w2 * (e2m + e3m));
}

// ----------------------------------------------------------------------------
// CLOSURE face mode: the boundary closures of the fused path's ring kernel
// (split_Jac3d_Stager_Warming_ker_boundary, OCFD_NS_Jacobian3d.cpp:828-2530),
// which that kernel applies near the x and y faces of the domain.
//
// WENO5 family (s[0..4] a 5-point stencil): the one- and two-candidate forms
// of OCFD_bound_Scheme.cpp:540-720 (eps = 1e-6, unit linear weights, weights
// 1/(12 eps + S)^2) and the three-candidate forms OCFD_Schemes.cpp:1110-1140
// (P) and :1170-1200 (M).  The P form builds its weights a0 and a1 from S1
// and S2 before they are accumulated (so from zero); that is reproduced.
// Operation order as in the reference.
// ----------------------------------------------------------------------------
constexpr double kEp5 = 1e-6;

double w5_p_lift(const double* s) {            // OCFD_bound_Scheme.cpp:560-576
    double S0 = 0.0, t;
    t = s[2] - 2.0 * s[3] + s[4];       S0 += 13 * t * t;
    t = 3.0 * s[2] - 4.0 * s[3] + s[4]; S0 += 3 * t * t;
    const double a0 = 1.0 / ((12.0 * kEp5 + S0) * (12.0 * kEp5 + S0));
    const double q03 = (2.0 * s[2] + 5.0 * s[3] - s[4]);
    return a0 * q03 / (6.0 * a0);
}
double w5_m_lift(const double* s) {            // OCFD_bound_Scheme.cpp:598-615
    double S2 = 0.0, t;
    t = s[4] - 2.0 * s[3] + s[2];       S2 += 13 * t * t;
    t = s[4] - 4.0 * s[3] + 3.0 * s[2]; S2 += 3 * t * t;
    const double a2 = 1.0 / ((12.0 * kEp5 + S2) * (12.0 * kEp5 + S2));
    const double q23 = (2.0 * s[4] - 7.0 * s[3] + 11.0 * s[2]);
    return a2 * q23 / (6.0 * a2);
}
double w5_p_right_plus(const double* s) {      // OCFD_bound_Scheme.cpp:617-641
    double S1 = 0.0, S2 = 0.0, t;
    t = s[1] - 2.0 * s[2] + s[3]; S1 += 13 * t * t;
    t = s[1] - s[3];              S1 += 3 * t * t;
    const double a1 = 1.0 / ((12.0 * kEp5 + S1) * (12.0 * kEp5 + S1));
    const double q13 = (-s[1] + 5.0 * s[2] + 2.0 * s[3]);
    t = s[0] - 2.0 * s[1] + s[2];       S2 += 13 * t * t;
    t = s[0] - 4.0 * s[1] + 3.0 * s[2]; S2 += 3 * t * t;
    const double a2 = 1.0 / ((12.0 * kEp5 + S2) * (12.0 * kEp5 + S2));
    const double q23 = (2.0 * s[0] - 7.0 * s[1] + 11.0 * s[2]);
    return (a1 * q13 + a2 * q23) / (6.0 * (a1 + a2));
}
double w5_p_lift_plus(const double* s) {       // OCFD_bound_Scheme.cpp:643-667
    double S0 = 0.0, S1 = 0.0, t;
    t = s[2] - 2.0 * s[3] + s[4];       S0 += 13 * t * t;
    t = 3.0 * s[2] - 4.0 * s[3] + s[4]; S0 += 3 * t * t;
    const double a0 = 1.0 / ((12.0 * kEp5 + S0) * (12.0 * kEp5 + S0));
    const double q03 = (2.0 * s[2] + 5.0 * s[3] - s[4]);
    t = s[1] - 2.0 * s[2] + s[3]; S1 += 13 * t * t;
    t = s[1] - s[3];              S1 += 3 * t * t;
    const double a1 = 1.0 / ((12.0 * kEp5 + S1) * (12.0 * kEp5 + S1));
    const double q13 = (-s[1] + 5.0 * s[2] + 2.0 * s[3]);
    return (a0 * q03 + a1 * q13) / (6.0 * (a0 + a1));
}
double w5_m_right_plus(const double* s) {      // OCFD_bound_Scheme.cpp:669-693
    double S0 = 0.0, S1 = 0.0, t;
    t = s[2] - 2.0 * s[1] + s[0];       S0 += 13 * t * t;
    t = 3.0 * s[2] - 4.0 * s[1] + s[0]; S0 += 3 * t * t;
    const double a0 = 1.0 / ((12.0 * kEp5 + S0) * (12.0 * kEp5 + S0));
    const double q03 = (2.0 * s[2] + 5.0 * s[1] - s[0]);
    t = s[3] - 2.0 * s[2] + s[1]; S1 += 13 * t * t;
    t = s[3] - s[1];              S1 += 3 * t * t;
    const double a1 = 1.0 / ((12.0 * kEp5 + S1) * (12.0 * kEp5 + S1));
    const double q13 = (-s[3] + 5.0 * s[2] + 2.0 * s[1]);
    return (a0 * q03 + a1 * q13) / (6.0 * (a0 + a1));
}
double w5_m_lift_plus(const double* s) {       // OCFD_bound_Scheme.cpp:695-719
    double S1 = 0.0, S2 = 0.0, t;
    t = s[3] - 2.0 * s[2] + s[1]; S1 += 13 * t * t;
    t = s[3] - s[1];              S1 += 3 * t * t;
    const double a1 = 1.0 / ((12.0 * kEp5 + S1) * (12.0 * kEp5 + S1));
    const double q13 = (-s[3] + 5.0 * s[2] + 2.0 * s[1]);
    t = s[4] - 2.0 * s[3] + s[2];       S2 += 13 * t * t;
    t = s[4] - 4.0 * s[3] + 3.0 * s[2]; S2 += 3 * t * t;
    const double a2 = 1.0 / ((12.0 * kEp5 + S2) * (12.0 * kEp5 + S2));
    const double q23 = (2.0 * s[4] - 7.0 * s[3] + 11.0 * s[2]);
    return (a1 * q13 + a2 * q23) / (6.0 * (a1 + a2));
}
double w5_p(const double* s) {                 // OCFD_Schemes.cpp:1110-1140
    double S0 = 0.0, S1 = 0.0, S2 = 0.0, t;
    t = s[2] - 2.0 * s[3] + s[4];       S0 += 13 * t * t;
    t = 3.0 * s[2] - 4.0 * s[3] + s[4]; S0 += 3 * t * t;
    // a0 from S1, S2 while they are still 0.0 (the reference's order)
    const double a0 = ((12.0 * kEp5 + S1) * (12.0 * kEp5 + S1)) *
                      ((12.0 * kEp5 + S2) * (12.0 * kEp5 + S2));
    const double q03 = (2.0 * s[2] + 5.0 * s[3] - s[4]);
    t = s[1] - 2.0 * s[2] + s[3]; S1 += 13 * t * t;
    t = s[1] - s[3];              S1 += 3 * t * t;
    const double a1 = ((12.0 * kEp5 + S0) * (12.0 * kEp5 + S0)) *
                      ((12.0 * kEp5 + S2) * (12.0 * kEp5 + S2));
    const double q13 = (-s[1] + 5.0 * s[2] + 2.0 * s[3]);
    t = s[0] - 2.0 * s[1] + s[2];       S2 += 13 * t * t;
    t = s[0] - 4.0 * s[1] + 3.0 * s[2]; S2 += 3 * t * t;
    const double a2 = ((12.0 * kEp5 + S0) * (12.0 * kEp5 + S0)) *
                      ((12.0 * kEp5 + S1) * (12.0 * kEp5 + S1));
    const double q23 = (2.0 * s[0] - 7.0 * s[1] + 11.0 * s[2]);
    return (a0 * q03 + a1 * q13 + a2 * q23) / (6.0 * (a0 + a1 + a2));
}
double w5_m(const double* s) {                 // OCFD_Schemes.cpp:1170-1200
    double S0 = 0.0, S1 = 0.0, S2 = 0.0, t;
    t = s[2] - 2.0 * s[1] + s[0];       S0 += 13 * t * t;
    t = 3.0 * s[2] - 4.0 * s[1] + s[0]; S0 += 3 * t * t;
    const double a0 = 1.0 / ((12.0 * kEp5 + S0) * (12.0 * kEp5 + S0));
    const double q03 = (2.0 * s[2] + 5.0 * s[1] - s[0]);
    t = s[3] - 2.0 * s[2] + s[1]; S1 += 13 * t * t;
    t = s[3] - s[1];              S1 += 3 * t * t;
    const double a1 = 1.0 / ((12.0 * kEp5 + S1) * (12.0 * kEp5 + S1));
    const double q13 = (-s[3] + 5.0 * s[2] + 2.0 * s[1]);
    t = s[4] - 2.0 * s[3] + s[2];       S2 += 13 * t * t;
    t = s[4] - 4.0 * s[3] + 3.0 * s[2]; S2 += 3 * t * t;
    const double a2 = 1.0 / ((12.0 * kEp5 + S2) * (12.0 * kEp5 + S2));
    const double q23 = (2.0 * s[4] - 7.0 * s[3] + 11.0 * s[2]);
    return (a0 * q03 + a1 * q13 + a2 * q23) / (6.0 * (a0 + a1 + a2));
}
// OCFD_Schemes.cpp:822-835
double sign_of(double x1, double x2) { return x2 >= 0 ? std::fabs(x1) : -std::fabs(x1); }
double minmod2(double x1, double x2) {
    return 0.5 * (sign_of(1.0, x1) + sign_of(1.0, x2)) * std::fmin(std::fabs(x1), std::fabs(x2));
}

// Closure value of face f (between cells f-1 and f, f = 0..n) of a line of n
// cells in the x (dir 0) or y (dir 1) direction; F[c] is the split flux of
// cell c (F[-4..n+3] valid), pm 0 for F+ (P faces), 1 for F- (M faces).  lo /
// hi: the low / high face of the direction is a CLOSURE face.  Returns false
// when face f keeps its WENO7-SYMBO value.  The per-face rules restate the
// ring kernel's x rules (OCFD_NS_Jacobian3d.cpp:1063-1069 P, :1079-1085 M) and
// y rules (:1515-1584), read as one value per face: every face value is the
// same from both cells that share it.  x and y differ at the high end: x
// extrapolates linearly and averages, y uses minmod2 forms and a copy.
bool closure_face(int pm, int dir, long f, long n, bool lo, bool hi, const double* F,
                  double* out) {
    if (pm == 0) {
        if (lo && f == 0) { *out = F[0]; return true; }
        if (lo && f == 1) { *out = w5_p_lift(F + f - 3); return true; }
        if (lo && f == 2) { *out = w5_p_lift_plus(F + f - 3); return true; }
        if ((lo && f == 3) || (hi && f == n - 2)) { *out = w5_p(F + f - 3); return true; }
        if (hi && f == n - 1) { *out = w5_p_right_plus(F + f - 3); return true; }
        if (hi && f == n) {
            *out = dir == 0 ? 1.5 * F[n - 1] - 0.5 * F[n - 2]
                            : F[n - 1] + 0.5 * minmod2(F[n - 1] - F[n - 2], F[n - 1] - F[n - 2]);
            return true;
        }
        return false;
    }
    if (lo && f == 0) { *out = w5_m_lift(F + f - 2); return true; }
    if (lo && f == 1) { *out = w5_m_lift_plus(F + f - 2); return true; }
    if ((lo && (f == 2 || f == 3)) || (hi && f == n - 3)) { *out = w5_m(F + f - 2); return true; }
    if (hi && f == n - 2) { *out = w5_m_right_plus(F + f - 2); return true; }
    if (hi && f == n - 1) {
        *out = dir == 0 ? 0.5 * F[n - 1] + 0.5 * F[n - 2]
                        : F[n - 1] - 0.5 * minmod2(F[n - 1] - F[n - 2], F[n - 1] - F[n - 2]);
        return true;
    }
    if (hi && f == n) {
        *out = dir == 0 ? 0.5 * F[n - 1] + 0.5 * F[n - 2] : F[n - 1];
        return true;
    }
    return false;
}

// ----------------------------------------------------------------------------
// Indexing helpers (reference: cuda_utility.h:16-27).
// ----------------------------------------------------------------------------
struct Dims {
    long nx, ny, nz, px, py, pz;     // interior and padded extents
    explicit Dims(const or_grid* g)
        : nx(g->nx), ny(g->ny), nz(g->nz),
          px(g->nx + 2 * OR_LAP), py(g->ny + 2 * OR_LAP), pz(g->nz + 2 * OR_LAP) {}
    // LAP-field index of interior coordinate (i,j,k), i in [-4, nx+4)
    long lap(long i, long j, long k) const {
        return (i + OR_LAP) + px * ((j + OR_LAP) + py * (k + OR_LAP));
    }
    long soa(long i, long j, long k, long var) const {
        return i + nx * (j + ny * (k + nz * var));
    }
    long lap_size() const { return px * py * pz; }
    long cells() const { return nx * ny * nz; }
};

}  // namespace

// ============================================================================
extern "C" {

double or_weno7_p(const double* s8) { return weno_p<double>(s8); }
double or_weno7_m(const double* s8) { return weno_m<double>(s8); }

void or_weno7_p_batch(const double* s, long n, double* out) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) out[i] = weno_p<double>(s + 8 * i);
}
void or_weno7_m_batch(const double* s, long n, double* out) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) out[i] = weno_m<double>(s + 8 * i);
}

// WENO5 closure family over n 5-point stencils; which: 0 P_lift, 1 P_lift_plus,
// 2 P, 3 P_right_plus, 4 M_lift, 5 M_lift_plus, 6 M, 7 M_right_plus, 8 minmod2
// of (s[0], s[1])
void or_weno5_batch(int which, const double* s, long n, double* out) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        const double* p = s + 5 * i;
        switch (which) {
            case 0: out[i] = w5_p_lift(p); break;
            case 1: out[i] = w5_p_lift_plus(p); break;
            case 2: out[i] = w5_p(p); break;
            case 3: out[i] = w5_p_right_plus(p); break;
            case 4: out[i] = w5_m_lift(p); break;
            case 5: out[i] = w5_m_lift_plus(p); break;
            case 6: out[i] = w5_m(p); break;
            case 7: out[i] = w5_m_right_plus(p); break;
            default: out[i] = minmod2(p[0], p[1]); break;
        }
    }
}

void or_split(double d, double u, double v, double w, double cc, double a1,
              double a2, double a3, double gamma, double epsl_sw, double* fp,
              double* fm) {
    sw_split<double>(d, u, v, w, cc, a1, a2, a3, gamma, epsl_sw, fp, fm);
}

void or_split_batch(const double* in, long n, double gamma, double epsl_sw,
                    double* fp, double* fm) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
        const double* p = in + 8 * i;
        sw_split<double>(p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], gamma,
                         epsl_sw, fp + 5 * i, fm + 5 * i);
    }
}

// Ghost-layer fill of one LAP field.  Replaces the reference's host-staged
// periodic self-exchange (OCFD_mpi_dev.cpp:123-290) with an in-place copy;
// OR_FACE_EXTRAP copies the nearest interior value (zero gradient).  Axes are
// filled x, then y, then z over the full padded extent of the other axes,
// so edge and corner ghosts are defined (the RHS never reads them).  An
// OR_FACE_EXTERNAL face keeps its ghost planes (a neighbouring subdomain's
// halo, unpacked by the caller as exchange_boundary_{x,y,z}_packed_dev do,
// OCFD_mpi_dev.cpp:185-290); the later axes' passes copy them into the edges.
void or_ghost_fill(const or_grid* g, double* f) {
    Dims D(g);
    const long L = OR_LAP;
    bool ext[6];
    for (int i = 0; i < 6; ++i) ext[i] = g->face_kind[i] == OR_FACE_EXTERNAL;
    // x
#pragma omp parallel for collapse(2) schedule(static)
    for (long k = -L; k < D.nz + L; ++k)
        for (long j = -L; j < D.ny + L; ++j)
            for (long l = 1; l <= L; ++l) {
                long lo = g->face_kind[0] == OR_FACE_PERIODIC ? D.nx - l : 0;
                long hi = g->face_kind[1] == OR_FACE_PERIODIC ? l - 1 : D.nx - 1;
                if (!ext[0]) f[D.lap(-l, j, k)] = f[D.lap(lo, j, k)];
                if (!ext[1]) f[D.lap(D.nx - 1 + l, j, k)] = f[D.lap(hi, j, k)];
            }
    // y
#pragma omp parallel for collapse(2) schedule(static)
    for (long k = -L; k < D.nz + L; ++k)
        for (long l = 1; l <= L; ++l)
            for (long i = -L; i < D.nx + L; ++i) {
                long lo = g->face_kind[2] == OR_FACE_PERIODIC ? D.ny - l : 0;
                long hi = g->face_kind[3] == OR_FACE_PERIODIC ? l - 1 : D.ny - 1;
                if (!ext[2]) f[D.lap(i, -l, k)] = f[D.lap(i, lo, k)];
                if (!ext[3]) f[D.lap(i, D.ny - 1 + l, k)] = f[D.lap(i, hi, k)];
            }
    // z
#pragma omp parallel for collapse(2) schedule(static)
    for (long l = 1; l <= L; ++l)
        for (long j = -L; j < D.ny + L; ++j)
            for (long i = -L; i < D.nx + L; ++i) {
                long lo = g->face_kind[4] == OR_FACE_PERIODIC ? D.nz - l : 0;
                long hi = g->face_kind[5] == OR_FACE_PERIODIC ? l - 1 : D.nz - 1;
                if (!ext[4]) f[D.lap(i, j, -l)] = f[D.lap(i, j, lo)];
                if (!ext[5]) f[D.lap(i, j, D.nz - 1 + l)] = f[D.lap(i, j, hi)];
            }
}

// cc = sqrt(T)/Ama on the whole padded field (commen_kernel.cpp:145-154,
// launched over the LAP-extended job by OCFD_NS_Jacobian3d.cpp:24-33).
void or_sound_speed(const or_grid* g, const double* T, double* cc) {
    Dims D(g);
    const long n = D.lap_size();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) cc[i] = std::sqrt(T[i]) / g->ama;
}

// ----------------------------------------------------------------------------
// Viscous terms: du_vis_Jacobian3d (OCFD_Stream.cpp:229-345).
//   1. first derivatives of u, v, w, T along the three computational
//      directions on the interior: central CD6 / CD8 through the ghosts
//      (OCFD_Schemes.cpp:97-104, :134-142; value / h, put_d0_kernel :74-95);
//   2. Sutherland viscosity (get_Amu_kernal, commen_kernel.cpp:123-132);
//   3. per direction: the viscous flux Ev1..4 on the interior
//      (vis_flux_ker, OCFD_NS_Jacobian3d.cpp:477-624), its ghosts filled by
//      the face kinds, its derivative along that direction, and
//      du[1..4] += J * derivative (YF_Pe_XF, commen_kernel.cpp:159-170).
// Constants as OCFD_init.cpp:380-396: Cp = 1/((g-1) Ama^2), Tsb = 110.4/Ref_T,
// amu_C0 = 1/Re*(1 + 110.4/Ref_T), heat-flux factor Cp/Pr.
// ----------------------------------------------------------------------------
namespace {
double cd6(const double* s) {
    return (45.0 * (s[4] - s[2]) - 9.0 * (s[5] - s[1]) + (s[6] - s[0])) / 60.0;
}
double cd8(const double* s) {
    return (672.0 * (s[5] - s[3]) - 168.0 * (s[6] - s[2]) + 32.0 * (s[7] - s[1]) -
            3.0 * (s[8] - s[0])) / 840.0;
}
// The reduced forms of the derivative next to a face whose DIF_BOUND flag is
// set (OCFD_D0bound_scheme_kernel, OCFD_bound_Scheme.cpp:82-240): at distance
// e = 0..3 from the face, a one-sided first difference, then 2nd-, 4th- and
// 6th-order central differences; c points at the stencil's centre.  Returns
// false where the central scheme applies.  The low face is tested first, as
// the reference does.
bool d0_bound_form(const double* c, long pos, long n, bool lo, bool hi, double* tmp) {
    long e;
    bool low;
    if (lo && pos < 4) {
        e = pos;
        low = true;
    } else if (hi && pos >= n - 4) {
        e = n - 1 - pos;
        low = false;
    } else {
        return false;
    }
    if (e == 0) *tmp = low ? (c[1] - c[0]) : (c[0] - c[-1]);
    else if (e == 1) *tmp = (c[1] - c[-1]) * 0.5;
    else if (e == 2) *tmp = (c[-2] - 8.0 * c[-1] + 8.0 * c[1] - c[2]) / 12.0;
    else *tmp = (c[3] - c[-3] - 9.0 * (c[2] - c[-2]) + 45.0 * (c[1] - c[-1])) / 60.0;
    return true;
}

// derivative along dir of LAP field f on the interior (dense out); d0b: the
// DIF_BOUND flags of the six faces (NULL: none), ignored on EXTERNAL faces
void d0_field(const or_grid* g, int scheme, int dir, const double* f, double* out,
              const int* d0b = nullptr) {
    Dims D(g);
    const long r = scheme == 6 ? 3 : 4;
    const double h = dir == 0 ? g->hx : dir == 1 ? g->hy : g->hz;
    const bool lo = d0b && d0b[2 * dir] && g->face_kind[2 * dir] != OR_FACE_EXTERNAL;
    const bool hi = d0b && d0b[2 * dir + 1] && g->face_kind[2 * dir + 1] != OR_FACE_EXTERNAL;
    const long n = dir == 0 ? D.nx : dir == 1 ? D.ny : D.nz;
#pragma omp parallel for collapse(2) schedule(static)
    for (long k = 0; k < D.nz; ++k)
        for (long j = 0; j < D.ny; ++j)
            for (long i = 0; i < D.nx; ++i) {
                double st[9];
                for (long q = -r; q <= r; ++q)
                    st[q + r] = f[dir == 0 ? D.lap(i + q, j, k)
                                           : dir == 1 ? D.lap(i, j + q, k) : D.lap(i, j, k + q)];
                double tmp;
                const long pos = dir == 0 ? i : dir == 1 ? j : k;
                if (!d0_bound_form(st + r, pos, n, lo, hi, &tmp))
                    tmp = scheme == 6 ? cd6(st) : cd8(st);
                out[i + D.nx * (j + D.ny * k)] = tmp / h;
            }
}
}  // namespace

void or_amu(const or_grid* g, const or_vis* vis, const double* T, double* amu) {
    Dims D(g);
    const double Tsb = 110.4 / vis->ref_t;
    const double amu_C0 = 1.0 / vis->re * (1.0 + 110.4 / vis->ref_t);
#pragma omp parallel for collapse(2) schedule(static)
    for (long k = 0; k < D.nz; ++k)
        for (long j = 0; j < D.ny; ++j)
            for (long i = 0; i < D.nx; ++i) {
                const double tmp = T[D.lap(i, j, k)];
                amu[i + D.nx * (j + D.ny * k)] = amu_C0 * std::sqrt(tmp * tmp * tmp) / (Tsb + tmp);
            }
}

// The viscous fluxes of all three directions (vis_flux_ker,
// OCFD_NS_Jacobian3d.cpp:477-624, per direction) into 12 LAP fields, direction
// dir component q at ev[(4 * dir + q) * lap_size]; interiors written, ghosts
// left as they are.
void or_vis_fluxes(const or_grid* g, const or_vis* vis, const double* u, const double* v,
                   const double* w, const double* T, const double* const* metrics,
                   const double* ajac, double* ev) {
    Dims D(g);
    const long N = D.cells();
    const double Cp = 1.0 / ((g->gamma - 1.0) * g->ama * g->ama);
    const double vfc = Cp / vis->pr;
    // grad[4*dir + q]: derivative along dir of (u, v, w, T)[q]
    std::vector<double> grad(12 * N), amu(N);
    const double* prim[4] = {u, v, w, T};
    for (int dir = 0; dir < 3; ++dir)
        for (int q = 0; q < 4; ++q)
            d0_field(g, vis->scheme, dir, prim[q], grad.data() + (4 * dir + q) * N,
                     vis->d0_bound);
    or_amu(g, vis, T, amu.data());
    auto met = [&](int m, long p) {       // akx..asz, Cartesian when metrics == NULL
        return metrics ? metrics[m][p] : (m == 0 || m == 4 || m == 8 ? 1.0 : 0.0);
    };
    for (int dir = 0; dir < 3; ++dir) {
        double* Ev = ev + 4 * dir * D.lap_size();
#pragma omp parallel for collapse(2) schedule(static)
        for (long k = 0; k < D.nz; ++k)
            for (long j = 0; j < D.ny; ++j)
                for (long i = 0; i < D.nx; ++i) {
                    const long c = i + D.nx * (j + D.ny * k), p = D.lap(i, j, k);
                    auto G = [&](int d, int q) { return grad[(4 * d + q) * N + c]; };
                    const double Akx = met(0, p), Aky = met(1, p), Akz = met(2, p);
                    const double Aix = met(3, p), Aiy = met(4, p), Aiz = met(5, p);
                    const double Asx = met(6, p), Asy = met(7, p), Asz = met(8, p);
                    const double ux = G(0, 0) * Akx + G(1, 0) * Aix + G(2, 0) * Asx;
                    const double vx = G(0, 1) * Akx + G(1, 1) * Aix + G(2, 1) * Asx;
                    const double wx = G(0, 2) * Akx + G(1, 2) * Aix + G(2, 2) * Asx;
                    const double uy = G(0, 0) * Aky + G(1, 0) * Aiy + G(2, 0) * Asy;
                    const double vy = G(0, 1) * Aky + G(1, 1) * Aiy + G(2, 1) * Asy;
                    const double wy = G(0, 2) * Aky + G(1, 2) * Aiy + G(2, 2) * Asy;
                    const double uz = G(0, 0) * Akz + G(1, 0) * Aiz + G(2, 0) * Asz;
                    const double vz = G(0, 1) * Akz + G(1, 1) * Aiz + G(2, 1) * Asz;
                    const double wz = G(0, 2) * Akz + G(1, 2) * Aiz + G(2, 2) * Asz;
                    const double div = ux + vy + wz;
                    const double Amu1 = amu[c];
                    const double s11 = (2.0 * ux - 2.0 / 3.0 * div) * Amu1;
                    const double s22 = (2.0 * vy - 2.0 / 3.0 * div) * Amu1;
                    const double s33 = (2.0 * wz - 2.0 / 3.0 * div) * Amu1;
                    const double s12 = (uy + vx) * Amu1;
                    const double s13 = (uz + wx) * Amu1;
                    const double s23 = (vz + wy) * Amu1;
                    const double Amuk = amu[c] * vfc;
                    const double Tx = G(0, 3) * Akx + G(1, 3) * Aix + G(2, 3) * Asx;
                    const double Ty = G(0, 3) * Aky + G(1, 3) * Aiy + G(2, 3) * Asy;
                    const double Tz = G(0, 3) * Akz + G(1, 3) * Aiz + G(2, 3) * Asz;
                    const double E1 = u[p] * s11 + v[p] * s12 + w[p] * s13 + Amuk * Tx;
                    const double E2 = u[p] * s12 + v[p] * s22 + w[p] * s23 + Amuk * Ty;
                    const double E3 = u[p] * s13 + v[p] * s23 + w[p] * s33 + Amuk * Tz;
                    const double Aj1 = ajac ? ajac[p] : 1.0;
                    const double akx = met(3 * dir, p) * Aj1;
                    const double aky = met(3 * dir + 1, p) * Aj1;
                    const double akz = met(3 * dir + 2, p) * Aj1;
                    const long L = D.lap_size();
                    Ev[p] = (akx * s11 + aky * s12 + akz * s13);
                    Ev[L + p] = (akx * s12 + aky * s22 + akz * s23);
                    Ev[2 * L + p] = (akx * s13 + aky * s23 + akz * s33);
                    Ev[3 * L + p] = (akx * E1 + aky * E2 + akz * E3);
                }
    }
}

// du[1..4] += J * d(Ev_dir)/d(dir) for one direction (the derivative and
// YF_Pe_XF accumulation of du_vis_Jacobian3d, OCFD_Stream.cpp:229-345), after
// the ghost fill of its four flux fields ev4 (4 LAP fields); an EXTERNAL face
// keeps the halo the caller put there.
void or_vis_div_add(const or_grid* g, const or_vis* vis, int dir, double* ev4,
                    const double* ajac, double* du) {
    Dims D(g);
    std::vector<double> dv(D.cells());
    for (int q = 0; q < 4; ++q) {
        double* e = ev4 + q * D.lap_size();
        or_ghost_fill(g, e);
        d0_field(g, vis->scheme, dir, e, dv.data(), vis->d0_bound);
#pragma omp parallel for collapse(2) schedule(static)
        for (long k = 0; k < D.nz; ++k)
            for (long j = 0; j < D.ny; ++j)
                for (long i = 0; i < D.nx; ++i) {
                    const long c = i + D.nx * (j + D.ny * k);
                    const double aj = ajac ? ajac[D.lap(i, j, k)] : 1.0;
                    du[D.soa(i, j, k, q + 1)] += aj * dv[c];
                }
    }
}

void or_du_vis(const or_grid* g, const or_vis* vis, const double* u, const double* v,
               const double* w, const double* T, const double* const* metrics,
               const double* ajac, double* du) {
    Dims D(g);
    std::vector<double> ev(12 * D.lap_size(), 0.0);
    or_vis_fluxes(g, vis, u, v, w, T, metrics, ajac, ev.data());
    for (int dir = 0; dir < 3; ++dir)
        or_vis_div_add(g, vis, dir, ev.data() + 4 * dir * D.lap_size(), ajac, du);
}

// Inviscid RHS (decomposed form of the BF3W operator), du overwritten.
void or_du_invis(const or_grid* g, const double* d, const double* u,
                 const double* v, const double* w, const double* cc,
                 const double* const* metrics, const double* ajac, double* du) {
    Dims D(g);
    const long L = OR_LAP;
    std::memset(du, 0, sizeof(double) * 5 * D.cells());  // OCFD_Stream.cpp:35
    const double h[3] = {g->hx, g->hy, g->hz};
    const long ext[3] = {D.nx, D.ny, D.nz};

    for (int dir = 0; dir < 3; ++dir) {
        // lines along dir; the two other interior indices enumerate the lines
        const long n = ext[dir];
        const long na = dir == 0 ? D.ny : D.nx;   // first transverse extent
        const long nb = dir == 2 ? D.ny : D.nz;   // second transverse extent
#pragma omp parallel
        {
            std::vector<double> fp(5 * (n + 2 * L)), fm(5 * (n + 2 * L));
#pragma omp for collapse(2) schedule(static)
            for (long b = 0; b < nb; ++b)
                for (long a = 0; a < na; ++a) {
                    auto at = [&](long s) -> long {
                        if (dir == 0) return D.lap(s, a, b);
                        if (dir == 1) return D.lap(a, s, b);
                        return D.lap(a, b, s);
                    };
                    auto cell = [&](long s, long var) -> long {
                        if (dir == 0) return D.soa(s, a, b, var);
                        if (dir == 1) return D.soa(a, s, b, var);
                        return D.soa(a, b, s, var);
                    };
                    // split on the line including 4 ghosts per side
                    for (long s = -L; s < n + L; ++s) {
                        const long p = at(s);
                        double a1, a2, a3;
                        if (metrics) {
                            a1 = metrics[3 * dir + 0][p];
                            a2 = metrics[3 * dir + 1][p];
                            a3 = metrics[3 * dir + 2][p];
                        } else {
                            a1 = dir == 0 ? 1.0 : 0.0;
                            a2 = dir == 1 ? 1.0 : 0.0;
                            a3 = dir == 2 ? 1.0 : 0.0;
                        }
                        double pp[5], mm[5];
                        sw_split<double>(d[p], u[p], v[p], w[p], cc[p], a1, a2,
                                         a3, g->gamma, g->epsl_sw, pp, mm);
                        for (int var = 0; var < 5; ++var) {
                            fp[var * (n + 2 * L) + (s + L)] = pp[var];
                            fm[var * (n + 2 * L) + (s + L)] = mm[var];
                        }
                    }
                    // faces i+1/2 for i = -1..n-1 use points i-3..i+4; in
                    // CLOSURE mode the faces near a CLOSURE x or y face take
                    // the ring kernel's closure values, and the y direction
                    // drops the M term of the last cell (the ring kernel
                    // computes it but never adds it, OCFD_NS_Jacobian3d.cpp:
                    // 1580-1583)
                    const bool lo = dir < 2 && g->face_kind[2 * dir] == OR_FACE_CLOSURE;
                    const bool hi = dir < 2 && g->face_kind[2 * dir + 1] == OR_FACE_CLOSURE;
                    std::vector<double> face(n + 1);
                    for (int pm = 0; pm < 2; ++pm)
                        for (int var = 0; var < 5; ++var) {
                            const double* line =
                                (pm == 0 ? fp.data() : fm.data()) + var * (n + 2 * L);
                            for (long i = -1; i < n; ++i) {
                                const double* st = line + (i - 3 + L);
                                if ((lo || hi) &&
                                    closure_face(pm, dir, i + 1, n, lo, hi, line + L, &face[i + 1]))
                                    continue;
                                face[i + 1] = pm == 0 ? weno_p<double>(st)
                                                      : weno_m<double>(st);
                            }
                            const long iend = (dir == 1 && pm == 1 && hi) ? n - 1 : n;
                            for (long i = 0; i < iend; ++i) {
                                const double J = ajac ? ajac[at(i)] : 1.0;
                                du[cell(i, var)] += -J * (face[i + 1] - face[i]) / h[dir];
                            }
                        }
                }
        }
    }
}

// commen_kernel.cpp:78-110 (cons_to_pri_kernel); Cv = 1/(g(g-1)Ama^2)
// (OCFD_init.cpp:380).  Writes LAP interiors of d,u,v,w,T,P (P may be NULL).
void or_cons_to_prim(const or_grid* g, const double* f, double* d, double* u,
                     double* v, double* w, double* T, double* P) {
    Dims D(g);
    const double cv = 1.0 / (g->gamma * (g->gamma - 1.0) * g->ama * g->ama);
#pragma omp parallel for collapse(2) schedule(static)
    for (long k = 0; k < D.nz; ++k)
        for (long j = 0; j < D.ny; ++j)
            for (long i = 0; i < D.nx; ++i) {
                const long p = D.lap(i, j, k);
                double d1 = f[D.soa(i, j, k, 0)];
                double u1 = f[D.soa(i, j, k, 1)] / d1;
                double v1 = f[D.soa(i, j, k, 2)] / d1;
                double w1 = f[D.soa(i, j, k, 3)] / d1;
                double t1 = f[D.soa(i, j, k, 4)];
                t1 = t1 - 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1);
                d[p] = d1; u[p] = u1; v[p] = v1; w[p] = w1;
                T[p] = t1 / (d1 * cv);
                if (P) P[p] = (t1 / d1) * (g->gamma - 1.0);
            }
}

// commen_kernel.cpp:33-67 (pri_to_cons_kernel).
void or_prim_to_cons(const or_grid* g, const double* d, const double* u,
                     const double* v, const double* w, const double* T, double* f) {
    Dims D(g);
    const double cv = 1.0 / (g->gamma * (g->gamma - 1.0) * g->ama * g->ama);
#pragma omp parallel for collapse(2) schedule(static)
    for (long k = 0; k < D.nz; ++k)
        for (long j = 0; j < D.ny; ++j)
            for (long i = 0; i < D.nx; ++i) {
                const long p = D.lap(i, j, k);
                const double d1 = d[p], u1 = u[p], v1 = v[p], w1 = w[p], t1 = T[p];
                f[D.soa(i, j, k, 0)] = d1;
                f[D.soa(i, j, k, 1)] = u1 * d1;
                f[D.soa(i, j, k, 2)] = v1 * d1;
                f[D.soa(i, j, k, 3)] = w1 * d1;
                f[D.soa(i, j, k, 4)] = d1 * ((u1 * u1 + v1 * v1 + w1 * w1) * 0.5 + cv * t1);
            }
}

// SSP-RK3 stage updates, OCFD_time.cpp:15-65 (ker1/ker2/ker3).
void or_time_advance(int krk, double dt, long n, double* f, const double* fn,
                     const double* du) {
    if (krk == 1) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) f[i] = fn[i] + dt * du[i];
    } else if (krk == 2) {
        const double a = 3.0 / 4.0, b = 1.0 / 4.0;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) f[i] = a * fn[i] + b * (f[i] + dt * du[i]);
    } else {
        const double a = 1.0 / 3.0, b = 2.0 / 3.0;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) f[i] = a * fn[i] + b * (f[i] + dt * du[i]);
    }
}

double or_compute_dt(const or_grid* g, const double* f, double cfl) {
    Dims D(g);
    const double cv = 1.0 / (g->gamma * (g->gamma - 1.0) * g->ama * g->ama);
    const double rx = 1.0 / g->hx, ry = 1.0 / g->hy, rz = 1.0 / g->hz;
    const double rr = std::sqrt(rx * rx + ry * ry + rz * rz);
    double smax = 0.0;
#pragma omp parallel for collapse(2) reduction(max : smax) schedule(static)
    for (long k = 0; k < D.nz; ++k)
        for (long j = 0; j < D.ny; ++j)
            for (long i = 0; i < D.nx; ++i) {
                double d1 = f[D.soa(i, j, k, 0)];
                double u1 = f[D.soa(i, j, k, 1)] / d1;
                double v1 = f[D.soa(i, j, k, 2)] / d1;
                double w1 = f[D.soa(i, j, k, 3)] / d1;
                double e = f[D.soa(i, j, k, 4)] - 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1);
                double T = e / (d1 * cv);
                double c = std::sqrt(T) / g->ama;
                double s = std::fabs(u1) * rx + std::fabs(v1) * ry + std::fabs(w1) * rz + c * rr;
                smax = s > smax ? s : smax;
            }
    return cfl / smax;
}

namespace {
struct Work {
    std::vector<double> d, u, v, w, T, P, cc, fn, du;
    explicit Work(const Dims& D)
        : d(D.lap_size()), u(D.lap_size()), v(D.lap_size()), w(D.lap_size()),
          T(D.lap_size()), P(D.lap_size()), cc(D.lap_size()),
          fn(5 * D.cells()), du(5 * D.cells()) {}
};

void rhs_from_cons(const or_grid* g, const double* f, Work& W,
                   const double* const* metrics, const double* ajac,
                   const or_vis* vis = nullptr) {
    or_cons_to_prim(g, f, W.d.data(), W.u.data(), W.v.data(), W.w.data(),
                    W.T.data(), W.P.data());
    or_ghost_fill(g, W.d.data());
    or_ghost_fill(g, W.u.data());
    or_ghost_fill(g, W.v.data());
    or_ghost_fill(g, W.w.data());
    or_ghost_fill(g, W.T.data());
    or_sound_speed(g, W.T.data(), W.cc.data());
    or_du_invis(g, W.d.data(), W.u.data(), W.v.data(), W.w.data(), W.cc.data(),
                metrics, ajac, W.du.data());
    if (vis)   // du_comput: inviscid, then viscous (OCFD_Stream.cpp:27-45)
        or_du_vis(g, vis, W.u.data(), W.v.data(), W.w.data(), W.T.data(), metrics, ajac,
                  W.du.data());
}
}  // namespace

int or_rhs_conserved(const or_grid* g, const double* f, double* du,
                     const double* const* metrics, const double* ajac) {
    Dims D(g);
    Work W(D);
    rhs_from_cons(g, f, W, metrics, ajac);
    std::memcpy(du, W.du.data(), sizeof(double) * 5 * D.cells());
    return 0;
}

int or_rhs_conserved_ns(const or_grid* g, const or_vis* vis, const double* f, double* du,
                        const double* const* metrics, const double* ajac) {
    Dims D(g);
    Work W(D);
    rhs_from_cons(g, f, W, metrics, ajac, vis);
    std::memcpy(du, W.du.data(), sizeof(double) * 5 * D.cells());
    return 0;
}

// Solver loop OCFD_NS_Solver.cpp:64-90 with all three SSP-RK3 stages: the
// state at the start of the step is kept in fn (the reference's pf/pfn swap).
int or_rk3_steps_ns(const or_grid* g, const or_vis* vis, double* f, double dt, int nsteps,
                    const double* const* metrics, const double* ajac) {
    Dims D(g);
    Work W(D);
    const long n = 5 * D.cells();
    for (int s = 0; s < nsteps; ++s) {
        std::memcpy(W.fn.data(), f, sizeof(double) * n);
        for (int krk = 1; krk <= 3; ++krk) {
            rhs_from_cons(g, f, W, metrics, ajac, vis);
            or_time_advance(krk, dt, n, f, W.fn.data(), W.du.data());
        }
    }
    return 0;
}

int or_rk3_steps(const or_grid* g, double* f, double dt, int nsteps,
                 const double* const* metrics, const double* ajac) {
    return or_rk3_steps_ns(g, nullptr, f, dt, nsteps, metrics, ajac);
}

// Algorithmic operation counts of one cell-RHS, from the same templates the
// oracle runs: 3 directions x (1 split + 5 vars x (P + M WENO) + 10 face
// differences of 4 operations each: subtract, times J, divide by h, accumulate).
void or_op_counts(double* out) {
    double s[8] = {1.0, 1.1, 0.9, 1.3, 1.2, 0.8, 1.05, 0.95};
    Cnt cs[8];
    for (int i = 0; i < 8; ++i) cs[i] = Cnt(s[i]);
    auto total = [](const OpTally& t) {
        return double(t.add + t.mul + t.div + t.sqrt + t.max);
    };
    g_tally = OpTally();
    Cnt fp[5], fm[5];
    sw_split<Cnt>(Cnt(1.0), Cnt(0.5), Cnt(0.1), Cnt(0.2), Cnt(1.0), Cnt(0.5),
                  Cnt(0.6), Cnt(0.7), 1.4, 1e-6, fp, fm);
    const OpTally split = g_tally;
    g_tally = OpTally();
    (void)weno_p<Cnt>(cs);
    const OpTally wp = g_tally;
    g_tally = OpTally();
    (void)weno_m<Cnt>(cs);
    const OpTally wm = g_tally;
    const double diff = 4.0;
    out[0] = total(split);
    out[1] = total(wp);
    out[2] = total(wm);
    out[3] = diff;
    out[4] = 3.0 * (total(split) + 5.0 * (total(wp) + total(wm)) + 10.0 * diff);
    out[5] = double(split.sqrt + split.div);
    out[6] = 3.0 * 5.0 * double(wp.div + wm.div);
}

void or_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int or_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
