// bf3w_rhs_impl.cuh -- fused BF3W inviscid RHS for sm_100a (device code).
//
// Included by the instantiation units bf3w_rhs_{f64,f32}{,_clo}.cu, each of
// which compiles one (precision, closure) slice of the kernels; the host
// dispatch is bf3w_rhs.cu.
//
// Replaces the reference's fused kernel split_Jac3d_Stager_Warming_ker
// (src/kernels/OCFD_split.cpp:36-3918) together with its boundary-ring kernel
// (src/solver/OCFD_NS_Jacobian3d.cpp:828-2530): one launch computes
//   du[v] = -J * sum_dir ( F^_dir(i+1/2) - F^_dir(i-1/2) ) / h_dir,
//   F^ = WENO7-SYMBO_P(F+) + WENO7-SYMBO_M(F-),  F+- = Steger-Warming split,
// on every cell of the job, with the ghost layers providing the boundary
// values (WENO7 everywhere: the reference's DIF_BOUND = 0 semantics).
//
// Design (B200 first, not a translation of the wave64 kernel):
//   * A CTA owns a BX x BY column footprint and sweeps it along z (the
//     reference's scanZ reuse).  The z-direction split fluxes of the last
//     9 planes live in a shared-memory ring, so every z face is reconstructed
//     exactly once and no split value goes through HBM (the reference
//     round-trips fpY/fmY/fpZ/fmZ through global scratch).
//   * Per plane, two barrier intervals:
//       A: x-split over (BX+8) x BY points and y-split over BX x (BY+8)
//          points into shared memory, the z-split of the plane 5 ahead into
//          the ring, and the z faces above the plane, whose stencils are all
//          in the ring already (1216 items at 16x8);
//       B: every x, y face of the plane as one work item (face, variable)
//          evaluating its P and M WENO once (1400 items at 16x8);
//     then the FP64 face difference writes du (no barrier needed before the
//     next plane's split interval: the arrays are disjoint).
//   * Primitive planes are staged with TMA tile loads (one thread issues
//     them, an mbarrier tracks their bytes), double-buffered one plane
//     ahead: the buffer of plane z holds its (BX+8) x (BY+8) box and the
//     BX x BY centre of plane z+5.  Fields whose box starts would not be
//     16-byte aligned are staged with per-thread cp.async instead.
//   * Stage mode (EPI, used by the solver and batches): instead of writing
//     du, the difference phase applies the SSP-RK3 stage to the conserved
//     state and writes the primitives of the new state to a second set of
//     LAP fields -- the separate stage kernel and the du round trip through
//     HBM disappear.  One thread per cell (the last BX*BY threads, which have
//     the least split work in the next interval) does all five variables,
//     so it owns its cell's f/fn staging (cp.async one plane ahead) and no
//     barrier guards it; the other threads go on to the next plane.
//   * Persistent grid, one CTA per SM.  Whole tile columns are swept round
//     robin (CTA b takes tiles b, b+G, ...), so the CTAs resident together
//     sweep neighbouring columns at the same z and their halo re-reads hit
//     L2; the (tile, plane) space of the tiles left over is then cut into
//     equal contiguous ranges, one per CTA, so every CTA ends with the same
//     number of planes (a range that crosses a tile boundary starts a new
//     sweep with its own 9-plane prologue).
//   * No tensor cores: nothing on this path is a contraction.  The bound is
//     the FP64 pipe (7266 algorithmic FLOP per cell).
#pragma once
#include <cstdio>

#include "ws_device.cuh"
#include "ws_internal.h"

namespace ws {

template <int BX, int BY, typename CT, bool EPI = false>
struct RhsLayout {
    static constexpr int BXY = BX * BY;
    static constexpr int SXW = BX + 8;        // x-split row width
    // x-split row pitch: for 4-byte types padded so that the 32 / BX rows a
    // warp's x faces read start on disjoint bank groups (unpadded, two rows
    // of a warp share banks and every such load takes two wavefronts)
    static constexpr int SXP = sizeof(CT) == 8 ? SXW : BX == 8 ? 24 : BX == 16 ? 48 : SXW;
    static_assert(SXP >= SXW, "x-split pitch");
    static constexpr int SYH = BY + 8;        // y-split rows
    static constexpr int BOXW = BX + 8, BOXH = BY + 8, BOX = BOXW * BOXH;
    static constexpr int STG = 5 * (BOX + BXY);   // doubles per staging buffer
    static constexpr int RING = 9;                // z planes held
    static constexpr int RS = 10 * BXY;           // ring slot stride (CT)
    static constexpr int N_STG = 2 * STG;         // double
    static constexpr int N_FX = 5 * BY * (BX + 1);
    static constexpr int N_FY = 5 * (BY + 1) * BX;
    // z faces of the last 3 planes: a plane's z faces are computed in
    // interval A while the previous plane's difference may still read two
    static constexpr int NFZS = 3;
    static constexpr int N_FZ = NFZS * 5 * BXY;
    static constexpr int N_FB = EPI ? 2 * 15 * BXY : 0;   // fn, f, viscous terms, x2
    static constexpr int N_RING = RING * RS;      // CT
    static constexpr int N_SX = 10 * BY * SXP;    // CT
    static constexpr int N_SY = 10 * SYH * BX;    // CT
    static constexpr size_t smem_bytes =
        (size_t)(N_STG + N_FX + N_FY + N_FZ + N_FB) * sizeof(double) +
        (size_t)(N_RING + N_SX + N_SY) * sizeof(CT);
    // two CTAs per SM when both fit (228 KB per SM, 1 KB reserved per CTA):
    // one CTA's barrier waits then overlap the other's arithmetic
    static constexpr int MINB = (2 * (smem_bytes + 128 + 1024) <= 228 * 1024) ? 2 : 1;
};

__device__ __forceinline__ size_t lap_index(int X, int Y, int Z, uint32_t pitch, int ny) {
    return (size_t)X + (size_t)pitch * ((size_t)Y + (size_t)(ny + 8) * (size_t)Z);
}
__device__ __forceinline__ size_t soa_index(const ws_soa& s, int i, int j, int k, int var) {
    return (size_t)i + (size_t)s.pitch * ((size_t)j + (size_t)s.length_Y *
                                          ((size_t)k + (size_t)s.length_Z * (size_t)var));
}
__device__ __forceinline__ double ldg_prim(const RhsArgs& a, int f, int X, int Y, int Z) {
    return __ldg(a.prim[f] + lap_index(X, Y, Z, a.ppitch[f], a.ny));
}
__device__ __forceinline__ double ldg_met(const RhsArgs& a, int m, int X, int Y, int Z) {
    return __ldg(a.met[m] + lap_index(X, Y, Z, a.mpitch[m], a.ny));
}

// Split of one point in direction DIR; metrics loaded from global when the
// grid is not Cartesian.
template <int DIR, bool UNI, typename CT>
__device__ __forceinline__ void split_point(const RhsArgs& a, const SplitK<CT>& k, double d,
                                            double u, double v, double w, double c, int X,
                                            int Y, int Z, CT out[10]) {
    if (UNI) {
        sw_split_cart<DIR, CT>(CT(d), CT(u), CT(v), CT(w), CT(c), k, out);
    } else {
        const CT a1 = CT(ldg_met(a, 3 * DIR + 0, X, Y, Z));
        const CT a2 = CT(ldg_met(a, 3 * DIR + 1, X, Y, Z));
        const CT a3 = CT(ldg_met(a, 3 * DIR + 2, X, Y, Z));
        sw_split_gen<CT>(CT(d), CT(u), CT(v), CT(w), CT(c), a1, a2, a3, k, out);
    }
}

// Face flux F^ = P(F+) + M(F-) of one face and variable from 8 staged split
// values each.  Element k of the P stencil is at bp[k*stride], minus `wrap`
// once k >= kw (the z ring wraps; x and y rows pass kw = 8); the M stencil is
// the reversed F- row at +pmoff.
// CHOL: FP64 indicators in the Cholesky form (plain RHS kernels), else the
// difference-chain form (stage kernels, which are at their register limit)
template <typename CT, bool CHOL = true>
__device__ __forceinline__ double face_flux(const CT* bp, int pmoff, int stride, int kw,
                                            int wrap);

template <>
__device__ __forceinline__ double face_flux<double, true>(const double* bp, int pmoff,
                                                          int stride, int kw, int wrap);
template <>
__device__ __forceinline__ double face_flux<double, false>(const double* bp, int pmoff,
                                                           int stride, int kw, int wrap);

template <bool CHOL>
__device__ __forceinline__ double face_flux_f64(const double* bp, int pmoff, int stride, int kw,
                                                int wrap) {
    double t[8], np, dp, nm, dm;
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = bp[k * stride - (k >= kw ? wrap : 0)];
    weno7_symbo_nd<CHOL>(t, np, dp);
    const double p3 = t[3];
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = bp[pmoff + (7 - k) * stride - ((7 - k) >= kw ? wrap : 0)];
    weno7_symbo_nd<CHOL>(t, nm, dm);
    const double m3 = t[3];
    return (p3 + m3) + (np * dm + nm * dp) / (dp * dm);
}
template <>
__device__ __forceinline__ double face_flux<double, true>(const double* bp, int pmoff,
                                                          int stride, int kw, int wrap) {
    return face_flux_f64<true>(bp, pmoff, stride, kw, wrap);
}
template <>
__device__ __forceinline__ double face_flux<double, false>(const double* bp, int pmoff,
                                                           int stride, int kw, int wrap) {
    return face_flux_f64<false>(bp, pmoff, stride, kw, wrap);
}

// mixed form: P and M in the two lanes of packed FP32x2 arithmetic; the face
// value is summed in FP32 and widened once (the face difference is FP64)
template <>
__device__ __forceinline__ double face_flux<float, true>(const float* bp, int pmoff, int stride,
                                                         int kw, int wrap);
template <>
__device__ __forceinline__ double face_flux<float, false>(const float* bp, int pmoff,
                                                          int stride, int kw, int wrap);
__device__ __forceinline__ double face_flux_f32(const float* bp, int pmoff, int stride, int kw,
                                                int wrap) {
    float2 t[8], n, d;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        t[k] = make_float2(bp[k * stride - (k >= kw ? wrap : 0)],
                           bp[pmoff + (7 - k) * stride - ((7 - k) >= kw ? wrap : 0)]);
    weno7_symbo_pm_f32x2(t, n, d);
    const float q = (n.x * d.y + n.y * d.x) * rcp_approx(d.x * d.y);
    return (double)((t[3].x + t[3].y) + q);
}
template <>
__device__ __forceinline__ double face_flux<float, true>(const float* bp, int pmoff, int stride,
                                                         int kw, int wrap) {
    return face_flux_f32(bp, pmoff, stride, kw, wrap);
}
template <>
__device__ __forceinline__ double face_flux<float, false>(const float* bp, int pmoff,
                                                          int stride, int kw, int wrap) {
    return face_flux_f32(bp, pmoff, stride, kw, wrap);
}

// CLOSURE face mode: value P + M of face f (between cells f-1 and f, f in
// 0..n) of an x (YDIR false) or y line of n cells, for a face next to a
// CLOSURE face (lo / hi: the low / high face of the direction is one).
// prow[k*stride] is F+ of cell f-4+k and mrow[k*stride] F- of that cell
// (k = 0..7, the WENO7 stencil of the face).  Each of P and M takes the ring
// kernel's closure value where one applies (the per-face rules of
// OCFD_NS_Jacobian3d.cpp:1063-1085 in x, :1515-1584 in y) and its WENO7
// value otherwise.  In y the ring kernel drops the M term of the last cell;
// the face above it (f == n, used by that cell only) carries M of face n-1
// instead of its own, which cancels the M term in that cell's difference.
// The same from the two stencils as arrays: sp[k] = F+ and sm[k] = F- of
// cell f-4+k.
__device__ __forceinline__ double closure_value_arr(const double sp[8], const double sm[8], int f,
                                                    int n, bool lo, bool hi, bool ydir) {
    double P, M, num, den;
    if (lo && f == 0) P = sp[4];
    else if (lo && f == 1) P = w5::p_lift(sp + 1);
    else if (lo && f == 2) P = w5::p_lift_plus(sp + 1);
    else if ((lo && f == 3) || (hi && f == n - 2)) P = w5::p3(sp + 1);
    else if (hi && f == n - 1) P = w5::p_right_plus(sp + 1);
    else if (hi && f == n)
        P = ydir ? sp[3] + 0.5 * w5::minmod2(sp[3] - sp[2], sp[3] - sp[2])
                 : 1.5 * sp[3] - 0.5 * sp[2];
    else {
        double t[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) t[k] = sp[k];
        weno7_symbo_nd<false>(t, num, den);
        P = sp[3] + num / den;
    }
    if (lo && f == 0) M = w5::m_lift(sm + 2);
    else if (lo && f == 1) M = w5::m_lift_plus(sm + 2);
    else if ((lo && (f == 2 || f == 3)) || (hi && f == n - 3)) M = w5::m3(sm + 2);
    else if (hi && f == n - 2) M = w5::m_right_plus(sm + 2);
    else if (hi && f == n - 1)
        M = ydir ? sm[4] - 0.5 * w5::minmod2(sm[4] - sm[3], sm[4] - sm[3])
                 : 0.5 * sm[4] + 0.5 * sm[3];
    else if (hi && f == n)      // y: M of face n-1 (see above)
        M = ydir ? sm[3] - 0.5 * w5::minmod2(sm[3] - sm[2], sm[3] - sm[2])
                 : 0.5 * sm[3] + 0.5 * sm[2];
    else {
        double t[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) t[k] = sm[7 - k];
        weno7_symbo_nd<false>(t, num, den);
        M = sm[4] + num / den;
    }
    return P + M;
}

template <typename CT>
__device__ __forceinline__ double closure_value(const CT* prow, const CT* mrow, int stride, int f,
                                             int n, bool lo, bool hi, bool ydir) {
    double sp[8], sm[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        sp[k] = (double)prow[k * stride];
        sm[k] = (double)mrow[k * stride];
    }
    return closure_value_arr(sp, sm, f, n, lo, hi, ydir);
}

// face f of a direction with n cells needs a closure value
__device__ __forceinline__ bool closure_face(int f, int n, int lo, int hi) {
    return (lo && f <= 3) || (hi && f >= n - 3);
}

// cp.async the primitive box of plane z (x: x0-4..x0+BX+3, y: y0-4..y0+BY+3)
// and the BX x BY centre of plane z+5 into one staging buffer.  Coordinates
// past the array (partial tiles, the last plane) are clamped into it; those
// values are never used.
template <int BX, int BY, int NT>
__device__ __forceinline__ void issue_stage(const RhsArgs& a, double* s, int x0, int y0,
                                            int z) {
    using L = RhsLayout<BX, BY, double>;
    const int zc = min(z + 5, a.nz + 7);
    for (int t = threadIdx.x; t < 5 * (L::BOX + L::BXY); t += NT) {
        int f, X, Y, Z;
        if (t < 5 * L::BOX) {
            f = t / L::BOX;
            const int r = t - f * L::BOX;
            const int yy = r / L::BOXW, xx = r - yy * L::BOXW;
            X = min(x0 - 4 + xx, a.nx + 7);
            Y = min(y0 - 4 + yy, a.ny + 7);
            Z = z;
        } else {
            const int t2 = t - 5 * L::BOX;
            f = t2 / L::BXY;
            const int c = t2 - f * L::BXY;
            X = min(x0 + c % BX, a.nx + 7);
            Y = min(y0 + c / BX, a.ny + 7);
            Z = zc;
        }
        cp_async8(s + t, a.prim[f] + lap_index(X, Y, Z, a.ppitch[f], a.ny));
    }
}

// TMA form of issue_stage, issued by one thread: the 5 boxes and 5 centres
// as 3D tiles completing on `bar`.  Box starts outside the array read zeros
// (partial tiles; never used).  GMAP: the maps live in global memory (the
// batched kernel's argument table) and are fenced for the tensor-map proxy
// before their first use in a sweep.
template <int BX, int BY, bool GMAP>
__device__ __forceinline__ void issue_stage_tma(const RhsArgs& a, double* s, int x0, int y0,
                                                int z, uint64_t* bar, bool first) {
    using L = RhsLayout<BX, BY, double>;
    if (GMAP && first) {
        for (int f = 0; f < 5; ++f) {
            asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;\n" ::"l"(
                             &a.tm_box[f])
                         : "memory");
            asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;\n" ::"l"(
                             &a.tm_ctr[f])
                         : "memory");
        }
    }
    mbar_expect_tx(bar, (uint32_t)(L::STG * sizeof(double)));
    const int zc = min(z + 5, a.nz + 7);
#pragma unroll
    for (int f = 0; f < 5; ++f) {
        tma_load_3d(s + f * L::BOX, &a.tm_box[f], x0 - 4, y0 - 4, z, bar);
        tma_load_3d(s + 5 * L::BOX + f * L::BXY, &a.tm_ctr[f], x0, y0, zc, bar);
    }
}

// a staging wait that gave up: recorded in the grid's status word (bit 1)
// or, for the drop-in path that has none, in this flag
// status bit 2: a staging wait gave up and the CTA stopped (every launch
// carries a status word: the grid's own, or the library's device error word)
__device__ __forceinline__ void report_stage_timeout(const RhsArgs& a) {
    if (a.status) atomicOr(a.status, 2);
}

// stage mode: cp.async fn (and, after stage 1, f; with viscous terms,
// those) of one cell into fb[v][col] (fn 0..4, f 5..9, viscous 10..14);
// `cell` is the SoA offset of the cell's variable 0 and vs the variable
// stride (f_in, fn and the viscous terms share one SoA shape)
__device__ __forceinline__ void issue_fcell(const RhsArgs& a, double* fb, int bxy, int col,
                                            size_t cell, size_t vs, int krk) {
#pragma unroll
    for (int v = 0; v < 5; ++v) cp_async8(fb + v * bxy + col, a.fn.ptr + cell + v * vs);
    if (krk > 1) {
#pragma unroll
        for (int v = 0; v < 5; ++v)
            cp_async8(fb + (5 + v) * bxy + col, a.f_in.ptr + cell + v * vs);
    }
    if (a.dvis.ptr) {
#pragma unroll
        for (int v = 0; v < 5; ++v)
            cp_async8(fb + (10 + v) * bxy + col, a.dvis.ptr + cell + v * vs);
    }
}

// stage mode: primitives of the new state q of one cell into p_out
// (commen_kernel.cpp:78-110; the divisions by rho, cv and Ama are taken as
// one reciprocal and products)
__device__ __forceinline__ void store_prims(const RhsArgs& a, const double q[5], int X, int Y,
                                            int z) {
    const double d1 = q[0], r = 1.0 / d1;
    const double u1 = q[1] * r, v1 = q[2] * r, w1 = q[3] * r;
    const double t1 = q[4] - 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1);
    const double T1 = t1 * r * a.rcv;
    const double vals[6] = {d1, u1, v1, w1, T1, sqrt(T1) * a.rama};
    const size_t idx = lap_index(X, Y, z, a.p_pitch, a.ny);
#pragma unroll
    for (int f = 0; f < 6; ++f) a.p_out[f][idx] = vals[f];
    if (!(d1 > 0.0 && T1 > 0.0 && T1 < INFINITY)) atomicOr(a.status, 1);
}

// Returns false when a TMA staging wait gave up (the caller then stops).
template <int BX, int BY, int NT, bool UNI, typename CT, bool EPI, bool GMAP, bool CLO>
__device__ __forceinline__ bool sweep(const RhsArgs& a, const SplitK<CT>& k, unsigned char* smem,
                                      int x0, int y0, int z0, int z1, int krk, uint64_t* bar,
                                      uint32_t& ph, bool& first) {
    using L = RhsLayout<BX, BY, CT, EPI>;
    constexpr int BXY = L::BXY, SXW = L::SXW, SXP = L::SXP, SYH = L::SYH, BOXW = L::BOXW,
                  BOX = L::BOX;
    constexpr int RS = L::RS;
    double* stg = reinterpret_cast<double*>(smem);       // [2][STG]
    double* fx = stg + L::N_STG;                         // [5][BY][BX+1]
    double* fy = fx + L::N_FX;                           // [5][BY+1][BX]
    double* fz = fy + L::N_FY;                           // [NFZS][5][BXY]
    double* fb = fz + L::N_FZ;                           // [2][15][BXY]   (stage mode)
    CT* ring = reinterpret_cast<CT*>(fb + L::N_FB);      // [9][10][BXY]
    CT* sxs = ring + L::N_RING;                          // [10][BY][SXP], rows of SXW
    CT* sys = sxs + L::N_SX;                             // [10][SYH][BX]
    const int tid = threadIdx.x;
    static_assert(NT >= BXY, "one thread per cell in the stage epilogue");
    static_assert(!EPI || UNI, "the stage epilogue is compiled for Cartesian grids");
    // stage mode: this thread's cell (dcol < 0: none) and its SoA offsets
    const int dcol = tid - (NT - BXY);
    const int dX = x0 + (dcol >= 0 ? dcol % BX : 0), dY = y0 + (dcol >= 0 ? dcol / BX : 0);
    const bool dcell = EPI && dcol >= 0 && dX < a.ex && dY < a.ey;
    const size_t fps = (size_t)a.fn.pitch * a.fn.length_Y;      // plane stride
    const size_t fvs = fps * a.fn.length_Z;                     // variable stride
    const size_t fc0 = dcell ? soa_index(a.fn, dX - 4, dY - 4, 0, 0) - 4 * fps : 0;

    const bool tma = a.tma != 0;
    if (!tma) issue_stage<BX, BY, NT>(a, stg, x0, y0, z0);
    else if (tid == 0) issue_stage_tma<BX, BY, GMAP>(a, stg, x0, y0, z0, &bar[0], first);
    first = false;
    if (dcell) issue_fcell(a, fb, BXY, dcol, fc0 + (size_t)z0 * fps, fvs, krk);
    cp_async_commit();

    // prologue: z split of planes z0-4 .. z0+4 into the ring
    for (int t = tid; t < 9 * BXY; t += NT) {
        const int pl = t / BXY, col = t - pl * BXY;
        const int Z = z0 - 4 + pl;
        const int X = min(x0 + col % BX, a.nx + 7), Y = min(y0 + col / BX, a.ny + 7);
        CT out[10];
        split_point<2, UNI, CT>(a, k, ldg_prim(a, 0, X, Y, Z), ldg_prim(a, 1, X, Y, Z),
                                ldg_prim(a, 2, X, Y, Z), ldg_prim(a, 3, X, Y, Z),
                                ldg_prim(a, 4, X, Y, Z), X, Y, Z, out);
        CT* dst = ring + (Z % 9) * RS + col;
#pragma unroll
        for (int c = 0; c < 10; ++c) dst[c * BXY] = out[c];
    }
    __syncthreads();
    {   // z face z0-1/2: stencil planes z0-4 .. z0+3
        const int s0 = (z0 - 4) % 9;
        for (int t = tid; t < 5 * BXY; t += NT) {
            const int var = t / BXY, col = t - var * BXY;
            fz[t] = face_flux<CT, !EPI>(ring + s0 * RS + var * BXY + col, 5 * BXY, RS, 9 - s0, 9 * RS);
        }
    }
    cp_async_wait<0>();
    {
        // a.hold_polls > 0 (failure-path test): wait on bar[2], on which
        // nothing ever arrives, for that many polls, so the timeout path runs
        const uint32_t want = ph & 1u;
        bool bad = false;
        if (tma) {
            bad = a.hold_polls > 0 ? !mbar_wait_bounded(&bar[2], 0u, a.hold_polls)
                                   : !mbar_wait_bounded(&bar[0], want);
            ph ^= 1u;
        }
        if (__syncthreads_or(bad)) {
            if (tid == 0) {
                report_stage_timeout(a);
                mbar_wait_bounded(&bar[0], want);     // the copies still in flight
            }
            return false;
        }
    }

    int prev = 0;
    for (int z = z0; z < z1; ++z) {
        const int b = (z - z0) & 1;
        const double* sb = stg + b * L::STG;

        // ---- interval A: x- and y-split of plane z, z-split of plane z+5
        constexpr unsigned NXS = SXW * BY, NYS = BX * SYH;
        unsigned ta = tid;
        for (; ta < NXS + NYS; ta += NT) {
            const int t = ta;
            CT out[10];
            if (t < NXS) {
                const int yy = t / SXW, xi = t - yy * SXW;
                const int bi = (yy + 4) * BOXW + xi;
                split_point<0, UNI, CT>(a, k, sb[bi], sb[BOX + bi], sb[2 * BOX + bi],
                                        sb[3 * BOX + bi], sb[4 * BOX + bi],
                                        min(x0 - 4 + xi, a.nx + 7), min(y0 + yy, a.ny + 7), z,
                                        out);
                CT* dst = sxs + yy * SXP + xi;
#pragma unroll
                for (int c = 0; c < 10; ++c) dst[c * BY * SXP] = out[c];
            } else {
                const int t2 = t - NXS;
                const int yi = t2 / BX, xx = t2 - yi * BX;
                const int bi = yi * BOXW + xx + 4;
                split_point<1, UNI, CT>(a, k, sb[bi], sb[BOX + bi], sb[2 * BOX + bi],
                                        sb[3 * BOX + bi], sb[4 * BOX + bi],
                                        min(x0 + xx, a.nx + 7), min(y0 - 4 + yi, a.ny + 7), z,
                                        out);
                CT* dst = sys + yi * BX + xx;
#pragma unroll
                for (int c = 0; c < 10; ++c) dst[c * SYH * BX] = out[c];
            }
        }
        const bool more = z + 1 < z1;
        ta -= NXS + NYS;
        if (more) {   // plane z+5 enters the ring (slot of plane z-4, last read by face z-1/2)
            for (; ta < BXY; ta += NT) {
                const int col = ta;
                const double* cb = sb + 5 * BOX + col;
                const int Z = z + 5;
                CT out[10];
                split_point<2, UNI, CT>(a, k, cb[0], cb[BXY], cb[2 * BXY], cb[3 * BXY],
                                        cb[4 * BXY], min(x0 + col % BX, a.nx + 7),
                                        min(y0 + col / BX, a.ny + 7), min(Z, a.nz + 7), out);
                CT* dst = ring + (Z % 9) * RS + col;
#pragma unroll
                for (int c = 0; c < 10; ++c) dst[c * BXY] = out[c];
            }
            ta -= BXY;
        }
        // z face z+1/2 (stencil planes z-3 .. z+4, in the ring since the last
        // interval) into the next slot, beside the splits (the previous
        // plane's difference may still read the two previous slots)
        const int cur = prev + 1 == L::NFZS ? 0 : prev + 1;
        {
            constexpr unsigned NZF = 5 * BXY;
            const int s0 = (z - 3) % 9;
            for (; ta < NZF; ta += NT)
                fz[cur * 5 * BXY + ta] =
                    face_flux<CT, !EPI>(ring + s0 * RS + ta, 5 * BXY, RS, 9 - s0, 9 * RS);
        }
        if (more) {
            if (!tma) {
                issue_stage<BX, BY, NT>(a, stg + (b ^ 1) * L::STG, x0, y0, z + 1);
                cp_async_commit();
            } else if (tid == 0) {
                issue_stage_tma<BX, BY, GMAP>(a, stg + (b ^ 1) * L::STG, x0, y0, z + 1,
                                              &bar[b ^ 1], false);
            }
        }
        __syncthreads();

        // ---- interval B: x and y faces of plane z
        // One round robin over the plane's items, split into loops by item
        // kind (no per-item branch chain): the x face right of each column
        // and the y face above each row (power-of-two index math), then the
        // left/bottom faces of the tile.
        constexpr unsigned NXR = 5 * BXY, NYR = 5 * BXY;
        constexpr unsigned NE = 5 * (BY + BX);
        unsigned t = tid;
        const bool clx = CLO && (a.clo[0] | a.clo[1]), cly = CLO && (a.clo[2] | a.clo[3]);
        for (; t < NXR; t += NT) {
            const unsigned var = t / BXY, r = t % BXY, yy = r / BX, xx = r % BX;
            const CT* bp = sxs + (var * BY + yy) * SXP + xx + 1;
            const int f = x0 - 3 + (int)xx;
            fx[(var * BY + yy) * (BX + 1) + xx + 1] =
                (clx && closure_face(f, a.nx, a.clo[0], a.clo[1]))
                    ? closure_value<CT>(bp, bp + 5 * BY * SXP, 1, f, a.nx, a.clo[0], a.clo[1],
                                        false)
                    : face_flux<CT, !EPI>(bp, 5 * BY * SXP, 1, 8, 0);
        }
        for (t -= NXR; t < NYR; t += NT) {
            const unsigned var = t / BXY, r = t % BXY, g = r / BX + 1, xx = r % BX;
            const CT* bp = sys + (var * SYH + g) * BX + xx;
            const int f = y0 - 4 + (int)g;
            fy[(var * (BY + 1) + g) * BX + xx] =
                (cly && closure_face(f, a.ny, a.clo[2], a.clo[3]))
                    ? closure_value<CT>(bp, bp + 5 * SYH * BX, BX, f, a.ny, a.clo[2], a.clo[3],
                                        true)
                    : face_flux<CT, !EPI>(bp, 5 * SYH * BX, BX, 8, 0);
        }
        for (t -= NYR; t < NE; t += NT) {
            if (t < 5 * BY) {
                const unsigned var = t / BY, yy = t % BY;
                const CT* bp = sxs + (var * BY + yy) * SXP;
                const int f = x0 - 4;
                fx[(var * BY + yy) * (BX + 1)] =
                    (clx && closure_face(f, a.nx, a.clo[0], a.clo[1]))
                        ? closure_value<CT>(bp, bp + 5 * BY * SXP, 1, f, a.nx, a.clo[0],
                                            a.clo[1], false)
                        : face_flux<CT, !EPI>(bp, 5 * BY * SXP, 1, 8, 0);
            } else {
                const unsigned var = (t - 5 * BY) / BX, xx = (t - 5 * BY) % BX;
                const CT* bp = sys + var * SYH * BX + xx;
                const int f = y0 - 4;
                fy[var * (BY + 1) * BX + xx] =
                    (cly && closure_face(f, a.ny, a.clo[2], a.clo[3]))
                        ? closure_value<CT>(bp, bp + 5 * SYH * BX, BX, f, a.ny, a.clo[2],
                                            a.clo[3], true)
                        : face_flux<CT, !EPI>(bp, 5 * SYH * BX, BX, 8, 0);
            }
        }
        cp_async_wait<0>();
        {   // the next plane's staging has landed (TMA: its barrier phase)
            const bool wt = tma && more;
            const uint32_t want = (ph >> (b ^ 1)) & 1u;
            const bool bad = wt && !mbar_wait_bounded(&bar[b ^ 1], want);
            if (wt) ph ^= 1u << (b ^ 1);
            if (__syncthreads_or(bad)) {
                if (tid == 0) {
                    report_stage_timeout(a);
                    mbar_wait_bounded(&bar[b ^ 1], want);   // the copies still in flight
                }
                return false;
            }
        }

        // ---- face difference of plane z (FP64): du, or the RK stage
        if (EPI) {
            if (dcell) {
                const double* fbz = fb + b * 15 * BXY;
                // the cell's coordinates and offsets are recomputed here rather
                // than kept live across the sweep (register pressure)
                const int dcol = tid - (NT - BXY);
                const int xx = dcol % BX, yy = dcol / BX;
                const int dX = x0 + xx, dY = y0 + yy;
                const size_t fps = (size_t)a.fn.pitch * a.fn.length_Y;
                const size_t fvs = fps * a.fn.length_Z;
                const size_t cell = soa_index(a.fn, dX - 4, dY - 4, z - 4, 0);
                double q[5];
#pragma unroll
                for (int var = 0; var < 5; ++var) {
                    const double* px = fx + (var * BY + yy) * (BX + 1) + xx;
                    const double* py = fy + (var * (BY + 1) + yy) * BX + xx;
                    const int i = var * BXY + dcol;
                    double r = (px[1] - px[0]) * a.rhx;
                    r = fma(py[BX] - py[0], a.rhy, r);
                    r = fma(fz[cur * 5 * BXY + i] - fz[prev * 5 * BXY + i], a.rhz, r);
                    const double fo = krk == 1 ? 0.0 : fbz[5 * BXY + i];
                    // Navier-Stokes: the viscous terms of this cell (staged with f, fn)
                    const double dv = a.dvis.ptr ? fbz[10 * BXY + i] : 0.0;
                    q[var] = ws_rk_stage(krk, fbz[i], fo, dv - r, a.dt);
                    a.f_out.ptr[cell + var * fvs] = q[var];
                }
                store_prims(a, q, dX, dY, z);
                if (more) {   // own cell of the next plane; fb[b^1] was last read by this thread
                    issue_fcell(a, fb + (b ^ 1) * 15 * BXY, BXY, dcol, cell + fps, fvs, krk);
                    cp_async_commit();
                }
            }
        } else {
            for (int t = tid; t < 5 * BXY; t += NT) {
                const int var = t / BXY, col = t - var * BXY;
                const int xx = col % BX, yy = col / BX;
                const int X = x0 + xx, Y = y0 + yy;
                if (X < a.ex && Y < a.ey) {
                    const double* px = fx + (var * BY + yy) * (BX + 1) + xx;
                    const double* py = fy + (var * (BY + 1) + yy) * BX + xx;
                    const double dfx = px[1] - px[0];
                    const double dfy = py[BX] - py[0];
                    const double dfz = fz[cur * 5 * BXY + t] - fz[prev * 5 * BXY + t];
                    double r = dfx * a.rhx;
                    r = fma(dfy, a.rhy, r);
                    r = fma(dfz, a.rhz, r);
                    const double J = UNI ? 1.0 : ldg_met(a, 9, X, Y, z);
                    a.du[(size_t)(X - a.sx) +
                         (size_t)a.du_pitch *
                             ((size_t)(Y - a.sy) +
                              (size_t)a.du_ly * ((size_t)(z - a.sz) + (size_t)a.du_lz * var))] =
                        -J * r;
                }
            }
        }
        prev = cur;
    }
    return true;
}

// One sweep.  In the kernels compiled for grids with CLOSURE faces (CLO),
// tiles that touch one (the x faces within 4 of a CLOSURE x face, the y
// faces within 4 of a CLOSURE y face) run the variant with the closure face
// values and all others the plain one; grids without CLOSURE faces run
// kernels that hold only the plain sweep.
template <int BX, int BY, int NT, bool UNI, typename CT, bool EPI, bool GMAP, bool CLO>
__device__ __forceinline__ bool run_sweep(const RhsArgs& a, const SplitK<CT>& k,
                                          unsigned char* smem, int x0, int y0, int z0, int z1,
                                          int krk, uint64_t* bar, uint32_t& ph, bool& first) {
    if (CLO) {
        const int fx0 = x0 - 4, fy0 = y0 - 4;    // first face of the tile in x and y
        const bool clo = (a.clo[0] && fx0 <= 3) || (a.clo[1] && fx0 + BX >= a.nx - 3) ||
                         (a.clo[2] && fy0 <= 3) || (a.clo[3] && fy0 + BY >= a.ny - 3);
        if (clo)
            return sweep<BX, BY, NT, UNI, CT, EPI, GMAP, true>(a, k, smem, x0, y0, z0, z1, krk,
                                                               bar, ph, first);
    }
    return sweep<BX, BY, NT, UNI, CT, EPI, GMAP, false>(a, k, smem, x0, y0, z0, z1, krk, bar, ph,
                                                        first);
}

// mbarriers of the two staging buffers (TMA path) and one nothing arrives on
// (the failure-path test waits on it), set up once per CTA
__device__ __forceinline__ void init_stage_barriers(uint64_t* bar) {
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init(&bar[2], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
}

template <int BX, int BY, int NT, bool UNI, typename CT, bool EPI, bool CLO>
__global__ void __launch_bounds__(NT, (RhsLayout<BX, BY, CT, EPI>::MINB))
    bf3w_rhs_kernel(const __grid_constant__ RhsArgs a, int krk) {
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    // TMA tile destinations must be 128-byte aligned: align explicitly (the
    // launch adds 128 bytes of slack)
    unsigned char* smem_raw = smem_dyn + ((128 - (smem_addr(smem_dyn) & 127)) & 127);
    __shared__ uint64_t bar[3];
    init_stage_barriers(bar);
    uint32_t ph = 0;
    bool first = true;
    const SplitK<CT> k = {CT(a.eps2), CT(a.hrg), CT(a.c1), CT(a.c3), CT(a.gm1)};
    const int G = gridDim.x, b = blockIdx.x;
    const long nzj = a.ez - a.sz;
    const int ntile = a.ntx * a.nty;
    // 1) whole-column sweeps, round robin: the CTAs running together sweep
    //    neighbouring tiles at the same z, so the halo re-reads hit L2
    const int full = ntile / G;
    for (int r = 0; r < full; ++r) {
        const int tile = b + r * G;
        const int x0 = a.sx + (tile % a.ntx) * BX, y0 = a.sy + (tile / a.ntx) * BY;
        for (int z = a.sz; z < a.ez; z += a.zc)
            if (!run_sweep<BX, BY, NT, UNI, CT, EPI, false, CLO>(a, k, smem_raw, x0, y0, z,
                                                        min(z + a.zc, a.ez), krk, bar, ph,
                                                        first))
                return;
    }
    // 2) the remaining tiles' (tile, plane) space cut into equal ranges
    const long total = (long)(ntile - full * G) * nzj;
    const long lo = total * b / G, hi = total * (b + 1) / G;
    long pos = lo;
    while (pos < hi) {
        const long tr = pos / nzj;
        const int zoff = (int)(pos - tr * nzj);
        const int len = (int)min(min(nzj - zoff, hi - pos), (long)a.zc);
        const int tile = full * G + (int)tr;
        if (!run_sweep<BX, BY, NT, UNI, CT, EPI, false, CLO>(a, k, smem_raw, a.sx + (tile % a.ntx) * BX,
                                                    a.sy + (tile / a.ntx) * BY, a.sz + zoff,
                                                    a.sz + zoff + len, krk, bar, ph, first))
            return;
        pos += len;
    }
}

// Batched form: one persistent launch over many grids.  The work is a list of
// items {grid, tile, first plane, end plane} (z runs of at most the scan
// length), longest first; each CTA takes the next item through an atomic
// counter (zeroed before the launch), so the long runs start early and the
// short ones fill in at the end.
template <int BX, int BY, int NT, bool UNI, typename CT, bool EPI, bool CLO>
__global__ void __launch_bounds__(NT, (RhsLayout<BX, BY, CT, EPI>::MINB))
    bf3w_rhs_batch_kernel(const RhsArgs* __restrict__ grids, const int4* __restrict__ items,
                          int nitems, unsigned* __restrict__ counter, int krk) {
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    // TMA tile destinations must be 128-byte aligned: align explicitly (the
    // launch adds 128 bytes of slack)
    unsigned char* smem_raw = smem_dyn + ((128 - (smem_addr(smem_dyn) & 127)) & 127);
    __shared__ uint64_t bar[3];
    __shared__ int next;
    init_stage_barriers(bar);
    uint32_t ph = 0;
    int fenced = -1;                  // grid whose tensor maps this CTA has fenced
    for (;;) {
        if (threadIdx.x == 0) next = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int it = next;
        __syncthreads();              // every thread has read `next`
        if (it >= nitems) return;
        const int4 w = items[it];
        const RhsArgs& a = grids[w.x];
        const SplitK<CT> k = {CT(a.eps2), CT(a.hrg), CT(a.c1), CT(a.c3), CT(a.gm1)};
        bool first = fenced != w.x;
        fenced = w.x;
        if (!run_sweep<BX, BY, NT, UNI, CT, EPI, true, CLO>(a, k, smem_raw,
                                                           a.sx + (w.y % a.ntx) * BX,
                                                           a.sy + (w.y / a.ntx) * BY, w.z, w.w,
                                                           krk, bar, ph, first))
            return;
    }
}

// ---------------------------------------------------------------------------
// Compiled tile shapes and per-slice launchers
// ---------------------------------------------------------------------------
inline constexpr TileCfg kCfgs[] = {{16, 8, 768}, {16, 8, 704}, {8, 8, 256}, {8, 8, 384}};
inline constexpr int kNumCfgs = sizeof(kCfgs) / sizeof(kCfgs[0]);

template <int BX, int BY, int NT, bool UNI, typename CT, bool EPI, bool CLO>
struct Launcher {
    static size_t smem() { return RhsLayout<BX, BY, CT, EPI>::smem_bytes + 128; }
    // attributes set and resident CTA count computed once per device
    static int max_ctas() {
        static int cached[64] = {0};
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
        if (cached[dev] > 0) return cached[dev];
        int sms = 0, per = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return 0;
        if (cudaFuncSetAttribute(bf3w_rhs_kernel<BX, BY, NT, UNI, CT, EPI, CLO>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem()) != cudaSuccess ||
            cudaFuncSetAttribute(bf3w_rhs_batch_kernel<BX, BY, NT, UNI, CT, EPI, CLO>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem()) != cudaSuccess)
            return 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per, bf3w_rhs_kernel<BX, BY, NT, UNI, CT, EPI, CLO>, NT, smem()) !=
            cudaSuccess)
            return 0;
        cached[dev] = sms * per;
        return cached[dev];
    }
    static int launch(const RhsArgs& a, int ctas, int krk, cudaStream_t st) {
        if (max_ctas() <= 0) return fail(WS_ERR_CUDA, "cannot prepare the RHS kernel");
        bf3w_rhs_kernel<BX, BY, NT, UNI, CT, EPI, CLO><<<ctas, NT, smem(), st>>>(a, krk);
        WS_CUDA(cudaGetLastError());
        return WS_OK;
    }
    static int launch_batch(const RhsArgs* grids, const BatchWork& w, int ctas, int krk,
                            cudaStream_t st) {
        if (max_ctas() <= 0) return fail(WS_ERR_CUDA, "cannot prepare the RHS kernel");
        WS_CUDA(cudaMemsetAsync(w.counter, 0, sizeof(unsigned), st));
        bf3w_rhs_batch_kernel<BX, BY, NT, UNI, CT, EPI, CLO>
            <<<ctas, NT, smem(), st>>>(grids, w.items, w.nitems, w.counter, krk);
        WS_CUDA(cudaGetLastError());
        return WS_OK;
    }
};

// One (precision, closure) slice of the kernels over every compiled tile
// shape; explicitly instantiated by its own translation unit.  The stage
// epilogue is compiled for Cartesian grids only (solver, batches).
template <typename CT, bool CLO>
struct RhsSlice {
    template <int BX, int BY, int NT>
    static int launch_t(const RhsArgs& a, bool uni, int ctas, int krk, cudaStream_t st) {
        if (krk > 0) {
            if (!uni) return fail(WS_ERR_UNSUPPORTED, "stage epilogue needs Cartesian metrics");
            return Launcher<BX, BY, NT, true, CT, true, CLO>::launch(a, ctas, krk, st);
        }
        return uni ? Launcher<BX, BY, NT, true, CT, false, CLO>::launch(a, ctas, 0, st)
                   : Launcher<BX, BY, NT, false, CT, false, CLO>::launch(a, ctas, 0, st);
    }
    template <int BX, int BY, int NT>
    static int batch_t(const RhsArgs* g, const BatchWork& w, bool uni, int ctas, int krk,
                       cudaStream_t st) {
        if (krk > 0) {
            if (!uni) return fail(WS_ERR_UNSUPPORTED, "stage epilogue needs Cartesian metrics");
            return Launcher<BX, BY, NT, true, CT, true, CLO>::launch_batch(g, w, ctas, krk, st);
        }
        return uni ? Launcher<BX, BY, NT, true, CT, false, CLO>::launch_batch(g, w, ctas, 0, st)
                   : Launcher<BX, BY, NT, false, CT, false, CLO>::launch_batch(g, w, ctas, 0, st);
    }
    template <int BX, int BY, int NT>
    static int max_t(bool uni, bool stage) {
        if (stage) return Launcher<BX, BY, NT, true, CT, true, CLO>::max_ctas();
        return uni ? Launcher<BX, BY, NT, true, CT, false, CLO>::max_ctas()
                   : Launcher<BX, BY, NT, false, CT, false, CLO>::max_ctas();
    }

    static int launch(int cfg, const RhsArgs& a, bool uni, int ctas, int krk, cudaStream_t st);
    static int launch_batch(int cfg, const RhsArgs* g, const BatchWork& w, bool uni, int ctas,
                            int krk, cudaStream_t st);
    static int max_ctas(int cfg, bool uni, bool stage);
};

template <typename CT, bool CLO>
int RhsSlice<CT, CLO>::launch(int cfg, const RhsArgs& a, bool uni, int ctas, int krk,
                              cudaStream_t st) {
    switch (cfg) {
        case 0: return launch_t<16, 8, 768>(a, uni, ctas, krk, st);
        case 1: return launch_t<16, 8, 704>(a, uni, ctas, krk, st);
        case 2: return launch_t<8, 8, 256>(a, uni, ctas, krk, st);
        case 3: return launch_t<8, 8, 384>(a, uni, ctas, krk, st);
        default: return fail(WS_ERR_INVALID, "unknown tile configuration");
    }
}
template <typename CT, bool CLO>
int RhsSlice<CT, CLO>::launch_batch(int cfg, const RhsArgs* g, const BatchWork& w, bool uni,
                                    int ctas, int krk, cudaStream_t st) {
    switch (cfg) {
        case 0: return batch_t<16, 8, 768>(g, w, uni, ctas, krk, st);
        case 1: return batch_t<16, 8, 704>(g, w, uni, ctas, krk, st);
        case 2: return batch_t<8, 8, 256>(g, w, uni, ctas, krk, st);
        case 3: return batch_t<8, 8, 384>(g, w, uni, ctas, krk, st);
        default: return fail(WS_ERR_INVALID, "unknown tile configuration");
    }
}
template <typename CT, bool CLO>
int RhsSlice<CT, CLO>::max_ctas(int cfg, bool uni, bool stage) {
    switch (cfg) {
        case 0: return max_t<16, 8, 768>(uni, stage);
        case 1: return max_t<16, 8, 704>(uni, stage);
        case 2: return max_t<8, 8, 256>(uni, stage);
        case 3: return max_t<8, 8, 384>(uni, stage);
        default: return 0;
    }
}

// each slice is compiled by its own translation unit only
extern template struct RhsSlice<double, false>;
extern template struct RhsSlice<double, true>;
extern template struct RhsSlice<float, false>;
extern template struct RhsSlice<float, true>;

}  // namespace ws
