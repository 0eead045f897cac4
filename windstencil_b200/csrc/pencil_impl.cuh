// pencil_impl.cuh -- BF3W inviscid RHS as three barrier-free line passes.
//
// Replaces, like the fused kernel (bf3w_rhs_impl.cuh), the reference's
// split_Jac3d_Stager_Warming_ker (src/kernels/OCFD_split.cpp:36-3918) and
// its boundary-ring kernel (src/solver/OCFD_NS_Jacobian3d.cpp:828-2530), with
// the same per-point arithmetic (ws_device.cuh).  The fused kernel sweeps a
// 2D column footprint along z with CTA barriers between its split and face
// intervals and recomputes the footprint's halo splits and edge faces.  Here
// every lane owns one grid line along the pass direction and marches it
// alone: per point it computes the Steger-Warming split of the point four
// ahead into a private 8-slot ring in shared memory, reconstructs the face
// above the current point from the ring (WENO7-SYMBO P and M), and adds the
// face difference of the point to du.  No lane reads another lane's ring, so
// there is no barrier and no halo work across lines; a warp's lanes own 32
// consecutive lines of the flattened pair of the other two axes, so there
// are no partial tiles, and each warp takes an equal contiguous share of the
// (line group, position) space.  The primitives of the next split and the
// du of the next point are loaded a step ahead, so that their latency
// overlaps the current step's reconstructions.
//
// A RHS is three passes, x (du =, or += onto viscous terms already stored in
// du), y (+=) and z (+=, or in stage mode the SSP-RK3 stage update and the
// primitives of the new state, as the fused kernel's epilogue).  du goes
// through HBM between the passes, which the compute-bound passes absorb
// (~320 B/cell against ~7.3 kFLOP/cell).
#pragma once
#include <type_traits>

#include "bf3w_rhs_impl.cuh"

namespace ws {

template <typename CT>
struct PencilLayout {
    static constexpr int RS = 10 * 32;            // ring slot stride (CT), lanes inner
    static constexpr int WARP = 8 * RS;           // one warp's ring
};

enum PencilMode { P_STORE = 0, P_ADD = 1, P_STAGE = 2 };

// Face value of variable v of face f (direction of n cells, CLOSURE flags lo /
// hi, ydir: the y forms) from a lane's ring column `col` of ns slots (slot
// stride 10 x 32, the stencil from slot s0 on): the closure value next to a
// CLOSURE face, the WENO7 value elsewhere.  Not inlined: the steps near the
// line ends call it, and one copy keeps the march loops' code within the
// instruction cache (inlined into those steps, the closure code doubled the
// y pass's time through instruction fetch stalls).
template <typename CT>
__device__ __noinline__ double pencil_closure_face(const CT* col, int s0, int ns, int v, int f,
                                                   int n, int lo, int hi, bool ydir) {
    constexpr int RS = 10 * 32;
    if (closure_face(f, n, lo, hi)) {
        double sp[8], sm[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int sk = s0 + k < ns ? s0 + k : s0 + k - ns;
            const CT* e = col + sk * RS;
            sp[k] = (double)e[v * 32];
            sm[k] = (double)e[(5 + v) * 32];
        }
        return closure_value_arr(sp, sm, f, n, lo, hi, ydir);
    }
    return face_flux<CT, true>(col + s0 * RS + v * 32, 5 * 32, RS, ns - s0, ns * RS);
}

// March length, first LAP position and line count of pass DIR over the job
// of `a`; the pass's work is its line groups (32 lines) x positions.
template <int DIR>
__device__ __forceinline__ long pencil_work(const RhsArgs& a, int& L) {
    const int nxj = a.ex - a.sx, nyj = a.ey - a.sy, nzj = a.ez - a.sz;
    L = DIR == 0 ? nxj : (DIR == 1 ? nyj : nzj);
    const long NL = DIR == 0 ? (long)nyj * nzj : (DIR == 1 ? (long)nxj * nzj : (long)nxj * nyj);
    return (NL + 31) / 32 * L;
}

// One segment of pass DIR (0 x, 1 y, 2 z): positions p0 .. p0+len-1 of the
// lines of group grp of the job of `a`, this lane's line marched with the
// lane's ring column `ring`.  CLO (y pass): faces next to a CLOSURE face of
// the grid (a.clo) take the closure rules of closure_value_arr; the lanes of
// a warp sit at the same y, so the branch is uniform.
template <int DIR, typename CT, bool UNI, int MODE, bool CLO = false>
__device__ __forceinline__ void pencil_segment(const RhsArgs& a, int krk, CT* ring, long grp,
                                               int p0, int len) {
    static_assert(MODE != P_STAGE || (DIR == 2 && UNI), "stage update: z pass, Cartesian");
    static_assert(!CLO || DIR == 1, "closure faces: y pass (the x pass is pencil_x_segment)");
    constexpr bool ADD = MODE != P_STORE;
    using P = PencilLayout<CT>;
    const int lane = threadIdx.x & 31;
    const SplitK<CT> k = {CT(a.eps2), CT(a.hrg), CT(a.c1), CT(a.c3), CT(a.gm1)};
    const int nxj = a.ex - a.sx, nyj = a.ey - a.sy, nzj = a.ez - a.sz;
    const int n1 = DIR == 0 ? nyj : nxj;              // fastest line axis
    const long NL = (long)n1 * (DIR == 2 ? nyj : nzj);
    const int m0 = DIR == 0 ? a.sx : (DIR == 1 ? a.sy : a.sz);
    const int mlast = (DIR == 0 ? a.nx : (DIR == 1 ? a.ny : a.nz)) + 7;   // last LAP index
    const double rh = DIR == 0 ? a.rhx : (DIR == 1 ? a.rhy : a.rhz);
    const size_t vs = (size_t)a.du_pitch * a.du_ly * a.du_lz;            // du variable stride
    const size_t fvs = MODE == P_STAGE ? (size_t)a.fn.pitch * a.fn.length_Y * a.fn.length_Z : 0;
    long l = grp * 32 + lane;
    const bool valid = l < NL;
    if (!valid) l = NL - 1;
    const int c1 = (int)(l % n1), c2 = (int)(l / n1);
    // LAP coordinates of march position m on this lane's line
    auto X = [&](int m) { return DIR == 0 ? m : a.sx + c1; };
    auto Y = [&](int m) { return DIR == 1 ? m : (DIR == 0 ? a.sy + c1 : a.sy + c2); };
    auto Z = [&](int m) { return DIR == 2 ? m : a.sz + c2; };
    auto load = [&](int m, double q[5]) {
        const int x = X(m), y = Y(m), z = Z(m);
#pragma unroll
        for (int f = 0; f < 5; ++f) q[f] = ldg_prim(a, f, x, y, z);
    };
    auto split_into = [&](int m, const double q[5]) {
        const int x = X(m), y = Y(m), z = Z(m);
        CT out[10];
        split_point<DIR, UNI, CT>(a, k, q[0], q[1], q[2], q[3], q[4], x, y, z, out);
        CT* dst = ring + (m & 7) * P::RS;
#pragma unroll
        for (int c = 0; c < 10; ++c) dst[c * 32] = out[c];
    };
    // du offset of march position m (job-relative); in stage mode the
    // conserved state has du's shape, offset by the interior origin
    auto du_at = [&](int m) {
        return (size_t)(X(m) - a.sx) +
               (size_t)a.du_pitch * ((size_t)(Y(m) - a.sy) + (size_t)a.du_ly * (size_t)(Z(m) - a.sz));
    };
    auto f_at = [&](int m) { return soa_index(a.fn, X(m) - 4, Y(m) - 4, Z(m) - 4, 0); };
    // face value of variable v above march position m (ring stencil from
    // slot s0 = (m - 3) & 7; face index m - 3 of the direction); the
    // closure test is compiled only into the steps of the closure zones
    const bool clo = CLO && (a.clo[2] | a.clo[3]);
    auto face = [&](int s0, int m, int v, auto cl) -> double {
        if constexpr (decltype(cl)::value)
            return pencil_closure_face<CT>(ring, s0, 8, v, m - 3, a.ny, a.clo[2], a.clo[3], true);
        else
            return face_flux<CT, true>(ring + s0 * P::RS + v * 32, 5 * 32, P::RS, 8 - s0,
                                       8 * P::RS);
    };

    const int ms = m0 + p0;
    for (int m = ms - 4; m < ms + 4; ++m) {
        double q[5];
        load(m, q);
        split_into(m, q);
    }
    double qn[5], dn[5], fnn[5], fin[5];
    load(ms + 4, qn);
    auto load_cell = [&](int m) {      // du (and the stage operands) of point m
        if (ADD) {
            const size_t o = du_at(m);
#pragma unroll
            for (int v = 0; v < 5; ++v) dn[v] = a.du[o + v * vs];
        }
        if (MODE == P_STAGE) {
            const size_t o = f_at(m);
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                fnn[v] = __ldg(a.fn.ptr + o + v * fvs);
                fin[v] = krk == 1 ? 0.0 : a.f_in.ptr[o + v * fvs];
            }
        }
    };
    if (valid) load_cell(ms);
    double fprev[5];
    {
        const int s0 = (ms - 4) & 7;
#pragma unroll
        for (int v = 0; v < 5; ++v)
            fprev[v] = face(s0, ms - 1, v, std::integral_constant<bool, CLO>{});
    }
    auto step = [&](int m, auto cl) {
        double q[5], dc[5], fnc[5], fic[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            q[f] = qn[f];
            dc[f] = dn[f];
            fnc[f] = fnn[f];
            fic[f] = fin[f];
        }
        load(min(m + 5, mlast), qn);
        if (valid && m + 1 < ms + len) load_cell(m + 1);
        split_into(m + 4, q);
        const int s0 = (m - 3) & 7;
        const double J = UNI ? 1.0 : ldg_met(a, 9, X(m), Y(m), Z(m));
        double r[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double fc = face(s0, m, v, cl);
            r[v] = -J * ((fc - fprev[v]) * rh);
            fprev[v] = fc;
        }
        if (!valid) return;
        if (MODE == P_STAGE) {
            const size_t o = f_at(m);
            double qs[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                qs[v] = ws_rk_stage(krk, fnc[v], fic[v], dc[v] + r[v], a.dt);
                a.f_out.ptr[o + v * fvs] = qs[v];
            }
            store_prims(a, qs, X(m), Y(m), Z(m));
        } else {
            const size_t o = du_at(m);
#pragma unroll
            for (int v = 0; v < 5; ++v) a.du[o + v * vs] = ADD ? dc[v] + r[v] : r[v];
        }
    };
    // closure zones: faces m - 3 <= 3 next to the low face, m - 3 >= n - 3
    // next to the high face (LAP positions m <= 6 and m >= n)
    const int me = ms + len;
    int z1 = ms, z2 = me;
    if (clo) {
        z1 = a.clo[2] ? max(ms, min(7, me)) : ms;
        z2 = a.clo[3] ? max(z1, min(a.ny, me)) : me;
    }
    int m = ms;
    if constexpr (CLO)
        for (; m < z1; ++m) step(m, std::true_type{});
    for (; m < z2; ++m) step(m, std::false_type{});
    if constexpr (CLO)
        for (; m < me; ++m) step(m, std::true_type{});
}

// One pass along DIR over the job of `a`: every warp takes an equal
// contiguous share of the (line group, position) space.
template <int DIR, int WPB, typename CT, bool UNI, int MODE, bool CLO = false>
__global__ void __launch_bounds__(WPB * 32, 1)
    pencil_rhs_kernel(const __grid_constant__ RhsArgs a, int krk) {
    using P = PencilLayout<CT>;
    extern __shared__ __align__(16) unsigned char pencil_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    CT* ring = reinterpret_cast<CT*>(pencil_smem) + warp * P::WARP + lane;
    int L = 0;
    const long total = pencil_work<DIR>(a, L);
    const long S = (long)gridDim.x * WPB, s = (long)blockIdx.x * WPB + warp;
    long pos = total * s / S;
    const long end = total * (s + 1) / S;
    while (pos < end) {
        const long grp = pos / L;
        const int p0 = (int)(pos - grp * L);
        const int len = (int)min((long)(L - p0), end - pos);
        pencil_segment<DIR, CT, UNI, MODE, CLO>(a, krk, ring, grp, p0, len);
        pos += len;
    }
}

// The same pass over the grids of a batch: argument table `grids`, and
// woff[i] the pass's work before grid i (woff[n] the total).  A warp's share
// may cross grids.
template <int DIR, int WPB, typename CT, int MODE, bool CLO = false>
__global__ void __launch_bounds__(WPB * 32, 1)
    pencil_batch_kernel(const RhsArgs* __restrict__ grids, const long* __restrict__ woff, int n,
                        int krk) {
    using P = PencilLayout<CT>;
    extern __shared__ __align__(16) unsigned char pencil_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    CT* ring = reinterpret_cast<CT*>(pencil_smem) + warp * P::WARP + lane;
    const long total = woff[n];
    const long S = (long)gridDim.x * WPB, s = (long)blockIdx.x * WPB + warp;
    long pos = total * s / S;
    const long end = total * (s + 1) / S;
    int lo = 0, hi = n;                    // the grid holding pos: woff[i] <= pos < woff[i+1]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (woff[mid] <= pos) lo = mid; else hi = mid;
    }
    int i = lo;
    while (pos < end) {
        while (woff[i + 1] <= pos) ++i;
        const RhsArgs& a = grids[i];
        int L = 0;
        pencil_work<DIR>(a, L);
        const long local = pos - woff[i];
        const long grp = local / L;
        const int p0 = (int)(local - grp * L);
        const int len = (int)min((long)(L - p0), end - pos);
        pencil_segment<DIR, CT, true, MODE, CLO>(a, krk, ring, grp, p0, len);
        pos += len;
    }
}

// The x pass, cooperative.  In the other passes a warp's 32 lines are
// consecutive in x, so the per-lane loads and du stores coalesce; in the x
// pass they are 32 consecutive y, and per lane every access is a separate
// L1 transaction (measured: MIO-throttle-bound, 3x the y pass's time in the
// mixed form).  Here the lanes still own their lines and reconstruct their
// own faces, but the loads and splits of the next C points of all 32 lines,
// and the stores of C points of du, are done by the warp together: lane
// (xi, yi) = (lane % C, lane / C) takes point xi of lines yi + r (32 / C),
// r < C, so each access covers 32 / C lines x C consecutive x.  A split is
// then written into the owning lane's ring column, so the ring holds 8 + C
// slots (a chunk of C faces spans 7 + C stencil points).  C = 4 for the
// mixed form; C = 2 for FP64, whose larger ring must leave room for 8 warps.
template <typename CT, int C_>
struct PencilXLayout {
    static constexpr int C = C_;                  // points per chunk (and lanes per line row)
    static constexpr int SLOTS = 8 + C;           // a chunk's 8-point stencils span 7 + C points
    static constexpr int RS = 10 * 32;
    static constexpr int RING = SLOTS * RS;       // CT
    static constexpr int DUS = 5 * C * 32;        // du staging, doubles
    static constexpr size_t WARP_BYTES = RING * sizeof(CT) + DUS * sizeof(double);
};
// chunk of the cooperative x pass: 4 for the mixed form, 2 for FP64 (whose
// ring is twice as large; 8 warps per CTA then still fit)
template <typename CT>
constexpr int pencil_x_chunk() { return sizeof(CT) == 4 ? 4 : 2; }

// One segment of the cooperative x pass (positions p0 .. p0+len-1 of the 32
// lines of group grp); wbase: the warp's ring and du staging.  CLO: faces
// next to a CLOSURE x face take the closure rules (uniform across the warp,
// whose lanes march the same x).
template <typename CT, bool UNI, int MODE, bool CLO = false>
__device__ __forceinline__ void pencil_x_segment(const RhsArgs& a, unsigned char* wbase,
                                                 long grp, int p0, int len) {
    static_assert(MODE != P_STAGE, "the x pass never applies the stage");
    constexpr bool ADD = MODE == P_ADD;
    using P = PencilXLayout<CT, pencil_x_chunk<CT>()>;
    constexpr int C = P::C, NS = P::SLOTS, LR = 32 / C;   // lines per load round
    const int lane = threadIdx.x & 31;
    CT* ringw = reinterpret_cast<CT*>(wbase);                       // [12][10][32]
    double* dus = reinterpret_cast<double*>(wbase + P::RING * sizeof(CT));   // [5][C][32]
    CT* ring = ringw + lane;                                        // this lane's column
    const SplitK<CT> k = {CT(a.eps2), CT(a.hrg), CT(a.c1), CT(a.c3), CT(a.gm1)};
    const int nyj = a.ey - a.sy, nzj = a.ez - a.sz;
    const int mlast = a.nx + 7;
    const size_t vs = (size_t)a.du_pitch * a.du_ly * a.du_lz;
    const long NL = (long)nyj * nzj;
    const int xi = lane % C, yi = lane / C;
    // this lane's own line, and the C lines it loads / stores for
    const long lo = min(grp * 32 + lane, NL - 1);
    const bool valid = grp * 32 + lane < NL;
    const int oy = a.sy + (int)(lo % nyj), oz = a.sz + (int)(lo / nyj);
    int cy[C], cz[C];
    bool cv[C];
#pragma unroll
    for (int r = 0; r < C; ++r) {
        const long l = grp * 32 + yi + LR * r;
        cv[r] = l < NL;
        const long lc = min(l, NL - 1);
        cy[r] = a.sy + (int)(lc % nyj);
        cz[r] = a.sz + (int)(lc / nyj);
    }
    // primitives of point x0 + xi of the C lines (x clamped), and their
    // splits into the owning lanes' ring columns (only xi < cnt)
    auto coop_load = [&](int x0, double q[C][5]) {
        const int x = min(x0 + xi, mlast);
#pragma unroll
        for (int r = 0; r < C; ++r)
#pragma unroll
            for (int f = 0; f < 5; ++f) q[r][f] = ldg_prim(a, f, x, cy[r], cz[r]);
    };
    auto coop_split = [&](int x0, int cnt, const double q[C][5]) {
        if (xi >= cnt) return;
        const int x = x0 + xi;
#pragma unroll
        for (int r = 0; r < C; ++r) {
            CT out[10];
            split_point<0, UNI, CT>(a, k, q[r][0], q[r][1], q[r][2], q[r][3], q[r][4], x,
                                    cy[r], cz[r], out);
            CT* dst = ringw + (x % NS) * P::RS + yi + LR * r;
#pragma unroll
            for (int c = 0; c < 10; ++c) dst[c * 32] = out[c];
        }
    };
    const bool clo = CLO && (a.clo[0] | a.clo[1]);
    // face value of variable v above point m (stencil from ring slot s0);
    // the closure test is compiled only into the chunks of the closure zones
    auto face = [&](int s0, int m, int v, auto cl) -> double {
        if constexpr (decltype(cl)::value)
            return pencil_closure_face<CT>(ring, s0, NS, v, m - 3, a.nx, a.clo[0], a.clo[1],
                                           false);
        else
            return face_flux<CT, true>(ring + s0 * P::RS + v * 32, 5 * 32, P::RS, NS - s0,
                                       NS * P::RS);
    };
    const int ms = a.sx + p0;
    double qb[C][5];
    for (int p = ms - 4; p < ms + 4; p += C) {   // the first 8 points
        coop_load(p, qb);
        coop_split(p, C, qb);
    }
    coop_load(ms + 4, qb);              // the first chunk's new points
    __syncwarp();
    double fprev[5];
    {
        const int s0 = (ms - 4) % NS;
#pragma unroll
        for (int v = 0; v < 5; ++v)
            fprev[v] = face(s0, ms - 1, v, std::integral_constant<bool, CLO>{});
    }
    // faces of this lane's line, steps mc .. mc+cnt-1, into the staging
    auto faces = [&](int mc, int cnt, auto cl) {
        for (int i = 0; i < cnt; ++i) {
            const int m = mc + i;
            const int s0 = (m - 3) % NS;
            const double J = UNI ? 1.0 : ldg_met(a, 9, m, oy, oz);
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                const double fc = face(s0, m, v, cl);
                dus[(v * C + i) * 32 + lane] = -J * ((fc - fprev[v]) * a.rhx);
                fprev[v] = fc;
            }
        }
    };
    for (int mc = ms; mc < ms + len; mc += C) {
        const int cnt = min(C, ms + len - mc);
        coop_split(mc + 4, cnt, qb);     // points mc+4 .. (slots of mc-4-C ..: dead)
        __syncwarp();
        if (mc + C < ms + len) coop_load(mc + C + 4, qb);
        // closure zones: faces m - 3 <= 3 (LAP m <= 6) next to the low x face,
        // m - 3 >= n - 3 (m >= n) next to the high one
        if constexpr (CLO) {
            if (clo && ((a.clo[0] && mc <= 6) || (a.clo[1] && mc + cnt - 1 >= a.nx)))
                faces(mc, cnt, std::true_type{});
            else
                faces(mc, cnt, std::false_type{});
        } else {
            faces(mc, cnt, std::false_type{});
        }
        __syncwarp();
        // du of the chunk: point mc + xi of lines yi + LR r
        if (xi < cnt) {
            const int x = mc + xi;
#pragma unroll
            for (int r = 0; r < C; ++r) {
                if (!cv[r]) continue;
                const size_t o = (size_t)(x - a.sx) +
                                 (size_t)a.du_pitch * ((size_t)(cy[r] - a.sy) +
                                                       (size_t)a.du_ly * (size_t)(cz[r] - a.sz));
#pragma unroll
                for (int v = 0; v < 5; ++v) {
                    const double r_ = dus[(v * C + xi) * 32 + yi + LR * r];
                    double* p = a.du + o + v * vs;
                    *p = ADD ? *p + r_ : r_;
                }
            }
        }
        (void)valid;
    }
    __syncwarp();
}

template <int WPB, typename CT, bool UNI, int MODE, bool CLO = false>
__global__ void __launch_bounds__(WPB * 32, 1)
    pencil_x_coop_kernel(const __grid_constant__ RhsArgs a) {
    extern __shared__ __align__(16) unsigned char pencil_smem[];
    const int warp = threadIdx.x >> 5;
    unsigned char* wbase = pencil_smem + warp * PencilXLayout<CT, pencil_x_chunk<CT>()>::WARP_BYTES;
    int L = 0;
    const long total = pencil_work<0>(a, L);
    const long S = (long)gridDim.x * WPB, s = (long)blockIdx.x * WPB + warp;
    long pos = total * s / S;
    const long end = total * (s + 1) / S;
    while (pos < end) {
        const long grp = pos / L;
        const int p0 = (int)(pos - grp * L);
        const int len = (int)min((long)(L - p0), end - pos);
        pencil_x_segment<CT, UNI, MODE, CLO>(a, wbase, grp, p0, len);
        pos += len;
    }
}

template <int WPB, typename CT, int MODE, bool CLO = false>
__global__ void __launch_bounds__(WPB * 32, 1)
    pencil_x_coop_batch_kernel(const RhsArgs* __restrict__ grids, const long* __restrict__ woff,
                               int n) {
    extern __shared__ __align__(16) unsigned char pencil_smem[];
    const int warp = threadIdx.x >> 5;
    unsigned char* wbase = pencil_smem + warp * PencilXLayout<CT, pencil_x_chunk<CT>()>::WARP_BYTES;
    const long total = woff[n];
    const long S = (long)gridDim.x * WPB, s = (long)blockIdx.x * WPB + warp;
    long pos = total * s / S;
    const long end = total * (s + 1) / S;
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (woff[mid] <= pos) lo = mid; else hi = mid;
    }
    int i = lo;
    while (pos < end) {
        while (woff[i + 1] <= pos) ++i;
        const RhsArgs& a = grids[i];
        int L = 0;
        pencil_work<0>(a, L);
        const long local = pos - woff[i];
        const long grp = local / L;
        const int p0 = (int)(local - grp * L);
        const int len = (int)min((long)(L - p0), end - pos);
        pencil_x_segment<CT, true, MODE, CLO>(a, wbase, grp, p0, len);
        pos += len;
    }
}

// Launch of a persistent line-pass kernel, one CTA per SM; the dynamic
// shared memory size is set and the SM count read once per device per kernel.
template <typename Kern, typename... Args>
int pencil_launch(Kern kern, int* blocks, int threads, size_t smem, cudaStream_t st,
                  Args... args) {
    int dev = 0;
    WS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(WS_ERR_UNSUPPORTED, "device ordinal >= 64");
    if (!blocks[dev]) {
        int sms = 0;
        WS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        WS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
        blocks[dev] = sms;
    }
    kern<<<blocks[dev], threads, smem, st>>>(args...);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
}

template <int WPB, typename CT, bool UNI>
struct PencilLauncher {
    static constexpr size_t SMEM = (size_t)WPB * PencilLayout<CT>::WARP * sizeof(CT);
    static constexpr int XW = 8;                       // warps of the cooperative x pass
    static constexpr size_t XSMEM = XW * PencilXLayout<CT, pencil_x_chunk<CT>()>::WARP_BYTES;
    // the stage pass holds more operands than the other passes: the mixed
    // form's runs with 12 warps (16 leave 128 registers), the FP64 one with 8
    static constexpr int SW = sizeof(CT) == 4 ? (WPB > 12 ? 12 : WPB) : (WPB > 8 ? 8 : WPB);
    static constexpr size_t SSMEM = (size_t)SW * PencilLayout<CT>::WARP * sizeof(CT);

    // one grid (job of a)
    template <int DIR, int MODE, bool CLO = false>
    static int one(const RhsArgs& a, int krk, cudaStream_t st) {
        constexpr int W = MODE == P_STAGE ? SW : WPB;
        static int blocks[64] = {0};
        return pencil_launch(pencil_rhs_kernel<DIR, W, CT, UNI, MODE, CLO>, blocks, W * 32,
                             MODE == P_STAGE ? SSMEM : SMEM, st, a, krk);
    }
    template <int MODE, bool CLO>
    static int xcoop(const RhsArgs& a, cudaStream_t st) {
        static int blocks[64] = {0};
        return pencil_launch(pencil_x_coop_kernel<XW, CT, UNI, MODE, CLO>, blocks, XW * 32,
                             XSMEM, st, a);
    }
    // the x and y passes (each pass's closure instance when the grid has a
    // CLOSURE face in its direction)
    static int xy(const RhsArgs& a, bool add_x, cudaStream_t st) {
        int rc;
        if (a.clo[0] | a.clo[1])
            rc = add_x ? xcoop<P_ADD, true>(a, st) : xcoop<P_STORE, true>(a, st);
        else
            rc = add_x ? xcoop<P_ADD, false>(a, st) : xcoop<P_STORE, false>(a, st);
        if (rc) return rc;
        return (a.clo[2] | a.clo[3]) ? one<1, P_ADD, true>(a, 0, st) : one<1, P_ADD>(a, 0, st);
    }
    // plain RHS: x (=, or += with add_x), y (+=), z (+=)
    static int rhs(const RhsArgs& a, bool add_x, cudaStream_t st) {
        int rc = xy(a, add_x, st);
        return rc ? rc : one<2, P_ADD>(a, 0, st);
    }
    // stage: x, y into du, then z with the stage update
    static int stage(const RhsArgs& a, bool add_x, int krk, cudaStream_t st) {
        if constexpr (UNI) {
            int rc = xy(a, add_x, st);
            return rc ? rc : one<2, P_STAGE>(a, krk, st);
        } else {
            return fail(WS_ERR_UNSUPPORTED, "stage update needs Cartesian metrics");
        }
    }

    // a batch: argument table g of n grids, woff = the three passes' work
    // prefix tables of n + 1 entries each (x, y, z); krk 0: RHS into each du;
    // clo: some grid has a CLOSURE face
    template <int DIR, int MODE, bool CLO = false>
    static int one_batch(const RhsArgs* g, const long* woff, int n, int krk, cudaStream_t st) {
        constexpr int W = MODE == P_STAGE ? SW : WPB;
        static int blocks[64] = {0};
        return pencil_launch(pencil_batch_kernel<DIR, W, CT, MODE, CLO>, blocks, W * 32,
                             MODE == P_STAGE ? SSMEM : SMEM, st, g, woff, n, krk);
    }
    template <bool CLO>
    static int xy_batch(const RhsArgs* g, const long* woff, int n, cudaStream_t st) {
        static int blocks[64] = {0};
        int rc = pencil_launch(pencil_x_coop_batch_kernel<XW, CT, P_STORE, CLO>, blocks, XW * 32,
                               XSMEM, st, g, woff, n);
        return rc ? rc : one_batch<1, P_ADD, CLO>(g, woff + (n + 1), n, 0, st);
    }
    static int batch(const RhsArgs* g, const long* woff, int n, int krk, bool clo,
                     cudaStream_t st) {
        int rc = clo ? xy_batch<true>(g, woff, n, st) : xy_batch<false>(g, woff, n, st);
        if (rc) return rc;
        if (!krk) return one_batch<2, P_ADD>(g, woff + 2 * (n + 1), n, 0, st);
        // the batched mixed stage pass (arguments read from global memory)
        // needs the registers of 8 warps per CTA
        if constexpr (sizeof(CT) == 4 && WPB != 8)
            return PencilLauncher<8, CT, true>::template one_batch<2, P_STAGE>(
                g, woff + 2 * (n + 1), n, krk, st);
        else
            return one_batch<2, P_STAGE>(g, woff + 2 * (n + 1), n, krk, st);
    }
};

}  // namespace ws
