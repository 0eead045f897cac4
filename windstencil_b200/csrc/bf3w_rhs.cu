// bf3w_rhs.cu -- fused BF3W inviscid RHS for sm_100a.
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
//   * A CTA owns a BX x BY column footprint and sweeps it along z over a chunk
//     of planes (the reference's scanZ reuse).  The z-direction split fluxes
//     of the last 8 planes live in a shared-memory ring, so every z face is
//     reconstructed exactly once and no split value goes through HBM (the
//     reference round-trips fpZ/fmZ through global scratch).
//   * Per plane: the x-split over (BX+8) x BY points and the y-split over
//     BX x (BY+8) points are staged in shared memory; every face flux is then
//     one work item (face, variable) that evaluates the P and M WENO of that
//     face once, so the only redundant faces are the BX and BY tile edges.
//   * The five primitive planes a step needs are brought in with cp.async,
//     double-buffered one plane ahead of the arithmetic.
//   * The grid is persistent (one CTA per SM, static round-robin over
//     (tile, z-chunk) work items).
//   * No tensor cores: nothing on this path is a contraction.  The bound is
//     the FP64 pipe (about 7.3 kFLOP per cell).
#include <cstdio>

#include "ws_device.cuh"
#include "ws_internal.h"

namespace ws {

template <int BX, int BY, typename CT>
struct RhsLayout {
    static constexpr int BXY = BX * BY;
    static constexpr int SXW = BX + 8;        // x-split row width
    static constexpr int SYH = BY + 8;        // y-split rows
    static constexpr int BOXW = BX + 8, BOXH = BY + 8, BOX = BOXW * BOXH;
    static constexpr int STG = 5 * (BOX + BXY);   // doubles per staging buffer
    static constexpr int N_STG = 2 * STG;         // double
    static constexpr int N_FX = 5 * BY * (BX + 1);
    static constexpr int N_FY = 5 * (BY + 1) * BX;
    static constexpr int N_FZ = 2 * 5 * BXY;
    static constexpr int N_RING = 8 * 10 * BXY;   // CT
    static constexpr int N_SX = 10 * BY * SXW;    // CT
    static constexpr int N_SY = 10 * SYH * BX;    // CT
    static constexpr size_t smem_bytes =
        (size_t)(N_STG + N_FX + N_FY + N_FZ) * sizeof(double) +
        (size_t)(N_RING + N_SX + N_SY) * sizeof(CT);
};

__device__ __forceinline__ size_t lap_index(int X, int Y, int Z, uint32_t pitch, int ny) {
    return (size_t)X + (size_t)pitch * ((size_t)Y + (size_t)(ny + 8) * (size_t)Z);
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

// P and M WENO of one face from 8 staged split values each; element k of the
// P stencil is at bp[idx(k)*stride], idx(k) = (k + rot) & mask (the z ring
// wraps, x and y rows do not), the M stencil is the reversed F- row at +pmoff.
template <typename CT>
__device__ __forceinline__ double face_flux(const CT* bp, int pmoff, int stride, int rot,
                                            int mask);

template <>
__device__ __forceinline__ double face_flux<double>(const double* bp, int pmoff, int stride,
                                                    int rot, int mask) {
    double t[8], np, dp, nm, dm;
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = bp[((k + rot) & mask) * stride];
    weno7_symbo_nd<double>(t, np, dp);
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = bp[pmoff + ((7 - k + rot) & mask) * stride];
    weno7_symbo_nd<double>(t, nm, dm);
    return np / dp + nm / dm;
}

template <>
__device__ __forceinline__ double face_flux<float>(const float* bp, int pmoff, int stride,
                                                   int rot, int mask) {
    float t[8], np, dp, nm, dm;
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = bp[((k + rot) & mask) * stride];
    weno7_symbo_nd<float>(t, np, dp);
#pragma unroll
    for (int k = 0; k < 8; ++k) t[k] = bp[pmoff + ((7 - k + rot) & mask) * stride];
    weno7_symbo_nd<float>(t, nm, dm);
    return (double)__fdividef(np, dp) + (double)__fdividef(nm, dm);
}

// cp.async the primitive box of plane z (x: x0-4..x0+BX+3, y: y0-4..y0+BY+3)
// and the BX x BY centre of plane z+4 into one staging buffer.
template <int BX, int BY, int NT>
__device__ __forceinline__ void issue_stage(const RhsArgs& a, double* s, int x0, int y0,
                                            int z) {
    using L = RhsLayout<BX, BY, double>;
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
            Z = z + 4;
        }
        cp_async8(s + t, a.prim[f] + lap_index(X, Y, Z, a.ppitch[f], a.ny));
    }
}

template <int BX, int BY, int NT, bool UNI, typename CT>
__global__ void __launch_bounds__(NT, 1) bf3w_rhs_kernel(const __grid_constant__ RhsArgs a) {
    using L = RhsLayout<BX, BY, CT>;
    constexpr int BXY = L::BXY, SXW = L::SXW, SYH = L::SYH, BOXW = L::BOXW, BOX = L::BOX;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* stg = reinterpret_cast<double*>(smem_raw);   // [2][STG]
    double* fx = stg + L::N_STG;                         // [5][BY][BX+1]
    double* fy = fx + L::N_FX;                           // [5][BY+1][BX]
    double* fz = fy + L::N_FY;                           // [2][5][BXY]
    CT* ring = reinterpret_cast<CT*>(fz + L::N_FZ);      // [8][10][BXY]
    CT* sxs = ring + L::N_RING;                          // [10][BY][SXW]
    CT* sys = sxs + L::N_SX;                             // [10][SYH][BX]

    const SplitK<CT> k = {CT(a.eps2), CT(a.hrg), CT(a.c1), CT(a.c3), CT(a.gm1)};
    const int tid = threadIdx.x;
    const int nwork = a.ntx * a.nty * a.nzc;

    for (int wi = blockIdx.x; wi < nwork; wi += gridDim.x) {
        const int tx = wi % a.ntx;
        const int rr = wi / a.ntx;
        const int ty = rr % a.nty, tz = rr / a.nty;
        const int x0 = a.sx + tx * BX, y0 = a.sy + ty * BY;
        const int z0 = a.sz + tz * a.zc;
        const int z1 = min(z0 + a.zc, a.ez);

        issue_stage<BX, BY, NT>(a, stg, x0, y0, z0);
        cp_async_commit();

        // prologue: z split of planes z0-4 .. z0+3 into the ring
        for (int t = tid; t < 8 * BXY; t += NT) {
            const int pl = t / BXY, col = t - pl * BXY;
            const int Z = z0 - 4 + pl;
            const int X = min(x0 + col % BX, a.nx + 7), Y = min(y0 + col / BX, a.ny + 7);
            CT out[10];
            split_point<2, UNI, CT>(a, k, ldg_prim(a, 0, X, Y, Z), ldg_prim(a, 1, X, Y, Z),
                                    ldg_prim(a, 2, X, Y, Z), ldg_prim(a, 3, X, Y, Z),
                                    ldg_prim(a, 4, X, Y, Z), X, Y, Z, out);
            CT* dst = ring + (Z & 7) * 10 * BXY + col;
#pragma unroll
            for (int c = 0; c < 10; ++c) dst[c * BXY] = out[c];
        }
        __syncthreads();
        // z face z0-1/2 (stencil planes z0-4 .. z0+3)
        for (int t = tid; t < 5 * BXY; t += NT) {
            const int var = t / BXY, col = t - var * BXY;
            fz[t] = face_flux<CT>(ring + var * BXY + col, 5 * BXY, 10 * BXY, (z0 - 4) & 7, 7);
        }
        int prev = 0;

        for (int z = z0; z < z1; ++z) {
            const int b = (z - z0) & 1;
            if (z + 1 < z1) {
                issue_stage<BX, BY, NT>(a, stg + (b ^ 1) * L::STG, x0, y0, z + 1);
                cp_async_commit();
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();

            // ---- split phase: x-split, y-split of plane z, z-split of plane z+4
            const double* sb = stg + b * L::STG;
            constexpr int NXS = SXW * BY, NYS = BX * SYH, NZS = BXY;
            for (int t = tid; t < NXS + NYS + NZS; t += NT) {
                CT out[10];
                if (t < NXS) {
                    const int yy = t / SXW, xi = t - yy * SXW;
                    const int bi = (yy + 4) * BOXW + xi;
                    split_point<0, UNI, CT>(a, k, sb[bi], sb[BOX + bi], sb[2 * BOX + bi],
                                            sb[3 * BOX + bi], sb[4 * BOX + bi],
                                            min(x0 - 4 + xi, a.nx + 7), min(y0 + yy, a.ny + 7),
                                            z, out);
                    CT* dst = sxs + yy * SXW + xi;
#pragma unroll
                    for (int c = 0; c < 10; ++c) dst[c * BY * SXW] = out[c];
                } else if (t < NXS + NYS) {
                    const int t2 = t - NXS;
                    const int yi = t2 / BX, xx = t2 - yi * BX;
                    const int bi = yi * BOXW + xx + 4;
                    split_point<1, UNI, CT>(a, k, sb[bi], sb[BOX + bi], sb[2 * BOX + bi],
                                            sb[3 * BOX + bi], sb[4 * BOX + bi],
                                            min(x0 + xx, a.nx + 7), min(y0 - 4 + yi, a.ny + 7),
                                            z, out);
                    CT* dst = sys + yi * BX + xx;
#pragma unroll
                    for (int c = 0; c < 10; ++c) dst[c * SYH * BX] = out[c];
                } else {
                    const int col = t - NXS - NYS;
                    const double* cb = sb + 5 * BOX + col;
                    split_point<2, UNI, CT>(a, k, cb[0], cb[BXY], cb[2 * BXY], cb[3 * BXY],
                                            cb[4 * BXY], min(x0 + col % BX, a.nx + 7),
                                            min(y0 + col / BX, a.ny + 7), z + 4, out);
                    CT* dst = ring + ((z + 4) & 7) * 10 * BXY + col;
#pragma unroll
                    for (int c = 0; c < 10; ++c) dst[c * BXY] = out[c];
                }
            }
            __syncthreads();

            // ---- face phase: every x, y face of plane z and the z face z+1/2
            const int cur = prev ^ 1;
            constexpr int NXF = (BX + 1) * BY * 5, NYF = BX * (BY + 1) * 5, NZF = BXY * 5;
            for (int t = tid; t < NXF + NYF + NZF; t += NT) {
                if (t < NXF) {
                    const int var = t / ((BX + 1) * BY);
                    const int r = t - var * (BX + 1) * BY;
                    const int yy = r / (BX + 1), f = r - yy * (BX + 1);
                    fx[t] = face_flux<CT>(sxs + (var * BY + yy) * SXW + f, 5 * BY * SXW, 1, 0, 15);
                } else if (t < NXF + NYF) {
                    const int t2 = t - NXF;
                    const int var = t2 / ((BY + 1) * BX);
                    const int r = t2 - var * (BY + 1) * BX;
                    const int g = r / BX, xx = r - g * BX;
                    fy[t2] = face_flux<CT>(sys + (var * SYH + g) * BX + xx, 5 * SYH * BX, BX, 0, 15);
                } else {
                    const int t3 = t - NXF - NYF;
                    const int var = t3 / BXY, col = t3 - var * BXY;
                    fz[cur * 5 * BXY + t3] =
                        face_flux<CT>(ring + var * BXY + col, 5 * BXY, 10 * BXY, (z - 3) & 7, 7);
                }
            }
            __syncthreads();

            // ---- difference phase: du of plane z (FP64)
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
                         (size_t)a.du_pitch * ((size_t)(Y - a.sy) +
                                               (size_t)a.du_ly * ((size_t)(z - a.sz) +
                                                                  (size_t)a.du_lz * var))] = -J * r;
                }
            }
            prev = cur;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Compiled tile shapes and host launch
// ---------------------------------------------------------------------------
namespace {
constexpr TileCfg kCfgs[] = {{16, 8, 512}, {16, 8, 256}, {16, 8, 576}};
constexpr int kNumCfgs = sizeof(kCfgs) / sizeof(kCfgs[0]);

template <int BX, int BY, int NT, bool UNI, typename CT>
struct Launcher {
    static void* fn() { return (void*)bf3w_rhs_kernel<BX, BY, NT, UNI, CT>; }
    static size_t smem() { return RhsLayout<BX, BY, CT>::smem_bytes; }
    static int launch(const RhsArgs& a, int ctas, cudaStream_t st) {
        static int prepared_dev = -1;
        int dev = 0;
        cudaGetDevice(&dev);
        if (prepared_dev != dev) {
            WS_CUDA(cudaFuncSetAttribute(bf3w_rhs_kernel<BX, BY, NT, UNI, CT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem()));
            prepared_dev = dev;
        }
        bf3w_rhs_kernel<BX, BY, NT, UNI, CT><<<ctas, NT, smem(), st>>>(a);
        WS_CUDA(cudaGetLastError());
        return WS_OK;
    }
    static int max_ctas() {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return 0;
        cudaFuncSetAttribute(bf3w_rhs_kernel<BX, BY, NT, UNI, CT>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem());
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per, bf3w_rhs_kernel<BX, BY, NT, UNI, CT>, NT, smem()) != cudaSuccess)
            return 0;
        return sms * per;
    }
};

template <int BX, int BY, int NT>
int dispatch_launch(const RhsArgs& a, int precision, bool uni, int ctas, cudaStream_t st) {
    if (precision == WS_MIXED) {
        return uni ? Launcher<BX, BY, NT, true, float>::launch(a, ctas, st)
                   : Launcher<BX, BY, NT, false, float>::launch(a, ctas, st);
    }
    return uni ? Launcher<BX, BY, NT, true, double>::launch(a, ctas, st)
               : Launcher<BX, BY, NT, false, double>::launch(a, ctas, st);
}
template <int BX, int BY, int NT>
int dispatch_max(int precision, bool uni) {
    if (precision == WS_MIXED)
        return uni ? Launcher<BX, BY, NT, true, float>::max_ctas()
                   : Launcher<BX, BY, NT, false, float>::max_ctas();
    return uni ? Launcher<BX, BY, NT, true, double>::max_ctas()
               : Launcher<BX, BY, NT, false, double>::max_ctas();
}
}  // namespace

int num_tile_cfgs() { return kNumCfgs; }
TileCfg tile_cfg(int i) { return kCfgs[i]; }
int find_tile_cfg(int bx, int by, int threads) {
    for (int i = 0; i < kNumCfgs; ++i)
        if (kCfgs[i].bx == bx && kCfgs[i].by == by && kCfgs[i].threads == threads) return i;
    return -1;
}

int launch_rhs(const RhsArgs& a, int precision, bool uniform, int cfg, int ctas,
               cudaStream_t st) {
    switch (cfg) {
        case 0: return dispatch_launch<16, 8, 512>(a, precision, uniform, ctas, st);
        case 1: return dispatch_launch<16, 8, 256>(a, precision, uniform, ctas, st);
        case 2: return dispatch_launch<16, 8, 576>(a, precision, uniform, ctas, st);
        default: return fail(WS_ERR_INVALID, "unknown tile configuration");
    }
}

int rhs_max_ctas(int precision, bool uniform, int cfg) {
    switch (cfg) {
        case 0: return dispatch_max<16, 8, 512>(precision, uniform);
        case 1: return dispatch_max<16, 8, 256>(precision, uniform);
        case 2: return dispatch_max<16, 8, 576>(precision, uniform);
        default: return 0;
    }
}

}  // namespace ws
