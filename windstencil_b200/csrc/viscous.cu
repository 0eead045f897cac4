// viscous.cu -- viscous terms of the Navier-Stokes RHS on the GPU.
//
// Replaces du_vis_Jacobian3d (OCFD_Stream.cpp:229-345): per RHS the reference
// runs 12 derivative kernels for u, v, w, T (du_viscous_Jacobian3d_init,
// OCFD_NS_Jacobian3d.cpp:455-475), and per direction the flux kernel
// vis_flux_ker (:477-624), a halo exchange of its four outputs, four
// derivative kernels and four accumulation kernels (YF_Pe_XF) -- 40 launches
// and 12 derivative fields in HBM.  Here:
//   vis_flux_kernel: one pass over the interior computes the 12 first
//     derivatives in registers (CD6/CD8 through the ghosts, value / h; the
//     reference's reduced forms next to DIF_BOUND faces), the
//     Sutherland viscosity (get_Amu_kernal, commen_kernel.cpp:123-132) and
//     the viscous fluxes Ev1..4 of all three directions (12 LAP fields; 9 on
//     Cartesian grids, where the symmetric stress entries share a field);
//   vis_ghost_kernel: the ghosts the divergence reads, each direction's
//     fluxes along their own axis only (one launch);
//   vis_div_kernel: one pass adds J * d(Ev_dir)/d(dir) of the three
//     directions to du[1..4] (or stores it, for the fused RK stage), x then y
//     then z as the reference accumulates.
// Per cell ~32 B of primitives in, 72-96 B of fluxes out and in again, 32-64
// B of du; the flux pass is bound by instruction issue, not by HBM.
#include "ws_internal.h"

namespace ws {
namespace {

struct VisArgs {
    const double* prim[4];     // u, v, w, T (LAP, ghosts filled)
    uint32_t ppitch[4];
    const double* met[10];     // akx..asz, ajac (uniform: unused)
    uint32_t mpitch[10];
    double* ev[12];            // flux q (0..3) of direction dir at ev[4 * dir + q], LAP
    uint32_t epitch;
    double* du;                // SoA [5][nz][ny][du_pitch]
    uint32_t du_pitch, du_ly, du_lz;
    int nx, ny, nz;
    double rh[3];              // 1 / (h * the difference's divisor: 60 CD6, 840 CD8)
    double h[3];               // grid spacing (the reduced boundary forms divide by it)
    double tsb, amu_c0, vfc;   // Sutherland constants, Cp/Pr
    int uniform, accumulate;
    // DIF_BOUND: reduced forms next to the low / high face of direction d
    // (the flag set and the face not EXTERNAL); any: some flag is on
    int d0lo[3], d0hi[3], any_d0;
};

__device__ __forceinline__ size_t lapi(int X, int Y, int Z, uint32_t pitch, int ny) {
    return (size_t)X + (size_t)pitch * ((size_t)Y + (size_t)(ny + 8) * (size_t)Z);
}

// Both passes march in z over a tile of VBX x VBY columns (the flux pass:
// VBX x FBY), one thread per column: a z derivative takes its values from
// the thread's own window of planes (registers), x and y derivatives from a
// tile of the current plane with an R-cell rim staged by the whole block.
// Each plane is read from HBM once (the rims and the window's lead plane come
// back through L2), instead of 8-point stencils re-read through the caches
// per point.  The next plane's tile arrives by cp.async while the current
// one is processed.  Work items are (column tile, chunk of VZC planes),
// chunk-major, so the blocks in flight share their rims and planes in L2.
constexpr int VBX = 32, VBY = 8, VNT = VBX * VBY, VZC = 16;
// the flux pass's tile height: 12 rows (12 warps per SM at 168 registers)
// measured fastest for CD8 against 8 (its window in registers then needs 232
// registers, 8 warps), 14 and 16 rows (128 registers, small spills)
constexpr int FBY = 12, FNT = VBX * FBY;

// central first difference from the differences d_m = f(+m) - f(-m), times
// the divisor of OCFD_Schemes.cpp:97-104 (CD6: /60) and :134-142 (CD8: /840),
// which the caller folds into its 1/h factor (one multiply instead of an
// IEEE division per derivative)
template <int R>
__device__ __forceinline__ double cdv(double d1, double d2, double d3, double d4) {
    if (R == 3) return 45.0 * d1 - 9.0 * d2 + d3;
    return 672.0 * d1 - 168.0 * d2 + 32.0 * d3 - 3.0 * d4;
}

// The kernels keep their fields in shared memory as interleaved pairs
// (double2: u|v, w|T; Ev1|Ev2, Ev3|Ev4), so one 16-byte load serves a stencil
// point of two fields: half the shared-memory instructions, which is what
// limits these passes (the MIO queue), at the same bytes.
// Differences of a pair along stride s (in double2 elements):
template <int R>
__device__ __forceinline__ double2 cd2(const double2* c, int s) {
    double d[2][4] = {};
#pragma unroll
    for (int m = 1; m <= R; ++m) {
        const double2 p = c[m * s], n = c[-m * s];
        d[0][m - 1] = p.x - n.x;
        d[1][m - 1] = p.y - n.y;
    }
    return make_double2(cdv<R>(d[0][0], d[0][1], d[0][2], d[0][3]),
                        cdv<R>(d[1][0], d[1][1], d[1][2], d[1][3]));
}

// The reference's reduced forms of the first difference next to a face whose
// DIF_BOUND flag is set (OCFD_D0bound_scheme_kernel, OCFD_bound_Scheme.cpp:
// 82-240), in its operation order: at distance e = 0..3 from the face a
// one-sided difference, then 2nd-, 4th- and 6th-order central differences.
// at(m) gives the stencil value at offset m (|m| <= 3).  Returns false where
// the central scheme applies (the low face is tested first, as there).
template <typename F>
__device__ __forceinline__ bool d0_form(F at, int pos, int n, bool lo, bool hi, double& t) {
    int e;
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
    if (e == 0) t = low ? at(1) - at(0) : at(0) - at(-1);
    else if (e == 1) t = (at(1) - at(-1)) * 0.5;
    else if (e == 2) t = (at(-2) - 8.0 * at(-1) + 8.0 * at(1) - at(2)) / 12.0;
    else t = (at(3) - at(-3) - 9.0 * (at(2) - at(-2)) + 45.0 * (at(1) - at(-1))) / 60.0;
    return true;
}

struct VisItem {
    int x0, y0, k0, k1;
};

template <int BY = VBY>
__host__ __device__ __forceinline__ long vis_items(int nx, int ny, int nz) {
    return (long)((nx + VBX - 1) / VBX) * ((ny + BY - 1) / BY) * ((nz + VZC - 1) / VZC);
}
template <int BY = VBY>
__device__ __forceinline__ long vis_items(const VisArgs& a) {
    return vis_items<BY>(a.nx, a.ny, a.nz);
}

template <int BY = VBY>
__device__ __forceinline__ VisItem vis_item(const VisArgs& a, long it) {
    const int ntx = (a.nx + VBX - 1) / VBX, nty = (a.ny + BY - 1) / BY;
    const long t = it % ((long)ntx * nty);
    VisItem w;
    w.x0 = (int)(t % ntx) * VBX;
    w.y0 = (int)(t / ntx) * BY;
    w.k0 = (int)(it / ((long)ntx * nty)) * VZC;
    w.k1 = min(a.nz, w.k0 + VZC);
    return w;
}

__device__ __forceinline__ void vcp8(void* smem, const void* gmem) {
    const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void vcp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void vcp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <int R>
constexpr size_t vis_flux_smem() {   // two buffers of the plane tile with its rim, pairs
    return 2 * (size_t)2 * (FBY + 2 * R) * (VBX + 2 * R) * sizeof(double2);
}
template <int R>
constexpr size_t vis_div_smem() {   // two buffers of the Ev_x, Ev_y tiles and of du
    return 2 * ((size_t)4 * VBY * (VBX + 2 * R) + 4 * (VBY + 2 * R) * VBX + 4 * VNT) *
           sizeof(double);
}

// Sutherland viscosity at temperature T (get_Amu_kernal, commen_kernel.cpp:123-132)
__device__ __forceinline__ double sutherland(const VisArgs& a, double T) {
    return a.amu_c0 * sqrt(T * T * T) / (a.tsb + T);
}

// Gradients of u, v, w, T (CD6/CD8, value / h), the Sutherland viscosity
// and the viscous fluxes Ev1..4 of all three directions (vis_flux_ker,
// OCFD_NS_Jacobian3d.cpp:477-624) at every interior cell.  A thread's z window
// (planes k-R .. k+R of its column, the four fields) lives in registers; the
// x and y stencils read the plane's tile with its rim from shared memory.
// The tiles arrive by cp.async into two buffers, the next plane's while the
// current one is processed, so one barrier per plane orders them; the
// window's lead values are loaded a plane ahead, and the viscosity (a
// square root and a division in series) is computed a plane ahead.
// D0: compiled with the DIF_BOUND reduced forms (grids with a flag set)
template <int R, bool UNI, bool D0>
__global__ void __launch_bounds__(FNT, 1) vis_flux_kernel(const __grid_constant__ VisArgs a) {
    constexpr int W = 2 * R + 1, TX = VBX + 2 * R, TY = FBY + 2 * R, TYX = TY * TX;
    constexpr int PS = (TYX + FNT - 1) / FNT;     // tile positions a thread stages per field
    extern __shared__ __align__(16) double vsm[];
    double2* tiles = reinterpret_cast<double2*>(vsm);  // [2 buffers][2 pairs][TY][TX]
    const int tid = threadIdx.x, lx = tid % VBX, ly = tid / VBX;
    const size_t plane_rows = (size_t)(a.ny + 8);
    const long items = vis_items<FBY>(a);
    int buf = 0;                                       // continues across items
    for (long it = blockIdx.x; it < items; it += gridDim.x) {
        const VisItem w = vis_item<FBY>(a, it);
        const int i = w.x0 + lx, j = w.y0 + ly;
        const bool own = i < a.nx && j < a.ny;
        const int X = min(i, a.nx - 1) + 4, Y = min(j, a.ny - 1) + 4;
        // in-plane offsets of this thread's column and of its tile positions
        // (LAP points clamped into the array: the clamped ones belong to no
        // stencil of an own cell), per field
        int col[4], so[4][PS];
#pragma unroll
        for (int q = 0; q < 4; ++q) col[q] = X + (int)a.ppitch[q] * Y;
#pragma unroll
        for (int p = 0; p < PS; ++p) {
            const int t = min(tid + p * FNT, TYX - 1), yy = t / TX, xx = t - yy * TX;
            const int tx = min(w.x0 - R + xx + 4, a.nx + 7), ty = min(w.y0 - R + yy + 4, a.ny + 7);
#pragma unroll
            for (int q = 0; q < 4; ++q) so[q][p] = tx + (int)a.ppitch[q] * ty;
        }
        auto plane = [&](int q, int k) {
            return a.prim[q] + (size_t)a.ppitch[q] * plane_rows * (size_t)(k + 4);
        };
        // plane k's tile into buffer b, pairs interleaved (u|v, w|T)
        auto stage = [&](int k, int b) {
            double* t = reinterpret_cast<double*>(tiles + b * 2 * TYX);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double* src = plane(q, k);
#pragma unroll
                for (int p = 0; p < PS; ++p)
                    if (tid + p * FNT < TYX)
                        vcp8(t + 2 * ((q >> 1) * TYX + tid + p * FNT) + (q & 1), src + so[q][p]);
            }
            vcp_commit();
        };
        stage(w.k0, buf);
        // window zw[q][m] = plane k - R + m; planes k0-R .. k0+R-1 go to
        // slots 1..2R, and each step shifts the lead plane k+R in
        double zw[4][W], lead[4];
#pragma unroll
        for (int m = 0; m < 2 * R; ++m)
#pragma unroll
            for (int q = 0; q < 4; ++q) zw[q][m + 1] = __ldg(plane(q, w.k0 - R + m) + col[q]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            zw[q][0] = 0.0;
            lead[q] = __ldg(plane(q, w.k0 + R) + col[q]);
        }
        double amu_n = sutherland(a, zw[3][R + 1]);       // plane k0
        for (int k = w.k0; k < w.k1; ++k) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
#pragma unroll
                for (int m = 0; m < 2 * R; ++m) zw[q][m] = zw[q][m + 1];
                zw[q][2 * R] = lead[q];
            }
            const double amu = amu_n;
            vcp_wait_all();
            __syncthreads();            // plane k's tile landed; buffer buf^1 is free
            const double2* tile = tiles + buf * 2 * TYX;
            if (k + 1 < w.k1) {
                stage(k + 1, buf ^ 1);
#pragma unroll
                for (int q = 0; q < 4; ++q) lead[q] = __ldg(plane(q, k + 1 + R) + col[q]);
                amu_n = sutherland(a, zw[3][R + 1]);
            }
            buf ^= 1;
            if (!own) continue;
            double g[4][3];
#pragma unroll
            for (int pr = 0; pr < 2; ++pr) {
                const double2* c = tile + (pr * TY + ly + R) * TX + lx + R;
                const double2 dx = cd2<R>(c, 1), dy = cd2<R>(c, TX);
                g[2 * pr][0] = dx.x * a.rh[0];
                g[2 * pr + 1][0] = dx.y * a.rh[0];
                g[2 * pr][1] = dy.x * a.rh[1];
                g[2 * pr + 1][1] = dy.y * a.rh[1];
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double* z = zw[q];
                g[q][2] = cdv<R>(z[R + 1] - z[R - 1], z[R + 2] - z[R - 2], z[R + 3] - z[R - 3],
                                 R == 4 ? z[R + 4] - z[0] : 0.0) *
                          a.rh[2];
            }
            if (D0) {           // DIF_BOUND: the reduced forms next to flagged faces
#pragma unroll
                for (int pr = 0; pr < 2; ++pr) {
                    const double2* c = tile + (pr * TY + ly + R) * TX + lx + R;
#pragma unroll
                    for (int hh = 0; hh < 2; ++hh) {
                        const int q = 2 * pr + hh;
                        auto cx = [&](int m) { return hh ? c[m].y : c[m].x; };
                        auto cy = [&](int m) { return hh ? c[m * TX].y : c[m * TX].x; };
                        auto cz = [&](int m) { return zw[q][R + m]; };
                        double t;
                        if (d0_form(cx, i, a.nx, a.d0lo[0], a.d0hi[0], t)) g[q][0] = t / a.h[0];
                        if (d0_form(cy, j, a.ny, a.d0lo[1], a.d0hi[1], t)) g[q][1] = t / a.h[1];
                        if (d0_form(cz, k, a.nz, a.d0lo[2], a.d0hi[2], t)) g[q][2] = t / a.h[2];
                    }
                }
            }
            const int Z = k + 4;
            // physical gradients (chain rule with akx..asz; Cartesian grids
            // take them as they are: the products with the unit metric give
            // the same values for finite gradients)
            double m[9], aj = 1.0, gx[4], gy[4], gz[4];
            if (UNI) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    gx[q] = g[q][0];
                    gy[q] = g[q][1];
                    gz[q] = g[q][2];
                }
            } else {
#pragma unroll
                for (int c = 0; c < 9; ++c) m[c] = __ldg(a.met[c] + lapi(X, Y, Z, a.mpitch[c], a.ny));
                aj = __ldg(a.met[9] + lapi(X, Y, Z, a.mpitch[9], a.ny));
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    gx[q] = g[q][0] * m[0] + g[q][1] * m[3] + g[q][2] * m[6];
                    gy[q] = g[q][0] * m[1] + g[q][1] * m[4] + g[q][2] * m[7];
                    gz[q] = g[q][0] * m[2] + g[q][1] * m[5] + g[q][2] * m[8];
                }
            }
            const double div = gx[0] + gy[1] + gz[2];
            const double s11 = (2.0 * gx[0] - 2.0 / 3.0 * div) * amu;
            const double s22 = (2.0 * gy[1] - 2.0 / 3.0 * div) * amu;
            const double s33 = (2.0 * gz[2] - 2.0 / 3.0 * div) * amu;
            const double s12 = (gy[0] + gx[1]) * amu;
            const double s13 = (gz[0] + gx[2]) * amu;
            const double s23 = (gz[1] + gy[2]) * amu;
            const double amuk = amu * a.vfc;
            const double u = zw[0][R], v = zw[1][R], wv = zw[2][R];
            const double E1 = u * s11 + v * s12 + wv * s13 + amuk * gx[3];
            const double E2 = u * s12 + v * s22 + wv * s23 + amuk * gy[3];
            const double E3 = u * s13 + v * s23 + wv * s33 + amuk * gz[3];
            const size_t o = lapi(X, Y, Z, a.epitch, a.ny);
            if (UNI) {
                // Ev of direction d: row d of the stress tensor and E_d; the
                // symmetric entries share a field (ev[4] = ev[1], ev[8] =
                // ev[2], ev[9] = ev[6], vis_flux_fields), so 9 are stored
                a.ev[0][o] = s11; a.ev[1][o] = s12; a.ev[2][o] = s13; a.ev[3][o] = E1;
                a.ev[5][o] = s22; a.ev[6][o] = s23; a.ev[7][o] = E2;
                a.ev[10][o] = s33; a.ev[11][o] = E3;
            } else {
#pragma unroll
                for (int dir = 0; dir < 3; ++dir) {
                    const double kx = m[3 * dir] * aj, ky = m[3 * dir + 1] * aj,
                                 kz = m[3 * dir + 2] * aj;
                    a.ev[4 * dir + 0][o] = kx * s11 + ky * s12 + kz * s13;
                    a.ev[4 * dir + 1][o] = kx * s12 + ky * s22 + kz * s23;
                    a.ev[4 * dir + 2][o] = kx * s13 + ky * s23 + kz * s33;
                    a.ev[4 * dir + 3][o] = kx * E1 + ky * E2 + kz * E3;
                }
            }
        }
    }
}

// du[1..4] (+)= J * (d Ev_x/dx + d Ev_y/dy + d Ev_z/dz), x then y then z as
// the reference accumulates (YF_Pe_XF per direction); du[0] = 0 when storing.
// The Ev_z window of a thread's column lives in registers; the next plane's
// Ev_x / Ev_y tiles (and du, accumulating) arrive by cp.async into the other
// of two shared-memory buffers while the current plane is processed.
template <int R, bool UNI, bool D0>
__global__ void __launch_bounds__(VNT, 2) vis_div_kernel(const __grid_constant__ VisArgs a) {
    constexpr int W = 2 * R + 1, XW = VBX + 2 * R, YH = VBY + 2 * R;
    constexpr int XF = VBY * XW, YF = YH * VBX;               // x-rim, y-rim tile per field
    constexpr int PX = (XF + VNT - 1) / VNT, PY = (YF + VNT - 1) / VNT;
    constexpr int BUF = 2 * XF + 2 * YF;                      // double2 per buffer
    extern __shared__ __align__(16) double vsm[];
    double2* tiles = reinterpret_cast<double2*>(vsm);         // [2][Ev_x pairs | Ev_y pairs]
    double* dus = vsm + 2 * 2 * BUF;                          // [2][4][VNT] du (accumulating)
    const int tid = threadIdx.x, lx = tid % VBX, ly = tid / VBX;
    const size_t eplane = (size_t)a.epitch * (size_t)(a.ny + 8);
    const long items = vis_items(a);
    for (long it = blockIdx.x; it < items; it += gridDim.x) {
        const VisItem w = vis_item(a, it);
        const int i = w.x0 + lx, j = w.y0 + ly;
        const bool own = i < a.nx && j < a.ny;
        const int X = min(i, a.nx - 1) + 4, Y = min(j, a.ny - 1) + 4;
        // in-plane offsets (the flux fields share one pitch): this column,
        // the x-rim and y-rim tile positions (clamped into the array)
        const int col = X + (int)a.epitch * Y;
        int xo[PX], yo[PY];
#pragma unroll
        for (int p = 0; p < PX; ++p) {
            const int t = min(tid + p * VNT, XF - 1), yy = t / XW, xx = t - yy * XW;
            xo[p] = min(w.x0 - R + xx + 4, a.nx + 7) + (int)a.epitch * (min(w.y0 + yy, a.ny - 1) + 4);
        }
#pragma unroll
        for (int p = 0; p < PY; ++p) {
            const int t = min(tid + p * VNT, YF - 1), yy = t / VBX, xx = t - yy * VBX;
            yo[p] = min(w.x0 + xx, a.nx - 1) + 4 + (int)a.epitch * min(w.y0 - R + yy + 4, a.ny + 7);
        }
        auto plane = [&](int c, int k) { return a.ev[c] + eplane * (size_t)(k + 4); };
        const size_t du_col = (size_t)min(i, a.nx - 1) + (size_t)a.du_pitch * (size_t)min(j, a.ny - 1);
        const size_t du_plane = (size_t)a.du_pitch * a.du_ly, du_var = du_plane * a.du_lz;
        // plane k's Ev_x / Ev_y tiles (pairs interleaved) and du into buffer b
        auto stage = [&](int k, int b) {
            double2* xt = tiles + b * BUF;
            double2* yt = xt + 2 * XF;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double* bx = plane(q, k);
                const double* by = plane(4 + q, k);
#pragma unroll
                for (int p = 0; p < PX; ++p)
                    if (tid + p * VNT < XF)
                        vcp8(reinterpret_cast<double*>(xt + (q >> 1) * XF + tid + p * VNT) + (q & 1),
                             bx + xo[p]);
#pragma unroll
                for (int p = 0; p < PY; ++p)
                    if (tid + p * VNT < YF)
                        vcp8(reinterpret_cast<double*>(yt + (q >> 1) * YF + tid + p * VNT) + (q & 1),
                             by + yo[p]);
                if (a.accumulate)
                    vcp8(dus + (b * 4 + q) * VNT + tid, a.du + du_col + du_plane * k + du_var * (q + 1));
            }
            vcp_commit();
        };
        __syncthreads();                  // the previous item's last buffer is read
        stage(w.k0, 0);
        // Ev_z window: zw[q][m] = plane k - R + m (m = 0..2R); filled with
        // planes k0-R .. k0+R-1 in slots 1..2R, the lead plane k0+R apart
        double zw[4][W], lead[4];
#pragma unroll
        for (int m = 0; m < 2 * R; ++m)
#pragma unroll
            for (int q = 0; q < 4; ++q) zw[q][m + 1] = __ldg(plane(8 + q, w.k0 - R + m) + col);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            zw[q][0] = 0.0;
            lead[q] = __ldg(plane(8 + q, w.k0 + R) + col);
        }
        for (int k = w.k0; k < w.k1; ++k) {
            const int b = (k - w.k0) & 1;
            vcp_wait_all();
            __syncthreads();              // buffer b landed; buffer b^1 read by every thread
            if (k + 1 < w.k1) stage(k + 1, b ^ 1);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
#pragma unroll
                for (int m = 0; m < 2 * R; ++m) zw[q][m] = zw[q][m + 1];
                zw[q][2 * R] = lead[q];
            }
            if (k + 1 < w.k1)
#pragma unroll
                for (int q = 0; q < 4; ++q) lead[q] = __ldg(plane(8 + q, k + 1 + R) + col);
            if (!own) continue;
            const int Z = k + 4;
            const double aj = UNI ? 1.0 : __ldg(a.met[9] + lapi(X, Y, Z, a.mpitch[9], a.ny));
            const double2* xt = tiles + b * BUF;
            const double2* yt = xt + 2 * XF;
#pragma unroll
            for (int pr = 0; pr < 2; ++pr) {
                const double2* cxp = xt + (pr * VBY + ly) * XW + lx + R;
                const double2* cyp = yt + (pr * YH + ly + R) * VBX + lx;
                const double2 dx = cd2<R>(cxp, 1);
                const double2 dy = cd2<R>(cyp, VBX);
                const double ddx[2] = {dx.x, dx.y}, ddy[2] = {dy.x, dy.y};
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int q = 2 * pr + h;
                    const double* z = zw[q];
                    const double dz = cdv<R>(z[R + 1] - z[R - 1], z[R + 2] - z[R - 2],
                                             z[R + 3] - z[R - 3], R == 4 ? z[R + 4] - z[0] : 0.0);
                    double vx = ddx[h] * a.rh[0], vy = ddy[h] * a.rh[1], vz = dz * a.rh[2];
                    if (D0) {           // DIF_BOUND: the reduced forms next to flagged faces
                        auto fx = [&](int m) { return h ? cxp[m].y : cxp[m].x; };
                        auto fy = [&](int m) { return h ? cyp[m * VBX].y : cyp[m * VBX].x; };
                        auto fz = [&](int m) { return z[R + m]; };
                        double t;
                        if (d0_form(fx, i, a.nx, a.d0lo[0], a.d0hi[0], t)) vx = t / a.h[0];
                        if (d0_form(fy, j, a.ny, a.d0lo[1], a.d0hi[1], t)) vy = t / a.h[1];
                        if (d0_form(fz, k, a.nz, a.d0lo[2], a.d0hi[2], t)) vz = t / a.h[2];
                    }
                    double acc = a.accumulate ? dus[(b * 4 + q) * VNT + tid] : 0.0;
                    acc += aj * vx;
                    acc += aj * vy;
                    acc += aj * vz;
                    a.du[du_col + du_plane * k + du_var * (q + 1)] = acc;
                }
            }
            if (!a.accumulate) a.du[du_col + du_plane * k] = 0.0;
        }
    }
}

// Ghosts of the flux fields where the divergence pass reads them: its
// stencils are one-dimensional, so Ev of direction d (fields 4d .. 4d+3)
// needs only the 8 ghost layers along axis d, at interior coordinates of the
// two other axes.  Values by the face kinds of that axis, as the full ghost
// fill sets them (periodic: wrapped; EXTERNAL: kept; else the boundary cell).
struct VisGhostArgs {
    double* ev[12];
    uint32_t pitch;
    int nx, ny, nz;
    int kind[6];
};

__device__ __forceinline__ int vis_ghost_src(int g, int n, int lo_kind, int hi_kind) {
    if (g < 4) return lo_kind == WS_FACE_PERIODIC ? g + n : lo_kind == WS_FACE_EXTERNAL ? g : 4;
    return hi_kind == WS_FACE_PERIODIC ? g - n : hi_kind == WS_FACE_EXTERNAL ? g : n + 3;
}

__global__ void vis_ghost_kernel(const __grid_constant__ VisGhostArgs a) {
    const long nx = a.nx, ny = a.ny, nz = a.nz;
    const long sx = 8 * ny * nz, sy = 8 * nx * nz, total = sx + sy + 8 * nx * ny;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
         t += (long)gridDim.x * blockDim.x) {
        int d, p[3], s;                     // axis, LAP point, its source along d
        if (t < sx) {                       // x layers fastest (two runs of 4)
            const int l = (int)(t % 8);
            const long r = t / 8;
            d = 0;
            p[0] = l < 4 ? l : (int)nx + l;
            p[1] = 4 + (int)(r % ny);
            p[2] = 4 + (int)(r / ny);
        } else if (t < sx + sy) {           // x fastest, then the y layer
            const long u = t - sx, r = u / nx;
            const int l = (int)(r % 8);
            d = 1;
            p[0] = 4 + (int)(u % nx);
            p[1] = l < 4 ? l : (int)ny + l;
            p[2] = 4 + (int)(r / 8);
        } else {                            // x fastest, y, then the z layer
            const long u = t - sx - sy, r = u / nx;
            const int l = (int)(r / ny);
            d = 2;
            p[0] = 4 + (int)(u % nx);
            p[1] = 4 + (int)(r % ny);
            p[2] = l < 4 ? l : (int)nz + l;
        }
        const int n = d == 0 ? a.nx : (d == 1 ? a.ny : a.nz);
        s = vis_ghost_src(p[d], n, a.kind[2 * d], a.kind[2 * d + 1]);
        if (s == p[d]) continue;
        const size_t o = lapi(p[0], p[1], p[2], a.pitch, a.ny);
        int q[3] = {p[0], p[1], p[2]};
        q[d] = s;
        const size_t os = lapi(q[0], q[1], q[2], a.pitch, a.ny);
#pragma unroll
        for (int c = 0; c < 4; ++c) a.ev[4 * d + c][o] = a.ev[4 * d + c][os];
    }
}

// Resident blocks of a viscous kernel on the current device, with its
// shared-memory attribute set; computed once per device (0 on failure).
template <typename K>
int vis_resident(K kernel, int threads, size_t smem, int* cache) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (cache[dev] > 0) return cache[dev];
    int sms = 0, per = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess)
        return 0;
    cache[dev] = sms * per;
    return cache[dev];
}

// persistent launch: min(work items, resident blocks); the CTA is VBX x BY
template <int BY, typename K>
int launch_vis(K kernel, size_t smem, int* cache, const ws_grid* g, const VisArgs& a,
               cudaStream_t st) {
    const int res = vis_resident(kernel, VBX * BY, smem, cache);
    if (res <= 0) return fail(WS_ERR_CUDA, "cannot prepare the viscous kernels");
    const long items = vis_items<BY>(g->nx, g->ny, g->nz);
    const int blocks = (int)std::max(1L, std::min(items, (long)res));
    kernel<<<blocks, VBX * BY, smem, st>>>(a);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
}

int flux_cache[8][64], div_cache[8][64];

}  // namespace

// flux fields held: 12, or 9 on Cartesian grids (Ev_x[1] = Ev_y[0] = s12,
// Ev_x[2] = Ev_z[0] = s13, Ev_y[2] = Ev_z[1] = s23 share a field)
static int vis_nfields(const ws_grid* g) { return g->metrics_uniform ? 9 : 12; }

size_t vis_workspace_bytes(const ws_grid* g) {
    return vis_nfields(g) * (size_t)lap_pitch(g->nx) * (g->ny + 8) * (g->nz + 8) *
           sizeof(double);
}

namespace {
VisArgs vis_args(const ws_grid* g, const ws_viscous* vis, const ws_field* prims,
                 const ws_metrics* m, ws_soa du, void* ws, bool accumulate) {
    VisArgs a{};
    if (prims)
        for (int q = 0; q < 4; ++q) {
            a.prim[q] = prims[q].ptr;
            a.ppitch[q] = prims[q].pitch;
        }
    a.uniform = g->metrics_uniform ? 1 : 0;
    if (!a.uniform) {
        const ws_field* mf = &m->akx;
        for (int c = 0; c < 10; ++c) {
            a.met[c] = mf[c].ptr;
            a.mpitch[c] = mf[c].pitch;
        }
    }
    ws_field ef[12];
    vis_flux_fields(g, ws, ef);
    for (int c = 0; c < 12; ++c) a.ev[c] = ef[c].ptr;
    a.epitch = ef[0].pitch;
    a.du = du.ptr;
    a.du_pitch = du.pitch;
    a.du_ly = du.length_Y;
    a.du_lz = du.length_Z;
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    const double dv = vis->scheme == 6 ? 60.0 : 840.0;
    a.rh[0] = 1.0 / (g->hx * dv); a.rh[1] = 1.0 / (g->hy * dv); a.rh[2] = 1.0 / (g->hz * dv);
    a.h[0] = g->hx; a.h[1] = g->hy; a.h[2] = g->hz;
    a.any_d0 = 0;
    for (int d = 0; d < 3; ++d) {
        a.d0lo[d] = vis->d0_bound[2 * d] && g->face_kind[2 * d] != WS_FACE_EXTERNAL;
        a.d0hi[d] = vis->d0_bound[2 * d + 1] && g->face_kind[2 * d + 1] != WS_FACE_EXTERNAL;
        a.any_d0 |= a.d0lo[d] | a.d0hi[d];
    }
    // OCFD_init.cpp:380-396
    const double Cp = 1.0 / ((g->gamma - 1.0) * g->ama * g->ama);
    a.tsb = 110.4 / vis->ref_t;
    a.amu_c0 = 1.0 / vis->re * (1.0 + 110.4 / vis->ref_t);
    a.vfc = Cp / vis->pr;
    a.accumulate = accumulate ? 1 : 0;
    return a;
}
}  // namespace

void vis_flux_fields(const ws_grid* g, void* ws, ws_field ev[12]) {
    static const int shared9[12] = {0, 1, 2, 3, 1, 4, 5, 6, 2, 5, 7, 8};
    const uint32_t ep = lap_pitch(g->nx);
    const size_t nlap = (size_t)ep * (g->ny + 8) * (g->nz + 8);
    double* e = static_cast<double*>(ws);
    const bool nine = vis_nfields(g) == 9;
    for (int c = 0; c < 12; ++c) ev[c] = ws_field{e + (nine ? shared9[c] : c) * nlap, ep, 0};
}

int launch_vis_flux(const ws_grid* g, const ws_viscous* vis, const ws_field prims[4],
                    const ws_metrics* m, void* ws, cudaStream_t st) {
    const VisArgs a = vis_args(g, vis, prims, m, ws_soa{}, ws, false);
    const bool cd6 = vis->scheme == 6, uni = a.uniform != 0, d0 = a.any_d0 != 0;
    const int c = (cd6 ? 0 : 4) + (uni ? 0 : 2) + (d0 ? 1 : 0);
    int rc;
    switch (c) {
        case 0: rc = launch_vis<FBY>(vis_flux_kernel<3, true, false>, vis_flux_smem<3>(), flux_cache[c], g, a, st); break;
        case 1: rc = launch_vis<FBY>(vis_flux_kernel<3, true, true>, vis_flux_smem<3>(), flux_cache[c], g, a, st); break;
        case 2: rc = launch_vis<FBY>(vis_flux_kernel<3, false, false>, vis_flux_smem<3>(), flux_cache[c], g, a, st); break;
        case 3: rc = launch_vis<FBY>(vis_flux_kernel<3, false, true>, vis_flux_smem<3>(), flux_cache[c], g, a, st); break;
        case 4: rc = launch_vis<FBY>(vis_flux_kernel<4, true, false>, vis_flux_smem<4>(), flux_cache[c], g, a, st); break;
        case 5: rc = launch_vis<FBY>(vis_flux_kernel<4, true, true>, vis_flux_smem<4>(), flux_cache[c], g, a, st); break;
        case 6: rc = launch_vis<FBY>(vis_flux_kernel<4, false, false>, vis_flux_smem<4>(), flux_cache[c], g, a, st); break;
        default: rc = launch_vis<FBY>(vis_flux_kernel<4, false, true>, vis_flux_smem<4>(), flux_cache[c], g, a, st); break;
    }
    if (rc) return rc;
    VisGhostArgs ga{};
    for (int c = 0; c < 12; ++c) ga.ev[c] = a.ev[c];
    ga.pitch = a.epitch;
    ga.nx = g->nx; ga.ny = g->ny; ga.nz = g->nz;
    for (int f = 0; f < 6; ++f) ga.kind[f] = g->face_kind[f];
    const long total = 8L * ((long)g->ny * g->nz + (long)g->nx * g->nz + (long)g->nx * g->ny);
    const int blocks = (int)std::min<long>((total + 255) / 256, 148L * 16);
    vis_ghost_kernel<<<blocks, 256, 0, st>>>(ga);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
}

int launch_vis_div(const ws_grid* g, const ws_viscous* vis, const ws_metrics* m, ws_soa du,
                   void* ws, bool accumulate, cudaStream_t st) {
    const VisArgs a = vis_args(g, vis, nullptr, m, du, ws, accumulate);
    const bool cd6 = vis->scheme == 6, uni = a.uniform != 0, d0 = a.any_d0 != 0;
    const int c = (cd6 ? 0 : 4) + (uni ? 0 : 2) + (d0 ? 1 : 0);
    switch (c) {
        case 0: return launch_vis<VBY>(vis_div_kernel<3, true, false>, vis_div_smem<3>(), div_cache[c], g, a, st);
        case 1: return launch_vis<VBY>(vis_div_kernel<3, true, true>, vis_div_smem<3>(), div_cache[c], g, a, st);
        case 2: return launch_vis<VBY>(vis_div_kernel<3, false, false>, vis_div_smem<3>(), div_cache[c], g, a, st);
        case 3: return launch_vis<VBY>(vis_div_kernel<3, false, true>, vis_div_smem<3>(), div_cache[c], g, a, st);
        case 4: return launch_vis<VBY>(vis_div_kernel<4, true, false>, vis_div_smem<4>(), div_cache[c], g, a, st);
        case 5: return launch_vis<VBY>(vis_div_kernel<4, true, true>, vis_div_smem<4>(), div_cache[c], g, a, st);
        case 6: return launch_vis<VBY>(vis_div_kernel<4, false, false>, vis_div_smem<4>(), div_cache[c], g, a, st);
        default: return launch_vis<VBY>(vis_div_kernel<4, false, true>, vis_div_smem<4>(), div_cache[c], g, a, st);
    }
}

// du[1..4] += (accumulate) or = viscous terms; du[0] = 0 when storing.
// prims: u, v, w, T LAP fields with ghosts filled; ws: vis_workspace_bytes(g).
int launch_du_vis(const ws_grid* g, const ws_viscous* vis, const ws_field prims[4],
                  const ws_metrics* m, ws_soa du, void* ws, bool accumulate, cudaStream_t st) {
    int rc = launch_vis_flux(g, vis, prims, m, ws, st);
    return rc ? rc : launch_vis_div(g, vis, m, du, ws, accumulate, st);
}

int check_viscous(const ws_viscous* vis) {
    if (!vis) return fail(WS_ERR_INVALID, "viscous parameters are NULL");
    if (!(vis->re > 0) || !(vis->pr > 0) || !(vis->ref_t > 0))
        return fail(WS_ERR_INVALID, "viscous: need Re, Pr, Ref_T > 0");
    if (vis->scheme != 6 && vis->scheme != 8)
        return fail(WS_ERR_INVALID, "viscous: scheme must be 6 (CD6) or 8 (CD8)");
    return WS_OK;
}

}  // namespace ws
