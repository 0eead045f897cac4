// viscous.cu -- viscous terms of the Navier-Stokes RHS on the GPU.
//
// Replaces du_vis_Jacobian3d (OCFD_Stream.cpp:229-345): per RHS the reference
// runs 12 derivative kernels for u, v, w, T (du_viscous_Jacobian3d_init,
// OCFD_NS_Jacobian3d.cpp:455-475), and per direction the flux kernel
// vis_flux_ker (:477-624), a halo exchange of its four outputs, four
// derivative kernels and four accumulation kernels (YF_Pe_XF) -- 40 launches
// and 12 derivative fields in HBM.  Here:
//   vis_flux_kernel: one pass over the interior computes the 12 first
//     derivatives in registers (CD6/CD8 through the ghosts, value / h), the
//     Sutherland viscosity (get_Amu_kernal, commen_kernel.cpp:123-132) and
//     the viscous fluxes Ev1..4 of all three directions (12 LAP fields);
//   ghost fill of those 12 fields by the face kinds (one launch per 8 fields);
//   vis_div_kernel: one pass adds J * d(Ev_dir)/d(dir) of the three
//     directions to du[1..4] (or stores it, for the fused RK stage), x then y
//     then z as the reference accumulates.
// Memory-bound: per cell ~32 B of primitives in (stencil re-reads hit L1/L2),
// 96 B of fluxes out and in again, 32-64 B of du.
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
    double rh[3];              // 1/h
    double tsb, amu_c0, vfc;   // Sutherland constants, Cp/Pr
    int uniform, accumulate;
};

__device__ __forceinline__ size_t lapi(int X, int Y, int Z, uint32_t pitch, int ny) {
    return (size_t)X + (size_t)pitch * ((size_t)Y + (size_t)(ny + 8) * (size_t)Z);
}

// central first difference (times h) along DIR at LAP point (X, Y, Z):
// OCFD_Schemes.cpp:97-104 (CD6) and :134-142 (CD8)
template <int R, int DIR>
__device__ __forceinline__ double cdiff(const double* f, uint32_t pitch, int ny, int X, int Y,
                                        int Z) {
    const long s = DIR == 0 ? 1 : DIR == 1 ? (long)pitch : (long)pitch * (ny + 8);
    const double* c = f + lapi(X, Y, Z, pitch, ny);
    if (R == 3)
        return (45.0 * (__ldg(c + s) - __ldg(c - s)) - 9.0 * (__ldg(c + 2 * s) - __ldg(c - 2 * s)) +
                (__ldg(c + 3 * s) - __ldg(c - 3 * s))) / 60.0;
    return (672.0 * (__ldg(c + s) - __ldg(c - s)) - 168.0 * (__ldg(c + 2 * s) - __ldg(c - 2 * s)) +
            32.0 * (__ldg(c + 3 * s) - __ldg(c - 3 * s)) -
            3.0 * (__ldg(c + 4 * s) - __ldg(c - 4 * s))) / 840.0;
}

// Blocks of 32 x 8 threads cover 32 x 8 cells of one plane, so the x and y
// neighbours of a stencil are mostly read by the same block (L1); the grid
// strides over the (x tile, y tile, plane) space.
template <int R>
__global__ void __launch_bounds__(256) vis_flux_kernel(const __grid_constant__ VisArgs a) {
    const int tx = (a.nx + 31) / 32, ty = (a.ny + 7) / 8;
    const long ntile = (long)tx * ty * a.nz;
    for (long b = blockIdx.x; b < ntile; b += gridDim.x) {
        const int i = (int)(b % tx) * 32 + threadIdx.x % 32;
        const long r = b / tx;
        const int j = (int)(r % ty) * 8 + threadIdx.x / 32, k = (int)(r / ty);
        if (i >= a.nx || j >= a.ny) continue;
        const int X = i + 4, Y = j + 4, Z = k + 4;
        // derivatives along the computational directions: g[q][dir]
        double g[4][3];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            g[q][0] = cdiff<R, 0>(a.prim[q], a.ppitch[q], a.ny, X, Y, Z) * a.rh[0];
            g[q][1] = cdiff<R, 1>(a.prim[q], a.ppitch[q], a.ny, X, Y, Z) * a.rh[1];
            g[q][2] = cdiff<R, 2>(a.prim[q], a.ppitch[q], a.ny, X, Y, Z) * a.rh[2];
        }
        double m[9], aj = 1.0;
        if (a.uniform) {
#pragma unroll
            for (int c = 0; c < 9; ++c) m[c] = (c == 0 || c == 4 || c == 8) ? 1.0 : 0.0;
        } else {
#pragma unroll
            for (int c = 0; c < 9; ++c) m[c] = __ldg(a.met[c] + lapi(X, Y, Z, a.mpitch[c], a.ny));
            aj = __ldg(a.met[9] + lapi(X, Y, Z, a.mpitch[9], a.ny));
        }
        // physical gradients (chain rule with akx..asz)
        double gx[4], gy[4], gz[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            gx[q] = g[q][0] * m[0] + g[q][1] * m[3] + g[q][2] * m[6];
            gy[q] = g[q][0] * m[1] + g[q][1] * m[4] + g[q][2] * m[7];
            gz[q] = g[q][0] * m[2] + g[q][1] * m[5] + g[q][2] * m[8];
        }
        const double Tc = __ldg(a.prim[3] + lapi(X, Y, Z, a.ppitch[3], a.ny));
        const double amu = a.amu_c0 * sqrt(Tc * Tc * Tc) / (a.tsb + Tc);
        const double div = gx[0] + gy[1] + gz[2];
        const double s11 = (2.0 * gx[0] - 2.0 / 3.0 * div) * amu;
        const double s22 = (2.0 * gy[1] - 2.0 / 3.0 * div) * amu;
        const double s33 = (2.0 * gz[2] - 2.0 / 3.0 * div) * amu;
        const double s12 = (gy[0] + gx[1]) * amu;
        const double s13 = (gz[0] + gx[2]) * amu;
        const double s23 = (gz[1] + gy[2]) * amu;
        const double amuk = amu * a.vfc;
        const double u = __ldg(a.prim[0] + lapi(X, Y, Z, a.ppitch[0], a.ny));
        const double v = __ldg(a.prim[1] + lapi(X, Y, Z, a.ppitch[1], a.ny));
        const double w = __ldg(a.prim[2] + lapi(X, Y, Z, a.ppitch[2], a.ny));
        const double E1 = u * s11 + v * s12 + w * s13 + amuk * gx[3];
        const double E2 = u * s12 + v * s22 + w * s23 + amuk * gy[3];
        const double E3 = u * s13 + v * s23 + w * s33 + amuk * gz[3];
        const size_t o = lapi(X, Y, Z, a.epitch, a.ny);
#pragma unroll
        for (int dir = 0; dir < 3; ++dir) {
            const double kx = m[3 * dir] * aj, ky = m[3 * dir + 1] * aj, kz = m[3 * dir + 2] * aj;
            a.ev[4 * dir + 0][o] = kx * s11 + ky * s12 + kz * s13;
            a.ev[4 * dir + 1][o] = kx * s12 + ky * s22 + kz * s23;
            a.ev[4 * dir + 2][o] = kx * s13 + ky * s23 + kz * s33;
            a.ev[4 * dir + 3][o] = kx * E1 + ky * E2 + kz * E3;
        }
    }
}

template <int R>
__global__ void __launch_bounds__(256) vis_div_kernel(const __grid_constant__ VisArgs a) {
    const int tx = (a.nx + 31) / 32, ty = (a.ny + 7) / 8;
    const long ntile = (long)tx * ty * a.nz;
    for (long b = blockIdx.x; b < ntile; b += gridDim.x) {
        const int i = (int)(b % tx) * 32 + threadIdx.x % 32;
        const long r = b / tx;
        const int j = (int)(r % ty) * 8 + threadIdx.x / 32, k = (int)(r / ty);
        if (i >= a.nx || j >= a.ny) continue;
        const int X = i + 4, Y = j + 4, Z = k + 4;
        const double aj = a.uniform ? 1.0 : __ldg(a.met[9] + lapi(X, Y, Z, a.mpitch[9], a.ny));
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double* d = a.du + (size_t)i +
                        (size_t)a.du_pitch * ((size_t)j + (size_t)a.du_ly *
                                                             ((size_t)k + (size_t)a.du_lz * (q + 1)));
            double acc = a.accumulate ? *d : 0.0;
            acc += aj * (cdiff<R, 0>(a.ev[q], a.epitch, a.ny, X, Y, Z) * a.rh[0]);
            acc += aj * (cdiff<R, 1>(a.ev[4 + q], a.epitch, a.ny, X, Y, Z) * a.rh[1]);
            acc += aj * (cdiff<R, 2>(a.ev[8 + q], a.epitch, a.ny, X, Y, Z) * a.rh[2]);
            *d = acc;
        }
        if (!a.accumulate)
            a.du[(size_t)i + (size_t)a.du_pitch * ((size_t)j + (size_t)a.du_ly * (size_t)k)] = 0.0;
    }
}

int grid_for(const ws_grid* g) {
    const long tiles = (long)((g->nx + 31) / 32) * ((g->ny + 7) / 8) * g->nz;
    return (int)std::max(1L, std::min(tiles, 148L * 8));
}

}  // namespace

size_t vis_workspace_bytes(const ws_grid* g) {
    return 12 * (size_t)lap_pitch(g->nx) * (g->ny + 8) * (g->nz + 8) * sizeof(double);
}

// du[1..4] += (accumulate) or = viscous terms; du[0] = 0 when storing.
// prims: u, v, w, T LAP fields with ghosts filled; ws: vis_workspace_bytes(g).
int launch_du_vis(const ws_grid* g, const ws_viscous* vis, const ws_field prims[4],
                  const ws_metrics* m, ws_soa du, void* ws, bool accumulate, cudaStream_t st) {
    VisArgs a{};
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
    const uint32_t ep = lap_pitch(g->nx);
    const size_t nlap = (size_t)ep * (g->ny + 8) * (g->nz + 8);
    double* e = static_cast<double*>(ws);
    for (int c = 0; c < 12; ++c) a.ev[c] = e + c * nlap;
    a.epitch = ep;
    a.du = du.ptr;
    a.du_pitch = du.pitch;
    a.du_ly = du.length_Y;
    a.du_lz = du.length_Z;
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    a.rh[0] = 1.0 / g->hx; a.rh[1] = 1.0 / g->hy; a.rh[2] = 1.0 / g->hz;
    // OCFD_init.cpp:380-396
    const double Cp = 1.0 / ((g->gamma - 1.0) * g->ama * g->ama);
    a.tsb = 110.4 / vis->ref_t;
    a.amu_c0 = 1.0 / vis->re * (1.0 + 110.4 / vis->ref_t);
    a.vfc = Cp / vis->pr;
    a.accumulate = accumulate ? 1 : 0;
    const int blocks = grid_for(g);
    if (vis->scheme == 6) vis_flux_kernel<3><<<blocks, 256, 0, st>>>(a);
    else vis_flux_kernel<4><<<blocks, 256, 0, st>>>(a);
    WS_CUDA(cudaGetLastError());
    ws_field ef[12];
    for (int c = 0; c < 12; ++c) ef[c] = ws_field{a.ev[c], ep, 0};
    int rc = launch_ghost_fill(g, ef, 8, st);
    if (!rc) rc = launch_ghost_fill(g, ef + 8, 4, st);
    if (rc) return rc;
    if (vis->scheme == 6) vis_div_kernel<3><<<blocks, 256, 0, st>>>(a);
    else vis_div_kernel<4><<<blocks, 256, 0, st>>>(a);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
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
