// ws_internal.h -- host-side declarations shared by the library's .cu/.cpp files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/windstencil_b200.h"

namespace ws {

// Error reporting: the message of the last failure, per host thread.
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
#define WS_CUDA(call)                                        \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return ::ws::cuda_fail(e_, #call); \
    } while (0)

// Arguments of the fused RHS kernel (one grid).
struct RhsArgs {
    const double* prim[5];     // d, u, v, w, cc at LAP element (0,0,0)
    uint32_t ppitch[5];
    const double* met[10];     // akx..asz, ajac (unused when metrics are uniform)
    uint32_t mpitch[10];
    double* du;
    uint32_t du_pitch, du_ly, du_lz;
    int nx, ny, nz;            // interior extents
    int sx, sy, sz, ex, ey, ez;   // job, LAP coordinates
    int ntx, nty, nzc, zc;     // tiles in x and y, z chunks and chunk length
    double rhx, rhy, rhz;      // 1/h
    double eps2, hrg, c1, c3, gm1;
};

// Tile configurations compiled into the library.
struct TileCfg {
    int bx, by, threads;
};
int num_tile_cfgs();
TileCfg tile_cfg(int i);
int find_tile_cfg(int bx, int by, int threads);   // index or -1

// Launch the fused RHS for one grid; cfg indexes the compiled tile shapes.
int launch_rhs(const RhsArgs& a, int precision, bool uniform, int cfg, int ctas,
               cudaStream_t st);
int rhs_max_ctas(int precision, bool uniform, int cfg);   // resident CTAs on the device

// Field kernels (field_kernels.cu).
struct FieldArgs {
    int nx, ny, nz;
};
int launch_sound_speed(const ws_grid* g, ws_job job, ws_field T, ws_field cc, cudaStream_t st);
int launch_ghost_fill(const ws_grid* g, const ws_field* f, int nf, cudaStream_t st);
int launch_cons_to_prim(const ws_grid* g, ws_soa f, ws_field d, ws_field u, ws_field v,
                        ws_field w, ws_field T, ws_field P, int* status, cudaStream_t st);
int launch_prim_to_cons(const ws_grid* g, ws_field d, ws_field u, ws_field v, ws_field w,
                        ws_field T, ws_soa f, cudaStream_t st);
int launch_time_advance(const ws_grid* g, int krk, double dt, ws_soa f, ws_soa fn, ws_soa du,
                        cudaStream_t st);
// Fused stage: f <- stage(krk), then cons->prim (d,u,v,w,T interiors) and
// cc on the interior; status word set on non-finite/rho<=0/p<=0.
int launch_stage_update(const ws_grid* g, int krk, double dt, ws_soa f, ws_soa fn, ws_soa du,
                        const ws_field prims[6], int* status, cudaStream_t st);
// Fill ghosts of d,u,v,w,T and recompute cc on ghost layers only.
int launch_ghost_fill_prims(const ws_grid* g, const ws_field prims[6], cudaStream_t st);

uint32_t lap_pitch(uint32_t nx);

}  // namespace ws
