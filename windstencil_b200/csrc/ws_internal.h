// ws_internal.h -- host-side declarations shared by the library's .cu/.cpp files.
#pragma once
#include <cuda.h>             // CUtensorMap (types only; the encoder is fetched at run time)
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#include <string>
#include <vector>

#include "../../include/windstencil_b200.h"

namespace ws {

// Grid checks shared by every entry point (extents, constants, face kinds,
// precision); WS_OK or the error code with its message set.
int validate_grid(const ws_grid* g);
// the library's device error word of the current device (launches without a
// per-grid status word report into it); NULL when it cannot be resolved
int* device_error_word();
// A maximum wave speed read back from launch_max_speed usable for a CFL time
// step: finite and positive (the reduction carries NaN and +inf through as
// NaN bits, so one bad cell makes the whole grid's maximum unusable).
inline bool wave_speed_ok(double m) { return std::isfinite(m) && m > 0; }
// a device status word as an error code: bit 2 (a staging wait gave up) ->
// WS_ERR_TIMEOUT, bit 1 (non-finite or non-physical state) -> WS_ERR_NONFINITE
inline int status_code(int v) {
    return (v & 2) ? WS_ERR_TIMEOUT : v ? WS_ERR_NONFINITE : WS_OK;
}
// any face of kind WS_FACE_EXTERNAL (ghosts written by the caller's halo exchange)
bool has_external(const ws_grid* g);
// 4 planes along `axis` of nf LAP fields <-> halo buffer [nf][b2][b1][b0]
// (b = the planes' box: 4 along the axis, the interior along the others):
// pack reads the interior planes next to face `side`, unpack writes the ghost
// planes beyond it
int launch_halo(const ws_grid* g, const ws_field* f, int nf, int axis, int side, double* buf,
                bool pack, cudaStream_t st);

// Error reporting: the message of the last failure, per host thread.
void set_error(const std::string& msg);
std::string last_error_message();       // this thread's last failure message
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
    int clo[4];                // CLOSURE faces: x-, x+, y-, y+ (0/1)
    // fused SSP-RK3 stage epilogue (solver and batches, whole interior):
    // f_out <- stage(fn, f_in, dt*du); d,u,v,w,T,cc of the new state into the
    // interiors of p_out (a second set of LAP fields: other CTAs still read
    // the current primitives).  f_in may alias f_out (stages 2 and 3).
    // f_in, fn and f_out share one SoA shape, the p_out fields one pitch.
    ws_soa f_in, fn, f_out;
    double* p_out[6];
    uint32_t p_pitch;
    double dt, rcv, rama;      // dt, 1/cv, 1/Ama
    int* status;
    // viscous terms of the stage (ptr NULL: none): du[0..4] added to the
    // inviscid RHS before the update; same SoA shape as fn
    ws_soa dvis;
    // TMA staging (tma != 0): per primitive, a map of its LAP array with the
    // (BX+8) x (BY+8) box of a plane and one with the BX x BY centre box.
    // Set only when every box start is 16-byte aligned (even job start x,
    // even pitches, 16-byte aligned fields); otherwise staging uses cp.async.
    int tma;
    // > 0 only in the failure-path test (environment WS_TEST_STAGE_WAIT):
    // the first staging wait polls, this many times, an mbarrier nothing
    // arrives on, so the kernel takes its timeout path (status bit 2, early
    // stop) without any fault
    int hold_polls;
    CUtensorMap tm_box[5], tm_ctr[5];
};

// fill the epilogue fields of `a` for one stage (WS_ERR_INVALID when the
// SoA shapes or the p_out pitches differ)
int set_rhs_stage(RhsArgs& a, const ws_grid* g, ws_soa f_in, ws_soa fn, ws_soa f_out,
                  const ws_field p_out[6], double dt, int* status);
// resident-CTA count for one grid's launch (0 on failure)
int rhs_ctas(const ws_grid* g, const RhsArgs& a, int cfg, bool stage);
// One fused RHS + SSP-RK3 stage krk over the whole interior (Cartesian):
// reads primitives p_in (ghosts filled), f_in and fn; writes f_out and the
// new primitives p_out.
// dvis.ptr may be NULL (no viscous terms).
// du: the grid's RHS buffer, which the line passes accumulate into (with
// viscous terms it holds them, and dvis is the same buffer).
int rhs_stage_enqueue(const ws_grid* g, const ws_field p_in[6], ws_soa f_in, ws_soa fn,
                      ws_soa f_out, const ws_field p_out[6], double dt, int krk, int* status,
                      ws_soa dvis, ws_soa du, ws_tile tile, cudaStream_t st);

// Viscous terms (viscous.cu): workspace size, parameter check, and du[1..4]
// += (accumulate) or = the viscous terms (du[0] = 0 when storing) from the
// LAP fields u, v, w, T (ghosts filled).
size_t vis_workspace_bytes(const ws_grid* g);
int check_viscous(const ws_viscous* vis);
int launch_du_vis(const ws_grid* g, const ws_viscous* vis, const ws_field prims[4],
                  const ws_metrics* m, ws_soa du, void* ws, bool accumulate, cudaStream_t st);
// the same in two passes: fluxes (+ the ghosts the divergence reads: each
// direction's fluxes along their own axis, by the face kinds), then the
// divergence; between them a slab's caller exchanges the x-direction
// fluxes' halos (EXTERNAL faces).  The workspace's 12 flux fields: direction
// dir, component q at ev[4 * dir + q].
void vis_flux_fields(const ws_grid* g, void* ws, ws_field ev[12]);
int launch_vis_flux(const ws_grid* g, const ws_viscous* vis, const ws_field prims[4],
                    const ws_metrics* m, void* ws, cudaStream_t st);
int launch_vis_div(const ws_grid* g, const ws_viscous* vis, const ws_metrics* m, ws_soa du,
                   void* ws, bool accumulate, cudaStream_t st);

// Tile configurations compiled into the library.
struct TileCfg {
    int bx, by, threads;
};
int num_tile_cfgs();
TileCfg tile_cfg(int i);
int find_tile_cfg(int bx, int by, int threads);   // index or -1
int default_cfg(int precision, bool stage);       // tuned default shape (stage kernel or plain RHS)

// The RHS as three line passes x, y, z (pencil_impl.cuh), wpb warps per CTA
// (0: the default), one CTA per SM; CLOSURE faces of the grid (a.clo) run the
// x and y passes' closure instances.  krk 0: the RHS into
// a.du; krk 1..3: the RHS into a.du, the z pass applying stage krk (a.f_in,
// a.fn -> a.f_out, primitives to a.p_out).  add_x: a.du already holds terms
// the RHS adds to (the viscous terms).
int launch_rhs_pencil(const RhsArgs& a, int precision, bool uniform, int wpb, int krk,
                      bool add_x, cudaStream_t st);
// The line passes over a batch: g the argument table of n Cartesian grids
// (each with its du), woff the x, y and z passes' work prefix tables (n + 1
// entries each, pencil_pass_work); krk as launch_rhs_pencil (no add_x); clo:
// some grid has a CLOSURE face (the x and y passes' closure instances).
int launch_rhs_pencil_batch(const RhsArgs* g, const long* woff, int n, int precision, int krk,
                            bool clo, cudaStream_t st);
long pencil_pass_work(const ws_grid& g, int dir);
// Whether a launch with tile selection `tile` runs the line passes: an
// explicit request (tile_x < 0, threads = 32 x warps per CTA or 0), or the
// default (all zeros); an explicit fused tile runs the fused kernel.
bool use_pencil(const ws_grid* g, ws_tile tile);

// Launch the fused RHS for one grid; cfg indexes the compiled tile shapes.
// krk == 0: write du; krk in 1..3: fused SSP-RK3 stage epilogue (Cartesian).
int launch_rhs(const RhsArgs& a, int precision, bool uniform, int cfg, int ctas, int krk,
               cudaStream_t st);
// resident CTAs of the kernel for (precision, metric kind, CLOSURE faces
// present, tile shape, stage epilogue)
int rhs_max_ctas(int precision, bool uniform, bool closure, int cfg, bool stage);
// Work of a batched RHS launch: items {grid, tile, first plane, end plane}
// in the order the CTAs take them, and the counter they take them by (the
// launch zeroes it first).
struct BatchWork {
    const int4* items;
    int nitems;
    unsigned* counter;
};
// Batched RHS over the grids of a device array of RhsArgs; all grids share
// precision, metric kind and tile shape; closure: some grid has CLOSURE faces.
int launch_rhs_batch(const RhsArgs* grids, const BatchWork& w, int precision, bool uniform,
                     bool closure, int cfg, int ctas, int krk, cudaStream_t st);
// Host-side RhsArgs of one grid and job (tile shape cfg, sweep cap scan).
RhsArgs make_rhs_args(const ws_grid* g, ws_job job, const ws_field prims[5],
                      const ws_metrics* m, ws_soa du, int cfg, int scan);

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
// Fill ghosts of d,u,v,w,T and recompute cc on ghost layers only.
int launch_ghost_fill_prims(const ws_grid* g, const ws_field prims[6], cudaStream_t st);

uint32_t lap_pitch(uint32_t nx);

// Batched ghost fill: per-grid argument blocks (opaque, size below) in
// device memory and a block table int2{grid, chunk}.
size_t ghost_args_size();
void fill_ghost_args(void* out, const ws_grid* g, const ws_field prims[6]);
long ghost_chunks(const ws_grid* g);
int launch_ghost_fill_batch(const void* grids, const int2* tab, int nblocks, cudaStream_t st);

// Device-resident state of one grid (used by the solver, batches and the
// server): f[2] and du SoA, two sets of d,u,v,w,T,cc LAP fields and a
// status word, in one allocation.  f[cur] is the current state and pr[cur]
// its primitives; a step writes the other buffer of each.
struct GridState {
    ws_grid g{};
    void* mem = nullptr;
    size_t bytes = 0;
    ws_soa f[2]{}, du{};
    ws_field pr[2][6]{};
    int* status = nullptr;
    int cur = 0;
    double dt = 0.0;
    const ws_field* prims() const { return pr[cur]; }
    // fused-stage arguments [2 * c + (stage == 2)] for state buffer c (with
    // their tensor maps), kept while the tile shape, sweep cap and dt stay
    // the same, so re-forming a batch does not re-encode them
    std::vector<RhsArgs> args;
    int args_cfg = -1, args_zc = 0;
    double args_dt = 0.0;
};
size_t grid_state_bytes(const ws_grid& g);
// stream-ordered allocation from the device's default memory pool
int grid_state_alloc(GridState& s, const ws_grid& g, cudaStream_t st);
void grid_state_free(GridState& s, cudaStream_t st);
// upload a dense conserved state and derive d,u,v,w,T,cc on the interior
int grid_state_upload(GridState& s, const double* f_host, cudaStream_t st);
int grid_state_download(GridState& s, double* f_host, cudaStream_t st);   // no sync
// d,u,v,w,T,cc (interiors) of the current conserved state f[cur]
int grid_state_derive(GridState& s, cudaStream_t st);

// A set of grids stepped together: one batched launch per kernel per stage.
// The kernel a batch of these grids runs for tile selection `tile`: -1 for
// the line passes (the default, or asked for by tile_x < 0), else a fused
// tile configuration (-2: not compiled).
int batch_kernel_cfg(const std::vector<GridState*>& grids, ws_tile tile);

class BatchRunner {
  public:
    BatchRunner() = default;
    ~BatchRunner();
    BatchRunner(const BatchRunner&) = delete;
    BatchRunner& operator=(const BatchRunner&) = delete;
    // (re)build the device tables for `grids` (all of one precision);
    // invalidates captured graphs
    // cfg < 0: the line passes (pencil_impl.cuh), else the fused kernel's tile
    int build(const std::vector<GridState*>& grids, int cfg, int zc, cudaStream_t st);
    int enqueue_rhs(cudaStream_t st);
    // the first RK stage only (leaves the current state unchanged; tuning)
    int enqueue_stage1(cudaStream_t st);
    // one SSP-RK3 step of every grid from its current buffer into the other
    int enqueue_step(cudaStream_t st);
    // nsteps steps (graph replay); flips every grid's current buffer
    int step(int nsteps, cudaStream_t st);
    // the same without graphs (a batch that changes every few steps)
    int step_eager(int nsteps, cudaStream_t st);
    int size() const { return (int)grids_.size(); }
    int cfg() const { return cfg_; }
    int zc() const { return zc_; }
    void release(cudaStream_t st);

  private:
    int upload_tables(cudaStream_t st);
    std::vector<GridState*> grids_;
    int precision_ = 0, cfg_ = 0, zc_ = 1 << 30, ctas_ = 0;
    bool closure_ = false;          // some grid has CLOSURE faces
    bool pencil_ = false;           // line passes instead of the fused kernel
    const long* d_woff_ = nullptr;  // line passes: x, y, z work prefix tables
    void* dev_ = nullptr;           // device tables
    size_t dev_bytes_ = 0;
    // With c = cur ^ p (p = step parity since build), a step reads f[c] and
    // writes f[1-c]; stages 1 and 3 read primitives pr[c] and write pr[1-c],
    // stage 2 the reverse.  d_rhs_[2*p + (stage == 2)] holds the RHS
    // arguments (with the stage epilogue) of every grid for that case, and
    // d_ghost_[s] the ghost-fill arguments of primitive set pr[cur ^ s].
    RhsArgs* d_rhs_[4] = {nullptr, nullptr, nullptr, nullptr};
    void* d_ghost_[2] = {nullptr, nullptr};
    BatchWork work_{nullptr, 0, nullptr};   // the RHS launches' work items
    int2* d_gtab_ = nullptr;
    int n_gtab_ = 0;
    int parity_ = 0;
    cudaStream_t cap_ = nullptr;
    cudaGraphExec_t exec_[2] = {nullptr, nullptr};
    void drop_graphs();
    std::vector<unsigned char> host_;
};

}  // namespace ws
