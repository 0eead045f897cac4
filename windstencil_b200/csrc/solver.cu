// solver.cu -- one grid, device-resident state, SSP-RK3 steps from CUDA graphs
// (Euler, or Navier-Stokes with ws_solver_set_viscous).
//
// Replaces the reference's time loop (src/solver/OCFD_NS_Solver.cpp:64-90)
// for the Euler system.  The reference's pf/pfn pointer swap becomes two
// captured graphs (state buffer 0 -> 1 and 1 -> 0), each holding three
// stages of
//   ghost fill (d,u,v,w,T,cc) -> fused RHS with the SSP-RK3 stage epilogue,
// which writes the stage's conserved state and its primitives into the other
// primitive buffer.  The reference's shipped loop runs stage 1 only
// (`KRK <= 1`, :77); all three stage formulas of OCFD_time.cpp:15-65 are used.
#include <cstring>
#include <vector>

#include "ws_internal.h"

namespace ws {
int rhs_enqueue(const ws_grid* g, ws_job job, const ws_field prims[5], const ws_metrics* m,
                ws_soa du, ws_tile tile, cudaStream_t st);
int launch_max_speed(const ws_grid* g, const ws_field prims[6], unsigned long long* out,
                     cudaStream_t st);
}  // namespace ws

using namespace ws;

struct ws_solver {
    GridState s;
    unsigned long long* scratch = nullptr;   // max wave speed
    cudaStream_t cap = nullptr;              // private capture stream
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    double graph_dt = 0.0;
    ws_tile tile{0, 0, 0, 0};
    // Navier-Stokes: viscous constants and the workspace of their fluxes
    bool viscous = false;
    ws_viscous vis{};
    void* vis_ws = nullptr;
    int next_stage = 1;                      // ws_solver_stage: the stage due next
    bool stage_begun = false;                // its first half is enqueued
};

namespace {
void drop_graphs(ws_solver* s) {
    for (auto& e : s->exec)
        if (e) {
            cudaGraphExecDestroy(e);
            e = nullptr;
        }
}

// du of the current state (ghost fill + RHS, + viscous terms)
int enqueue_rhs(ws_solver* s, cudaStream_t st) {
    GridState& g = s->s;
    int rc = launch_ghost_fill_prims(&g.g, g.prims(), st);
    if (rc) return rc;
    ws_job job{{4, 4, 4}, {g.g.nx + 4, g.g.ny + 4, g.g.nz + 4}};
    const ws_field* p = g.prims();
    const ws_field p5[5] = {p[0], p[1], p[2], p[3], p[5]};
    rc = rhs_enqueue(&g.g, job, p5, nullptr, g.du, s->tile, st);
    if (rc || !s->viscous) return rc;
    const ws_field p4[4] = {p[1], p[2], p[3], p[4]};
    return launch_du_vis(&g.g, &s->vis, p4, nullptr, g.du, s->vis_ws, true, st);
}

// primitives that stage krk of a step from state buffer c reads
const ws_field* stage_input(const GridState& g, int c, int krk) {
    return g.pr[krk == 2 ? 1 - c : c];
}

// Stage krk of the SSP-RK3 step from state buffer c into 1-c; primitives
// pr[c] -> pr[1-c] (stage 1), pr[1-c] -> pr[c] (stage 2), pr[c] -> pr[1-c]
// (stage 3).  First half: ghost fill of the stage's input (faces that are
// not EXTERNAL) and, with viscous terms, their flux pass.
int enqueue_stage_begin(ws_solver* s, int c, int krk, cudaStream_t st) {
    GridState& g = s->s;
    const ws_field* pin = stage_input(g, c, krk);
    int rc = launch_ghost_fill_prims(&g.g, pin, st);
    if (rc || !s->viscous) return rc;
    const ws_field p4[4] = {pin[1], pin[2], pin[3], pin[4]};
    return launch_vis_flux(&g.g, &s->vis, p4, nullptr, s->vis_ws, st);
}

// Second half: the viscous terms' divergence into du (stored), then the fused
// RHS with the stage update, which adds them to the inviscid RHS.
int enqueue_stage_end(ws_solver* s, int c, int krk, double dt, cudaStream_t st) {
    GridState& g = s->s;
    const ws_field* pin = stage_input(g, c, krk);
    const ws_field* pout = g.pr[krk == 2 ? c : 1 - c];
    ws_soa dvis{};
    if (s->viscous) {
        int rc = launch_vis_div(&g.g, &s->vis, nullptr, g.du, s->vis_ws, false, st);
        if (rc) return rc;
        dvis = g.du;
    }
    return rhs_stage_enqueue(&g.g, pin, g.f[1 - c], g.f[c], g.f[1 - c], pout, dt, krk,
                             g.status, dvis, g.du, s->tile, st);
}

int enqueue_stage(ws_solver* s, int c, int krk, double dt, cudaStream_t st) {
    int rc = enqueue_stage_begin(s, c, krk, st);
    return rc ? rc : enqueue_stage_end(s, c, krk, dt, st);
}

// one SSP-RK3 step from state buffer c into 1-c
int enqueue_step(ws_solver* s, int c, double dt, cudaStream_t st) {
    for (int krk = 1; krk <= 3; ++krk)
        if (int rc = enqueue_stage(s, c, krk, dt, st)) return rc;
    return WS_OK;
}

int capture(ws_solver* s, double dt) {
    drop_graphs(s);
    for (int c = 0; c < 2; ++c) {
        cudaGraph_t graph = nullptr;
        WS_CUDA(cudaStreamBeginCapture(s->cap, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(s, c, dt, s->cap);
        cudaError_t e = cudaStreamEndCapture(s->cap, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&s->exec[c], graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    }
    s->graph_dt = dt;
    return WS_OK;
}
}  // namespace

extern "C" {

int ws_solver_create(const ws_grid* g, ws_solver** out) {
    if (!out) return fail(WS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!g) return fail(WS_ERR_INVALID, "grid is NULL");
    if (int rc = validate_grid(g)) return rc;
    if (g->precision != WS_FP64 && g->precision != WS_MIXED)
        return fail(WS_ERR_INVALID, "precision must be WS_FP64 or WS_MIXED");
    if (!g->metrics_uniform)
        return fail(WS_ERR_UNSUPPORTED, "the solver holds Cartesian grids only");
    ws_solver* s = new (std::nothrow) ws_solver();
    if (!s) return fail(WS_ERR_ALLOC, "host allocation failed");
    int rc = grid_state_alloc(s->s, *g, nullptr);
    cudaError_t e = cudaSuccess;
    if (rc == WS_OK) e = cudaMalloc(&s->scratch, sizeof(unsigned long long));
    if (rc == WS_OK && e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&s->cap, cudaStreamNonBlocking);
    if (rc == WS_OK && e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
    if (rc != WS_OK || e != cudaSuccess) {
        ws_solver_destroy(s);
        return rc != WS_OK ? rc : cuda_fail(e, "ws_solver_create");
    }
    *out = s;
    return WS_OK;
}

void ws_solver_destroy(ws_solver* s) {
    if (!s) return;
    drop_graphs(s);
    if (s->cap) cudaStreamDestroy(s->cap);
    cudaFree(s->scratch);
    cudaFree(s->vis_ws);
    grid_state_free(s->s, nullptr);
    cudaStreamSynchronize(nullptr);
    delete s;
}

int ws_solver_set_tile(ws_solver* s, ws_tile tile) {
    if (!s) return fail(WS_ERR_INVALID, "solver is NULL");
    if (tile.tile_x >= 0 && (tile.tile_x || tile.tile_y || tile.threads) &&
        find_tile_cfg(tile.tile_x, tile.tile_y, tile.threads) < 0)
        return fail(WS_ERR_UNSUPPORTED, "tile shape not compiled in this build");
    s->tile = tile;
    drop_graphs(s);
    return WS_OK;
}

int ws_solver_set_viscous(ws_solver* s, const ws_viscous* vis) {
    if (!s) return fail(WS_ERR_INVALID, "solver is NULL");
    if (!vis) {
        s->viscous = false;
        drop_graphs(s);
        return WS_OK;
    }
    if (int rc = check_viscous(vis)) return rc;
    if (!s->vis_ws) {
        WS_CUDA(cudaMalloc(&s->vis_ws, vis_workspace_bytes(&s->s.g)));
        WS_CUDA(cudaMemset(s->vis_ws, 0, vis_workspace_bytes(&s->s.g)));
    }
    s->vis = *vis;
    s->viscous = true;
    drop_graphs(s);
    return WS_OK;
}

int ws_solver_save(ws_solver* s, const char* path, int32_t istep, double tt,
                   ws_stream_t stream) {
    if (!s || !path) return fail(WS_ERR_INVALID, "NULL argument");
    const ws_grid& g = s->s.g;
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    std::vector<double> f(5 * n), p(5 * n);
    int rc = ws_solver_get_state(s, f.data(), stream);
    if (rc) return rc;
    const double cv = 1.0 / (g.gamma * (g.gamma - 1.0) * g.ama * g.ama);
    for (size_t c = 0; c < n; ++c) {    // cons_to_pri_kernel, commen_kernel.cpp:78-110
        const double d1 = f[c];
        const double u1 = f[n + c] / d1, v1 = f[2 * n + c] / d1, w1 = f[3 * n + c] / d1;
        double T1 = f[4 * n + c] - 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1);
        T1 = T1 / (d1 * cv);
        p[c] = d1; p[n + c] = u1; p[2 * n + c] = v1; p[3 * n + c] = w1; p[4 * n + c] = T1;
    }
    return ws_restart_write(path, g.nx, g.ny, g.nz, istep, tt, p.data());
}

int ws_solver_load(ws_solver* s, const char* path, int32_t* istep, double* tt,
                   ws_stream_t stream) {
    if (!s || !path || !istep || !tt) return fail(WS_ERR_INVALID, "NULL argument");
    const ws_grid& g = s->s.g;
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    std::vector<double> p(5 * n), f(5 * n);
    int rc = ws_restart_read(path, g.nx, g.ny, g.nz, istep, tt, p.data());
    if (rc) return rc;
    const double cv = 1.0 / (g.gamma * (g.gamma - 1.0) * g.ama * g.ama);
    for (size_t c = 0; c < n; ++c) {    // pri_to_cons_kernel, commen_kernel.cpp:33-70
        const double d = p[c], u = p[n + c], v = p[2 * n + c], w = p[3 * n + c];
        f[c] = d; f[n + c] = u * d; f[2 * n + c] = v * d; f[3 * n + c] = w * d;
        f[4 * n + c] = d * ((u * u + v * v + w * w) * 0.5 + cv * p[4 * n + c]);
    }
    s->next_stage = 1;
    s->stage_begun = false;
    rc = grid_state_upload(s->s, f.data(), (cudaStream_t)stream);
    if (rc) return rc;
    WS_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return WS_OK;
}

int ws_solver_set_state(ws_solver* s, const double* f_host, ws_stream_t stream) {
    if (!s || !f_host) return fail(WS_ERR_INVALID, "NULL argument");
    s->next_stage = 1;
    s->stage_begun = false;
    return grid_state_upload(s->s, f_host, (cudaStream_t)stream);
}

int ws_solver_get_state(ws_solver* s, double* f_host, ws_stream_t stream) {
    if (!s || !f_host) return fail(WS_ERR_INVALID, "NULL argument");
    int rc = grid_state_download(s->s, f_host, (cudaStream_t)stream);
    if (rc) return rc;
    WS_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return WS_OK;
}

int ws_solver_get_state_async(ws_solver* s, double* f_host, ws_stream_t stream) {
    if (!s || !f_host) return fail(WS_ERR_INVALID, "NULL argument");
    return grid_state_download(s->s, f_host, (cudaStream_t)stream);
}

int ws_solver_get_rhs(ws_solver* s, double* du_host, ws_stream_t stream) {
    if (!s || !du_host) return fail(WS_ERR_INVALID, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)5 * s->s.g.nx * s->s.g.ny * s->s.g.nz;
    WS_CUDA(cudaMemcpyAsync(du_host, s->s.du.ptr, n * sizeof(double), cudaMemcpyDeviceToHost,
                            st));
    WS_CUDA(cudaStreamSynchronize(st));
    return WS_OK;
}

int ws_solver_fields(ws_solver* s, ws_soa* f, ws_soa* du, ws_field prims[6]) {
    if (!s) return fail(WS_ERR_INVALID, "solver is NULL");
    if (f) *f = s->s.f[s->s.cur];
    if (du) *du = s->s.du;
    if (prims)
        for (int i = 0; i < 6; ++i) prims[i] = s->s.prims()[i];
    return WS_OK;
}

int ws_solver_rhs(ws_solver* s, ws_stream_t stream) {
    if (!s) return fail(WS_ERR_INVALID, "solver is NULL");
    if (s->viscous && has_external(&s->s.g))
        return fail(WS_ERR_UNSUPPORTED, "viscous RHS of an EXTERNAL grid: the fluxes' "
                                        "halos come from ws_solver_stage_begin / _end");
    return enqueue_rhs(s, (cudaStream_t)stream);
}

int ws_solver_compute_dt(ws_solver* s, double cfl, double* dt, ws_stream_t stream) {
    if (!s || !dt) return fail(WS_ERR_INVALID, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    WS_CUDA(cudaMemsetAsync(s->scratch, 0, sizeof(unsigned long long), st));
    int rc = launch_max_speed(&s->s.g, s->s.prims(), s->scratch, st);
    if (rc) return rc;
    unsigned long long bits = 0;
    WS_CUDA(cudaMemcpyAsync(&bits, s->scratch, sizeof bits, cudaMemcpyDeviceToHost, st));
    WS_CUDA(cudaStreamSynchronize(st));
    double m;
    std::memcpy(&m, &bits, sizeof m);
    if (!wave_speed_ok(m))
        return fail(WS_ERR_NONFINITE, "maximum wave speed is not finite and positive");
    *dt = cfl / m;
    return WS_OK;
}

int ws_solver_step(ws_solver* s, double dt, int nsteps, ws_stream_t stream) {
    if (!s) return fail(WS_ERR_INVALID, "solver is NULL");
    if (nsteps < 0 || !(dt > 0)) return fail(WS_ERR_INVALID, "need dt > 0 and nsteps >= 0");
    if (has_external(&s->s.g))
        return fail(WS_ERR_UNSUPPORTED, "a grid with EXTERNAL faces steps by stages "
                                        "(ws_solver_stage) with a halo exchange before each");
    if (s->next_stage != 1 || s->stage_begun)
        return fail(WS_ERR_INVALID, "a staged step is in progress");
    if (!s->exec[0] || s->graph_dt != dt) {
        int rc = capture(s, dt);
        if (rc) return rc;
    }
    cudaStream_t st = (cudaStream_t)stream;
    for (int i = 0; i < nsteps; ++i) {
        WS_CUDA(cudaGraphLaunch(s->exec[s->s.cur], st));
        s->s.cur ^= 1;
    }
    return WS_OK;
}

int ws_solver_stage_fields(ws_solver* s, int krk, ws_field prims[6]) {
    if (!s || !prims) return fail(WS_ERR_INVALID, "NULL argument");
    if (krk < 1 || krk > 3) return fail(WS_ERR_INVALID, "krk must be 1, 2 or 3");
    const ws_field* p = stage_input(s->s, s->s.cur, krk);
    for (int i = 0; i < 6; ++i) prims[i] = p[i];
    return WS_OK;
}

namespace {
int check_stage(ws_solver* s, int krk, bool begun) {
    if (!s) return fail(WS_ERR_INVALID, "solver is NULL");
    if (krk != s->next_stage)
        return fail(WS_ERR_INVALID, "stage " + std::to_string(krk) + " called when stage " +
                                        std::to_string(s->next_stage) + " is due");
    if (s->stage_begun != begun)
        return fail(WS_ERR_INVALID, begun ? "stage end without its begin"
                                          : "the stage's first half is already enqueued");
    return WS_OK;
}

void advance_stage(ws_solver* s, int krk) {
    s->stage_begun = false;
    if (krk == 3) {
        s->s.cur ^= 1;
        s->next_stage = 1;
    } else {
        s->next_stage = krk + 1;
    }
}
}  // namespace

int ws_solver_stage(ws_solver* s, int krk, double dt, ws_stream_t stream) {
    if (int rc = check_stage(s, krk, false)) return rc;
    if (!(dt > 0)) return fail(WS_ERR_INVALID, "need dt > 0");
    if (s->viscous && has_external(&s->s.g))
        return fail(WS_ERR_UNSUPPORTED, "with viscous terms an EXTERNAL grid stages in two "
                                        "halves (ws_solver_stage_begin / _end) with the "
                                        "fluxes' halo exchange between them");
    int rc = enqueue_stage(s, s->s.cur, krk, dt, (cudaStream_t)stream);
    if (rc) return rc;
    advance_stage(s, krk);
    return WS_OK;
}

int ws_solver_stage_begin(ws_solver* s, int krk, ws_stream_t stream) {
    if (int rc = check_stage(s, krk, false)) return rc;
    int rc = enqueue_stage_begin(s, s->s.cur, krk, (cudaStream_t)stream);
    if (rc) return rc;
    s->stage_begun = true;
    return WS_OK;
}

int ws_solver_stage_end(ws_solver* s, int krk, double dt, ws_stream_t stream) {
    if (int rc = check_stage(s, krk, true)) return rc;
    if (!(dt > 0)) return fail(WS_ERR_INVALID, "need dt > 0");
    int rc = enqueue_stage_end(s, s->s.cur, krk, dt, (cudaStream_t)stream);
    if (rc) return rc;
    advance_stage(s, krk);
    return WS_OK;
}

int ws_solver_stage_flux_fields(ws_solver* s, int axis, ws_field ev_axis[4]) {
    if (!s || !ev_axis) return fail(WS_ERR_INVALID, "NULL argument");
    if (axis < 0 || axis > 2) return fail(WS_ERR_INVALID, "axis must be 0, 1 or 2");
    if (!s->viscous) return fail(WS_ERR_INVALID, "the solver has no viscous terms");
    ws_field ev[12];
    vis_flux_fields(&s->s.g, s->vis_ws, ev);
    for (int q = 0; q < 4; ++q) ev_axis[q] = ev[4 * axis + q];
    return WS_OK;
}

int ws_solver_status(ws_solver* s, int* status, ws_stream_t stream) {
    if (!s || !status) return fail(WS_ERR_INVALID, "NULL argument");
    int v = 0;
    cudaStream_t st = (cudaStream_t)stream;
    WS_CUDA(cudaMemcpyAsync(&v, s->s.status, sizeof v, cudaMemcpyDeviceToHost, st));
    WS_CUDA(cudaStreamSynchronize(st));
    *status = status_code(v);
    return WS_OK;
}

}  // extern "C"
