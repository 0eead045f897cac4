// solver.cu -- one grid, device-resident state, SSP-RK3 steps from CUDA graphs.
//
// Replaces the reference's time loop (src/solver/OCFD_NS_Solver.cpp:64-90)
// for the Euler system: the pf/pfn pointer swap becomes two captured graphs
// (state A -> B and B -> A), each holding three stages of
//   ghost fill (d,u,v,w,T,cc) -> fused RHS -> stage update + cons->prim + cc.
// The reference's shipped loop runs stage 1 only (`KRK <= 1`, :77); all three
// stage formulas of OCFD_time.cpp:15-65 are used here.
#include <cstring>

#include "ws_internal.h"

namespace ws {
int rhs_enqueue(const ws_grid* g, ws_job job, const ws_field prims[5], const ws_metrics* m,
                ws_soa du, ws_tile tile, cudaStream_t st);

namespace {
__global__ void max_speed_kernel(ws_field d, ws_field u, ws_field v, ws_field w, ws_field cc,
                                 int nx, int ny, int nz, double rx, double ry, double rz,
                                 unsigned long long* out) {
    const long n = (long)nx * ny * nz;
    const double rr = sqrt(rx * rx + ry * ry + rz * rz);
    double m = 0.0;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx) + 4;
        const long r = t / nx;
        const int j = (int)(r % ny) + 4, k = (int)(r / ny) + 4;
        auto at = [&](const ws_field& f) {
            return f.ptr[(size_t)i + (size_t)f.pitch * ((size_t)j + (size_t)(ny + 8) * k)];
        };
        const double s = fabs(at(u)) * rx + fabs(at(v)) * ry + fabs(at(w)) * rz + at(cc) * rr;
        m = fmax(m, s);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}
}  // namespace
}  // namespace ws

using namespace ws;

struct ws_solver {
    ws_grid g;
    int dev = 0;
    double* soa_buf = nullptr;      // f[0], f[1], du
    double* lap_buf = nullptr;      // d, u, v, w, T, cc
    int* status = nullptr;          // device status word
    unsigned long long* scratch = nullptr;
    ws_soa f[2], du;
    ws_field prims[6];
    int cur = 0;                    // buffer holding the current state
    cudaStream_t cap = nullptr;     // private capture stream
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    double graph_dt = 0.0;
    ws_tile tile{0, 0, 0, 0};
};

namespace {
void drop_graphs(ws_solver* s) {
    for (auto& e : s->exec)
        if (e) {
            cudaGraphExecDestroy(e);
            e = nullptr;
        }
}

int enqueue_rhs(ws_solver* s, cudaStream_t st) {
    int rc = launch_ghost_fill_prims(&s->g, s->prims, st);
    if (rc) return rc;
    ws_job job{{4, 4, 4}, {s->g.nx + 4, s->g.ny + 4, s->g.nz + 4}};
    const ws_field p5[5] = {s->prims[0], s->prims[1], s->prims[2], s->prims[3], s->prims[5]};
    return rhs_enqueue(&s->g, job, p5, nullptr, s->du, s->tile, st);
}

// one SSP-RK3 step from state f[src] into f[1-src]
int enqueue_step(ws_solver* s, int src, double dt, cudaStream_t st) {
    for (int krk = 1; krk <= 3; ++krk) {
        int rc = enqueue_rhs(s, st);
        if (rc) return rc;
        rc = launch_stage_update(&s->g, krk, dt, s->f[1 - src], s->f[src], s->du, s->prims,
                                 s->status, st);
        if (rc) return rc;
    }
    return WS_OK;
}

int capture(ws_solver* s, double dt) {
    drop_graphs(s);
    for (int src = 0; src < 2; ++src) {
        cudaGraph_t graph = nullptr;
        WS_CUDA(cudaStreamBeginCapture(s->cap, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(s, src, dt, s->cap);
        cudaError_t e = cudaStreamEndCapture(s->cap, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&s->exec[src], graph, 0);
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
    if (g->lap != WS_LAP || g->nx < 4 || g->ny < 4 || g->nz < 4)
        return fail(WS_ERR_INVALID, "invalid grid");
    if (!g->metrics_uniform)
        return fail(WS_ERR_UNSUPPORTED, "the solver holds Cartesian grids only");
    ws_solver* s = new (std::nothrow) ws_solver();
    if (!s) return fail(WS_ERR_ALLOC, "host allocation failed");
    s->g = *g;
    cudaGetDevice(&s->dev);
    const size_t ncell = (size_t)g->nx * g->ny * g->nz;
    const uint32_t lp = lap_pitch(g->nx);
    const size_t nlap = (size_t)lp * (g->ny + 8) * (g->nz + 8);
    cudaError_t e = cudaMalloc(&s->soa_buf, sizeof(double) * 15 * ncell);
    if (e == cudaSuccess) e = cudaMalloc(&s->lap_buf, sizeof(double) * 6 * nlap);
    if (e == cudaSuccess) e = cudaMalloc(&s->status, 64);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemset(s->lap_buf, 0, sizeof(double) * 6 * nlap);
    if (e == cudaSuccess) e = cudaMemset(s->soa_buf, 0, sizeof(double) * 15 * ncell);
    if (e == cudaSuccess) e = cudaMemset(s->status, 0, 64);
    if (e != cudaSuccess) {
        ws_solver_destroy(s);
        return cuda_fail(e, "ws_solver_create");
    }
    s->scratch = reinterpret_cast<unsigned long long*>(s->status + 8);
    for (int b = 0; b < 3; ++b) {
        ws_soa q{s->soa_buf + b * 5 * ncell, g->nx, g->ny, g->nz, 0};
        if (b < 2) s->f[b] = q; else s->du = q;
    }
    for (int i = 0; i < 6; ++i) s->prims[i] = ws_field{s->lap_buf + i * nlap, lp, 0};
    *out = s;
    return WS_OK;
}

void ws_solver_destroy(ws_solver* s) {
    if (!s) return;
    drop_graphs(s);
    if (s->cap) cudaStreamDestroy(s->cap);
    cudaFree(s->soa_buf);
    cudaFree(s->lap_buf);
    cudaFree(s->status);
    delete s;
}

int ws_solver_set_tile(ws_solver* s, ws_tile tile) {
    if (!s) return fail(WS_ERR_INVALID, "solver is NULL");
    if ((tile.tile_x || tile.tile_y || tile.threads) &&
        find_tile_cfg(tile.tile_x, tile.tile_y, tile.threads) < 0)
        return fail(WS_ERR_UNSUPPORTED, "tile shape not compiled in this build");
    s->tile = tile;
    drop_graphs(s);
    return WS_OK;
}

int ws_solver_set_state(ws_solver* s, const double* f_host, ws_stream_t stream) {
    if (!s || !f_host) return fail(WS_ERR_INVALID, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)5 * s->g.nx * s->g.ny * s->g.nz;
    WS_CUDA(cudaMemcpyAsync(s->f[s->cur].ptr, f_host, n * sizeof(double), cudaMemcpyHostToDevice,
                            st));
    int rc = launch_cons_to_prim(&s->g, s->f[s->cur], s->prims[0], s->prims[1], s->prims[2],
                                 s->prims[3], s->prims[4], ws_field{nullptr, 0, 0}, s->status, st);
    if (rc) return rc;
    ws_job job{{4, 4, 4}, {s->g.nx + 4, s->g.ny + 4, s->g.nz + 4}};
    return launch_sound_speed(&s->g, job, s->prims[4], s->prims[5], st);
}

int ws_solver_get_state(ws_solver* s, double* f_host, ws_stream_t stream) {
    if (!s || !f_host) return fail(WS_ERR_INVALID, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)5 * s->g.nx * s->g.ny * s->g.nz;
    WS_CUDA(cudaMemcpyAsync(f_host, s->f[s->cur].ptr, n * sizeof(double), cudaMemcpyDeviceToHost,
                            st));
    WS_CUDA(cudaStreamSynchronize(st));
    return WS_OK;
}

int ws_solver_get_rhs(ws_solver* s, double* du_host, ws_stream_t stream) {
    if (!s || !du_host) return fail(WS_ERR_INVALID, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)5 * s->g.nx * s->g.ny * s->g.nz;
    WS_CUDA(cudaMemcpyAsync(du_host, s->du.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    WS_CUDA(cudaStreamSynchronize(st));
    return WS_OK;
}

int ws_solver_fields(ws_solver* s, ws_soa* f, ws_soa* du, ws_field prims[6]) {
    if (!s) return fail(WS_ERR_INVALID, "solver is NULL");
    if (f) *f = s->f[s->cur];
    if (du) *du = s->du;
    if (prims)
        for (int i = 0; i < 6; ++i) prims[i] = s->prims[i];
    return WS_OK;
}

int ws_solver_rhs(ws_solver* s, ws_stream_t stream) {
    if (!s) return fail(WS_ERR_INVALID, "solver is NULL");
    return enqueue_rhs(s, (cudaStream_t)stream);
}

int ws_solver_compute_dt(ws_solver* s, double cfl, double* dt, ws_stream_t stream) {
    if (!s || !dt) return fail(WS_ERR_INVALID, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    WS_CUDA(cudaMemsetAsync(s->scratch, 0, sizeof(unsigned long long), st));
    const long n = (long)s->g.nx * s->g.ny * s->g.nz;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    max_speed_kernel<<<blocks, 256, 0, st>>>(s->prims[0], s->prims[1], s->prims[2], s->prims[3],
                                              s->prims[5], s->g.nx, s->g.ny, s->g.nz,
                                              1.0 / s->g.hx, 1.0 / s->g.hy, 1.0 / s->g.hz,
                                              s->scratch);
    WS_CUDA(cudaGetLastError());
    unsigned long long bits = 0;
    WS_CUDA(cudaMemcpyAsync(&bits, s->scratch, sizeof bits, cudaMemcpyDeviceToHost, st));
    WS_CUDA(cudaStreamSynchronize(st));
    double m;
    std::memcpy(&m, &bits, sizeof m);
    if (!(m > 0)) return fail(WS_ERR_NONFINITE, "maximum wave speed is not positive");
    *dt = cfl / m;
    return WS_OK;
}

int ws_solver_step(ws_solver* s, double dt, int nsteps, ws_stream_t stream) {
    if (!s) return fail(WS_ERR_INVALID, "solver is NULL");
    if (nsteps < 0 || !(dt > 0)) return fail(WS_ERR_INVALID, "need dt > 0 and nsteps >= 0");
    if (!s->exec[0] || s->graph_dt != dt) {
        int rc = capture(s, dt);
        if (rc) return rc;
    }
    cudaStream_t st = (cudaStream_t)stream;
    for (int i = 0; i < nsteps; ++i) {
        WS_CUDA(cudaGraphLaunch(s->exec[s->cur], st));
        s->cur ^= 1;
    }
    return WS_OK;
}

int ws_solver_status(ws_solver* s, int* status, ws_stream_t stream) {
    if (!s || !status) return fail(WS_ERR_INVALID, "NULL argument");
    int v = 0;
    cudaStream_t st = (cudaStream_t)stream;
    WS_CUDA(cudaMemcpyAsync(&v, s->status, sizeof v, cudaMemcpyDeviceToHost, st));
    WS_CUDA(cudaStreamSynchronize(st));
    *status = v ? WS_ERR_NONFINITE : WS_OK;
    return WS_OK;
}

}  // extern "C"
