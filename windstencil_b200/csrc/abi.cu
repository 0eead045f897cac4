// abi.cu -- extern "C" entry points of libwindstencil_b200.so.
//
// Argument checking, error reporting and the one-grid solver whose SSP-RK3
// step is one captured CUDA graph (ghost fill -> RHS -> stage update, three
// times).  Reference counterparts are named in include/windstencil_b200.h.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include <cstdlib>

#include "ws_internal.h"

namespace ws {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
std::string last_error_message() { return g_last_error; }
int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? WS_ERR_ALLOC : WS_ERR_CUDA;
}

namespace {

int check_grid(const ws_grid* g) {
    if (!g) return fail(WS_ERR_INVALID, "grid is NULL");
    if (g->lap != WS_LAP) return fail(WS_ERR_INVALID, "grid.lap must be 4");
    if (g->nx < 4 || g->ny < 4 || g->nz < 4)
        return fail(WS_ERR_INVALID, "grid extents must be >= 4 in every direction");
    if (g->nx > (1u << 20) || g->ny > (1u << 20) || g->nz > (1u << 20))
        return fail(WS_ERR_INVALID, "grid extent too large");
    if (!(g->hx > 0 && g->hy > 0 && g->hz > 0)) return fail(WS_ERR_INVALID, "h must be > 0");
    if (!(g->gamma > 1.0) || !(g->ama > 0) || !(g->epsl_sw >= 0))
        return fail(WS_ERR_INVALID, "need gamma > 1, ama > 0, epsl_sw >= 0");
    for (int i = 0; i < 6; ++i) {
        const int k = g->face_kind[i];
        if (k != WS_FACE_PERIODIC && k != WS_FACE_EXTRAP && k != WS_FACE_CLOSURE &&
            k != WS_FACE_EXTERNAL)
            return fail(WS_ERR_INVALID, "face_kind must be a ws_face_kind value");

        if (k == WS_FACE_CLOSURE && i >= 4)
            return fail(WS_ERR_UNSUPPORTED, "CLOSURE faces are x and y faces only "
                                            "(the reference closes z through its ghosts)");
        if (k == WS_FACE_CLOSURE && (i < 2 ? g->nx : g->ny) < 8)
            return fail(WS_ERR_INVALID, "a CLOSURE direction needs >= 8 cells");
    }
    if (g->precision != WS_FP64 && g->precision != WS_MIXED)
        return fail(WS_ERR_INVALID, "precision must be WS_FP64 or WS_MIXED");
    return WS_OK;
}

int check_field(const ws_grid* g, ws_field f, const char* name) {
    if (!f.ptr) return fail(WS_ERR_INVALID, std::string(name) + ": NULL pointer");
    if (f.pitch < g->nx + 8) return fail(WS_ERR_INVALID, std::string(name) + ": pitch < nx+8");
    if ((reinterpret_cast<uintptr_t>(f.ptr) & 7) != 0)
        return fail(WS_ERR_INVALID, std::string(name) + ": pointer not 8-byte aligned");
    return WS_OK;
}

int check_soa(ws_soa s, uint32_t ex, uint32_t ey, uint32_t ez, const char* name) {
    if (!s.ptr) return fail(WS_ERR_INVALID, std::string(name) + ": NULL pointer");
    if (s.pitch < ex || s.length_Y < ey || s.length_Z < ez)
        return fail(WS_ERR_INVALID, std::string(name) + ": SoA smaller than the job");
    if ((reinterpret_cast<uintptr_t>(s.ptr) & 7) != 0)
        return fail(WS_ERR_INVALID, std::string(name) + ": pointer not 8-byte aligned");
    return WS_OK;
}

int check_job(const ws_grid* g, ws_job j) {
    if (j.start.x < 4 || j.start.y < 4 || j.start.z < 4 || j.end.x > g->nx + 4 ||
        j.end.y > g->ny + 4 || j.end.z > g->nz + 4)
        return fail(WS_ERR_INVALID, "job must lie inside the interior [4, n+4)");
    return WS_OK;
}

bool job_empty(ws_job j) {
    return j.end.x <= j.start.x || j.end.y <= j.start.y || j.end.z <= j.start.z;
}

}  // namespace

// default tile shape (measured on B200 at 600x128x128): FP64 16x8 columns /
// 768 threads, one CTA per SM -- 24 warps hide the FP64 and barrier
// latencies better than 16 within an 80-register budget; mixed 8x8 / 384
// threads, two CTAs per SM (one CTA's barrier waits overlap the other's
// arithmetic).
// Measured at 600x128x128 on B200: 16x8 with 704 threads in every form (the
// sweep's two intervals hold 1216 and 1400 items, which 704 threads run in
// two nearly full rounds each); the mixed form's 8x8/384 (two CTAs per SM)
// measures 1% slower for the plain RHS and 7% for the stage kernel.
int default_cfg(int precision, bool stage) {
    (void)precision;
    (void)stage;
    return 1;
}

namespace {
// sweep length cap: unlimited (each persistent CTA sweeps its whole share)
int default_scan(const ws_grid*) { return 1 << 30; }

}  // namespace

namespace {
// cuTensorMapEncodeTiled from the driver, looked up once (nullptr when the
// driver does not provide it: staging then stays on cp.async)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static const EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return static_cast<EncodeTiledFn>(nullptr);
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// 3D map of one LAP field (x: nx+8, y: ny+8, z: nz+8 elements) with a
// bw x bh x 1 box; false when the field breaks TMA's alignment rules
bool encode_lap_map(CUtensorMap* map, const ws_grid* g, const ws_field& f, int bw, int bh) {
    const EncodeTiledFn fn = encode_tiled();
    if (!fn || !f.ptr || (reinterpret_cast<uintptr_t>(f.ptr) & 15) || (f.pitch & 1) ||
        f.pitch < (uint32_t)g->nx + 8)
        return false;
    const cuuint64_t dims[3] = {(cuuint64_t)g->nx + 8, (cuuint64_t)g->ny + 8,
                                (cuuint64_t)g->nz + 8};
    const cuuint64_t strides[2] = {(cuuint64_t)f.pitch * 8,
                                   (cuuint64_t)f.pitch * (g->ny + 8) * 8};
    const cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, f.ptr, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace

RhsArgs make_rhs_args(const ws_grid* g, ws_job job, const ws_field prims[5],
                      const ws_metrics* m, ws_soa du, int cfg, int scan) {
    const TileCfg c = tile_cfg(cfg);
    RhsArgs a{};
    for (int i = 0; i < 5; ++i) {
        a.prim[i] = prims[i].ptr;
        a.ppitch[i] = prims[i].pitch;
    }
    const bool uni = g->metrics_uniform != 0;
    if (!uni) {
        const ws_field* mf = &m->akx;
        for (int i = 0; i < 10; ++i) {
            a.met[i] = mf[i].ptr;
            a.mpitch[i] = mf[i].pitch;
        }
    }
    a.du = du.ptr;
    a.du_pitch = du.pitch;
    a.du_ly = du.length_Y;
    a.du_lz = du.length_Z;
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    a.sx = job.start.x; a.sy = job.start.y; a.sz = job.start.z;
    a.ex = job.end.x; a.ey = job.end.y; a.ez = job.end.z;
    a.ntx = (a.ex - a.sx + c.bx - 1) / c.bx;
    a.nty = (a.ey - a.sy + c.by - 1) / c.by;
    a.zc = scan;
    a.nzc = (a.ez - a.sz + scan - 1) / scan;
    a.rhx = 1.0 / g->hx; a.rhy = 1.0 / g->hy; a.rhz = 1.0 / g->hz;
    a.eps2 = g->epsl_sw * g->epsl_sw;
    a.hrg = 0.5 / g->gamma;
    a.c1 = 2.0 * (g->gamma - 1.0);
    a.c3 = (3.0 - g->gamma) / (2.0 * (g->gamma - 1.0));
    a.gm1 = g->gamma - 1.0;
    for (int i = 0; i < 4; ++i) a.clo[i] = g->face_kind[i] == WS_FACE_CLOSURE ? 1 : 0;
    // TMA staging: box starts at x = sx - 4 + k*bx and centres at sx + k*bx
    // are even (16-byte aligned for doubles) when sx is even
    bool tma = (job.start.x % 2) == 0;
    for (int i = 0; i < 5 && tma; ++i)
        tma = encode_lap_map(&a.tm_box[i], g, prims[i], c.bx + 8, c.by + 8) &&
              encode_lap_map(&a.tm_ctr[i], g, prims[i], c.bx, c.by);
    a.tma = tma ? 1 : 0;
    a.status = device_error_word();     // the stage epilogue sets the grid's own
    const char* hold = std::getenv("WS_TEST_STAGE_WAIT");
    a.hold_polls = hold ? std::max(0, std::atoi(hold)) : 0;
    return a;
}

int set_rhs_stage(RhsArgs& a, const ws_grid* g, ws_soa f_in, ws_soa fn, ws_soa f_out,
                  const ws_field p_out[6], double dt, int* status) {
    auto same = [](const ws_soa& x, const ws_soa& y) {
        return x.pitch == y.pitch && x.length_Y == y.length_Y && x.length_Z == y.length_Z;
    };
    if (!same(f_in, fn) || !same(fn, f_out))
        return fail(WS_ERR_INVALID, "stage epilogue: f_in, fn, f_out need one SoA shape");
    a.f_in = f_in;
    a.fn = fn;
    a.f_out = f_out;
    for (int i = 0; i < 6; ++i) {
        if (p_out[i].pitch != p_out[0].pitch)
            return fail(WS_ERR_INVALID, "stage epilogue: output fields need one pitch");
        a.p_out[i] = p_out[i].ptr;
    }
    a.p_pitch = p_out[0].pitch;
    a.dt = dt;
    a.rcv = g->gamma * (g->gamma - 1.0) * g->ama * g->ama;   // 1/cv, OCFD_init.cpp:380
    a.rama = 1.0 / g->ama;
    a.status = status;
    return WS_OK;
}

// persistent grid: one CTA per resident slot, but no more than keeps every
// CTA at >= 16 planes of work once the tile columns run out
int rhs_ctas(const ws_grid* g, const RhsArgs& a, int cfg, bool stage) {
    const long ntile = (long)a.ntx * a.nty;
    const long planes = ntile * (a.ez - a.sz);
    const bool clo = a.clo[0] | a.clo[1] | a.clo[2] | a.clo[3];
    int ctas = rhs_max_ctas(g->precision, g->metrics_uniform != 0, clo, cfg, stage);
    if (ctas <= 0) return 0;
    const long want = ntile >= ctas ? ctas : std::max(ntile, planes / 16);
    if (want < ctas) ctas = (int)std::max(1L, want);
    return ctas;
}

int tile_index(const ws_grid* g, ws_tile tile, bool stage, int* cfg) {
    *cfg = default_cfg(g->precision, stage);
    if (tile.tile_x || tile.tile_y || tile.threads) {
        *cfg = find_tile_cfg(tile.tile_x, tile.tile_y, tile.threads);
        if (*cfg < 0) return fail(WS_ERR_UNSUPPORTED, "tile shape not compiled in this build");
    }
    return WS_OK;
}

// Fill RhsArgs and launch; shared by the drop-in entry and the solver.
bool use_pencil(const ws_grid* g, ws_tile tile) {
    (void)g;
    if (tile.tile_x < 0) return true;
    return !(tile.tile_x || tile.tile_y || tile.threads);
}

namespace {
int check_pencil(const ws_grid* g, ws_tile tile) {
    (void)g;
    if (tile.threads % 32) return fail(WS_ERR_INVALID, "line passes: threads = 32 x warps");
    return WS_OK;
}
}  // namespace

int rhs_enqueue(const ws_grid* g, ws_job job, const ws_field prims[5], const ws_metrics* m,
                ws_soa du, ws_tile tile, cudaStream_t st) {
    if (use_pencil(g, tile)) {
        int rc = check_pencil(g, tile);
        if (rc) return rc;
        const RhsArgs a = make_rhs_args(g, job, prims, m, du, 0, 1);
        return launch_rhs_pencil(a, g->precision, g->metrics_uniform != 0, tile.threads / 32, 0,
                                 false, st);
    }
    int cfg = 0;
    int rc = tile_index(g, tile, false, &cfg);
    if (rc) return rc;
    const int scan = tile.scan_z > 0 ? tile.scan_z : default_scan(g);
    const RhsArgs a = make_rhs_args(g, job, prims, m, du, cfg, scan);
    const int ctas = rhs_ctas(g, a, cfg, false);
    if (ctas <= 0) return fail(WS_ERR_CUDA, "cannot size the persistent grid");
    return launch_rhs(a, g->precision, g->metrics_uniform != 0, cfg, ctas, 0, st);
}

// One fused RHS + SSP-RK3 stage over the whole interior (Cartesian grids):
// reads primitives p_in (ghosts filled), f_in and fn; writes f_out and the
// new primitives p_out.
int rhs_stage_enqueue(const ws_grid* g, const ws_field p_in[6], ws_soa f_in, ws_soa fn,
                      ws_soa f_out, const ws_field p_out[6], double dt, int krk, int* status,
                      ws_soa dvis, ws_soa du, ws_tile tile, cudaStream_t st) {
    if (use_pencil(g, tile)) {
        int rc = check_pencil(g, tile);
        if (rc) return rc;
        if (du.pitch != fn.pitch || du.length_Y != fn.length_Y || du.length_Z != fn.length_Z)
            return fail(WS_ERR_INVALID, "line passes: du needs the state's shape");
        ws_job job{{4, 4, 4}, {g->nx + 4, g->ny + 4, g->nz + 4}};
        const ws_field p5[5] = {p_in[0], p_in[1], p_in[2], p_in[3], p_in[5]};
        RhsArgs a = make_rhs_args(g, job, p5, nullptr, du, 0, 1);
        if ((rc = set_rhs_stage(a, g, f_in, fn, f_out, p_out, dt, status))) return rc;
        return launch_rhs_pencil(a, g->precision, true, tile.threads / 32, krk,
                                 dvis.ptr != nullptr, st);
    }
    int cfg = 0;
    int rc = tile_index(g, tile, true, &cfg);
    if (rc) return rc;
    const int scan = tile.scan_z > 0 ? tile.scan_z : default_scan(g);
    ws_job job{{4, 4, 4}, {g->nx + 4, g->ny + 4, g->nz + 4}};
    const ws_field p5[5] = {p_in[0], p_in[1], p_in[2], p_in[3], p_in[5]};
    RhsArgs a = make_rhs_args(g, job, p5, nullptr, ws_soa{}, cfg, scan);
    if ((rc = set_rhs_stage(a, g, f_in, fn, f_out, p_out, dt, status))) return rc;
    if (dvis.ptr) {
        if (dvis.pitch != fn.pitch || dvis.length_Y != fn.length_Y ||
            dvis.length_Z != fn.length_Z)
            return fail(WS_ERR_INVALID, "stage epilogue: viscous terms need the state's shape");
        a.dvis = dvis;
    }
    const int ctas = rhs_ctas(g, a, cfg, true);
    if (ctas <= 0) return fail(WS_ERR_CUDA, "cannot size the persistent grid");
    return launch_rhs(a, g->precision, true, cfg, ctas, krk, st);
}

int validate_grid(const ws_grid* g) { return check_grid(g); }

// One word per device for the launches that have no per-grid status word.
__device__ int g_ws_device_error;

int* device_error_word() {
    static int* cache[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    if (!cache[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_ws_device_error) != cudaSuccess) return nullptr;
        cache[dev] = static_cast<int*>(p);
    }
    return cache[dev];
}

bool has_external(const ws_grid* g) {
    for (int i = 0; i < 6; ++i)
        if (g->face_kind[i] == WS_FACE_EXTERNAL) return true;
    return false;
}

}  // namespace ws

using namespace ws;

// ============================================================================
extern "C" {

int ws_abi_version(void) { return WS_ABI_VERSION; }

int ws_last_error(char* buf, size_t n) {
    if (!buf || n == 0) return WS_ERR_INVALID;
    std::snprintf(buf, n, "%s", g_last_error.c_str());
    return WS_OK;
}

uint32_t ws_lap_pitch(uint32_t nx) { return lap_pitch(nx); }

int ws_du_invis_jacobian3d_init(const ws_grid* g, ws_job job, ws_field T, ws_field cc,
                                ws_stream_t stream) {
    int rc;
    if ((rc = check_grid(g))) return rc;
    if ((rc = check_job(g, job))) return rc;
    if ((rc = check_field(g, T, "T")) || (rc = check_field(g, cc, "cc"))) return rc;
    if (job_empty(job)) return WS_OK;
    return launch_sound_speed(g, job, T, cc, (cudaStream_t)stream);
}

size_t ws_du_vis_workspace_bytes(const ws_grid* g) {
    return g ? vis_workspace_bytes(g) : 0;
}

int ws_du_vis_jacobian3d(const ws_grid* g, const ws_viscous* vis, ws_field u, ws_field v,
                         ws_field w, ws_field T, const ws_metrics* metrics, ws_soa du,
                         void* workspace, size_t workspace_bytes, ws_stream_t stream) {
    int rc;
    if ((rc = check_grid(g)) || (rc = check_viscous(vis))) return rc;
    if (has_external(g))
        return fail(WS_ERR_UNSUPPORTED, "viscous terms on a grid with EXTERNAL faces");
    if ((rc = check_field(g, u, "u")) || (rc = check_field(g, v, "v")) ||
        (rc = check_field(g, w, "w")) || (rc = check_field(g, T, "T")))
        return rc;
    if (!g->metrics_uniform) {
        if (!metrics) return fail(WS_ERR_INVALID, "metrics are NULL for a non-uniform grid");
        const ws_field* mf = &metrics->akx;
        for (int i = 0; i < 10; ++i)
            if ((rc = check_field(g, mf[i], "metric"))) return rc;
    }
    if ((rc = check_soa(du, g->nx, g->ny, g->nz, "du"))) return rc;
    if (!workspace || workspace_bytes < vis_workspace_bytes(g))
        return fail(WS_ERR_INVALID, "viscous workspace missing or smaller than "
                                    "ws_du_vis_workspace_bytes()");
    if (reinterpret_cast<uintptr_t>(workspace) & 15)
        return fail(WS_ERR_INVALID, "viscous workspace must be 16-byte aligned");
    const ws_field p4[4] = {u, v, w, T};
    return launch_du_vis(g, vis, p4, metrics, du, workspace, true, (cudaStream_t)stream);
}

int ws_du_invis_jacobian3d_tiled(const ws_grid* g, ws_job job, ws_field d, ws_field u,
                                 ws_field v, ws_field w, ws_field cc,
                                 const ws_metrics* metrics, ws_soa du, ws_tile tile,
                                 ws_stream_t stream) {
    int rc;
    if ((rc = check_grid(g))) return rc;
    if ((rc = check_job(g, job))) return rc;
    const ws_field prims[5] = {d, u, v, w, cc};
    const char* names[5] = {"d", "u", "v", "w", "cc"};
    for (int i = 0; i < 5; ++i)
        if ((rc = check_field(g, prims[i], names[i]))) return rc;
    if (!g->metrics_uniform) {
        if (!metrics) return fail(WS_ERR_INVALID, "metrics required when metrics_uniform == 0");
        const ws_field* mf = &metrics->akx;
        for (int i = 0; i < 10; ++i)
            if ((rc = check_field(g, mf[i], "metric field"))) return rc;
    }
    if (job_empty(job)) return WS_OK;
    if ((rc = check_soa(du, job.end.x - job.start.x, job.end.y - job.start.y,
                        job.end.z - job.start.z, "du")))
        return rc;
    return rhs_enqueue(g, job, prims, metrics, du, tile, (cudaStream_t)stream);
}

int ws_du_invis_jacobian3d(const ws_grid* g, ws_job job, ws_field d, ws_field u, ws_field v,
                           ws_field w, ws_field cc, const ws_metrics* metrics, ws_soa du,
                           ws_stream_t stream) {
    ws_tile t{0, 0, 0, 0};
    return ws_du_invis_jacobian3d_tiled(g, job, d, u, v, w, cc, metrics, du, t, stream);
}

int ws_ghost_fill(const ws_grid* g, const ws_field* fields, int nfields, ws_stream_t stream) {
    int rc;
    if ((rc = check_grid(g))) return rc;
    if (!fields || nfields < 1 || nfields > 8)
        return fail(WS_ERR_INVALID, "ghost fill takes 1..8 fields");
    for (int i = 0; i < nfields; ++i)
        if ((rc = check_field(g, fields[i], "field"))) return rc;
    return launch_ghost_fill(g, fields, nfields, (cudaStream_t)stream);
}

int ws_device_error(int* flags, ws_stream_t stream) {
    if (!flags) return fail(WS_ERR_INVALID, "flags is NULL");
    int* w = device_error_word();
    if (!w) return fail(WS_ERR_CUDA, "cannot resolve the device error word");
    cudaStream_t st = (cudaStream_t)stream;
    int v = 0;
    WS_CUDA(cudaMemcpyAsync(&v, w, sizeof v, cudaMemcpyDeviceToHost, st));
    WS_CUDA(cudaMemsetAsync(w, 0, sizeof(int), st));
    WS_CUDA(cudaStreamSynchronize(st));
    *flags = v;
    return WS_OK;
}

size_t ws_halo_bytes(const ws_grid* g, int axis, int nfields) {
    if (!g || nfields < 1 || nfields > 8 || axis < 0 || axis > 2) return 0;
    const size_t n[3] = {g->nx, g->ny, g->nz};
    size_t c = (size_t)nfields * 4 * sizeof(double);
    for (int d = 0; d < 3; ++d)
        if (d != axis) c *= n[d];
    return c;
}

namespace {
int halo_call(const ws_grid* g, const ws_field* fields, int nfields, int axis, int side,
              const void* buf, bool pack, ws_stream_t stream) {
    int rc;
    if ((rc = check_grid(g))) return rc;
    if (!fields || nfields < 1 || nfields > 8)
        return fail(WS_ERR_INVALID, "a halo takes 1..8 fields");
    if (axis < 0 || axis > 2) return fail(WS_ERR_INVALID, "axis must be 0, 1 or 2");
    if (side != 0 && side != 1) return fail(WS_ERR_INVALID, "side must be 0 or 1");
    if (!buf || (reinterpret_cast<uintptr_t>(buf) & 7))
        return fail(WS_ERR_INVALID, "halo buffer NULL or not 8-byte aligned");
    for (int i = 0; i < nfields; ++i)
        if ((rc = check_field(g, fields[i], "field"))) return rc;
    return launch_halo(g, fields, nfields, axis, side,
                       const_cast<double*>(static_cast<const double*>(buf)), pack,
                       (cudaStream_t)stream);
}
}  // namespace

int ws_halo_pack(const ws_grid* g, const ws_field* fields, int nfields, int axis, int side,
                 void* buf, ws_stream_t stream) {
    return halo_call(g, fields, nfields, axis, side, buf, true, stream);
}

int ws_halo_unpack(const ws_grid* g, const ws_field* fields, int nfields, int axis, int side,
                   const void* buf, ws_stream_t stream) {
    return halo_call(g, fields, nfields, axis, side, buf, false, stream);
}

size_t ws_halo_x_bytes(const ws_grid* g, int nfields) { return ws_halo_bytes(g, 0, nfields); }

int ws_halo_pack_x(const ws_grid* g, const ws_field* fields, int nfields, int side, void* buf,
                   ws_stream_t stream) {
    return halo_call(g, fields, nfields, 0, side, buf, true, stream);
}

int ws_halo_unpack_x(const ws_grid* g, const ws_field* fields, int nfields, int side,
                     const void* buf, ws_stream_t stream) {
    return halo_call(g, fields, nfields, 0, side, buf, false, stream);
}

int ws_cons_to_prim(const ws_grid* g, ws_soa f, ws_field d, ws_field u, ws_field v, ws_field w,
                    ws_field T, ws_field P, ws_stream_t stream) {
    int rc;
    if ((rc = check_grid(g))) return rc;
    if ((rc = check_soa(f, g->nx, g->ny, g->nz, "f"))) return rc;
    const ws_field fs[5] = {d, u, v, w, T};
    for (int i = 0; i < 5; ++i)
        if ((rc = check_field(g, fs[i], "primitive"))) return rc;
    if (P.ptr && (rc = check_field(g, P, "P"))) return rc;
    return launch_cons_to_prim(g, f, d, u, v, w, T, P, nullptr, (cudaStream_t)stream);
}

int ws_prim_to_cons(const ws_grid* g, ws_field d, ws_field u, ws_field v, ws_field w, ws_field T,
                    ws_soa f, ws_stream_t stream) {
    int rc;
    if ((rc = check_grid(g))) return rc;
    if ((rc = check_soa(f, g->nx, g->ny, g->nz, "f"))) return rc;
    const ws_field fs[5] = {d, u, v, w, T};
    for (int i = 0; i < 5; ++i)
        if ((rc = check_field(g, fs[i], "primitive"))) return rc;
    return launch_prim_to_cons(g, d, u, v, w, T, f, (cudaStream_t)stream);
}

int ws_time_advance(const ws_grid* g, int krk, double dt, ws_soa f, ws_soa fn, ws_soa du,
                    ws_stream_t stream) {
    int rc;
    if ((rc = check_grid(g))) return rc;
    if (krk < 1 || krk > 3) return fail(WS_ERR_INVALID, "krk must be 1, 2 or 3");
    if ((rc = check_soa(f, g->nx, g->ny, g->nz, "f")) ||
        (rc = check_soa(fn, g->nx, g->ny, g->nz, "fn")) ||
        (rc = check_soa(du, g->nx, g->ny, g->nz, "du")))
        return rc;
    return launch_time_advance(g, krk, dt, f, fn, du, (cudaStream_t)stream);
}

}  // extern "C"
