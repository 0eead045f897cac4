// batch.cu -- many independent grids stepped together.
//
// The reference solves one grid per MPI rank (src/solver/OCFD_NS_Solver.cpp);
// this file adds what it does not have: device-resident states of many
// uneven grids, advanced by SSP-RK3 with two batched launches per stage
// (ghost fill; fused RHS with the stage update), the step replayed from a CUDA
// graph, and an autotuner that times the compiled tile shapes on the batch.
#include <algorithm>
#include <cfloat>
#include <cstring>
#include <memory>
#include <utility>
#include <vector>

#include "ws_internal.h"

namespace ws {

namespace {
size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Work items of a batched RHS launch: every tile's z column cut into runs
// of at most zc planes, {grid, tile, first plane, end plane} (LAP z),
// longest first (a run costs its planes plus about one plane of prologue,
// whatever the tile's fill), so that the CTAs, taking them in turn, start
// the long runs early; equal runs keep grid and tile order, so CTAs that run
// together sweep neighbouring columns.
std::vector<int4> batch_items(const std::vector<GridState*>& grids, int cfg, int zc) {
    const TileCfg t = tile_cfg(cfg);
    std::vector<std::pair<int, int4>> w;
    for (int i = 0; i < (int)grids.size(); ++i) {
        const ws_grid& g = grids[i]->g;
        const int ntiles = (((int)g.nx + t.bx - 1) / t.bx) * (((int)g.ny + t.by - 1) / t.by);
        for (int tile = 0; tile < ntiles; ++tile)
            for (int z = 0; z < (int)g.nz; z += zc) {
                const int len = std::min(zc, (int)g.nz - z);
                w.push_back({len + 1, make_int4(i, tile, 4 + z, 4 + z + len)});
            }
    }
    std::stable_sort(w.begin(), w.end(),
                     [](const auto& l, const auto& r) { return l.first > r.first; });
    std::vector<int4> out(w.size());
    for (size_t k = 0; k < w.size(); ++k) out[k] = w[k].second;
    return out;
}

__global__ void max_speed_kernel(ws_field u, ws_field v, ws_field w, ws_field cc, int nx,
                                 int ny, int nz, double rx, double ry, double rz,
                                 unsigned long long* out) {
    const long n = (long)nx * ny * nz;
    const double rr = sqrt(rx * rx + ry * ry + rz * rz);
    double m = 0.0;
    bool bad = false;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx) + 4;
        const long r = t / nx;
        const int j = (int)(r % ny) + 4, k = (int)(r / ny) + 4;
        auto at = [&](const ws_field& f) {
            return f.ptr[(size_t)i + (size_t)f.pitch * ((size_t)j + (size_t)(ny + 8) * k)];
        };
        const double s = fabs(at(u)) * rx + fabs(at(v)) * ry + fabs(at(w)) * rz + at(cc) * rr;
        // a NaN or infinite speed must reach the result, which fmax would
        // drop (NaN) or the host could read as a valid maximum (+inf)
        bad |= !(s <= DBL_MAX);
        m = fmax(m, s);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    // positive doubles order like their bit patterns; the quiet-NaN pattern
    // 0x7ff8... lies above every finite value and +inf, so it wins the max
    const unsigned long long bits =
        __any_sync(0xffffffffu, bad) ? 0x7ff8000000000000ull
                                     : (unsigned long long)__double_as_longlong(m);
    if ((threadIdx.x & 31) == 0) atomicMax(out, bits);
}
}  // namespace

// max over the interior of |u|/hx + |v|/hy + |w|/hz + c*sqrt(hx^-2+hy^-2+hz^-2)
// as the bits of a non-negative double, atomically max-ed into *out (*out must
// start at 0); a NaN or infinite speed in any cell yields NaN bits instead
int launch_max_speed(const ws_grid* g, const ws_field prims[6], unsigned long long* out,
                     cudaStream_t st) {
    const long n = (long)g->nx * g->ny * g->nz;
    int blocks = (int)std::min<long>((n + 255) / 256, 148L * 8);
    max_speed_kernel<<<std::max(blocks, 1), 256, 0, st>>>(prims[1], prims[2], prims[3], prims[5],
                                                          g->nx, g->ny, g->nz, 1.0 / g->hx,
                                                          1.0 / g->hy, 1.0 / g->hz, out);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
}

// ---------------------------------------------------------------------------
// GridState
// ---------------------------------------------------------------------------
size_t grid_state_bytes(const ws_grid& g) {
    const size_t ncell = (size_t)g.nx * g.ny * g.nz;
    const size_t nlap = (size_t)lap_pitch(g.nx) * (g.ny + 8) * (g.nz + 8);
    return 3 * align256(5 * ncell * sizeof(double)) + 12 * align256(nlap * sizeof(double)) + 256;
}

int grid_state_alloc(GridState& s, const ws_grid& g, cudaStream_t st) {
    s.g = g;
    s.args.clear();
    s.args_cfg = -1;
    s.bytes = grid_state_bytes(g);
    WS_CUDA(cudaMallocAsync(&s.mem, s.bytes, st));
    WS_CUDA(cudaMemsetAsync(s.mem, 0, s.bytes, st));
    const size_t ncell = (size_t)g.nx * g.ny * g.nz;
    const uint32_t lp = lap_pitch(g.nx);
    const size_t nlap = (size_t)lp * (g.ny + 8) * (g.nz + 8);
    unsigned char* p = static_cast<unsigned char*>(s.mem);
    for (int b = 0; b < 3; ++b) {
        ws_soa q{reinterpret_cast<double*>(p), g.nx, g.ny, g.nz, 0};
        if (b < 2) s.f[b] = q; else s.du = q;
        p += align256(5 * ncell * sizeof(double));
    }
    for (int b = 0; b < 2; ++b)
        for (int i = 0; i < 6; ++i) {
            s.pr[b][i] = ws_field{reinterpret_cast<double*>(p), lp, 0};
            p += align256(nlap * sizeof(double));
        }
    s.status = reinterpret_cast<int*>(p);
    s.cur = 0;
    return WS_OK;
}

void grid_state_free(GridState& s, cudaStream_t st) {
    if (s.mem) cudaFreeAsync(s.mem, st);
    s.mem = nullptr;
}

int grid_state_derive(GridState& s, cudaStream_t st) {
    const ws_field* p = s.pr[s.cur];
    int rc = launch_cons_to_prim(&s.g, s.f[s.cur], p[0], p[1], p[2], p[3], p[4],
                                 ws_field{nullptr, 0, 0}, s.status, st);
    if (rc) return rc;
    ws_job job{{4, 4, 4}, {s.g.nx + 4, s.g.ny + 4, s.g.nz + 4}};
    return launch_sound_speed(&s.g, job, p[4], p[5], st);
}

int grid_state_upload(GridState& s, const double* f_host, cudaStream_t st) {
    const size_t n = (size_t)5 * s.g.nx * s.g.ny * s.g.nz;
    WS_CUDA(cudaMemsetAsync(s.status, 0, sizeof(int), st));     // a new state, a new status
    WS_CUDA(cudaMemcpyAsync(s.f[s.cur].ptr, f_host, n * sizeof(double), cudaMemcpyHostToDevice,
                            st));
    return grid_state_derive(s, st);
}

int grid_state_download(GridState& s, double* f_host, cudaStream_t st) {
    const size_t n = (size_t)5 * s.g.nx * s.g.ny * s.g.nz;
    WS_CUDA(cudaMemcpyAsync(f_host, s.f[s.cur].ptr, n * sizeof(double), cudaMemcpyDeviceToHost,
                            st));
    return WS_OK;
}

// ---------------------------------------------------------------------------
// BatchRunner
// ---------------------------------------------------------------------------
BatchRunner::~BatchRunner() { release(nullptr); }

void BatchRunner::drop_graphs() {
    for (auto& e : exec_)
        if (e) {
            cudaGraphExecDestroy(e);
            e = nullptr;
        }
}

void BatchRunner::release(cudaStream_t st) {
    drop_graphs();
    if (dev_) cudaFreeAsync(dev_, st);
    dev_ = nullptr;
    dev_bytes_ = 0;
    if (cap_) cudaStreamDestroy(cap_);
    cap_ = nullptr;
    grids_.clear();
}

int batch_kernel_cfg(const std::vector<GridState*>& grids, ws_tile tile) {
    (void)grids;
    if (tile.tile_x < 0) return -1;
    if (tile.tile_x || tile.tile_y || tile.threads) {
        const int c = find_tile_cfg(tile.tile_x, tile.tile_y, tile.threads);
        return c < 0 ? -2 : c;
    }
    return -1;
}

int BatchRunner::build(const std::vector<GridState*>& grids, int cfg, int zc, cudaStream_t st) {
    drop_graphs();
    grids_ = grids;
    pencil_ = cfg < 0;
    if (pencil_) cfg = 0;       // argument tables as for tile 0 (its fields unused)
    cfg_ = cfg;
    zc_ = zc > 0 ? zc : (1 << 30);
    parity_ = 0;
    const int n = (int)grids.size();
    if (n == 0) return WS_OK;
    precision_ = grids[0]->g.precision;
    for (auto* s : grids)
        if (s->g.precision != precision_ || !s->g.metrics_uniform)
            return fail(WS_ERR_INVALID, "a batch holds Cartesian grids of one precision");
    long n_gtab = 0;
    for (auto* s : grids) n_gtab += ghost_chunks(&s->g);
    if (n_gtab > (1L << 30)) return fail(WS_ERR_INVALID, "batch too large");
    n_gtab_ = (int)n_gtab;
    // persistent CTAs of the RHS launches
    closure_ = false;
    for (auto* s : grids)
        for (int i = 0; i < 4; ++i) closure_ |= s->g.face_kind[i] == WS_FACE_CLOSURE;
    const int maxc = rhs_max_ctas(precision_, true, closure_, cfg_, true);
    if (maxc <= 0) return fail(WS_ERR_CUDA, "cannot size the persistent grid");
    const TileCfg tc = tile_cfg(cfg);
    long planes = 0;
    for (auto* s : grids)
        planes += (long)(((int)s->g.nx + tc.bx - 1) / tc.bx) *
                  (((int)s->g.ny + tc.by - 1) / tc.by) * s->g.nz;
    ctas_ = (int)std::max(1L, std::min<long>(maxc, std::max<long>(1, planes / 16)));
    // the RHS launches' work items: z runs of at most zc planes per tile, and
    // short enough (down to 8 planes) that a small batch still gives every
    // CTA two items or more (whole columns would leave most SMs idle on a few
    // small grids)
    const long fill = std::max(8L, (planes + 2L * ctas_ - 1) / (2L * ctas_));
    const std::vector<int4> items = batch_items(grids, cfg, (int)std::min<long>(zc_, fill));
    // layout of the device tables: 4 RhsArgs sets, work items + their
    // counter, 2 ghost sets, block table
    const size_t gsz = ghost_args_size();
    size_t o = 0, o_rhs[4], o_gh[2];
    for (int k = 0; k < 4; ++k) {
        o_rhs[k] = o;
        o = align256(o + n * sizeof(RhsArgs));
    }
    const size_t o_items = o;
    o = align256(o + items.size() * sizeof(int4));
    const size_t o_ctr = o;
    o = align256(o + sizeof(unsigned));
    for (int k = 0; k < 2; ++k) {
        o_gh[k] = o;
        o = align256(o + n * gsz);
    }
    const size_t o_gt = o;
    o = align256(o_gt + n_gtab * sizeof(int2));
    const size_t o_woff = o;           // line passes: 3 x (n + 1) work prefixes
    const size_t bytes = align256(o_woff + 3 * (size_t)(n + 1) * sizeof(long));
    host_.assign(bytes, 0);
    unsigned char* h = host_.data();
    if (!items.empty())
        std::memcpy(h + o_items, items.data(), items.size() * sizeof(int4));
    int2* hgt = reinterpret_cast<int2*>(h + o_gt);
    long* hw = reinterpret_cast<long*>(h + o_woff);
    for (int dir = 0; dir < 3; ++dir) {
        long* w = hw + dir * (n + 1);
        w[0] = 0;
        for (int i = 0; i < n; ++i) w[i + 1] = w[i] + pencil_pass_work(grids[i]->g, dir);
    }
    long gi = 0;
    for (int i = 0; i < n; ++i) {
        GridState* s = grids[i];
        if (s->args.size() != 4 || s->args_cfg != cfg || s->args_zc != zc_ ||
            s->args_dt != s->dt) {
            ws_job job{{4, 4, 4}, {s->g.nx + 4, s->g.ny + 4, s->g.nz + 4}};
            s->args.resize(4);
            for (int c = 0; c < 2; ++c)
                for (int two = 0; two < 2; ++two) {
                    // stage 2 reads pr[1-c] and writes pr[c]; stages 1 and 3 the reverse
                    const ws_field* pin = s->pr[two ? 1 - c : c];
                    const ws_field* pout = s->pr[two ? c : 1 - c];
                    const ws_field p5[5] = {pin[0], pin[1], pin[2], pin[3], pin[5]};
                    RhsArgs& a = s->args[2 * c + two];
                    a = make_rhs_args(&s->g, job, p5, nullptr, s->du, cfg, zc_);
                    int rc = set_rhs_stage(a, &s->g, s->f[1 - c], s->f[c], s->f[1 - c], pout,
                                           s->dt, s->status);
                    if (rc) return rc;
                }
            s->args_cfg = cfg;
            s->args_zc = zc_;
            s->args_dt = s->dt;
        }
        for (int p = 0; p < 2; ++p) {
            const int c = s->cur ^ p;
            for (int two = 0; two < 2; ++two)
                std::memcpy(h + o_rhs[2 * p + two] + i * sizeof(RhsArgs), &s->args[2 * c + two],
                            sizeof(RhsArgs));
            fill_ghost_args(h + o_gh[p] + i * gsz, &s->g, s->pr[c]);
        }
        for (long c = 0; c < ghost_chunks(&s->g); ++c) hgt[gi++] = make_int2(i, (int)c);
    }
    if (bytes > dev_bytes_) {
        if (dev_) cudaFreeAsync(dev_, st);
        dev_ = nullptr;
        WS_CUDA(cudaMallocAsync(&dev_, bytes, st));
        dev_bytes_ = bytes;
    }
    unsigned char* d = static_cast<unsigned char*>(dev_);
    for (int k = 0; k < 4; ++k) d_rhs_[k] = reinterpret_cast<RhsArgs*>(d + o_rhs[k]);
    work_ = {reinterpret_cast<const int4*>(d + o_items), (int)items.size(),
             reinterpret_cast<unsigned*>(d + o_ctr)};
    for (int k = 0; k < 2; ++k) d_ghost_[k] = d + o_gh[k];
    d_gtab_ = reinterpret_cast<int2*>(d + o_gt);
    d_woff_ = reinterpret_cast<const long*>(d + o_woff);
    int rc = upload_tables(st);
    if (rc) return rc;
    return WS_OK;
}

int BatchRunner::upload_tables(cudaStream_t st) {
    WS_CUDA(cudaMemcpyAsync(dev_, host_.data(), host_.size(), cudaMemcpyHostToDevice, st));
    // host_ must stay unchanged until the copy has read it
    WS_CUDA(cudaStreamSynchronize(st));
    return WS_OK;
}

// du of every grid's current state; d_rhs_[2 * parity_] reads pr[cur]
int BatchRunner::enqueue_rhs(cudaStream_t st) {
    if (grids_.empty()) return WS_OK;
    int rc = launch_ghost_fill_batch(d_ghost_[parity_], d_gtab_, n_gtab_, st);
    if (rc) return rc;
    if (pencil_)
        return launch_rhs_pencil_batch(d_rhs_[2 * parity_], d_woff_, (int)grids_.size(),
                                       precision_, 0, closure_, st);
    return launch_rhs_batch(d_rhs_[2 * parity_], work_, precision_, true, closure_, cfg_, ctas_, 0,
                            st);
}

// stage 1 alone: reads f[cur], pr[cur] and writes only the other buffers,
// so it can be repeated without changing the current state
int BatchRunner::enqueue_stage1(cudaStream_t st) {
    if (grids_.empty()) return WS_OK;
    int rc = launch_ghost_fill_batch(d_ghost_[parity_], d_gtab_, n_gtab_, st);
    if (rc) return rc;
    if (pencil_)
        return launch_rhs_pencil_batch(d_rhs_[2 * parity_], d_woff_, (int)grids_.size(),
                                       precision_, 1, closure_, st);
    return launch_rhs_batch(d_rhs_[2 * parity_], work_, precision_, true, closure_, cfg_, ctas_, 1,
                            st);
}

int BatchRunner::enqueue_step(cudaStream_t st) {
    if (grids_.empty()) return WS_OK;
    for (int krk = 1; krk <= 3; ++krk) {
        const int two = krk == 2;
        int rc = launch_ghost_fill_batch(d_ghost_[parity_ ^ two], d_gtab_, n_gtab_, st);
        if (rc) return rc;
        rc = pencil_ ? launch_rhs_pencil_batch(d_rhs_[2 * parity_ + two], d_woff_,
                                               (int)grids_.size(), precision_, krk, closure_, st)
                     : launch_rhs_batch(d_rhs_[2 * parity_ + two], work_, precision_, true,
                                        closure_, cfg_, ctas_, krk, st);
        if (rc) return rc;
    }
    return WS_OK;
}

int BatchRunner::step_eager(int nsteps, cudaStream_t st) {
    if (grids_.empty()) return WS_OK;
    for (int i = 0; i < nsteps; ++i) {
        int rc = enqueue_step(st);
        if (rc) return rc;
        parity_ ^= 1;
        for (auto* s : grids_) s->cur ^= 1;
    }
    return WS_OK;
}

int BatchRunner::step(int nsteps, cudaStream_t st) {
    if (grids_.empty() || nsteps <= 0) return WS_OK;
    if (!exec_[0]) {
        if (!cap_) WS_CUDA(cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking));
        const int keep = parity_;
        for (int p = 0; p < 2; ++p) {
            parity_ = p;
            cudaGraph_t graph = nullptr;
            WS_CUDA(cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal));
            int rc = enqueue_step(cap_);
            cudaError_t e = cudaStreamEndCapture(cap_, &graph);
            if (rc) {
                if (graph) cudaGraphDestroy(graph);
                parity_ = keep;
                return rc;
            }
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&exec_[p], graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
        }
        parity_ = keep;
    }
    for (int i = 0; i < nsteps; ++i) {
        WS_CUDA(cudaGraphLaunch(exec_[parity_], st));
        parity_ ^= 1;
        for (auto* s : grids_) s->cur ^= 1;
    }
    return WS_OK;
}

}  // namespace ws

using namespace ws;

// ===========================================================================
// C ABI
// ===========================================================================
struct ws_batch {
    std::vector<GridState> states;
    BatchRunner runner;
    ws_tile tile{0, 0, 0, 0};
    bool dirty = true;
};

namespace {
int batch_ready(ws_batch* b, cudaStream_t st) {
    if (!b->dirty) return WS_OK;
    std::vector<GridState*> ptrs;
    for (auto& s : b->states) ptrs.push_back(&s);
    const int cfg = batch_kernel_cfg(ptrs, b->tile);
    if (cfg == -2) return fail(WS_ERR_UNSUPPORTED, "tile shape not compiled in this build");
    int rc = b->runner.build(ptrs, cfg, b->tile.scan_z, st);
    if (rc == WS_OK) b->dirty = false;
    return rc;
}
}  // namespace

extern "C" {

int ws_batch_create(const ws_grid* grids, int n, ws_batch** out) {
    if (!out) return fail(WS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!grids || n <= 0) return fail(WS_ERR_INVALID, "need at least one grid");
    for (int i = 0; i < n; ++i) {
        const ws_grid& g = grids[i];
        if (int rc = validate_grid(&g)) return rc;
        if (has_external(&g))
            return fail(WS_ERR_UNSUPPORTED, "EXTERNAL faces need a halo exchange");
        if (g.lap != WS_LAP || g.nx < 4 || g.ny < 4 || g.nz < 4 || !g.metrics_uniform ||
            (g.precision != WS_FP64 && g.precision != WS_MIXED) ||
            g.precision != grids[0].precision)
            return fail(WS_ERR_INVALID, "batch grids: Cartesian, n >= 4, one precision");
    }
    std::unique_ptr<ws_batch> b(new (std::nothrow) ws_batch());
    if (!b) return fail(WS_ERR_ALLOC, "host allocation failed");
    b->states.resize(n);
    for (int i = 0; i < n; ++i) {
        int rc = grid_state_alloc(b->states[i], grids[i], nullptr);
        if (rc) {
            for (auto& s : b->states) grid_state_free(s, nullptr);
            return rc;
        }
    }
    WS_CUDA(cudaStreamSynchronize(nullptr));
    *out = b.release();
    return WS_OK;
}

void ws_batch_destroy(ws_batch* b) {
    if (!b) return;
    cudaDeviceSynchronize();
    b->runner.release(nullptr);
    for (auto& s : b->states) grid_state_free(s, nullptr);
    cudaStreamSynchronize(nullptr);
    delete b;
}

int ws_batch_size(ws_batch* b) { return b ? (int)b->states.size() : 0; }

int ws_batch_set_state(ws_batch* b, int i, const double* f_host, ws_stream_t stream) {
    if (!b || !f_host || i < 0 || i >= (int)b->states.size())
        return fail(WS_ERR_INVALID, "bad batch index or NULL state");
    return grid_state_upload(b->states[i], f_host, (cudaStream_t)stream);
}

int ws_batch_get_state(ws_batch* b, int i, double* f_host, ws_stream_t stream) {
    if (!b || !f_host || i < 0 || i >= (int)b->states.size())
        return fail(WS_ERR_INVALID, "bad batch index or NULL state");
    int rc = grid_state_download(b->states[i], f_host, (cudaStream_t)stream);
    if (rc) return rc;
    WS_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return WS_OK;
}

int ws_batch_get_rhs(ws_batch* b, int i, double* du_host, ws_stream_t stream) {
    if (!b || !du_host || i < 0 || i >= (int)b->states.size())
        return fail(WS_ERR_INVALID, "bad batch index or NULL buffer");
    const GridState& s = b->states[i];
    const size_t n = (size_t)5 * s.g.nx * s.g.ny * s.g.nz;
    cudaStream_t st = (cudaStream_t)stream;
    WS_CUDA(cudaMemcpyAsync(du_host, s.du.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    WS_CUDA(cudaStreamSynchronize(st));
    return WS_OK;
}

int ws_batch_compute_dt(ws_batch* b, double cfl, double* dt_out, ws_stream_t stream) {
    if (!b || !dt_out) return fail(WS_ERR_INVALID, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int n = (int)b->states.size();
    unsigned long long* d = nullptr;
    WS_CUDA(cudaMallocAsync(&d, n * sizeof(unsigned long long), st));
    WS_CUDA(cudaMemsetAsync(d, 0, n * sizeof(unsigned long long), st));
    for (int i = 0; i < n; ++i) {
        int rc = launch_max_speed(&b->states[i].g, b->states[i].prims(), d + i, st);
        if (rc) return rc;
    }
    std::vector<unsigned long long> h(n);
    WS_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            st));
    WS_CUDA(cudaFreeAsync(d, st));
    WS_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) {
        double m;
        std::memcpy(&m, &h[i], sizeof m);
        if (!wave_speed_ok(m))
            return fail(WS_ERR_NONFINITE, "grid " + std::to_string(i) +
                                              ": maximum wave speed is not finite and positive");
        dt_out[i] = cfl / m;
    }
    return WS_OK;
}

int ws_batch_set_dt(ws_batch* b, const double* dt) {
    if (!b || !dt) return fail(WS_ERR_INVALID, "NULL argument");
    for (size_t i = 0; i < b->states.size(); ++i) {
        if (!(dt[i] > 0)) return fail(WS_ERR_INVALID, "dt must be > 0");
        b->states[i].dt = dt[i];
    }
    b->dirty = true;
    return WS_OK;
}

int ws_batch_set_tile(ws_batch* b, ws_tile tile) {
    if (!b) return fail(WS_ERR_INVALID, "batch is NULL");
    if (tile.tile_x >= 0 && (tile.tile_x || tile.tile_y || tile.threads) &&
        find_tile_cfg(tile.tile_x, tile.tile_y, tile.threads) < 0)
        return fail(WS_ERR_UNSUPPORTED, "tile shape not compiled in this build");
    b->tile = tile;
    b->dirty = true;
    return WS_OK;
}

int ws_batch_get_tile(ws_batch* b, ws_tile* tile) {
    if (!b || !tile) return fail(WS_ERR_INVALID, "NULL argument");
    *tile = b->tile;
    return WS_OK;
}

int ws_batch_rhs(ws_batch* b, ws_stream_t stream) {
    if (!b) return fail(WS_ERR_INVALID, "batch is NULL");
    int rc = batch_ready(b, (cudaStream_t)stream);
    if (rc) return rc;
    return b->runner.enqueue_rhs((cudaStream_t)stream);
}

int ws_batch_step(ws_batch* b, int nsteps, ws_stream_t stream) {
    if (!b) return fail(WS_ERR_INVALID, "batch is NULL");
    for (auto& s : b->states)
        if (!(s.dt > 0)) return fail(WS_ERR_INVALID, "set dt (ws_batch_set_dt) before stepping");
    int rc = batch_ready(b, (cudaStream_t)stream);
    if (rc) return rc;
    return b->runner.step(nsteps, (cudaStream_t)stream);
}

int ws_batch_status(ws_batch* b, int* status, ws_stream_t stream) {
    if (!b || !status) return fail(WS_ERR_INVALID, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    for (size_t i = 0; i < b->states.size(); ++i)
        WS_CUDA(cudaMemcpyAsync(&status[i], b->states[i].status, sizeof(int),
                                cudaMemcpyDeviceToHost, st));
    WS_CUDA(cudaStreamSynchronize(st));
    for (size_t i = 0; i < b->states.size(); ++i) status[i] = status_code(status[i]);
    return WS_OK;
}

// Times the candidate kernels on the first RK stage of this batch (ghost
// fill + RHS and stage update; the current state is left as it was) and
// keeps the fastest; returns its tile selection in *chosen.  Candidates: the
// line passes (tile_x = -1) and every compiled tile shape of the fused
// kernel with two sweep caps.
int ws_batch_autotune(ws_batch* b, ws_tile* chosen, ws_stream_t stream) {
    if (!b) return fail(WS_ERR_INVALID, "batch is NULL");
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    WS_CUDA(cudaEventCreate(&e0));
    WS_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    ws_tile best_tile{0, 0, 0, 0};
    std::vector<ws_tile> cand{ws_tile{-1, 0, 0, 0}};
    for (int c = 0; c < num_tile_cfgs(); ++c)
        for (int cap : {0, 32}) {
            const TileCfg tc = tile_cfg(c);
            cand.push_back(ws_tile{tc.bx, tc.by, cap, tc.threads});
        }
    for (const ws_tile& t : cand) {
        b->tile = t;
        b->dirty = true;
        int rc = batch_ready(b, st);
        if (rc == WS_OK) rc = b->runner.enqueue_stage1(st);    // warm-up
        if (rc) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return rc;
        }
        cudaEventRecord(e0, st);
        for (int r = 0; r < 2; ++r) b->runner.enqueue_stage1(st);
        cudaEventRecord(e1, st);
        WS_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            best_tile = b->tile;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tile = best_tile;
    b->dirty = true;
    if (chosen) *chosen = best_tile;
    return batch_ready(b, st);
}

}  // extern "C"
