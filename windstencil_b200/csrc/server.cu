// server.cu -- continuous-batching solve server.
//
// No reference counterpart: the reference runs one solve per MPI job.  A solve
// request is (grid, initial state, number of SSP-RK3 steps, CFL, precision).
// A host thread runs the loop
//   admit  : move queued requests to active slots while the HBM state budget
//            and the slot limit allow; upload (or generate) the initial state
//            and compute its time step on the device;
//   tick   : SSP-RK3 steps of every active grid -- two batched launches per
//            stage and precision (BatchRunner) -- up to the next completion
//            (at most 4 steps while the queue is empty);
//   retire : grids that reached their step count copy their state back, free
//            their slot and record their latency.
// Requests arriving while others run are admitted at the next tick, so their
// work shares the device with the running ones; a grid's arithmetic does not
// depend on what else is in the batch.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "ws_internal.h"

namespace ws {
int launch_max_speed(const ws_grid* g, const ws_field prims[6], unsigned long long* out,
                     cudaStream_t st);

namespace {

// ---- seeded synthetic initial state on the device -------------------------
// Periodic Sod-type state: left rho = 1, p = 1/gamma; right rho = 0.125,
// p = 0.1/gamma (jump at x_jump * nx); u = mach; v, w and rho carry 1%
// uniform noise from a counter-based hash (splitmix64) of (seed, cell, field).
__device__ __forceinline__ double hash_uniform(unsigned long long seed, unsigned long long n) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (n + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;   // [-1, 1)
}

__global__ void synth_state_kernel(ws_soa f, int nx, int ny, int nz, double gamma, double ama,
                                   double mach, double x_jump, unsigned long long seed) {
    const long n = (long)nx * ny * nz;
    const double cv = 1.0 / (gamma * (gamma - 1.0) * ama * ama);
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx);
        const long r = t / nx;
        const int j = (int)(r % ny), k = (int)(r / ny);
        const bool left = (i + 0.5) < x_jump * nx;
        double d = left ? 1.0 : 0.125;
        const double p = (left ? 1.0 : 0.1) / gamma;
        d *= 1.0 + 0.01 * hash_uniform(seed, 3 * (unsigned long long)t);
        const double u = mach * ama;
        const double v = 0.01 * hash_uniform(seed, 3 * (unsigned long long)t + 1);
        const double w = 0.01 * hash_uniform(seed, 3 * (unsigned long long)t + 2);
        const double T = gamma * ama * ama * p / d;
        const size_t o = (size_t)i + (size_t)f.pitch * ((size_t)j + (size_t)f.length_Y * k);
        const size_t vs = (size_t)f.pitch * f.length_Y * f.length_Z;
        f.ptr[o] = d;
        f.ptr[o + vs] = u * d;
        f.ptr[o + 2 * vs] = v * d;
        f.ptr[o + 3 * vs] = w * d;
        f.ptr[o + 4 * vs] = d * ((u * u + v * v + w * w) * 0.5 + cv * T);
    }
}

// status words of the active grids, gathered into one array for one copy
__global__ void gather_status_kernel(int* const* words, int n, int* out) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) out[i] = *words[i];
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

enum { RQ_QUEUED = 0, RQ_RUNNING = 1, RQ_DONE = 2, RQ_FAILED = 3 };

struct Req {
    uint64_t id = 0;
    ws_request r{};
    GridState st;
    int steps_done = 0;
    int state = RQ_QUEUED;
    int error = WS_OK;
    double t_submit = 0, t_admit = 0, t_done = 0;
    size_t bytes = 0;
};

}  // namespace
}  // namespace ws

using namespace ws;

struct ws_server {
    ws_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> queue;
    std::map<uint64_t, std::unique_ptr<Req>> reqs;
    std::vector<Req*> active;
    uint64_t next_id = 1;
    size_t used = 0;
    bool stop = false;
    int dev = 0;
    std::thread th;
    cudaStream_t stream = nullptr;
    BatchRunner runner[2];          // per precision
    bool rebuild = true;
    // status words of the active grids (device table of pointers, gathered
    // after every tick so that a request whose state turned non-finite stops
    // at once instead of stepping NaNs to its step count)
    int** d_words = nullptr;
    int* d_status = nullptr;
    int* h_status = nullptr;        // pinned
    int** h_words = nullptr;        // pinned: the pointer table's upload source
    int n_words = 0, cap_words = 0;
    // statistics
    std::vector<double> latencies;
    double served_cell_rhs = 0, executed_cell_rhs = 0, t_start = 0, t_last = 0;
    long ticks = 0, admitted = 0, completed = 0, failed = 0, max_active_seen = 0;
    double busy_s = 0;
    double t_admit = 0, t_rebuild = 0, t_steps = 0, t_retire = 0;   // per-phase host clock
    double active_cells = 0;
};

namespace {

constexpr int kTickSteps = 4;

double cells_of(const Req* q) {
    return (double)q->r.grid.nx * q->r.grid.ny * q->r.grid.nz;
}

// FIFO admission: memory (HBM budget) and compute (active cells) both cap the
// running set; the compute cap keeps a tick short once the device is full,
// so admitted requests finish sooner instead of all slowing down together.
int admit_locked(ws_server* s, std::vector<Req*>& fresh) {
    double cells = s->active_cells;
    for (Req* q : fresh) cells += cells_of(q);
    while (!s->queue.empty() && (int)s->active.size() + (int)fresh.size() < s->cfg.max_active) {
        Req* q = s->reqs[s->queue.front()].get();
        const bool idle = s->active.empty() && fresh.empty();
        if (!idle && cells + cells_of(q) > (double)s->cfg.max_active_cells) break;
        if (s->used + q->bytes > s->cfg.hbm_budget_bytes) {
            if (s->active.empty() && fresh.empty()) {       // can never fit
                q->state = RQ_FAILED;
                q->error = WS_ERR_BUDGET;
                s->queue.pop_front();
                s->failed++;
                s->cv_done.notify_all();
                continue;
            }
            break;                                          // wait for memory
        }
        s->queue.pop_front();
        s->used += q->bytes;
        cells += cells_of(q);
        q->state = RQ_RUNNING;
        q->t_admit = now_s();
        fresh.push_back(q);
    }
    return WS_OK;
}

// device work of admission: allocate, initial state, time step
int start_requests(ws_server* s, std::vector<Req*>& fresh) {
    cudaStream_t st = s->stream;
    const int n = (int)fresh.size();
    if (!n) return WS_OK;
    unsigned long long* d = nullptr;
    WS_CUDA(cudaMallocAsync(&d, n * sizeof(unsigned long long), st));
    WS_CUDA(cudaMemsetAsync(d, 0, n * sizeof(unsigned long long), st));
    for (int i = 0; i < n; ++i) {
        Req* q = fresh[i];
        int rc = grid_state_alloc(q->st, q->r.grid, st);
        if (rc) return rc;
        if (q->r.f0_host) {
            rc = grid_state_upload(q->st, q->r.f0_host, st);
        } else {
            const ws_grid& g = q->r.grid;
            const long cells = (long)g.nx * g.ny * g.nz;
            synth_state_kernel<<<(int)std::min<long>((cells + 255) / 256, 148L * 8), 256, 0, st>>>(
                q->st.f[q->st.cur], g.nx, g.ny, g.nz, g.gamma, g.ama, q->r.synth_mach,
                q->r.synth_x_jump, q->r.synth_seed);
            WS_CUDA(cudaGetLastError());
            rc = grid_state_derive(q->st, st);
        }
        if (rc) return rc;
        if (q->r.dt > 0) continue;
        rc = launch_max_speed(&q->r.grid, q->st.prims(), d + i, st);
        if (rc) return rc;
    }
    std::vector<unsigned long long> h(n);
    WS_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            st));
    WS_CUDA(cudaFreeAsync(d, st));
    WS_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) {
        Req* q = fresh[i];
        if (q->r.dt > 0) {
            q->st.dt = q->r.dt;
        } else {
            double m;
            std::memcpy(&m, &h[i], sizeof m);
            q->st.dt = wave_speed_ok(m) ? q->r.cfl / m : 0.0;   // 0: the request fails
        }
    }
    return WS_OK;
}

void finish(ws_server* s, Req* q, int error) {
    q->t_done = now_s();
    q->state = error ? RQ_FAILED : RQ_DONE;
    q->error = error;
    s->used -= q->bytes;
    if (error) {
        s->failed++;
    } else {
        s->completed++;
        s->latencies.push_back(q->t_done - q->t_submit);
        const ws_grid& g = q->r.grid;
        s->served_cell_rhs += 3.0 * q->r.nsteps * (double)g.nx * g.ny * g.nz;
    }
}

void loop(ws_server* s) {
    cudaSetDevice(s->dev);
    cudaStream_t st = s->stream;
    for (;;) {
        std::vector<Req*> fresh;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->active.empty())
                s->cv_work.wait_for(lk, std::chrono::milliseconds(50),
                                    [&] { return s->stop || !s->queue.empty(); });
            if (s->stop) break;
            admit_locked(s, fresh);
        }
        const double t0 = now_s();
        double tp = t0;
        auto phase = [&](double& acc) {
            const double t = now_s();
            acc += t - tp;
            tp = t;
        };
        if (!fresh.empty()) {
            int rc = start_requests(s, fresh);
            std::lock_guard<std::mutex> lk(s->mu);
            for (Req* q : fresh) {
                if (rc || !(q->st.dt > 0)) {
                    grid_state_free(q->st, st);
                    finish(s, q, rc ? rc : WS_ERR_NONFINITE);
                } else {
                    s->active.push_back(q);
                    s->active_cells += cells_of(q);
                    s->admitted++;
                }
            }
            s->rebuild = true;
            s->max_active_seen = std::max<long>(s->max_active_seen, (long)s->active.size());
            s->cv_done.notify_all();
        }
        phase(s->t_admit);
        if (s->active.empty()) continue;
        if (s->rebuild) {
            for (int p = 0; p < 2; ++p) {
                std::vector<GridState*> g;
                for (Req* q : s->active)
                    if (q->r.grid.precision == p) g.push_back(&q->st);
                const ws_tile& t = s->cfg.tile;
                int cfg = batch_kernel_cfg(g, t);
                if (cfg == -2) cfg = -1;        // a shape not compiled: the line passes
                s->runner[p].build(g, cfg, t.scan_z, st);
            }
            const int na = (int)s->active.size();
            if (na > s->cap_words) {
                cudaStreamSynchronize(st);      // the old tables are idle
                cudaFree(s->d_words);
                cudaFree(s->d_status);
                if (s->h_status) cudaFreeHost(s->h_status);
                if (s->h_words) cudaFreeHost(s->h_words);
                s->cap_words = std::max(na, 2 * s->cap_words);
                if (cudaMalloc(&s->d_words, s->cap_words * sizeof(int*)) != cudaSuccess ||
                    cudaMalloc(&s->d_status, s->cap_words * sizeof(int)) != cudaSuccess ||
                    cudaMallocHost(&s->h_status, s->cap_words * sizeof(int)) != cudaSuccess ||
                    cudaMallocHost(&s->h_words, s->cap_words * sizeof(int*)) != cudaSuccess) {
                    cudaGetLastError();
                    s->d_words = nullptr;
                    s->d_status = nullptr;
                    s->h_status = nullptr;
                    s->h_words = nullptr;
                    s->cap_words = 0;
                }
            }
            s->n_words = 0;
            if (s->cap_words >= na) {
                // the previous upload from h_words was complete at the last
                // tick's synchronisation
                for (int i = 0; i < na; ++i) s->h_words[i] = s->active[i]->st.status;
                cudaMemcpyAsync(s->d_words, s->h_words, na * sizeof(int*), cudaMemcpyHostToDevice,
                                st);
                s->n_words = na;
            }
            s->rebuild = false;
        }
        phase(s->t_rebuild);
        // steps this tick: up to the first completion; at most kTickSteps
        // while nothing waits in the queue (a request arriving now is then
        // admitted within that many steps)
        int k = 1 << 30;
        for (Req* q : s->active) k = std::min(k, q->r.nsteps - q->steps_done);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->queue.empty()) k = std::min(k, kTickSteps);
        }
        k = std::max(k, 1);
        // the batch changes every few ticks: launch the steps directly
        // rather than capture a graph for each new batch
        for (int p = 0; p < 2; ++p) s->runner[p].step_eager(k, st);
        if (s->n_words > 0) {
            gather_status_kernel<<<1, 256, 0, st>>>(s->d_words, s->n_words, s->d_status);
            cudaMemcpyAsync(s->h_status, s->d_status, s->n_words * sizeof(int),
                            cudaMemcpyDeviceToHost, st);
        }
        cudaStreamSynchronize(st);
        phase(s->t_steps);
        s->ticks++;
        s->executed_cell_rhs += 3.0 * k * s->active_cells;
        std::vector<Req*> done;
        for (size_t i = 0; i < s->active.size(); ++i) {
            Req* q = s->active[i];
            q->steps_done += k;
            // finished, or already failed (its status word is set)
            if (q->steps_done >= q->r.nsteps ||
                ((int)i < s->n_words && s->h_status[i] != 0))
                done.push_back(q);
        }
        if (!done.empty()) {
            int err = WS_OK;
            for (Req* q : done) {
                if (q->r.result_host &&
                    grid_state_download(q->st, q->r.result_host, st) != WS_OK)
                    err = WS_ERR_CUDA;
            }
            std::vector<int> status(done.size(), 0);
            for (size_t i = 0; i < done.size(); ++i)
                cudaMemcpyAsync(&status[i], done[i]->st.status, sizeof(int),
                                cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
            std::lock_guard<std::mutex> lk(s->mu);
            for (size_t i = 0; i < done.size(); ++i) {
                Req* q = done[i];
                grid_state_free(q->st, st);
                s->active.erase(std::find(s->active.begin(), s->active.end(), q));
                s->active_cells -= cells_of(q);
                finish(s, q, err ? err : status_code(status[i]));
            }
            s->rebuild = true;
            s->cv_done.notify_all();
        }
        phase(s->t_retire);
        s->busy_s += now_s() - t0;
        s->t_last = now_s();
    }
}

size_t request_bytes(const ws_grid& g) { return grid_state_bytes(g) + 4096; }

}  // namespace

extern "C" {

int ws_server_create(const ws_server_config* cfg, ws_server** out) {
    if (!out) return fail(WS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    std::unique_ptr<ws_server> s(new (std::nothrow) ws_server());
    if (!s) return fail(WS_ERR_ALLOC, "host allocation failed");
    if (cfg) s->cfg = *cfg;
    if (s->cfg.hbm_budget_bytes == 0) s->cfg.hbm_budget_bytes = (size_t)80 << 30;
    if (s->cfg.max_active <= 0) s->cfg.max_active = 4096;
    if (s->cfg.max_active_cells <= 0) s->cfg.max_active_cells = 32.0e6;
    WS_CUDA(cudaGetDevice(&s->dev));
    WS_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    // keep freed request memory in the pool instead of returning it to the OS,
    // and grow the pool once now to the working set the active-cell cap allows
    // (~330 B of state per cell): growing it request by request maps new
    // memory at every admission (measured ~23 ms per request, a fifth of the
    // loop's time under load)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, s->dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        const size_t warm = std::min<size_t>(s->cfg.hbm_budget_bytes,
                                             (size_t)(s->cfg.max_active_cells * 400.0));
        void* p = nullptr;
        if (cudaMallocAsync(&p, warm, s->stream) == cudaSuccess) {
            cudaFreeAsync(p, s->stream);
            cudaStreamSynchronize(s->stream);
        }
        cudaGetLastError();     // a device too small to warm this much is not an error
    }
    s->t_start = now_s();
    ws_server* raw = s.get();
    s->th = std::thread([raw] { loop(raw); });
    *out = s.release();
    return WS_OK;
}

void ws_server_destroy(ws_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->th.joinable()) s->th.join();
    for (auto& kv : s->reqs)
        if (kv.second->st.mem) grid_state_free(kv.second->st, s->stream);
    for (auto& r : s->runner) r.release(s->stream);
    cudaStreamSynchronize(s->stream);
    if (s->d_words) cudaFree(s->d_words);
    if (s->d_status) cudaFree(s->d_status);
    if (s->h_status) cudaFreeHost(s->h_status);
    if (s->h_words) cudaFreeHost(s->h_words);
    cudaStreamDestroy(s->stream);
    delete s;
}

int ws_server_submit(ws_server* s, const ws_request* r, uint64_t* id) {
    if (!s || !r) return fail(WS_ERR_INVALID, "NULL argument");
    const ws_grid& g = r->grid;
    if (int rc = validate_grid(&g)) return rc;
    if (has_external(&g))
        return fail(WS_ERR_UNSUPPORTED, "EXTERNAL faces need a halo exchange");
    if (g.lap != WS_LAP || g.nx < 4 || g.ny < 4 || g.nz < 4 || !g.metrics_uniform ||
        (g.precision != WS_FP64 && g.precision != WS_MIXED))
        return fail(WS_ERR_INVALID, "request grid: Cartesian, n >= 4, FP64 or mixed");
    if (r->nsteps < 1 || (!(r->dt > 0) && !(r->cfl > 0)))
        return fail(WS_ERR_INVALID, "request needs nsteps >= 1 and dt > 0 or cfl > 0");
    auto q = std::make_unique<Req>();
    q->r = *r;
    q->bytes = request_bytes(g);
    q->t_submit = now_s();
    std::lock_guard<std::mutex> lk(s->mu);
    if (q->bytes > s->cfg.hbm_budget_bytes)
        return fail(WS_ERR_BUDGET, "request state exceeds the server's HBM budget");
    q->id = s->next_id++;
    if (id) *id = q->id;
    s->queue.push_back(q->id);
    s->reqs[q->id] = std::move(q);
    s->cv_work.notify_all();
    return WS_OK;
}

int ws_server_poll(ws_server* s, uint64_t id, int* state, double* latency_s) {
    if (!s) return fail(WS_ERR_INVALID, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(WS_ERR_NOT_FOUND, "unknown request id");
    Req* q = it->second.get();
    if (state) *state = q->state;
    if (latency_s) *latency_s = q->state >= RQ_DONE ? q->t_done - q->t_submit : -1.0;
    return q->state == RQ_FAILED ? q->error : WS_OK;
}

int ws_server_wait(ws_server* s, uint64_t id, double timeout_s) {
    if (!s) return fail(WS_ERR_INVALID, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(WS_ERR_NOT_FOUND, "unknown request id");
    Req* q = it->second.get();
    const bool ok = s->cv_done.wait_for(
        lk, std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9),
        [&] { return q->state >= RQ_DONE; });
    if (!ok) return fail(WS_ERR_TIMEOUT, "request not finished within the timeout");
    if (q->state == RQ_FAILED) return fail(q->error, "request failed");
    return WS_OK;
}

int ws_server_get_stats(ws_server* s, ws_server_stats* out) {
    if (!s || !out) return fail(WS_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    std::vector<double> l = s->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) {
        if (l.empty()) return -1.0;
        const size_t i = std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5));
        return l[i];
    };
    std::memset(out, 0, sizeof *out);
    out->submitted = (long)s->reqs.size();
    out->queued = (long)s->queue.size();
    out->active = (long)s->active.size();
    out->completed = s->completed;
    out->failed = s->failed;
    out->ticks = s->ticks;
    out->max_active = s->max_active_seen;
    out->hbm_in_use = s->used;
    out->p50_latency_s = pct(0.50);
    out->p99_latency_s = pct(0.99);
    out->mean_latency_s = l.empty() ? -1.0 : [&] {
        double a = 0;
        for (double v : l) a += v;
        return a / l.size();
    }();
    out->served_cell_rhs = s->served_cell_rhs;
    out->executed_cell_rhs = s->executed_cell_rhs;
    out->busy_s = s->busy_s;
    out->admit_s = s->t_admit;
    out->rebuild_s = s->t_rebuild;
    out->steps_s = s->t_steps;
    out->retire_s = s->t_retire;
    out->elapsed_s = now_s() - s->t_start;
    return WS_OK;
}

// Forget finished requests (keeps the statistics).
int ws_server_release(ws_server* s, uint64_t id) {
    if (!s) return fail(WS_ERR_INVALID, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(WS_ERR_NOT_FOUND, "unknown request id");
    if (it->second->state < RQ_DONE) return fail(WS_ERR_BUSY, "request still queued or running");
    s->reqs.erase(it);
    return WS_OK;
}

}  // extern "C"
