// dt_static.cu -- CFL time step of caller-owned grids without any allocation.
//
// ws_batch_compute_dt reduces the maximum wave speed of each grid into a
// scratch array it allocates per call (cudaMallocAsync), and the solver keeps
// its own allocated accumulator.  Some callers cannot allocate device memory
// from inside their time loop: a host code that owns every device buffer
// through its own arena and treats allocation after start-up as an error (as
// a drop-in for the reference's inviscid path, whose host code allocates all
// fields once at start-up), or a code running under a hard device-memory cap
// where a late allocation can fail; cudaMalloc and cudaFree also wait for the
// device, which stalls a loop that is otherwise asynchronous.  For them,
// ws_compute_dt_static keeps its scratch in a fixed array compiled into the
// library instead.
//
// The array lives in every GPU that loads the library, for the life of the
// process (WS_DT_STATIC_MAX_GRIDS x 8 bytes).  Every call uses the same
// array and leaves its last contents there, so each call first clears the
// entries it uses, and calls whose device work overlaps (two streams, two
// host threads) race on it: serialise them.  Host code never dereferences
// the array's name -- in host code that name stands for a host-side shadow,
// not the device address -- the device address is looked up once per device
// with cudaGetSymbolAddress on the first call made with that device current
// and kept for the life of the process, so a cudaDeviceReset after that
// first call is not supported (the module reloads at another address).
#include <cstring>
#include <mutex>

#include "ws_internal.h"

namespace ws {
int launch_max_speed(const ws_grid* g, const ws_field prims[6], unsigned long long* out,
                     cudaStream_t st);
}

namespace {

// bits of a non-negative double per grid: max wave speed
static __device__ __align__(256) unsigned long long g_dt_scratch[WS_DT_STATIC_MAX_GRIDS];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned long long* g_addr[kMaxDevices] = {nullptr};

// device address of g_dt_scratch on the current device (set up once per device)
int scratch_address(unsigned long long** out) {
    int dev = 0;
    WS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return ws::fail(WS_ERR_UNSUPPORTED, "device ordinal beyond the static-scratch table");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_dt_scratch);
        if (e != cudaSuccess) return ws::cuda_fail(e, "cudaGetSymbolAddress(g_dt_scratch)");
        g_addr[dev] = static_cast<unsigned long long*>(p);
    }
    *out = g_addr[dev];
    return WS_OK;
}

}  // namespace

extern "C" int ws_compute_dt_static(const ws_grid* grids, const ws_field* prims, int n,
                                    double cfl, double* dt_out, ws_stream_t stream) {
    using namespace ws;
    if (!grids || !prims || !dt_out) return fail(WS_ERR_INVALID, "NULL argument");
    if (n < 1 || n > WS_DT_STATIC_MAX_GRIDS)
        return fail(WS_ERR_INVALID,
                    "ws_compute_dt_static: n must be 1.." + std::to_string(WS_DT_STATIC_MAX_GRIDS) +
                        " grids (the size of its fixed scratch array)");
    if (!(cfl > 0)) return fail(WS_ERR_INVALID, "cfl must be > 0");
    for (int i = 0; i < n; ++i) {
        const ws_grid& g = grids[i];
        if (g.lap != WS_LAP || g.nx < 1 || g.ny < 1 || g.nz < 1 || !(g.hx > 0) || !(g.hy > 0) ||
            !(g.hz > 0))
            return fail(WS_ERR_INVALID, "invalid grid " + std::to_string(i));
        for (int f = 0; f < 4; ++f)
            if (!prims[4 * i + f].ptr || prims[4 * i + f].pitch < g.nx + 8)
                return fail(WS_ERR_INVALID, "grid " + std::to_string(i) +
                                                ": u, v, w, cc need a pointer and pitch >= nx+8");
    }
    unsigned long long* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // the array keeps the previous call's maxima: clear the entries used
    WS_CUDA(cudaMemsetAsync(scratch, 0, (size_t)n * sizeof(unsigned long long), st));
    for (int i = 0; i < n; ++i) {
        // launch_max_speed reads u, v, w, cc from slots 1, 2, 3, 5
        const ws_field six[6] = {ws_field{}, prims[4 * i], prims[4 * i + 1], prims[4 * i + 2],
                                 ws_field{}, prims[4 * i + 3]};
        rc = launch_max_speed(&grids[i], six, scratch + i, st);
        if (rc) return rc;
    }
    // one copy of the n maxima, one synchronisation (32 KB on the stack at most)
    unsigned long long bits[WS_DT_STATIC_MAX_GRIDS];
    WS_CUDA(cudaMemcpyAsync(bits, scratch, (size_t)n * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, st));
    WS_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) {
        double v;
        std::memcpy(&v, &bits[i], sizeof v);
        if (!wave_speed_ok(v))
            return fail(WS_ERR_NONFINITE, "grid " + std::to_string(i) +
                                              ": maximum wave speed is not finite and positive");
        dt_out[i] = cfl / v;
    }
    return WS_OK;
}
