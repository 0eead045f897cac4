// blocks.cu -- one grid split into blocks and stepped from C++.
//
// Replaces the reference's MPI decomposition and per-stage exchange: the
// NPX0 x NPY0 x NPZ0 process grid (OCFD_mpi.c:102-197), the packed plane
// exchange exchange_boundary_{x,y,z}_packed_dev (OCFD_mpi_dev.cpp:123-290)
// and the stage loop around it (OCFD_NS_Solver.cpp:64-90).  The reference
// copies every packed plane set through host memory and a blocking
// MPI_Sendrecv; here the planes stay on the device: a pack kernel, NCCL
// point-to-point sends between GPUs (or, for blocks sharing a process, the
// neighbour's pack buffer read in place), an unpack kernel, all in stream
// order.  Each block steps with its own ws_solver on a grid whose shared
// faces are WS_FACE_EXTERNAL.  The stencils are one-dimensional, so no edge
// or corner ghosts are needed and the axes' exchanges are independent.
//
// NCCL is loaded at run time (dlopen of libnccl.so.2): in a process that
// already holds NCCL (PyTorch's), the same library serves both.
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "ws_internal.h"

namespace ws {
namespace {

// ---- NCCL entry points, resolved once -------------------------------------
struct Nccl {
    bool tried = false, ok = false;
    std::string why;
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t,
                         cudaStream_t) = nullptr;
    ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t,
                               ncclComm_t, cudaStream_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
};

Nccl& nccl() {
    static Nccl n;
    if (n.tried) return n;
    n.tried = true;
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
        const char* e = dlerror();
        n.why = std::string("cannot load libnccl.so.2: ") + (e ? e : "?");
        return n;
    }
    bool all = true;
    auto sym = [&](auto& fn, const char* name) {
        fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
        if (!fn) {
            all = false;
            n.why = std::string("libnccl.so.2 lacks ") + name;
        }
    };
    sym(n.get_unique_id, "ncclGetUniqueId");
    sym(n.comm_init_rank, "ncclCommInitRank");
    sym(n.comm_destroy, "ncclCommDestroy");
    sym(n.group_start, "ncclGroupStart");
    sym(n.group_end, "ncclGroupEnd");
    sym(n.send, "ncclSend");
    sym(n.recv, "ncclRecv");
    sym(n.all_reduce, "ncclAllReduce");
    sym(n.error_string, "ncclGetErrorString");
    n.ok = all;
    return n;
}

int nccl_fail(ncclResult_t r, const char* what) {
    const char* s = nccl().error_string ? nccl().error_string(r) : "?";
    return fail(WS_ERR_COMM, std::string(what) + ": " + s);
}
#define WS_NCCL(call)                                              \
    do {                                                           \
        ncclResult_t r_ = (call);                                  \
        if (r_ != ncclSuccess) return nccl_fail(r_, #call);        \
    } while (0)

}  // namespace

// The point-to-point messages of one exchange of a block, in the order they
// are posted (one NCCL group): per axis, the send of the low planes, the
// send of the high planes, the receive of the high ghosts, the receive of
// the low ghosts.  NCCL matches the messages between two ranks in order, so
// with a two-block periodic ring (the same peer on both sides) the first
// message from the peer (its low planes) lands in the high ghosts and the
// second in the low ones; every rank walks the axes in the same order.
int exchange_plan(const ws_block_info& b, ws_p2p_op* ops, int cap) {
    int n = 0;
    auto put = [&](int kind, int peer, int axis, int side) {
        if (n < cap) ops[n] = ws_p2p_op{kind, peer, axis, side};
        ++n;
    };
    for (int ax = 0; ax < 3; ++ax) {
        const int lo = b.nbr[ax][0], hi = b.nbr[ax][1];
        if (lo >= 0) put(0, lo, ax, 0);
        if (hi >= 0) put(0, hi, ax, 1);
        if (hi >= 0) put(1, hi, ax, 1);
        if (lo >= 0) put(1, lo, ax, 0);
    }
    return n;
}

namespace {

// (first cell, cells) of part k of an axis of n cells split in P parts: the
// first n % P parts one cell wider (OCFD_mpi.c:124-145)
void part_extent(int n, int P, int k, int& first, int& cells) {
    const int base = n / P, rem = n % P;
    cells = base + (k < rem ? 1 : 0);
    first = k * base + std::min(k, rem);
}

}  // namespace

int decompose_block(const ws_grid* g, const int32_t dims[3], int32_t index, ws_block_info* out) {
    if (!g || !dims || !out) return fail(WS_ERR_INVALID, "NULL argument");
    for (int ax = 0; ax < 3; ++ax)
        if (dims[ax] < 1) return fail(WS_ERR_INVALID, "dims: three positive part counts");
    const long total = (long)dims[0] * dims[1] * dims[2];
    if (index < 0 || index >= total) return fail(WS_ERR_INVALID, "block index out of range");
    const int n_glob[3] = {(int)g->nx, (int)g->ny, (int)g->nz};
    for (int ax = 0; ax < 3; ++ax) {
        const int lo = g->face_kind[2 * ax], hi = g->face_kind[2 * ax + 1];
        if ((lo == WS_FACE_PERIODIC) != (hi == WS_FACE_PERIODIC))
            return fail(WS_ERR_INVALID, "axis " + std::to_string(ax) +
                                            " must be periodic at both faces or at neither");
        if (lo == WS_FACE_EXTERNAL || hi == WS_FACE_EXTERNAL)
            return fail(WS_ERR_INVALID, "the grid to split must not have EXTERNAL faces");
        if (n_glob[ax] < dims[ax])
            return fail(WS_ERR_INVALID, "cannot split " + std::to_string(n_glob[ax]) +
                                            " cells into " + std::to_string(dims[ax]) + " parts");
    }
    ws_block_info b{};
    b.index = index;
    b.coords[0] = index % dims[0];
    b.coords[1] = (index / dims[0]) % dims[1];
    b.coords[2] = index / (dims[0] * dims[1]);
    for (int ax = 0; ax < 3; ++ax) {
        const int P = dims[ax], k = b.coords[ax];
        const int lo = g->face_kind[2 * ax], hi = g->face_kind[2 * ax + 1];
        part_extent(n_glob[ax], P, k, b.origin[ax], b.n[ax]);
        int fl = lo, fh = hi;
        b.nbr[ax][0] = b.nbr[ax][1] = -1;
        if (P > 1) {
            const bool periodic = lo == WS_FACE_PERIODIC;
            const int left = k > 0 ? k - 1 : (periodic ? P - 1 : -1);
            const int right = k < P - 1 ? k + 1 : (periodic ? 0 : -1);
            int c[3] = {b.coords[0], b.coords[1], b.coords[2]};
            if (left >= 0) {
                c[ax] = left;
                b.nbr[ax][0] = c[0] + dims[0] * (c[1] + dims[1] * c[2]);
                fl = WS_FACE_EXTERNAL;
            }
            if (right >= 0) {
                c[ax] = right;
                b.nbr[ax][1] = c[0] + dims[0] * (c[1] + dims[1] * c[2]);
                fh = WS_FACE_EXTERNAL;
            }
        }
        // a ghost plane set comes from one neighbour's 4 nearest planes
        const int need = (fl == WS_FACE_CLOSURE || fh == WS_FACE_CLOSURE) ? 8 : 4;
        if (b.n[ax] < need)
            return fail(WS_ERR_INVALID, "block " + std::to_string(index) + " has " +
                                            std::to_string(b.n[ax]) + " cells along axis " +
                                            std::to_string(ax) + "; needs >= " +
                                            std::to_string(need));
        b.faces[2 * ax] = fl;
        b.faces[2 * ax + 1] = fh;
    }
    *out = b;
    return WS_OK;
}

}  // namespace ws

using namespace ws;

namespace {
// One block in this process: its grid, solver and halo buffers (per split
// axis and side, sized for the primitives' halo; the flux halo uses the
// leading part).
struct LocalBlock {
    ws_block_info info{};
    ws_grid g{};
    ws_solver* s = nullptr;
    double* send[3][2] = {};
    double* recv[3][2] = {};
};

constexpr int kPrimFields = 6;   // d, u, v, w, T, cc
constexpr int kFluxFields = 4;   // one direction's viscous fluxes Ev1..4
enum HaloKind { PRIMS, FLUX };
}  // namespace

struct ws_blocks {
    ws_grid g{};
    int32_t dims[3] = {1, 1, 1};
    std::vector<LocalBlock> blk;
    std::vector<int> local;      // block index -> position in blk, or -1
    bool viscous = false;
    int krk = 1;                 // the stage due next
    // NCCL (one block per rank)
    ncclComm_t comm = nullptr;
    int rank = 0, nranks = 1;
    double* d_min = nullptr;     // all-reduce scratch
};

namespace {
void release(ws_blocks* b) {
    for (auto& l : b->blk) {
        for (int ax = 0; ax < 3; ++ax)
            for (int sd = 0; sd < 2; ++sd) {
                cudaFree(l.send[ax][sd]);
                cudaFree(l.recv[ax][sd]);
            }
        ws_solver_destroy(l.s);
    }
    b->blk.clear();
    cudaFree(b->d_min);
    b->d_min = nullptr;
    if (b->comm && nccl().comm_destroy) nccl().comm_destroy(b->comm);
    b->comm = nullptr;
}

int add_block(ws_blocks* b, int index, bool remote) {
    LocalBlock l;
    int rc = decompose_block(&b->g, b->dims, index, &l.info);
    if (rc) return rc;
    l.g = b->g;
    l.g.nx = (uint32_t)l.info.n[0];
    l.g.ny = (uint32_t)l.info.n[1];
    l.g.nz = (uint32_t)l.info.n[2];
    for (int f = 0; f < 6; ++f) l.g.face_kind[f] = l.info.faces[f];
    b->blk.push_back(l);                 // owned from here (release frees it)
    LocalBlock& m = b->blk.back();
    if ((rc = ws_solver_create(&m.g, &m.s))) return rc;
    for (int ax = 0; ax < 3; ++ax)
        for (int sd = 0; sd < 2; ++sd) {
            if (m.info.nbr[ax][sd] < 0) continue;
            const size_t bytes = ws_halo_bytes(&m.g, ax, kPrimFields);
            if (cudaMalloc(&m.send[ax][sd], bytes) != cudaSuccess ||
                (remote && cudaMalloc(&m.recv[ax][sd], bytes) != cudaSuccess)) {
                cudaGetLastError();
                return fail(WS_ERR_ALLOC, "halo buffers");
            }
        }
    return WS_OK;
}
}  // namespace

namespace {
// the fields of a halo: the stage's primitives, or direction `axis`'s fluxes
int halo_fields(const ws_blocks* b, const LocalBlock& l, HaloKind kind, int axis,
                ws_field f[kPrimFields], int* nf) {
    if (kind == PRIMS) {
        *nf = kPrimFields;
        return ws_solver_stage_fields(l.s, b->krk, f);
    }
    *nf = kFluxFields;
    return ws_solver_stage_flux_fields(l.s, axis, f);
}

// Every block of the grid in this process: per axis, each block packs the
// planes next to its shared faces, then each unpacks its neighbours' packs
// into its ghost planes (no copy in between).
int exchange_local(ws_blocks* b, HaloKind kind, cudaStream_t st) {
    for (int ax = 0; ax < 3; ++ax) {
        for (auto& l : b->blk) {
            ws_field f[kPrimFields];
            int nf = 0;
            for (int sd = 0; sd < 2; ++sd) {
                if (l.info.nbr[ax][sd] < 0) continue;
                int rc = halo_fields(b, l, kind, ax, f, &nf);
                if (rc || (rc = ws_halo_pack(&l.g, f, nf, ax, sd, l.send[ax][sd],
                                             (ws_stream_t)st)))
                    return rc;
            }
        }
        for (auto& l : b->blk) {
            ws_field f[kPrimFields];
            int nf = 0;
            for (int sd = 0; sd < 2; ++sd) {
                const int nb = l.info.nbr[ax][sd];
                if (nb < 0) continue;
                const LocalBlock& o = b->blk[b->local[nb]];
                int rc = halo_fields(b, l, kind, ax, f, &nf);
                if (rc || (rc = ws_halo_unpack(&l.g, f, nf, ax, sd, o.send[ax][1 - sd],
                                               (ws_stream_t)st)))
                    return rc;
            }
        }
    }
    return WS_OK;
}

// One block per rank: pack every shared face, post the sends and receives
// of exchange_plan as one NCCL group, unpack.
int exchange_nccl(ws_blocks* b, HaloKind kind, cudaStream_t st) {
    LocalBlock& l = b->blk[0];
    ws_field f[3][kPrimFields];
    int nf[3] = {0, 0, 0};
    size_t count[3] = {0, 0, 0};
    bool any = false;
    for (int ax = 0; ax < 3; ++ax) {
        if (l.info.nbr[ax][0] < 0 && l.info.nbr[ax][1] < 0) continue;
        any = true;
        int rc = halo_fields(b, l, kind, ax, f[ax], &nf[ax]);
        if (rc) return rc;
        count[ax] = ws_halo_bytes(&l.g, ax, nf[ax]) / sizeof(double);
        for (int sd = 0; sd < 2; ++sd)
            if (l.info.nbr[ax][sd] >= 0 &&
                (rc = ws_halo_pack(&l.g, f[ax], nf[ax], ax, sd, l.send[ax][sd], (ws_stream_t)st)))
                return rc;
    }
    if (!any) return WS_OK;
    ws_p2p_op ops[12];
    const int nops = exchange_plan(l.info, ops, 12);
    Nccl& n = nccl();
    WS_NCCL(n.group_start());
    ncclResult_t r = ncclSuccess;
    for (int i = 0; i < nops && r == ncclSuccess; ++i) {
        const ws_p2p_op& o = ops[i];
        r = o.kind == 0
                ? n.send(l.send[o.axis][o.side], count[o.axis], ncclFloat64, o.peer, b->comm, st)
                : n.recv(l.recv[o.axis][o.side], count[o.axis], ncclFloat64, o.peer, b->comm, st);
    }
    const ncclResult_t re = n.group_end();       // closes the group in every case
    if (r != ncclSuccess) return nccl_fail(r, "ncclSend / ncclRecv");
    if (re != ncclSuccess) return nccl_fail(re, "ncclGroupEnd");
    for (int ax = 0; ax < 3; ++ax)
        for (int sd = 0; sd < 2; ++sd) {
            if (l.info.nbr[ax][sd] < 0) continue;
            int rc = ws_halo_unpack(&l.g, f[ax], nf[ax], ax, sd, l.recv[ax][sd], (ws_stream_t)st);
            if (rc) return rc;
        }
    return WS_OK;
}

int exchange(ws_blocks* b, HaloKind kind, cudaStream_t st) {
    return b->comm ? exchange_nccl(b, kind, st) : exchange_local(b, kind, st);
}

// stage b->krk of every local block: primitives' halo, first half, fluxes'
// halo (viscous), second half with the stage update
int stage(ws_blocks* b, double dt, cudaStream_t st) {
    int rc = exchange(b, PRIMS, st);
    if (rc) return rc;
    for (auto& l : b->blk)
        if ((rc = ws_solver_stage_begin(l.s, b->krk, (ws_stream_t)st))) return rc;
    if (b->viscous && (rc = exchange(b, FLUX, st))) return rc;
    for (auto& l : b->blk)
        if ((rc = ws_solver_stage_end(l.s, b->krk, dt, (ws_stream_t)st))) return rc;
    b->krk = b->krk % 3 + 1;
    return WS_OK;
}
}  // namespace

extern "C" {

int ws_blocks_decompose(const ws_grid* g, const int32_t dims[3], int32_t index,
                        ws_block_info* out) {
    return decompose_block(g, dims, index, out);
}

int ws_blocks_exchange_plan(const ws_grid* g, const int32_t dims[3], int32_t index,
                            ws_p2p_op* ops, int32_t cap, int32_t* count) {
    if (!count || (cap > 0 && !ops)) return fail(WS_ERR_INVALID, "NULL argument");
    ws_block_info b{};
    if (int rc = decompose_block(g, dims, index, &b)) return rc;
    *count = exchange_plan(b, ops, cap);
    return WS_OK;
}

int ws_nccl_unique_id(void* id) {
    if (!id) return fail(WS_ERR_INVALID, "NULL argument");
    Nccl& n = nccl();
    if (!n.ok) return fail(WS_ERR_UNSUPPORTED, n.why);
    ncclUniqueId u;
    WS_NCCL(n.get_unique_id(&u));
    std::memcpy(id, u.internal, sizeof u.internal);
    return WS_OK;
}

int ws_blocks_create(const ws_grid* g, const int32_t dims[3], const void* nccl_id, int32_t rank,
                     ws_blocks** out) {
    if (!g || !dims || !out) return fail(WS_ERR_INVALID, "NULL argument");
    *out = nullptr;
    ws_blocks* b = new ws_blocks;
    b->g = *g;
    for (int ax = 0; ax < 3; ++ax) b->dims[ax] = dims[ax];
    ws_block_info probe{};
    int rc = decompose_block(g, dims, 0, &probe);        // validates g and dims
    const long total = rc ? 0 : (long)dims[0] * dims[1] * dims[2];
    b->local.assign(total, -1);
    if (!rc && !nccl_id) {
        for (int i = 0; i < total && !rc; ++i) {
            b->local[i] = i;
            rc = add_block(b, i, false);
        }
    } else if (!rc) {
        b->nranks = (int)total;
        b->rank = rank;
        if (rank < 0 || rank >= total) {
            rc = fail(WS_ERR_INVALID, "rank out of range of the dims' product");
        } else if (!nccl().ok) {
            rc = fail(WS_ERR_UNSUPPORTED, nccl().why);
        } else {
            b->local[rank] = 0;
            rc = add_block(b, rank, true);
            if (!rc && cudaMalloc(&b->d_min, sizeof(double)) != cudaSuccess) {
                cudaGetLastError();
                rc = fail(WS_ERR_ALLOC, "all-reduce scratch");
            }
            if (!rc) {
                ncclUniqueId u;
                std::memcpy(u.internal, nccl_id, sizeof u.internal);
                const ncclResult_t r = nccl().comm_init_rank(&b->comm, (int)total, u, rank);
                if (r != ncclSuccess) {
                    b->comm = nullptr;
                    rc = nccl_fail(r, "ncclCommInitRank");
                }
            }
        }
    }
    if (rc) {
        release(b);
        delete b;
        return rc;
    }
    *out = b;
    return WS_OK;
}

void ws_blocks_destroy(ws_blocks* b) {
    if (!b) return;
    release(b);
    delete b;
}

int ws_blocks_count(ws_blocks* b, int32_t* count) {
    if (!b || !count) return fail(WS_ERR_INVALID, "NULL argument");
    *count = (int32_t)b->blk.size();
    return WS_OK;
}

int ws_blocks_info(ws_blocks* b, int32_t i, ws_block_info* out) {
    if (!b || !out) return fail(WS_ERR_INVALID, "NULL argument");
    if (i < 0 || i >= (int32_t)b->blk.size()) return fail(WS_ERR_INVALID, "no such local block");
    *out = b->blk[i].info;
    return WS_OK;
}

int ws_blocks_solver(ws_blocks* b, int32_t i, ws_solver** s) {
    if (!b || !s) return fail(WS_ERR_INVALID, "NULL argument");
    if (i < 0 || i >= (int32_t)b->blk.size()) return fail(WS_ERR_INVALID, "no such local block");
    *s = b->blk[i].s;
    return WS_OK;
}

int ws_blocks_set_viscous(ws_blocks* b, const ws_viscous* vis) {
    if (!b) return fail(WS_ERR_INVALID, "blocks are NULL");
    if (b->krk != 1) return fail(WS_ERR_INVALID, "a step is in progress");
    for (auto& l : b->blk)
        if (int rc = ws_solver_set_viscous(l.s, vis)) return rc;
    b->viscous = vis != nullptr;
    return WS_OK;
}

int ws_blocks_step(ws_blocks* b, double dt, int nsteps, ws_stream_t stream) {
    if (!b) return fail(WS_ERR_INVALID, "blocks are NULL");
    if (nsteps < 0 || !(dt > 0)) return fail(WS_ERR_INVALID, "need dt > 0 and nsteps >= 0");
    for (int i = 0; i < 3 * nsteps; ++i)
        if (int rc = stage(b, dt, (cudaStream_t)stream)) return rc;
    return WS_OK;
}

int ws_blocks_compute_dt(ws_blocks* b, double cfl, double* dt, ws_stream_t stream) {
    if (!b || !dt) return fail(WS_ERR_INVALID, "NULL argument");
    double m = 0.0;
    bool first = true;
    int rc = WS_OK;
    for (auto& l : b->blk) {
        double d = 0.0;
        if ((rc = ws_solver_compute_dt(l.s, cfl, &d, stream))) break;
        m = first ? d : std::min(m, d);
        first = false;
    }
    if (b->comm) {
        // every rank takes the all-reduce, also after a local failure (which
        // contributes -1), so that no rank waits in it for good; then all of
        // them return an error
        const std::string local_error = rc ? last_error_message() : std::string();
        if (rc) m = -1.0;
        cudaStream_t st = (cudaStream_t)stream;
        WS_CUDA(cudaMemcpyAsync(b->d_min, &m, sizeof m, cudaMemcpyHostToDevice, st));
        WS_NCCL(nccl().all_reduce(b->d_min, b->d_min, 1, ncclFloat64, ncclMin, b->comm, st));
        WS_CUDA(cudaMemcpyAsync(&m, b->d_min, sizeof m, cudaMemcpyDeviceToHost, st));
        WS_CUDA(cudaStreamSynchronize(st));
        if (rc) return fail(rc, local_error);
        if (!(m > 0)) return fail(WS_ERR_NONFINITE, "another rank's time step failed");
    } else if (rc) {
        return rc;
    }
    *dt = m;
    return WS_OK;
}

int ws_blocks_status(ws_blocks* b, int* status, ws_stream_t stream) {
    if (!b || !status) return fail(WS_ERR_INVALID, "NULL argument");
    int worst = 0;
    for (auto& l : b->blk) {
        int s = 0;
        if (int rc = ws_solver_status(l.s, &s, stream)) return rc;
        worst = std::max(worst, s);
    }
    *status = worst;
    return WS_OK;
}

}  // extern "C"
