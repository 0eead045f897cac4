// field_kernels.cu -- bandwidth kernels around the RHS: sound speed, ghost
// fill, prim<->cons, SSP-RK3 stage updates; single-grid and batched forms.
//
// Reference counterparts:
//   sound speed    src/kernels/commen_kernel.cpp:145-154 (launched over the
//                  LAP-extended job by OCFD_NS_Jacobian3d.cpp:24-33)
//   ghost fill     src/mpi/OCFD_mpi_dev.cpp:123-290 (host-staged periodic
//                  self-exchange; here an in-place device copy)
//   halo planes    cudaFieldBoundaryPack/Unpack_kernel with the jobs of
//                  exchange_boundary_{x,y,z}_packed_dev, OCFD_mpi_dev.cpp:137-290
//   cons->prim     src/kernels/commen_kernel.cpp:78-119
//   prim->cons     src/kernels/commen_kernel.cpp:33-73
//   RK3 stages     src/solver/OCFD_time.cpp:15-91
#include "ws_internal.h"

namespace ws {

namespace {

__device__ __forceinline__ size_t lap_idx(int i, int j, int k, uint32_t pitch, int ny) {
    return (size_t)i + (size_t)pitch * ((size_t)j + (size_t)(ny + 8) * (size_t)k);
}
__device__ __forceinline__ size_t soa_idx(int i, int j, int k, int var, const ws_soa& s) {
    return (size_t)i + (size_t)s.pitch * ((size_t)j + (size_t)s.length_Y *
                                          ((size_t)k + (size_t)s.length_Z * (size_t)var));
}

// source index of a (possibly ghost) LAP index along one axis: an interior
// index, or the ghost index itself on an EXTERNAL face (its value comes from
// the neighbour's halo and is kept)
__device__ __forceinline__ int ghost_src(int i, int n, int lo_kind, int hi_kind) {
    if (i < 4)
        return lo_kind == WS_FACE_PERIODIC ? i + n : lo_kind == WS_FACE_EXTERNAL ? i : 4;
    if (i >= n + 4)
        return hi_kind == WS_FACE_PERIODIC ? i - n : hi_kind == WS_FACE_EXTERNAL ? i : n + 3;
    return i;
}

__host__ __device__ __forceinline__ long ghost_count(int nx, int ny, int nz) {
    const long px = nx + 8, py = ny + 8;
    return 8 * px * py + 8 * px * (long)nz + 8 * (long)ny * nz;
}

// t-th point of the 4-layer ghost shell (edges and corners included):
// z slabs (full xy planes), then y slabs at interior z, then x slabs.
__device__ __forceinline__ void ghost_point(long t, int nx, int ny, int nz, int& i, int& j,
                                            int& k) {
    const long px = nx + 8, py = ny + 8;
    const long nzs = 8 * px * py, nys = 8 * px * (long)nz;
    if (t < nzs) {
        const long pl = t / (px * py), r = t - pl * (px * py);
        k = pl < 4 ? (int)pl : (int)(nz + pl);
        j = (int)(r / px);
        i = (int)(r - (long)j * px);
    } else if (t < nzs + nys) {
        const long t2 = t - nzs;
        const long row = t2 / px;
        i = (int)(t2 - row * px);
        const int rj = (int)(row % 8);
        k = 4 + (int)(row / 8);
        j = rj < 4 ? rj : ny + rj;
    } else {
        const long t3 = t - nzs - nys;
        const long line = t3 / 8;
        const int ri = (int)(t3 - line * 8);
        i = ri < 4 ? ri : nx + ri;
        j = 4 + (int)(line % ny);
        k = 4 + (int)(line / ny);
    }
}

struct GhostArgs {
    double* ptr[8];
    uint32_t pitch[8];
    int nf;
    int nx, ny, nz;
    int kind[6];
};

// value at a ghost point = value at the wrapped / clamped coordinates.  The
// source is an interior point, or a ghost of an EXTERNAL face at interior
// coordinates of the two other axes (which this pass never writes), so one
// pass fills every face without ordering between them; those EXTERNAL ghosts
// map onto themselves and are skipped.
__device__ __forceinline__ void ghost_fill_point(const GhostArgs& a, long t) {
    int i, j, k;
    ghost_point(t, a.nx, a.ny, a.nz, i, j, k);
    const int si = ghost_src(i, a.nx, a.kind[0], a.kind[1]);
    const int sj = ghost_src(j, a.ny, a.kind[2], a.kind[3]);
    const int sk = ghost_src(k, a.nz, a.kind[4], a.kind[5]);
    if (si == i && sj == j && sk == k) return;
    for (int f = 0; f < a.nf; ++f) {
        double* p = a.ptr[f];
        p[lap_idx(i, j, k, a.pitch[f], a.ny)] = p[lap_idx(si, sj, sk, a.pitch[f], a.ny)];
    }
}

__global__ void ghost_fill_kernel(const __grid_constant__ GhostArgs a) {
    const long total = ghost_count(a.nx, a.ny, a.nz);
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
         t += (long)gridDim.x * blockDim.x)
        ghost_fill_point(a, t);
}

struct HaloArgs {
    double* ptr[8];
    uint32_t pitch[8];
    int nf, ny;
    int b[3];        // box extents in x, y, z (4 along the halo's axis)
    int o[3];        // box origin, LAP coordinates
    double* buf;     // [nf][b2][b1][b0]
    int pack;        // 1: planes -> buf, 0: buf -> planes
};

// one double per thread in buffer order (x fastest): the 4 planes along the
// halo's axis over the interior of the two other axes
__global__ void halo_kernel(const __grid_constant__ HaloArgs a) {
    const long per = (long)a.b[0] * a.b[1] * a.b[2];
    const long total = (long)a.nf * per;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
         t += (long)gridDim.x * blockDim.x) {
        const int f = (int)(t / per);
        long r = t - (long)f * per;
        const int i = (int)(r % a.b[0]);
        r /= a.b[0];
        const int j = (int)(r % a.b[1]);
        const int k = (int)(r / a.b[1]);
        double* p = a.ptr[f] + lap_idx(a.o[0] + i, a.o[1] + j, a.o[2] + k, a.pitch[f], a.ny);
        if (a.pack)
            a.buf[t] = *p;
        else
            *p = a.buf[t];
    }
}

__global__ void sound_speed_kernel(ws_field T, ws_field cc, int i0, int j0, int k0, int ni,
                                   int nj, int nk, int ny, double ama) {
    const long n = (long)ni * nj * nk;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        const int i = i0 + (int)(t % ni);
        const long r = t / ni;
        const int j = j0 + (int)(r % nj), k = k0 + (int)(r / nj);
        cc.ptr[lap_idx(i, j, k, cc.pitch, ny)] = sqrt(T.ptr[lap_idx(i, j, k, T.pitch, ny)]) / ama;
    }
}

struct PrimArgs {
    ws_soa f;
    ws_field d, u, v, w, T, P;
    int nx, ny, nz;
    double cv, gamma;
    int* status;
};

__global__ void cons_to_prim_kernel(const __grid_constant__ PrimArgs a) {
    const long n = (long)a.nx * a.ny * a.nz;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % a.nx);
        const long r = t / a.nx;
        const int j = (int)(r % a.ny), k = (int)(r / a.ny);
        const double d1 = a.f.ptr[soa_idx(i, j, k, 0, a.f)];
        const double u1 = a.f.ptr[soa_idx(i, j, k, 1, a.f)] / d1;
        const double v1 = a.f.ptr[soa_idx(i, j, k, 2, a.f)] / d1;
        const double w1 = a.f.ptr[soa_idx(i, j, k, 3, a.f)] / d1;
        double t1 = a.f.ptr[soa_idx(i, j, k, 4, a.f)];
        t1 = t1 - 0.5 * d1 * (u1 * u1 + v1 * v1 + w1 * w1);
        const int I = i + 4, J = j + 4, K = k + 4;
        a.d.ptr[lap_idx(I, J, K, a.d.pitch, a.ny)] = d1;
        a.u.ptr[lap_idx(I, J, K, a.u.pitch, a.ny)] = u1;
        a.v.ptr[lap_idx(I, J, K, a.v.pitch, a.ny)] = v1;
        a.w.ptr[lap_idx(I, J, K, a.w.pitch, a.ny)] = w1;
        const double T1 = t1 / (d1 * a.cv);
        a.T.ptr[lap_idx(I, J, K, a.T.pitch, a.ny)] = T1;
        if (a.P.ptr) a.P.ptr[lap_idx(I, J, K, a.P.pitch, a.ny)] = (t1 / d1) * (a.gamma - 1.0);
        if (a.status && !(d1 > 0.0 && T1 > 0.0 && T1 < INFINITY)) atomicOr(a.status, 1);
    }
}

__global__ void prim_to_cons_kernel(const __grid_constant__ PrimArgs a) {
    const long n = (long)a.nx * a.ny * a.nz;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % a.nx);
        const long r = t / a.nx;
        const int j = (int)(r % a.ny), k = (int)(r / a.ny);
        const int I = i + 4, J = j + 4, K = k + 4;
        const double d1 = a.d.ptr[lap_idx(I, J, K, a.d.pitch, a.ny)];
        const double u1 = a.u.ptr[lap_idx(I, J, K, a.u.pitch, a.ny)];
        const double v1 = a.v.ptr[lap_idx(I, J, K, a.v.pitch, a.ny)];
        const double w1 = a.w.ptr[lap_idx(I, J, K, a.w.pitch, a.ny)];
        const double T1 = a.T.ptr[lap_idx(I, J, K, a.T.pitch, a.ny)];
        a.f.ptr[soa_idx(i, j, k, 0, a.f)] = d1;
        a.f.ptr[soa_idx(i, j, k, 1, a.f)] = u1 * d1;
        a.f.ptr[soa_idx(i, j, k, 2, a.f)] = v1 * d1;
        a.f.ptr[soa_idx(i, j, k, 3, a.f)] = w1 * d1;
        a.f.ptr[soa_idx(i, j, k, 4, a.f)] = d1 * ((u1 * u1 + v1 * v1 + w1 * w1) * 0.5 + a.cv * T1);
    }
}

// RK3 stage coefficients, OCFD_time.cpp:15-65: f = a*fn + b*(f + dt*du),
// stage 1 f = fn + dt*du.
__device__ __forceinline__ double rk_stage(int krk, double fn, double f, double du, double dt) {
    if (krk == 1) return fn + dt * du;
    if (krk == 2) return (3.0 / 4.0) * fn + (1.0 / 4.0) * (f + dt * du);
    return (1.0 / 3.0) * fn + (2.0 / 3.0) * (f + dt * du);
}

struct StageArgs {
    ws_soa f, fn, du;
    int nx, ny, nz, krk;
    double dt;
};

__global__ void time_advance_kernel(const __grid_constant__ StageArgs a) {
    const long n = (long)a.nx * a.ny * a.nz;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n;
         t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % a.nx);
        const long r = t / a.nx;
        const int j = (int)(r % a.ny), k = (int)(r / a.ny);
#pragma unroll
        for (int var = 0; var < 5; ++var) {
            const size_t p = soa_idx(i, j, k, var, a.f);
            const double fo = a.f.ptr[p];
            const double fnv = a.fn.ptr[soa_idx(i, j, k, var, a.fn)];
            const double duv = a.du.ptr[soa_idx(i, j, k, var, a.du)];
            a.f.ptr[p] = rk_stage(a.krk, fnv, fo, duv, a.dt);
        }
    }
}

// ---- batched forms: block b works on grid tab[b].x, chunk tab[b].y of
// kBatchChunk points (a host-built table; no search on the device)
constexpr int kBatchThreads = 256;
constexpr long kBatchChunk = 256L * 8;

__global__ void ghost_fill_batch_kernel(const GhostArgs* __restrict__ grids,
                                        const int2* __restrict__ tab) {
    const int2 e = tab[blockIdx.x];
    const GhostArgs& a = grids[e.x];
    const long total = ghost_count(a.nx, a.ny, a.nz);
    const long t0 = (long)e.y * kBatchChunk;
    const long t1 = min(total, t0 + kBatchChunk);
    for (long t = t0 + threadIdx.x; t < t1; t += blockDim.x) ghost_fill_point(a, t);
}

int grid_for(long n, int threads) {
    long b = (n + threads - 1) / threads;
    const long cap = 148L * 16;
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

}  // namespace

int launch_ghost_fill(const ws_grid* g, const ws_field* f, int nf, cudaStream_t st) {
    if (nf < 1 || nf > 8) return fail(WS_ERR_INVALID, "ghost fill: 1..8 fields");
    GhostArgs a{};
    for (int i = 0; i < nf; ++i) {
        a.ptr[i] = f[i].ptr;
        a.pitch[i] = f[i].pitch;
    }
    a.nf = nf;
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    for (int i = 0; i < 6; ++i) a.kind[i] = g->face_kind[i];
    ghost_fill_kernel<<<grid_for(ghost_count(g->nx, g->ny, g->nz), 256), 256, 0, st>>>(a);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
}

int launch_halo(const ws_grid* g, const ws_field* f, int nf, int axis, int side, double* buf,
                bool pack, cudaStream_t st) {
    if (nf < 1 || nf > 8) return fail(WS_ERR_INVALID, "halo: 1..8 fields");
    if (axis < 0 || axis > 2) return fail(WS_ERR_INVALID, "halo: axis must be 0, 1 or 2");
    HaloArgs a{};
    for (int i = 0; i < nf; ++i) {
        a.ptr[i] = f[i].ptr;
        a.pitch[i] = f[i].pitch;
    }
    a.nf = nf;
    a.ny = g->ny;
    const int n[3] = {(int)g->nx, (int)g->ny, (int)g->nz};
    for (int d = 0; d < 3; ++d) {
        a.b[d] = d == axis ? 4 : n[d];
        a.o[d] = 4;
    }
    // pack: interior planes 4..7 (low) / n..n+3 (high);
    // unpack: ghost planes 0..3 (low) / n+4..n+7 (high)
    a.o[axis] = pack ? (side == 0 ? 4 : n[axis]) : (side == 0 ? 0 : n[axis] + 4);
    a.buf = buf;
    a.pack = pack ? 1 : 0;
    const long total = (long)nf * a.b[0] * a.b[1] * a.b[2];
    halo_kernel<<<grid_for(total, 256), 256, 0, st>>>(a);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
}

int launch_sound_speed(const ws_grid* g, ws_job job, ws_field T, ws_field cc, cudaStream_t st) {
    const int i0 = (int)job.start.x - 4, j0 = (int)job.start.y - 4, k0 = (int)job.start.z - 4;
    const int ni = (int)(job.end.x - job.start.x) + 8, nj = (int)(job.end.y - job.start.y) + 8,
              nk = (int)(job.end.z - job.start.z) + 8;
    const long n = (long)ni * nj * nk;
    sound_speed_kernel<<<grid_for(n, 256), 256, 0, st>>>(T, cc, i0, j0, k0, ni, nj, nk, g->ny,
                                                          g->ama);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
}

int launch_cons_to_prim(const ws_grid* g, ws_soa f, ws_field d, ws_field u, ws_field v,
                        ws_field w, ws_field T, ws_field P, int* status, cudaStream_t st) {
    PrimArgs a{};
    a.f = f; a.d = d; a.u = u; a.v = v; a.w = w; a.T = T; a.P = P;
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    a.cv = 1.0 / (g->gamma * (g->gamma - 1.0) * g->ama * g->ama);
    a.gamma = g->gamma;
    a.status = status;
    cons_to_prim_kernel<<<grid_for((long)g->nx * g->ny * g->nz, 256), 256, 0, st>>>(a);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
}

int launch_prim_to_cons(const ws_grid* g, ws_field d, ws_field u, ws_field v, ws_field w,
                        ws_field T, ws_soa f, cudaStream_t st) {
    PrimArgs a{};
    a.f = f; a.d = d; a.u = u; a.v = v; a.w = w; a.T = T;
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    a.cv = 1.0 / (g->gamma * (g->gamma - 1.0) * g->ama * g->ama);
    a.gamma = g->gamma;
    prim_to_cons_kernel<<<grid_for((long)g->nx * g->ny * g->nz, 256), 256, 0, st>>>(a);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
}

int launch_time_advance(const ws_grid* g, int krk, double dt, ws_soa f, ws_soa fn, ws_soa du,
                        cudaStream_t st) {
    StageArgs a{};
    a.f = f; a.fn = fn; a.du = du;
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz; a.krk = krk; a.dt = dt;
    time_advance_kernel<<<grid_for((long)g->nx * g->ny * g->nz, 256), 256, 0, st>>>(a);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
}

int launch_ghost_fill_prims(const ws_grid* g, const ws_field prims[6], cudaStream_t st) {
    return launch_ghost_fill(g, prims, 6, st);
}

// ---- batched launches ----------------------------------------------------
size_t ghost_args_size() { return sizeof(GhostArgs); }

void fill_ghost_args(void* out, const ws_grid* g, const ws_field prims[6]) {
    GhostArgs a{};
    for (int i = 0; i < 6; ++i) {
        a.ptr[i] = prims[i].ptr;
        a.pitch[i] = prims[i].pitch;
    }
    a.nf = 6;
    a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
    for (int i = 0; i < 6; ++i) a.kind[i] = g->face_kind[i];
    *reinterpret_cast<GhostArgs*>(out) = a;
}

long ghost_chunks(const ws_grid* g) {
    return (ghost_count(g->nx, g->ny, g->nz) + kBatchChunk - 1) / kBatchChunk;
}
int launch_ghost_fill_batch(const void* grids, const int2* tab, int nblocks, cudaStream_t st) {
    if (nblocks <= 0) return WS_OK;
    ghost_fill_batch_kernel<<<nblocks, kBatchThreads, 0, st>>>(
        reinterpret_cast<const GhostArgs*>(grids), tab);
    WS_CUDA(cudaGetLastError());
    return WS_OK;
}

uint32_t lap_pitch(uint32_t nx) {
    // rows padded to a multiple of 32 doubles (256 B)
    return ((nx + 8 + 31) / 32) * 32;
}

}  // namespace ws
