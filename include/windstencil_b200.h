/*
 * windstencil_b200.h -- C ABI of the B200 (sm_100a) BF3W inviscid RHS library.
 *
 * libwindstencil_b200.so replaces WindStencil's inviscid hot path: the fused
 * BF3W kernel (src/kernels/OCFD_split.cpp:36-3918), its driver and boundary
 * ring kernel (src/solver/OCFD_NS_Jacobian3d.cpp:24-414, :828-2530), the sound
 * speed / prim<->cons / RK-stage kernels around it, and the host-staged halo
 * exchange (src/mpi/OCFD_mpi_dev.cpp:123-290) on one GPU.
 *
 * Conventions (all entry points):
 *   - plain C types, device pointers in ws_field / ws_soa, sizes in elements;
 *   - the return value is WS_OK (0) or a WS_ERR_* code; nothing aborts and the
 *     message of the last failure on the calling thread is in ws_last_error();
 *   - work is enqueued on the given stream (NULL = legacy default stream) and
 *     no entry point synchronises the host, except where its comment says so;
 *   - LAP fields are [nz+8][ny+8][pitch >= nx+8] doubles, x fastest, 4 ghost
 *     layers on every side; SoA arrays are [5][length_Z][length_Y][pitch]
 *     doubles (reference index macros, include/windstencil/cuda_utility.h:16-27).
 */
#ifndef WINDSTENCIL_B200_H
#define WINDSTENCIL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(WS_BUILDING_LIB) && defined(__GNUC__)
#define WS_API __attribute__((visibility("default")))
#else
#define WS_API
#endif

#define WS_LAP 4
#define WS_NVARS 5
#define WS_ABI_VERSION 1

/* cudaStream_t without including the CUDA headers */
typedef struct CUstream_st* ws_stream_t;

/* == cudaField (include/windstencil/cuda_commen.h:48-54, HIP layout). */
typedef struct ws_field {
    double* ptr;        /* device pointer to element (0,0,0) of the LAP array */
    uint32_t pitch;     /* row pitch in elements                              */
    uint32_t dummy0;
} ws_field;

/* == cudaSoA (include/windstencil/cuda_commen.h:64-72). */
typedef struct ws_soa {
    double* ptr;        /* device pointer to element (0,0,0) of variable 0    */
    uint32_t pitch;     /* row pitch in elements                              */
    uint32_t length_Y;  /* rows per plane                                      */
    uint32_t length_Z;  /* planes per variable                                 */
    uint32_t dummy0;
} ws_soa;

typedef struct ws_dim3 { uint32_t x, y, z; } ws_dim3;

/* == cudaJobPackage (include/windstencil/cuda_commen.h:98-106): the cells
 * [start, end) in LAP coordinates (interior = [4, n+4)). */
typedef struct ws_job { ws_dim3 start, end; } ws_job;

enum ws_face_kind {
    WS_FACE_PERIODIC = 0,   /* ghosts wrap (the reference's periodic self-exchange) */
    WS_FACE_EXTRAP = 1,     /* zero-gradient ghosts (copy of the boundary cell)     */
    /* x and y faces only: zero-gradient ghosts, and the faces next to it take
     * the boundary closures of the reference's fused path (its ring kernel
     * split_Jac3d_Stager_Warming_ker_boundary, OCFD_NS_Jacobian3d.cpp:
     * 1063-1085 for x and :1515-1584 for y): WENO5 one-sided forms, linear
     * extrapolation / averages (x) or minmod2 forms (y) at the high end, and
     * the reference's dropped M term of the last y cell.  >= 8 cells.       */
    WS_FACE_CLOSURE = 2,
    /* the face is shared with a neighbouring subdomain (a block of a grid
     * split along x, y and/or z); its 4 ghost planes over the interior of
     * the other two axes are written by the caller (ws_halo_unpack), as the
     * reference's exchange_boundary_{x,y,z}_packed_dev do
     * (OCFD_mpi_dev.cpp:123-290); the ghost fill leaves them.  Faces next to
     * it are reconstructed with WENO7 through those ghosts. */
    WS_FACE_EXTERNAL = 3
};

enum ws_precision {
    WS_FP64 = 0,            /* the drop-in: every operation in FP64                  */
    WS_MIXED = 1            /* FP32 split, smoothness indicators, weights and
                               candidates; FP64 state, face difference and RK3      */
};

enum ws_status {
    WS_OK = 0,
    WS_ERR_INVALID = 1,     /* bad argument (sizes, job, pitch, alignment)  */
    WS_ERR_CUDA = 2,        /* a CUDA runtime call failed                    */
    WS_ERR_ALLOC = 3,       /* device or host allocation failed              */
    WS_ERR_UNSUPPORTED = 4, /* configuration this build does not implement   */
    WS_ERR_NONFINITE = 5,   /* device status: non-finite value, rho<=0, p<=0 */
    WS_ERR_TIMEOUT = 6,     /* a bounded device wait gave up                 */
    WS_ERR_BUDGET = 7,      /* admission would exceed the HBM budget         */
    WS_ERR_BUSY = 8,        /* object in use / queue full                    */
    WS_ERR_NOT_FOUND = 9,   /* unknown request id                            */
    WS_ERR_IO = 10,         /* file missing, short or not in the expected format */
    WS_ERR_COMM = 11        /* a communication library call (NCCL) failed       */
};

/* Grid and physics constants.  Replaces the reference's __constant__ set
 * (src/runtime/parameters_d.cpp:12-35) and the derived constants of
 * OCFD_init.cpp:379-407 (Cv, split_C1, split_C3 are derived from gamma, ama). */
typedef struct ws_grid {
    uint32_t nx, ny, nz;      /* interior extents                                */
    uint32_t lap;             /* ghost width; must be WS_LAP                      */
    double hx, hy, hz;        /* grid spacing (reference default 1/(N-1))         */
    double gamma;             /* Gamma                                            */
    double ama;               /* Ama (reference Mach number)                      */
    double epsl_sw;           /* EPSL_SW, Steger-Warming entropy fix              */
    int32_t face_kind[6];     /* x-, x+, y-, y+, z-, z+ : enum ws_face_kind       */
    int32_t precision;        /* enum ws_precision                                */
    int32_t metrics_uniform;  /* 1: Cartesian metrics xi=(1,0,0), eta=(0,1,0),
                                 zeta=(0,0,1) and J=1; metric fields not read    */
} ws_grid;

/* Metric fields (LAP), the reference's pAkx_d..pAsz_d and pAjac_d
 * (include/windstencil/parameters_d.h:37-63). */
typedef struct ws_metrics {
    ws_field akx, aky, akz;   /* xi   gradient */
    ws_field aix, aiy, aiz;   /* eta  gradient */
    ws_field asx, asy, asz;   /* zeta gradient */
    ws_field ajac;            /* Jacobian J    */
} ws_metrics;

/* Kernel selection.  All zeros (the default) and tile_x < 0 select the line
 * passes: three barrier-free passes (x, y, z) in which each lane marches one
 * grid line (with tile_x < 0, threads = 32 x warps per CTA, or 0 for the
 * tuned count).  Any other tile_x, tile_y, threads select the fused tile
 * sweep: a CTA of `threads` threads owns tile_x x tile_y columns and sweeps
 * them along z; scan_z caps the planes of one sweep (0: no cap, each
 * persistent CTA sweeps its whole share of planes).  Both give the same
 * results, CLOSURE faces included. */
typedef struct ws_tile {
    int32_t tile_x, tile_y, scan_z, threads;
} ws_tile;

/* ------------------------------------------------------------------------ */
/* Library                                                                   */
/* ------------------------------------------------------------------------ */
WS_API int  ws_abi_version(void);
/* Copies the message of the last failure on this thread (NUL-terminated). */
WS_API int  ws_last_error(char* buf, size_t n);
/* Elements of the LAP-field row pitch this library allocates for extent nx+8
 * (a multiple of 32). */
WS_API uint32_t ws_lap_pitch(uint32_t nx);
/* Device-side errors of the launches that carry no per-grid status word
 * (the drop-in RHS entry points): bit value 2 = a staging wait of the fused
 * RHS gave up (bounded wait on its TMA copies) and the launch stopped early,
 * leaving du incomplete.  Reads and clears the word of the current device;
 * synchronises `stream`.  The solver, batches and server report the same bit
 * in their own status words (WS_ERR_TIMEOUT). */
WS_API int ws_device_error(int* flags, ws_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Drop-in kernels (explicit arguments)                                      */
/* ------------------------------------------------------------------------ */

/* cc = sqrt(T)/Ama over the job extended by 4 ghost layers.
 * Replaces du_invis_Jacobian3d_init (OCFD_NS_Jacobian3d.cpp:24-33) and
 * sound_speed_kernel (commen_kernel.cpp:145-154). */
WS_API int ws_du_invis_jacobian3d_init(const ws_grid* g, ws_job job, ws_field T, ws_field cc,
                                ws_stream_t stream);

/* du (SoA, written with `=`) = BF3W inviscid RHS on the job's cells from the
 * LAP primitives d,u,v,w and sound speed cc (ghosts filled).  metrics may be
 * NULL when g->metrics_uniform is 1.  du(x,y,z) is addressed relative to
 * job.start.  Replaces du_invis_Jacobian3d_x (OCFD_NS_Jacobian3d.cpp:133-414:
 * the fused kernel OCFD_split.cpp:36-3918 plus the boundary ring kernel
 * :828-2530); needs no workspace and allocates nothing. */
WS_API int ws_du_invis_jacobian3d(const ws_grid* g, ws_job job, ws_field d, ws_field u,
                           ws_field v, ws_field w, ws_field cc, const ws_metrics* metrics,
                           ws_soa du, ws_stream_t stream);

/* Same, with an explicit tile shape (autotuner and tests). */
WS_API int ws_du_invis_jacobian3d_tiled(const ws_grid* g, ws_job job, ws_field d, ws_field u,
                                 ws_field v, ws_field w, ws_field cc,
                                 const ws_metrics* metrics, ws_soa du, ws_tile tile,
                                 ws_stream_t stream);

/* Viscous constants of the Navier-Stokes RHS: Reynolds number, Prandtl
 * number, Sutherland reference temperature Ref_T (Sutherland constant
 * 110.4 K, viscosity 1/Re at T = 1) and the central-difference order of the
 * derivatives, 6 or 8 (the reference's Scheme_vis_ID 203 / 204).
 * d0_bound: the reference's DIF_BOUND flags (D0_bound, parameters.c:175,
 * :225), faces x-, x+, y-, y+, z-, z+.  Nonzero: in the four cells next to
 * that face the viscous derivatives (gradients and flux divergence) take the
 * reference's reduced forms (OCFD_bound, OCFD_bound_Scheme.cpp:432-452, and
 * OCFD_D0bound_scheme_kernel, :82-240): a one-sided first difference at the
 * face, then 2nd-, 4th- and 6th-order central differences; zero: the central
 * difference through the ghosts.  Ignored on EXTERNAL faces (a neighbouring
 * block's, not a physical, boundary). */
typedef struct ws_viscous {
    double re, pr, ref_t;
    int32_t scheme;
    int32_t dummy0;
    int32_t d0_bound[6];
} ws_viscous;

/* Device workspace that ws_du_vis_jacobian3d needs for grid g (bytes): the
 * viscous flux fields as LAP arrays, 12 of them, or 9 on a Cartesian grid
 * (metrics_uniform), where the symmetric stress entries share a field. */
WS_API size_t ws_du_vis_workspace_bytes(const ws_grid* g);

/* du[1..4] (SoA, whole interior) += viscous terms of momentum and energy from
 * the LAP fields u, v, w, T (ghosts filled); du[0] is left as it is.
 * Replaces du_vis_Jacobian3d (OCFD_Stream.cpp:229-345: gradient kernels
 * OCFD_NS_Jacobian3d.cpp:455-475, vis_flux_ker :477-624 per direction,
 * halo exchange of the fluxes, derivative and YF_Pe_XF accumulation), with
 * the fluxes' ghosts filled by g->face_kind.  workspace: caller-owned device
 * memory of ws_du_vis_workspace_bytes(g) (the reference keeps the same
 * fields as globals); the call allocates nothing.  WS_ERR_UNSUPPORTED for a
 * grid with WS_FACE_EXTERNAL faces: the fluxes' halos need an exchange of
 * their own between the two passes (ws_solver_stage_begin / _end). */
WS_API int ws_du_vis_jacobian3d(const ws_grid* g, const ws_viscous* vis, ws_field u, ws_field v,
                                ws_field w, ws_field T, const ws_metrics* metrics, ws_soa du,
                                void* workspace, size_t workspace_bytes, ws_stream_t stream);

/* ------------------------------------------------------------------------ */
/* The reference's on-disk formats (one domain, little-endian, Fortran-style  */
/* records: int32 length | data | int32 length; each 3D field is nz plane     */
/* records of nx*ny float64, x fastest).                                     */
/* ------------------------------------------------------------------------ */
/* Restart file OCFD%08d.dat (OCFD_save / read_file, src/io/OCFD_IO.c:24-226):
 * header record (int32 Istep, float64 tt), then d, u, v, w, T.
 * prims: host [5][nz][ny][nx] in that order. */
WS_API int ws_restart_write(const char* path, int nx, int ny, int nz, int32_t istep, double tt,
                            const double* prims);
WS_API int ws_restart_read(const char* path, int nx, int ny, int nz, int32_t* istep, double* tt,
                           double* prims);
/* Metrics file OCFD3d-Jacobi.dat (OCFD_Comput_Jacobian3d.cpp:120-211): no
 * header; x, y, z, akx, aky, akz, aix, aiy, aiz, asx, asy, asz, ajac.
 * fields: host [13][nz][ny][nx] in that order (interiors; ghosts are filled
 * afterwards, e.g. with ws_ghost_fill). */
WS_API int ws_metrics_write(const char* path, int nx, int ny, int nz, const double* fields);
WS_API int ws_metrics_read(const char* path, int nx, int ny, int nz, double* fields);

/* In-place ghost fill (4 layers) of nfields LAP fields by g->face_kind.
 * Replaces exchange_boundary_xyz_packed_dev (OCFD_mpi_dev.cpp:123-290) on one
 * GPU: no host staging, no MPI. */
WS_API int ws_ghost_fill(const ws_grid* g, const ws_field* fields, int nfields, ws_stream_t stream);

/* Halo planes of a grid split into blocks (the reference's MPI decomposition
 * NPX0 x NPY0 x NPZ0, OCFD_mpi.c:102-145, with one subdomain per GPU).
 * axis 0, 1, 2 = x, y, z; side 0 is the low face, side 1 the high face.  A
 * halo buffer holds nfields x the 4 planes along the axis over the interior
 * of the other two, x fastest: [field][z][y][x] with 4 x planes (axis 0),
 * [field][z][4][x] (axis 1), [field][4][y][x] (axis 2) -- the packed layout
 * of cudaFieldBoundaryPack_kernel (OCFD_mpi_dev.cpp:137-152).  Buffers are
 * device memory, 8-byte aligned; 1 <= nfields <= 8. */
WS_API size_t ws_halo_bytes(const ws_grid* g, int axis, int nfields);
/* Interior planes next to face (axis, side) (side 0: 4..7; side 1: n..n+3
 * in LAP coordinates along the axis) -> buf: the sends of
 * exchange_boundary_{x,y,z}_packed_dev; side 0 goes to the low neighbour. */
WS_API int ws_halo_pack(const ws_grid* g, const ws_field* fields, int nfields, int axis,
                        int side, void* buf, ws_stream_t stream);
/* buf -> the ghost planes beyond face (axis, side) (side 0: 0..3; side 1:
 * n+4..n+7): the receives.  The low ghosts take the low neighbour's side-1
 * planes, and the reverse. */
WS_API int ws_halo_unpack(const ws_grid* g, const ws_field* fields, int nfields, int axis,
                          int side, const void* buf, ws_stream_t stream);
/* The x-axis forms of the three above (axis 0). */
WS_API size_t ws_halo_x_bytes(const ws_grid* g, int nfields);
WS_API int ws_halo_pack_x(const ws_grid* g, const ws_field* fields, int nfields, int side,
                          void* buf, ws_stream_t stream);
WS_API int ws_halo_unpack_x(const ws_grid* g, const ws_field* fields, int nfields, int side,
                            const void* buf, ws_stream_t stream);

/* Conserved (SoA f) -> LAP interiors of d,u,v,w,T and P (P.ptr may be NULL).
 * Replaces get_duvwT / cons_to_pri_kernel (commen_kernel.cpp:78-119). */
WS_API int ws_cons_to_prim(const ws_grid* g, ws_soa f, ws_field d, ws_field u, ws_field v,
                    ws_field w, ws_field T, ws_field P, ws_stream_t stream);

/* LAP primitives -> conserved SoA f.
 * Replaces pri_to_cons_kernel_warp (commen_kernel.cpp:33-73). */
WS_API int ws_prim_to_cons(const ws_grid* g, ws_field d, ws_field u, ws_field v, ws_field w,
                    ws_field T, ws_soa f, ws_stream_t stream);

/* SSP-RK3 stage krk in {1,2,3}: f <- stage(fn, f, dt*du).
 * Replaces OCFD_time_advance (OCFD_time.cpp:15-91). */
WS_API int ws_time_advance(const ws_grid* g, int krk, double dt, ws_soa f, ws_soa fn, ws_soa du,
                    ws_stream_t stream);

/* CFL time step of n caller-owned grids, allocating nothing.
 * No counterpart in the reference (it takes DT as an input).
 * For callers that must not allocate device memory after start-up: a host
 * code that owns every device buffer in its own arena (as the reference's
 * time loop does) or runs under a hard device-memory cap, and any loop that
 * cannot afford the device-wide wait that cudaMalloc/cudaFree imply.  The
 * other dt entry points use allocated scratch; this one reduces into a fixed
 * array of WS_DT_STATIC_MAX_GRIDS entries compiled into the library, present
 * on every GPU that loads it until the process exits.
 * prims: 4 LAP fields per grid, in the order u, v, w, cc.
 * dt_out[i] = cfl / max over grid i's interior of
 *             |u|/hx + |v|/hy + |w|/hz + cc*sqrt(hx^-2 + hy^-2 + hz^-2).
 * n above WS_DT_STATIC_MAX_GRIDS is rejected with WS_ERR_INVALID; a grid with
 * a NaN or infinite wave speed in any cell gives WS_ERR_NONFINITE.  The first
 * call with a given device current looks up the array's device address and
 * keeps it until exit; make that first call before any stream capture, and
 * do not call cudaDeviceReset after it.  All calls share the array (each
 * clears the entries it uses first), so calls whose work overlaps on the GPU
 * race: serialise them.  Every call copies the maxima to the host and
 * synchronises `stream` before it returns. */
#define WS_DT_STATIC_MAX_GRIDS 4096
WS_API int ws_compute_dt_static(const ws_grid* grids, const ws_field* prims, int n, double cfl,
                                double* dt_out, ws_stream_t stream);

/* ------------------------------------------------------------------------ */
/* One grid, device-resident, SSP-RK3 step as one CUDA graph                 */
/* Replaces the time loop NS_solver_real (OCFD_NS_Solver.cpp:64-90) with all  */
/* three RK stages.                                                           */
/* ------------------------------------------------------------------------ */
typedef struct ws_solver ws_solver;

/* Allocates the state (f, fn, du SoA; d,u,v,w,T,cc LAP) on the current device. */
WS_API int  ws_solver_create(const ws_grid* g, ws_solver** out);
WS_API void ws_solver_destroy(ws_solver* s);
/* Uploads a dense conserved state [5][nz][ny][nx] from host memory. */
WS_API int  ws_solver_set_state(ws_solver* s, const double* f_host, ws_stream_t stream);
/* Downloads the conserved state; synchronises `stream`. */
WS_API int  ws_solver_get_state(ws_solver* s, double* f_host, ws_stream_t stream);
/* The same download, only enqueued on `stream` (the host does not wait): f_host
 * must stay valid, and is complete, once the stream has passed the copy (the
 * caller synchronises).  With pinned f_host the copy runs on a copy engine
 * beside kernels of other streams, so a caller with several solvers can
 * overlap one's transfers with another's steps. */
WS_API int  ws_solver_get_state_async(ws_solver* s, double* f_host, ws_stream_t stream);
/* Downloads du of the last ws_solver_rhs() (a step uses du as its
 * accumulator, so read it before stepping); synchronises `stream`. */
WS_API int  ws_solver_get_rhs(ws_solver* s, double* du_host, ws_stream_t stream);
/* Device descriptors of the state (f, du SoA; d,u,v,w,T,cc LAP). */
WS_API int  ws_solver_fields(ws_solver* s, ws_soa* f, ws_soa* du, ws_field prims[6]);
/* CFL time step of the current state; synchronises `stream`. */
WS_API int  ws_solver_compute_dt(ws_solver* s, double cfl, double* dt, ws_stream_t stream);
/* du of the current state (prims, ghost fill, cc, RHS). */
WS_API int  ws_solver_rhs(ws_solver* s, ws_stream_t stream);
/* nsteps SSP-RK3 steps with time step dt, replayed from one CUDA graph.
 * WS_ERR_UNSUPPORTED for a grid with WS_FACE_EXTERNAL faces (those step by
 * stages, with a halo exchange before each). */
WS_API int  ws_solver_step(ws_solver* s, double dt, int nsteps, ws_stream_t stream);
/* One SSP-RK3 stage, krk = 1, 2, 3 in that order (stage 3 completes the step
 * and makes its result the current state): ghost fill of the stage's input
 * primitives on every face that is not WS_FACE_EXTERNAL, then the fused RHS
 * with the stage update.  Before each stage the caller writes the EXTERNAL
 * faces' ghost planes into ws_solver_stage_fields(s, krk).  The reference's
 * loop body per stage: exchange_boundary_xyz_packed_dev, du_comput,
 * OCFD_time_advance (OCFD_NS_Solver.cpp:64-90).  WS_ERR_INVALID when krk is
 * not the next stage. */
WS_API int  ws_solver_stage(ws_solver* s, int krk, double dt, ws_stream_t stream);
/* The primitive fields d,u,v,w,T,cc that stage krk reads (stage 1: the
 * current state's). */
WS_API int  ws_solver_stage_fields(ws_solver* s, int krk, ws_field prims[6]);
/* ws_solver_stage in two halves, for a block with viscous terms: the first
 * (ghost fill, viscous flux pass with the fluxes' own ghost fill) and the
 * second (viscous divergence, fused RHS + stage update).  Between them the
 * caller exchanges, along each axis with EXTERNAL faces, the halos of that
 * direction's four viscous fluxes (ws_solver_stage_flux_fields; d/dx needs
 * the x fluxes' x ghosts, and so on), as the reference exchanges Ev1..4
 * between vis_flux_ker and its derivatives (OCFD_Stream.cpp:229-345).
 * ws_solver_stage with viscous terms on an EXTERNAL grid returns
 * WS_ERR_UNSUPPORTED. */
WS_API int  ws_solver_stage_begin(ws_solver* s, int krk, ws_stream_t stream);
WS_API int  ws_solver_stage_end(ws_solver* s, int krk, double dt, ws_stream_t stream);
/* The four viscous flux fields of direction `axis` (Ev1..4, LAP) in the
 * solver's workspace; WS_ERR_INVALID without viscous terms. */
WS_API int  ws_solver_stage_flux_fields(ws_solver* s, int axis, ws_field ev_axis[4]);
/* Device status word: 0, WS_ERR_NONFINITE, or WS_ERR_TIMEOUT (a staging
 * wait of the fused RHS gave up); synchronises `stream`. */
WS_API int  ws_solver_status(ws_solver* s, int* status, ws_stream_t stream);
WS_API int  ws_solver_set_tile(ws_solver* s, ws_tile tile);
/* Current state to / from a restart file (d, u, v, w, T from / to the
 * conserved state with the formulas of cons_to_pri_kernel / pri_to_cons_kernel,
 * commen_kernel.cpp:33-110); synchronise `stream`. */
WS_API int  ws_solver_save(ws_solver* s, const char* path, int32_t istep, double tt,
                           ws_stream_t stream);
WS_API int  ws_solver_load(ws_solver* s, const char* path, int32_t* istep, double* tt,
                           ws_stream_t stream);
/* Navier-Stokes: every RHS adds the viscous terms (NULL: Euler again).  The
 * solver keeps their workspace; the RK stage adds them before its update.
 * A grid with WS_FACE_EXTERNAL faces then steps with ws_solver_stage_begin /
 * _end. */
WS_API int  ws_solver_set_viscous(ws_solver* s, const ws_viscous* vis);

/* ------------------------------------------------------------------------ */
/* One grid split into blocks, stepped from C++                              */
/* ------------------------------------------------------------------------ */
/* Block `index` of g split into dims[0] x dims[1] x dims[2] blocks, the
 * reference's MPI decomposition: rank = px + NPX0 * (py + NPY0 * pz)
 * (OCFD_mpi.c:102-121); per axis n / P cells, the first n % P blocks one
 * wider (:124-145); neighbours wrapped on a periodic axis, none (-1) at the
 * ends of another or on an axis in one part (:176-197).  Faces shared with a
 * neighbour are WS_FACE_EXTERNAL.  An axis must be periodic at both faces or
 * at neither; g has no EXTERNAL faces; a block needs 4 cells per axis (8
 * with a CLOSURE face on it). */
typedef struct ws_block_info {
    int32_t index, coords[3], origin[3], n[3];
    int32_t nbr[3][2];      /* neighbour block per axis, low / high side; -1: none */
    int32_t faces[6];       /* the block grid's face kinds */
} ws_block_info;
WS_API int ws_blocks_decompose(const ws_grid* g, const int32_t dims[3], int32_t index,
                               ws_block_info* out);

/* A set of blocks stepped with SSP-RK3 from C++ (the time loop of
 * OCFD_NS_Solver.cpp:64-90): before every stage the halos of the stage's
 * primitives (d, u, v, w, T, cc) are packed on the device, exchanged and
 * unpacked into the neighbours' ghost planes (exchange_boundary_{x,y,z}_
 * packed_dev, OCFD_mpi_dev.cpp:123-290); with viscous terms each direction's
 * four fluxes are exchanged the same way between the flux pass and the
 * divergence.  Everything is enqueued on the caller's stream.
 *   nccl_id NULL: every block of the grid lives in this process, on the
 *     current device; a block's ghosts come straight from its neighbour's
 *     packed planes (a single-GPU stand-in for a multi-GPU run).
 *   nccl_id (ws_nccl_unique_id on one rank, passed to all): this process
 *     owns block `rank` of a job of dims[0] x dims[1] x dims[2] ranks, one
 *     per GPU (the current device); the packed planes go to the neighbours
 *     with NCCL point-to-point sends, one group per exchange.  NCCL is loaded
 *     at run time (libnccl.so.2, the one already in the process if any).
 * Block states are read and written through each block's solver
 * (ws_blocks_solver; the block's part of the global state, ws_block_info). */
typedef struct ws_blocks ws_blocks;
WS_API int  ws_nccl_unique_id(void* id /* 128 bytes */);
/* The point-to-point messages block `index` posts in one exchange over
 * NCCL, in posting order (kind 0 send of the planes next to face (axis,
 * side), 1 receive into the ghosts beyond it; peer = block index): per axis
 * the low planes' send, the high planes' send, the high ghosts' receive,
 * the low ghosts' receive.  NCCL matches two ranks' messages in order, so
 * every send lands in the ghosts it was packed for, a two-block periodic
 * ring included.  *count = the number of messages (at most 12; ops holds the
 * first cap). */
typedef struct ws_p2p_op { int32_t kind, peer, axis, side; } ws_p2p_op;
WS_API int  ws_blocks_exchange_plan(const ws_grid* g, const int32_t dims[3], int32_t index,
                                    ws_p2p_op* ops, int32_t cap, int32_t* count);
WS_API int  ws_blocks_create(const ws_grid* g, const int32_t dims[3], const void* nccl_id,
                             int32_t rank, ws_blocks** out);
WS_API void ws_blocks_destroy(ws_blocks* b);
/* blocks in this process, and their descriptions / solvers (owned by b) */
WS_API int  ws_blocks_count(ws_blocks* b, int32_t* count);
WS_API int  ws_blocks_info(ws_blocks* b, int32_t i, ws_block_info* out);
WS_API int  ws_blocks_solver(ws_blocks* b, int32_t i, ws_solver** s);
/* Navier-Stokes on every block (NULL: Euler); every rank makes the same call */
WS_API int  ws_blocks_set_viscous(ws_blocks* b, const ws_viscous* vis);
/* nsteps SSP-RK3 steps of dt; every rank makes the same calls */
WS_API int  ws_blocks_step(ws_blocks* b, double dt, int nsteps, ws_stream_t stream);
/* global CFL time step: the minimum over all blocks (NCCL all-reduce over
 * the ranks); synchronises `stream` */
WS_API int  ws_blocks_compute_dt(ws_blocks* b, double cfl, double* dt, ws_stream_t stream);
/* the largest status word of this process's blocks; synchronises `stream` */
WS_API int  ws_blocks_status(ws_blocks* b, int* status, ws_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Many independent grids, device-resident, stepped together: per RK stage   */
/* one batched ghost fill, one persistent fused-RHS launch over all grids,   */
/* one batched stage update; the step is replayed from a CUDA graph.  No     */
/* reference counterpart (the reference solves one grid per MPI rank).       */
/* All grids: Cartesian (metrics_uniform = 1), one precision, no EXTERNAL   */
/* faces.                                                                    */
/* ------------------------------------------------------------------------ */
typedef struct ws_batch ws_batch;

WS_API int  ws_batch_create(const ws_grid* grids, int n, ws_batch** out);
WS_API void ws_batch_destroy(ws_batch* b);
WS_API int  ws_batch_size(ws_batch* b);
/* dense conserved state [5][nz][ny][nx] of grid i */
WS_API int  ws_batch_set_state(ws_batch* b, int i, const double* f_host, ws_stream_t stream);
WS_API int  ws_batch_get_state(ws_batch* b, int i, double* f_host, ws_stream_t stream);
/* du of grid i after the last ws_batch_rhs() (a step overwrites it, as for
 * the solver); synchronises `stream`. */
WS_API int  ws_batch_get_rhs(ws_batch* b, int i, double* du_host, ws_stream_t stream);
/* CFL time step of every grid (dt_out[n]); synchronises `stream` */
WS_API int  ws_batch_compute_dt(ws_batch* b, double cfl, double* dt_out, ws_stream_t stream);
WS_API int  ws_batch_set_dt(ws_batch* b, const double* dt);
WS_API int  ws_batch_set_tile(ws_batch* b, ws_tile tile);
WS_API int  ws_batch_get_tile(ws_batch* b, ws_tile* tile);
/* du of every grid's current state */
WS_API int  ws_batch_rhs(ws_batch* b, ws_stream_t stream);
/* nsteps SSP-RK3 steps of every grid */
WS_API int  ws_batch_step(ws_batch* b, int nsteps, ws_stream_t stream);
/* per-grid status (0, WS_ERR_NONFINITE or WS_ERR_TIMEOUT); synchronises `stream` */
WS_API int  ws_batch_status(ws_batch* b, int* status, ws_stream_t stream);
/* times the compiled tile shapes on this batch's RHS and keeps the fastest */
WS_API int  ws_batch_autotune(ws_batch* b, ws_tile* chosen, ws_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Continuous-batching solve server.  No reference counterpart.  A host      */
/* thread admits queued requests while the HBM state budget and the slot     */
/* limit allow, keeps their state on the device, advances every active grid  */
/* one SSP-RK3 step per tick (one batched launch per kernel per stage and    */
/* precision) and retires grids that reached their step count.               */
/* ------------------------------------------------------------------------ */
typedef struct ws_server ws_server;

typedef struct ws_server_config {
    size_t hbm_budget_bytes;  /* device memory for request states (0: 80 GiB) */
    int32_t max_active;       /* concurrent grids (0: 4096)                    */
    ws_tile tile;             /* kernel tile shape (zeroes: default)           */
    double max_active_cells;  /* cells stepped per tick; admission waits above
                                 it once the device is full (0: 3.2e7)         */
} ws_server_config;

typedef struct ws_request {
    ws_grid grid;             /* Cartesian, FP64 or mixed                      */
    int32_t nsteps;           /* SSP-RK3 steps                                 */
    double cfl;               /* dt = cfl / max wave speed of the initial state */
    double dt;                /* > 0: use this dt instead of cfl               */
    const double* f0_host;    /* dense conserved initial state [5][nz][ny][nx];
                                 read at admission, keep it valid until then;
                                 NULL: seeded synthetic state (below)          */
    uint64_t synth_seed;      /* periodic Sod-type state: rho 1 | 0.125,       */
    double synth_mach;        /* p 1/gamma | 0.1/gamma, u = mach, 1% noise     */
    double synth_x_jump;      /* jump position as a fraction of nx             */
    double* result_host;      /* final conserved state is copied here (or NULL) */
} ws_request;

typedef struct ws_server_stats {
    long submitted, queued, active, completed, failed, ticks, max_active;
    size_t hbm_in_use;
    double p50_latency_s, p99_latency_s, mean_latency_s;  /* submit -> result */
    double served_cell_rhs;    /* cell-RHS evaluations of completed requests  */
    double executed_cell_rhs;  /* cell-RHS evaluations run, finished or not   */
    double busy_s, elapsed_s;
    /* host clock spent by the loop in each phase: admission (allocation,
     * initial state, time step), batch table rebuild, the steps (launch to
     * completion), retirement (result copies, status) */
    double admit_s, rebuild_s, steps_s, retire_s;
} ws_server_stats;

enum ws_request_state { WS_RQ_QUEUED = 0, WS_RQ_RUNNING = 1, WS_RQ_DONE = 2, WS_RQ_FAILED = 3 };

WS_API int  ws_server_create(const ws_server_config* cfg, ws_server** out);
/* stops the loop, frees every request's device state */
WS_API void ws_server_destroy(ws_server* s);
WS_API int  ws_server_submit(ws_server* s, const ws_request* r, uint64_t* id);
/* state = enum ws_request_state; latency (submit -> done) or -1 */
WS_API int  ws_server_poll(ws_server* s, uint64_t id, int* state, double* latency_s);
/* blocks until the request is done (WS_ERR_TIMEOUT after timeout_s > 0) */
WS_API int  ws_server_wait(ws_server* s, uint64_t id, double timeout_s);
WS_API int  ws_server_get_stats(ws_server* s, ws_server_stats* out);
/* forgets a finished request */
WS_API int  ws_server_release(ws_server* s, uint64_t id);

#ifdef __cplusplus
}
#endif
#endif /* WINDSTENCIL_B200_H */
