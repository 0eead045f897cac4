/*
 * oracle.h -- CPU restatement of WindStencil's inviscid (BF3W) right-hand side.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * path in windstencil_b200/ and the timed CPU baseline of bench.py.  Nothing in
 * the product links, loads or calls it; only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / --impl reference legs do.
 *
 * Parity status: the scalar kernels (Steger-Warming split, WENO7-SYMBO P/M,
 * prim<->cons, sound speed, SSP-RK3 stage formulas) are pinned bit-for-bit
 * against the reference's own functions compiled for the host by
 * oracle/build_ref.py (tests/test_oracle_pin.py).  The reference ships no golden
 * vectors or known-answer tests; the whole-field assembly is pinned by
 * property tests (free-stream preservation, telescoping conservation, axis
 * permutation, P/M mirror) and by committed golden checksums
 * (tests/golden/).
 *
 * Layout (dense, no pitch padding):
 *   LAP field  : [nz+8][ny+8][nx+8], x fastest, ghost width 4 on every side
 *                (reference: get_Field_LAP, include/windstencil/cuda_utility.h:17)
 *   SoA        : [5][nz][ny][nx], x fastest, interior only
 *                (reference: get_SoA, include/windstencil/cuda_utility.h:26)
 */
#ifndef WS_ORACLE_H
#define WS_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_LAP 4

/* CLOSURE (x and y faces only): zero-gradient ghosts, and the faces next to
 * it take the boundary closures of the fused path's ring kernel.
 * EXTERNAL: ghost planes written by the caller (a halo from a neighbouring
 * subdomain); the ghost fill keeps them. */
enum { OR_FACE_PERIODIC = 0, OR_FACE_EXTRAP = 1, OR_FACE_CLOSURE = 2, OR_FACE_EXTERNAL = 3 };

typedef struct or_grid {
    int nx, ny, nz;            /* interior extents                                  */
    double hx, hy, hz;         /* grid spacing (reference: OCFD_init.cpp:29-31)    */
    double gamma;              /* ratio of specific heats                          */
    double ama;                /* reference Mach number (Ama)                      */
    double epsl_sw;            /* Steger-Warming entropy fix (EPSL_SW)             */
    int face_kind[6];          /* x-, x+, y-, y+, z-, z+ : OR_FACE_*               */
} or_grid;

/* Viscous terms (du_vis_Jacobian3d, OCFD_Stream.cpp:229-345): Reynolds and
 * Prandtl numbers, the Sutherland reference temperature Ref_T (Sutherland
 * constant 110.4 K) and the central difference order (6: Scheme_vis_ID 203,
 * 8: 204). */
typedef struct or_vis {
    double re, pr, ref_t;
    int scheme;
    int d0_bound[6];   /* DIF_BOUND per face (x-, x+, y-, y+, z-, z+): reduced forms */
} or_vis;

/* scalar kernels ------------------------------------------------------------ */
double or_weno7_p(const double* s8);
double or_weno7_m(const double* s8);
void   or_weno7_p_batch(const double* s8n, long n, double* out);
void   or_weno7_m_batch(const double* s8n, long n, double* out);
/* WENO5 closure family on n 5-point stencils (which: see oracle.cpp) */
void   or_weno5_batch(int which, const double* s5n, long n, double* out);
void   or_split(double d, double u, double v, double w, double cc,
                double a1, double a2, double a3, double gamma, double epsl_sw,
                double* fp5, double* fm5);
void   or_split_batch(const double* in8n, long n, double gamma, double epsl_sw,
                      double* fp5n, double* fm5n);

/* field kernels ------------------------------------------------------------- */
void   or_ghost_fill(const or_grid* g, double* lap_field);
void   or_sound_speed(const or_grid* g, const double* T, double* cc);
/* du (SoA, overwritten) = inviscid RHS from LAP primitives.  metrics: NULL for
 * Cartesian (xi=(1,0,0), eta=(0,1,0), zeta=(0,0,1)), else 9 LAP fields in the
 * order Akx,Aky,Akz, Aix,Aiy,Aiz, Asx,Asy,Asz.  ajac: NULL for J=1. */
void   or_du_invis(const or_grid* g, const double* d, const double* u,
                   const double* v, const double* w, const double* cc,
                   const double* const* metrics, const double* ajac, double* du);
void   or_cons_to_prim(const or_grid* g, const double* f, double* d, double* u,
                       double* v, double* w, double* T, double* P);
void   or_prim_to_cons(const or_grid* g, const double* d, const double* u,
                       const double* v, const double* w, const double* T, double* f);
void   or_time_advance(int krk, double dt, long n, double* f, const double* fn,
                       const double* du);

/* whole solver ------------------------------------------------------------- */
/* CFL time step from conserved state f (SoA). */
double or_compute_dt(const or_grid* g, const double* f, double cfl);
/* nsteps SSP-RK3 steps of the Euler system, f (SoA) updated in place.
 * Returns 0, or -1 on allocation failure. */
/* viscosity mu(T) on the interior (dense nx*ny*nz) */
void   or_amu(const or_grid* g, const or_vis* vis, const double* T, double* amu);
/* du (SoA) += viscous terms of momentum and energy (vars 1..4) from LAP
 * u, v, w, T with filled ghosts; metrics as or_du_invis */
void   or_du_vis(const or_grid* g, const or_vis* vis, const double* u, const double* v,
                 const double* w, const double* T, const double* const* metrics,
                 const double* ajac, double* du);
/* du_vis in two steps (for subdomains whose x-flux halos come from a
 * neighbour between them): the 12 viscous flux fields (direction dir,
 * component q at ev + (4*dir+q)*lap_size, interiors), then per direction the
 * ghost fill of its 4 fields and du[1..4] += J * d(Ev_dir)/d(dir). */
void   or_vis_fluxes(const or_grid* g, const or_vis* vis, const double* u, const double* v,
                     const double* w, const double* T, const double* const* metrics,
                     const double* ajac, double* ev);
void   or_vis_div_add(const or_grid* g, const or_vis* vis, int dir, double* ev4,
                      const double* ajac, double* du);
/* Navier-Stokes forms of or_rhs_conserved / or_rk3_steps (vis may be NULL) */
int    or_rhs_conserved_ns(const or_grid* g, const or_vis* vis, const double* f, double* du,
                           const double* const* metrics, const double* ajac);
int    or_rk3_steps_ns(const or_grid* g, const or_vis* vis, double* f, double dt, int nsteps,
                       const double* const* metrics, const double* ajac);
int    or_rk3_steps(const or_grid* g, double* f, double dt, int nsteps,
                    const double* const* metrics, const double* ajac);
/* du from conserved state f: cons->prim, ghost fill, sound speed, RHS. */
int    or_rhs_conserved(const or_grid* g, const double* f, double* du,
                        const double* const* metrics, const double* ajac);

/* algorithmic operation counts (one call each), see or_op_counts() in .cpp:
 * out[0] split ops, out[1] WENO-P ops, out[2] WENO-M ops,
 * out[3] face-difference ops per cell per direction and per var (P and M),
 * out[4] FLOP per cell-RHS, out[5] of which sqrt+div in split,
 * out[6] of which div in WENO (per cell). */
void   or_op_counts(double* out);
void   or_set_threads(int n);
int    or_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
