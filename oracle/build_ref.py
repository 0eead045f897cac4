#!/usr/bin/env python3
"""Build the reference's own scalar kernels for the host (test infrastructure).

The reference (WindStencil) is HIP-only and cannot be built here as a whole:
hipcc, ROCm and MPI are absent and its fused kernel assumes 64-lane
wavefronts.  Its per-point arithmetic, however, is plain C inside a handful of
functions.  This recipe reads those functions *where they lie* in the mounted
reference tree, places them behind a small shim that maps the HIP qualifiers
and the index macros to host C++, compiles them with g++ into
``oracle/_ref/libwsref.so`` and deletes the generated translation unit, so no
reference source is kept (``oracle/_ref/`` is git-ignored).

Functions taken from the reference (path within the WindStencil tree):
  src/kernels/OCFD_Schemes.cpp        OCFD_weno7_SYMBO_kernel_P_opt, _M_opt,
                                      OCFD_weno5_kernel_P, _M, sign, minmod2
  src/boundary/OCFD_bound_Scheme.cpp  OCFD_weno5_kernel_P_lift, _P_lift_plus,
                                      _P_right_plus, _M_lift, _M_lift_plus,
                                      _M_right_plus
  src/kernels/OCFD_Schemes.cpp        OCFD_kernel_CD6, OCFD_kernel_CD8
  src/solver/OCFD_NS_Jacobian3d.cpp   vis_flux_ker
  src/kernels/commen_kernel.cpp       get_Amu_kernal, YF_Pe_XF
  src/solver/OCFD_NS_Jacobian3d.cpp   split_Jac3d_Stager_Warming_ker_origin
  src/kernels/commen_kernel.cpp       cons_to_pri_kernel, pri_to_cons_kernel,
                                      sound_speed_kernel
  src/solver/OCFD_time.cpp            OCFD_time_advance_ker1/2/3
  include/windstencil/cuda_utility.h  get_Field / get_Field_LAP / get_SoA /
                                      get_SoA_LAP index macros

The host drivers below (``ref_*``) are this project's code: they set the
HIP thread coordinates for every point and call the reference function, and
``ref_du_invis`` assembles the decomposed RHS from the reference's split and
WENO functions with the loop of oracle/oracle.cpp (or_du_invis); for CLOSURE
faces it takes the face values near them from the reference's WENO5 closure
functions, by the per-face rules this project reads out of the fused path's
ring kernel (OCFD_NS_Jacobian3d.cpp:1063-1085 x, :1515-1584 y).

Only tests/ and bench.py's CPU-baseline legs use the result, as the checker.
Usage:  python oracle/build_ref.py [--ref /path/to/reference] [--native]
        (the tree defaults to $WS_REFERENCE, else the recipe's mount point)
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
# Where this recipe looks for the reference tree: --ref, else $WS_REFERENCE,
# else the read-only mount of the machine the recipe was written for.
MOUNT_REF = "/root/reference"


def reference_tree() -> str | None:
    """The reference tree to read, or None when none is mounted."""
    ref = os.environ.get("WS_REFERENCE", MOUNT_REF)
    return ref if os.path.isdir(os.path.join(ref, "src")) else None

FUNCS = [
    ("src/kernels/OCFD_Schemes.cpp", "OCFD_weno7_SYMBO_kernel_P_opt"),
    ("src/kernels/OCFD_Schemes.cpp", "OCFD_weno7_SYMBO_kernel_M_opt"),
    ("src/kernels/OCFD_Schemes.cpp", "sign"),
    ("src/kernels/OCFD_Schemes.cpp", "minmod2"),
    ("src/kernels/OCFD_Schemes.cpp", "OCFD_weno5_kernel_P"),
    ("src/kernels/OCFD_Schemes.cpp", "OCFD_weno5_kernel_M"),
    ("src/boundary/OCFD_bound_Scheme.cpp", "OCFD_weno5_kernel_P_lift"),
    ("src/boundary/OCFD_bound_Scheme.cpp", "OCFD_weno5_kernel_P_lift_plus"),
    ("src/boundary/OCFD_bound_Scheme.cpp", "OCFD_weno5_kernel_P_right_plus"),
    ("src/boundary/OCFD_bound_Scheme.cpp", "OCFD_weno5_kernel_M_lift"),
    ("src/boundary/OCFD_bound_Scheme.cpp", "OCFD_weno5_kernel_M_lift_plus"),
    ("src/boundary/OCFD_bound_Scheme.cpp", "OCFD_weno5_kernel_M_right_plus"),
    ("src/boundary/OCFD_bound_Scheme.cpp", "OCFD_D0bound_scheme_kernel"),
    ("src/kernels/OCFD_Schemes.cpp", "OCFD_kernel_CD6"),
    ("src/kernels/OCFD_Schemes.cpp", "OCFD_kernel_CD8"),
    ("src/solver/OCFD_NS_Jacobian3d.cpp", "vis_flux_ker"),
    ("src/kernels/commen_kernel.cpp", "get_Amu_kernal"),
    ("src/kernels/commen_kernel.cpp", "YF_Pe_XF"),
    ("src/solver/OCFD_NS_Jacobian3d.cpp", "split_Jac3d_Stager_Warming_ker_origin"),
    ("src/kernels/commen_kernel.cpp", "pri_to_cons_kernel"),
    ("src/kernels/commen_kernel.cpp", "cons_to_pri_kernel"),
    ("src/kernels/commen_kernel.cpp", "sound_speed_kernel"),
    ("src/solver/OCFD_time.cpp", "OCFD_time_advance_ker1"),
    ("src/solver/OCFD_time.cpp", "OCFD_time_advance_ker2"),
    ("src/solver/OCFD_time.cpp", "OCFD_time_advance_ker3"),
]
MACROS = [("include/windstencil/cuda_utility.h",
           ["get_Field", "get_Field_LAP", "get_SoA", "get_SoA_LAP"])]

SHIM_HEAD = r"""
// ---- host shim for HIP device code (generated; not committed) ----
#include <cmath>
#include <cstring>
#include <vector>
using std::sqrt; using std::fmax; using std::fmin; using std::abs;
typedef double REAL;
#define LAP 4
#define __device__
#define __global__
#define __host__
#define __forceinline__ inline
struct dim3 { unsigned x, y, z;
  dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {} };
static thread_local dim3 threadIdx(0, 0, 0), blockIdx(0, 0, 0), blockDim(1, 1, 1);
struct cudaField { REAL* ptr; unsigned pitch; unsigned dummy0; };
struct cudaSoA { REAL* ptr; unsigned pitch, length_Y, length_Z, dummy0; };
struct cudaJobPackage { dim3 start, end;
  cudaJobPackage() {}
  cudaJobPackage(const dim3& s, const dim3& e) : start(s), end(e) {} };
static thread_local REAL epsl_sw_d, Gamma_d, split_C1_d, split_C3_d, Cv_d, Ama_d, dt_d;
static thread_local unsigned ny_d, nz_d, ny_2lap_d, nz_2lap_d;
static thread_local REAL vis_flux_init_c_d, amu_C0_d, Tsb_d;
"""

DRIVERS = r"""
// ---- host drivers (this project's code) ----
namespace {
void set_consts(double gamma, double ama, double eps) {
  Gamma_d = gamma; Ama_d = ama; epsl_sw_d = eps;
  // derived constants as the reference forms them (OCFD_init.cpp:380-386)
  Cv_d = 1.0 / (gamma * (gamma - 1.0) * ama * ama);
  split_C1_d = 2.0 * (gamma - 1.0);
  split_C3_d = (3.0 - gamma) / (2.0 * (gamma - 1.0));
}
void set_dims(int nx, int ny, int nz) {
  ny_d = ny; nz_d = nz; ny_2lap_d = ny + 2 * LAP; nz_2lap_d = nz + 2 * LAP; (void)nx;
}
cudaField fld(double* p, int nx) { cudaField f; f.ptr = p; f.pitch = nx + 2 * LAP; f.dummy0 = 0; return f; }
cudaSoA soa(double* p, int nx, int ny, int nz) {
  cudaSoA s; s.ptr = p; s.pitch = nx; s.length_Y = ny; s.length_Z = nz; s.dummy0 = 0; return s; }
}

extern "C" {
double ref_weno_p(const double* s) { REAL t[8]; std::memcpy(t, s, sizeof t);
  return OCFD_weno7_SYMBO_kernel_P_opt(t); }
double ref_weno_m(const double* s) { REAL t[8]; std::memcpy(t, s, sizeof t);
  return OCFD_weno7_SYMBO_kernel_M_opt(t); }
void ref_weno_p_batch(const double* s, long n, double* out) {
  #pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) out[i] = ref_weno_p(s + 8 * i); }
void ref_weno_m_batch(const double* s, long n, double* out) {
  #pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) out[i] = ref_weno_m(s + 8 * i); }

// WENO5 closure family, same order as the oracle's or_weno5_batch
void ref_weno5_batch(int which, const double* s, long n, double* out) {
  #pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) {
    REAL t[5]; std::memcpy(t, s + 5 * i, sizeof t);
    switch (which) {
      case 0: out[i] = OCFD_weno5_kernel_P_lift(t); break;
      case 1: out[i] = OCFD_weno5_kernel_P_lift_plus(t); break;
      case 2: out[i] = OCFD_weno5_kernel_P(t); break;
      case 3: out[i] = OCFD_weno5_kernel_P_right_plus(t); break;
      case 4: out[i] = OCFD_weno5_kernel_M_lift(t); break;
      case 5: out[i] = OCFD_weno5_kernel_M_lift_plus(t); break;
      case 6: out[i] = OCFD_weno5_kernel_M(t); break;
      case 7: out[i] = OCFD_weno5_kernel_M_right_plus(t); break;
      default: out[i] = minmod2(t[0], t[1]); break;
    }
  }
}

// one-point fields: pitch 1 and unit padded extents make every index 0 (+var)
void ref_split_batch(const double* in, long n, double gamma, double eps,
                     double* fp, double* fm) {
  #pragma omp parallel
  {
    set_consts(gamma, 1.0, eps);
    ny_2lap_d = 1; nz_2lap_d = 1;
    #pragma omp for schedule(static)
    for (long i = 0; i < n; ++i) {
      double p[8]; std::memcpy(p, in + 8 * i, sizeof p);
      cudaField f[8];
      for (int k = 0; k < 8; ++k) { f[k].ptr = p + k; f[k].pitch = 1; f[k].dummy0 = 0; }
      cudaSoA sp{fp + 5 * i, 1, 1, 1, 0}, sm{fm + 5 * i, 1, 1, 1, 0};
      threadIdx = dim3(0, 0, 0); blockIdx = dim3(0, 0, 0); blockDim = dim3(1, 1, 1);
      cudaJobPackage job(dim3(0, 0, 0), dim3(1, 1, 1));
      split_Jac3d_Stager_Warming_ker_origin(f[0], f[1], f[2], f[3], f[4], sp, sm,
                                            f[5], f[6], f[7], job);
    }
  }
}

void ref_cons_to_prim(int nx, int ny, int nz, double gamma, double ama, double* f,
                      double* d, double* u, double* v, double* w, double* T, double* P) {
  #pragma omp parallel
  {
    set_consts(gamma, ama, 0.0); set_dims(nx, ny, nz);
    cudaJobPackage job(dim3(0, 0, 0), dim3(nx, ny, nz));
    #pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
      threadIdx = dim3(i, j, k);
      cons_to_pri_kernel(soa(f, nx, ny, nz), fld(d, nx), fld(u, nx), fld(v, nx), fld(w, nx),
                         fld(T, nx), fld(P, nx), job);
    }
  }
}

void ref_prim_to_cons(int nx, int ny, int nz, double gamma, double ama, double* d,
                      double* u, double* v, double* w, double* T, double* f) {
  #pragma omp parallel
  {
    set_consts(gamma, ama, 0.0); set_dims(nx, ny, nz);
    cudaJobPackage job(dim3(0, 0, 0), dim3(nx, ny, nz));
    #pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
      threadIdx = dim3(i, j, k);
      pri_to_cons_kernel(soa(f, nx, ny, nz), fld(d, nx), fld(u, nx), fld(v, nx), fld(w, nx),
                         fld(T, nx), job);
    }
  }
}

void ref_sound_speed(int nx, int ny, int nz, double ama, double* T, double* cc) {
  #pragma omp parallel
  {
    set_consts(1.4, ama, 0.0); set_dims(nx, ny, nz);
    cudaJobPackage job(dim3(0, 0, 0), dim3(nx + 2 * LAP, ny + 2 * LAP, nz + 2 * LAP));
    #pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz + 2 * LAP; ++k) for (int j = 0; j < ny + 2 * LAP; ++j)
      for (int i = 0; i < nx + 2 * LAP; ++i) {
        threadIdx = dim3(i, j, k);
        sound_speed_kernel(fld(T, nx), fld(cc, nx), job);
      }
  }
}

// f_lap may be NULL (stage 3 then writes into a scratch LAP copy)
void ref_time_advance(int krk, double dt, int nx, int ny, int nz, double* f, double* fn,
                      double* du) {
  std::vector<double> lap;
  if (krk == 3) lap.assign((size_t)5 * (nx + 2 * LAP) * (ny + 2 * LAP) * (nz + 2 * LAP), 0.0);
  #pragma omp parallel
  {
    set_dims(nx, ny, nz); dt_d = dt;
    cudaJobPackage job(dim3(0, 0, 0), dim3(nx, ny, nz));
    cudaSoA sl{lap.empty() ? nullptr : lap.data(), (unsigned)(nx + 2 * LAP),
               (unsigned)(ny + 2 * LAP), (unsigned)(nz + 2 * LAP), 0};
    #pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
      threadIdx = dim3(i, j, k);
      if (krk == 1) OCFD_time_advance_ker1(soa(f, nx, ny, nz), soa(fn, nx, ny, nz), soa(du, nx, ny, nz), job);
      else if (krk == 2) OCFD_time_advance_ker2(soa(f, nx, ny, nz), soa(fn, nx, ny, nz), soa(du, nx, ny, nz), job);
      else OCFD_time_advance_ker3(soa(f, nx, ny, nz), soa(fn, nx, ny, nz), soa(du, nx, ny, nz), sl, job);
    }
  }
}

// Face value of the ring kernel's closures for face f (between cells f-1
// and f) of a line of n cells (F[c] = split flux of cell c); false: WENO7.
// The rules read out of OCFD_NS_Jacobian3d.cpp:1063-1085 (x) and :1515-1584
// (y), as one value per face.
bool ref_closure_face(int pm, int dir, long f, long n, bool lo, bool hi, REAL* F, double* out) {
  if (pm == 0) {
    if (lo && f == 0) { *out = F[0]; return true; }
    if (lo && f == 1) { *out = OCFD_weno5_kernel_P_lift(F + f - 3); return true; }
    if (lo && f == 2) { *out = OCFD_weno5_kernel_P_lift_plus(F + f - 3); return true; }
    if ((lo && f == 3) || (hi && f == n - 2)) { *out = OCFD_weno5_kernel_P(F + f - 3); return true; }
    if (hi && f == n - 1) { *out = OCFD_weno5_kernel_P_right_plus(F + f - 3); return true; }
    if (hi && f == n) {
      *out = dir == 0 ? 1.5*F[n - 1] - 0.5*F[n - 2]
                      : F[n - 1]+0.5*minmod2(F[n - 1] -F[n - 2], F[n - 1] -F[n - 2]);
      return true;
    }
    return false;
  }
  if (lo && f == 0) { *out = OCFD_weno5_kernel_M_lift(F + f - 2); return true; }
  if (lo && f == 1) { *out = OCFD_weno5_kernel_M_lift_plus(F + f - 2); return true; }
  if ((lo && (f == 2 || f == 3)) || (hi && f == n - 3)) { *out = OCFD_weno5_kernel_M(F + f - 2); return true; }
  if (hi && f == n - 2) { *out = OCFD_weno5_kernel_M_right_plus(F + f - 2); return true; }
  if (hi && f == n - 1) {
    *out = dir == 0 ? 0.5 *F[n - 1] + 0.5 *F[n - 2]
                    : F[n - 1]-0.5*minmod2(F[n - 1] - F[n - 2], F[n - 1] - F[n - 2]);
    return true;
  }
  if (hi && f == n) { *out = dir == 0 ? 0.5 *F[n - 1] + 0.5 *F[n - 2] : F[n - 1]; return true; }
  return false;
}

// Decomposed inviscid RHS from the reference's split and WENO functions; the
// loop structure is or_du_invis() of oracle/oracle.cpp.  Cartesian metrics
// when metrics == NULL, J = 1 when ajac == NULL.  Ghosts must be filled by
// the caller; face_kind (may be NULL) marks CLOSURE faces (value 2).
void ref_du_invis(int nx, int ny, int nz, double hx, double hy, double hz, double gamma,
                  double eps, const double* d, const double* u, const double* v,
                  const double* w, const double* cc, const double* const* metrics,
                  const double* ajac, double* du, const int* face_kind) {
  const long px = nx + 2 * LAP, py = ny + 2 * LAP;
  auto lap = [&](long i, long j, long k) { return (i + LAP) + px * ((j + LAP) + py * (k + LAP)); };
  const double h[3] = {hx, hy, hz};
  const long ext[3] = {nx, ny, nz};
  std::memset(du, 0, sizeof(double) * 5 * (size_t)nx * ny * nz);
  for (int dir = 0; dir < 3; ++dir) {
    const long n = ext[dir];
    const long na = dir == 0 ? ny : nx, nb = dir == 2 ? ny : nz;
    #pragma omp parallel
    {
      set_consts(gamma, 1.0, eps);
      ny_2lap_d = 1; nz_2lap_d = 1;
      std::vector<double> fp(5 * (n + 2 * LAP)), fm(5 * (n + 2 * LAP)), face(n + 1);
      #pragma omp for collapse(2) schedule(static)
      for (long b = 0; b < nb; ++b) for (long a = 0; a < na; ++a) {
        auto at = [&](long s) { return dir == 0 ? lap(s, a, b) : dir == 1 ? lap(a, s, b) : lap(a, b, s); };
        auto cell = [&](long s, long var) {
          long i = dir == 0 ? s : a, j = dir == 1 ? s : (dir == 0 ? a : b), k = dir == 2 ? s : b;
          return i + nx * (j + ny * (k + nz * var)); };
        for (long s = -LAP; s < n + LAP; ++s) {
          const long p = at(s);
          double in[8] = {d[p], u[p], v[p], w[p], cc[p],
                          metrics ? metrics[3 * dir][p] : (dir == 0 ? 1.0 : 0.0),
                          metrics ? metrics[3 * dir + 1][p] : (dir == 1 ? 1.0 : 0.0),
                          metrics ? metrics[3 * dir + 2][p] : (dir == 2 ? 1.0 : 0.0)};
          double pp[5], mm[5];
          cudaField f[8];
          for (int q = 0; q < 8; ++q) { f[q].ptr = in + q; f[q].pitch = 1; f[q].dummy0 = 0; }
          cudaSoA sp{pp, 1, 1, 1, 0}, sm{mm, 1, 1, 1, 0};
          threadIdx = dim3(0, 0, 0);
          cudaJobPackage job(dim3(0, 0, 0), dim3(1, 1, 1));
          split_Jac3d_Stager_Warming_ker_origin(f[0], f[1], f[2], f[3], f[4], sp, sm, f[5], f[6], f[7], job);
          for (int var = 0; var < 5; ++var) {
            fp[var * (n + 2 * LAP) + s + LAP] = pp[var];
            fm[var * (n + 2 * LAP) + s + LAP] = mm[var];
          }
        }
        const bool lo = face_kind && dir < 2 && face_kind[2 * dir] == 2;
        const bool hi = face_kind && dir < 2 && face_kind[2 * dir + 1] == 2;
        for (int pm = 0; pm < 2; ++pm) for (int var = 0; var < 5; ++var) {
          double* line = (pm == 0 ? fp.data() : fm.data()) + var * (n + 2 * LAP);
          for (long i = -1; i < n; ++i) {
            REAL* st = line + (i - 3 + LAP);
            if ((lo || hi) && ref_closure_face(pm, dir, i + 1, n, lo, hi, line + LAP, &face[i + 1]))
              continue;
            face[i + 1] = pm == 0 ? OCFD_weno7_SYMBO_kernel_P_opt(st) : OCFD_weno7_SYMBO_kernel_M_opt(st);
          }
          // the ring kernel never adds the y M term of the last cell
          const long iend = (dir == 1 && pm == 1 && hi) ? n - 1 : n;
          for (long i = 0; i < iend; ++i) {
            const double J = ajac ? ajac[at(i)] : 1.0;
            du[cell(i, var)] += -J * (face[i + 1] - face[i]) / h[dir];
          }
        }
      }
    }
  }
}
// Viscous terms (du_vis_Jacobian3d) from the reference's vis_flux_ker,
// get_Amu_kernal, OCFD_kernel_CD6/CD8 and YF_Pe_XF, with the loop structure
// of or_du_vis() in oracle/oracle.cpp: derivatives of u, v, w, T through
// the ghosts (value / h, as put_d0_kernel), viscosity, then per direction
// the flux on the interior, its ghosts filled by face_kind, its derivative
// and du[1..4] += J * derivative.  metrics / ajac may be NULL (Cartesian).
void ref_du_vis(int nx, int ny, int nz, double hx, double hy, double hz, double gamma,
                double ama, double re, double pr, double ref_t, int scheme, double* u,
                double* v, double* w, double* T, const double* const* metrics,
                const double* ajac, double* du, const int* face_kind, const int* d0b) {
  const long px = nx + 2 * LAP, py = ny + 2 * LAP, pz = nz + 2 * LAP, L = px * py * pz;
  const long N = (long)nx * ny * nz;
  auto lap = [&](long i, long j, long k) { return (i + LAP) + px * ((j + LAP) + py * (k + LAP)); };
  const double h[3] = {hx, hy, hz};
  const long r = scheme == 6 ? 3 : 4;
  // Cartesian metrics as fields when none are given
  std::vector<double> unit(L, 1.0), zero(L, 0.0);
  const double* M[9];
  for (int m = 0; m < 9; ++m)
    M[m] = metrics ? metrics[m] : (m == 0 || m == 4 || m == 8 ? unit.data() : zero.data());
  const double* J = ajac ? ajac : unit.data();
  auto cf = [&](const double* p, long pitch) { cudaField f; f.ptr = const_cast<double*>(p);
    f.pitch = (unsigned)pitch; f.dummy0 = 0; return f; };
  // the flags OCFD_bound (OCFD_bound_Scheme.cpp:432-452) sets for one domain
  // whose job spans the interior: x = 4/5/6 with the low face's DIF_BOUND,
  // y = 4/5/6 with the high face's; EXTERNAL faces are a neighbour's boundary
  auto flags = [&](int dir) {
    dim3 fl(dir + 1, 0, 0);
    if (d0b[2 * dir] && face_kind[2 * dir] != 3) fl.x = dir + 4;
    if (d0b[2 * dir + 1] && face_kind[2 * dir + 1] != 3) fl.y = dir + 4;
    return fl;
  };
  auto d0 = [&](const double* f, int dir, double* out) {
    const dim3 fl = flags(dir);
    const cudaJobPackage job(dim3(LAP, LAP, LAP), dim3(nx + LAP, ny + LAP, nz + LAP));
    #pragma omp parallel for collapse(2) schedule(static)
    for (long k = 0; k < nz; ++k) for (long j = 0; j < ny; ++j) for (long i = 0; i < nx; ++i) {
      REAL st[9];
      for (long q = -r; q <= r; ++q)
        st[q + r] = f[dir == 0 ? lap(i + q, j, k) : dir == 1 ? lap(i, j + q, k) : lap(i, j, k + q)];
      REAL tmp;
      // OCFD_CD6_kernel / OCFD_CD8_kernel (OCFD_Schemes.cpp:107-160): the
      // boundary forms first, the central scheme where they do not apply
      int flag = OCFD_D0bound_scheme_kernel(&tmp, fl, dim3(i, j, k), &st[0], (int)-r, job);
      if (flag != 0) tmp = scheme == 6 ? OCFD_kernel_CD6(st) : OCFD_kernel_CD8(st);
      out[i + nx * (j + ny * k)] = tmp / h[dir];
    }
  };
  auto ghost = [&](double* f) {      // periodic wrap / zero gradient, x then y then z
    for (long k = -LAP; k < nz + LAP; ++k) for (long j = -LAP; j < ny + LAP; ++j)
      for (long l = 1; l <= LAP; ++l) {
        f[lap(-l, j, k)] = f[lap(face_kind[0] == 0 ? nx - l : 0, j, k)];
        f[lap(nx - 1 + l, j, k)] = f[lap(face_kind[1] == 0 ? l - 1 : nx - 1, j, k)];
      }
    for (long k = -LAP; k < nz + LAP; ++k) for (long l = 1; l <= LAP; ++l)
      for (long i = -LAP; i < nx + LAP; ++i) {
        f[lap(i, -l, k)] = f[lap(i, face_kind[2] == 0 ? ny - l : 0, k)];
        f[lap(i, ny - 1 + l, k)] = f[lap(i, face_kind[3] == 0 ? l - 1 : ny - 1, k)];
      }
    for (long l = 1; l <= LAP; ++l) for (long j = -LAP; j < ny + LAP; ++j)
      for (long i = -LAP; i < nx + LAP; ++i) {
        f[lap(i, j, -l)] = f[lap(i, j, face_kind[4] == 0 ? nz - l : 0)];
        f[lap(i, j, nz - 1 + l)] = f[lap(i, j, face_kind[5] == 0 ? l - 1 : nz - 1)];
      }
  };
  std::vector<double> grad(12 * N), amu(N), Ev(4 * L), dv(N);
  double* prim[4] = {u, v, w, T};
  for (int dir = 0; dir < 3; ++dir) for (int q = 0; q < 4; ++q)
    d0(prim[q], dir, grad.data() + (4 * dir + q) * N);
  #pragma omp parallel
  {
    set_consts(gamma, ama, 0.0); set_dims(nx, ny, nz);
    // OCFD_init.cpp:380-396
    const double Cp = 1.0 / ((gamma - 1.0) * ama * ama);
    Tsb_d = 110.4 / ref_t;
    amu_C0_d = 1.0 / re * (1.0 + 110.4 / ref_t);
    vis_flux_init_c_d = Cp / pr;
    cudaJobPackage job0(dim3(0, 0, 0), dim3(nx, ny, nz));
    #pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
      threadIdx = dim3(i, j, k); blockIdx = dim3(0, 0, 0); blockDim = dim3(1, 1, 1);
      get_Amu_kernal(cf(amu.data(), nx), cf(T, px), job0);
    }
  }
  auto G = [&](int dir, int q) { return cf(grad.data() + (4 * dir + q) * N, nx); };
  for (int dir = 0; dir < 3; ++dir) {
    std::fill(Ev.begin(), Ev.end(), 0.0);
    #pragma omp parallel
    {
      set_consts(gamma, ama, 0.0); set_dims(nx, ny, nz);
      const double Cp = 1.0 / ((gamma - 1.0) * ama * ama);
      vis_flux_init_c_d = Cp / pr;
      cudaJobPackage job(dim3(LAP, LAP, LAP), dim3(nx + LAP, ny + LAP, nz + LAP));
      #pragma omp for collapse(2) schedule(static)
      for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
        threadIdx = dim3(i, j, k); blockIdx = dim3(0, 0, 0); blockDim = dim3(1, 1, 1);
        vis_flux_ker(G(0, 0), G(0, 1), G(0, 2), G(1, 0), G(1, 1), G(1, 2), G(2, 0), G(2, 1),
                     G(2, 2), G(0, 3), G(1, 3), G(2, 3), cf(amu.data(), nx),
                     cf(u, px), cf(v, px), cf(w, px),
                     cf(M[3 * dir], px), cf(M[3 * dir + 1], px), cf(M[3 * dir + 2], px),
                     cf(J, px), cf(M[0], px), cf(M[1], px), cf(M[2], px), cf(M[3], px),
                     cf(M[4], px), cf(M[5], px), cf(M[6], px), cf(M[7], px), cf(M[8], px),
                     cf(Ev.data(), px), cf(Ev.data() + L, px), cf(Ev.data() + 2 * L, px),
                     cf(Ev.data() + 3 * L, px), job);
      }
    }
    for (int q = 0; q < 4; ++q) {
      double* e = Ev.data() + q * L;
      ghost(e);
      d0(e, dir, dv.data());
      #pragma omp parallel
      {
        set_dims(nx, ny, nz);
        cudaJobPackage job0(dim3(0, 0, 0), dim3(nx, ny, nz));
        #pragma omp for collapse(2) schedule(static)
        for (int k = 0; k < nz; ++k) for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) {
          threadIdx = dim3(i, j, k); blockIdx = dim3(0, 0, 0); blockDim = dim3(1, 1, 1);
          YF_Pe_XF(cf(du + (q + 1) * N, nx), cf(dv.data(), nx), cf(J, px), job0);
        }
      }
    }
  }
}
}  // extern "C"
"""


def extract_function(text: str, name: str) -> str:
    """Return the full definition of function `name` (signature + body)."""
    m = re.search(r"^[^\n;{}]*\b" + re.escape(name) + r"\s*\(", text, re.M)
    while m:
        # skip commented-out lines and prototypes
        start = m.start()
        line = text[start:text.find("\n", start)]
        if not line.lstrip().startswith("//"):
            i = text.find("{", m.end())
            semi = text.find(";", m.end())
            if i != -1 and (semi == -1 or i < semi):
                depth, j = 0, i
                while j < len(text):
                    if text[j] == "{":
                        depth += 1
                    elif text[j] == "}":
                        depth -= 1
                        if depth == 0:
                            return text[start:j + 1]
                    j += 1
        m = re.compile(r"^[^\n;{}]*\b" + re.escape(name) + r"\s*\(", re.M).search(text, m.end())
    raise RuntimeError(f"function {name} not found")


def extract_macro(text: str, name: str) -> str:
    m = re.search(r"^#define\s+" + re.escape(name) + r"\(.*$", text, re.M)
    if not m:
        raise RuntimeError(f"macro {name} not found")
    return m.group(0)


def build(ref: str, native: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    parts = [SHIM_HEAD]
    for hdr, names in MACROS:
        txt = open(os.path.join(ref, hdr), encoding="utf-8", errors="replace").read()
        parts += [extract_macro(txt, n) for n in names]
    for src, name in FUNCS:
        txt = open(os.path.join(ref, src), encoding="utf-8", errors="replace").read()
        parts.append(extract_function(txt, name))
    parts.append(DRIVERS)
    tu = os.path.join(OUT_DIR, "wsref_tu.cpp")
    so = os.path.join(OUT_DIR, "libwsref.so")
    with open(tu, "w") as f:
        f.write("\n\n".join(parts))
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    arch = "-march=native" if native else "-march=x86-64-v2"
    cmd = [cxx, "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-fno-fast-math", arch, "-w", "-o", so, tu]
    try:
        subprocess.run(cmd, check=True)
    finally:
        os.remove(tu)          # keep no reference source on disk
    return so


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("WS_REFERENCE", MOUNT_REF))
    ap.add_argument("--native", action="store_true")
    a = ap.parse_args()
    if not os.path.isdir(os.path.join(a.ref, "src")):
        print(f"reference tree not found at {a.ref}; nothing built", file=sys.stderr)
        return 1
    print(build(a.ref, a.native))
    return 0


if __name__ == "__main__":
    sys.exit(main())
