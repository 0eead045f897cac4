"""ctypes bindings of the CPU oracle (test infrastructure only).

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs as
the checker; the product package never imports this module.

`Oracle` wraps oracle/liboracle.so (the restatement, oracle/oracle.cpp).
`RefFunctions` wraps oracle/_ref/libwsref.so (the reference's own scalar
kernels built for the host by oracle/build_ref.py) when it has been built.
Arrays are numpy float64 in the dense layouts of oracle/oracle.h:
LAP field (nz+8, ny+8, nx+8) and SoA (5, nz, ny, nx).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LAP = 4
FACE_PERIODIC, FACE_EXTRAP, FACE_CLOSURE, FACE_EXTERNAL = 0, 1, 2, 3
# WENO5 closure family, in the order of or_weno5_batch / ref_weno5_batch
WENO5_FORMS = ("p_lift", "p_lift_plus", "p", "p_right_plus", "m_lift", "m_lift_plus",
               "m", "m_right_plus", "minmod2")

_dp = C.POINTER(C.c_double)


class OrGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double),
                ("gamma", C.c_double), ("ama", C.c_double), ("epsl_sw", C.c_double),
                ("face_kind", C.c_int * 6)]


class OrVis(C.Structure):
    """Viscous constants: Re, Pr, Sutherland Ref_T, central-difference order 6 or 8,
    DIF_BOUND flags per face (the reduced boundary forms of the derivatives)."""
    _fields_ = [("re", C.c_double), ("pr", C.c_double), ("ref_t", C.c_double),
                ("scheme", C.c_int), ("d0_bound", C.c_int * 6)]


def make_vis(re=500.0, pr=0.72, ref_t=288.15, scheme=8, d0_bound=(0,) * 6) -> OrVis:
    v = OrVis()
    v.re, v.pr, v.ref_t, v.scheme = re, pr, ref_t, scheme
    for i, b in enumerate(d0_bound):
        v.d0_bound[i] = int(b)
    return v


def make_grid(nx, ny, nz, hx=None, hy=None, hz=None, gamma=1.4, ama=1.0,
              epsl_sw=1e-6, face_kind=(0, 0, 0, 0, 0, 0)) -> OrGrid:
    """Grid spacing defaults to the reference's h = 1/(N-1) (OCFD_init.cpp:29-31)."""
    g = OrGrid()
    g.nx, g.ny, g.nz = nx, ny, nz
    g.hx = hx if hx is not None else 1.0 / (nx - 1.0)
    g.hy = hy if hy is not None else 1.0 / (ny - 1.0)
    g.hz = hz if hz is not None else 1.0 / (nz - 1.0)
    g.gamma, g.ama, g.epsl_sw = gamma, ama, epsl_sw
    for i, k in enumerate(face_kind):
        g.face_kind[i] = int(k)
    return g


def _p(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _ptr_array(arrs):
    if arrs is None:
        return None
    t = (_dp * len(arrs))(*[_p(a) for a in arrs])
    return t


def build_oracle(native: bool = False, out: str | None = None) -> str:
    """Compile liboracle.so (portable) or a -march=native copy at `out`."""
    if native:
        out = out or os.path.join(HERE, "liboracle_native.so")
        subprocess.run(["make", "-s", "-C", HERE, "native", f"OUT={out}"], check=True)
        return out
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return os.path.join(HERE, "liboracle.so")


class Oracle:
    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build_oracle()
        L = C.CDLL(path)
        self.lib = L
        L.or_weno7_p.restype = C.c_double
        L.or_weno7_m.restype = C.c_double
        L.or_compute_dt.restype = C.c_double
        L.or_get_threads.restype = C.c_int
        L.or_split_batch.argtypes = [_dp, C.c_long, C.c_double, C.c_double, _dp, _dp]
        L.or_weno7_p_batch.argtypes = [_dp, C.c_long, _dp]
        L.or_weno7_m_batch.argtypes = [_dp, C.c_long, _dp]
        L.or_weno5_batch.argtypes = [C.c_int, _dp, C.c_long, _dp]
        L.or_time_advance.argtypes = [C.c_int, C.c_double, C.c_long, _dp, _dp, _dp]

    # -- scalar kernels ----------------------------------------------------
    def weno_p(self, s: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(-1, 8)
        out = np.empty(len(s))
        self.lib.or_weno7_p_batch(_p(s), len(s), _p(out))
        return out

    def weno_m(self, s: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(-1, 8)
        out = np.empty(len(s))
        self.lib.or_weno7_m_batch(_p(s), len(s), _p(out))
        return out

    def weno5(self, form: str, s: np.ndarray) -> np.ndarray:
        """WENO5 closure form (WENO5_FORMS) on rows of 5 points."""
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(-1, 5)
        out = np.empty(len(s))
        self.lib.or_weno5_batch(WENO5_FORMS.index(form), _p(s), len(s), _p(out))
        return out

    def split(self, pts: np.ndarray, gamma=1.4, epsl_sw=1e-6):
        """pts (n, 8) = d,u,v,w,cc,a1,a2,a3 -> (fp (n,5), fm (n,5))."""
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 8)
        fp = np.empty((len(pts), 5))
        fm = np.empty((len(pts), 5))
        self.lib.or_split_batch(_p(pts), len(pts), gamma, epsl_sw, _p(fp), _p(fm))
        return fp, fm

    # -- field kernels -----------------------------------------------------
    def ghost_fill(self, g: OrGrid, field: np.ndarray) -> None:
        self.lib.or_ghost_fill(C.byref(g), _p(field))

    def sound_speed(self, g: OrGrid, T: np.ndarray) -> np.ndarray:
        cc = np.empty_like(T)
        self.lib.or_sound_speed(C.byref(g), _p(T), _p(cc))
        return cc

    def du_invis(self, g: OrGrid, d, u, v, w, cc, metrics=None, ajac=None) -> np.ndarray:
        du = np.empty((5, g.nz, g.ny, g.nx))
        self.lib.or_du_invis(C.byref(g), _p(d), _p(u), _p(v), _p(w), _p(cc),
                             _ptr_array(metrics), _p(ajac), _p(du))
        return du

    def cons_to_prim(self, g: OrGrid, f: np.ndarray):
        shp = (g.nz + 2 * LAP, g.ny + 2 * LAP, g.nx + 2 * LAP)
        out = [np.zeros(shp) for _ in range(6)]
        self.lib.or_cons_to_prim(C.byref(g), _p(f), *[_p(a) for a in out])
        return out  # d, u, v, w, T, P

    def prim_to_cons(self, g: OrGrid, d, u, v, w, T) -> np.ndarray:
        f = np.empty((5, g.nz, g.ny, g.nx))
        self.lib.or_prim_to_cons(C.byref(g), _p(d), _p(u), _p(v), _p(w), _p(T), _p(f))
        return f

    def time_advance(self, krk, dt, f, fn, du) -> None:
        self.lib.or_time_advance(krk, dt, f.size, _p(f), _p(fn), _p(du))

    # -- solver ------------------------------------------------------------
    def compute_dt(self, g: OrGrid, f: np.ndarray, cfl: float) -> float:
        return self.lib.or_compute_dt(C.byref(g), _p(f), C.c_double(cfl))

    def rk3_steps(self, g: OrGrid, f: np.ndarray, dt: float, nsteps: int,
                  metrics=None, ajac=None) -> np.ndarray:
        out = np.array(f, dtype=np.float64, order="C", copy=True)
        rc = self.lib.or_rk3_steps(C.byref(g), _p(out), C.c_double(dt), nsteps,
                                   _ptr_array(metrics), _p(ajac))
        if rc != 0:
            raise MemoryError("oracle rk3 allocation failed")
        return out

    def du_vis(self, g: OrGrid, vis: OrVis, u, v, w, T, metrics=None, ajac=None,
               du=None) -> np.ndarray:
        """du[1..4] += viscous terms (du zero when not given)."""
        du = np.zeros((5, g.nz, g.ny, g.nx)) if du is None else du
        self.lib.or_du_vis(C.byref(g), C.byref(vis), _p(u), _p(v), _p(w), _p(T),
                           _ptr_array(metrics), _p(ajac), _p(du))
        return du

    def vis_fluxes(self, g: OrGrid, vis: OrVis, u, v, w, T, metrics=None, ajac=None):
        """12 viscous flux LAP fields (3*4, nz+8, ny+8, nx+8): direction-major."""
        shp = (12, g.nz + 2 * LAP, g.ny + 2 * LAP, g.nx + 2 * LAP)
        ev = np.zeros(shp)
        self.lib.or_vis_fluxes(C.byref(g), C.byref(vis), _p(u), _p(v), _p(w), _p(T),
                               _ptr_array(metrics), _p(ajac), _p(ev))
        return ev

    def vis_div_add(self, g: OrGrid, vis: OrVis, direction: int, ev4: np.ndarray, du,
                    ajac=None) -> None:
        """Ghost fill of ev4 (4 LAP fields, in place) and du[1..4] += J d/d(dir)."""
        assert ev4.flags.c_contiguous and ev4.shape[0] == 4
        self.lib.or_vis_div_add(C.byref(g), C.byref(vis), direction, _p(ev4), _p(ajac), _p(du))

    def rhs_conserved_ns(self, g: OrGrid, vis: OrVis, f: np.ndarray, metrics=None,
                         ajac=None) -> np.ndarray:
        du = np.empty_like(f)
        self.lib.or_rhs_conserved_ns(C.byref(g), C.byref(vis), _p(f), _p(du),
                                     _ptr_array(metrics), _p(ajac))
        return du

    def rk3_steps_ns(self, g: OrGrid, vis: OrVis, f: np.ndarray, dt: float, nsteps: int,
                     metrics=None, ajac=None) -> np.ndarray:
        out = np.array(f, dtype=np.float64, order="C", copy=True)
        rc = self.lib.or_rk3_steps_ns(C.byref(g), C.byref(vis), _p(out), C.c_double(dt),
                                      nsteps, _ptr_array(metrics), _p(ajac))
        if rc != 0:
            raise MemoryError("oracle rk3 allocation failed")
        return out

    def rhs_conserved(self, g: OrGrid, f: np.ndarray, metrics=None, ajac=None) -> np.ndarray:
        du = np.empty_like(f)
        self.lib.or_rhs_conserved(C.byref(g), _p(f), _p(du), _ptr_array(metrics), _p(ajac))
        return du

    def op_counts(self) -> dict:
        out = (C.c_double * 7)()
        self.lib.or_op_counts(out)
        keys = ["split", "weno_p", "weno_m", "diff", "flop_per_cell",
                "split_sqrt_div", "weno_div_per_cell"]
        return dict(zip(keys, list(out)))

    def set_threads(self, n: int) -> None:
        self.lib.or_set_threads(int(n))

    def threads(self) -> int:
        return self.lib.or_get_threads()


class RefFunctions:
    """The reference's own scalar kernels built for the host (oracle/_ref)."""

    PATH = os.path.join(HERE, "_ref", "libwsref.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.PATH)

    def __init__(self, path: str | None = None):
        L = C.CDLL(path or self.PATH)
        self.lib = L
        L.ref_weno_p.restype = C.c_double
        L.ref_weno_m.restype = C.c_double
        L.ref_split_batch.argtypes = [_dp, C.c_long, C.c_double, C.c_double, _dp, _dp]
        L.ref_weno_p_batch.argtypes = [_dp, C.c_long, _dp]
        L.ref_weno_m_batch.argtypes = [_dp, C.c_long, _dp]
        L.ref_weno5_batch.argtypes = [C.c_int, _dp, C.c_long, _dp]
        L.ref_cons_to_prim.argtypes = [C.c_int] * 3 + [C.c_double] * 2 + [_dp] * 7
        L.ref_prim_to_cons.argtypes = [C.c_int] * 3 + [C.c_double] * 2 + [_dp] * 6
        L.ref_sound_speed.argtypes = [C.c_int] * 3 + [C.c_double, _dp, _dp]
        L.ref_time_advance.argtypes = [C.c_int, C.c_double] + [C.c_int] * 3 + [_dp] * 3
        L.ref_du_invis.argtypes = ([C.c_int] * 3 + [C.c_double] * 5 + [_dp] * 5 +
                                   [C.POINTER(_dp), _dp, _dp, C.POINTER(C.c_int)])
        L.ref_du_vis.argtypes = ([C.c_int] * 3 + [C.c_double] * 8 + [C.c_int] + [_dp] * 4 +
                                 [C.POINTER(_dp), _dp, _dp, C.POINTER(C.c_int),
                                  C.POINTER(C.c_int)])

    def weno_p(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(-1, 8)
        out = np.empty(len(s))
        self.lib.ref_weno_p_batch(_p(s), len(s), _p(out))
        return out

    def weno_m(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(-1, 8)
        out = np.empty(len(s))
        self.lib.ref_weno_m_batch(_p(s), len(s), _p(out))
        return out

    def weno5(self, form, s):
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(-1, 5)
        out = np.empty(len(s))
        self.lib.ref_weno5_batch(WENO5_FORMS.index(form), _p(s), len(s), _p(out))
        return out

    def split(self, pts, gamma=1.4, epsl_sw=1e-6):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 8)
        fp = np.empty((len(pts), 5))
        fm = np.empty((len(pts), 5))
        self.lib.ref_split_batch(_p(pts), len(pts), gamma, epsl_sw, _p(fp), _p(fm))
        return fp, fm

    def cons_to_prim(self, g: OrGrid, f, out=None):
        """d, u, v, w, T, P as LAP fields (interiors written; `out` reused when given)."""
        if out is None:
            shp = (g.nz + 2 * LAP, g.ny + 2 * LAP, g.nx + 2 * LAP)
            out = [np.zeros(shp) for _ in range(6)]
        self.lib.ref_cons_to_prim(g.nx, g.ny, g.nz, g.gamma, g.ama, _p(f), *[_p(a) for a in out])
        return out

    def prim_to_cons(self, g: OrGrid, d, u, v, w, T):
        f = np.empty((5, g.nz, g.ny, g.nx))
        self.lib.ref_prim_to_cons(g.nx, g.ny, g.nz, g.gamma, g.ama, _p(d), _p(u), _p(v),
                                  _p(w), _p(T), _p(f))
        return f

    def sound_speed(self, g: OrGrid, T, out=None):
        cc = np.empty_like(T) if out is None else out
        self.lib.ref_sound_speed(g.nx, g.ny, g.nz, g.ama, _p(T), _p(cc))
        return cc

    def time_advance(self, krk, dt, g: OrGrid, f, fn, du):
        self.lib.ref_time_advance(krk, dt, g.nx, g.ny, g.nz, _p(f), _p(fn), _p(du))

    def du_invis(self, g: OrGrid, d, u, v, w, cc, metrics=None, ajac=None, out=None):
        du = np.empty((5, g.nz, g.ny, g.nx)) if out is None else out
        kinds = (C.c_int * 6)(*[g.face_kind[i] for i in range(6)])
        self.lib.ref_du_invis(g.nx, g.ny, g.nz, g.hx, g.hy, g.hz, g.gamma, g.epsl_sw,
                              _p(d), _p(u), _p(v), _p(w), _p(cc), _ptr_array(metrics),
                              _p(ajac), _p(du), kinds)
        return du

    def du_vis(self, g: OrGrid, vis: OrVis, u, v, w, T, metrics=None, ajac=None, du=None):
        du = np.zeros((5, g.nz, g.ny, g.nx)) if du is None else du
        kinds = (C.c_int * 6)(*[g.face_kind[i] for i in range(6)])
        d0b = (C.c_int * 6)(*[vis.d0_bound[i] for i in range(6)])
        self.lib.ref_du_vis(g.nx, g.ny, g.nz, g.hx, g.hy, g.hz, g.gamma, g.ama, vis.re,
                            vis.pr, vis.ref_t, vis.scheme, _p(u), _p(v), _p(w), _p(T),
                            _ptr_array(metrics), _p(ajac), _p(du), kinds, d0b)
        return du


class RefRK3:
    """SSP-RK3 time steps assembled from the reference's own scalar kernels
    built for the host (oracle/_ref): per stage cons_to_pri_kernel, the ghost
    fill (the oracle's restatement of the periodic / boundary halo), the
    sound speed, the decomposed inviscid RHS and OCFD_time_advance_ker1/2/3
    (the solver loop of OCFD_NS_Solver.cpp:64-90 with all three stages, as
    or_rk3_steps runs it).  Every array is allocated once; a step allocates
    nothing.  Used by bench.py's reference arm and CPU baseline only."""

    def __init__(self, g: OrGrid, f: np.ndarray, ref: RefFunctions | None = None,
                 oracle: Oracle | None = None):
        self.g = g
        self.ref = ref or RefFunctions()
        self.o = oracle or Oracle()
        shp = (g.nz + 2 * LAP, g.ny + 2 * LAP, g.nx + 2 * LAP)
        self.prims = [np.zeros(shp) for _ in range(6)]    # d, u, v, w, T, P
        self.cc = np.zeros(shp)
        self.f = np.array(f, dtype=np.float64, order="C", copy=True)
        self.fn = np.empty_like(self.f)
        self.du = np.empty_like(self.f)

    def rhs(self) -> np.ndarray:
        g = self.g
        self.ref.cons_to_prim(g, self.f, out=self.prims)
        for x in self.prims[:5]:
            self.o.ghost_fill(g, x)
        self.ref.sound_speed(g, self.prims[4], out=self.cc)
        d, u, v, w = self.prims[:4]
        return self.ref.du_invis(g, d, u, v, w, self.cc, out=self.du)

    def step(self, dt: float) -> None:
        np.copyto(self.fn, self.f)
        for krk in (1, 2, 3):
            self.rhs()
            self.ref.time_advance(krk, dt, self.g, self.f, self.fn, self.du)
