"""windstencil_b200 -- B200 (sm_100a) BF3W inviscid RHS behind a C ABI.

Python mirror of include/windstencil_b200.h for tests, benchmarks and
Python callers.  Device memory comes from torch (plumbing only); every
computation runs in libwindstencil_b200.so, and importing the compute entry
points fails loudly when the library has not been built.

Reference interface this mirrors (WindStencil, src/):
  du_invis_Jacobian3d_init  solver/OCFD_NS_Jacobian3d.cpp:24-33   -> du_invis_jacobian3d_init
  du_invis_Jacobian3d_x     solver/OCFD_NS_Jacobian3d.cpp:133-414 -> du_invis_jacobian3d
  exchange_boundary_xyz_packed_dev  mpi/OCFD_mpi_dev.cpp:123-290 -> ghost_fill (one domain),
                                     halo_pack / halo_unpack + halo.SlabStepper (blocks)
  get_duvwT / cons_to_pri_kernel     kernels/commen_kernel.cpp:78-119 -> cons_to_prim
  pri_to_cons_kernel_warp            kernels/commen_kernel.cpp:33-73  -> prim_to_cons
  OCFD_time_advance                  solver/OCFD_time.cpp:15-91        -> time_advance
  NS_solver_real (time loop)         solver/OCFD_NS_Solver.cpp:64-90   -> Solver
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._abi import (FACE_CLOSURE, FACE_EXTERNAL, FACE_EXTRAP, FACE_PERIODIC, FP64, LAP, MIXED,
                   WsDim3, WsError,
                   WsField, WsGrid, WsJob, WsMetrics, WsSoa, WsTile, WsViscous, check,
                   header_symbols, last_error, load)

__all__ = [
    "FACE_CLOSURE", "FACE_EXTERNAL", "FACE_EXTRAP", "FACE_PERIODIC", "FP64", "MIXED", "LAP",
    "WsError", "Grid", "make_grid", "halo_bytes", "halo_pack", "halo_unpack", "halo_x_bytes",
    "halo_pack_x", "halo_unpack_x",
    "device_error",
    "lap_tensor", "soa_tensor", "field_desc", "soa_desc", "interior_job", "du_invis_jacobian3d",
    "du_vis_jacobian3d", "viscous", "restart_write", "restart_read", "metrics_write",
    "metrics_read",
    "du_invis_jacobian3d_init", "ghost_fill", "cons_to_prim", "prim_to_cons", "time_advance",
    "Solver", "load", "header_symbols", "last_error",
]


@dataclass
class Grid:
    """Grid and physics constants (ws_grid).  h defaults to 1/(N-1), the
    reference's convention (OCFD_init.cpp:29-31)."""
    nx: int
    ny: int
    nz: int
    hx: float | None = None
    hy: float | None = None
    hz: float | None = None
    gamma: float = 1.4
    ama: float = 1.0
    epsl_sw: float = 1e-6
    faces: tuple = (FACE_PERIODIC,) * 6
    precision: int = FP64
    metrics_uniform: bool = True

    def __post_init__(self):
        self.hx = self.hx if self.hx is not None else 1.0 / (self.nx - 1.0)
        self.hy = self.hy if self.hy is not None else 1.0 / (self.ny - 1.0)
        self.hz = self.hz if self.hz is not None else 1.0 / (self.nz - 1.0)

    def c(self) -> WsGrid:
        g = WsGrid()
        g.nx, g.ny, g.nz, g.lap = self.nx, self.ny, self.nz, LAP
        g.hx, g.hy, g.hz = self.hx, self.hy, self.hz
        g.gamma, g.ama, g.epsl_sw = self.gamma, self.ama, self.epsl_sw
        for i, k in enumerate(self.faces):
            g.face_kind[i] = int(k)
        g.precision = int(self.precision)
        g.metrics_uniform = 1 if self.metrics_uniform else 0
        return g

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def make_grid(nx, ny, nz, **kw) -> Grid:
    return Grid(nx, ny, nz, **kw)


def _torch():
    import torch
    return torch


def lap_pitch(nx: int) -> int:
    return int(load().ws_lap_pitch(nx))


def lap_tensor(g: Grid, n: int | None = None, device="cuda", fill=0.0):
    """LAP field(s): (nz+8, ny+8, pitch) float64, pitch = ws_lap_pitch(nx)."""
    torch = _torch()
    shape = (g.nz + 2 * LAP, g.ny + 2 * LAP, lap_pitch(g.nx))
    if n is not None:
        shape = (n,) + shape
    return torch.full(shape, fill, dtype=torch.float64, device=device)


def soa_tensor(g: Grid, device="cuda"):
    torch = _torch()
    return torch.zeros((5, g.nz, g.ny, g.nx), dtype=torch.float64, device=device)


def field_desc(t) -> WsField:
    """ws_field of a (nz+8, ny+8, pitch) float64 tensor (contiguous rows)."""
    assert t.dtype.itemsize == 8 and t.dim() == 3 and t.stride(-1) == 1
    assert t.stride(0) == t.stride(1) * t.shape[1], "planes must be contiguous"
    return WsField(t.data_ptr(), t.stride(1), 0)


def soa_desc(t) -> WsSoa:
    """ws_soa of a (5, Lz, Ly, pitch) float64 tensor."""
    assert t.dtype.itemsize == 8 and t.dim() == 4 and t.stride(-1) == 1
    assert t.stride(1) == t.stride(2) * t.shape[2] and t.stride(0) == t.stride(1) * t.shape[1]
    return WsSoa(t.data_ptr(), t.stride(2), t.shape[2], t.shape[1], 0)


def interior_job(g: Grid) -> WsJob:
    """The reference's job for the whole interior (OCFD_Stream.cpp:193)."""
    return WsJob(WsDim3(LAP, LAP, LAP), WsDim3(g.nx + LAP, g.ny + LAP, g.nz + LAP))


def _stream(stream):
    if stream is None:
        return _torch().cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def _metrics(m):
    if m is None:
        return None
    if isinstance(m, WsMetrics):
        return C.byref(m)
    mm = WsMetrics(*[field_desc(t) for t in m])   # 10 tensors: akx..asz, ajac
    return C.byref(mm)


def viscous(re=500.0, pr=0.72, ref_t=288.15, scheme=8, d0_bound=(0,) * 6) -> WsViscous:
    """ws_viscous: Reynolds and Prandtl numbers, Sutherland Ref_T, CD order 6 or 8,
    and the per-face reduced boundary forms of the derivatives (DIF_BOUND)."""
    return WsViscous(re, pr, ref_t, scheme, 0, (C.c_int32 * 6)(*[int(b) for b in d0_bound]))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def restart_write(path: str, prims, istep: int = 0, tt: float = 0.0) -> None:
    """prims: float64 [5, nz, ny, nx] (d, u, v, w, T) to an OCFD%08d.dat file."""
    a = np.ascontiguousarray(prims, dtype=np.float64)
    _, nz, ny, nx = a.shape
    check(load().ws_restart_write(path.encode(), nx, ny, nz, istep, tt, _dp(a)))


def restart_read(path: str, nx: int, ny: int, nz: int):
    """(Istep, tt, prims [5, nz, ny, nx]) from an OCFD%08d.dat file."""
    a = np.empty((5, nz, ny, nx))
    i, t = C.c_int32(), C.c_double()
    check(load().ws_restart_read(path.encode(), nx, ny, nz, C.byref(i), C.byref(t), _dp(a)))
    return i.value, t.value, a


def metrics_write(path: str, fields) -> None:
    """fields: float64 [13, nz, ny, nx] (x, y, z, akx..asz, ajac)."""
    a = np.ascontiguousarray(fields, dtype=np.float64)
    _, nz, ny, nx = a.shape
    check(load().ws_metrics_write(path.encode(), nx, ny, nz, _dp(a)))


def metrics_read(path: str, nx: int, ny: int, nz: int):
    a = np.empty((13, nz, ny, nx))
    check(load().ws_metrics_read(path.encode(), nx, ny, nz, _dp(a)))
    return a


def du_vis_jacobian3d(g: Grid, vis, u, v, w, T, du, metrics=None, workspace=None,
                      stream=None) -> None:
    """du[1..4] += viscous terms (ws_du_vis_jacobian3d); the workspace is a
    device tensor of at least ws_du_vis_workspace_bytes(g) bytes (allocated
    here when not given)."""
    torch = _torch()
    gc = g.c()
    lib = load()
    need = int(lib.ws_du_vis_workspace_bytes(C.byref(gc)))
    if workspace is None:
        workspace = torch.empty(need // 8 + 2, dtype=torch.float64, device=du.device)
    vp = vis if isinstance(vis, WsViscous) else viscous(**vis)
    mp = None
    if metrics is not None:
        mm = metrics if isinstance(metrics, WsMetrics) else WsMetrics(
            *[field_desc(t) for t in metrics])
        mp = C.byref(mm)
    fs = [field_desc(t) for t in (u, v, w, T)]
    check(lib.ws_du_vis_jacobian3d(C.byref(gc), C.byref(vp), *fs, mp, soa_desc(du),
                                   C.c_void_p(workspace.data_ptr()),
                                   workspace.numel() * workspace.element_size(),
                                   _stream(stream)))


def du_invis_jacobian3d_init(g: Grid, job: WsJob, T, cc, stream=None) -> None:
    gc = g.c()
    check(load().ws_du_invis_jacobian3d_init(C.byref(gc), job, field_desc(T), field_desc(cc),
                                             _stream(stream)))


def du_invis_jacobian3d(g: Grid, job: WsJob, d, u, v, w, cc, du, metrics=None, tile=None,
                        stream=None) -> None:
    """du = BF3W inviscid RHS (ws_du_invis_jacobian3d / _tiled)."""
    gc = g.c()
    fs = [field_desc(t) for t in (d, u, v, w, cc)]
    if metrics is not None:
        mm = metrics if isinstance(metrics, WsMetrics) else WsMetrics(
            *[field_desc(t) for t in metrics])
        mp = C.byref(mm)
    else:
        mp = None
    if tile is None:
        rc = load().ws_du_invis_jacobian3d(C.byref(gc), job, *fs, mp, soa_desc(du),
                                           _stream(stream))
    else:
        rc = load().ws_du_invis_jacobian3d_tiled(C.byref(gc), job, *fs, mp, soa_desc(du),
                                                 WsTile(*tile), _stream(stream))
    check(rc)


def ghost_fill(g: Grid, fields, stream=None) -> None:
    gc = g.c()
    arr = (WsField * len(fields))(*[field_desc(t) for t in fields])
    check(load().ws_ghost_fill(C.byref(gc), arr, len(fields), _stream(stream)))


def device_error(stream=None) -> int:
    """Read and clear the device error word of the launches without a
    per-grid status (ws_device_error): 2 = a staging wait gave up."""
    v = C.c_int()
    check(load().ws_device_error(C.byref(v), _stream(stream)))
    return v.value


def halo_bytes(g: Grid, axis: int, nfields: int) -> int:
    """Bytes of one side's halo along `axis`: nfields x 4 planes over the
    interior of the other two axes."""
    gc = g.c()
    return int(load().ws_halo_bytes(C.byref(gc), axis, nfields))


def halo_x_bytes(g: Grid, nfields: int) -> int:
    return halo_bytes(g, 0, nfields)


def _halo(fn, g: Grid, fields, axis: int, side: int, buf, stream):
    gc = g.c()
    arr = (WsField * len(fields))(*[f if isinstance(f, WsField) else field_desc(f)
                                    for f in fields])
    assert buf.dtype.itemsize == 8 and buf.is_contiguous()
    assert buf.numel() * 8 >= halo_bytes(g, axis, len(fields)), "halo buffer too small"
    check(fn(C.byref(gc), arr, len(fields), axis, side, buf.data_ptr(), _stream(stream)))


def halo_pack(g: Grid, fields, axis: int, side: int, buf, stream=None) -> None:
    """Interior planes next to face (axis, side) (side 0 low, 1 high) of LAP
    fields (tensors or WsField) -> buf (contiguous float64 device tensor)."""
    _halo(load().ws_halo_pack, g, fields, axis, side, buf, stream)


def halo_unpack(g: Grid, fields, axis: int, side: int, buf, stream=None) -> None:
    """buf -> the ghost planes beyond face (axis, side) of the fields."""
    _halo(load().ws_halo_unpack, g, fields, axis, side, buf, stream)


def halo_pack_x(g: Grid, fields, side: int, buf, stream=None) -> None:
    halo_pack(g, fields, 0, side, buf, stream)


def halo_unpack_x(g: Grid, fields, side: int, buf, stream=None) -> None:
    halo_unpack(g, fields, 0, side, buf, stream)


def cons_to_prim(g: Grid, f, d, u, v, w, T, P=None, stream=None) -> None:
    gc = g.c()
    pd = field_desc(P) if P is not None else WsField(None, 0, 0)
    check(load().ws_cons_to_prim(C.byref(gc), soa_desc(f), *[field_desc(t) for t in
                                                              (d, u, v, w, T)], pd,
                                 _stream(stream)))


def prim_to_cons(g: Grid, d, u, v, w, T, f, stream=None) -> None:
    gc = g.c()
    check(load().ws_prim_to_cons(C.byref(gc), *[field_desc(t) for t in (d, u, v, w, T)],
                                 soa_desc(f), _stream(stream)))


def time_advance(g: Grid, krk: int, dt: float, f, fn, du, stream=None) -> None:
    gc = g.c()
    check(load().ws_time_advance(C.byref(gc), krk, dt, soa_desc(f), soa_desc(fn), soa_desc(du),
                                 _stream(stream)))


class Solver:
    """One device-resident grid stepped by SSP-RK3 CUDA graphs (ws_solver_*)."""

    def __init__(self, g: Grid):
        self.g = g
        self._gc = g.c()
        h = C.c_void_p()
        check(load().ws_solver_create(C.byref(self._gc), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            load().ws_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, f_host, stream=None):
        """f_host: C-contiguous float64 numpy (5, nz, ny, nx)."""
        import numpy as np
        a = np.ascontiguousarray(f_host, dtype=np.float64)
        self._keep = a
        check(load().ws_solver_set_state(self.h, a.ctypes.data, _stream(stream)))

    def get_state(self, stream=None):
        import numpy as np
        out = np.empty((5, self.g.nz, self.g.ny, self.g.nx))
        check(load().ws_solver_get_state(self.h, out.ctypes.data, _stream(stream)))
        return out

    def get_rhs(self, stream=None):
        """du of the last rhs() (a step uses du as scratch: read it first)."""
        import numpy as np
        out = np.empty((5, self.g.nz, self.g.ny, self.g.nx))
        check(load().ws_solver_get_rhs(self.h, out.ctypes.data, _stream(stream)))
        return out

    def fields(self):
        f, du = WsSoa(), WsSoa()
        prims = (WsField * 6)()
        check(load().ws_solver_fields(self.h, C.byref(f), C.byref(du), prims))
        return f, du, list(prims)

    def compute_dt(self, cfl: float, stream=None) -> float:
        dt = C.c_double()
        check(load().ws_solver_compute_dt(self.h, cfl, C.byref(dt), _stream(stream)))
        return dt.value

    def rhs(self, stream=None):
        check(load().ws_solver_rhs(self.h, _stream(stream)))

    def step(self, dt: float, nsteps: int = 1, stream=None):
        check(load().ws_solver_step(self.h, dt, nsteps, _stream(stream)))

    def stage(self, krk: int, dt: float, stream=None):
        """One SSP-RK3 stage (1, 2, 3 in order); EXTERNAL ghosts come from the caller."""
        check(load().ws_solver_stage(self.h, krk, dt, _stream(stream)))

    def stage_fields(self, krk: int):
        """WsField descriptors of d,u,v,w,T,cc that stage krk reads."""
        prims = (WsField * 6)()
        check(load().ws_solver_stage_fields(self.h, krk, prims))
        return list(prims)

    def stage_begin(self, krk: int, stream=None):
        """First half of a stage: ghost fill, viscous flux pass."""
        check(load().ws_solver_stage_begin(self.h, krk, _stream(stream)))

    def stage_end(self, krk: int, dt: float, stream=None):
        """Second half: viscous divergence, fused RHS + stage update."""
        check(load().ws_solver_stage_end(self.h, krk, dt, _stream(stream)))

    def stage_flux_fields(self, axis: int = 0):
        """WsField descriptors of direction `axis`'s four viscous fluxes."""
        ev = (WsField * 4)()
        check(load().ws_solver_stage_flux_fields(self.h, axis, ev))
        return list(ev)

    def status(self, stream=None) -> int:
        s = C.c_int()
        check(load().ws_solver_status(self.h, C.byref(s), _stream(stream)))
        return s.value

    def set_tile(self, tile):
        check(load().ws_solver_set_tile(self.h, WsTile(*tile)))

    def save(self, path: str, istep: int = 0, tt: float = 0.0, stream=None) -> None:
        """Current state to a restart file (OCFD%08d.dat format)."""
        check(load().ws_solver_save(self.h, path.encode(), istep, tt, _stream(stream)))

    def load_restart(self, path: str, stream=None):
        """State from a restart file; returns (Istep, tt)."""
        i, t = C.c_int32(), C.c_double()
        check(load().ws_solver_load(self.h, path.encode(), C.byref(i), C.byref(t),
                                    _stream(stream)))
        return i.value, t.value

    def set_viscous(self, vis):
        """Navier-Stokes with ws_viscous constants (a WsViscous, a dict with
        re, pr, ref_t, scheme, or None for Euler)."""
        if vis is None:
            check(load().ws_solver_set_viscous(self.h, None))
            return
        v = vis if isinstance(vis, WsViscous) else viscous(**vis)
        check(load().ws_solver_set_viscous(self.h, C.byref(v)))


class Batch:
    """Many device-resident grids stepped together (ws_batch_*)."""

    def __init__(self, grids):
        self.grids = list(grids)
        arr = (WsGrid * len(self.grids))(*[g.c() for g in self.grids])
        h = C.c_void_p()
        check(load().ws_batch_create(arr, len(self.grids), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            load().ws_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.grids)

    def set_state(self, i, f_host, stream=None):
        import numpy as np
        a = np.ascontiguousarray(f_host, dtype=np.float64)
        check(load().ws_batch_set_state(self.h, i, a.ctypes.data, _stream(stream)))
        _abi_sync(stream)

    def get_state(self, i, stream=None):
        import numpy as np
        g = self.grids[i]
        out = np.empty((5, g.nz, g.ny, g.nx))
        check(load().ws_batch_get_state(self.h, i, out.ctypes.data, _stream(stream)))
        return out

    def get_rhs(self, i, stream=None):
        """du of grid i after the last rhs() (a step overwrites it)."""
        import numpy as np
        g = self.grids[i]
        out = np.empty((5, g.nz, g.ny, g.nx))
        check(load().ws_batch_get_rhs(self.h, i, out.ctypes.data, _stream(stream)))
        return out

    def compute_dt(self, cfl, stream=None):
        import numpy as np
        out = np.empty(len(self.grids))
        check(load().ws_batch_compute_dt(self.h, cfl, out.ctypes.data_as(C.POINTER(C.c_double)),
                                         _stream(stream)))
        return out

    def set_dt(self, dts):
        import numpy as np
        a = np.ascontiguousarray(dts, dtype=np.float64)
        check(load().ws_batch_set_dt(self.h, a.ctypes.data_as(C.POINTER(C.c_double))))

    def set_tile(self, tile):
        check(load().ws_batch_set_tile(self.h, WsTile(*tile)))

    def rhs(self, stream=None):
        check(load().ws_batch_rhs(self.h, _stream(stream)))

    def step(self, nsteps=1, stream=None):
        check(load().ws_batch_step(self.h, nsteps, _stream(stream)))

    def status(self, stream=None):
        arr = (C.c_int * len(self.grids))()
        check(load().ws_batch_status(self.h, arr, _stream(stream)))
        return list(arr)

    def autotune(self, stream=None):
        t = WsTile()
        check(load().ws_batch_autotune(self.h, C.byref(t), _stream(stream)))
        return (t.tile_x, t.tile_y, t.scan_z, t.threads)


class Server:
    """Continuous-batching solve server (ws_server_*)."""

    def __init__(self, hbm_budget_bytes=80 << 30, max_active=4096, tile=(0, 0, 0, 0),
                 max_active_cells=0.0):
        from ._abi import WsServerConfig
        cfg = WsServerConfig(hbm_budget_bytes, max_active, WsTile(*tile), max_active_cells)
        h = C.c_void_p()
        check(load().ws_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self._keep = {}

    def close(self):
        if self.h:
            load().ws_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, grid: Grid, nsteps, cfl=0.5, dt=0.0, f0=None, seed=0, mach=1.0,
               x_jump=0.5, want_result=True):
        """Queue a solve; returns the request id.  f0: dense conserved state
        (numpy) or None for the seeded synthetic state on the device."""
        import numpy as np
        from ._abi import WsRequest
        res = np.empty((5, grid.nz, grid.ny, grid.nx)) if want_result else None
        f0a = None if f0 is None else np.ascontiguousarray(f0, dtype=np.float64)
        r = WsRequest(grid.c(), nsteps, cfl, dt, None if f0a is None else f0a.ctypes.data,
                      seed, mach, x_jump, None if res is None else res.ctypes.data)
        rid = C.c_uint64()
        check(load().ws_server_submit(self.h, C.byref(r), C.byref(rid)))
        self._keep[rid.value] = (f0a, res)
        return rid.value

    def poll(self, rid):
        st, lat = C.c_int(), C.c_double()
        rc = load().ws_server_poll(self.h, rid, C.byref(st), C.byref(lat))
        return st.value, lat.value, rc

    def wait(self, rid, timeout=0.0):
        check(load().ws_server_wait(self.h, rid, timeout))
        return self._keep[rid][1]

    def result(self, rid):
        return self._keep[rid][1]

    def release(self, rid):
        check(load().ws_server_release(self.h, rid))
        self._keep.pop(rid, None)

    def stats(self) -> dict:
        from ._abi import WsServerStats
        s = WsServerStats()
        check(load().ws_server_get_stats(self.h, C.byref(s)))
        return {n: getattr(s, n) for n, _ in WsServerStats._fields_}


def _abi_sync(stream):
    """Host buffers handed to an asynchronous upload must outlive it."""
    if stream is None:
        _torch().cuda.current_stream().synchronize()
    else:
        getattr(stream, "synchronize", lambda: None)()
