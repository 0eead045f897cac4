"""ctypes declarations of include/windstencil_b200.h.

The structures mirror the C layouts exactly; `load()` opens the in-tree
libwindstencil_b200.so and raises if it is missing -- there is no CPU or
pure-Python fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwindstencil_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "windstencil_b200.h")

LAP = 4
FACE_PERIODIC, FACE_EXTRAP, FACE_CLOSURE, FACE_EXTERNAL = 0, 1, 2, 3
FP64, MIXED = 0, 1

WS_OK = 0
WS_ERR_NONFINITE = 5
ERRORS = {1: "WS_ERR_INVALID", 2: "WS_ERR_CUDA", 3: "WS_ERR_ALLOC", 4: "WS_ERR_UNSUPPORTED",
          5: "WS_ERR_NONFINITE", 6: "WS_ERR_TIMEOUT", 7: "WS_ERR_BUDGET", 8: "WS_ERR_BUSY",
          9: "WS_ERR_NOT_FOUND", 10: "WS_ERR_IO", 11: "WS_ERR_COMM"}


class WsField(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("pitch", C.c_uint32), ("dummy0", C.c_uint32)]


class WsSoa(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("pitch", C.c_uint32), ("length_Y", C.c_uint32),
                ("length_Z", C.c_uint32), ("dummy0", C.c_uint32)]


class WsDim3(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32), ("z", C.c_uint32)]


class WsJob(C.Structure):
    _fields_ = [("start", WsDim3), ("end", WsDim3)]


class WsGrid(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32), ("lap", C.c_uint32),
                ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double),
                ("gamma", C.c_double), ("ama", C.c_double), ("epsl_sw", C.c_double),
                ("face_kind", C.c_int32 * 6), ("precision", C.c_int32),
                ("metrics_uniform", C.c_int32)]


class WsMetrics(C.Structure):
    _fields_ = [(n, WsField) for n in
                ("akx", "aky", "akz", "aix", "aiy", "aiz", "asx", "asy", "asz", "ajac")]


class WsViscous(C.Structure):
    _fields_ = [("re", C.c_double), ("pr", C.c_double), ("ref_t", C.c_double),
                ("scheme", C.c_int32), ("dummy0", C.c_int32), ("d0_bound", C.c_int32 * 6)]


class WsBlockInfo(C.Structure):
    _fields_ = [("index", C.c_int32), ("coords", C.c_int32 * 3), ("origin", C.c_int32 * 3),
                ("n", C.c_int32 * 3), ("nbr", (C.c_int32 * 2) * 3), ("faces", C.c_int32 * 6)]


class WsP2pOp(C.Structure):
    _fields_ = [("kind", C.c_int32), ("peer", C.c_int32), ("axis", C.c_int32),
                ("side", C.c_int32)]


class WsTile(C.Structure):
    _fields_ = [("tile_x", C.c_int32), ("tile_y", C.c_int32), ("scan_z", C.c_int32),
                ("threads", C.c_int32)]


class WsServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("max_active", C.c_int32), ("tile", WsTile),
                ("max_active_cells", C.c_double)]


class WsRequest(C.Structure):
    _fields_ = [("grid", WsGrid), ("nsteps", C.c_int32), ("cfl", C.c_double),
                ("dt", C.c_double), ("f0_host", C.c_void_p), ("synth_seed", C.c_uint64),
                ("synth_mach", C.c_double), ("synth_x_jump", C.c_double),
                ("result_host", C.c_void_p)]


class WsServerStats(C.Structure):
    _fields_ = [(n, C.c_long) for n in ("submitted", "queued", "active", "completed", "failed",
                                        "ticks", "max_active")] + [
        ("hbm_in_use", C.c_size_t), ("p50_latency_s", C.c_double),
        ("p99_latency_s", C.c_double), ("mean_latency_s", C.c_double),
        ("served_cell_rhs", C.c_double), ("executed_cell_rhs", C.c_double),
        ("busy_s", C.c_double), ("elapsed_s", C.c_double), ("admit_s", C.c_double),
        ("rebuild_s", C.c_double), ("steps_s", C.c_double), ("retire_s", C.c_double)]


_P = C.c_void_p
_I = C.c_int
_DP = C.POINTER(C.c_double)
SIGNATURES = {
    "ws_abi_version": (_I, []),
    "ws_last_error": (_I, [C.c_char_p, C.c_size_t]),
    "ws_lap_pitch": (C.c_uint32, [C.c_uint32]),
    "ws_device_error": (_I, [C.POINTER(_I), _P]),
    "ws_du_invis_jacobian3d_init": (_I, [C.POINTER(WsGrid), WsJob, WsField, WsField, _P]),
    "ws_du_invis_jacobian3d": (_I, [C.POINTER(WsGrid), WsJob] + [WsField] * 5 +
                               [C.POINTER(WsMetrics), WsSoa, _P]),
    "ws_du_invis_jacobian3d_tiled": (_I, [C.POINTER(WsGrid), WsJob] + [WsField] * 5 +
                                     [C.POINTER(WsMetrics), WsSoa, WsTile, _P]),
    "ws_ghost_fill": (_I, [C.POINTER(WsGrid), C.POINTER(WsField), _I, _P]),
    "ws_halo_bytes": (C.c_size_t, [C.POINTER(WsGrid), _I, _I]),
    "ws_halo_pack": (_I, [C.POINTER(WsGrid), C.POINTER(WsField), _I, _I, _I, _P, _P]),
    "ws_halo_unpack": (_I, [C.POINTER(WsGrid), C.POINTER(WsField), _I, _I, _I, _P, _P]),
    "ws_halo_x_bytes": (C.c_size_t, [C.POINTER(WsGrid), _I]),
    "ws_halo_pack_x": (_I, [C.POINTER(WsGrid), C.POINTER(WsField), _I, _I, _P, _P]),
    "ws_halo_unpack_x": (_I, [C.POINTER(WsGrid), C.POINTER(WsField), _I, _I, _P, _P]),
    "ws_cons_to_prim": (_I, [C.POINTER(WsGrid), WsSoa] + [WsField] * 6 + [_P]),
    "ws_prim_to_cons": (_I, [C.POINTER(WsGrid)] + [WsField] * 5 + [WsSoa, _P]),
    "ws_time_advance": (_I, [C.POINTER(WsGrid), _I, C.c_double, WsSoa, WsSoa, WsSoa, _P]),
    "ws_solver_create": (_I, [C.POINTER(WsGrid), C.POINTER(_P)]),
    "ws_solver_destroy": (None, [_P]),
    "ws_solver_set_state": (_I, [_P, _P, _P]),
    "ws_solver_get_state": (_I, [_P, _P, _P]),
    "ws_solver_get_state_async": (_I, [_P, _P, _P]),
    "ws_solver_get_rhs": (_I, [_P, _P, _P]),
    "ws_solver_fields": (_I, [_P, C.POINTER(WsSoa), C.POINTER(WsSoa), C.POINTER(WsField)]),
    "ws_solver_compute_dt": (_I, [_P, C.c_double, C.POINTER(C.c_double), _P]),
    "ws_solver_rhs": (_I, [_P, _P]),
    "ws_solver_step": (_I, [_P, C.c_double, _I, _P]),
    "ws_solver_stage": (_I, [_P, _I, C.c_double, _P]),
    "ws_solver_stage_fields": (_I, [_P, _I, C.POINTER(WsField)]),
    "ws_solver_stage_begin": (_I, [_P, _I, _P]),
    "ws_solver_stage_end": (_I, [_P, _I, C.c_double, _P]),
    "ws_solver_stage_flux_fields": (_I, [_P, _I, C.POINTER(WsField)]),
    "ws_solver_status": (_I, [_P, C.POINTER(_I), _P]),
    "ws_solver_set_tile": (_I, [_P, WsTile]),
    "ws_solver_set_viscous": (_I, [_P, C.POINTER(WsViscous)]),
    "ws_solver_save": (_I, [_P, C.c_char_p, C.c_int32, C.c_double, _P]),
    "ws_solver_load": (_I, [_P, C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_double), _P]),
    "ws_restart_write": (_I, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int32, C.c_double,
                              _DP]),
    "ws_restart_read": (_I, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int32),
                             C.POINTER(C.c_double), _DP]),
    "ws_metrics_write": (_I, [C.c_char_p, C.c_int, C.c_int, C.c_int, _DP]),
    "ws_metrics_read": (_I, [C.c_char_p, C.c_int, C.c_int, C.c_int, _DP]),
    "ws_du_vis_workspace_bytes": (C.c_size_t, [C.POINTER(WsGrid)]),
    "ws_du_vis_jacobian3d": (_I, [C.POINTER(WsGrid), C.POINTER(WsViscous)] + [WsField] * 4 +
                             [C.POINTER(WsMetrics), WsSoa, _P, C.c_size_t, _P]),
    "ws_blocks_decompose": (_I, [C.POINTER(WsGrid), C.POINTER(C.c_int32), C.c_int32,
                                 C.POINTER(WsBlockInfo)]),
    "ws_nccl_unique_id": (_I, [_P]),
    "ws_blocks_exchange_plan": (_I, [C.POINTER(WsGrid), C.POINTER(C.c_int32), C.c_int32,
                                     C.POINTER(WsP2pOp), C.c_int32, C.POINTER(C.c_int32)]),
    "ws_blocks_create": (_I, [C.POINTER(WsGrid), C.POINTER(C.c_int32), _P, C.c_int32,
                              C.POINTER(_P)]),
    "ws_blocks_destroy": (None, [_P]),
    "ws_blocks_count": (_I, [_P, C.POINTER(C.c_int32)]),
    "ws_blocks_info": (_I, [_P, C.c_int32, C.POINTER(WsBlockInfo)]),
    "ws_blocks_solver": (_I, [_P, C.c_int32, C.POINTER(_P)]),
    "ws_blocks_set_viscous": (_I, [_P, C.POINTER(WsViscous)]),
    "ws_blocks_step": (_I, [_P, C.c_double, _I, _P]),
    "ws_blocks_compute_dt": (_I, [_P, C.c_double, C.POINTER(C.c_double), _P]),
    "ws_blocks_status": (_I, [_P, C.POINTER(_I), _P]),
    "ws_batch_create": (_I, [C.POINTER(WsGrid), _I, C.POINTER(_P)]),
    "ws_batch_destroy": (None, [_P]),
    "ws_batch_size": (_I, [_P]),
    "ws_batch_set_state": (_I, [_P, _I, _P, _P]),
    "ws_batch_get_state": (_I, [_P, _I, _P, _P]),
    "ws_batch_get_rhs": (_I, [_P, _I, _P, _P]),
    "ws_batch_compute_dt": (_I, [_P, C.c_double, C.POINTER(C.c_double), _P]),
    "ws_batch_set_dt": (_I, [_P, C.POINTER(C.c_double)]),
    "ws_batch_set_tile": (_I, [_P, WsTile]),
    "ws_batch_get_tile": (_I, [_P, C.POINTER(WsTile)]),
    "ws_batch_rhs": (_I, [_P, _P]),
    "ws_batch_step": (_I, [_P, _I, _P]),
    "ws_batch_status": (_I, [_P, C.POINTER(_I), _P]),
    "ws_batch_autotune": (_I, [_P, C.POINTER(WsTile), _P]),
    "ws_compute_dt_static": (_I, [C.POINTER(WsGrid), C.POINTER(WsField), _I, C.c_double,
                                  C.POINTER(C.c_double), _P]),
    "ws_server_create": (_I, [C.POINTER(WsServerConfig), C.POINTER(_P)]),
    "ws_server_destroy": (None, [_P]),
    "ws_server_submit": (_I, [_P, C.POINTER(WsRequest), C.POINTER(C.c_uint64)]),
    "ws_server_poll": (_I, [_P, C.c_uint64, C.POINTER(_I), C.POINTER(C.c_double)]),
    "ws_server_wait": (_I, [_P, C.c_uint64, C.c_double]),
    "ws_server_get_stats": (_I, [_P, C.POINTER(WsServerStats)]),
    "ws_server_release": (_I, [_P, C.c_uint64]),
}

_lib = None


class WsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def header_symbols() -> list[str]:
    """Every function the public header declares."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^WS_API\s+[\w\s\*]+?\b(ws_\w+)\s*\(", txt, re.M)))


def load(path: str | None = None) -> C.CDLL:
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(
            f"{p} is missing: build it with `make -C windstencil_b200` "
            "(there is no fallback implementation)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        if hasattr(lib, name):
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().ws_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != WS_OK:
        raise WsError(rc, last_error())
