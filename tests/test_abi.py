"""The C-ABI library loads, exports every symbol the header declares, and
rejects invalid arguments with WS_ERR_INVALID before touching a device (so
these run without a GPU)."""
import ctypes as C

import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import _abi


def test_library_exports_header_symbols():
    lib = ws.load()
    declared = ws.header_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # every declared symbol has a ctypes signature in the Python mirror
    assert set(declared) <= set(_abi.SIGNATURES), set(declared) - set(_abi.SIGNATURES)


def test_abi_version_and_pitch():
    lib = ws.load()
    assert lib.ws_abi_version() == 1
    for nx in (1, 24, 25, 600, 1000):
        p = lib.ws_lap_pitch(nx)
        assert p >= nx + 8 and p % 32 == 0


def test_struct_layouts():
    # cudaField / cudaSoA / cudaJobPackage layouts of the reference (LP64)
    assert C.sizeof(_abi.WsField) == 16
    assert C.sizeof(_abi.WsSoa) == 24
    assert C.sizeof(_abi.WsJob) == 24
    assert _abi.WsGrid.face_kind.offset == 64


def _fake_field(p=4096):
    return _abi.WsField(0x10000, p, 0)


def _rc(fn, *args):
    lib = ws.load()
    rc = getattr(lib, fn)(*args)
    return rc, ws.last_error()


def test_invalid_arguments_rejected():
    g = ws.Grid(16, 8, 8).c()
    job = ws.interior_job(ws.Grid(16, 8, 8))
    f = _fake_field()
    du = _abi.WsSoa(0x10000, 16, 8, 8, 0)
    # bad lap
    g.lap = 3
    rc, msg = _rc("ws_du_invis_jacobian3d", C.byref(g), job, f, f, f, f, f, None, du, None)
    assert rc == 1 and "lap" in msg
    g.lap = 4
    # job outside the interior
    bad = _abi.WsJob(_abi.WsDim3(3, 4, 4), _abi.WsDim3(20, 12, 12))
    rc, msg = _rc("ws_du_invis_jacobian3d", C.byref(g), bad, f, f, f, f, f, None, du, None)
    assert rc == 1 and "job" in msg
    # pitch too small
    small = _abi.WsField(0x10000, 10, 0)
    rc, msg = _rc("ws_du_invis_jacobian3d", C.byref(g), job, small, f, f, f, f, None, du, None)
    assert rc == 1 and "pitch" in msg
    # NULL field
    rc, msg = _rc("ws_du_invis_jacobian3d", C.byref(g), job, _abi.WsField(None, 64, 0), f, f, f,
                  f, None, du, None)
    assert rc == 1 and "NULL" in msg
    # du too small for the job
    rc, msg = _rc("ws_du_invis_jacobian3d", C.byref(g), job, f, f, f, f, f, None,
                  _abi.WsSoa(0x10000, 8, 8, 8, 0), None)
    assert rc == 1 and "SoA" in msg
    # general metrics without metric fields
    g.metrics_uniform = 0
    rc, msg = _rc("ws_du_invis_jacobian3d", C.byref(g), job, f, f, f, f, f, None, du, None)
    assert rc == 1 and "metrics" in msg
    g.metrics_uniform = 1
    # bad precision / face kind
    g.precision = 7
    assert _rc("ws_du_invis_jacobian3d", C.byref(g), job, f, f, f, f, f, None, du, None)[0] == 1
    g.precision = 0
    g.face_kind[2] = 9
    assert _rc("ws_ghost_fill", C.byref(g), C.byref(f), 1, None)[0] == 1
    g.face_kind[2] = 0
    # krk out of range
    assert _rc("ws_time_advance", C.byref(g), 4, 1.0, du, du, du, None)[0] == 1
    # tile shape not compiled
    rc, msg = _rc("ws_du_invis_jacobian3d_tiled", C.byref(g), job, f, f, f, f, f, None, du,
                  _abi.WsTile(7, 3, 8, 99), None)
    assert rc == 4


def test_python_error_type():
    with pytest.raises(ws.WsError) as e:
        _abi.check(1)
    assert e.value.code == 1


def test_grid_defaults_follow_reference():
    g = ws.Grid(64, 32, 16)
    assert g.hx == 1.0 / 63 and g.hy == 1.0 / 31 and g.hz == 1.0 / 15
    c = g.c()
    assert c.lap == 4 and c.metrics_uniform == 1
    assert np.isclose(c.gamma, 1.4)
