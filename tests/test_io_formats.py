"""The reference's on-disk formats: restart files (OCFD%08d.dat, OCFD_IO.c)
and metrics files (OCFD3d-Jacobi.dat, OCFD_Comput_Jacobian3d.cpp).

The byte layout is written out here independently of the library (record
markers int32 12 around the header, int32 nx*ny*8 around every z plane) so
a file the reference would write is read back, and the library's files are
byte-identical to it.  CPU only."""
import struct

import numpy as np
import pytest

import windstencil_b200 as ws


def _fortran_restart(nx, ny, nz, istep, tt, prims):
    out = bytearray(struct.pack("<iidi", 12, istep, tt, 12))
    m = struct.pack("<i", nx * ny * 8)
    for q in range(5):
        for k in range(nz):
            out += m + np.ascontiguousarray(prims[q, k], dtype="<f8").tobytes() + m
    return bytes(out)


def _fortran_fields(fields):
    _, nz, ny, nx = fields.shape
    out = bytearray()
    m = struct.pack("<i", nx * ny * 8)
    for q in range(fields.shape[0]):
        for k in range(nz):
            out += m + np.ascontiguousarray(fields[q, k], dtype="<f8").tobytes() + m
    return bytes(out)


def test_restart_read_reference_layout(tmp_path):
    nx, ny, nz = 7, 5, 3
    prims = np.random.default_rng(40).normal(size=(5, nz, ny, nx))
    p = tmp_path / "OCFD00000042.dat"
    p.write_bytes(_fortran_restart(nx, ny, nz, 42, 0.125, prims))
    istep, tt, got = ws.restart_read(str(p), nx, ny, nz)
    assert istep == 42 and tt == 0.125
    assert np.array_equal(got, prims)


def test_restart_write_is_reference_layout(tmp_path):
    nx, ny, nz = 6, 4, 5
    prims = np.random.default_rng(41).normal(size=(5, nz, ny, nx))
    p = tmp_path / "OCFD00000007.dat"
    ws.restart_write(str(p), prims, istep=7, tt=3.5)
    assert p.read_bytes() == _fortran_restart(nx, ny, nz, 7, 3.5, prims)


def test_metrics_round_trip_and_layout(tmp_path):
    nx, ny, nz = 5, 4, 3
    fields = np.random.default_rng(42).normal(size=(13, nz, ny, nx))
    p = tmp_path / "OCFD3d-Jacobi.dat"
    ws.metrics_write(str(p), fields)
    assert p.read_bytes() == _fortran_fields(fields)
    assert np.array_equal(ws.metrics_read(str(p), nx, ny, nz), fields)


@pytest.mark.parametrize("damage", ["short", "marker", "header", "grid"])
def test_restart_rejects_bad_files(tmp_path, damage):
    nx, ny, nz = 4, 4, 2
    raw = bytearray(_fortran_restart(nx, ny, nz, 1, 0.0, np.zeros((5, nz, ny, nx))))
    if damage == "short":
        raw = raw[:-3]
    elif damage == "marker":
        raw[20] ^= 0x01                  # first plane record's leading marker
    elif damage == "header":
        raw[0] = 13
    p = tmp_path / "bad.dat"
    p.write_bytes(bytes(raw))
    n = (nx + 1) if damage == "grid" else nx
    with pytest.raises(ws.WsError, match="WS_ERR_IO"):
        ws.restart_read(str(p), n, ny, nz)


def test_missing_file(tmp_path):
    with pytest.raises(ws.WsError, match="WS_ERR_IO"):
        ws.metrics_read(str(tmp_path / "none.dat"), 4, 4, 4)


@pytest.mark.gpu
def test_solver_save_load_round_trip(cuda, tmp_path):
    from windstencil_b200 import workloads as wl
    g = ws.Grid(20, 12, 8, faces=(1, 1, 0, 0, 0, 0))
    f0 = wl.sod_state(20, 12, 8, seed=43)
    s = ws.Solver(g)
    s.set_state(f0)
    s.step(1e-3, 2)
    a = s.get_state()
    p = tmp_path / "OCFD00000002.dat"
    s.save(str(p), istep=2, tt=2e-3)
    s2 = ws.Solver(g)
    assert s2.load_restart(str(p)) == (2, 2e-3)
    b = s2.get_state()
    assert np.abs(b - a).max() <= 1e-14 * np.abs(a).max()
    s.close()
    s2.close()
