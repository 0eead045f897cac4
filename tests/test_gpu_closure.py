"""CLOSURE face mode on the GPU against the oracle.

A CLOSURE x or y face gives the faces next to it the boundary closures of the
reference's fused path (its ring kernel): one-sided WENO5 forms, linear
extrapolation / averages (x) or minmod2 forms (y) at the high end, and the
reference's dropped M term of the last y cell.  The oracle's closure forms
are pinned bit for bit to the reference's own functions
(tests/test_oracle_pin.py).  Tolerance as for the other FP64 paths: rel.
L-inf per field <= 1e-12; the mixed form within its one-RHS budget.  Both
kernels run every case: the line passes (the default, and tile_x < 0) and
the fused tile sweep (an explicit tile).
"""
import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import workloads as wl
from oracle.oracle import make_grid as or_grid
from tests.conftest import rel_l2, rel_linf

pytestmark = pytest.mark.gpu
TOL = 1e-12
CL, EX, PE = ws.FACE_CLOSURE, ws.FACE_EXTRAP, ws.FACE_PERIODIC

LINES = (-1, 0, 0, 0)
FUSED = (16, 8, 0, 704)
FACES = [(CL, CL, PE, PE, PE, PE), (PE, PE, CL, CL, PE, PE), (CL, CL, CL, CL, EX, EX),
         (CL, EX, EX, CL, PE, PE), (EX, CL, CL, PE, PE, PE)]


def _rhs(g, f0, tile=None):
    s = ws.Solver(g)
    if tile:
        s.set_tile(tile)
    s.set_state(f0)
    s.rhs()
    out = s.get_rhs()
    s.close()
    return out


@pytest.mark.parametrize("path", [None, FUSED])
@pytest.mark.parametrize("faces", FACES)
@pytest.mark.parametrize("shape", [(40, 24, 10), (19, 13, 7), (8, 8, 5)])
def test_closure_rhs_fp64(oracle, cuda, faces, shape, path):
    f0 = wl.fourier_state(*shape, seed=21)
    ref = oracle.rhs_conserved(or_grid(*shape, face_kind=faces), f0)
    out = _rhs(ws.Grid(*shape, faces=faces), f0, path)
    assert rel_linf(out, ref).max() <= TOL


@pytest.mark.parametrize("warps", [0, 8])
def test_closure_rhs_line_passes_explicit(oracle, cuda, warps):
    shape, faces = (45, 38, 11), (CL, CL, CL, CL, EX, EX)
    f0 = wl.sod_state(*shape, seed=27)
    ref = oracle.rhs_conserved(or_grid(*shape, face_kind=faces), f0)
    out = _rhs(ws.Grid(*shape, faces=faces), f0, (-1, 0, 0, 32 * warps))
    assert rel_linf(out, ref).max() <= TOL


@pytest.mark.parametrize("tile", [(16, 8, 0, 768), (8, 8, 0, 384), (16, 8, 3, 704),
                                  (8, 8, 5, 256)])
def test_closure_rhs_tiles(oracle, cuda, tile):
    shape, faces = (37, 21, 9), (CL, CL, CL, CL, PE, PE)
    f0 = wl.sod_state(*shape, seed=22)
    ref = oracle.rhs_conserved(or_grid(*shape, face_kind=faces), f0)
    out = _rhs(ws.Grid(*shape, faces=faces), f0, tile)
    assert rel_linf(out, ref).max() <= TOL


@pytest.mark.parametrize("path", [None, FUSED])
def test_closure_drop_in_subjob(oracle, cuda, path):
    # a job away from the origin still places the closures at the grid's faces
    from tests.test_gpu_parity import _case
    g = ws.Grid(30, 20, 12, faces=(CL, CL, CL, CL, PE, PE))
    for job in (ws.WsJob(ws.WsDim3(4, 4, 4), ws.WsDim3(34, 24, 16)),
                ws.WsJob(ws.WsDim3(7, 5, 6), ws.WsDim3(34, 24, 13)),
                ws.WsJob(ws.WsDim3(30, 21, 4), ws.WsDim3(34, 24, 16))):
        out, ref = _case(oracle, cuda, g, wl.fourier_state(30, 20, 12, seed=23), tile=path,
                         job=job)
        assert rel_linf(out, ref).max() <= TOL


@pytest.mark.parametrize("path", [None, FUSED])
def test_closure_solver_steps(oracle, cuda, path):
    nx, ny, nz = 48, 24, 8
    faces = (CL, CL, CL, CL, PE, PE)
    og = or_grid(nx, ny, nz, face_kind=faces)
    f0 = wl.fourier_state(nx, ny, nz, seed=24)
    dt = oracle.compute_dt(og, f0, 0.5)
    ref = oracle.rk3_steps(og, f0, dt, 5)
    s = ws.Solver(ws.Grid(nx, ny, nz, faces=faces))
    if path:
        s.set_tile(path)
    s.set_state(f0)
    s.step(dt, 5)
    out = s.get_state()
    assert s.status() == 0
    s.close()
    assert rel_linf(out, ref).max() <= TOL


@pytest.mark.parametrize("path", [None, FUSED])
@pytest.mark.parametrize("faces", [(CL, CL, CL, CL, PE, PE), (EX, CL, CL, EX, PE, PE)])
def test_closure_mixed_rhs(oracle, cuda, faces, path):
    shape = (40, 24, 10)
    f0 = wl.fourier_state(*shape, seed=25)
    ref = oracle.rhs_conserved(or_grid(*shape, face_kind=faces), f0)
    out = _rhs(ws.Grid(*shape, faces=faces, precision=ws.MIXED), f0, path)
    assert rel_l2(out, ref).max() <= 5e-5
    assert rel_linf(out, ref).max() <= 1e-4


@pytest.mark.parametrize("path", [None, FUSED])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_closure_batch_matches_solver(cuda, path, precision):
    # a batch mixing closure and periodic grids; each grid steps as alone
    prec = ws.MIXED if precision == "mixed" else ws.FP64
    shapes = [(24, 16, 8), (33, 12, 9), (20, 20, 6)]
    faces = [(CL, CL, PE, PE, PE, PE), (PE, PE, CL, CL, PE, PE), (PE,) * 6]
    grids = [ws.Grid(*s, faces=f, precision=prec) for s, f in zip(shapes, faces)]
    states = [wl.fourier_state(*s, seed=26 + i) for i, s in enumerate(shapes)]
    b = ws.Batch(grids)
    if path:
        b.set_tile(path)
    for i, f in enumerate(states):
        b.set_state(i, f)
    dts = b.compute_dt(0.5)
    b.set_dt(dts)
    b.step(3)
    for i, (g, f) in enumerate(zip(grids, states)):
        s = ws.Solver(g)
        if path:
            s.set_tile(path)
        s.set_state(f)
        s.step(dts[i], 3)
        a = s.get_state()
        s.close()
        tol = 1e-13 if prec == ws.FP64 else 1e-6
        assert rel_linf(b.get_state(i), a).max() <= tol, i
    b.close()


def test_closure_rejected_in_z_and_on_short_lines(cuda):
    with pytest.raises(ws.WsError):
        ws.Solver(ws.Grid(16, 16, 16, faces=(PE, PE, PE, PE, CL, CL)))
    with pytest.raises(ws.WsError):
        ws.Solver(ws.Grid(7, 16, 16, faces=(CL, CL, PE, PE, PE, PE)))
