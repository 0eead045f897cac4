"""ws_compute_dt_static: the CFL time step for callers that cannot allocate
device memory (an arena-owning host code, a hard memory cap, or a loop that
cannot take the device-wide wait of cudaMalloc/cudaFree).  Its scratch is a
fixed array inside the library; it must agree with the allocating dt entry
points, and a second call must not see the first call's maxima.

This file is named to run last: if it fails, a run stopped at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import _abi
from windstencil_b200 import workloads as wl

pytestmark = pytest.mark.gpu

SHAPES = [(40, 24, 16), (33, 17, 20), (64, 32, 16)]
MACH = [2.5, 0.4, 1.2]          # distinct maxima so stale slots would show


def _static_dt(grids, fields, cfl, stream):
    n = len(grids)
    garr = (_abi.WsGrid * n)(*[g.c() for g in grids])
    farr = (_abi.WsField * (4 * n))(*[f for quad in fields for f in quad])
    out = (C.c_double * n)()
    _abi.check(ws.load().ws_compute_dt_static(garr, farr, n, cfl, out, stream))
    return np.array(out[:])


def test_dt_static_matches_allocating_entry_points(cuda):
    grids = [ws.Grid(*s) for s in SHAPES]
    states = [wl.batch_state(wl.GridSpec(*s, mach=m, x_jump=0.4, seed=i))
              for i, (s, m) in enumerate(zip(SHAPES, MACH))]
    solvers, quads, ref = [], [], []
    for g, f in zip(grids, states):
        s = ws.Solver(g)
        s.set_state(f)
        ref.append(s.compute_dt(0.5))                 # solver's allocated scratch
        _, _, p = s.fields()
        quads.append((p[1], p[2], p[3], p[5]))        # u, v, w, cc
        solvers.append(s)
    b = ws.Batch(grids)
    for i, f in enumerate(states):
        b.set_state(i, f)
    ref_batch = b.compute_dt(0.5)                     # cudaMallocAsync scratch
    b.close()
    assert np.array_equal(np.array(ref), ref_batch)

    stream = cuda.cuda.current_stream().cuda_stream
    first = _static_dt(grids, quads, 0.5, stream)
    assert np.allclose(first, ref, rtol=1e-15, atol=0)
    # second call, grids in another order: the shared array must have been
    # cleared, or slot 0 would keep the first call's larger maximum
    order = [1, 2, 0]
    second = _static_dt([grids[i] for i in order], [quads[i] for i in order], 0.5, stream)
    assert np.allclose(second, [ref[i] for i in order], rtol=1e-15, atol=0)
    for s in solvers:
        s.close()


def test_dt_static_full_table(cuda):
    """n = WS_DT_STATIC_MAX_GRIDS: every slot, the last included, is cleared,
    reduced and read back (one small grid's fields behind every slot)."""
    n = ws_max()
    g = ws.Grid(16, 8, 8)
    s = ws.Solver(g)
    s.set_state(wl.fourier_state(16, 8, 8, seed=3))
    ref = s.compute_dt(0.5)
    _, _, p = s.fields()
    stream = cuda.cuda.current_stream().cuda_stream
    out = _static_dt([g] * n, [(p[1], p[2], p[3], p[5])] * n, 0.5, stream)
    assert out.shape == (n,) and np.all(out == ref)
    s.close()


@pytest.mark.parametrize("kind", ["nan", "inf"])
def test_dt_static_nonfinite(cuda, kind):
    """A NaN or infinite wave speed in one cell of the second grid gives
    WS_ERR_NONFINITE naming that grid, not a dt."""
    shp = (24, 16, 12)
    f_ok = wl.fourier_state(*shp, seed=31)
    f_bad = f_ok.copy()
    f_bad[1, 5, 7, 11] = np.nan if kind == "nan" else np.inf
    solvers, quads = [], []
    for f in (f_ok, f_bad):
        s = ws.Solver(ws.Grid(*shp))
        s.set_state(f)
        _, _, p = s.fields()
        quads.append((p[1], p[2], p[3], p[5]))
        solvers.append(s)
    stream = cuda.cuda.current_stream().cuda_stream
    with pytest.raises(ws.WsError) as e:
        _static_dt([ws.Grid(*shp)] * 2, quads, 0.5, stream)
    assert e.value.code == 5 and "grid 1" in str(e.value)
    for s in solvers:
        s.close()


def test_dt_static_rejects_too_many_grids(cuda):
    g = ws.Grid(8, 8, 8).c()
    f = _abi.WsField(0x10000, 32, 0)
    garr = (_abi.WsGrid * 1)(g)
    farr = (_abi.WsField * 4)(f, f, f, f)
    out = (C.c_double * 1)()
    rc = ws.load().ws_compute_dt_static(garr, farr, ws_max() + 1, 0.5, out, None)
    assert rc == 1 and "4096" in ws.last_error()


def ws_max():
    import re
    txt = open(_abi.HEADER).read()
    return int(re.search(r"#define WS_DT_STATIC_MAX_GRIDS (\d+)", txt).group(1))
