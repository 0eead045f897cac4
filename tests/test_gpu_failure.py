"""Failure detection on the GPU without a fault: the fused RHS's bounded
staging wait.

Every wait of the kernels on their TMA copies is bounded; when one gives up
the CTA waits (again bounded) for its copies still in flight, sets status
bit 2 and stops.  The test makes the wait run out without anything being
wrong: with WS_TEST_STAGE_WAIT=n the first staging wait of each CTA polls,
n times, an mbarrier that nothing ever arrives on.  The tests check that the
host reads the failure (ws_device_error for the drop-in entry,
ws_solver_status -> WS_ERR_TIMEOUT for the stage kernel) and that the
context stays usable: the next launches are correct against the oracle.
"""
import ctypes as C

import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import workloads as wl
from oracle.oracle import make_grid as or_grid
from tests.conftest import rel_linf

pytestmark = pytest.mark.gpu
SHAPE = (64, 32, 16)
HOLD = "64"
# the fused kernel's tile shape: the waits are its TMA staging waits (the
# default FP64 path, the line passes, loads with plain global loads and has
# no wait to run out)
FUSED = (16, 8, 0, 704)


def _rhs_drop_in(s, g):
    """Ghost fill, then the drop-in entry on the solver's fields."""
    lib, gc = ws.load(), g.c()
    _, du, prims = s.fields()
    ws.check(lib.ws_ghost_fill(C.byref(gc), (ws.WsField * 6)(*prims), 6, None))
    ws.check(lib.ws_du_invis_jacobian3d_tiled(C.byref(gc), ws.interior_job(g), prims[0],
                                              prims[1], prims[2], prims[3], prims[5], None, du,
                                              ws.WsTile(*FUSED), None))


def test_drop_in_wait_timeout_reported(oracle, cuda, monkeypatch):
    g = ws.Grid(*SHAPE)
    f0 = wl.fourier_state(*SHAPE, seed=41)
    s = ws.Solver(g)
    s.set_state(f0)
    assert ws.device_error() in (0, 2)            # clear whatever an earlier test left
    monkeypatch.setenv("WS_TEST_STAGE_WAIT", HOLD)
    _rhs_drop_in(s, g)
    assert ws.device_error() == 2                 # reported, and cleared by the read
    assert ws.device_error() == 0
    monkeypatch.delenv("WS_TEST_STAGE_WAIT")
    _rhs_drop_in(s, g)                            # the context is still usable
    assert ws.device_error() == 0
    ref = oracle.rhs_conserved(or_grid(*SHAPE), f0)
    assert rel_linf(s.get_rhs(), ref).max() <= 1e-12
    s.close()


def test_stage_kernel_wait_timeout_reported(oracle, cuda, monkeypatch):
    g = ws.Grid(*SHAPE)
    f0 = wl.fourier_state(*SHAPE, seed=42)
    og = or_grid(*SHAPE)
    dt = oracle.compute_dt(og, f0, 0.5)
    s = ws.Solver(g)
    s.set_tile(FUSED)
    s.set_state(f0)
    monkeypatch.setenv("WS_TEST_STAGE_WAIT", HOLD)
    s.step(dt * 0.5, 1)                           # captured with the forced wait
    assert s.status() == 6                        # WS_ERR_TIMEOUT
    monkeypatch.delenv("WS_TEST_STAGE_WAIT")
    s.set_state(f0)                               # new state, new status word
    assert s.status() == 0
    s.step(dt, 2)                                 # new dt: recaptured without it
    assert s.status() == 0
    ref = oracle.rk3_steps(og, f0, dt, 2)
    assert rel_linf(s.get_state(), ref).max() <= 1e-12
    s.close()
