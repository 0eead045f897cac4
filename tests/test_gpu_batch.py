"""Batched solves of many uneven grids (one persistent RHS launch per RK stage
for all grids) against the one-grid path and the oracle."""
import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import workloads as wl
from oracle.oracle import make_grid as or_grid
from tests.conftest import rel_linf

pytestmark = pytest.mark.gpu
FUSED = (16, 8, 0, 704)      # the fused kernel's default tile (the default batch runs line passes)

SHAPES = [(33, 17, 16), (48, 20, 31), (16, 16, 16), (70, 9, 12), (25, 40, 5), (64, 32, 16)]


def _states(shapes, seed=0):
    out = []
    for i, (nx, ny, nz) in enumerate(shapes):
        spec = wl.GridSpec(nx, ny, nz, mach=0.3 + 0.4 * i, x_jump=0.3 + 0.07 * i, seed=seed + i)
        out.append(wl.batch_state(spec))
    return out


def test_batch_rhs_matches_oracle_and_single(oracle, cuda):
    grids = [ws.Grid(*s) for s in SHAPES]
    states = _states(SHAPES)
    b = ws.Batch(grids)
    for i, f in enumerate(states):
        b.set_state(i, f)
    b.rhs()
    for i, (g, f) in enumerate(zip(grids, states)):
        out = b.get_rhs(i)
        ref = oracle.rhs_conserved(or_grid(g.nx, g.ny, g.nz), f)
        assert rel_linf(out, ref).max() <= 1e-12, (i, SHAPES[i])
        s = ws.Solver(g)
        s.set_state(f)
        s.rhs()
        assert np.array_equal(s.get_rhs(), out), i
        s.close()
    b.close()


@pytest.mark.parametrize("precision", [ws.FP64, ws.MIXED])
def test_batch_steps_match_single(cuda, precision):
    shapes = SHAPES[:4]
    grids = [ws.Grid(*s, precision=precision) for s in shapes]
    states = _states(shapes, seed=10)
    b = ws.Batch(grids)
    for i, f in enumerate(states):
        b.set_state(i, f)
    dts = b.compute_dt(0.5)
    b.set_dt(dts)
    b.step(5)
    assert b.status() == [0] * len(grids)
    for i, (g, f) in enumerate(zip(grids, states)):
        s = ws.Solver(g)
        s.set_state(f)
        assert s.compute_dt(0.5) == dts[i]
        s.step(dts[i], 5)
        a = s.get_state()
        s.close()
        out = b.get_state(i)
        assert rel_linf(out, a).max() <= (1e-13 if precision == ws.FP64 else 1e-6), i
    b.close()


def test_batch_autotune_keeps_results(cuda):
    grids = [ws.Grid(*s) for s in SHAPES]
    states = _states(SHAPES, seed=20)
    b = ws.Batch(grids)
    for i, f in enumerate(states):
        b.set_state(i, f)
    b.rhs()
    before = [b.get_rhs(i) for i in range(len(grids))]
    tile = b.autotune()
    assert (tile[0], tile[1], tile[3]) in {(16, 8, 768), (16, 8, 704), (8, 8, 256), (8, 8, 384)}
    b.rhs()
    for i in range(len(grids)):
        assert np.array_equal(b.get_rhs(i), before[i])
    b.close()


def test_batch_nonfinite_status(cuda):
    """A bad initial state (negative density) is reported for that grid only."""
    shapes = SHAPES[:3]
    grids = [ws.Grid(*s) for s in shapes]
    states = _states(shapes, seed=30)
    states[1] = states[1].copy()
    states[1][0, 2, 3, 4] = -1.0
    b = ws.Batch(grids)
    for i, f in enumerate(states):
        b.set_state(i, f)
    assert b.status() == [0, 5, 0]
    b.close()


def test_batch_whole_column_runs_match_single(cuda):
    """The fused kernel's batch with every work item a whole tile column (the
    small batches above cut their columns into runs of 8 or more planes):
    the RHS equals the one-grid path bit for bit, two steps within 1e-13.
    (A step uses du as scratch, so the RHS is read before stepping.)"""
    shapes = [(128, 64, 40), (120, 56, 40), (96, 64, 33), (128, 50, 40)] * 2
    grids = [ws.Grid(*s) for s in shapes]
    states = _states(shapes, seed=20)
    b = ws.Batch(grids)
    b.set_tile(FUSED)
    for i, f in enumerate(states):
        b.set_state(i, f)
    b.rhs()
    rhs = [b.get_rhs(i) for i in range(len(grids))]
    dts = b.compute_dt(0.5)
    b.set_dt(dts)
    b.step(2)
    assert b.status() == [0] * len(grids)
    for i, (g, f) in enumerate(zip(grids, states)):
        s = ws.Solver(g)
        s.set_tile(FUSED)
        s.set_state(f)
        s.rhs()
        assert np.array_equal(s.get_rhs(), rhs[i]), i
        s.step(dts[i], 2)
        assert rel_linf(b.get_state(i), s.get_state()).max() <= 1e-13, i
        s.close()
    b.close()
