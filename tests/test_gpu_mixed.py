"""Mixed-precision form (FP32 split, smoothness indicators, weights and
candidates; FP64 state, face difference and SSP-RK3) against FP64.

Error measures are per conserved field: rel. L2 = ||a-b||_2 / ||b||_2 and
rel. L-inf = max|a-b| / max|b|.  Stated budget: rel. L2 <= 1e-6 of the state
after 100 steps on the 600x128x128 Fourier workload (the benchmark's mixed
configuration); one RHS evaluation within rel. L2 <= 5e-5, rel. L-inf <= 1e-4.

The Sod-type states with 1% cell noise are chaotic under WENO: the FP64
solution itself moves by ~10% in v, w after 100 steps when its initial state
is perturbed by 1e-12 (the FP64 oracle shows the same), so long-horizon mixed-vs-FP64
comparisons use the smooth Fourier workload; Sod is compared on one RHS.
"""
import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import workloads as wl
from oracle.oracle import make_grid as or_grid
from tests.conftest import rel_l2, rel_linf

pytestmark = pytest.mark.gpu


def _rhs(g, f0):
    s = ws.Solver(g)
    s.set_state(f0)
    s.rhs()
    out = s.get_rhs()
    s.close()
    return out


@pytest.mark.parametrize("case", ["fourier", "sod"])
def test_mixed_rhs_vs_fp64_oracle(oracle, cuda, case):
    nx, ny, nz = 64, 32, 16
    faces = (1, 1, 0, 0, 0, 0) if case == "sod" else (0,) * 6
    f0 = wl.fourier_state(nx, ny, nz, 1) if case == "fourier" else wl.sod_state(nx, ny, nz, 2)
    ref = oracle.rhs_conserved(or_grid(nx, ny, nz, face_kind=faces), f0)
    out = _rhs(ws.Grid(nx, ny, nz, faces=faces, precision=ws.MIXED), f0)
    assert np.all(np.isfinite(out))
    assert rel_l2(out, ref).max() <= 5e-5
    assert rel_linf(out, ref).max() <= 1e-4


def test_mixed_high_mach_finite(cuda):
    """Mach 3 periodic Sod jump: indicators large enough to overflow a
    product of four FP32 weights must stay finite."""
    spec = wl.GridSpec(48, 16, 16, mach=3.0, x_jump=0.4, seed=5)
    f0 = wl.batch_state(spec)
    g = ws.Grid(48, 16, 16, precision=ws.MIXED)
    out = _rhs(g, f0)
    ref = _rhs(ws.Grid(48, 16, 16), f0)
    assert np.all(np.isfinite(out))
    assert rel_l2(out, ref).max() <= 5e-5


def test_mixed_state_budget_config3(cuda):
    """600x128x128 Fourier workload, 100 SSP-RK3 steps at CFL 0.5:
    mixed vs FP64 rel. L2 <= 1e-6 per conserved field."""
    nx, ny, nz = 600, 128, 128
    f0 = wl.fourier_state(nx, ny, nz, seed=1)
    s64 = ws.Solver(ws.Grid(nx, ny, nz))
    s64.set_state(f0)
    dt = s64.compute_dt(0.5)
    s64.step(dt, 100)
    a = s64.get_state()
    s64.close()
    s32 = ws.Solver(ws.Grid(nx, ny, nz, precision=ws.MIXED))
    s32.set_state(f0)
    s32.step(dt, 100)
    b = s32.get_state()
    assert s32.status() == 0
    s32.close()
    err = rel_l2(b, a)
    assert err.max() <= 1e-6, err
