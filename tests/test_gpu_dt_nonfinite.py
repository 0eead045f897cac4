"""The CFL time step refuses a state with a NaN or infinite wave speed.

The wave-speed maximum is reduced on the device as the bit patterns of
non-negative doubles; a NaN cell must not drop out of the maximum (as it
would through fmax) and an infinite one must not come back as a valid
maximum (dt = cfl/inf = 0).  Both end in WS_ERR_NONFINITE on the solver's
and the batch's dt entry points.
"""
import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import workloads as wl

pytestmark = pytest.mark.gpu
SHAPE = (24, 16, 12)


def poisoned(kind, cell=(5, 7, 11)):
    """A smooth state with one bad momentum value: NaN, or +inf."""
    f = wl.fourier_state(*SHAPE, seed=31)
    k, j, i = cell
    f[1, k, j, i] = np.nan if kind == "nan" else np.inf
    return f


@pytest.mark.parametrize("kind", ["nan", "inf"])
def test_solver_dt_nonfinite(cuda, kind):
    s = ws.Solver(ws.Grid(*SHAPE))
    try:
        s.set_state(poisoned(kind))
        with pytest.raises(ws.WsError) as e:
            s.compute_dt(0.5)
        assert e.value.code == 5                      # WS_ERR_NONFINITE
        s.set_state(wl.fourier_state(*SHAPE, seed=31))
        assert np.isfinite(s.compute_dt(0.5)) and s.compute_dt(0.5) > 0
    finally:
        s.close()


@pytest.mark.parametrize("kind", ["nan", "inf"])
def test_batch_dt_nonfinite(cuda, kind):
    b = ws.Batch([ws.Grid(*SHAPE), ws.Grid(*SHAPE)])
    try:
        b.set_state(0, wl.fourier_state(*SHAPE, seed=31))
        b.set_state(1, poisoned(kind))
        with pytest.raises(ws.WsError) as e:
            b.compute_dt(0.5)
        assert e.value.code == 5 and "grid 1" in str(e.value)
    finally:
        b.close()
