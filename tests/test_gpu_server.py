"""Continuous-batching server: results are the same alone and in a mix of
uneven grids, precisions and step counts admitted while others run; HBM
budget admission; failures stay with their request."""
import time

import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import workloads as wl
from tests.conftest import rel_linf

pytestmark = pytest.mark.gpu


def _solo(grid, f0, nsteps):
    s = ws.Solver(grid)
    s.set_state(f0)
    dt = s.compute_dt(0.5)
    s.step(dt, nsteps)
    out = s.get_state()
    s.close()
    return out


def test_server_single_request_matches_solver(cuda):
    g = ws.Grid(40, 24, 16)
    f0 = wl.fourier_state(40, 24, 16, seed=3)
    srv = ws.Server()
    rid = srv.submit(g, 7, cfl=0.5, f0=f0)
    out = srv.wait(rid, timeout=60)
    srv.close()
    assert rel_linf(out, _solo(g, f0, 7)).max() <= 1e-13


@pytest.mark.parametrize("precision", [ws.FP64, ws.MIXED])
def test_server_same_alone_and_in_mix(cuda, precision):
    """The probe request gives the same result alone and when admitted into
    a running mix of other requests (different sizes, precisions, steps)."""
    probe_grid = ws.Grid(36, 20, 18, precision=precision)
    probe_f0 = wl.batch_state(wl.GridSpec(36, 20, 18, mach=1.2, x_jump=0.4, seed=9))
    srv = ws.Server()
    alone = srv.wait(srv.submit(probe_grid, 12, cfl=0.5, f0=probe_f0), timeout=120).copy()
    srv.close()

    srv = ws.Server()
    rng = np.random.default_rng(5)
    others = []
    for i in range(10):
        nx, ny, nz = int(rng.integers(16, 64)), int(rng.integers(8, 40)), int(rng.integers(8, 40))
        prec = ws.FP64 if i % 2 else ws.MIXED
        g = ws.Grid(nx, ny, nz, precision=prec)
        others.append(srv.submit(g, int(rng.integers(5, 30)), cfl=0.5, seed=100 + i,
                                 mach=float(rng.uniform(0.3, 3.0)),
                                 x_jump=float(rng.uniform(0.25, 0.75))))
        if i == 4:
            time.sleep(0.05)          # the probe joins while the first ones run
            rid = srv.submit(probe_grid, 12, cfl=0.5, f0=probe_f0)
    mixed = srv.wait(rid, timeout=120)
    for o in others:
        srv.wait(o, timeout=120)
    st = srv.stats()
    srv.close()
    assert st["completed"] == 11 and st["failed"] == 0
    assert st["max_active"] >= 2
    tol = 1e-13 if precision == ws.FP64 else 1e-6
    assert rel_linf(mixed, alone).max() <= tol


def test_server_budget_admission(cuda):
    g = ws.Grid(48, 32, 32)
    per = None
    srv0 = ws.Server()
    rid = srv0.submit(g, 2, cfl=0.5, seed=1)
    srv0.wait(rid, timeout=60)
    per = srv0.stats()["served_cell_rhs"]
    srv0.close()
    assert per > 0
    # a budget of ~1.5 states: requests run one at a time, all complete
    nbytes = 48 * 32 * 32 * 8 * 15 + 6 * 64 * 40 * 40 * 8 + 8192
    srv = ws.Server(hbm_budget_bytes=int(1.5 * nbytes) + 65536)
    ids = [srv.submit(g, 3, cfl=0.5, seed=i) for i in range(4)]
    for i in ids:
        srv.wait(i, timeout=60)
    st = srv.stats()
    assert st["completed"] == 4 and st["max_active"] == 1
    # a request that can never fit is refused at submission
    big = ws.Grid(256, 128, 128)
    with pytest.raises(ws.WsError) as e:
        srv.submit(big, 1, cfl=0.5)
    assert e.value.code == 7
    srv.close()


def test_server_failure_isolated(cuda):
    """A request with a non-physical initial state fails alone."""
    g = ws.Grid(24, 16, 12)
    good = wl.fourier_state(24, 16, 12, seed=4)
    bad = good.copy()
    bad[0, 3, 4, 5] = -1.0          # negative density
    srv = ws.Server()
    a = srv.submit(g, 4, dt=1e-4, f0=bad)
    b = srv.submit(g, 4, dt=1e-4, f0=good)
    with pytest.raises(ws.WsError) as e:
        srv.wait(a, timeout=60)
    assert e.value.code == 5
    out = srv.wait(b, timeout=60)
    assert np.all(np.isfinite(out))
    st = srv.stats()
    srv.close()
    assert st["failed"] == 1 and st["completed"] == 1
    assert st["p50_latency_s"] > 0


def test_server_synthetic_state_matches_host_generator(cuda):
    """The server's seeded device-side initial state equals the host
    generator workloads.synth_state (same counter-based hash)."""
    nx, ny, nz = 30, 12, 10
    g = ws.Grid(nx, ny, nz)
    srv = ws.Server()
    rid = srv.submit(g, 1, dt=1e-4, seed=77, mach=1.5, x_jump=0.45)
    out = srv.wait(rid, timeout=60)
    srv.close()
    f0 = wl.synth_state(nx, ny, nz, 77, 1.5, 0.45)
    s = ws.Solver(g)
    s.set_state(f0)
    s.step(1e-4, 1)
    ref = s.get_state()
    s.close()
    assert rel_linf(out, ref).max() <= 1e-13
