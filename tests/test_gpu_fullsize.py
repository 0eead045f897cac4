"""GPU parity at the benchmark's full sizes.

The benchmark's FP64 workload (Sod state along x, 1% noise, extrapolation in
x, periodic y and z) at 600x128x128 and 480x512x64, checked against the CPU
oracle on the same inputs, rel. L-inf per field <= 1e-12: one RHS through
the drop-in entry (ws_du_invis_jacobian3d) at both sizes, and two SSP-RK3
steps of the graph-captured solver (fused RHS + stage kernel) at
600x128x128, and the Navier-Stokes RHS (inviscid + viscous terms) of the
benchmark's viscous workload at 600x128x128.  Beside them, two size-independent properties on the GPU
alone at 600x128x128: a uniform state has a zero RHS, and on a fully
periodic grid the face differences telescope (sum of du = 0 to round-off).
The oracle takes a few seconds per RHS at these sizes on the host cores.
"""
import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import workloads as wl
from oracle.oracle import make_grid as or_grid
from tests.conftest import rel_linf
from tests.test_gpu_parity import _case

pytestmark = pytest.mark.gpu
TOL = 1e-12
SOD_FACES = (ws.FACE_EXTRAP, ws.FACE_EXTRAP, 0, 0, 0, 0)


@pytest.mark.parametrize("shape", [(600, 128, 128), (480, 512, 64)])
def test_full_size_rhs_matches_oracle(oracle, cuda, shape):
    g = ws.Grid(*shape, faces=SOD_FACES)
    out, ref = _case(oracle, cuda, g, wl.sod_state(*shape, seed=2))
    assert np.all(np.isfinite(out))
    assert rel_linf(out, ref).max() <= TOL


def test_full_size_steps_match_oracle(oracle, cuda):
    nx, ny, nz = 600, 128, 128
    g = ws.Grid(nx, ny, nz, faces=SOD_FACES)
    og = or_grid(nx, ny, nz, face_kind=SOD_FACES)
    f0 = wl.sod_state(nx, ny, nz, seed=2)
    dt = oracle.compute_dt(og, f0, 0.5)
    ref = oracle.rk3_steps(og, f0, dt, 2)
    s = ws.Solver(g)
    try:
        s.set_state(f0)
        assert abs(s.compute_dt(0.5) - dt) <= 1e-14 * dt
        s.step(dt, 2)
        assert s.status() == 0
        assert rel_linf(s.get_state(), ref).max() <= TOL
    finally:
        s.close()


def _gpu_rhs(g, f):
    s = ws.Solver(g)
    try:
        s.set_state(f)
        s.rhs()
        return s.get_rhs()
    finally:
        s.close()


def test_full_size_free_stream_and_conservation(cuda):
    nx, ny, nz = 600, 128, 128
    shp = (nz, ny, nx)
    d = np.full(shp, 1.3)
    f = wl.prim_to_cons(d, np.full(shp, 0.7), np.full(shp, -0.2), np.full(shp, 0.1),
                        np.full(shp, 0.9))
    du = _gpu_rhs(ws.Grid(nx, ny, nz, faces=SOD_FACES), f)
    assert np.max(np.abs(du)) <= 1e-12

    du = _gpu_rhs(ws.Grid(nx, ny, nz), wl.fourier_state(nx, ny, nz, seed=3))
    assert np.all(np.isfinite(du))
    for v in range(5):
        assert abs(np.sum(du[v])) <= 1e-12 * np.sum(np.abs(du[v]))


def test_full_size_navier_stokes_rhs_matches_oracle(oracle, cuda):
    """The benchmark's Navier-Stokes workload (Re 1e4, Pr 0.72, Sutherland
    Ref_T 288.15, CD8) at 600x128x128: inviscid + viscous RHS of the solver
    against the oracle's rhs_conserved_ns."""
    from oracle.oracle import make_vis
    nx, ny, nz = 600, 128, 128
    vis = dict(re=1e4, pr=0.72, ref_t=288.15, scheme=8)
    og = or_grid(nx, ny, nz, face_kind=SOD_FACES)
    f0 = wl.sod_state(nx, ny, nz, seed=2)
    ref = oracle.rhs_conserved_ns(og, make_vis(**vis), f0)
    s = ws.Solver(ws.Grid(nx, ny, nz, faces=SOD_FACES))
    try:
        s.set_viscous(vis)
        s.set_state(f0)
        s.rhs()
        assert rel_linf(s.get_rhs(), ref).max() <= TOL
    finally:
        s.close()
