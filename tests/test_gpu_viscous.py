"""Viscous terms (Navier-Stokes) on the GPU against the oracle.

The oracle's viscous restatement is pinned bit for bit to the reference's own
vis_flux_ker / get_Amu_kernal / CD6 / CD8 / YF_Pe_XF (tests/test_oracle_pin.py).
FP64 tolerance as elsewhere: rel. L-inf per field <= 1e-12.
"""
import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import workloads as wl
from oracle.oracle import make_grid as or_grid, make_vis
from tests.conftest import rel_linf
from tests.test_gpu_parity import oracle_prims, to_lap

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _vis(scheme):
    return dict(re=400.0, pr=0.72, ref_t=260.0, scheme=scheme)


@pytest.mark.parametrize("scheme", [6, 8])
@pytest.mark.parametrize("faces", [(0, 0, 0, 0, 0, 0), (1, 1, 0, 0, 1, 1), (2, 2, 2, 2, 0, 0)])
def test_du_vis_drop_in(oracle, cuda, scheme, faces):
    nx, ny, nz = 24, 14, 10
    g = ws.Grid(nx, ny, nz, faces=faces)
    og = or_grid(nx, ny, nz, face_kind=faces)
    d, u, v, w, T, cc = oracle_prims(oracle, og, wl.fourier_state(nx, ny, nz, seed=31))
    base = np.random.default_rng(32).normal(size=(5, nz, ny, nx))
    ref = oracle.du_vis(og, make_vis(**_vis(scheme)), u, v, w, T, du=base.copy())
    du = cuda.from_numpy(base.copy()).cuda()
    ws.du_vis_jacobian3d(g, _vis(scheme), *(to_lap(cuda, g, a) for a in (u, v, w, T)), du)
    cuda.cuda.synchronize()
    assert rel_linf(du.cpu().numpy(), ref).max() <= TOL


def test_du_vis_general_metrics(oracle, cuda):
    nx, ny, nz = 18, 12, 9
    g = ws.Grid(nx, ny, nz, metrics_uniform=False)
    og = or_grid(nx, ny, nz)
    d, u, v, w, T, cc = oracle_prims(oracle, og, wl.fourier_state(nx, ny, nz, seed=33))
    rng = np.random.default_rng(34)
    shp = d.shape
    metrics = [rng.uniform(0.6, 1.4, shp) if i % 4 == 0 else rng.uniform(-0.3, 0.3, shp)
               for i in range(9)]
    ajac = rng.uniform(0.8, 1.2, shp)
    ref = oracle.du_vis(og, make_vis(**_vis(8)), u, v, w, T, metrics, ajac)
    du = cuda.zeros((5, nz, ny, nx), dtype=cuda.float64, device="cuda")
    mdev = [to_lap(cuda, g, a) for a in metrics + [ajac]]
    ws.du_vis_jacobian3d(g, _vis(8), *(to_lap(cuda, g, a) for a in (u, v, w, T)), du,
                         metrics=mdev)
    cuda.cuda.synchronize()
    assert rel_linf(du.cpu().numpy(), ref).max() <= TOL


@pytest.mark.parametrize("faces", [(0, 0, 0, 0, 0, 0), (1, 1, 0, 0, 0, 0)])
def test_ns_solver_rhs_and_steps(oracle, cuda, faces):
    nx, ny, nz = 32, 16, 12
    og = or_grid(nx, ny, nz, face_kind=faces)
    vis = make_vis(**_vis(8))
    f0 = wl.fourier_state(nx, ny, nz, seed=35)
    s = ws.Solver(ws.Grid(nx, ny, nz, faces=faces))
    s.set_viscous(_vis(8))
    s.set_state(f0)
    s.rhs()
    ref_du = oracle.rhs_conserved_ns(og, vis, f0)
    assert rel_linf(s.get_rhs(), ref_du).max() <= TOL
    dt = oracle.compute_dt(og, f0, 0.4)
    ref = oracle.rk3_steps_ns(og, vis, f0, dt, 5)
    s.step(dt, 5)
    out = s.get_state()
    assert s.status() == 0
    s.close()
    assert rel_linf(out, ref).max() <= TOL


def test_ns_solver_back_to_euler(oracle, cuda):
    nx, ny, nz = 16, 12, 8
    f0 = wl.fourier_state(nx, ny, nz, seed=36)
    s = ws.Solver(ws.Grid(nx, ny, nz))
    s.set_viscous(_vis(6))
    s.set_viscous(None)
    s.set_state(f0)
    s.rhs()
    ref = oracle.rhs_conserved(or_grid(nx, ny, nz), f0)
    assert rel_linf(s.get_rhs(), ref).max() <= TOL
    s.close()


def test_viscous_rejects_bad_input(cuda):
    g = ws.Grid(16, 12, 8)
    s = ws.Solver(g)
    with pytest.raises(ws.WsError):
        s.set_viscous(dict(re=100.0, pr=0.7, ref_t=288.0, scheme=4))
    with pytest.raises(ws.WsError):
        s.set_viscous(dict(re=-1.0, pr=0.7, ref_t=288.0, scheme=8))
    s.close()
    f = [ws.lap_tensor(g) for _ in range(4)]
    du = cuda.zeros((5, 8, 12, 16), dtype=cuda.float64, device="cuda")
    small = cuda.empty(16, dtype=cuda.float64, device="cuda")
    with pytest.raises(ws.WsError):
        ws.du_vis_jacobian3d(g, _vis(8), *f, du, workspace=small)


@pytest.mark.parametrize("scheme", [6, 8])
@pytest.mark.parametrize("faces,d0b", [((1, 1, 0, 0, 1, 1), (1, 1, 0, 0, 0, 0)),
                                       ((1, 1, 1, 1, 0, 0), (1, 1, 1, 1, 1, 1)),
                                       ((1, 1, 0, 0, 1, 1), (0, 1, 1, 0, 1, 0))])
def test_du_vis_dif_bound(oracle, cuda, scheme, faces, d0b):
    """DIF_BOUND: the reference's reduced derivative forms in the four cells
    next to flagged faces (gradients and flux divergence), against the oracle
    (pinned to the reference's OCFD_D0bound_scheme_kernel), general metrics in
    the last case."""
    nx, ny, nz = 22, 13, 11
    general = d0b == (0, 1, 1, 0, 1, 0)
    g = ws.Grid(nx, ny, nz, faces=faces, metrics_uniform=not general)
    og = or_grid(nx, ny, nz, face_kind=faces)
    d, u, v, w, T, cc = oracle_prims(oracle, og, wl.fourier_state(nx, ny, nz, seed=37))
    metrics = ajac = mdev = None
    if general:
        rng = np.random.default_rng(38)
        shp = d.shape
        metrics = [rng.uniform(0.6, 1.4, shp) if i % 4 == 0 else rng.uniform(-0.3, 0.3, shp)
                   for i in range(9)]
        ajac = rng.uniform(0.8, 1.2, shp)
        mdev = [to_lap(cuda, g, a) for a in metrics + [ajac]]
    vis = dict(_vis(scheme), d0_bound=d0b)
    base = np.random.default_rng(39).normal(size=(5, nz, ny, nx))
    ref = oracle.du_vis(og, make_vis(**vis), u, v, w, T, metrics, ajac, du=base.copy())
    plain = oracle.du_vis(og, make_vis(**_vis(scheme)), u, v, w, T, metrics, ajac,
                          du=base.copy())
    assert not np.array_equal(ref, plain)         # the flags change the boundary cells
    du = cuda.from_numpy(base.copy()).cuda()
    ws.du_vis_jacobian3d(g, vis, *(to_lap(cuda, g, a) for a in (u, v, w, T)), du, metrics=mdev)
    cuda.cuda.synchronize()
    assert rel_linf(du.cpu().numpy(), ref).max() <= TOL


def test_ns_solver_dif_bound_steps(oracle, cuda):
    """The solver with DIF_BOUND on the x faces: RHS and 3 steps against the
    oracle."""
    nx, ny, nz = 28, 14, 10
    faces = (1, 1, 0, 0, 0, 0)
    vis = dict(_vis(8), d0_bound=(1, 1, 0, 0, 0, 0))
    og = or_grid(nx, ny, nz, face_kind=faces)
    f0 = wl.fourier_state(nx, ny, nz, seed=40)
    s = ws.Solver(ws.Grid(nx, ny, nz, faces=faces))
    s.set_viscous(vis)
    s.set_state(f0)
    s.rhs()
    assert rel_linf(s.get_rhs(), oracle.rhs_conserved_ns(og, make_vis(**vis), f0)).max() <= TOL
    dt = oracle.compute_dt(og, f0, 0.4)
    s.step(dt, 3)
    ref = oracle.rk3_steps_ns(og, make_vis(**vis), f0, dt, 3)
    assert rel_linf(s.get_state(), ref).max() <= TOL
    s.close()
