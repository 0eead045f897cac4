"""GPU parity of the CUDA path (through the C ABI) against the CPU oracle.

Tolerance: FP64 path, rel. L-inf per field <= 1e-12 (the target the port is
held to; the two differ only by FMA contraction and summation order).  The
mixed form is checked against its stated error budget in test_gpu_mixed.py.
"""
import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import workloads as wl
from oracle.oracle import make_grid as or_grid
from tests.conftest import rel_linf

pytestmark = pytest.mark.gpu
TOL = 1e-12


def to_lap(torch, g, a):
    """numpy (nz+8, ny+8, nx+8) -> pitched device LAP tensor."""
    t = ws.lap_tensor(g)
    t[:, :, :g.nx + 8] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t


def oracle_prims(oracle, og, f):
    d, u, v, w, T, _ = oracle.cons_to_prim(og, f)
    for a in (d, u, v, w, T):
        oracle.ghost_fill(og, a)
    cc = oracle.sound_speed(og, T)
    return d, u, v, w, T, cc


def _case(oracle, torch, g, f, metrics=None, ajac=None, tile=None, job=None, lap=None):
    og = or_grid(g.nx, g.ny, g.nz, g.hx, g.hy, g.hz, g.gamma, g.ama, g.epsl_sw, g.faces)
    d, u, v, w, T, cc = oracle_prims(oracle, og, f)
    ref = oracle.du_invis(og, d, u, v, w, cc, metrics, ajac)
    dev = [(lap or to_lap)(torch, g, a) for a in (d, u, v, w, cc)]
    mdev = None
    if metrics is not None:
        mdev = [to_lap(torch, g, a) for a in list(metrics) + [ajac]]
    job = job or ws.interior_job(g)
    ex = job.end.x - job.start.x
    ey = job.end.y - job.start.y
    ez = job.end.z - job.start.z
    du = torch.full((5, ez, ey, ex), np.nan, dtype=torch.float64, device="cuda")
    ws.du_invis_jacobian3d(g, job, *dev, du, metrics=mdev, tile=tile)
    torch.cuda.synchronize()
    sx, sy, sz = job.start.x - 4, job.start.y - 4, job.start.z - 4
    ref = ref[:, sz:sz + ez, sy:sy + ey, sx:sx + ex]
    return du.cpu().numpy(), ref


@pytest.mark.parametrize("shape", [(64, 32, 16), (17, 9, 6), (40, 24, 37), (5, 4, 4)])
def test_rhs_fp64_periodic(oracle, cuda, shape):
    g = ws.Grid(*shape)
    out, ref = _case(oracle, cuda, g, wl.fourier_state(*shape, seed=3))
    assert np.all(np.isfinite(out))
    assert rel_linf(out, ref).max() <= TOL


def test_rhs_fp64_extrap_x(oracle, cuda):
    g = ws.Grid(48, 20, 12, faces=(ws.FACE_EXTRAP, ws.FACE_EXTRAP, 0, 0, 0, 0))
    out, ref = _case(oracle, cuda, g, wl.sod_state(48, 20, 12, seed=5))
    assert rel_linf(out, ref).max() <= TOL


def test_rhs_fp64_all_extrap(oracle, cuda):
    g = ws.Grid(21, 14, 11, faces=(ws.FACE_EXTRAP,) * 6)
    out, ref = _case(oracle, cuda, g, wl.sod_state(21, 14, 11, seed=6))
    assert rel_linf(out, ref).max() <= TOL


def test_rhs_fp64_general_metrics(oracle, cuda):
    g = ws.Grid(33, 18, 10, metrics_uniform=False)
    rng = np.random.default_rng(7)
    shp = (10 + 8, 18 + 8, 33 + 8)
    metrics = [rng.uniform(0.6, 1.4, shp) if i % 4 == 0 else rng.uniform(-0.3, 0.3, shp)
               for i in range(9)]
    ajac = rng.uniform(0.8, 1.2, shp)
    out, ref = _case(oracle, cuda, g, wl.fourier_state(33, 18, 10, seed=8), metrics, ajac)
    assert rel_linf(out, ref).max() <= TOL


@pytest.mark.parametrize("tile", [(16, 8, 1, 768), (16, 8, 5, 704), (16, 8, 32, 768),
                                  (16, 8, 0, 704), (16, 8, 3, 768), (8, 8, 0, 256),
                                  (8, 8, 7, 384), (8, 8, 0, 384)])
def test_rhs_tiles_and_scans(oracle, cuda, tile):
    g = ws.Grid(37, 19, 23)
    out, ref = _case(oracle, cuda, g, wl.fourier_state(37, 19, 23, seed=9), tile=tile)
    assert rel_linf(out, ref).max() <= TOL


def test_rhs_subjob(oracle, cuda):
    g = ws.Grid(30, 20, 18)
    job = ws.WsJob(ws.WsDim3(7, 5, 9), ws.WsDim3(29, 21, 20))
    out, ref = _case(oracle, cuda, g, wl.fourier_state(30, 20, 18, seed=10), job=job)
    assert rel_linf(out, ref).max() <= TOL


def test_ghost_fill_exact(oracle, cuda):
    for faces in [(0,) * 6, (1, 1, 0, 0, 1, 0), (1,) * 6]:
        g = ws.Grid(19, 7, 5, faces=faces)
        og = or_grid(19, 7, 5, face_kind=faces)
        rng = np.random.default_rng(11)
        a = rng.normal(size=(5 + 8, 7 + 8, 19 + 8))
        t = to_lap(cuda, g, a)
        ws.ghost_fill(g, [t])
        oracle.ghost_fill(og, a)
        assert np.array_equal(t[:, :, :27].cpu().numpy(), a)


def test_prim_cons_roundtrip(oracle, cuda):
    g = ws.Grid(23, 11, 9)
    og = or_grid(23, 11, 9)
    f = wl.fourier_state(23, 11, 9, seed=12)
    fdev = cuda.from_numpy(f).cuda()
    prims = [ws.lap_tensor(g) for _ in range(6)]
    ws.cons_to_prim(g, fdev, *prims)
    ref = oracle.cons_to_prim(og, f)
    cuda.cuda.synchronize()
    for a, b in zip(prims, ref):
        av = a[4:-4, 4:-4, 4:27].cpu().numpy()
        bv = b[4:-4, 4:-4, 4:27]
        assert np.max(np.abs(av - bv)) <= 1e-14 * max(1.0, np.max(np.abs(bv)))
    f2 = ws.soa_tensor(g)
    ws.prim_to_cons(g, *prims[:5], f2)
    assert rel_linf(f2.cpu().numpy(), f).max() <= 1e-14


@pytest.mark.parametrize("krk", [1, 2, 3])
def test_time_advance(oracle, cuda, krk):
    g = ws.Grid(16, 8, 6)
    rng = np.random.default_rng(20 + krk)
    f, fn, du = (rng.normal(size=(5, 6, 8, 16)) for _ in range(3))
    tf, tfn, tdu = (cuda.from_numpy(x).cuda() for x in (f, fn, du))
    ws.time_advance(g, krk, 2.5e-3, tf, tfn, tdu)
    oracle.time_advance(krk, 2.5e-3, f, fn, du)
    assert rel_linf(tf.cpu().numpy(), f).max() <= 1e-15


def test_solver_config1_10_steps(oracle, cuda):
    """Plain FP64 3D Euler, 64x32x16 periodic, Fourier state with a contact,
    SSP-RK3 at CFL 0.5, 10 steps: rel. L-inf <= 1e-12 per conserved field."""
    nx, ny, nz = 64, 32, 16
    g = ws.Grid(nx, ny, nz)
    og = or_grid(nx, ny, nz)
    f0 = wl.fourier_state(nx, ny, nz, seed=1)
    dt = oracle.compute_dt(og, f0, 0.5)
    ref = oracle.rk3_steps(og, f0, dt, 10)
    s = ws.Solver(g)
    s.set_state(f0)
    dt_gpu = s.compute_dt(0.5)
    assert abs(dt_gpu - dt) <= 1e-14 * dt
    s.step(dt, 10)
    out = s.get_state()
    assert s.status() == 0
    err = rel_linf(out, ref)
    assert err.max() <= TOL, err


def test_solver_extrap_sod(oracle, cuda):
    nx, ny, nz = 60, 16, 8
    faces = (1, 1, 0, 0, 0, 0)
    g = ws.Grid(nx, ny, nz, faces=faces)
    og = or_grid(nx, ny, nz, face_kind=faces)
    f0 = wl.sod_state(nx, ny, nz, seed=2)
    dt = oracle.compute_dt(og, f0, 0.5)
    ref = oracle.rk3_steps(og, f0, dt, 5)
    s = ws.Solver(g)
    s.set_state(f0)
    s.step(dt, 5)
    assert rel_linf(s.get_state(), ref).max() <= TOL


def test_solver_rhs_matches_oracle(oracle, cuda):
    nx, ny, nz = 40, 16, 12
    g = ws.Grid(nx, ny, nz)
    og = or_grid(nx, ny, nz)
    f0 = wl.fourier_state(nx, ny, nz, seed=4)
    s = ws.Solver(g)
    s.set_state(f0)
    s.rhs()
    out = s.get_rhs()
    ref = oracle.rhs_conserved(og, f0)
    assert rel_linf(out, ref).max() <= TOL


def test_rhs_subjob_even_start(oracle, cuda):
    # even job start in x: the primitive planes are staged with TMA tiles
    g = ws.Grid(30, 20, 18)
    job = ws.WsJob(ws.WsDim3(6, 5, 9), ws.WsDim3(29, 21, 20))
    out, ref = _case(oracle, cuda, g, wl.fourier_state(30, 20, 18, seed=11), job=job)
    assert rel_linf(out, ref).max() <= TOL


@pytest.mark.parametrize("layout", ["odd_pitch", "offset_8_bytes"])
def test_rhs_fields_tma_cannot_stage(oracle, cuda, layout):
    # fields whose rows or base break the 16-byte rule of TMA tiles: the
    # kernel stages them with cp.async instead, with the same results
    g = ws.Grid(30, 14, 12)

    def lap(torch, g, a):
        if layout == "odd_pitch":      # rows of 39 doubles
            t = torch.zeros((g.nz + 8, g.ny + 8, g.nx + 9), dtype=torch.float64, device="cuda")
        else:                          # rows of 40 doubles, base 8 bytes past 16-byte alignment
            t = torch.zeros((g.nz + 8, g.ny + 8, g.nx + 10), dtype=torch.float64,
                            device="cuda")[:, :, 1:g.nx + 9]
        t[:, :, :g.nx + 8] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        return t
    out, ref = _case(oracle, cuda, g, wl.fourier_state(30, 14, 12, seed=12), lap=lap)
    assert rel_linf(out, ref).max() <= TOL
