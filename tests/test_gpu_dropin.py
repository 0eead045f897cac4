"""The drop-in C call sequence, driven through the C ABI with raw device
buffers as a reference time loop would: per stage cons_to_prim -> ghost fill
-> ws_du_invis_jacobian3d_init (sound speed on the padded job range) ->
ws_du_invis_jacobian3d -> ws_time_advance, against the oracle.

Tolerances: the sound speed is bit-exact (IEEE sqrt and division on both
sides, sqrt(T)/Ama as sound_speed_kernel, commen_kernel.cpp:145-154); the
time loop is held to rel. L-inf <= 1e-12 per field after 10 steps.
"""
import ctypes as C

import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import workloads as wl
from oracle.oracle import make_grid as or_grid
from tests.conftest import rel_linf

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _lap_odd_pitch(torch, g, fill=np.nan):
    """A LAP field whose pitch is odd (nx + 9 elements), so rows are not
    16-byte aligned."""
    pitch = g.nx + 9
    t = torch.full((g.nz + 8, g.ny + 8, pitch), fill, dtype=torch.float64, device="cuda")
    return t


def _init_case(oracle, torch, g, job, odd_pitch=False):
    og = or_grid(g.nx, g.ny, g.nz, gamma=g.gamma, ama=g.ama, face_kind=g.faces)
    rng = np.random.default_rng(21)
    T = rng.uniform(0.2, 3.0, size=(g.nz + 8, g.ny + 8, g.nx + 8))
    ref = oracle.sound_speed(og, T)            # whole padded field
    if odd_pitch:
        Td, cc = _lap_odd_pitch(torch, g, 0.0), _lap_odd_pitch(torch, g)
    else:
        Td, cc = ws.lap_tensor(g), ws.lap_tensor(g, fill=np.nan)
    Td[:, :, :g.nx + 8] = torch.from_numpy(T).cuda()
    ws.du_invis_jacobian3d_init(g, job, Td, cc)
    torch.cuda.synchronize()
    out = cc[:, :, :g.nx + 8].cpu().numpy()
    # the job's cells plus 4 ghost layers on every side (the reference's
    # du_invis_Jacobian3d_init range, OCFD_NS_Jacobian3d.cpp:24-33)
    xs, ys, zs = job.start.x - 4, job.start.y - 4, job.start.z - 4
    xe, ye, ze = job.end.x + 4, job.end.y + 4, job.end.z + 4
    inside = np.zeros(out.shape, dtype=bool)
    inside[zs:ze, ys:ye, xs:xe] = True
    return out, ref, inside


@pytest.mark.parametrize("ama", [1.0, 0.7])
def test_init_padded_range(oracle, cuda, ama):
    g = ws.Grid(29, 13, 11, ama=ama)
    out, ref, inside = _init_case(oracle, cuda, g, ws.interior_job(g))
    assert inside.all()
    assert np.array_equal(out, ref)


def test_init_subjob(oracle, cuda):
    g = ws.Grid(30, 20, 18)
    job = ws.WsJob(ws.WsDim3(7, 5, 9), ws.WsDim3(29, 21, 20))
    out, ref, inside = _init_case(oracle, cuda, g, job)
    assert np.array_equal(out[inside], ref[inside])
    assert np.all(np.isnan(out[~inside]))       # nothing written outside the range


def test_init_odd_pitch(oracle, cuda):
    g = ws.Grid(21, 9, 7)
    job = ws.WsJob(ws.WsDim3(5, 4, 6), ws.WsDim3(24, 13, 11))
    out, ref, inside = _init_case(oracle, cuda, g, job, odd_pitch=True)
    assert np.array_equal(out[inside], ref[inside])
    assert np.all(np.isnan(out[~inside]))


def test_init_empty_job_writes_nothing(oracle, cuda):
    g = ws.Grid(12, 8, 8)
    job = ws.WsJob(ws.WsDim3(6, 6, 6), ws.WsDim3(6, 12, 12))
    cc = ws.lap_tensor(g, fill=np.nan)
    ws.du_invis_jacobian3d_init(g, job, ws.lap_tensor(g, fill=1.0), cc)
    cuda.cuda.synchronize()
    assert bool(cuda.isnan(cc[:, :, :g.nx + 8]).all())


@pytest.mark.parametrize("tile", [None, (-1, 0, 0, 0), (16, 8, 0, 704)])
def test_rhs_empty_job_writes_nothing(cuda, tile):
    """A job with no cells in one direction returns WS_OK and launches
    nothing, on the line passes and the tile sweep alike."""
    g = ws.Grid(12, 8, 8)
    prims = [ws.lap_tensor(g, fill=1.0) for _ in range(5)]
    du = cuda.full((5, 4, 4, 4), np.nan, dtype=cuda.float64, device="cuda")
    for job in (ws.WsJob(ws.WsDim3(6, 6, 6), ws.WsDim3(6, 10, 10)),
                ws.WsJob(ws.WsDim3(6, 6, 6), ws.WsDim3(10, 6, 10)),
                ws.WsJob(ws.WsDim3(6, 6, 6), ws.WsDim3(10, 10, 6))):
        ws.du_invis_jacobian3d(g, job, *prims, du, tile=tile)
    cuda.cuda.synchronize()
    assert bool(cuda.isnan(du).all())


def _c_time_loop(torch, g, f0, dt, nsteps):
    """INTEGRATION's drop-in sequence through the C ABI, on one stream."""
    lib = ws.load()
    gc = g.c()
    gp = C.byref(gc)
    stream = torch.cuda.Stream()
    sh = C.c_void_p(stream.cuda_stream)
    job = ws.interior_job(g)
    f = torch.from_numpy(f0).cuda()
    fn, du = torch.empty_like(f), torch.empty_like(f)
    prims = [ws.lap_tensor(g) for _ in range(6)]      # d, u, v, w, T, P
    cc = ws.lap_tensor(g)
    pd = [ws.field_desc(t) for t in prims]
    fcc = ws.field_desc(cc)
    sf, sfn, sdu = ws.soa_desc(f), ws.soa_desc(fn), ws.soa_desc(du)
    gh = (ws.WsField * 5)(*pd[:5])
    check = ws._abi.check
    with torch.cuda.stream(stream):
        for _ in range(nsteps):
            fn.copy_(f)                                 # the solver's f -> fn copy
            for krk in (1, 2, 3):
                check(lib.ws_cons_to_prim(gp, sf, *pd, sh))
                check(lib.ws_ghost_fill(gp, gh, 5, sh))
                check(lib.ws_du_invis_jacobian3d_init(gp, job, pd[4], fcc, sh))
                check(lib.ws_du_invis_jacobian3d(gp, job, pd[0], pd[1], pd[2], pd[3], fcc,
                                                 None, sdu, sh))
                check(lib.ws_time_advance(gp, krk, C.c_double(dt), sf, sfn, sdu, sh))
        check(lib.ws_cons_to_prim(gp, sf, *pd, sh))
    stream.synchronize()
    flags = C.c_int()
    check(lib.ws_device_error(C.byref(flags), sh))
    return f.cpu().numpy(), [t[:, :, :g.nx + 8].cpu().numpy() for t in prims[:5]], flags.value


def test_c_sequence_config1_10_steps(oracle, cuda):
    """The 64x32x16 periodic configuration, 10 SSP-RK3 steps at CFL 0.5."""
    nx, ny, nz = 64, 32, 16
    g = ws.Grid(nx, ny, nz)
    og = or_grid(nx, ny, nz)
    f0 = wl.fourier_state(nx, ny, nz, seed=1)
    dt = oracle.compute_dt(og, f0, 0.5)
    out, prims, flags = _c_time_loop(cuda, g, f0, dt, 10)
    ref = oracle.rk3_steps(og, f0, dt, 10)
    assert flags == 0
    assert rel_linf(out, ref).max() <= TOL
    # the primitives the sequence leaves behind are those of the final state
    rp = oracle.cons_to_prim(og, ref)
    for a, b in zip(prims, rp[:5]):
        s = (slice(4, nz + 4), slice(4, ny + 4), slice(4, nx + 4))
        assert np.max(np.abs(a[s] - b[s])) <= TOL * np.max(np.abs(b[s]))


def test_c_sequence_extrap_x(oracle, cuda):
    """Same sequence on the headline face kinds (x extrapolation, y/z periodic)."""
    nx, ny, nz = 40, 16, 12
    faces = (ws.FACE_EXTRAP, ws.FACE_EXTRAP, 0, 0, 0, 0)
    g = ws.Grid(nx, ny, nz, faces=faces)
    og = or_grid(nx, ny, nz, face_kind=faces)
    f0 = wl.sod_state(nx, ny, nz, seed=2)
    dt = oracle.compute_dt(og, f0, 0.5)
    out, _, flags = _c_time_loop(cuda, g, f0, dt, 4)
    assert flags == 0
    assert rel_linf(out, oracle.rk3_steps(og, f0, dt, 4)).max() <= TOL


def test_get_state_async_matches_get_state(cuda):
    """ws_solver_get_state_async enqueues the download only: after the
    caller synchronises the stream, the pinned buffer holds the same state as
    ws_solver_get_state's; two solvers on two streams, stepped in turn with
    their downloads in flight, give the states they give alone."""
    shape = (40, 24, 16)
    g = ws.Grid(*shape, faces=(ws.FACE_EXTRAP, ws.FACE_EXTRAP, 0, 0, 0, 0))
    f0 = wl.sod_state(*shape, seed=43)
    lib = ws.load()
    ref = ws.Solver(g)
    ref.set_state(f0)
    dt = ref.compute_dt(0.5)
    ref.step(dt, 2)
    want = ref.get_state()
    ref.close()
    streams = [cuda.cuda.Stream(), cuda.cuda.Stream()]
    solvers = [ws.Solver(g), ws.Solver(g)]
    inp = cuda.from_numpy(np.ascontiguousarray(f0)).pin_memory()
    outs = [cuda.empty(f0.shape, dtype=cuda.float64).pin_memory() for _ in range(2)]
    try:
        for k in (0, 1):
            ws.check(lib.ws_solver_set_state(solvers[k].h, inp.numpy().ctypes.data,
                                             streams[k].cuda_stream))
            solvers[k].step(dt, 2, stream=streams[k])
            ws.check(lib.ws_solver_get_state_async(solvers[k].h, outs[k].numpy().ctypes.data,
                                                   streams[k].cuda_stream))
        for st in streams:
            st.synchronize()
        for k in (0, 1):
            assert np.array_equal(outs[k].numpy(), want)
        with pytest.raises(ws.WsError):
            ws.check(lib.ws_solver_get_state_async(solvers[0].h, None, None))
    finally:
        for s in solvers:
            s.close()
