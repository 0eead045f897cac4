"""x slabs on the GPU: the halo pack / unpack kernels, the ghost fill of
EXTERNAL faces, the per-stage solver entry points, and whole SSP-RK3 runs of
a grid split into slabs (all slabs on this GPU, halos passed between them in
process) against the same grid stepped whole.

A slab's cells see exactly the values the whole grid's cells see (the halo
carries the neighbour's d, u, v, w, T, cc), so the split run must agree with
the whole-grid run bit for bit wherever both use the same compiled kernel;
the oracle bounds both at rel. L-inf 1e-12 per field.
"""
import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import halo
from windstencil_b200 import workloads as wl
from oracle.oracle import make_grid as or_grid
from tests.conftest import rel_linf

pytestmark = pytest.mark.gpu
PE, EX, CL, XT = ws.FACE_PERIODIC, ws.FACE_EXTRAP, ws.FACE_CLOSURE, ws.FACE_EXTERNAL


def _rand_fields(torch, g, n, seed):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    t = ws.lap_tensor(g, n)
    t.copy_(torch.rand(t.shape, generator=gen, device="cuda", dtype=torch.float64))
    return [t[i] for i in range(n)]


@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("nf", [1, 6])
@pytest.mark.parametrize("shape", [(19, 13, 7), (40, 24, 10)])
def test_halo_pack_unpack(cuda, nf, shape, axis):
    torch = cuda
    faces = [PE] * 6
    faces[2 * axis] = faces[2 * axis + 1] = XT
    g = ws.Grid(*shape, faces=tuple(faces))
    n = list(shape)
    fields = _rand_fields(torch, g, nf, 5)
    nb = ws.halo_bytes(g, axis, nf) // 8
    box = [n[0], n[1], n[2]]
    box[axis] = 4
    assert nb == nf * box[0] * box[1] * box[2]
    if axis == 0:
        assert ws.halo_x_bytes(g, nf) // 8 == nb

    def planes(f, a0):         # (z, y, x) slices: 4 planes along axis from a0
        sl = [slice(a0, a0 + 4) if d == axis else slice(4, n[d] + 4) for d in range(3)]
        return f[sl[2], sl[1], sl[0]]
    for side, a0 in ((0, 4), (1, n[axis])):
        buf = torch.full((nb,), -1.0, dtype=torch.float64, device="cuda")
        ws.halo_pack(g, fields, axis, side, buf)
        want = torch.stack([planes(f, a0) for f in fields]).reshape(-1)
        assert torch.equal(buf, want)
    for side, a0 in ((0, 0), (1, n[axis] + 4)):
        before = [f.clone() for f in fields]
        buf = torch.rand(nb, dtype=torch.float64, device="cuda")
        ws.halo_unpack(g, fields, axis, side, buf)
        b = buf.reshape(nf, box[2], box[1], box[0])
        for q, f in enumerate(fields):
            assert torch.equal(planes(f, a0), b[q])
            mask = torch.ones_like(f, dtype=torch.bool)
            sl = [slice(a0, a0 + 4) if d == axis else slice(4, n[d] + 4) for d in range(3)]
            mask[sl[2], sl[1], sl[0]] = False
            assert torch.equal(f[mask], before[q][mask])      # nothing else written
    torch.cuda.synchronize()


@pytest.mark.parametrize("faces", [(XT, XT, PE, EX, PE, PE), (EX, XT, EX, EX, PE, EX),
                                   (XT, CL, CL, CL, PE, PE), (PE, PE, XT, XT, EX, XT),
                                   (XT, XT, XT, XT, XT, XT)])
def test_ghost_fill_external(oracle, cuda, faces):
    """EXTERNAL ghosts over the interior of the other axes are kept; every
    other ghost as the oracle's fill (edges from the kept planes)."""
    torch = cuda
    shape = (21, 11, 9)
    nx, ny, nz = shape
    g = ws.Grid(*shape, faces=faces)
    (f,) = _rand_fields(torch, g, 1, 9)
    host = f[:, :, :nx + 8].cpu().numpy().copy()
    ws.ghost_fill(g, [f])
    oracle.ghost_fill(or_grid(*shape, face_kind=faces), host)
    got = f[:, :, :nx + 8].cpu().numpy()
    assert np.array_equal(got, host)


def _run_whole(g, f0, dt, nsteps):
    s = ws.Solver(g)
    s.set_state(f0)
    s.step(dt, nsteps)
    out = s.get_state()
    assert s.status() == 0
    s.close()
    return out


def test_stages_equal_step(cuda):
    g = ws.Grid(33, 20, 12, faces=(EX, EX, PE, PE, PE, PE))
    f0 = wl.sod_state(g.nx, g.ny, g.nz, seed=31)
    s = ws.Solver(g)
    s.set_state(f0)
    dt = s.compute_dt(0.5)
    assert [p.ptr for p in s.stage_fields(1)] == [p.ptr for p in s.fields()[2]]
    for _ in range(2):
        for krk in (1, 2, 3):
            s.stage(krk, dt)
    staged = s.get_state()
    s.close()
    assert np.array_equal(staged, _run_whole(g, f0, dt, 2))


def test_stage_rules(cuda):
    g = ws.Grid(16, 16, 16, faces=(XT, EX, PE, PE, PE, PE))
    s = ws.Solver(g)
    s.set_state(wl.fourier_state(16, 16, 16, seed=2))
    with pytest.raises(ws.WsError, match="WS_ERR_INVALID"):
        s.stage(2, 1e-4)                                   # stage 1 is due
    with pytest.raises(ws.WsError, match="WS_ERR_UNSUPPORTED"):
        s.step(1e-4, 1)                                    # EXTERNAL: staged only
    s.stage(1, 1e-4)
    s.set_state(wl.fourier_state(16, 16, 16, seed=2))      # a new state restarts at 1
    s.stage(1, 1e-4)
    s.close()
    with pytest.raises(ws.WsError, match="WS_ERR_UNSUPPORTED"):
        ws.Batch([g])


def test_stage_halves_rules(cuda):
    g = ws.Grid(16, 16, 16, faces=(XT, EX, PE, PE, PE, PE))
    s = ws.Solver(g)
    s.set_state(wl.fourier_state(16, 16, 16, seed=2))
    with pytest.raises(ws.WsError, match="WS_ERR_INVALID"):
        s.stage_flux_fields()                              # no viscous terms
    with pytest.raises(ws.WsError, match="WS_ERR_INVALID"):
        s.stage_end(1, 1e-4)                               # end without begin
    s.set_viscous(ws.viscous())
    assert len(s.stage_flux_fields()) == 4
    assert [f.ptr for f in s.stage_flux_fields(2)] != [f.ptr for f in s.stage_flux_fields(0)]
    with pytest.raises(ws.WsError, match="WS_ERR_UNSUPPORTED"):
        s.stage(1, 1e-4)                                   # the flux halo is needed
    with pytest.raises(ws.WsError, match="WS_ERR_UNSUPPORTED"):
        s.rhs()
    s.stage_begin(1)
    with pytest.raises(ws.WsError, match="WS_ERR_INVALID"):
        s.stage_begin(1)                                   # already begun
    s.stage_end(1, 1e-4)
    s.stage_begin(2)
    s.stage_end(2, 1e-4)
    s.close()


CASES = [
    ("periodic_2", (64, 24, 12), (PE,) * 6, 2, ws.FP64),
    ("periodic_3_ragged", (70, 20, 10), (PE,) * 6, 3, ws.FP64),
    ("extrap_4", (96, 16, 12), (EX, EX, PE, PE, PE, PE), 4, ws.FP64),
    ("closure_2", (64, 24, 10), (CL, CL, CL, CL, PE, PE), 2, ws.FP64),
    ("mixed_periodic_2", (64, 24, 12), (PE,) * 6, 2, ws.MIXED),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_slabs_match_whole_grid(oracle, cuda, case):
    _, shape, faces, parts, prec = case
    g = ws.Grid(*shape, faces=faces, precision=prec)
    f0 = wl.sod_state(*shape, seed=17)
    nsteps = 3
    st = halo.in_process(g, parts)
    try:
        st.set_state(f0)
        whole = ws.Solver(g)
        whole.set_state(f0)
        dt = whole.compute_dt(0.5)
        whole.close()
        assert st.compute_dt(0.5) == dt
        st.step(dt, nsteps)
        got = halo.join_state(st.get_state())
        assert st.status() == 0
    finally:
        st.close()
    want = _run_whole(g, f0, dt, nsteps)
    diff = rel_linf(got, want).max()
    if CL in faces:
        # the end slabs run the closure kernel, the middle ones the plain one;
        # the whole grid runs the closure kernel everywhere
        assert diff <= 1e-13, diff
    else:
        assert np.array_equal(got, want), diff
    if prec == ws.FP64:
        ref = oracle.rk3_steps(or_grid(*shape, face_kind=faces), f0, dt, nsteps)
        assert rel_linf(got, ref).max() <= 1e-12


NS_CASES = [
    ("ns_periodic_2_cd8", (64, 20, 12), (PE,) * 6, 2, 8),
    ("ns_extrap_3_cd6", (66, 16, 12), (EX, EX, PE, PE, PE, PE), 3, 6),
]


@pytest.mark.parametrize("case", NS_CASES, ids=[c[0] for c in NS_CASES])
def test_ns_slabs_match_whole_grid(oracle, cuda, case):
    """Navier-Stokes on slabs: the stage halo and, between the viscous flux
    and divergence passes, the x fluxes' halo."""
    from oracle.oracle import make_vis
    _, shape, faces, parts, scheme = case
    vis = dict(re=200.0, pr=0.72, ref_t=288.15, scheme=scheme)
    g = ws.Grid(*shape, faces=faces)
    f0 = wl.fourier_state(*shape, seed=23)
    nsteps = 3
    whole = ws.Solver(g)
    whole.set_viscous(vis)
    whole.set_state(f0)
    dt = whole.compute_dt(0.3)
    whole.step(dt, nsteps)
    want = whole.get_state()
    whole.close()
    st = halo.in_process(g, parts)
    try:
        st.set_viscous(vis)
        st.set_state(f0)
        st.step(dt, nsteps)
        got = halo.join_state(st.get_state())
        assert st.status() == 0
    finally:
        st.close()
    assert np.array_equal(got, want), rel_linf(got, want).max()
    ref = oracle.rk3_steps_ns(or_grid(*shape, face_kind=faces), make_vis(**vis), f0, dt, nsteps)
    assert rel_linf(got, ref).max() <= 1e-12


def _gloo_rank(rank, world, port, shape, faces, vis, nsteps, out_dir):
    """One rank of a gloo group: its slab on the one GPU of this machine,
    halos staged through host memory (no device-side waiting between the
    ranks' kernels)."""
    import datetime
    import os

    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        g = ws.Grid(*shape, faces=faces)
        f0 = wl.fourier_state(*shape, seed=29)
        st = halo.distributed(g)
        st.set_viscous(vis)
        st.set_state(f0)
        dt = st.compute_dt(0.4)
        st.step(dt, nsteps)
        np.save(os.path.join(out_dir, f"slab{rank}.npy"), st.get_state()[0])
        np.save(os.path.join(out_dir, f"dt{rank}.npy"), np.array([dt, st.status()]))
        st.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", [("euler_periodic_2", (PE,) * 6, 2, None),
                                  ("ns_extrap_3", (EX, EX, PE, PE, PE, PE), 3,
                                   dict(re=200.0, pr=0.72, ref_t=288.15, scheme=8))],
                         ids=lambda c: c[0])
def test_distributed_slabs_gloo_match_whole_grid(cuda, case):
    """halo.distributed end to end in separate processes (one slab each,
    DistExchange over gloo with host staging): the multi-GPU code path with
    the transport swapped, against the whole grid bit for bit."""
    import socket
    import tempfile

    import torch.multiprocessing as mp
    _, faces, parts, vis = case
    shape, nsteps = (60, 16, 12), 3
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_gloo_rank, args=(parts, port, shape, faces, vis, nsteps, d),
                           nprocs=parts, join=True, start_method="spawn")
        got = halo.join_state([np.load(f"{d}/slab{r}.npy") for r in range(parts)])
        meta = [np.load(f"{d}/dt{r}.npy") for r in range(parts)]
    g = ws.Grid(*shape, faces=faces)
    f0 = wl.fourier_state(*shape, seed=29)
    s = ws.Solver(g)
    s.set_viscous(vis)
    s.set_state(f0)
    dt = s.compute_dt(0.4)
    s.step(dt, nsteps)
    want = s.get_state()
    s.close()
    assert all(m[0] == dt and m[1] == 0 for m in meta)
    assert np.array_equal(got, want), rel_linf(got, want).max()


BLOCK_CASES = [
    ("periodic_2x2x1", (48, 40, 12), (PE,) * 6, (2, 2, 1), ws.FP64, None),
    ("mixedfaces_1x2x2", (40, 34, 20), (EX, EX, PE, PE, EX, EX), (1, 2, 2), ws.FP64, None),
    ("periodic_2x2x2", (48, 32, 24), (PE,) * 6, (2, 2, 2), ws.FP64, None),
    ("mixedprec_2x2x1", (48, 40, 12), (PE,) * 6, (2, 2, 1), ws.MIXED, None),
    ("ns_2x2x1", (48, 40, 12), (EX, EX, PE, PE, PE, PE), (2, 2, 1), ws.FP64,
     dict(re=200.0, pr=0.72, ref_t=288.15, scheme=8)),
]


@pytest.mark.parametrize("case", BLOCK_CASES, ids=[c[0] for c in BLOCK_CASES])
def test_blocks_match_whole_grid(cuda, case):
    """Blocks along several axes on one GPU, halos handed over in process."""
    _, shape, faces, dims, prec, vis = case
    g = ws.Grid(*shape, faces=faces, precision=prec)
    f0 = wl.fourier_state(*shape, seed=19)
    whole = ws.Solver(g)
    whole.set_viscous(vis)
    whole.set_state(f0)
    dt = whole.compute_dt(0.3)
    whole.step(dt, 3)
    want = whole.get_state()
    whole.close()
    st = halo.in_process(g, dims=dims)
    try:
        st.set_viscous(vis)
        st.set_state(f0)
        assert st.compute_dt(0.3) == dt
        st.step(dt, 3)
        got = halo.join_state(st.get_state(), [r.block for r in st.runners])
        assert st.status() == 0
    finally:
        st.close()
    assert np.array_equal(got, want), rel_linf(got, want).max()


def _gloo_block_rank(rank, world, port, shape, faces, dims, nsteps, out_dir):
    import datetime
    import os

    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        g = ws.Grid(*shape, faces=faces)
        st = halo.distributed(g, dims=dims)
        st.set_state(wl.fourier_state(*shape, seed=31))
        dt = st.compute_dt(0.4)
        st.step(dt, nsteps)
        np.save(os.path.join(out_dir, f"block{rank}.npy"), st.get_state()[0])
        np.save(os.path.join(out_dir, f"dt{rank}.npy"), np.array([dt, st.status()]))
        st.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_distributed_blocks_gloo_match_whole_grid(cuda):
    """halo.distributed over a 2 x 2 x 1 process grid in four processes
    sharing the GPU (gloo, host-staged), against the whole grid."""
    import socket
    import tempfile

    import torch.multiprocessing as mp
    shape, faces, dims, nsteps = (48, 40, 12), (EX, EX, PE, PE, PE, PE), (2, 2, 1), 2
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    blocks = halo.decompose_blocks(ws.Grid(*shape, faces=faces), dims)
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_gloo_block_rank, args=(4, port, shape, faces, dims, nsteps, d),
                           nprocs=4, join=True, start_method="spawn")
        got = halo.join_state([np.load(f"{d}/block{r}.npy") for r in range(4)], blocks)
        meta = [np.load(f"{d}/dt{r}.npy") for r in range(4)]
    g = ws.Grid(*shape, faces=faces)
    s = ws.Solver(g)
    s.set_state(wl.fourier_state(*shape, seed=31))
    dt = s.compute_dt(0.4)
    s.step(dt, nsteps)
    want = s.get_state()
    s.close()
    assert all(m[0] == dt and m[1] == 0 for m in meta)
    assert np.array_equal(got, want), rel_linf(got, want).max()


# -- the C++ stepper (ws_blocks_*) against the Python stage sequence ---------
NATIVE_CASES = [
    ("slabs_3", (70, 20, 10), (PE,) * 6, (3, 1, 1), None),
    ("closure_2x2", (48, 40, 10), (CL, CL, CL, CL, PE, PE), (2, 2, 1), None),
    ("ns_2x1x2", (48, 16, 24), (EX, EX, PE, PE, PE, PE), (2, 1, 2),
     dict(re=200.0, pr=0.72, ref_t=288.15, scheme=8)),
]


@pytest.mark.parametrize("case", NATIVE_CASES, ids=[c[0] for c in NATIVE_CASES])
def test_native_stepper_matches_python_sequence(cuda, case):
    """halo.in_process runs the library's C++ stepper; the Python sequence
    (native=False) over the same kernels gives the same bits."""
    _, shape, faces, dims, vis = case
    g = ws.Grid(*shape, faces=faces)
    f0 = wl.fourier_state(*shape, seed=37)
    out = []
    for native in (True, False):
        st = halo.in_process(g, dims=dims, native=native)
        try:
            st.set_viscous(vis)
            st.set_state(f0)
            dt = st.compute_dt(0.3)
            st.step(dt, 2)
            out.append((dt, halo.join_state(st.get_state(), [r.block for r in st.runners])))
            assert st.status() == 0
        finally:
            st.close()
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1]), rel_linf(out[0][1], out[1][1]).max()


def test_native_stepper_one_rank_nccl(cuda):
    """The C++ stepper's NCCL mode with a one-rank communicator on this GPU
    (its all-reduce of the time step; one block has no neighbour) against
    the whole-grid solver."""
    shape, faces = (40, 24, 16), (PE,) * 6
    g = ws.Grid(*shape, faces=faces)
    f0 = wl.sod_state(*shape, seed=41)
    whole = ws.Solver(g)
    whole.set_state(f0)
    dt = whole.compute_dt(0.5)
    whole.step(dt, 3)
    want = whole.get_state()
    whole.close()
    st = halo.NativeBlocks(g, (1, 1, 1), halo.nccl_unique_id(), 0)
    try:
        st.set_state(f0)
        assert st.compute_dt(0.5) == dt
        st.step(dt, 3)
        got = st.get_state()[0]
        assert st.status() == 0
    finally:
        st.close()
    assert np.array_equal(got, want)


def test_native_stepper_rejects_bad_input(cuda):
    g = ws.Grid(32, 16, 8)
    with pytest.raises(ws.WsError):
        halo.NativeBlocks(g, (2, 1, 1), halo.nccl_unique_id(), 5)     # rank >= 2
    with pytest.raises(ws.WsError):
        halo.NativeBlocks(ws.Grid(12, 8, 8), (4, 1, 1))               # 3-cell slabs
    st = halo.NativeBlocks(g, (2, 1, 1))
    try:
        with pytest.raises(ws.WsError):
            st.step(0.0, 1)
    finally:
        st.close()


@pytest.mark.parametrize("nccl", [False, True])
def test_native_stepper_dt_failure_is_collective(cuda, nccl):
    """A non-finite state makes ws_blocks_compute_dt fail; in NCCL mode the
    failing rank still takes the all-reduce (so no other rank would wait in
    it for good) and the communicator serves the next call."""
    shape = (32, 16, 8)
    g = ws.Grid(*shape)
    f0 = wl.fourier_state(*shape, seed=47)
    bad = f0.copy()
    bad[4, 3, 5, 7] = np.nan
    st = (halo.NativeBlocks(g, (1, 1, 1), halo.nccl_unique_id(), 0) if nccl
          else halo.NativeBlocks(g, (2, 1, 1)))
    try:
        st.set_state(bad)
        with pytest.raises(ws.WsError):
            st.compute_dt(0.5)
        st.set_state(f0)
        whole = ws.Solver(g)
        whole.set_state(f0)
        assert st.compute_dt(0.5) == whole.compute_dt(0.5)
        whole.close()
    finally:
        st.close()
