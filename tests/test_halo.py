"""Slab decomposition along x and the x-halo exchange (windstencil_b200.halo),
checked on the CPU: the split against the reference's rule, and whole runs
of SlabStepper over oracle slabs, in one process and as gloo ranks
(world_size 2 and 3), against the oracle on the undivided grid, bit for bit."""
import ctypes as C
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle.oracle import make_grid as or_make_grid
from windstencil_b200 import (FACE_CLOSURE, FACE_EXTERNAL, FACE_EXTRAP, FACE_PERIODIC, Grid,
                              WsError, workloads as wl)
from windstencil_b200.halo import (DistExchange, LocalExchange, SlabStepper, decompose,
                                   decompose_blocks, join_state, slab_extents, split_state)

from halo_oracle import OracleSlab


def _or_grid(g: Grid):
    return or_make_grid(g.nx, g.ny, g.nz, hx=g.hx, hy=g.hy, hz=g.hz, gamma=g.gamma, ama=g.ama,
                        epsl_sw=g.epsl_sw, face_kind=g.faces)


def _state(g: Grid, seed=3):
    return wl.sod_state(g.nx, g.ny, g.nz, seed=seed)


# -- the split ---------------------------------------------------------------
@pytest.mark.parametrize("nx,parts", [(64, 2), (65, 2), (67, 4), (600, 8), (9, 1), (31, 5)])
def test_slab_extents_follow_reference_split(nx, parts):
    """OCFD_mpi.c:124-145: nx = NX/NPX0 (+1 for npx < NX % NPX0), offset
    NX/NPX0 * k + min(k, NX % NPX0)."""
    ext = slab_extents(nx, parts)
    for k, (x0, n) in enumerate(ext):
        assert n == nx // parts + (1 if k < nx % parts else 0)
        assert x0 == nx // parts * k + min(k, nx % parts)
    assert sum(n for _, n in ext) == nx


def test_decompose_neighbours_and_faces():
    g = Grid(64, 16, 8, faces=(FACE_PERIODIC,) * 6)
    s = decompose(g, 4)
    assert [(x.left, x.right) for x in s] == [(3, 1), (0, 2), (1, 3), (2, 0)]
    assert all(x.faces[:2] == (FACE_EXTERNAL, FACE_EXTERNAL) for x in s)
    g = Grid(64, 16, 8, faces=(FACE_CLOSURE, FACE_EXTRAP) + (FACE_PERIODIC,) * 4)
    s = decompose(g, 3)
    assert [(x.left, x.right) for x in s] == [(None, 1), (0, 2), (1, None)]
    assert s[0].faces[:2] == (FACE_CLOSURE, FACE_EXTERNAL)
    assert s[1].faces[:2] == (FACE_EXTERNAL, FACE_EXTERNAL)
    assert s[2].faces[:2] == (FACE_EXTERNAL, FACE_EXTRAP)
    assert all(x.faces[2:] == g.faces[2:] for x in s)
    one = decompose(g, 1)[0]
    assert one.faces == tuple(g.faces) and one.left is None and one.right is None


def test_decompose_rejects_thin_or_mixed():
    with pytest.raises(ValueError):
        decompose(Grid(12, 8, 8, faces=(FACE_PERIODIC,) * 6), 4)        # 3 cells a slab
    with pytest.raises(ValueError):
        decompose(Grid(28, 8, 8, faces=(FACE_CLOSURE, FACE_EXTRAP) + (0,) * 4), 4)  # 7 < 8
    with pytest.raises(ValueError):
        decompose(Grid(32, 8, 8, faces=(FACE_PERIODIC, FACE_EXTRAP) + (0,) * 4), 2)


@pytest.mark.parametrize("dims", [(2, 1, 1), (4, 1, 1), (3, 2, 1), (2, 2, 2), (1, 3, 2), (1, 1, 1)])
@pytest.mark.parametrize("faces", [(FACE_PERIODIC,) * 6,
                                   (FACE_CLOSURE, FACE_EXTRAP, FACE_PERIODIC, FACE_PERIODIC,
                                    FACE_EXTRAP, FACE_EXTRAP),
                                   (FACE_EXTRAP, FACE_EXTRAP, FACE_CLOSURE, FACE_CLOSURE,
                                    FACE_PERIODIC, FACE_PERIODIC)])
def test_native_decomposition_matches(dims, faces):
    """ws_blocks_decompose (the C++ stepper's split) equals decompose_blocks:
    extents, neighbours, face kinds, block order."""
    from windstencil_b200.halo import native_decompose
    g = Grid(67, 33, 19, faces=faces)
    assert native_decompose(g, dims) == decompose_blocks(g, dims)


def test_native_decomposition_rejects_like_python():
    from windstencil_b200.halo import native_decompose
    bad = [(Grid(12, 8, 8, faces=(FACE_PERIODIC,) * 6), (4, 1, 1)),
           (Grid(28, 8, 8, faces=(FACE_CLOSURE, FACE_EXTRAP) + (0,) * 4), (4, 1, 1)),
           (Grid(32, 8, 8, faces=(FACE_PERIODIC, FACE_EXTRAP) + (0,) * 4), (2, 1, 1)),
           (Grid(32, 8, 8, faces=(FACE_EXTERNAL, FACE_EXTRAP) + (0,) * 4), (2, 1, 1)),
           (Grid(32, 8, 8), (0, 1, 1))]
    for g, dims in bad:
        with pytest.raises(ValueError):
            decompose_blocks(g, dims)
        with pytest.raises(WsError):
            native_decompose(g, dims)


@pytest.mark.parametrize("dims", [(2, 1, 1), (3, 1, 1), (2, 2, 1), (2, 2, 2), (1, 2, 3),
                                  (4, 1, 2)])
@pytest.mark.parametrize("periodic", [True, False])
def test_native_nccl_plan_matches_in_order(dims, periodic):
    """The C++ stepper's NCCL exchange posts each rank's messages in
    ws_blocks_exchange_plan's order, and NCCL matches the messages between
    two ranks in posting order.  Simulated over all ranks: every send finds a
    receive, and the k-th send from a to b (planes next to face (axis, s))
    meets the k-th receive at b from a, which fills the ghosts beyond face
    (axis, 1 - s) -- the neighbour's opposite face -- along the same axis;
    each shared face is received exactly once."""
    from windstencil_b200.halo import native_exchange_plan
    k = FACE_PERIODIC if periodic else FACE_EXTRAP
    g = Grid(48, 40, 32, faces=(k,) * 6)
    blocks = decompose_blocks(g, dims)
    plans = [native_exchange_plan(g, dims, b.index) for b in blocks]
    sends, recvs = {}, {}
    for a, plan in enumerate(plans):
        for kind, peer, axis, side in plan:
            (sends if kind == "send" else recvs).setdefault((a, peer) if kind == "send"
                                                            else (peer, a), []).append((axis, side))
    assert sends.keys() == recvs.keys()
    for (a, b), out in sends.items():
        into = recvs[(a, b)]
        assert len(out) == len(into)
        for (ax_s, s), (ax_r, r) in zip(out, into):
            assert ax_s == ax_r and r == 1 - s
            assert blocks[a].nbr[ax_s][s] == b and blocks[b].nbr[ax_r][r] == a
    for b, plan in zip(blocks, plans):
        got = sorted((ax, sd) for kind, _, ax, sd in plan if kind == "recv")
        assert got == sorted((ax, sd) for ax in range(3) for sd in b.sides(ax))


def test_abi_halo_argument_checks():
    """Halo entry points validate their arguments before any device work."""
    from windstencil_b200 import _abi
    lib = _abi.load()
    g = Grid(16, 12, 10, faces=(FACE_EXTERNAL, 0, FACE_EXTERNAL, 0, 0, FACE_EXTERNAL)).c()
    fields = (_abi.WsField * 1)(_abi.WsField(8, 32, 0))
    assert lib.ws_halo_pack(C.byref(g), fields, 1, 3, 0, 8, None) == 1      # bad axis
    assert lib.ws_halo_pack(C.byref(g), fields, 1, 1, 2, 8, None) == 1      # bad side
    assert lib.ws_halo_unpack(C.byref(g), fields, 9, 2, 0, 8, None) == 1    # 9 fields
    assert lib.ws_halo_pack_x(C.byref(g), fields, 1, 2, 8, None) == 1
    assert lib.ws_halo_bytes(C.byref(g), 0, 6) == 6 * 10 * 12 * 4 * 8
    assert lib.ws_halo_bytes(C.byref(g), 1, 6) == 6 * 10 * 4 * 16 * 8
    assert lib.ws_halo_bytes(C.byref(g), 2, 6) == 6 * 4 * 12 * 16 * 8
    assert lib.ws_halo_x_bytes(C.byref(g), 6) == lib.ws_halo_bytes(C.byref(g), 0, 6)
    g.face_kind[0] = 7
    assert lib.ws_ghost_fill(C.byref(g), fields, 1, None) == 1


# -- whole runs over oracle slabs --------------------------------------------
VIS = dict(re=200.0, pr=0.72, ref_t=288.15, scheme=8)
PE3 = (FACE_PERIODIC,) * 6
MIX = (FACE_EXTRAP, FACE_EXTRAP, FACE_PERIODIC, FACE_PERIODIC, FACE_EXTRAP, FACE_EXTRAP)
CLO = (FACE_CLOSURE, FACE_CLOSURE, FACE_CLOSURE, FACE_CLOSURE, FACE_PERIODIC, FACE_PERIODIC)
# blocks: (grid, dims, viscous constants)
BLOCK_CASES = {
    "periodic_2x2x1": (Grid(24, 20, 10, faces=PE3), (2, 2, 1), None),
    "periodic_1x2x2": (Grid(20, 18, 16, faces=PE3), (1, 2, 2), None),
    "mixed_2x1x2": (Grid(26, 12, 17, faces=MIX), (2, 1, 2), None),
    "closure_2x2x1": (Grid(32, 24, 8, faces=CLO), (2, 2, 1), None),
    "periodic_2x2x2": (Grid(20, 16, 12, faces=PE3), (2, 2, 2), None),
    "ns_mixed_2x2x1": (Grid(24, 20, 10, faces=MIX), (2, 2, 1), dict(VIS, scheme=6)),
    "ns_periodic_1x2x2": (Grid(12, 18, 16, faces=PE3), (1, 2, 2), VIS),
}
CASES = {
    "periodic_2": (Grid(40, 12, 10, faces=(FACE_PERIODIC,) * 6), 2, None),
    "periodic_3": (Grid(37, 12, 10, faces=(FACE_PERIODIC,) * 6), 3, None),
    "extrap_3": (Grid(36, 12, 10, faces=(FACE_EXTRAP, FACE_EXTRAP) + (FACE_PERIODIC,) * 4), 3,
                 None),
    "closure_2": (Grid(32, 12, 10, faces=(FACE_CLOSURE, FACE_CLOSURE, FACE_CLOSURE,
                                          FACE_CLOSURE, FACE_PERIODIC, FACE_PERIODIC)), 2, None),
    "ns_periodic_2": (Grid(40, 12, 10, faces=(FACE_PERIODIC,) * 6), 2, VIS),
    "ns_extrap_3": (Grid(36, 12, 10, faces=(FACE_EXTRAP, FACE_EXTRAP) + (FACE_PERIODIC,) * 4),
                    3, dict(VIS, scheme=6)),
}
NSTEPS = 2


def _reference_run(oracle, g, f, nsteps, vis=None):
    from oracle.oracle import make_vis
    og = _or_grid(g)
    dt = oracle.compute_dt(og, f, 0.5)
    if vis is None:
        return dt, oracle.rk3_steps(og, f, dt, nsteps)
    return dt, oracle.rk3_steps_ns(og, make_vis(**vis), f, dt, nsteps)


@pytest.mark.parametrize("case", sorted(CASES))
def test_slabs_in_one_process_match_whole_grid(oracle, case):
    g, parts, vis = CASES[case]
    f = _state(g)
    dt, want = _reference_run(oracle, g, f, NSTEPS, vis)
    st = SlabStepper([OracleSlab(oracle, g, s) for s in decompose(g, parts)], LocalExchange())
    st.set_viscous(vis)
    assert st.viscous == (vis is not None)
    st.set_state(f)
    assert st.compute_dt(0.5) == dt
    st.step(dt, NSTEPS)
    got = join_state(st.get_state())
    assert np.array_equal(got, want)


def test_decompose_blocks_reference_order_and_neighbours():
    """Rank = npx + NPX0 * (npy + NPY0 * npz) (OCFD_mpi.c:111-113); per-axis
    extents by the reference's rule; periodic axes wrap, others end."""
    g = Grid(30, 20, 12, faces=MIX)
    blocks = decompose_blocks(g, (3, 2, 2))
    assert [b.index for b in blocks] == list(range(12))
    for b in blocks:
        px, py, pz = b.coords
        assert b.index == px + 3 * (py + 2 * pz)
        assert (b.origin[0], b.n[0]) == slab_extents(30, 3)[px]
        assert (b.origin[1], b.n[1]) == slab_extents(20, 2)[py]
        assert (b.origin[2], b.n[2]) == slab_extents(12, 2)[pz]
    b = blocks[0]                                       # (0, 0, 0)
    assert b.nbr[0] == (None, 1) and b.nbr[1] == (3, 3) and b.nbr[2] == (None, 6)
    assert b.faces == (FACE_EXTRAP, FACE_EXTERNAL, FACE_EXTERNAL, FACE_EXTERNAL,
                       FACE_EXTRAP, FACE_EXTERNAL)
    b = blocks[11]                                      # (2, 1, 1)
    assert b.nbr[0] == (10, None) and b.nbr[1] == (8, 8) and b.nbr[2] == (5, None)
    assert b.faces[0] == FACE_EXTERNAL and b.faces[1] == FACE_EXTRAP
    f = np.random.default_rng(1).random((5, 12, 20, 30))
    parts = [split_state(f, x) for x in blocks]
    assert np.array_equal(join_state(parts, blocks), f)
    with pytest.raises(ValueError):
        decompose_blocks(Grid(30, 12, 12, faces=MIX), (3, 4, 1))      # 3 cells along y


@pytest.mark.parametrize("case", sorted(BLOCK_CASES))
def test_blocks_in_one_process_match_whole_grid(oracle, case):
    g, dims, vis = BLOCK_CASES[case]
    f = _state(g)
    dt, want = _reference_run(oracle, g, f, NSTEPS, vis)
    blocks = decompose_blocks(g, dims)
    st = SlabStepper([OracleSlab(oracle, g, b) for b in blocks], LocalExchange())
    st.set_viscous(vis)
    st.set_state(f)
    assert st.compute_dt(0.5) == dt
    st.step(dt, NSTEPS)
    assert np.array_equal(join_state(st.get_state(), blocks), want)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, case, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist
    from oracle.oracle import Oracle
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        oracle = Oracle()
        oracle.set_threads(1)
        g, parts, vis = CASES[case]
        assert parts == world
        slab = decompose(g, world)[rank]
        st = SlabStepper([OracleSlab(oracle, g, slab)], DistExchange())
        st.set_viscous(vis)
        st.set_state(_state(g))
        dt = st.compute_dt(0.5)
        st.step(dt, NSTEPS)
        np.save(os.path.join(out_dir, f"slab{rank}.npy"), st.get_state()[0])
        np.save(os.path.join(out_dir, f"dt{rank}.npy"), np.array([dt]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["periodic_2", "periodic_3", "closure_2", "ns_periodic_2",
                                  "ns_extrap_3"])
def test_gloo_ranks_match_whole_grid(oracle, case):
    """One slab per gloo rank: DistExchange's sends / receives (a two-rank
    periodic ring has the same rank on both sides), the viscous fluxes' halo
    and the dt reduction."""
    g, parts, vis = CASES[case]
    f = _state(g)
    dt, want = _reference_run(oracle, g, f, NSTEPS, vis)
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(parts, _free_port(), case, d), nprocs=parts,
                           join=True, start_method="spawn")
        got = join_state([np.load(os.path.join(d, f"slab{r}.npy")) for r in range(parts)])
        dts = [float(np.load(os.path.join(d, f"dt{r}.npy"))[0]) for r in range(parts)]
    assert dts == [dt] * parts
    assert np.array_equal(got, want)


def _dt_failure_rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist
    from oracle.oracle import Oracle
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        oracle = Oracle()
        oracle.set_threads(1)
        g = Grid(32, 12, 8, faces=(FACE_PERIODIC,) * 6)

        class FailingSlab(OracleSlab):          # a block whose dt fails, planted on the CPU
            def local_dt(self, cfl):
                raise WsError(5, "planted: non-finite wave speed")

        slab = decompose(g, world)[rank]
        runner = (FailingSlab if rank == 1 else OracleSlab)(oracle, g, slab)
        st = SlabStepper([runner], DistExchange())
        st.set_state(_state(g))
        try:
            st.compute_dt(0.5)
            outcome = "returned"
        except WsError:
            outcome = "raised"
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as fh:
            fh.write(outcome)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_dt_failure_is_collective():
    """A rank whose block's time step fails still takes the dt reduction
    (contributing -1), so the other rank does not wait in it for good, and
    every rank raises."""
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_dt_failure_rank_main, args=(2, _free_port(), d), nprocs=2,
                           join=True, start_method="spawn")
        got = [open(os.path.join(d, f"rank{r}.txt")).read() for r in range(2)]
    assert got == ["raised", "raised"]


def _block_rank_main(rank, world, port, case, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist
    from oracle.oracle import Oracle
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        oracle = Oracle()
        oracle.set_threads(1)
        g, dims, vis = BLOCK_CASES[case]
        block = decompose_blocks(g, dims)[rank]
        st = SlabStepper([OracleSlab(oracle, g, block)], DistExchange())
        st.set_viscous(vis)
        st.set_state(_state(g))
        dt = st.compute_dt(0.5)
        st.step(dt, NSTEPS)
        np.save(os.path.join(out_dir, f"block{rank}.npy"), st.get_state()[0])
        np.save(os.path.join(out_dir, f"dt{rank}.npy"), np.array([dt]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["periodic_2x2x1", "mixed_2x1x2", "ns_periodic_1x2x2"])
def test_gloo_block_ranks_match_whole_grid(oracle, case):
    """One block per gloo rank (4 ranks): the exchange along every split axis,
    two-rank periodic rings on each, the viscous fluxes' halos per direction."""
    g, dims, vis = BLOCK_CASES[case]
    world = dims[0] * dims[1] * dims[2]
    f = _state(g)
    dt, want = _reference_run(oracle, g, f, NSTEPS, vis)
    blocks = decompose_blocks(g, dims)
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_block_rank_main, args=(world, _free_port(), case, d), nprocs=world,
                           join=True, start_method="spawn")
        got = join_state([np.load(os.path.join(d, f"block{r}.npy")) for r in range(world)],
                         blocks)
        dts = [float(np.load(os.path.join(d, f"dt{r}.npy"))[0]) for r in range(world)]
    assert dts == [dt] * world
    assert np.array_equal(got, want)


def test_split_state_round_trip():
    g = Grid(37, 6, 5)
    f = np.random.default_rng(0).random((5, 5, 6, 37))
    parts = [split_state(f, s) for s in decompose(g, 3)]
    assert [p.shape[-1] for p in parts] == [13, 12, 12]
    assert np.array_equal(join_state(parts), f)
