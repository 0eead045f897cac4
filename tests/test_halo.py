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
                                   join_state, slab_extents, split_state)

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


def test_abi_rejects_external_outside_x():
    """EXTERNAL is an x-face kind only; the check runs before any device work."""
    from windstencil_b200 import _abi
    lib = _abi.load()
    g = Grid(16, 16, 16, faces=(0, 0, FACE_EXTERNAL, 0, 0, 0)).c()
    h = C.c_void_p()
    assert lib.ws_solver_create(C.byref(g), C.byref(h)) == 4        # WS_ERR_UNSUPPORTED
    g = Grid(16, 16, 16, faces=(FACE_EXTERNAL, 0, 0, 0, 0, 0)).c()
    fields = (_abi.WsField * 1)(_abi.WsField(8, 32, 0))
    assert lib.ws_halo_pack_x(C.byref(g), fields, 1, 2, 8, None) == 1   # bad side
    assert lib.ws_halo_unpack_x(C.byref(g), fields, 9, 0, 8, None) == 1  # 9 fields
    assert lib.ws_halo_x_bytes(C.byref(g), 6) == 6 * 16 * 16 * 4 * 8
    g.face_kind[0] = 7
    assert lib.ws_ghost_fill(C.byref(g), fields, 1, None) == 1


# -- whole runs over oracle slabs --------------------------------------------
VIS = dict(re=200.0, pr=0.72, ref_t=288.15, scheme=8)
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


def test_split_state_round_trip():
    g = Grid(37, 6, 5)
    f = np.random.default_rng(0).random((5, 5, 6, 37))
    parts = [split_state(f, s) for s in decompose(g, 3)]
    assert [p.shape[-1] for p in parts] == [13, 12, 12]
    assert np.array_equal(join_state(parts), f)
