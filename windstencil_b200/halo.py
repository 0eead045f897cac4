"""halo -- one grid split into blocks along x, y and z (slabs along x are the
common case), stepped with a halo exchange before every SSP-RK3 stage.

Replaces the reference's MPI decomposition and its per-RHS exchange:

  process grid   NPX0 x NPY0 x NPZ0 ranks, rank = npx + NPX0 * (npy + NPY0 *
                 npz) (OCFD_mpi.c:102-121)
  extents        per axis n = N_GLOBAL / NP, the first N_GLOBAL % NP
                 subdomains one cell wider (OCFD_mpi.c:124-145 and its y, z
                 counterparts)
  neighbours     ID_XM1 / ID_XP1 and the y, z ones (OCFD_mpi.c:176-197):
                 wrapped when the axis is periodic, none at the ends of a
                 non-periodic axis
  exchange       exchange_boundary_{x,y,z}_packed_dev (OCFD_mpi_dev.cpp:
                 123-290): the 4 interior planes next to each shared face,
                 packed over the interior of the other two axes, go to the
                 neighbour on that side and land in its ghost planes
  time loop      OCFD_NS_Solver.cpp:64-90: exchange, du_comput, time advance

The reference copies every packed plane set through host memory and a
blocking MPI_Sendrecv.  Here the planes stay on the device: a pack kernel,
point-to-point sends over NVLink (NCCL through torch.distributed, one rank
per GPU), an unpack kernel, all ordered on the current stream; blocks that
share a process unpack straight from their neighbour's pack buffer.  Each
block steps with its fused RHS + stage kernel (ws_solver_stage) on a grid
whose shared faces are WS_FACE_EXTERNAL.  The stencils are one-dimensional,
so no edge or corner ghosts are needed and the axes' exchanges are
independent of each other.

The stage's halo carries d, u, v, w, T and cc: every ghost value the stage
reads (the reference exchanges d, u, v, w, T and recomputes cc on the padded
field; cc travels here instead of being recomputed).  With viscous terms a
second halo per stage carries, along each axis, that direction's four
viscous fluxes between their flux pass and their divergence, as the
reference exchanges Ev1..4 between vis_flux_ker and their derivatives
(OCFD_Stream.cpp:229-345).

The stage sequence exists twice.  NativeBlocks drives the C++ stepper of
libwindstencil_b200.so (ws_blocks_*: decomposition, pack, exchange, unpack
and stages in C++; blocks in one process read each other's packs, blocks on
separate GPUs exchange through NCCL loaded by the library).  SlabStepper is
the same sequence in Python over CudaBlock runners and an exchange object;
anything with CudaBlock's methods can stand in for a block (the CPU tests run
the oracle that way over gloo ranks), and DistExchange moves the packs with
torch.distributed.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from dataclasses import dataclass

import numpy as np

from . import (FACE_CLOSURE, FACE_EXTERNAL, FACE_PERIODIC, Grid, Solver, WsError, halo_bytes,
               halo_pack, halo_unpack)
from . import _abi

HALO_FIELDS = 6          # d, u, v, w, T, cc
FLUX_FIELDS = 4          # one direction's viscous fluxes Ev1..4
PRIMS, FLUX = "prims", "flux"       # the two halos of a stage
LO, HI = 0, 1            # the faces of an axis


def slab_extents(nx: int, parts: int) -> list[tuple[int, int]]:
    """(first global cell, cells) of each part of an axis: the reference's
    split (OCFD_mpi.c:124-145), the remainder going to the first parts."""
    if parts < 1 or nx < parts:
        raise ValueError(f"cannot split {nx} cells into {parts} parts")
    base, rem = divmod(nx, parts)
    out, x0 = [], 0
    for k in range(parts):
        n = base + (1 if k < rem else 0)
        out.append((x0, n))
        x0 += n
    return out


@dataclass(frozen=True)
class Block:
    """Block `index` of a dims[0] x dims[1] x dims[2] process grid (index x
    fastest): global cells [origin, origin + n) per axis, the neighbours'
    indices per axis and side (None at a non-periodic end or when the axis
    is not split) and the block's face kinds."""
    index: int
    dims: tuple
    coords: tuple
    origin: tuple
    n: tuple
    nbr: tuple          # ((lo, hi) for x, y, z)
    faces: tuple

    # the x-slab view
    @property
    def parts(self) -> int:
        return self.dims[0]

    @property
    def x0(self) -> int:
        return self.origin[0]

    @property
    def nx(self) -> int:
        return self.n[0]

    @property
    def left(self):
        return self.nbr[0][LO]

    @property
    def right(self):
        return self.nbr[0][HI]

    def sides(self, axis: int) -> list[int]:
        return [s for s in (LO, HI) if self.nbr[axis][s] is not None]


Slab = Block


def block_index(dims, coords) -> int:
    return coords[0] + dims[0] * (coords[1] + dims[1] * coords[2])


def decompose_blocks(grid: Grid, dims) -> list[Block]:
    """Split `grid` into dims[0] x dims[1] x dims[2] blocks.  Faces shared
    with a neighbour become WS_FACE_EXTERNAL; the grid's own faces stay at
    the ends of each axis.  An axis split in one part keeps its faces (a
    periodic axis wraps onto itself)."""
    dims = tuple(int(d) for d in dims)
    if len(dims) != 3 or min(dims) < 1:
        raise ValueError("dims: three positive part counts")
    n_glob = (grid.nx, grid.ny, grid.nz)
    per = []
    for ax in range(3):
        lo, hi = grid.faces[2 * ax], grid.faces[2 * ax + 1]
        if (lo == FACE_PERIODIC) != (hi == FACE_PERIODIC):
            raise ValueError(f"axis {ax} must be periodic at both faces or at neither")
        if FACE_EXTERNAL in (lo, hi):
            raise ValueError("the grid to split must not have EXTERNAL faces")
        per.append(slab_extents(n_glob[ax], dims[ax]))
    blocks = []
    for pz in range(dims[2]):
        for py in range(dims[1]):
            for px in range(dims[0]):
                c = (px, py, pz)
                origin, n, nbr, faces = [], [], [], []
                for ax in range(3):
                    P, k = dims[ax], c[ax]
                    lo, hi = grid.faces[2 * ax], grid.faces[2 * ax + 1]
                    o, m = per[ax][k]
                    origin.append(o)
                    n.append(m)
                    if P == 1:
                        nb = (None, None)
                        fk = (lo, hi)
                    else:
                        periodic = lo == FACE_PERIODIC
                        left = k - 1 if k > 0 else (P - 1 if periodic else None)
                        right = k + 1 if k < P - 1 else (0 if periodic else None)
                        nb = tuple(None if kk is None else
                                   block_index(dims, c[:ax] + (kk,) + c[ax + 1:])
                                   for kk in (left, right))
                        fk = (FACE_EXTERNAL if left is not None else lo,
                              FACE_EXTERNAL if right is not None else hi)
                    # a ghost plane set comes from one neighbour's 4 nearest planes
                    need = 8 if FACE_CLOSURE in fk else 4
                    if m < need:
                        raise ValueError(f"block {c} has {m} cells along axis {ax}; "
                                         f"needs >= {need}")
                    nbr.append(nb)
                    faces.extend(fk)
                blocks.append(Block(block_index(dims, c), dims, c, tuple(origin), tuple(n),
                                    tuple(nbr), tuple(faces)))
    return blocks


def decompose(grid: Grid, parts: int) -> list[Block]:
    """Split `grid` into `parts` slabs along x."""
    return decompose_blocks(grid, (parts, 1, 1))


def block_grid(grid: Grid, block: Block) -> Grid:
    """The block's own grid: its extents and face kinds, the global spacing."""
    return dataclasses.replace(grid, nx=block.n[0], ny=block.n[1], nz=block.n[2], hx=grid.hx,
                               hy=grid.hy, hz=grid.hz, faces=tuple(block.faces))


slab_grid = block_grid


def split_state(f: np.ndarray, block: Block) -> np.ndarray:
    """The block's part of a dense conserved state (5, nz, ny, nx)."""
    (x0, y0, z0), (nx, ny, nz) = block.origin, block.n
    return np.ascontiguousarray(f[:, z0:z0 + nz, y0:y0 + ny, x0:x0 + nx])


def join_state(parts: list[np.ndarray], blocks: list[Block] | None = None) -> np.ndarray:
    """The whole state from the blocks' states (x slabs: in slab order)."""
    if blocks is None:
        return np.concatenate(parts, axis=-1)
    ext = [0, 0, 0]
    for b in blocks:
        for ax in range(3):
            ext[ax] = max(ext[ax], b.origin[ax] + b.n[ax])
    out = np.empty((5, ext[2], ext[1], ext[0]))
    for p, b in zip(parts, blocks):
        (x0, y0, z0), (bx, by, bz) = b.origin, b.n
        out[:, z0:z0 + bz, y0:y0 + by, x0:x0 + bx] = p
    return out


class CudaBlock:
    """One block's state and kernels on the current CUDA device: a ws_solver
    over the block grid, plus send and receive halo buffers per split axis
    (sized for the larger halo; the flux halo uses their leading part)."""

    def __init__(self, grid: Grid, block: Block):
        import torch
        self.slab = self.block = block
        self.grid = block_grid(grid, block)
        self.solver = Solver(self.grid)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.n, self._send, self._recv = {}, {}, {}
        for ax in range(3):
            if not block.sides(ax):
                continue
            self.n[ax, PRIMS] = halo_bytes(self.grid, ax, HALO_FIELDS) // 8
            self.n[ax, FLUX] = halo_bytes(self.grid, ax, FLUX_FIELDS) // 8
            self._send[ax] = [torch.empty(self.n[ax, PRIMS], dtype=torch.float64, device=dev)
                              for _ in range(2)]
            self._recv[ax] = [torch.empty(self.n[ax, PRIMS], dtype=torch.float64, device=dev)
                              for _ in range(2)]
        self.krk = 1     # the stage due next
        self.viscous = False

    def set_viscous(self, vis) -> None:
        self.solver.set_viscous(vis)
        self.viscous = vis is not None

    def set_state(self, f_block: np.ndarray) -> None:
        self.solver.set_state(f_block)
        self.krk = 1

    def get_state(self) -> np.ndarray:
        return self.solver.get_state()

    def send(self, axis: int, side: int, kind: str = PRIMS):
        return self._send[axis][side][:self.n[axis, kind]]

    def recv(self, axis: int, side: int, kind: str = PRIMS):
        return self._recv[axis][side][:self.n[axis, kind]]

    def _fields(self, axis, kind):
        if kind == PRIMS:
            return self.solver.stage_fields(self.krk)
        return self.solver.stage_flux_fields(axis)

    def pack(self, axis: int, side: int, kind: str = PRIMS) -> None:
        """Planes next to face (axis, side) of the halo's fields -> send buffer."""
        halo_pack(self.grid, self._fields(axis, kind), axis, side, self.send(axis, side, kind))

    def unpack(self, axis: int, side: int, buf, kind: str = PRIMS) -> None:
        """buf -> ghost planes beyond face (axis, side) of the halo's fields."""
        halo_unpack(self.grid, self._fields(axis, kind), axis, side, buf)

    def begin(self) -> None:
        """First half of the due stage (ghost fill, viscous flux pass)."""
        self.solver.stage_begin(self.krk)

    def end(self, dt: float) -> None:
        """Second half (viscous divergence, fused RHS + stage update)."""
        self.solver.stage_end(self.krk, dt)
        self.krk = self.krk % 3 + 1

    def local_dt(self, cfl: float) -> float:
        return self.solver.compute_dt(cfl)

    def status(self) -> int:
        return self.solver.status()

    def close(self) -> None:
        self.solver.close()


CudaSlab = CudaBlock


class LocalExchange:
    """Every block lives in this process (one or several devices with peer
    access): each block's ghost planes come straight from its neighbour's
    send buffer; no copy in between."""

    def run(self, runners: list, kind: str = PRIMS) -> None:
        by_index = {r.block.index: r for r in runners}
        for ax in range(3):
            for r in runners:
                for side in r.block.sides(ax):
                    r.pack(ax, side, kind)
            for r in runners:
                for side in r.block.sides(ax):
                    nb = by_index[r.block.nbr[ax][side]]
                    r.unpack(ax, side, nb.send(ax, 1 - side, kind), kind)

    def min(self, x: float) -> float:
        return x


class DistExchange:
    """One block per rank of a torch.distributed group, block index = group
    rank: point-to-point sends of the packed planes, issued as one batch.
    With NCCL the device buffers go straight over NVLink; with a backend
    that moves host memory only (gloo) device buffers are staged through
    pinned host copies, as the reference stages its packs for MPI.

    Per axis, sends go low planes first and receives take the high ghosts
    first, and each message is tagged with its axis and the side it was
    packed from, so a two-block periodic ring (the same rank on both sides)
    matches too; the axes follow each other in the same order on every
    rank."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.device_p2p = dist.get_backend(group) == "nccl"
        self._host = {}

    def _peer(self, index: int) -> int:
        if self.group is None:
            return index
        return self.dist.get_global_rank(self.group, index)

    def _staged(self, t, key):
        """The buffer the transport moves: t itself, or its pinned host twin."""
        if self.device_p2p or not t.is_cuda:
            return t
        h = self._host.get(key)
        if h is None or h.numel() != t.numel():
            import torch
            h = torch.empty(t.numel(), dtype=t.dtype).pin_memory()
            self._host[key] = h
        return h

    def run(self, runners: list, kind: str = PRIMS) -> None:
        dist = self.dist
        if len(runners) != 1:
            raise ValueError("DistExchange runs one block per rank")
        r = runners[0]
        b = r.block
        axes = [ax for ax in range(3) if b.sides(ax)]
        send, recv = {}, {}
        for ax in axes:
            for side in b.sides(ax):
                r.pack(ax, side, kind)
                send[ax, side] = self._staged(r.send(ax, side, kind), ("s", ax, side, kind))
                recv[ax, side] = self._staged(r.recv(ax, side, kind), ("r", ax, side, kind))
                if send[ax, side] is not r.send(ax, side, kind):
                    send[ax, side].copy_(r.send(ax, side, kind))   # synchronous D2H
        ops = []
        for ax in axes:
            lo, hi = b.nbr[ax]
            if lo is not None:
                ops.append(dist.P2POp(dist.isend, send[ax, LO], self._peer(lo), self.group,
                                      2 * ax + LO))
            if hi is not None:
                ops.append(dist.P2POp(dist.isend, send[ax, HI], self._peer(hi), self.group,
                                      2 * ax + HI))
                ops.append(dist.P2POp(dist.irecv, recv[ax, HI], self._peer(hi), self.group,
                                      2 * ax + LO))
            if lo is not None:
                ops.append(dist.P2POp(dist.irecv, recv[ax, LO], self._peer(lo), self.group,
                                      2 * ax + HI))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for ax in axes:
            for side in b.sides(ax):
                buf = r.recv(ax, side, kind)
                if recv[ax, side] is not buf:
                    buf.copy_(recv[ax, side], non_blocking=True)   # pinned -> device, in order
                r.unpack(ax, side, buf, kind)

    def min(self, x: float) -> float:
        import torch
        dist = self.dist
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        return float(t.item())


class SlabStepper:
    """SSP-RK3 steps of a grid split into blocks: before each stage the halos
    of the stage's input are exchanged, then every local block runs its
    fused stage.  `runners` are this process's blocks."""

    def __init__(self, runners: list, exchange):
        self.runners = runners
        self.exchange = exchange

    def stage(self, dt: float) -> None:
        self.exchange.run(self.runners, PRIMS)
        for r in self.runners:
            r.begin()
        if self.viscous:
            self.exchange.run(self.runners, FLUX)
        for r in self.runners:
            r.end(dt)

    @property
    def viscous(self) -> bool:
        return any(r.viscous for r in self.runners)

    def set_viscous(self, vis) -> None:
        """Navier-Stokes on every block (ws_viscous constants; None: Euler).
        Every rank must make the same choice: it adds an exchange per stage."""
        for r in self.runners:
            r.set_viscous(vis)

    def step(self, dt: float, nsteps: int = 1) -> None:
        if not dt > 0:
            raise ValueError("dt must be > 0")
        for _ in range(nsteps * 3):
            self.stage(dt)

    def compute_dt(self, cfl: float) -> float:
        """Global CFL time step: the minimum of the blocks' (the maximum wave
        speed over the whole grid).  Every rank takes the reduction, also when
        its own blocks fail (they contribute -1), so that no rank waits in it
        for good; then every rank raises."""
        err = None
        try:
            local = min(r.local_dt(cfl) for r in self.runners)
        except WsError as e:
            local, err = -1.0, e
        if not local > 0:                      # NaN or a failure
            local = -1.0
        dt = self.exchange.min(local)
        if err is not None:
            raise err
        if not dt > 0:
            raise WsError(_abi.WS_ERR_NONFINITE, "a block's maximum wave speed is not finite "
                                                 "and positive")
        return dt

    def set_state(self, f_global: np.ndarray) -> None:
        for r in self.runners:
            r.set_state(split_state(f_global, r.block))

    def get_state(self) -> list[np.ndarray]:
        """This process's blocks' states, in block order."""
        return [r.get_state() for r in self.runners]

    def status(self) -> int:
        return max(r.status() for r in self.runners)

    def close(self) -> None:
        for r in self.runners:
            r.close()


BlockStepper = SlabStepper


def in_process(grid: Grid, parts=None, dims=None, native: bool = True):
    """All blocks on the current CUDA device (a single-GPU stand-in for a
    multi-GPU run: same kernels, same halos, no waits between blocks):
    `parts` x slabs, or a dims[0] x dims[1] x dims[2] process grid.  native:
    the library's C++ stepper (NativeBlocks), else the Python sequence."""
    dims = tuple(dims) if dims is not None else (parts, 1, 1)
    if native:
        return NativeBlocks(grid, dims)
    return SlabStepper([CudaBlock(grid, b) for b in decompose_blocks(grid, dims)],
                       LocalExchange())


def distributed(grid: Grid, group=None, dims=None, native: bool = False):
    """This rank's block of `grid` split over the ranks of `group` (one GPU
    per rank, the current CUDA device): x slabs, or `dims` whose product is
    the group size.  native: the library's C++ stepper over its own NCCL
    communicator (the id travels over `group`; NCCL ranks = group ranks),
    else the Python sequence over torch.distributed."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dims = tuple(dims) if dims is not None else (world, 1, 1)
    if dims[0] * dims[1] * dims[2] != world:
        raise ValueError(f"dims {dims} do not match {world} ranks")
    rank = dist.get_rank(group)
    if native:
        box = [nccl_unique_id() if rank == 0 else None]
        dist.broadcast_object_list(box, src=dist.get_global_rank(group, 0) if group else 0,
                                   group=group)
        return NativeBlocks(grid, dims, box[0], rank)
    block = decompose_blocks(grid, dims)[rank]
    return SlabStepper([CudaBlock(grid, block)], DistExchange(group))


# ---- the C++ stepper ---------------------------------------------------------

def _block_of(info, dims) -> Block:
    nbr = tuple(tuple(None if info.nbr[ax][sd] < 0 else int(info.nbr[ax][sd])
                      for sd in (LO, HI)) for ax in range(3))
    return Block(int(info.index), tuple(dims), tuple(info.coords), tuple(info.origin),
                 tuple(info.n), nbr, tuple(info.faces))


def native_decompose(grid: Grid, dims) -> list[Block]:
    """The library's decomposition (ws_blocks_decompose) of `grid` into
    dims[0] x dims[1] x dims[2] blocks."""
    from . import check, load
    d = (C.c_int32 * 3)(*dims)
    gc = grid.c()
    out = []
    for i in range(max(1, d[0] * d[1] * d[2])):      # index 0 also checks dims
        info = _abi.WsBlockInfo()
        check(load().ws_blocks_decompose(C.byref(gc), d, i, C.byref(info)))
        out.append(_block_of(info, dims))
    return out


def native_exchange_plan(grid: Grid, dims, index: int) -> list[tuple]:
    """The messages block `index` posts in one NCCL exchange of the C++
    stepper (ws_blocks_exchange_plan), in order: (kind "send" / "recv",
    peer block, axis, side)."""
    from . import check, load
    d = (C.c_int32 * 3)(*dims)
    gc = grid.c()
    ops = (_abi.WsP2pOp * 12)()
    n = C.c_int32()
    check(load().ws_blocks_exchange_plan(C.byref(gc), d, index, ops, 12, C.byref(n)))
    return [("send" if o.kind == 0 else "recv", o.peer, o.axis, o.side) for o in ops[:n.value]]


class _BlockSolver(Solver):
    """A block's ws_solver, owned by the ws_blocks object."""

    def __init__(self, g: Grid, handle):
        self.g = g
        self._gc = g.c()
        self.h = handle

    def close(self):
        self.h = None


class NativeRunner:
    """One block of a NativeBlocks stepper in this process."""

    def __init__(self, grid: Grid, block: Block, handle):
        self.block = self.slab = block
        self.grid = block_grid(grid, block)
        self.solver = _BlockSolver(self.grid, handle)

    def set_state(self, f_block: np.ndarray) -> None:
        self.solver.set_state(f_block)

    def get_state(self) -> np.ndarray:
        return self.solver.get_state()


class NativeBlocks:
    """SSP-RK3 steps of `grid` split into dims[0] x dims[1] x dims[2] blocks,
    stepped by the library's C++ stepper (ws_blocks_*).  nccl_id None: every
    block in this process on the current device; else this process owns
    block `rank` and exchanges with the other ranks over NCCL."""

    def __init__(self, grid: Grid, dims, nccl_id: bytes | None = None, rank: int = 0):
        from . import check, load
        self.grid = grid
        self.dims = tuple(int(v) for v in dims)
        self._gc = grid.c()
        d = (C.c_int32 * 3)(*self.dims)
        h = C.c_void_p()
        idbuf = None
        if nccl_id is not None:
            idbuf = C.create_string_buffer(bytes(nccl_id), 128)
        check(load().ws_blocks_create(C.byref(self._gc), d, idbuf, int(rank), C.byref(h)))
        self.h = h
        n = C.c_int32()
        check(load().ws_blocks_count(self.h, C.byref(n)))
        self.runners = []
        for i in range(n.value):
            info = _abi.WsBlockInfo()
            check(load().ws_blocks_info(self.h, i, C.byref(info)))
            sh = C.c_void_p()
            check(load().ws_blocks_solver(self.h, i, C.byref(sh)))
            self.runners.append(NativeRunner(grid, _block_of(info, self.dims), sh))
        self.viscous = False

    def set_viscous(self, vis) -> None:
        from . import check, load, viscous
        if vis is None:
            check(load().ws_blocks_set_viscous(self.h, None))
        else:
            v = vis if isinstance(vis, _abi.WsViscous) else viscous(**vis)
            check(load().ws_blocks_set_viscous(self.h, C.byref(v)))
        self.viscous = vis is not None

    def step(self, dt: float, nsteps: int = 1, stream=None) -> None:
        from . import _stream, check, load
        check(load().ws_blocks_step(self.h, dt, nsteps, _stream(stream)))

    def compute_dt(self, cfl: float, stream=None) -> float:
        from . import _stream, check, load
        dt = C.c_double()
        check(load().ws_blocks_compute_dt(self.h, cfl, C.byref(dt), _stream(stream)))
        return dt.value

    def set_state(self, f_global: np.ndarray) -> None:
        for r in self.runners:
            r.set_state(split_state(f_global, r.block))

    def get_state(self) -> list[np.ndarray]:
        """This process's blocks' states, in block order."""
        return [r.get_state() for r in self.runners]

    def status(self, stream=None) -> int:
        from . import _stream, check, load
        s = C.c_int()
        check(load().ws_blocks_status(self.h, C.byref(s), _stream(stream)))
        return s.value

    def close(self) -> None:
        from . import load
        if self.h:
            load().ws_blocks_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def nccl_unique_id() -> bytes:
    """A new NCCL communicator id (ws_nccl_unique_id), for NativeBlocks."""
    from . import check, load
    buf = C.create_string_buffer(128)
    check(load().ws_nccl_unique_id(buf))
    return buf.raw
