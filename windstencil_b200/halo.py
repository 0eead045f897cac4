"""halo -- one grid split into slabs along x, stepped with an x-halo exchange
before every SSP-RK3 stage.

Replaces the reference's MPI x decomposition and its per-RHS exchange:

  slab extents   OCFD_mpi.c:124-145 (nx = NX_GLOBAL / NPX0; the first
                 NX_GLOBAL % NPX0 subdomains one cell wider; offsets i_offset)
  neighbours     ID_XM1 / ID_XP1 (OCFD_mpi.c:176-197): wrapped when x is
                 periodic, none at the ends of a non-periodic x
  exchange       exchange_boundary_x_packed_dev (OCFD_mpi_dev.cpp:185-218):
                 the 4 interior planes next to each x face, packed
                 [field][z][y][x] over interior y, z, go to the neighbour on
                 that side and land in its ghost planes
  time loop      OCFD_NS_Solver.cpp:64-90: exchange, du_comput, time advance

The reference copies every packed plane set through host memory and a
blocking MPI_Sendrecv.  Here the planes stay on the device: a pack kernel,
point-to-point sends over NVLink (NCCL through torch.distributed, one rank
per GPU), an unpack kernel, all ordered on the current stream; slabs that
share a process unpack straight from their neighbour's pack buffer.  Each
slab steps with its fused RHS + stage kernel (ws_solver_stage) on a grid
whose shared x faces are WS_FACE_EXTERNAL.

The stage's halo carries d, u, v, w, T and cc: every ghost value the stage
reads (the reference exchanges d, u, v, w, T and recomputes cc on the padded
field; cc travels here instead of being recomputed).  With viscous terms a
second halo per stage carries the four x-direction viscous fluxes between
their flux pass and their divergence, as the reference exchanges Ev1..4
between vis_flux_ker and their derivatives (OCFD_Stream.cpp:229-345).

This module holds the decomposition, the exchange and the stage sequence;
the per-slab kernels live in libwindstencil_b200.so (CudaSlab).  Anything
with CudaSlab's methods can stand in for it (the CPU tests run the oracle
that way over gloo ranks).
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass

import numpy as np

from . import (FACE_CLOSURE, FACE_EXTERNAL, FACE_PERIODIC, Grid, Solver, halo_pack_x,
               halo_unpack_x, halo_x_bytes)

HALO_FIELDS = 6          # d, u, v, w, T, cc
FLUX_FIELDS = 4          # x-direction viscous fluxes Ev1..4
PRIMS, FLUX = "prims", "flux"       # the two halos of a stage
LO, HI = 0, 1            # x faces of a slab


def slab_extents(nx: int, parts: int) -> list[tuple[int, int]]:
    """(first global x cell, cells) of each slab: the reference's split
    (OCFD_mpi.c:124-145), the remainder going to the first slabs."""
    if parts < 1 or nx < parts:
        raise ValueError(f"cannot split {nx} cells into {parts} slabs")
    base, rem = divmod(nx, parts)
    out, x0 = [], 0
    for k in range(parts):
        n = base + (1 if k < rem else 0)
        out.append((x0, n))
        x0 += n
    return out


@dataclass(frozen=True)
class Slab:
    """Slab `index` of `parts`: global x cells [x0, x0 + nx), its neighbours'
    indices (None at a non-periodic end) and its face kinds."""
    index: int
    parts: int
    x0: int
    nx: int
    left: int | None
    right: int | None
    faces: tuple


def decompose(grid: Grid, parts: int) -> list[Slab]:
    """Split `grid` into `parts` slabs along x.  Shared faces become
    WS_FACE_EXTERNAL; the grid's own x faces stay at the two ends.  One slab
    keeps the grid as it is (a periodic x wraps onto itself)."""
    lo, hi = grid.faces[0], grid.faces[1]
    if (lo == FACE_PERIODIC) != (hi == FACE_PERIODIC):
        raise ValueError("x must be periodic at both faces or at neither")
    if FACE_EXTERNAL in (lo, hi):
        raise ValueError("the grid to split must not have EXTERNAL faces")
    periodic = lo == FACE_PERIODIC
    slabs = []
    for k, (x0, n) in enumerate(slab_extents(grid.nx, parts)):
        if parts == 1:
            left = right = None
            faces = tuple(grid.faces)
        else:
            left = k - 1 if k > 0 else (parts - 1 if periodic else None)
            right = k + 1 if k < parts - 1 else (0 if periodic else None)
            faces = (FACE_EXTERNAL if left is not None else lo,
                     FACE_EXTERNAL if right is not None else hi) + tuple(grid.faces[2:])
        # a ghost plane set comes from one neighbour's 4 nearest planes
        need = 8 if FACE_CLOSURE in faces[:2] else 4
        if n < need:
            raise ValueError(f"slab {k} has {n} cells along x; needs >= {need}")
        slabs.append(Slab(k, parts, x0, n, left, right, faces))
    return slabs


def slab_grid(grid: Grid, slab: Slab) -> Grid:
    """The slab's own grid: its x extent and face kinds, the global spacing."""
    return dataclasses.replace(grid, nx=slab.nx, hx=grid.hx, hy=grid.hy, hz=grid.hz,
                               faces=tuple(slab.faces))


def split_state(f: np.ndarray, slab: Slab) -> np.ndarray:
    """The slab's part of a dense conserved state (5, nz, ny, nx)."""
    return np.ascontiguousarray(f[..., slab.x0:slab.x0 + slab.nx])


def join_state(parts: list[np.ndarray]) -> np.ndarray:
    return np.concatenate(parts, axis=-1)


class CudaSlab:
    """One slab's state and kernels on the current CUDA device: a ws_solver
    over the slab grid, plus its send and receive halo buffers (sized for the
    larger halo; the flux halo uses their leading part)."""

    def __init__(self, grid: Grid, slab: Slab):
        import torch
        self.slab = slab
        self.grid = slab_grid(grid, slab)
        self.solver = Solver(self.grid)
        self.n = {PRIMS: halo_x_bytes(self.grid, HALO_FIELDS) // 8,
                  FLUX: halo_x_bytes(self.grid, FLUX_FIELDS) // 8}
        dev = torch.device("cuda", torch.cuda.current_device())
        self._send = [torch.empty(self.n[PRIMS], dtype=torch.float64, device=dev)
                      for _ in range(2)]
        self._recv = [torch.empty(self.n[PRIMS], dtype=torch.float64, device=dev)
                      for _ in range(2)]
        self.krk = 1     # the stage due next
        self.viscous = False

    def set_viscous(self, vis) -> None:
        self.solver.set_viscous(vis)
        self.viscous = vis is not None

    def set_state(self, f_slab: np.ndarray) -> None:
        self.solver.set_state(f_slab)
        self.krk = 1

    def get_state(self) -> np.ndarray:
        return self.solver.get_state()

    def send(self, side: int, kind: str = PRIMS):
        return self._send[side][:self.n[kind]]

    def recv(self, side: int, kind: str = PRIMS):
        return self._recv[side][:self.n[kind]]

    def _fields(self, kind):
        if kind == PRIMS:
            return self.solver.stage_fields(self.krk)
        return self.solver.stage_flux_fields()

    def pack(self, side: int, kind: str = PRIMS) -> None:
        """Planes next to face `side` of the halo's fields -> send(side, kind)."""
        halo_pack_x(self.grid, self._fields(kind), side, self.send(side, kind))

    def unpack(self, side: int, buf, kind: str = PRIMS) -> None:
        """buf -> ghost planes beyond face `side` of the halo's fields."""
        halo_unpack_x(self.grid, self._fields(kind), side, buf)

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


def _sides(slab: Slab):
    return [s for s, nb in ((LO, slab.left), (HI, slab.right)) if nb is not None]


class LocalExchange:
    """Every slab lives in this process (one or several devices with peer
    access): each slab's ghost planes come straight from its neighbour's
    send buffer; no copy in between."""

    def run(self, runners: list, kind: str = PRIMS) -> None:
        by_index = {r.slab.index: r for r in runners}
        for r in runners:
            for side in _sides(r.slab):
                r.pack(side, kind)
        for r in runners:
            if r.slab.left is not None:
                r.unpack(LO, by_index[r.slab.left].send(HI, kind), kind)
            if r.slab.right is not None:
                r.unpack(HI, by_index[r.slab.right].send(LO, kind), kind)

    def min(self, x: float) -> float:
        return x


class DistExchange:
    """One slab per rank of a torch.distributed group, slab index = group
    rank: point-to-point sends of the packed planes, issued as one batch.
    With NCCL the device buffers go straight over NVLink; with a backend
    that moves host memory only (gloo) device buffers are staged through
    pinned host copies, as the reference stages its packs for MPI.

    Order and tags make a two-slab periodic ring (both neighbours the same
    rank) match as well: sends go low planes first, receives take the high
    ghosts first, and each message is tagged with the side it was packed
    from (0 low, 1 high)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.device_p2p = dist.get_backend(group) == "nccl"
        self._host = {}

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

    def _peer(self, index: int) -> int:
        if self.group is None:
            return index
        return self.dist.get_global_rank(self.group, index)

    def run(self, runners: list, kind: str = PRIMS) -> None:
        dist = self.dist
        if len(runners) != 1:
            raise ValueError("DistExchange runs one slab per rank")
        r = runners[0]
        s = r.slab
        sides = _sides(s)
        for side in sides:
            r.pack(side, kind)
        send = {side: self._staged(r.send(side, kind), ("s", side, kind)) for side in sides}
        recv = {side: self._staged(r.recv(side, kind), ("r", side, kind)) for side in sides}
        for side in sides:
            if send[side] is not r.send(side, kind):
                send[side].copy_(r.send(side, kind))      # synchronous device -> host
        ops = []
        if s.left is not None:
            ops.append(dist.P2POp(dist.isend, send[LO], self._peer(s.left), self.group, LO))
        if s.right is not None:
            ops.append(dist.P2POp(dist.isend, send[HI], self._peer(s.right), self.group, HI))
            ops.append(dist.P2POp(dist.irecv, recv[HI], self._peer(s.right), self.group, LO))
        if s.left is not None:
            ops.append(dist.P2POp(dist.irecv, recv[LO], self._peer(s.left), self.group, HI))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for side in sides:
            buf = r.recv(side, kind)
            if recv[side] is not buf:
                buf.copy_(recv[side], non_blocking=True)  # pinned host -> device, stream-ordered
            r.unpack(side, buf, kind)

    def min(self, x: float) -> float:
        import torch
        dist = self.dist
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        return float(t.item())


class SlabStepper:
    """SSP-RK3 steps of a grid split into x slabs: before each stage the x
    halos of the stage's input are exchanged, then every local slab runs its
    fused stage.  `runners` are this process's slabs."""

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
        """Navier-Stokes on every slab (ws_viscous constants; None: Euler).
        Every rank must make the same choice: it adds an exchange per stage."""
        for r in self.runners:
            r.set_viscous(vis)

    def step(self, dt: float, nsteps: int = 1) -> None:
        if not dt > 0:
            raise ValueError("dt must be > 0")
        for _ in range(nsteps * 3):
            self.stage(dt)

    def compute_dt(self, cfl: float) -> float:
        """Global CFL time step: the minimum of the slabs' (the maximum wave
        speed over the whole grid)."""
        return self.exchange.min(min(r.local_dt(cfl) for r in self.runners))

    def set_state(self, f_global: np.ndarray) -> None:
        for r in self.runners:
            r.set_state(split_state(f_global, r.slab))

    def get_state(self) -> list[np.ndarray]:
        """This process's slabs' states, in slab order."""
        return [r.get_state() for r in self.runners]

    def status(self) -> int:
        return max(r.status() for r in self.runners)

    def close(self) -> None:
        for r in self.runners:
            r.close()


def in_process(grid: Grid, parts: int) -> SlabStepper:
    """All `parts` slabs on the current CUDA device (a single-GPU stand-in
    for a multi-GPU run: same kernels, same halos, no waits between slabs)."""
    return SlabStepper([CudaSlab(grid, s) for s in decompose(grid, parts)], LocalExchange())


def distributed(grid: Grid, group=None) -> SlabStepper:
    """This rank's slab of `grid` split over the ranks of `group` (one GPU
    per rank, the current CUDA device)."""
    import torch.distributed as dist
    parts = dist.get_world_size(group)
    index = dist.get_rank(group)
    slab = decompose(grid, parts)[index]
    return SlabStepper([CudaSlab(grid, slab)], DistExchange(group))
