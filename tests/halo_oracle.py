"""A slab of windstencil_b200.halo stepped by the CPU oracle (test checker).

OracleSlab has CudaSlab's methods (pack / unpack / stage / local_dt /
set_state / get_state / status), so SlabStepper, LocalExchange and
DistExchange run unchanged over it: on gloo ranks on the CPU, the
decomposition, the exchange pattern and the stage sequence of the
multi-GPU path are checked against the oracle on the whole grid.

Each stage follows the oracle's rhs_from_cons (oracle/oracle.cpp): prims of
the stage's state, ghost fill of d, u, v, w, T (EXTERNAL x faces keep the
unpacked halo), cc = sqrt(T)/ama on the padded field, inviscid RHS, SSP-RK3
update (OCFD_time.cpp:15-65).
"""
from __future__ import annotations

import numpy as np
import torch

from oracle.oracle import make_grid as or_make_grid
from windstencil_b200.halo import HALO_FIELDS, Slab, slab_grid

L = 4


class OracleSlab:
    def __init__(self, oracle, grid, slab: Slab):
        self.o = oracle
        self.slab = slab
        g = slab_grid(grid, slab)
        self.grid = g
        self.og = or_make_grid(g.nx, g.ny, g.nz, hx=g.hx, hy=g.hy, hz=g.hz, gamma=g.gamma,
                               ama=g.ama, epsl_sw=g.epsl_sw, face_kind=g.faces)
        n = HALO_FIELDS * g.nz * g.ny * 4
        self.send = [torch.zeros(n, dtype=torch.float64) for _ in range(2)]
        self.recv = [torch.zeros(n, dtype=torch.float64) for _ in range(2)]
        self.f = None
        self.fn = None
        self.prims = None
        self.krk = 1

    def set_state(self, f_slab):
        self.f = np.array(f_slab, dtype=np.float64, order="C", copy=True)
        self.prims = None
        self.krk = 1

    def get_state(self):
        return self.f.copy()

    def _inputs(self):
        if self.prims is None:
            d, u, v, w, T, _ = self.o.cons_to_prim(self.og, self.f)
            cc = self.o.sound_speed(self.og, T)
            self.prims = [d, u, v, w, T, cc]
        return self.prims

    def _planes(self, side, ghost):
        g = self.grid
        if ghost:
            x0 = 0 if side == 0 else g.nx + L
        else:
            x0 = L if side == 0 else g.nx
        return (slice(L, g.nz + L), slice(L, g.ny + L), slice(x0, x0 + 4))

    def pack(self, side):
        sl = self._planes(side, ghost=False)
        buf = np.stack([p[sl] for p in self._inputs()])
        self.send[side].copy_(torch.from_numpy(buf.reshape(-1)))

    def unpack(self, side, buf):
        g = self.grid
        b = buf.cpu().numpy().reshape(HALO_FIELDS, g.nz, g.ny, 4)
        sl = self._planes(side, ghost=True)
        for q, p in enumerate(self._inputs()):
            p[sl] = b[q]

    def stage(self, dt):
        d, u, v, w, T, _ = self._inputs()
        if self.krk == 1:
            self.fn = self.f.copy()
        for p in (d, u, v, w, T):
            self.o.ghost_fill(self.og, p)
        cc = self.o.sound_speed(self.og, T)
        du = self.o.du_invis(self.og, d, u, v, w, cc)
        self.o.time_advance(self.krk, dt, self.f, self.fn, du)
        self.prims = None
        self.krk = self.krk % 3 + 1

    def local_dt(self, cfl):
        return self.o.compute_dt(self.og, self.f, cfl)

    def status(self):
        return 0

    def close(self):
        pass
