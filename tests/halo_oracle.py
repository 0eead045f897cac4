"""A block of windstencil_b200.halo stepped by the CPU oracle (test checker).

OracleSlab has CudaBlock's methods (send / recv / pack / unpack / begin /
end / local_dt / set_state / get_state / set_viscous / status), so
SlabStepper, LocalExchange and DistExchange run unchanged over it: on gloo
ranks on the CPU, the decomposition, the exchange pattern and the stage
sequence of the multi-GPU path are checked against the oracle on the whole
grid.

Each stage follows the oracle's rhs_from_cons (oracle/oracle.cpp): prims of
the stage's state, ghost fill of d, u, v, w, T (EXTERNAL faces keep the
unpacked halo), cc = sqrt(T)/ama on the padded field, inviscid RHS; with
viscous terms the 12 flux fields, each direction's fluxes' halo along its
axis, and per direction the flux ghost fill and divergence added to du;
then the SSP-RK3 update (OCFD_time.cpp:15-65).
"""
from __future__ import annotations

import numpy as np
import torch

from oracle.oracle import make_grid as or_make_grid
from oracle.oracle import make_vis
from windstencil_b200.halo import FLUX, HALO_FIELDS, PRIMS, Block, block_grid

L = 4


class OracleSlab:
    def __init__(self, oracle, grid, block: Block):
        self.o = oracle
        self.slab = self.block = block
        g = block_grid(grid, block)
        self.grid = g
        self.og = or_make_grid(g.nx, g.ny, g.nz, hx=g.hx, hy=g.hy, hz=g.hz, gamma=g.gamma,
                               ama=g.ama, epsl_sw=g.epsl_sw, face_kind=g.faces)
        n = (g.nx, g.ny, g.nz)
        self.n, self._send, self._recv = {}, {}, {}
        for ax in range(3):
            plane = 4 * n[(ax + 1) % 3] * n[(ax + 2) % 3]
            self.n[ax, PRIMS] = HALO_FIELDS * plane
            self.n[ax, FLUX] = 4 * plane
            self._send[ax] = [torch.zeros(self.n[ax, PRIMS], dtype=torch.float64)
                              for _ in range(2)]
            self._recv[ax] = [torch.zeros(self.n[ax, PRIMS], dtype=torch.float64)
                              for _ in range(2)]
        self.f = self.fn = self.prims = self.du = self.ev = None
        self.vis = None
        self.viscous = False
        self.krk = 1

    def set_viscous(self, vis):
        """vis: dict of re, pr, ref_t, scheme (as windstencil_b200.viscous) or None."""
        self.vis = make_vis(**vis) if vis is not None else None
        self.viscous = vis is not None

    def set_state(self, f_slab):
        self.f = np.array(f_slab, dtype=np.float64, order="C", copy=True)
        self.prims = None
        self.krk = 1

    def get_state(self):
        return self.f.copy()

    def send(self, axis, side, kind=PRIMS):
        return self._send[axis][side][:self.n[axis, kind]]

    def recv(self, axis, side, kind=PRIMS):
        return self._recv[axis][side][:self.n[axis, kind]]

    def _inputs(self):
        if self.prims is None:
            d, u, v, w, T, _ = self.o.cons_to_prim(self.og, self.f)
            cc = self.o.sound_speed(self.og, T)
            self.prims = [d, u, v, w, T, cc]
        return self.prims

    def _fields(self, axis, kind):
        if kind == PRIMS:
            return self._inputs()
        return [self.ev[4 * axis + q] for q in range(4)]

    def _planes(self, axis, side, ghost):
        """(z, y, x) slices of the 4 planes along `axis` (interior elsewhere)."""
        g = self.grid
        n = (g.nx, g.ny, g.nz)
        if ghost:
            a0 = 0 if side == 0 else n[axis] + L
        else:
            a0 = L if side == 0 else n[axis]
        sl = [slice(a0, a0 + 4) if ax == axis else slice(L, n[ax] + L) for ax in range(3)]
        return (sl[2], sl[1], sl[0])

    def _shape(self, axis, nf):
        g = self.grid
        n = [g.nx, g.ny, g.nz]
        n[axis] = 4
        return (nf, n[2], n[1], n[0])

    def pack(self, axis, side, kind=PRIMS):
        sl = self._planes(axis, side, ghost=False)
        buf = np.stack([p[sl] for p in self._fields(axis, kind)])
        self.send(axis, side, kind).copy_(torch.from_numpy(buf.reshape(-1)))

    def unpack(self, axis, side, buf, kind=PRIMS):
        fields = self._fields(axis, kind)
        b = buf.cpu().numpy().reshape(self._shape(axis, len(fields)))
        sl = self._planes(axis, side, ghost=True)
        for q, p in enumerate(fields):
            p[sl] = b[q]

    def begin(self):
        d, u, v, w, T, _ = self._inputs()
        if self.krk == 1:
            self.fn = self.f.copy()
        for p in (d, u, v, w, T):
            self.o.ghost_fill(self.og, p)
        cc = self.o.sound_speed(self.og, T)
        self.du = self.o.du_invis(self.og, d, u, v, w, cc)
        if self.viscous:
            self.ev = self.o.vis_fluxes(self.og, self.vis, u, v, w, T)

    def end(self, dt):
        if self.viscous:     # du_comput: inviscid, then viscous (OCFD_Stream.cpp:27-45)
            for direction in range(3):
                self.o.vis_div_add(self.og, self.vis, direction,
                                   self.ev[4 * direction:4 * direction + 4], self.du)
        self.o.time_advance(self.krk, dt, self.f, self.fn, self.du)
        self.prims = self.du = self.ev = None
        self.krk = self.krk % 3 + 1

    def local_dt(self, cfl):
        return self.o.compute_dt(self.og, self.f, cfl)

    def status(self):
        return 0

    def close(self):
        pass
