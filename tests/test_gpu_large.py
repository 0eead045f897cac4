"""A grid whose du holds more than 2^31 elements (64-bit offsets everywhere).

1024x1024x448 periodic, built on the device as 28 copies along z of a
1024x1024x16 periodic state, so its exact RHS is the small grid's RHS
repeated along z: du of the large grid (5 x 448 x 1024 x 1024 = 2.35e9
doubles, 18.8 GB; primitives 5 x 3.9 GB) must equal, bit for bit, the small
grid's du in every copy, and the small grid's du matches the oracle within
the FP64 tolerance.  About 40 GB of device memory.
"""
import numpy as np
import pytest

import windstencil_b200 as ws
from windstencil_b200 import workloads as wl
from tests.conftest import rel_linf
from tests.test_gpu_parity import _case

pytestmark = pytest.mark.gpu
NX, NY, NZ, REPS = 1024, 1024, 16, 28


def test_du_beyond_2_31_elements(oracle, cuda):
    torch = cuda
    h = 1.0 / 255.0
    small = ws.Grid(NX, NY, NZ, hx=h, hy=h, hz=h)
    big = ws.Grid(NX, NY, NZ * REPS, hx=h, hy=h, hz=h)
    assert 5 * big.nz * big.ny * big.nx > 2 ** 31

    # the small grid: device RHS against the oracle on the same primitives
    prims = []

    def keep(torch, g, a):        # device LAP field of a, kept for the large grid
        t = ws.lap_tensor(g)
        t[:, :, :g.nx + 8] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        prims.append(t)
        return t

    out, ref = _case(oracle, torch, small, wl.fourier_state(NX, NY, NZ, seed=21), lap=keep)
    assert rel_linf(out, ref).max() <= 1e-12
    du_small = torch.from_numpy(out).cuda()
    del out, ref

    # the large grid: interior planes repeat the small interior, ghost planes
    # (periodic) are the small grid's
    L = 4
    bigp = []
    for p in prims:
        q = ws.lap_tensor(big)
        q[:L] = p[:L]
        q[L + big.nz:] = p[L + NZ:]
        q[L:L + big.nz] = p[L:L + NZ].repeat(REPS, 1, 1)
        bigp.append(q)
    del prims
    du = torch.empty((5, big.nz, NY, NX), dtype=torch.float64, device="cuda")
    ws.du_invis_jacobian3d(big, ws.interior_job(big), *bigp, du)
    torch.cuda.synchronize()
    assert ws.device_error() == 0
    for r in range(REPS):
        assert torch.equal(du[:, r * NZ:(r + 1) * NZ], du_small), r

