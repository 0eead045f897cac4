"""Small profiling case for the fused RHS kernels.

Runs one fused-RHS evaluation per requested precision on a Sod state
(x extrapolation, y/z periodic) through the one-grid solver and, with
--step, one SSP-RK3 step after it (three launches of the RHS with the stage
epilogue), so that a profiler can capture exactly those launches, e.g.

    ncu --set full --clock-control none -k regex:bf3w_rhs -c 2 -o prof \
        python -m windstencil_b200.profile_case --nx 600 --ny 128 --nz 64

The default 600x128x64 case holds ~1 GB on the device and its inputs exceed
the 126 MB L2, so DRAM counters stay meaningful.  --viscous N adds N
evaluations of the viscous terms (ws_du_vis_jacobian3d, CD8, Re 1e4) on the
FP64 grid: the flux pass, the flux ghost fill and the divergence pass.
--batch N instead steps N grids of the batched workload (nx log-uniform in
[32, 256], ny, nz in [16, 128], periodic) together, one SSP-RK3 step per
precision after one warm-up step: three launches each of the batched ghost
fill and of the batched RHS + stage kernel.
"""
from __future__ import annotations

import argparse
import ctypes as C


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=600)
    ap.add_argument("--ny", type=int, default=128)
    ap.add_argument("--nz", type=int, default=64)
    ap.add_argument("--precision", default="fp64,mixed")
    ap.add_argument("--tile", default="", help="tile_x,tile_y,scan_z,threads")
    ap.add_argument("--step", action="store_true", help="also one SSP-RK3 step")
    ap.add_argument("--viscous", type=int, default=0, help="viscous-term evaluations")
    ap.add_argument("--batch", type=int, default=0, help="grids of the batched workload")
    a = ap.parse_args()

    import torch

    import windstencil_b200 as ws
    from windstencil_b200 import workloads as wl

    if a.batch:
        _batch(a, ws, wl)
        return
    f0 = wl.sod_state(a.nx, a.ny, a.nz, seed=2)
    for name in a.precision.split(","):
        prec = ws.MIXED if name == "mixed" else ws.FP64
        g = ws.Grid(a.nx, a.ny, a.nz, faces=(1, 1, 0, 0, 0, 0), precision=prec)
        s = ws.Solver(g)
        if a.tile:
            s.set_tile(tuple(int(v) for v in a.tile.split(",")))
        s.set_state(f0)
        s.rhs()
        if a.step:
            s.step(s.compute_dt(0.5), 1)
        if a.viscous and prec == ws.FP64:
            _, du, prims = s.fields()     # descriptors of the solver's state
            lib, gc = ws.load(), g.c()
            need = int(lib.ws_du_vis_workspace_bytes(C.byref(gc)))
            work = torch.zeros(need // 8 + 2, dtype=torch.float64, device="cuda")
            vis = ws.viscous(re=1.0e4, pr=0.72, ref_t=288.15, scheme=8)
            for _ in range(a.viscous):
                ws.check(lib.ws_du_vis_jacobian3d(
                    C.byref(gc), C.byref(vis), prims[1], prims[2], prims[3], prims[4], None,
                    du, C.c_void_p(work.data_ptr()), work.numel() * 8,
                    torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        s.close()
    print("ok")


def _batch(a, ws, wl) -> None:
    import torch
    specs = wl.batch_specs(a.batch, seed=4)
    states = [wl.batch_state(sp) for sp in specs]
    for name in a.precision.split(","):
        prec = ws.MIXED if name == "mixed" else ws.FP64
        b = ws.Batch([ws.Grid(sp.nx, sp.ny, sp.nz, precision=prec) for sp in specs])
        if a.tile:
            b.set_tile(tuple(int(v) for v in a.tile.split(",")))
        for i, f in enumerate(states):
            b.set_state(i, f)
        b.set_dt(b.compute_dt(0.5))
        b.step(1)
        b.step(1)
        torch.cuda.synchronize()
        b.close()
    print("ok")


if __name__ == "__main__":
    main()
