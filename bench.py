#!/usr/bin/env python3
"""Benchmark of the BF3W inviscid RHS on B200 (one JSON line on rank 0).

Workload (default): plain FP64 fused RHS on the 600x128x128 grid of the
benchmark configuration "Plain FP64 fused RHS at 600x128x128 and 480x512x64":
4 ghost cells, periodic in y and z, zero-gradient extrapolation in x, seeded
Sod state (left rho=1, p=1; right rho=0.125, p=0.1; 1% noise), SSP-RK3 at
CFL 0.5.  One bench step = one SSP-RK3 time step = 3 RHS evaluations
(ghost fill -> fused RHS -> stage update, x3), replayed from a CUDA graph.

  value          Gcell-RHS/s = cells x 3 x K / device time of K steps
                 (CUDA events, max over ranks; state 1.2 GB > L2, no flush
                 needed)
  e2e            the same metric through the C ABI with host buffers: every
                 step uploads the conserved state from pinned host memory,
                 steps, and downloads it again
  roofline       the fused RHS kernel alone, timed with CUDA events on its
                 launch stream; algorithmic FLOP = WS_FLOP_PER_CELL x cells;
                 FP64-pipe bound, peak = FP64 FMA throughput measured in this
                 run by a DFMA microkernel (MEASURED_PEAKS.json has no FP64
                 figure); HBM fraction against MEASURED_PEAKS hbm_gbs
  cpu_baseline   the reference's own scalar kernels built for the host
                 (oracle/_ref), else the oracle port, on this machine's cores

--impl reference runs only the CPU reference arm (rank 0) on the same
workload and metric.  --gpus N > 1 runs N independent replicas (one grid per
rank, weak scaling; the single-grid path has no exchange step at one grid per
GPU).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOP_PER_CELL = 7266.0      # oracle.or_op_counts(): algorithmic FLOP per cell-RHS
BYTES_PER_CELL = 80.0       # 5 FP64 primitives in + 5 FP64 du out (Cartesian metrics)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=600)
    ap.add_argument("--ny", type=int, default=128)
    ap.add_argument("--nz", type=int, default=128)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    return ap.parse_args()


def workload_name(a):
    return (f"fp64 fused RHS {a.nx}x{a.ny}x{a.nz}, Sod (rho 1/0.125, p 1/0.1, 1% noise), "
            "x extrapolation, y/z periodic, SSP-RK3 CFL 0.5")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                self.out = ""

    def summary(self):
        if not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.strip().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_arm(a, seconds, reference_preferred=True):
    """Time the CPU inviscid RHS on the workload's grid (bounded sample)."""
    from oracle.oracle import Oracle, RefFunctions, make_grid
    from windstencil_b200 import workloads as wl
    o = Oracle()
    kind = "port"
    rhs = o.du_invis
    if reference_preferred and RefFunctions.available():
        r = RefFunctions()
        rhs = r.du_invis
        kind = "reference"
    og = make_grid(a.nx, a.ny, a.nz, face_kind=(1, 1, 0, 0, 0, 0))
    f = wl.sod_state(a.nx, a.ny, a.nz, seed=2)
    d, u, v, w, T, _ = o.cons_to_prim(og, f)
    for x in (d, u, v, w, T):
        o.ghost_fill(og, x)
    cc = o.sound_speed(og, T)
    cores = o.threads()
    rhs(og, d, u, v, w, cc)         # warm-up (page-in, thread pool)
    n = 0
    t0 = time.perf_counter()
    while True:
        rhs(og, d, u, v, w, cc)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 50:
            break
    value = a.nx * a.ny * a.nz * n / el / 1e9
    sample = (f"{n} full inviscid RHS evaluation(s) of the {a.nx}x{a.ny}x{a.nz} grid in "
              f"{el:.1f} s ({'reference scalar kernels built for the host' if kind == 'reference' else 'oracle port'}, "
              f"OpenMP over {cores} threads)")
    return {"value": value, "unit": "Gcell-RHS/s", "cores": cores, "kind": kind,
            "sample": sample}


def run_reference(a, rank, world):
    if rank != 0:
        return
    from oracle.oracle import Oracle, RefFunctions, make_grid
    from windstencil_b200 import workloads as wl
    o = Oracle()
    kind = "port"
    rhs = o.du_invis
    if RefFunctions.available():
        rhs = RefFunctions().du_invis
        kind = "reference"
    # each step: one inviscid RHS on a 16-plane z-slab of the grid (bounded sample)
    nzs = min(a.nz, 16)
    og = make_grid(a.nx, a.ny, nzs, hz=1.0 / (a.nz - 1.0), face_kind=(1, 1, 0, 0, 0, 0))
    f = wl.sod_state(a.nx, a.ny, nzs, seed=2)
    d, u, v, w, T, _ = o.cons_to_prim(og, f)
    for x in (d, u, v, w, T):
        o.ghost_fill(og, x)
    cc = o.sound_speed(og, T)
    for _ in range(a.warmup):
        rhs(og, d, u, v, w, cc)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        rhs(og, d, u, v, w, cc)
    el = time.perf_counter() - t0
    value = a.nx * a.ny * nzs * a.steps / el / 1e9
    sample = (f"each step: one inviscid RHS on a {a.nx}x{a.ny}x{nzs} slab of the workload "
              f"(same x/y extents, spacing and state recipe)")
    line = {"metric": "Gcell-RHS/s", "value": value, "unit": "Gcell-RHS/s", "impl": "reference",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": el / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(a), "grid": [a.nx, a.ny, a.nz],
                       "inputs_exceed_l2": True},
            "cpu_baseline": {"value": value, "unit": "Gcell-RHS/s", "cores": o.threads(),
                             "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "Gcell-RHS/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(a, rank, world, dist):
    import torch
    import windstencil_b200 as ws
    from windstencil_b200 import workloads as wl

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    prec = ws.MIXED if a.precision == "mixed" else ws.FP64
    faces = (ws.FACE_EXTRAP, ws.FACE_EXTRAP, 0, 0, 0, 0)
    g = ws.Grid(a.nx, a.ny, a.nz, faces=faces, precision=prec)
    cells = g.cells
    f0 = wl.sod_state(a.nx, a.ny, a.nz, seed=2 + rank)
    s = ws.Solver(g)
    stream = torch.cuda.Stream()
    s.set_state(f0, stream=stream)
    dt = s.compute_dt(0.5, stream=stream)

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- whole-job value: K SSP-RK3 steps from the captured graphs
    s.step(dt, a.warmup, stream=stream)
    stream.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        s.step(dt, a.steps, stream=stream)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    status = s.status(stream=stream)
    value = world * cells * 3 * a.steps / (ms * 1e-3) / 1e9

    # ---- dominant kernel alone: the fused RHS through the drop-in entry point
    f_desc, du_desc, prims = s.fields()
    gc = g.c()
    lib = ws.load()
    import ctypes as C
    job = ws.interior_job(g)
    p5 = [prims[0], prims[1], prims[2], prims[3], prims[5]]
    nrhs = max(3, a.steps)
    for _ in range(2):
        ws._abi.check(lib.ws_du_invis_jacobian3d(C.byref(gc), job, *p5, None, du_desc,
                                                 stream.cuda_stream))
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0.record(stream)
    for _ in range(nrhs):
        ws._abi.check(lib.ws_du_invis_jacobian3d(C.byref(gc), job, *p5, None, du_desc,
                                                 stream.cuda_stream))
    k1.record(stream)
    k1.synchronize()
    rhs_ms = k0.elapsed_time(k1) / nrhs
    peak = fp64_peak_tflops(torch, stream)
    achieved = FLOP_PER_CELL * cells / (rhs_ms * 1e-3) / 1e12
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    traffic = measured_traffic(a)
    roof = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if peak else None, "traffic": traffic,
            "kernel": "bf3w_rhs_kernel", "kernel_ms": rhs_ms,
            "peak_source": "DFMA microkernel measured in this run (of measured)",
            "algorithmic_flop_per_cell": FLOP_PER_CELL,
            "algorithmic_bytes_per_cell": BYTES_PER_CELL,
            "hbm_achieved_gbs": BYTES_PER_CELL * cells / (rhs_ms * 1e-3) / 1e9,
            "hbm_peak_gbs": hbm}

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not a.no_e2e:
        host = torch.empty((5, a.nz, a.ny, a.nx), dtype=torch.float64).pin_memory()
        host.copy_(torch.from_numpy(f0))
        hp = host.numpy()
        ptr = hp.ctypes.data
        n_e2e = max(2, min(a.steps, 10))
        for _ in range(1):
            ws._abi.check(lib.ws_solver_set_state(s.h, ptr, stream.cuda_stream))
            s.step(dt, 1, stream=stream)
            ws._abi.check(lib.ws_solver_get_state(s.h, ptr, stream.cuda_stream))
        barrier()
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        q0.record(stream)
        for _ in range(n_e2e):
            ws._abi.check(lib.ws_solver_set_state(s.h, ptr, stream.cuda_stream))
            s.step(dt, 1, stream=stream)
            ws._abi.check(lib.ws_solver_get_state(s.h, ptr, stream.cuda_stream))
        q1.record(stream)
        q1.synchronize()
        wall = time.perf_counter() - w0
        ems = q0.elapsed_time(q1)
        if dist is not None:
            t = torch.tensor([ems], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        nbytes = 5 * cells * 8
        e2e = {"value": world * cells * 3 * n_e2e / (ems * 1e-3) / 1e9, "unit": "Gcell-RHS/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "steps": n_e2e, "wall_s": wall,
               "note": "every step: pinned host state -> device, one SSP-RK3 step, "
                       "state -> pinned host, through ws_solver_set_state/step/get_state"}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_arm(a, a.cpu_seconds)

    s.close()
    if rank == 0:
        line = {"metric": "Gcell-RHS/s", "value": value, "unit": "Gcell-RHS/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if prec == ws.FP64 else "f64 state / f32 flux",
                "data": "synthetic",
                "config": {"workload": workload_name(a) if prec == ws.FP64 else
                           workload_name(a).replace("fp64", "mixed"),
                           "grid": [a.nx, a.ny, a.nz], "rhs_per_step": 3, "cfl": 0.5,
                           "dt": dt, "inputs_exceed_l2": True,
                           "parallelism": f"replicas{world}"},
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": 9 * a.steps, "clocks": clk.summary(),
                "device_status": status}
        print(json.dumps(line), flush=True)


_PEAK = None


def fp64_peak_tflops(torch, stream):
    import ctypes as C
    import windstencil_b200 as ws
    lib = ws.load()
    if not hasattr(lib, "ws_probe_fp64_peak"):
        return None
    lib.ws_probe_fp64_peak.restype = C.c_int
    lib.ws_probe_fp64_peak.argtypes = [C.POINTER(C.c_double), C.c_void_p]
    out = C.c_double()
    ws._abi.check(lib.ws_probe_fp64_peak(C.byref(out), stream.cuda_stream))
    return out.value


def measured_traffic(a):
    """DRAM bytes per RHS launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "bf3w_rhs_fp64_600x128x128.json")
    try:
        d = json.load(open(p))
        if d.get("grid") == [a.nx, a.ny, a.nz]:
            return d.get("dram_bytes_per_launch")
    except Exception:
        pass
    return None


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist_
        if a.impl == "ours":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
            dist_.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        else:
            dist_.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
        dist = dist_
    try:
        if a.impl == "reference":
            run_reference(a, rank, world)
        else:
            run_ours(a, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
