#!/usr/bin/env python3
"""Benchmark of the BF3W inviscid RHS on B200 (one JSON line on rank 0).

Headline workload: plain FP64 RHS on the 600x128x128 grid of the benchmark
configuration "Plain FP64 fused RHS at 600x128x128 and 480x512x64": 4 ghost
cells, periodic in y and z, zero-gradient extrapolation in x, seeded Sod
state (left rho=1, p=1; right rho=0.125, p=0.1; 1% noise), SSP-RK3 at CFL
0.5.  One bench step = one SSP-RK3 time step = 3 RHS evaluations, each a
ghost fill and the x, y and z line passes, the last applying the stage update
(12 launches), replayed from a CUDA graph.

  value          Gcell-RHS/s = cells x 3 x K / device time of K steps
                 (CUDA events, max over ranks; the state is 1.2 GB > L2, so
                 no flush is needed)
  e2e            the same metric through the C ABI with host buffers: every
                 step uploads the conserved state from pinned host memory,
                 steps, and downloads it again
  roofline       one RHS (the three line passes) through the drop-in entry
                 point, timed with CUDA events on its launch stream;
                 algorithmic FLOP = 7266 per cell (the oracle's operation
                 count); FP64-pipe bound, peak = FP64 FMA throughput measured
                 in this run by a DFMA microkernel (MEASURED_PEAKS.json has no
                 FP64 figure); the HBM side uses MEASURED_PEAKS hbm_gbs
  cpu_baseline   the reference's own scalar kernels built for the host
                 (oracle/_ref), else the oracle port, on this machine's cores:
                 whole SSP-RK3 steps of the same grid
  mixed          the mixed-precision form on the 600x128x128 Fourier
                 workload: speed-up over FP64 (RHS and step), state error
                 after 100 steps (rel. L2 / L-inf per conserved field), and
                 its roofline against the FP32 FMA peak measured in this run
  grid_480x512x64  the second size of the FP64 workload: RHS alone (both
                 forms) and whole SSP-RK3 steps
  navier_stokes  the headline grid with the viscous terms added (CD8,
                 Re 1e4): whole SSP-RK3 steps and the viscous terms alone
  batched        256 uneven periodic grids, 50 SSP-RK3 steps, FP64 and mixed,
                 against one-grid-at-a-time FP64 solves of the same grids
                 (device time, and per request end to end)
  served         Poisson arrivals of solve requests into the continuous-
                 batching server; p50/p99 latency and served throughput

--impl reference runs only the CPU reference arm (rank 0): whole SSP-RK3
steps of the headline grid with the reference's own scalar kernels, on the
same config and metric.  --gpus N > 1 (one rank per GPU under torchrun)
steps one grid split into N blocks of nx x ny x nz, one per GPU (x slabs, or
the process grid --dims px,py,pz), with the halos exchanged over NCCL before
every RK stage (weak scaling: each GPU keeps the single-GPU workload's cells).
--profile-case runs a short fixed launch sequence for a profiler instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOP_PER_CELL = 7266.0      # oracle or_op_counts(): algorithmic FLOP per cell-RHS
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
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-second", action="store_true")
    ap.add_argument("--no-ns", action="store_true")
    ap.add_argument("--no-slabs", action="store_true")
    ap.add_argument("--dims", default="",
                    help="with --gpus N > 1: the process grid px,py,pz (product N); "
                         "default N,1,1 (x slabs)")
    ap.add_argument("--backend", default="nccl", choices=["nccl", "gloo"],
                    help="process group of --gpus N > 1; gloo stages the halos through "
                         "host memory, so ranks may share a GPU (a test of the "
                         "multi-rank path on one device)")
    ap.add_argument("--halo", default="torch", choices=["torch", "native"],
                    help="with --gpus N > 1: the stage sequence in Python with the halos "
                         "over torch.distributed (torch), or the library's C++ stepper "
                         "with its own NCCL communicator (native; needs --backend nccl)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--batch-grids", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=50)
    ap.add_argument("--serial-grids", type=int, default=32)
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-rate-low", type=float, default=6.0)
    ap.add_argument("--serve-seconds", type=float, default=60.0)    # the configuration's window
    ap.add_argument("--serve-drain", type=float, default=20.0)
    # --profile-case: a short fixed sequence of launches for ncu (no timing)
    ap.add_argument("--profile-case", action="store_true",
                    help="run a small profiling case instead of the benchmark: one fused "
                         "RHS per --precision on the Sod grid --nx --ny --nz (and with "
                         "--step one SSP-RK3 step, with --viscous N that many viscous-term "
                         "evaluations); with --profile-batch N, one warm-up and one timed "
                         "SSP-RK3 step of N grids of the batched workload per precision")
    ap.add_argument("--precision", default="fp64,mixed")
    ap.add_argument("--tile", default="", help="tile_x,tile_y,scan_z,threads")
    ap.add_argument("--step", action="store_true")
    ap.add_argument("--viscous", type=int, default=0)
    ap.add_argument("--profile-batch", type=int, default=0)
    return ap.parse_args()


def process_dims(a, world):
    """The process grid of a multi-GPU run: --dims px,py,pz, else N x 1 x 1."""
    if a.dims:
        d = tuple(int(v) for v in a.dims.split(","))
        if len(d) != 3 or d[0] * d[1] * d[2] != world:
            raise SystemExit(f"--dims {a.dims} does not match {world} GPUs")
        return d
    return (world, 1, 1)


def workload_name(a, world=1):
    if world == 1:
        return (f"fp64 fused RHS {a.nx}x{a.ny}x{a.nz}, Sod (rho 1/0.125, p 1/0.1, 1% noise), "
                "x extrapolation, y/z periodic, SSP-RK3 CFL 0.5")
    d = process_dims(a, world)
    return (f"fp64 fused RHS {a.nx * d[0]}x{a.ny * d[1]}x{a.nz * d[2]} split into "
            f"{d[0]}x{d[1]}x{d[2]} blocks of {a.nx}x{a.ny}x{a.nz} (one per GPU, halos "
            "exchanged over NCCL every RK stage), Sod per block (rho 1/0.125, p 1/0.1, "
            "1% noise), x extrapolation, y/z periodic, SSP-RK3 CFL 0.5")


L2_BYTES = 126e6                # B200 L2


def config_of(a, world, **kw):
    # per GPU, the five primitive LAP fields a step reads (plus f, fn, du)
    prim_bytes = 5 * 8 * (a.nx + 8) * (a.ny + 8) * (a.nz + 8)
    d = process_dims(a, world) if world > 1 else (1, 1, 1)
    c = {"workload": workload_name(a, world),
         "grid": [a.nx * d[0], a.ny * d[1], a.nz * d[2]],
         "grid_per_gpu": [a.nx, a.ny, a.nz], "rhs_per_step": 3, "cfl": 0.5,
         "inputs_exceed_l2": prim_bytes > L2_BYTES,
         "parallelism": "single" if world == 1 else "blocks%dx%dx%d" % d}
    c.update(kw)
    return c


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
        sm, smax, pw, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.strip().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
                pw.append(float(p[3]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(pw) if pw else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU arms (the oracle is the checker / reported baseline, never the product)
# ---------------------------------------------------------------------------
def _cpu_stepper(nx, ny, nz):
    """The headline workload stepped on the host: SSP-RK3 steps assembled from
    the reference's own scalar kernels (oracle/_ref, kind "reference"), else
    the oracle port's own step (kind "port")."""
    from oracle.oracle import Oracle, RefFunctions, RefRK3, make_grid
    from windstencil_b200 import workloads as wl
    o = Oracle()
    og = make_grid(nx, ny, nz, face_kind=(1, 1, 0, 0, 0, 0))
    f = wl.sod_state(nx, ny, nz, seed=2)
    dt = o.compute_dt(og, f, 0.5)
    if RefFunctions.available():
        st = RefRK3(og, f, oracle=o)
        return o, "reference", (lambda: st.step(dt)), dt
    state = {"f": f}

    def port_step():
        state["f"] = o.rk3_steps(og, state["f"], dt, 1)
    return o, "port", port_step, dt


def cpu_arm(a, seconds):
    """Bounded sample: whole SSP-RK3 steps of the headline grid for ~`seconds`."""
    o, kind, step, _ = _cpu_stepper(a.nx, a.ny, a.nz)
    step()                          # warm-up (page-in, thread pool)
    n, t0 = 0, time.perf_counter()
    while True:
        step()
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 20:
            break
    what = ("reference scalar kernels built for the host" if kind == "reference"
            else "oracle port")
    return {"value": a.nx * a.ny * a.nz * 3 * n / el / 1e9, "unit": "Gcell-RHS/s",
            "cores": o.threads(), "kind": kind,
            "sample": f"{n} SSP-RK3 step(s) (3 inviscid RHS each) of the {a.nx}x{a.ny}x{a.nz} "
                      f"grid in {el:.1f} s ({what}, OpenMP over {o.threads()} threads)"}


def run_reference(a, rank, world):
    """The reference arm: the headline workload's SSP-RK3 steps on the host
    cores, one bench step = one time step (3 RHS evaluations and the stage
    updates), on the same grid, state, dt and metric as the GPU arm."""
    if rank != 0:
        return
    o, kind, step, dt = _cpu_stepper(a.nx, a.ny, a.nz)
    for _ in range(a.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        step()
    el = time.perf_counter() - t0
    value = a.nx * a.ny * a.nz * 3 * a.steps / el / 1e9
    what = ("the reference's own scalar kernels built for the host (cons_to_pri, sound "
            "speed, Steger-Warming split, WENO7-SYMBO P/M, time advance ker1/2/3), "
            "decomposed RHS loop, OpenMP" if kind == "reference" else "the oracle port")
    sample = (f"each step: one whole SSP-RK3 time step of the {a.nx}x{a.ny}x{a.nz} grid "
              f"(3 inviscid RHS + stage updates) with {what}")
    line = {"metric": "Gcell-RHS/s", "value": value, "unit": "Gcell-RHS/s", "impl": "reference",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": el / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(a, world), "dt": dt,
            "cpu_baseline": {"value": value, "unit": "Gcell-RHS/s", "cores": o.threads(),
                             "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "Gcell-RHS/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arms
# ---------------------------------------------------------------------------
def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _peak(ws, name):
    """Attainable FMA throughput (TFLOP/s) measured now by the measurement
    utility libws_peaks.so (name: "fp64" or "fp32")."""
    import ctypes as C
    lib = C.CDLL(os.path.join(ROOT, "windstencil_b200", "libws_peaks.so"))
    fn = getattr(lib, f"wsp_{name}_fma_peak")
    fn.argtypes = [C.POINTER(C.c_double), C.c_void_p]
    fn.restype = C.c_int
    out = C.c_double()
    rc = fn(C.byref(out), None)
    if rc != 0:
        raise RuntimeError(f"FMA peak measurement failed (CUDA error {rc})")
    return out.value


def time_rhs_kernel(torch, ws, g, solver, stream, reps):
    """Mean device time of one RHS (the line passes, the default kernel) through
    the drop-in entry point."""
    import ctypes as C
    _, du_desc, prims = solver.fields()
    gc = g.c()
    lib = ws.load()
    job = ws.interior_job(g)
    p5 = [prims[0], prims[1], prims[2], prims[3], prims[5]]
    call = lambda: ws._abi.check(lib.ws_du_invis_jacobian3d(   # noqa: E731
        C.byref(gc), job, *p5, None, du_desc, stream.cuda_stream))
    for _ in range(2):
        call()
    e0, e1 = _events(torch)
    e0.record(stream)
    for _ in range(reps):
        call()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def bench_mixed(a, torch, ws, wl, stream):
    """Mixed form vs FP64 on the 600x128x128 Fourier workload, 100 steps."""
    nx, ny, nz = a.nx, a.ny, a.nz
    f0 = wl.fourier_state(nx, ny, nz, seed=1)
    res = {"workload": f"{nx}x{ny}x{nz} periodic Fourier state with contact, 100 SSP-RK3 "
                       "steps at CFL 0.5",
           "error_measure": "per conserved field: rel. L2 = |a-b|_2/|b|_2, "
                            "rel. L-inf = max|a-b|/max|b|, mixed vs FP64 on this GPU"}
    out = {}
    for name, prec in (("fp64", ws.FP64), ("mixed", ws.MIXED)):
        g = ws.Grid(nx, ny, nz, precision=prec)
        s = ws.Solver(g)
        s.set_state(f0, stream=stream)
        if name == "fp64":
            dt = s.compute_dt(0.5, stream=stream)
        out[name + "_kernel_ms"] = time_rhs_kernel(torch, ws, g, s, stream, 10)
        s.step(dt, 2, stream=stream)
        s.set_state(f0, stream=stream)
        e0, e1 = _events(torch)
        e0.record(stream)
        s.step(dt, 100, stream=stream)
        e1.record(stream)
        e1.synchronize()
        out[name + "_step_ms"] = e0.elapsed_time(e1) / 100
        out[name + "_state"] = s.get_state(stream=stream)
        s.close()
    a64, a32 = out["fp64_state"], out["mixed_state"]
    l2 = [float(np.linalg.norm(a32[i] - a64[i]) / np.linalg.norm(a64[i])) for i in range(5)]
    li = [float(np.max(np.abs(a32[i] - a64[i])) / np.max(np.abs(a64[i]))) for i in range(5)]
    cells = nx * ny * nz
    peak32 = _peak(ws, "fp32")
    res.update({
        "kernel_ms_fp64": out["fp64_kernel_ms"], "kernel_ms_mixed": out["mixed_kernel_ms"],
        "kernel_speedup_vs_fp64": out["fp64_kernel_ms"] / out["mixed_kernel_ms"],
        "value": cells * 3 / (out["mixed_step_ms"] * 1e-3) / 1e9,
        "value_fp64_same_workload": cells * 3 / (out["fp64_step_ms"] * 1e-3) / 1e9,
        "unit": "Gcell-RHS/s",
        "step_speedup_vs_fp64": out["fp64_step_ms"] / out["mixed_step_ms"],
        "state_rel_l2": l2, "state_rel_linf": li, "max_rel_l2": max(l2),
        "fp32_peak_tflops_measured": peak32,
        "rhs_gcell_s": cells / (out["mixed_kernel_ms"] * 1e-3) / 1e9})
    # the mixed RHS against the FP32 FMA peak measured now (its reconstruction
    # runs as packed FP32x2 FMAs; the face difference and stage stay FP64)
    ach = FLOP_PER_CELL * cells / (out["mixed_kernel_ms"] * 1e-3) / 1e12
    res["roofline"] = {"bound": "fp32", "achieved": ach, "peak": peak32, "unit": "TFLOP/s",
                       "frac": ach / peak32 if peak32 else None,
                       "kernel": "line passes x, y, z (mixed form), one RHS",
                       "kernel_ms": out["mixed_kernel_ms"],
                       "peak_source": "FP32 FMA microkernel measured in this run (of measured)",
                       "algorithmic_flop_per_cell": FLOP_PER_CELL}
    return res


def bench_second_grid(a, torch, ws, wl, stream, peak64):
    """The second size of the FP64 workload, 480x512x64 (same faces and state
    recipe): the RHS kernel alone in both forms and whole SSP-RK3 steps."""
    nx, ny, nz = 480, 512, 64
    cells = nx * ny * nz
    f0 = wl.sod_state(nx, ny, nz, seed=3)
    faces = (ws.FACE_EXTRAP, ws.FACE_EXTRAP, 0, 0, 0, 0)
    res = {"workload": f"{nx}x{ny}x{nz} Sod state, periodic y/z, extrapolation in x"}
    for name, prec in (("fp64", ws.FP64), ("mixed", ws.MIXED)):
        g = ws.Grid(nx, ny, nz, faces=faces, precision=prec)
        s = ws.Solver(g)
        s.set_state(f0, stream=stream)
        dt = s.compute_dt(0.5, stream=stream)
        kms = time_rhs_kernel(torch, ws, g, s, stream, 10)
        s.step(dt, 3, stream=stream)
        e0, e1 = _events(torch)
        e0.record(stream)
        s.step(dt, 20, stream=stream)
        e1.record(stream)
        e1.synchronize()
        sms = e0.elapsed_time(e1) / 20
        s.close()
        tf = FLOP_PER_CELL * cells / (kms * 1e-3) / 1e12
        res[name] = {"kernel_ms": kms, "rhs_gcell_s": cells / (kms * 1e-3) / 1e9,
                     "step_ms": sms, "value": cells * 3 / (sms * 1e-3) / 1e9,
                     "unit": "Gcell-RHS/s", "achieved_tflops": tf}
        if name == "fp64":
            res[name]["frac_of_fp64_peak"] = tf / peak64 if peak64 else None
    res["kernel_speedup_mixed_vs_fp64"] = res["fp64"]["kernel_ms"] / res["mixed"]["kernel_ms"]
    return res


def bench_slabs_one_gpu(a, torch, ws, wl, stream, parts=2):
    """The multi-GPU path's per-stage work on one GPU: a (parts*nx) x ny x nz
    grid split into `parts` x slabs, all on this GPU (halo pack, hand-over
    in process, unpack, ghost fill, fused stage per slab and stage, launched
    eagerly), against the same grid stepped whole from its graphs."""
    from windstencil_b200 import halo
    faces = (ws.FACE_EXTRAP, ws.FACE_EXTRAP, 0, 0, 0, 0)
    g = ws.Grid(a.nx * parts, a.ny, a.nz, faces=faces)
    f0 = wl.sod_state(g.nx, g.ny, g.nz, seed=12)
    steps = max(3, min(a.steps, 20))
    whole = ws.Solver(g)
    whole.set_state(f0, stream=stream)
    dt = whole.compute_dt(0.5, stream=stream)
    whole.step(dt, 3, stream=stream)
    e0, e1 = _events(torch)
    e0.record(stream)
    whole.step(dt, steps, stream=stream)
    e1.record(stream)
    e1.synchronize()
    ms_whole = e0.elapsed_time(e1) / steps
    whole.close()
    with torch.cuda.stream(stream):
        st = halo.in_process(g, parts)
        st.set_state(f0)
        st.step(dt, 3)
        e0.record(stream)
        st.step(dt, steps)
        e1.record(stream)
    e1.synchronize()
    ms_slabs = e0.elapsed_time(e1) / steps
    status = st.status()
    st.close()
    return {"workload": f"{g.nx}x{g.ny}x{g.nz} Sod, x extrapolation, split into {parts} x "
                        f"slabs of {a.nx}x{a.ny}x{a.nz} on one GPU",
            "steps": steps, "step_ms_whole_grid": ms_whole, "step_ms_slabs": ms_slabs,
            "slab_overhead": ms_slabs / ms_whole - 1.0,
            "halo_bytes_per_stage_per_face": ws.halo_x_bytes(g, halo.HALO_FIELDS),
            "device_status": status,
            "stepper": "C++ (ws_blocks_step: decomposition, pack, exchange, unpack and "
                       "stages in the library)",
            "note": "slabs: per stage per slab a halo pack and unpack per shared face, "
                    "ghost fill, RHS line passes with the stage; the exchange between GPUs (NCCL) is "
                    "not in this number"}


def bench_navier_stokes(a, torch, ws, wl, stream):
    """Navier-Stokes (inviscid + viscous terms, CD8, Re 1e4) on the headline
    grid: whole SSP-RK3 steps, and the viscous terms alone through the
    drop-in entry point.  Re 1e4 keeps the viscous stability limit of the
    0.5-CFL convective time step (dx = 1/599) from binding."""
    nx, ny, nz = a.nx, a.ny, a.nz
    cells = nx * ny * nz
    vis = dict(re=1.0e4, pr=0.72, ref_t=288.15, scheme=8)
    faces = (ws.FACE_EXTRAP, ws.FACE_EXTRAP, 0, 0, 0, 0)
    g = ws.Grid(nx, ny, nz, faces=faces)
    f0 = wl.sod_state(nx, ny, nz, seed=2)
    s = ws.Solver(g)
    s.set_viscous(vis)
    s.set_state(f0, stream=stream)
    dt = s.compute_dt(0.5, stream=stream)
    s.step(dt, 3, stream=stream)
    e0, e1 = _events(torch)
    e0.record(stream)
    s.step(dt, 20, stream=stream)
    e1.record(stream)
    e1.synchronize()
    sms = e0.elapsed_time(e1) / 20
    status = s.status(stream=stream)
    # viscous terms alone (drop-in, caller workspace) on the current state
    _, du, prims = s.fields()
    import ctypes as C
    lib = ws.load()
    gc = g.c()
    need = int(lib.ws_du_vis_workspace_bytes(C.byref(gc)))
    work = torch.empty(need // 8 + 2, dtype=torch.float64, device="cuda")
    vp = ws.viscous(**vis)
    call = lambda: ws._abi.check(lib.ws_du_vis_jacobian3d(   # noqa: E731
        C.byref(gc), C.byref(vp), prims[1], prims[2], prims[3], prims[4], None, du,
        C.c_void_p(work.data_ptr()), need + 16, stream.cuda_stream))
    call()
    e0.record(stream)
    for _ in range(10):
        call()
    e1.record(stream)
    e1.synchronize()
    vms = e0.elapsed_time(e1) / 10
    s.close()
    return {"workload": f"{nx}x{ny}x{nz} Sod, Navier-Stokes (Re 1e4, Pr 0.72, Sutherland "
                        "Ref_T 288.15, CD8 viscous derivatives), SSP-RK3 CFL 0.5",
            "value": cells * 3 / (sms * 1e-3) / 1e9, "unit": "Gcell-RHS/s", "step_ms": sms,
            "viscous_terms_ms": vms,
            "viscous_hbm_gbs_lower_bound": 224.0 * cells / (vms * 1e-3) / 1e9,
            "note": "viscous_terms_ms: gradients + fluxes pass, flux ghost fill, divergence "
                    "pass through ws_du_vis_jacobian3d; ~224 B/cell of compulsory traffic "
                    "(4 primitives in, 12 fluxes out and in, du[1..4] read and written)",
            "device_status": status}


def bench_batch(a, torch, ws, wl, stream):
    specs = wl.batch_specs(a.batch_grids, seed=4)
    cells = sum(s.cells for s in specs)
    states = [wl.batch_state(s) for s in specs]
    res = {"workload": f"{len(specs)} periodic grids, nx log-U[32,256], ny,nz log-U[16,128], "
                       "Mach U[0.3,3], Sod jump at a seeded x, 1% noise; "
                       f"{a.batch_steps} SSP-RK3 steps at CFL 0.5",
           "grids": len(specs), "cells": cells}
    dts = None
    for name, prec in (("fp64", ws.FP64), ("mixed", ws.MIXED)):
        b = ws.Batch([ws.Grid(s.nx, s.ny, s.nz, precision=prec) for s in specs])
        for i, f in enumerate(states):
            b.set_state(i, f, stream=stream)
        if dts is None:
            dts = b.compute_dt(0.5, stream=stream)
        b.set_dt(dts)
        tile = b.autotune(stream=stream)
        b.step(2, stream=stream)
        for i, f in enumerate(states):       # same stream: ordered after the warm-up
            b.set_state(i, f, stream=stream)
        stream.synchronize()
        e0, e1 = _events(torch)
        e0.record(stream)
        b.step(a.batch_steps, stream=stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        st = b.status()
        b.close()
        pencil = tile[0] < 0
        res[name] = {"value": cells * 3 * a.batch_steps / (ms * 1e-3) / 1e9,
                     "unit": "Gcell-RHS/s", "ms_per_step": ms / a.batch_steps,
                     "tile": list(tile),
                     "kernel": "line passes (x, y, z)" if pencil else "fused tile sweep",
                     "nonfinite_grids": int(sum(1 for x in st if x)),
                     "launches_per_step": 12 if pencil else 6}
    # one grid at a time, FP64, same grids (a sample of them), same steps:
    # device time of the steps alone, and each request end to end (state
    # upload from host memory, dt, the steps, result download; wall clock)
    nser = min(a.serial_grids, len(specs))
    tot_ms, tot_e2e, ser_cells = 0.0, 0.0, 0
    for i in range(nser):
        s = specs[i]
        sol = ws.Solver(ws.Grid(s.nx, s.ny, s.nz))
        sol.set_state(states[i], stream=stream)
        sol.step(dts[i], 1, stream=stream)
        sol.set_state(states[i], stream=stream)
        e0, e1 = _events(torch)
        e0.record(stream)
        sol.step(dts[i], a.batch_steps, stream=stream)
        e1.record(stream)
        e1.synchronize()
        tot_ms += e0.elapsed_time(e1)
        t0 = time.perf_counter()
        sol.set_state(states[i], stream=stream)
        dt_i = sol.compute_dt(0.5, stream=stream)
        sol.step(dt_i, a.batch_steps, stream=stream)
        sol.get_state(stream=stream)
        tot_e2e += time.perf_counter() - t0
        ser_cells += s.cells
        sol.close()
    serial = ser_cells * 3 * a.batch_steps / (tot_ms * 1e-3) / 1e9
    res["one_grid_at_a_time_fp64"] = {
        "value": serial, "unit": "Gcell-RHS/s",
        "sample": f"grids 0..{nser - 1} of the batch, each solved alone with ws_solver "
                  f"({a.batch_steps} steps, graph-captured; device time of the steps)"}
    res["one_grid_at_a_time_fp64_per_request"] = {
        "value": ser_cells * 3 * a.batch_steps / tot_e2e / 1e9, "unit": "Gcell-RHS/s",
        "sample": f"the same grids, each request end to end on the host clock: state upload "
                  f"from host memory, CFL dt, {a.batch_steps} steps, state download (solver "
                  "created beforehand)"}
    res["speedup_fp64_vs_per_request"] = res["fp64"]["value"] / \
        res["one_grid_at_a_time_fp64_per_request"]["value"]
    res["speedup_fp64_vs_one_at_a_time"] = res["fp64"]["value"] / serial
    res["speedup_mixed_vs_one_at_a_time"] = res["mixed"]["value"] / serial
    return res, serial


def bench_serve(a, ws, wl, serial_rate, rate, seconds, drain, seed=5, host_io=False):
    """Poisson arrivals into the continuous-batching server (bounded run).
    host_io: every request uploads its initial state from host memory and
    copies its final state back (latency includes both); else the initial
    state is generated on the device and no result is copied."""
    rng = np.random.default_rng(seed)
    specs = wl.batch_specs(int(rate * seconds * 1.2) + 16, seed=seed)
    pool = []
    if host_io:         # a pool of host states, reused in turn (grid matches state)
        pool = [(sp, wl.batch_state(sp)) for sp in specs[:32]]
    srv = ws.Server(hbm_budget_bytes=80 << 30)
    t0 = time.perf_counter()
    t_next = 0.0
    ids, offered_work = [], 0.0
    pending = []

    def release_done():
        keep = []
        for rid in pending:
            state = srv.poll(rid)[0]
            if state >= 2:              # done or failed: free its host buffers
                srv.release(rid)
            else:
                keep.append(rid)
        pending[:] = keep
    i = 0
    while True:
        now = time.perf_counter() - t0
        if now >= seconds:
            break
        if now < t_next:
            if host_io:
                release_done()
            time.sleep(min(t_next - now, 0.01))
            continue
        s, f0 = pool[i % len(pool)] if host_io else (specs[i % len(specs)], None)
        nsteps = int(rng.integers(50, 501))
        prec = ws.FP64 if rng.random() < 0.5 else ws.MIXED
        g = ws.Grid(s.nx, s.ny, s.nz, precision=prec)
        rid = srv.submit(g, nsteps, cfl=0.5, f0=f0, seed=s.seed, mach=s.mach, x_jump=s.x_jump,
                         want_result=host_io)
        ids.append(rid)
        if host_io:
            pending.append(rid)
        offered_work += 3.0 * nsteps * s.cells
        i += 1
        t_next += rng.exponential(1.0 / rate)
    deadline = time.perf_counter() + drain
    while time.perf_counter() < deadline:
        st = srv.stats()
        if st["completed"] + st["failed"] >= len(ids):
            break
        if host_io:
            release_done()
        time.sleep(0.2)
    st = srv.stats()
    wall = time.perf_counter() - t0
    srv.close()
    served = st["served_cell_rhs"] / wall / 1e9
    executed = st["executed_cell_rhs"] / wall / 1e9
    return {
        "arrivals": "Poisson", "rate_per_s": rate, "arrival_window_s": seconds,
        "offered_requests": len(ids), "completed": st["completed"], "failed": st["failed"],
        "unfinished_at_stop": len(ids) - st["completed"] - st["failed"],
        "wall_s": wall, "p50_latency_s": st["p50_latency_s"],
        "p99_latency_s": st["p99_latency_s"], "mean_latency_s": st["mean_latency_s"],
        "latency_over": ("completed requests (submit -> initial state uploaded from host "
                         "memory, steps, result copied to host memory)" if host_io else
                         "completed requests (submit -> result on the device)"),
        "max_concurrent_grids": st["max_active"], "ticks": st["ticks"],
        "loop_seconds": {k: st[k] for k in ("admit_s", "rebuild_s", "steps_s", "retire_s")},
        "offered_gcell_rhs_s": offered_work / seconds / 1e9,
        "served_gcell_rhs_s": served, "executed_gcell_rhs_s": executed, "unit": "Gcell-RHS/s",
        "served_vs_one_at_a_time_fp64": served / serial_rate if serial_rate else None,
        "executed_vs_one_at_a_time_fp64": executed / serial_rate if serial_rate else None,
        "requests": "grid as the batched workload, steps U[50,500], FP64 or mixed 50/50, "
                    "80 GiB state budget, " +
                    ("initial states from a pool of 32 host states (seeded), results copied "
                     "back" if host_io else "seeded initial state generated on the device"),
        "note": "admission: FIFO under the HBM budget and a 3.2e7 active-cell cap; "
                "arrivals stop at the end of the window, latency percentiles cover the "
                "requests finished by the drain deadline; served counts finished requests' "
                "work, executed all device work in the window"}


def max_over_ranks(torch, dist, x):
    """The maximum of x over the ranks (x itself on one GPU)."""
    if dist is None:
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def pipelined_e2e(a, torch, ws, g, f0, dt, host, cells, n_steps, nsolv=3):
    """The e2e leg with the transfers overlapped: nsolv solvers on their own
    streams take the steps in turn; each step uploads its input state from
    pinned host memory (ws_solver_set_state), takes one SSP-RK3 step and
    downloads its result into its solver's pinned buffer
    (ws_solver_get_state_async), so the solvers' uploads and downloads run on
    the copy engines while another steps (per stream the three are in series,
    hence more than two solvers).  Every step still moves its whole state
    both ways."""
    lib = ws.load()
    st = [torch.cuda.Stream() for _ in range(nsolv)]
    solvers = [ws.Solver(g) for _ in range(nsolv)]
    outs = [torch.empty_like(host).pin_memory() for _ in range(nsolv)]
    inp = host.numpy().ctypes.data
    try:
        def one(i):
            k = i % nsolv
            ws._abi.check(lib.ws_solver_set_state(solvers[k].h, inp, st[k].cuda_stream))
            solvers[k].step(dt, 1, stream=st[k])
            ws._abi.check(lib.ws_solver_get_state_async(
                solvers[k].h, outs[k].numpy().ctypes.data, st[k].cuda_stream))
        for i in range(nsolv):      # graphs captured, buffers touched
            one(i)
        torch.cuda.synchronize()
        q0, q1 = _events(torch)
        w0 = time.perf_counter()
        q0.record(st[0])
        for x in st[1:]:
            x.wait_event(q0)
        steps = nsolv * n_steps
        for i in range(steps):
            one(i)
        for x in st[1:]:
            qb = torch.cuda.Event()
            qb.record(x)
            st[0].wait_event(qb)
        q1.record(st[0])
        q1.synchronize()
        wall = time.perf_counter() - w0
        ms = q0.elapsed_time(q1)
        ok = all(s.status(stream=x) == 0 for s, x in zip(solvers, st))
    finally:
        for s in solvers:
            s.close()
    return {"value": cells * 3 * steps / (ms * 1e-3) / 1e9, "steps": steps,
            "wall_s": wall, "pipelined": True, "solvers": nsolv, "device_status_ok": ok,
            "note": f"{nsolv} solvers on their own streams take the steps in turn; every step: its "
                    "input state pinned host -> device (ws_solver_set_state), one SSP-RK3 "
                    "step, its result device -> its own pinned host buffer "
                    "(ws_solver_get_state_async); one solver's transfers overlap another's "
                    "step. serial_value: the same with one solver, each step waiting for "
                    "its download"}


def run_ours(a, rank, world, dist):
    import torch
    import windstencil_b200 as ws
    from windstencil_b200 import workloads as wl

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local % torch.cuda.device_count())
    faces = (ws.FACE_EXTRAP, ws.FACE_EXTRAP, 0, 0, 0, 0)
    f0 = wl.sod_state(a.nx, a.ny, a.nz, seed=2 + rank)
    stream = torch.cuda.Stream()
    if world == 1:
        # one grid: the step's graphs (ghost fill + x, y, z line passes with the stage, x3)
        g = ws.Grid(a.nx, a.ny, a.nz, faces=faces)
        s = ws.Solver(g)
        s.set_state(f0, stream=stream)
        dt = s.compute_dt(0.5, stream=stream)
        launches_per_step = 12      # 3 x (ghost fill + x, y, z line passes)

        def run_steps(n):
            s.step(dt, n, stream=stream)
    else:
        # this rank's block of one (px*nx) x (py*ny) x (pz*nz) grid (x slabs
        # by default); per stage: halo pack, NCCL send/recv with the
        # neighbours, unpack, ghost fill, fused stage
        from windstencil_b200 import halo
        dims = process_dims(a, world)
        gg = ws.Grid(a.nx * dims[0], a.ny * dims[1], a.nz * dims[2], faces=faces)
        with torch.cuda.stream(stream):
            if a.halo == "native" and a.backend != "nccl":
                raise SystemExit("--halo native needs --backend nccl (one GPU per rank)")
            stepper = halo.distributed(gg, dims=dims, native=a.halo == "native")
            runner = stepper.runners[0]
            runner.set_state(f0)
            dt = stepper.compute_dt(0.5)
        g, s = runner.grid, runner.solver
        sides = sum(len(runner.block.sides(ax)) for ax in range(3))
        launches_per_step = 3 * (4 + 2 * sides)

        def run_steps(n):
            with torch.cuda.stream(stream):
                stepper.step(dt, n)
    cells = g.cells

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- whole-job value: K SSP-RK3 steps
    run_steps(a.warmup)
    stream.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    with ClockSampler(local) as clk:
        e0.record(stream)
        run_steps(a.steps)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(torch, dist, e0.elapsed_time(e1))
    status = s.status(stream=stream)
    value = world * cells * 3 * a.steps / (ms * 1e-3) / 1e9

    # ---- dominant kernel alone (drop-in entry point, same stream)
    rhs_ms = time_rhs_kernel(torch, ws, g, s, stream, max(3, min(a.steps, 20)))
    peak = _peak(ws, "fp64")
    achieved = FLOP_PER_CELL * cells / (rhs_ms * 1e-3) / 1e12
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    roof = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if peak else None, "traffic": measured_traffic(a),
            "kernel": "one RHS = pencil_x_coop_kernel<8,double,1,0> + "
                      "pencil_rhs_kernel<1|2,8,double,1,1> (x, y, z line passes)",
            "kernel_ms": rhs_ms,
            "peak_source": "DFMA microkernel measured in this run (of measured)",
            "algorithmic_flop_per_cell": FLOP_PER_CELL,
            "algorithmic_bytes_per_cell": BYTES_PER_CELL,
            "rhs_gcell_s": cells / (rhs_ms * 1e-3) / 1e9,
            "hbm_achieved_gbs": BYTES_PER_CELL * cells / (rhs_ms * 1e-3) / 1e9,
            "hbm_peak_gbs": peaks.get("hbm_gbs"), "hbm_peak_source": "MEASURED_PEAKS.json"}
    if roof["traffic"]:
        roof["hbm_measured_gbs"] = roof["traffic"] / (rhs_ms * 1e-3) / 1e9

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not a.no_e2e:
        import ctypes as C  # noqa: F401
        lib = ws.load()
        host = torch.empty((5, a.nz, a.ny, a.nx), dtype=torch.float64).pin_memory()
        host.copy_(torch.from_numpy(f0))
        ptr = host.numpy().ctypes.data
        n_e2e = max(2, min(a.steps, 10))

        def one():
            ws._abi.check(lib.ws_solver_set_state(s.h, ptr, stream.cuda_stream))
            run_steps(1)
            ws._abi.check(lib.ws_solver_get_state(s.h, ptr, stream.cuda_stream))
        one()
        barrier()
        q0, q1 = _events(torch)
        w0 = time.perf_counter()
        q0.record(stream)
        for _ in range(n_e2e):
            one()
        q1.record(stream)
        q1.synchronize()
        wall = time.perf_counter() - w0
        ems = max_over_ranks(torch, dist, q0.elapsed_time(q1))
        nbytes = 5 * cells * 8
        serial = world * cells * 3 * n_e2e / (ems * 1e-3) / 1e9
        e2e = {"value": serial, "unit": "Gcell-RHS/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "steps": n_e2e, "wall_s": wall,
               "note": "every step: pinned host state -> device, one SSP-RK3 step, "
                       "state -> pinned host, through ws_solver_set_state/step/get_state"}
        if world == 1:
            e2e.update(pipelined_e2e(a, torch, ws, g, f0, dt, host, cells, n_e2e))
            e2e["serial_value"] = serial
    if world == 1:
        s.close()
    else:
        stepper.close()

    extra = {}
    if rank == 0 and world == 1:
        if not a.no_mixed:
            extra["mixed"] = bench_mixed(a, torch, ws, wl, stream)
        if not a.no_second:
            extra["grid_480x512x64"] = bench_second_grid(a, torch, ws, wl, stream, peak)
        if not a.no_slabs:
            extra["x_slabs_one_gpu"] = bench_slabs_one_gpu(a, torch, ws, wl, stream)
        if not a.no_ns:
            extra["navier_stokes"] = bench_navier_stokes(a, torch, ws, wl, stream)
        serial = None
        if not a.no_batch:
            extra["batched"], serial = bench_batch(a, torch, ws, wl, stream)
        if not a.no_serve:
            # the configuration's offered load (200/s, far above one GPU) and a
            # load one B200 sustains, where latency is not queueing-bound
            extra["served"] = bench_serve(a, ws, wl, serial, a.serve_rate, a.serve_seconds,
                                          a.serve_drain)
            extra["served_sustainable"] = bench_serve(a, ws, wl, serial, a.serve_rate_low,
                                                      a.serve_seconds, a.serve_drain, seed=6)
            extra["served_host_io"] = bench_serve(a, ws, wl, serial, a.serve_rate_low,
                                                  a.serve_seconds, a.serve_drain, seed=7,
                                                  host_io=True)
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_arm(a, a.cpu_seconds)

    if rank == 0:
        line = {"metric": "Gcell-RHS/s", "value": value, "unit": "Gcell-RHS/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic",
                "config": config_of(a, world), "dt": dt,
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches_per_step * a.steps, "clocks": clk.summary(),
                "device_status": status}
        if world > 1:
            line["halo_transport"] = (
                "NCCL point-to-point, device buffers, stage sequence in C++ (ws_blocks_step)"
                if a.halo == "native" else
                "NCCL point-to-point, device buffers, stage sequence in Python"
                if a.backend == "nccl" else "gloo, staged through pinned host memory")
        line.update(extra)
        print(json.dumps(line), flush=True)


def profile_case(a):
    """A small, fixed launch sequence for a profiler to capture, e.g.

        ncu --set full --clock-control none -k regex:bf3w_rhs -c 2 -o prof \
            python bench.py --profile-case --nz 64 --precision fp64

    600x128x64 holds ~1 GB on the device and its inputs exceed the 126 MB L2,
    so DRAM counters stay meaningful.  Nothing is timed or printed but "ok"."""
    import torch
    import windstencil_b200 as ws
    from windstencil_b200 import workloads as wl
    import ctypes as C

    tile = tuple(int(v) for v in a.tile.split(",")) if a.tile else None
    if a.profile_batch:
        specs = wl.batch_specs(a.profile_batch, seed=4)
        states = [wl.batch_state(sp) for sp in specs]
        for name in a.precision.split(","):
            prec = ws.MIXED if name == "mixed" else ws.FP64
            b = ws.Batch([ws.Grid(sp.nx, sp.ny, sp.nz, precision=prec) for sp in specs])
            if tile:
                b.set_tile(tile)
            for i, f in enumerate(states):
                b.set_state(i, f)
            b.set_dt(b.compute_dt(0.5))
            b.step(1)
            b.step(1)
            torch.cuda.synchronize()
            b.close()
        print("ok")
        return
    f0 = wl.sod_state(a.nx, a.ny, a.nz, seed=2)
    for name in a.precision.split(","):
        prec = ws.MIXED if name == "mixed" else ws.FP64
        g = ws.Grid(a.nx, a.ny, a.nz, faces=(1, 1, 0, 0, 0, 0), precision=prec)
        s = ws.Solver(g)
        if tile:
            s.set_tile(tile)
        s.set_state(f0)
        s.rhs()
        if a.step:
            s.step(s.compute_dt(0.5), 1)
        if a.viscous and prec == ws.FP64:
            _, du, prims = s.fields()
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


def measured_traffic(a):
    """DRAM bytes of one RHS (the three line passes) from the committed ncu
    summary, if it was measured on this grid."""
    p = os.path.join(ROOT, "profiles", "pencil_rhs_fp64_600x128x128.json")
    try:
        d = json.load(open(p))
        if d.get("grid") == [a.nx, a.ny, a.nz]:
            return d.get("dram_bytes_per_launch")
    except Exception:
        pass
    return None


def main():
    a = parse()
    if a.profile_case:
        profile_case(a)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist_
        if a.impl == "ours":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")) %
                                  torch.cuda.device_count())
            dist_.init_process_group(a.backend, timeout=datetime.timedelta(seconds=300))
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
