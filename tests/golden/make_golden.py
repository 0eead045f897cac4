#!/usr/bin/env python3
"""Writes tests/golden/config1_golden.json from the reference's own kernels.

Case: the 64x32x16 periodic configuration (Fourier state with a contact,
seed 1, gamma 1.4, Ama 1), SSP-RK3 at CFL 0.5.  The arithmetic is the
reference's: its scalar kernels (cons_to_pri_kernel, sound_speed_kernel, the
decomposed inviscid RHS built from split_Jac3d_Stager_Warming_ker_origin and
OCFD_weno7_SYMBO_kernel_P_opt/_M_opt, OCFD_time_advance_ker1/2/3) built for
the host by oracle/build_ref.py into oracle/_ref.  The ghost layers of the
periodic single-domain case are filled by plain copies (what the reference's
self send/receive halo exchange does on one rank), with the oracle's ghost
fill.  The time step comes from the CFL rule both the oracle and the GPU
solver use (the reference takes DT as an input).

Stored: seeds and sizes, dt, SHA-256 of the float64 (little-endian, C order)
initial state, RHS of the initial state and state after 10 steps, and for
the latter two 128 seeded sample cells (exact values as float.hex) plus
per-field maxima, so the GPU path can be checked against the reference's
numbers without the reference tree.

Run from the repository root, where the reference tree is mounted:
    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle, RefFunctions, make_grid  # noqa: E402
from windstencil_b200 import workloads as wl  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "config1_golden.json")
NX, NY, NZ, SEED, CFL, NSTEPS, NSAMPLE = 64, 32, 16, 1, 0.5, 10, 128


def sha256(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def ref_rhs(ref, orc, g, f):
    d, u, v, w, T, _ = ref.cons_to_prim(g, f)
    for x in (d, u, v, w, T):
        orc.ghost_fill(g, x)
    cc = ref.sound_speed(g, T)
    return ref.du_invis(g, d, u, v, w, cc)


def ref_rk3(ref, orc, g, f0, dt, nsteps):
    f = np.array(f0, dtype=np.float64, copy=True)
    for _ in range(nsteps):
        fn = f.copy()
        for krk in (1, 2, 3):
            du = ref_rhs(ref, orc, g, f)
            ref.time_advance(krk, dt, g, f, fn, du)
    return f


def samples(a, idx):
    flat = a.reshape(5, -1)
    return {"cells": idx.tolist(),
            "values": [[float(flat[v, i]).hex() for i in idx] for v in range(5)],
            "field_absmax": [float(np.abs(flat[v]).max()).hex() for v in range(5)]}


def main():
    if not RefFunctions.available():
        from oracle import build_ref
        build_ref.build(os.environ.get("WS_REFERENCE", build_ref.DEFAULT_REF))
    ref, orc = RefFunctions(), Oracle()
    g = make_grid(NX, NY, NZ)
    f0 = wl.fourier_state(NX, NY, NZ, seed=SEED)
    dt = orc.compute_dt(g, f0, CFL)
    du0 = ref_rhs(ref, orc, g, f0)
    f10 = ref_rk3(ref, orc, g, f0, dt, NSTEPS)
    idx = np.sort(np.random.default_rng(2024).choice(NX * NY * NZ, NSAMPLE, replace=False))
    out = {
        "case": f"{NX}x{NY}x{NZ} periodic, fourier_state seed {SEED}, gamma 1.4, Ama 1, "
                f"SSP-RK3 CFL {CFL}",
        "generated_by": "tests/golden/make_golden.py (reference scalar kernels, oracle/_ref)",
        "grid": [NX, NY, NZ], "seed": SEED, "cfl": CFL, "steps": NSTEPS,
        "dt": float(dt).hex(),
        "sha256_f0": sha256(f0), "sha256_du0": sha256(du0), "sha256_f10": sha256(f10),
        "du0": samples(du0, idx), "f10": samples(f10, idx),
    }
    with open(OUT, "w") as fh:
        json.dump(out, fh, separators=(",", ":"))
        fh.write("\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
