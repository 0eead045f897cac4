"""Golden vectors of the reference's own arithmetic (tests/golden).

tests/golden/config1_golden.json was written by tests/golden/make_golden.py
from the reference's scalar kernels built for the host: the RHS of the
64x32x16 periodic configuration's initial state and its state after 10
SSP-RK3 steps.  The oracle must reproduce them bit for bit (SHA-256); the
CUDA path must match the sampled cells within rel. 1e-12 of each field's
maximum (FMA contraction and summation order differ from the reference's).
These tests need neither the reference tree nor oracle/_ref.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.oracle import make_grid
from windstencil_b200 import workloads as wl

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "config1_golden.json")
TOL = 1e-12


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as fh:
        return json.load(fh)


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def _case(golden):
    nx, ny, nz = golden["grid"]
    return nx, ny, nz, wl.fourier_state(nx, ny, nz, seed=golden["seed"])


def _check_samples(out, ref):
    flat = out.reshape(5, -1)
    idx = np.array(ref["cells"])
    for v in range(5):
        want = np.array([float.fromhex(x) for x in ref["values"][v]])
        scale = float.fromhex(ref["field_absmax"][v])
        err = np.abs(flat[v, idx] - want).max() / scale
        assert err <= TOL, (v, err)


def test_initial_state_generator_is_stable(golden):
    assert _sha(_case(golden)[3]) == golden["sha256_f0"]


def test_oracle_reproduces_reference_rhs_bitexact(oracle, golden):
    nx, ny, nz, f0 = _case(golden)
    du = oracle.rhs_conserved(make_grid(nx, ny, nz), f0)
    assert _sha(du) == golden["sha256_du0"]


def test_oracle_reproduces_reference_10_steps_bitexact(oracle, golden):
    nx, ny, nz, f0 = _case(golden)
    g = make_grid(nx, ny, nz)
    dt = oracle.compute_dt(g, f0, golden["cfl"])
    assert dt == float.fromhex(golden["dt"])
    f10 = oracle.rk3_steps(g, f0, dt, golden["steps"])
    assert _sha(f10) == golden["sha256_f10"]


@pytest.mark.gpu
def test_gpu_rhs_and_10_steps_match_reference_golden(cuda, golden):
    import windstencil_b200 as ws
    nx, ny, nz, f0 = _case(golden)
    s = ws.Solver(ws.Grid(nx, ny, nz))
    s.set_state(f0)
    s.rhs()
    _check_samples(s.get_rhs(), golden["du0"])
    s.step(float.fromhex(golden["dt"]), golden["steps"])
    out = s.get_state()
    assert s.status() == 0
    _check_samples(out, golden["f10"])
    s.close()
