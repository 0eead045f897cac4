"""Seeded synthetic initial states for the benchmark configurations.

The reference ships no input decks, meshes or datasets; its paper grids are
sizes only.  These generators produce the states the benchmark configurations
describe, from numpy's PCG64 with a fixed seed per configuration and grid, in
FP64 on the host; the same arrays feed the GPU path and the CPU oracle.

Units follow the reference (Ama = 1 by default): p = rho*T/(gamma*Ama^2),
c = sqrt(T)/Ama, Cv = 1/(gamma*(gamma-1)*Ama^2) (OCFD_init.cpp:380).

  fourier_state : rho = 1 + sum of 8 Fourier modes (integer wavenumber
                  components 1..4, amplitudes U[0, 0.05], phases U[0, 2pi)),
                  times 2 for x > L/2 (a contact); u = 0.5 (Mach 0.5 at T=1)
                  plus the same kind of perturbation; v, w perturbation only;
                  p = 1/gamma.  Periodic in every direction.
  sod_state     : left rho=1, p=1; right rho=0.125, p=0.1 (jump at x = L/2);
                  u = 0; v, w = 1% uniform noise; rho times (1 + 1% noise).
  batch_specs   : uneven periodic grids, nx log-uniform in [32, 256], ny, nz
                  log-uniform in [16, 128], freestream Mach U[0.3, 3.0], a Sod
                  jump at a seeded x position, 1% noise.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def _modes(rng, nx, ny, nz, nmodes=8, amp=0.05):
    """sum_m a_m sin(2 pi (kx x/Lx + ky y/Ly + kz z/Lz) + phi_m) on the grid
    x_i = i*h (L = n*h), through separable complex exponentials."""
    k = rng.integers(1, 5, size=(nmodes, 3))
    a = rng.uniform(0.0, amp, size=nmodes)
    phi = rng.uniform(0.0, 2.0 * np.pi, size=nmodes)
    out = np.zeros((nz, ny, nx))
    ix, iy, iz = np.arange(nx), np.arange(ny), np.arange(nz)
    for m in range(nmodes):
        ex = np.exp(2j * np.pi * k[m, 0] * ix / nx)
        ey = np.exp(2j * np.pi * k[m, 1] * iy / ny)
        ez = np.exp(2j * np.pi * k[m, 2] * iz / nz) * np.exp(1j * phi[m])
        out += a[m] * np.imag(ez[:, None, None] * ey[None, :, None] * ex[None, None, :])
    return out


def prim_to_cons(d, u, v, w, T, gamma=1.4, ama=1.0):
    """Conserved SoA (5, nz, ny, nx) from interior primitives, in the order of
    pri_to_cons_kernel (commen_kernel.cpp:33-67)."""
    cv = 1.0 / (gamma * (gamma - 1.0) * ama * ama)
    f = np.empty((5,) + d.shape)
    f[0] = d
    f[1] = u * d
    f[2] = v * d
    f[3] = w * d
    f[4] = d * ((u * u + v * v + w * w) * 0.5 + cv * T)
    return f


def fourier_state(nx, ny, nz, seed=1, gamma=1.4, ama=1.0):
    rng = np.random.default_rng(seed)
    d = 1.0 + _modes(rng, nx, ny, nz)
    d[:, :, np.arange(nx) * 2 > nx] *= 2.0
    u = 0.5 * ama * 1.0 + _modes(rng, nx, ny, nz)
    v = _modes(rng, nx, ny, nz)
    w = _modes(rng, nx, ny, nz)
    p = np.full_like(d, 1.0 / gamma)
    T = gamma * ama * ama * p / d
    return prim_to_cons(d, u, v, w, T, gamma, ama)


def sod_state(nx, ny, nz, seed=2, gamma=1.4, ama=1.0, x_jump=0.5):
    rng = np.random.default_rng(seed)
    left = (np.arange(nx) + 0.5) < x_jump * nx
    d = np.where(left, 1.0, 0.125)[None, None, :] * np.ones((nz, ny, nx))
    p = np.where(left, 1.0, 0.1)[None, None, :] * np.ones((nz, ny, nx))
    d = d * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, size=d.shape))
    u = np.zeros_like(d)
    v = 0.01 * rng.uniform(-1.0, 1.0, size=d.shape)
    w = 0.01 * rng.uniform(-1.0, 1.0, size=d.shape)
    T = gamma * ama * ama * p / d
    return prim_to_cons(d, u, v, w, T, gamma, ama)


@dataclass
class GridSpec:
    nx: int
    ny: int
    nz: int
    mach: float
    x_jump: float
    seed: int

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def batch_specs(n=256, seed=4, nx_range=(32, 256), nyz_range=(16, 128),
                mach_range=(0.3, 3.0)) -> list[GridSpec]:
    rng = np.random.default_rng(seed)
    lx = rng.uniform(np.log(nx_range[0]), np.log(nx_range[1]), size=n)
    ly = rng.uniform(np.log(nyz_range[0]), np.log(nyz_range[1]), size=n)
    lz = rng.uniform(np.log(nyz_range[0]), np.log(nyz_range[1]), size=n)
    mach = rng.uniform(*mach_range, size=n)
    xj = rng.uniform(0.25, 0.75, size=n)
    seeds = rng.integers(0, 2**31 - 1, size=n)
    return [GridSpec(int(round(np.exp(a))), int(round(np.exp(b))), int(round(np.exp(c))),
                     float(m), float(x), int(s))
            for a, b, c, m, x, s in zip(lx, ly, lz, mach, xj, seeds)]


def batch_state(spec: GridSpec, gamma=1.4, ama=1.0):
    """Periodic Sod-type state moving at the spec's Mach number."""
    rng = np.random.default_rng(spec.seed)
    nx, ny, nz = spec.nx, spec.ny, spec.nz
    left = (np.arange(nx) + 0.5) < spec.x_jump * nx
    d = np.where(left, 1.0, 0.125)[None, None, :] * np.ones((nz, ny, nx))
    p = np.where(left, 1.0 / gamma, 0.1 / gamma)[None, None, :] * np.ones((nz, ny, nx))
    d = d * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, size=d.shape))
    u = np.full_like(d, spec.mach * ama)        # c = 1 on the left state
    v = 0.01 * rng.uniform(-1.0, 1.0, size=d.shape)
    w = 0.01 * rng.uniform(-1.0, 1.0, size=d.shape)
    T = gamma * ama * ama * p / d
    return prim_to_cons(d, u, v, w, T, gamma, ama)


_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix_uniform(seed, n):
    """[-1, 1) from the splitmix64 finaliser of seed + golden*(n+1) (Steele,
    Lea and Flood 2014); the same counter-based hash as the server's device
    generator, so host and device build identical synthetic states."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + np.uint64(0x9E3779B97F4A7C15) * (n.astype(np.uint64) + np.uint64(1))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) * 2.0 - 1.0


def synth_state(nx, ny, nz, seed, mach, x_jump, gamma=1.4, ama=1.0):
    """Host copy of the server's seeded synthetic request state (ws_request
    with f0_host == NULL): periodic Sod-type jump moving at `mach`, 1% noise."""
    t = np.arange(nx * ny * nz, dtype=np.int64).reshape(nz, ny, nx)
    left = (np.arange(nx) + 0.5) < x_jump * nx
    d = np.where(left, 1.0, 0.125)[None, None, :] * np.ones((nz, ny, nx))
    p = np.where(left, 1.0, 0.1)[None, None, :] / gamma * np.ones((nz, ny, nx))
    d = d * (1.0 + 0.01 * _splitmix_uniform(seed, 3 * t))
    u = np.full_like(d, mach * ama)
    v = 0.01 * _splitmix_uniform(seed, 3 * t + 1)
    w = 0.01 * _splitmix_uniform(seed, 3 * t + 2)
    T = gamma * ama * ama * p / d
    return prim_to_cons(d, u, v, w, T, gamma, ama)


def lap_from_interior(a, lap=4, pitch=None):
    """Dense LAP array (nz+8, ny+8, pitch or nx+8) with `a` in the interior."""
    nz, ny, nx = a.shape
    out = np.zeros((nz + 2 * lap, ny + 2 * lap, pitch or nx + 2 * lap))
    out[lap:lap + nz, lap:lap + ny, lap:lap + nx] = a
    return out
