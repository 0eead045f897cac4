"""Pins the CPU oracle to the reference's own code.

The reference ships no golden vectors or known-answer tests for this path.
oracle/build_ref.py builds the reference's own scalar kernels for the host;
these tests require the oracle (oracle/oracle.cpp) to agree with them
bit-for-bit (both built with -ffp-contract=off).
"""
import numpy as np
import pytest

from oracle.oracle import LAP, make_grid


def _stencils(n, seed):
    rng = np.random.default_rng(seed)
    s = rng.standard_normal((n, 8)) * rng.uniform(1e-3, 30.0, (n, 1)) + rng.uniform(-5, 5, (n, 1))
    # smooth, constant, step, spike and zero stencils
    x = np.linspace(0, 1, 8)
    s[:100] = np.sin(2 * np.pi * x * rng.uniform(0.1, 2, (100, 1)))
    s[100:200] = rng.uniform(-3, 3, (100, 1))
    s[200:300] = np.where(x > rng.uniform(0, 1, (100, 1)), 1.0, 0.125)
    s[300:400] = 0.0
    s[300:400, 3] = rng.uniform(-1, 1, 100)
    s[400:500] = 0.0
    return s


def test_weno_p_m_bitexact(oracle, reffn):
    s = _stencils(300_000, 11)
    assert np.array_equal(oracle.weno_p(s), reffn.weno_p(s))
    assert np.array_equal(oracle.weno_m(s), reffn.weno_m(s))


def test_weno_mirror(oracle):
    s = _stencils(50_000, 12)
    assert np.array_equal(oracle.weno_m(s), oracle.weno_p(s[:, ::-1]))


def test_split_bitexact(oracle, reffn):
    rng = np.random.default_rng(13)
    n = 50_000
    pts = np.column_stack([
        rng.uniform(0.05, 5.0, n), rng.normal(0, 2, n), rng.normal(0, 1, n), rng.normal(0, 1, n),
        rng.uniform(0.1, 3.0, n), rng.normal(0, 1, (n, 3))])
    pts[:1000, 5:] = [1.0, 0.0, 0.0]
    pts[1000:2000, 5:] = [0.0, 1.0, 0.0]
    for gamma, eps in [(1.4, 1e-6), (1.67, 0.0), (1.3, 0.1)]:
        fp, fm = oracle.split(pts, gamma, eps)
        rfp, rfm = reffn.split(pts, gamma, eps)
        assert np.array_equal(fp, rfp) and np.array_equal(fm, rfm)


def _prims(g, seed):
    rng = np.random.default_rng(seed)
    shp = (g.nz + 2 * LAP, g.ny + 2 * LAP, g.nx + 2 * LAP)
    d = rng.uniform(0.5, 2.0, shp)
    u = rng.normal(0.3, 0.5, shp)
    v = rng.normal(0, 0.3, shp)
    w = rng.normal(0, 0.3, shp)
    T = rng.uniform(0.5, 1.5, shp)
    return d, u, v, w, T


def test_field_kernels_bitexact(oracle, reffn):
    g = make_grid(13, 9, 7, gamma=1.4, ama=0.8)
    d, u, v, w, T = _prims(g, 14)
    f = oracle.prim_to_cons(g, d, u, v, w, T)
    assert np.array_equal(f, reffn.prim_to_cons(g, d, u, v, w, T))
    a = oracle.cons_to_prim(g, f)
    b = reffn.cons_to_prim(g, f)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert np.array_equal(oracle.sound_speed(g, T), reffn.sound_speed(g, T))
    rng = np.random.default_rng(15)
    for krk in (1, 2, 3):
        f0 = rng.normal(size=f.shape)
        fn = rng.normal(size=f.shape)
        du = rng.normal(size=f.shape)
        a1, b1 = f0.copy(), f0.copy()
        oracle.time_advance(krk, 1.7e-3, a1, fn, du)
        reffn.time_advance(krk, 1.7e-3, g, b1, fn, du)
        assert np.array_equal(a1, b1)


@pytest.mark.parametrize("general", [False, True])
def test_du_invis_bitexact(oracle, reffn, general):
    g = make_grid(19, 11, 9)
    d, u, v, w, T = _prims(g, 16)
    cc = oracle.sound_speed(g, T)
    metrics = ajac = None
    if general:
        rng = np.random.default_rng(17)
        shp = d.shape
        metrics = [np.ascontiguousarray(rng.uniform(0.5, 1.5, shp) if i % 4 == 0 else
                                        rng.uniform(-0.3, 0.3, shp)) for i in range(9)]
        ajac = rng.uniform(0.7, 1.3, shp)
    a = oracle.du_invis(g, d, u, v, w, cc, metrics, ajac)
    b = reffn.du_invis(g, d, u, v, w, cc, metrics, ajac)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("form", ["p_lift", "p_lift_plus", "p", "p_right_plus", "m_lift",
                                  "m_lift_plus", "m", "m_right_plus", "minmod2"])
def test_weno5_closures_bitexact(oracle, reffn, form):
    # the CLOSURE mode's WENO5 family and minmod2, including the reference's
    # weight order of OCFD_weno5_kernel_P
    rng = np.random.default_rng(18)
    s = rng.standard_normal((200_000, 5)) * rng.uniform(1e-3, 30.0, (200_000, 1))
    s[:1000] = rng.uniform(-2, 2, (1000, 1))                      # constant
    s[1000:2000] = np.where(np.arange(5) > 2, 1.0, 0.125)         # step
    s[2000:2100, :2] = 0.0                                        # minmod2 zeros
    s[2100:2200, 1] = -s[2100:2200, 0]                            # opposite signs
    assert np.array_equal(oracle.weno5(form, s), reffn.weno5(form, s))


@pytest.mark.parametrize("faces", [(2, 2, 0, 0, 0, 0), (0, 0, 2, 2, 0, 0), (2, 2, 2, 2, 1, 1),
                                   (2, 1, 1, 2, 0, 0), (1, 2, 2, 0, 0, 0)])
def test_du_invis_closure_bitexact(oracle, reffn, faces):
    # CLOSURE faces: the ring kernel's boundary closures near the x / y faces
    g = make_grid(17, 13, 9, face_kind=faces)
    d, u, v, w, T = _prims(g, 19)
    for a in (d, u, v, w, T):
        oracle.ghost_fill(g, a)
    cc = oracle.sound_speed(g, T)
    a = oracle.du_invis(g, d, u, v, w, cc)
    b = reffn.du_invis(g, d, u, v, w, cc)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("scheme", [6, 8])
@pytest.mark.parametrize("general", [False, True])
@pytest.mark.parametrize("faces,d0b", [((0, 0, 0, 0, 0, 0), (0,) * 6),
                                       ((1, 1, 0, 0, 1, 1), (0,) * 6),
                                       ((1, 1, 0, 0, 1, 1), (1, 1, 0, 1, 1, 0)),
                                       ((1, 1, 1, 1, 0, 0), (1, 1, 1, 1, 1, 1))])
def test_du_vis_bitexact(oracle, reffn, scheme, general, faces, d0b):
    # viscous terms: CD6/CD8 gradients, Sutherland viscosity, viscous fluxes
    # per direction and their divergence, added to du[1..4]; with DIF_BOUND
    # flags the reduced forms next to flagged faces come from the reference's
    # OCFD_D0bound_scheme_kernel (periodic faces included, as the reference
    # applies them wherever the flag is set)
    from oracle.oracle import make_vis
    g = make_grid(14, 10, 9, face_kind=faces, ama=0.7)
    vis = make_vis(re=300.0, pr=0.72, ref_t=250.0, scheme=scheme, d0_bound=d0b)
    d, u, v, w, T = _prims(g, 20)
    for a in (u, v, w, T):
        oracle.ghost_fill(g, a)
    metrics = ajac = None
    if general:
        rng = np.random.default_rng(21)
        shp = d.shape
        metrics = [np.ascontiguousarray(rng.uniform(0.5, 1.5, shp) if i % 4 == 0 else
                                        rng.uniform(-0.3, 0.3, shp)) for i in range(9)]
        ajac = rng.uniform(0.7, 1.3, shp)
    base = np.random.default_rng(22).normal(size=(5, g.nz, g.ny, g.nx))
    a = oracle.du_vis(g, vis, u, v, w, T, metrics, ajac, base.copy())
    b = reffn.du_vis(g, vis, u, v, w, T, metrics, ajac, base.copy())
    assert np.array_equal(a, b)
    assert np.array_equal(a[0], base[0])        # no viscous mass term


def test_ref_rk3_steps_bitexact(oracle, reffn):
    """The reference arm's time step (the reference's scalar kernels per
    stage: cons_to_pri, ghost fill, sound speed, decomposed RHS, time advance
    ker1/2/3) equals the oracle's SSP-RK3 steps bit for bit, on the headline
    face kinds (extrapolation in x, periodic y and z)."""
    from oracle.oracle import RefRK3, make_grid
    from windstencil_b200 import workloads as wl
    g = make_grid(24, 16, 12, face_kind=(1, 1, 0, 0, 0, 0))
    f = wl.sod_state(24, 16, 12, seed=2)
    dt = oracle.compute_dt(g, f, 0.5)
    st = RefRK3(g, f, ref=reffn, oracle=oracle)
    for _ in range(2):
        st.step(dt)
    assert np.array_equal(st.f, oracle.rk3_steps(g, f, dt, 2))
