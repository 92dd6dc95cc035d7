"""Parity of the CUDA library with the CPU oracle (bit-exact, FP64).

Both sides start from the same initial state; after every step dt must be
identical and after the run the whole reference-layout state must be identical:
variables 1-8 in every cell (ghosts included) and the right-face B (9-11)
everywhere except the last ghost layer of its direction, which the reference
never refreshes and never reads.
"""
import numpy as np
import pytest

from dumses_hybrid_b200 import Context, Params, condinit
from _oracle import Oracle

pytestmark = pytest.mark.gpu


def compare_states(ug, uo, params):
    assert np.isfinite(ug[..., :8]).all()
    d = ug[..., :8] != uo[..., :8]
    if d.any():
        idx = np.argwhere(d)[:5]
        diff = np.max(np.abs(ug[..., :8] - uo[..., :8]))
        raise AssertionError(f"{int(d.sum())} values differ (max abs {diff:.3e}); first (i,j,k,v): {idx.tolist()}")
    nx, ny, nz, _ = ug.shape
    assert np.array_equal(ug[:-1, :, :, 8], uo[:-1, :, :, 8])
    if params.ndim > 1:
        assert np.array_equal(ug[:, :-1, :, 9], uo[:, :-1, :, 9])
    else:
        assert np.array_equal(ug[..., 9], uo[..., 9])  # ndim = 1: the frozen right y face
    if params.ndim == 3:
        assert np.array_equal(ug[:, :, :-1, 10], uo[:, :, :-1, 10])
    else:
        assert np.array_equal(ug[..., 10], uo[..., 10])


def run_pair(params, ic, nsteps, use_run=False, **ickw):
    u0 = condinit(params, ic, **ickw)
    o = Oracle(params)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    t_o = 0.0
    dts_o = []
    for _ in range(nsteps):
        t_o, dt = o.step(t_o)
        dts_o.append(dt)
    with Context(params) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        t_g = 0.0
        dts_g = []
        if use_run:
            t_g, _ = g.run(nsteps, t_g)
        else:
            for _ in range(nsteps):
                dt = g.compute_dt()
                g.godunov(dt, t_g)
                if params.fargo:
                    g.fargo_update(dt)
                g.boundary(t_g, dt)
                t_g = t_g + dt
                dts_g.append(dt)
        ug = g.download()
    if not use_run:
        assert dts_g == dts_o
    assert t_g == t_o
    compare_states(ug, o.uin, params)
    return ug


OT16 = Params(ndim=3, nx=16, ny=16, nz=16, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1, gamma=5 / 3, courant=0.8)
MRI_TEST = Params(ndim=3, iso=1, nx=16, ny=32, nz=16, xmin=-0.5, xmax=0.5, ymin=0.0, ymax=4.0, zmin=-0.5, zmax=0.5,
                  gamma=1.001, ciso=1e-3, omega0=1e-3, courant=0.8, bdtypex="shearingbox")
MRI_FARGO = Params(ndim=3, iso=1, nx=16, ny=32, nz=16, xmin=-0.25, xmax=0.25, ymin=-0.5, ymax=0.5, zmin=-0.25,
                   zmax=0.25, ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True)
LOOP2D = Params(ndim=2, nx=32, ny=16, nz=1, xmin=-1, xmax=1, ymin=-0.5, ymax=0.5, courant=0.7)


def test_orszag_tang_3d_steps():
    run_pair(OT16, "orszag_tang", 6)


def test_orszag_tang_3d_device_loop():
    run_pair(OT16, "orszag_tang", 6, use_run=True)


def test_field_loop_2d():
    run_pair(LOOP2D, "field_loop", 8)


def test_field_loop_2d_device_loop():
    run_pair(LOOP2D, "field_loop", 8, use_run=True)


def test_mri_shearing_box():
    run_pair(MRI_TEST, "mri_test", 6, beta=1000.0, amp=0.0)


def test_mri_shearing_box_kicks():
    p = Params(**{**MRI_TEST.__dict__, "ciso": 1.0, "omega0": 1.0, "gamma": 5 / 3, "xmin": -0.25, "xmax": 0.25,
                  "ymin": -0.5, "ymax": 0.5, "zmin": -0.25, "zmax": 0.25})
    run_pair(p, "mri", 6, beta=1000.0, amp=0.1, seed=3)


def test_mri_fargo():
    run_pair(MRI_FARGO, "mri", 6, beta=1000.0, amp=0.1, seed=5)


def test_mri_fargo_device_loop():
    run_pair(MRI_FARGO, "mri", 6, use_run=True, beta=1000.0, amp=0.1, seed=5)


@pytest.mark.parametrize("riemann,riemann2d,slope", [
    ("hll", "llf", 2), ("llf", "upwind", 1), ("upwind", "hlla", 2), ("hlld", "hlld", 3), ("hlld", "llf", 0),
])
def test_solver_and_limiter_variants_3d(riemann, riemann2d, slope):
    p = Params(**{**OT16.__dict__, "riemann": riemann, "riemann2d": riemann2d, "slope_type": slope})
    run_pair(p, "orszag_tang", 4)


@pytest.mark.parametrize("riemann,riemann2d,slope", [("hll", "upwind", 2), ("llf", "hlla", 3), ("hlld", "llf", 1)])
def test_solver_and_limiter_variants_2d(riemann, riemann2d, slope):
    p = Params(**{**LOOP2D.__dict__, "riemann": riemann, "riemann2d": riemann2d, "slope_type": slope})
    run_pair(p, "field_loop", 4)


def test_zero_gradient_boundaries():
    p = Params(**{**OT16.__dict__, "bdtypex": "zero_gradient", "bdtypez": "zero_gradient"})
    run_pair(p, "orszag_tang", 4)


def test_mri_fargo_zero_gradient_z():
    # FARGO's EMFs on the top z faces read the face field there (fargo.f90:146-177), which
    # the preceding godunov updated; with a zero-gradient z boundary it differs from the
    # field of the last active plane
    p = Params(**{**MRI_FARGO.__dict__, "bdtypez": "zero_gradient"})
    run_pair(p, "mri", 5, beta=1000.0, amp=0.1, seed=29)


def test_isothermal_rotating_periodic():
    # Coriolis + shear source terms without the shearing boundary
    p = Params(**{**MRI_TEST.__dict__, "bdtypex": "periodic", "ciso": 1.0, "omega0": 1.0, "gamma": 5 / 3,
                  "xmin": -0.25, "xmax": 0.25, "ymin": -0.5, "ymax": 0.5, "zmin": -0.25, "zmax": 0.25})
    run_pair(p, "mri", 4, beta=400.0, amp=0.1, seed=11)


def test_uneven_grid_orszag_tang():
    p = Params(**{**OT16.__dict__, "nx": 24, "ny": 12, "nz": 20})
    run_pair(p, "orszag_tang", 3)


def test_stage_fluxes_and_emfs():
    """Face fluxes and edge EMFs of one Godunov step against the oracle's arrays."""
    P = OT16
    u0 = condinit(P, "orszag_tang")
    o = Oracle(P)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    dt = o.compute_dt()
    o.godunov(dt, 0.0)
    nx, ny, nz = P.nx, P.ny, P.nz
    F = (nx + 1) * (ny + 1) * (nz + 1)
    flux = o.array(0).reshape((nx + 1, ny + 1, nz + 1, 8, 3), order="F")
    emf = [o.array(w).reshape((nx + 6, ny + 6, nz + 6), order="F") for w in (1, 2, 3)]
    with Context(P) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        assert g.compute_dt() == dt
        g.godunov(dt, 0.0)
        for d in range(3):
            gf = g.debug_array(d, F * 6).reshape((nz + 1, ny + 1, nx + 1, 6)).transpose(3, 0, 1, 2)
            hi = [nx + 1 if d == 0 else nx, ny + 1 if d == 1 else ny, nz + 1 if d == 2 else nz]
            for comp, var in ((0, 0), (1, 4), (2, 1), (3, 2), (4, 3)):
                a = gf[comp, : hi[2], : hi[1], : hi[0]].transpose(2, 1, 0)
                b = flux[: hi[0], : hi[1], : hi[2], var, d]
                assert np.array_equal(a, b), f"flux dir {d} var {var}: max diff {np.max(np.abs(a - b))}"
        for e in range(3):
            ge = g.debug_array(3 + e, F).reshape((nz + 1, ny + 1, nx + 1)).transpose(2, 1, 0)
            hi = [nx if e == 0 else nx + 1, ny if e == 1 else ny + 1, nz if e == 2 else nz + 1]
            a = ge[: hi[0], : hi[1], : hi[2]]
            b = emf[e][3: 3 + hi[0], 3: 3 + hi[1], 3: 3 + hi[2]]
            assert np.array_equal(a, b), f"emf {e}: max diff {np.max(np.abs(a - b))}"


def test_history_sums_match_oracle():
    p = Params(**{**MRI_FARGO.__dict__})
    u0 = condinit(p, "mri", beta=1000.0, amp=0.1, seed=5)
    o = Oracle(p)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    with Context(p) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        t, _ = g.run(3, 0.0)
        h_g = g.history()
    t_o = 0.0
    for _ in range(3):
        t_o, _ = o.step(t_o)
    h_o = o.history()
    scale = np.maximum(np.abs(h_o), 1e-300)
    # FP64 sums in a different (tree) order: relative 1e-12, div B at round-off
    for q in (0, 1, 2, 3, 4, 5, 6, 7):
        assert abs(h_g[q] - h_o[q]) <= 1e-12 * scale[q] + 1e-18, (q, h_g[q], h_o[q])
    assert abs(h_g[8]) < 1e-9 and abs(h_o[8]) < 1e-9


def test_default_history_sums_match_oracle():
    """The default history routine of the problems without their own (src/subroutines/history.f90,
    Maxwell stress of B_x B_z, Reynolds stress of v_x v_z), on a 3D Orszag-Tang state after 3 steps,
    FP64 and FP32, against the oracle's restatement; the MRI variant on the same state differs."""
    p = Params(ndim=3, nx=16, ny=24, nz=12, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1, gamma=5 / 3,
               courant=0.8)
    u0 = condinit(p, "orszag_tang")
    o = Oracle(p)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    t_o = 0.0
    for _ in range(3):
        t_o, _ = o.step(t_o)
    h_o = o.history("default")
    scale = np.maximum(np.abs(h_o), 1e-300)
    # FP64: the same sums in another (tree) order, 1e-12; FP32: the state is within ~1e-5 of FP64
    for prec, tol in (("fp64", 1e-12), ("fp32", 1e-3)):
        with Context(Params(**{**p.__dict__, "precision": prec})) as g:
            g.upload(u0)
            g.boundary(0.0, 0.0)
            g.run(3, 0.0)
            h_g = g.history("default")
            h_m = g.history("mri")
        for q in (0, 1, 2, 3, 4, 5, 6, 7):
            assert abs(h_g[q] - h_o[q]) <= tol * scale[q] + (1e-15 if prec == "fp64" else 1e-6 * h_o[4]), \
                (prec, q, h_g[q], h_o[q])
        assert abs(h_g[8]) < 1e-9 and abs(h_o[8]) < 1e-9
        assert not np.isclose(h_m[1], h_g[1])


def tube_1d(nx: int, bdtype: str, omega0: float = 0.0, riemann: str = "hlld") -> tuple[Params, np.ndarray]:
    """A 1D Riemann problem with field: left rho 1, P 1, B_y 1; right rho 0.125, P 0.1, B_y -1;
    B_x 0.75 and a transverse velocity and B_z on both sides (the Brio-Wu-like tube), with the
    right y and z faces (vars 10, 11) set to the left faces, as a problem's condinit sets them."""
    p = Params(ndim=1, iso=0, nx=nx, ny=1, nz=1, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0,
               gamma=2.0, courant=0.8, slope_type=2, riemann=riemann, riemann2d="hlld", bdtypex=bdtype,
               omega0=omega0)
    u = np.zeros(p.shape, order="F")
    xc = (np.arange(nx + 6) - 2.5) / nx
    left = xc < 0.5
    rho = np.where(left, 1.0, 0.125)
    pres = np.where(left, 1.0, 0.1)
    bx, by, bz = 0.75, np.where(left, 1.0, -1.0), 0.3 * np.sin(2 * np.pi * xc)
    vy = 0.1 * np.cos(2 * np.pi * xc)
    u[:, 0, 0, 0] = rho
    u[:, 0, 0, 2] = rho * vy
    u[:, 0, 0, 4] = pres / (p.gamma - 1.0) + 0.5 * rho * vy ** 2 + 0.5 * (bx * bx + by * by + bz * bz)
    for v, b in ((5, bx), (6, by), (7, bz), (8, bx), (9, by), (10, bz)):
        u[:, 0, 0, v] = b
    return p, u


@pytest.mark.parametrize("bdtype,omega0,riemann", [("zero_gradient", 0.0, "hlld"), ("periodic", 0.0, "hlld"),
                                                   ("zero_gradient", 0.0, "hll"), ("zero_gradient", 0.0, "llf"),
                                                   ("zero_gradient", 0.0, "upwind"), ("periodic", 1.0, "hlld")])
def test_one_dimensional_scheme_matches_oracle(bdtype, omega0, riemann):
    """NDIM = 1 (trace1d, the x solves, every field updated by its x flux, the frozen right y and z
    faces of the reference): 40 steps of an MHD tube, every dt and the final state bit-identical,
    the rotation terms and the B_z shear flux included (omega0 > 0), and the history line."""
    p, u0 = tube_1d(128, bdtype, omega0, riemann)
    o = Oracle(p)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    with Context(p) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        t_g = t_o = 0.0
        for _ in range(40):
            dt_o = o.compute_dt()
            dt_g = g.compute_dt()
            assert dt_g == dt_o
            o.godunov(dt_o, t_o)
            o.boundary(t_o, dt_o)
            g.godunov(dt_g, t_g)
            g.boundary(t_g, dt_g)
            t_o = t_o + dt_o
            t_g = t_g + dt_g
        ug = g.download()
        h = g.history("default")
        t_r, _ = g.run(3, t_g)
        ur = g.download()
    compare_states(ug, o.uin, p)
    assert np.array_equal(h[:3], o.history("1d")) and not np.any(h[3:])
    for _ in range(3):
        t_o, _ = o.step(t_o)
    assert t_r == t_o
    compare_states(ur, o.uin, p)
    # the right y and z faces keep their initial values in the active cells (the ghost fill copies them)
    assert np.array_equal(ur[3:-3, ..., 9:11], u0[3:-3, ..., 9:11])


def test_field_loop_full_run_to_t2():
    """The 2D field-loop configuration as specified (128x64 on [-1,1]x[-0.5,0.5], HLLD + CT, MC, CFL 0.7,
    v = (2, 1), A_z = 1e-3 (0.3 - r)) run to t = 2: every step's dt and the final state bit-identical."""
    p = Params(ndim=2, nx=128, ny=64, nz=1, xmin=-1, xmax=1, ymin=-0.5, ymax=0.5, courant=0.7)
    u0 = condinit(p, "field_loop")
    o = Oracle(p)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    t_o, n = 0.0, 0
    while t_o < 2.0:
        t_o, _ = o.step(t_o)
        n += 1
    with Context(p) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        t_g, _ = g.run(n, 0.0)
        ug = g.download()
    assert t_g == t_o and n > 100
    compare_states(ug, o.uin, p)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_state_reads_between_dt_and_godunov(tmp_path, precision):
    """compute_dt leaves the primitive variables for godunov; a download or a dump in between
    (both use that buffer as scratch in FP64) must not change the step's result."""
    p = Params(**{**MRI_FARGO.__dict__, "precision": precision})
    u0 = condinit(p, "mri", beta=1000.0, amp=0.1, seed=5)
    out = []
    for interleave in (False, True):
        with Context(p) as g:
            g.upload(u0)
            g.boundary(0.0, 0.0)
            t = 0.0
            for _ in range(3):
                dt = g.compute_dt()
                if interleave:
                    g.download()
                    g.dump(tmp_path / "d.bin", t, dt)
                g.godunov(dt, t)
                g.fargo_update(dt)
                g.boundary(t, dt)
                t += dt
            out.append(g.download())
    assert np.array_equal(out[0], out[1])
