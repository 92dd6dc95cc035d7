"""Dissipation (physics.f90:272-664) on the GPU against the oracle: the FP64 path
bit-identical (state after every step, dt sequence), called step by step or inside
dg_run; the FP32 path within a stated relative L1."""
import numpy as np
import pytest

from dumses_hybrid_b200 import Context, Params, condinit
from _oracle import Oracle
from test_parity_gpu import compare_states

pytestmark = pytest.mark.gpu

OT16 = Params(ndim=3, nx=16, ny=16, nz=16, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1, gamma=5 / 3, courant=0.8)
MRI_FARGO = Params(ndim=3, iso=1, nx=16, ny=32, nz=16, xmin=-0.25, xmax=0.25, ymin=-0.5, ymax=0.5, zmin=-0.25,
                   zmax=0.25, ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True)
LOOP2D = Params(ndim=2, nx=32, ny=16, nz=1, xmin=-1, xmax=1, ymin=-0.5, ymax=0.5, courant=0.7)


def run_pair(params, ic, nsteps, use_run=False, **ickw):
    u0 = condinit(params, ic, **ickw)
    o = Oracle(params)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    t_o, dts_o = 0.0, []
    for _ in range(nsteps):
        t_o, dt = o.step(t_o)
        dts_o.append(dt)
    with Context(params) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        t_g, dts_g = 0.0, []
        if use_run:
            t_g, _ = g.run(nsteps, t_g)
        else:
            for _ in range(nsteps):
                dt = g.compute_dt()
                g.godunov(dt, t_g)
                if params.fargo:
                    g.fargo_update(dt)
                g.boundary(t_g, dt)
                g.dissipation(t_g, dt)
                t_g = t_g + dt
                dts_g.append(dt)
        ug = g.download()
    if not use_run:
        assert dts_g == dts_o
    assert t_g == t_o
    compare_states(ug, o.uin, params)
    return ug, o.uin.copy()


@pytest.mark.parametrize("nu,eta", [(2e-3, 0.0), (0.0, 2e-3), (1e-3, 3e-3)])
def test_orszag_tang_dissipative(nu, eta):
    p = Params(**{**OT16.__dict__, "nu": nu, "eta": eta})
    run_pair(p, "orszag_tang", 4)


def test_orszag_tang_dissipative_device_loop():
    p = Params(**{**OT16.__dict__, "nu": 1e-3, "eta": 1e-3})
    run_pair(p, "orszag_tang", 4, use_run=True)


def test_mri_fargo_dissipative():
    """Isothermal shearing box with FARGO: the resistive CT keeps the outer x face, the
    viscous energy flux is off (ISO = 1)."""
    p = Params(**{**MRI_FARGO.__dict__, "nu": 1e-3, "eta": 2e-3})
    run_pair(p, "mri", 4, beta=1000.0, amp=0.1, seed=5)
    run_pair(p, "mri", 4, use_run=True, beta=1000.0, amp=0.1, seed=5)


def test_field_loop_2d_dissipative():
    p = Params(**{**LOOP2D.__dict__, "nu": 1e-3, "eta": 1e-3})
    run_pair(p, "field_loop", 6)
    run_pair(p, "field_loop", 6, use_run=True)


def test_dissipation_is_noop_without_coefficients():
    with Context(OT16) as g:
        g.upload(condinit(OT16, "orszag_tang"))
        g.boundary(0.0, 0.0)
        u0 = g.download()
        g.dissipation(0.0, 1e-3)
        assert np.array_equal(g.download(), u0)


@pytest.mark.parametrize("p", [Params(**{**OT16.__dict__, "nu": 1e-3, "eta": 2e-3}),
                               Params(**{**MRI_FARGO.__dict__, "nu": 1e-3, "eta": 2e-3})])
def test_fp32_dissipative_within_tolerance(p):
    """FP32 path with dissipation: relative L1 per variable below 1e-4 after 10 steps."""
    ic, kw = ("orszag_tang", {}) if not p.fargo else ("mri", dict(beta=1000.0, amp=0.1, seed=5))
    u0 = condinit(p, ic, **kw)
    out = {}
    for prec in ("fp64", "fp32"):
        q = Params(**{**p.__dict__, "precision": prec})
        with Context(q) as g:
            g.upload(u0)
            g.boundary(0.0, 0.0)
            g.run(10, 0.0)
            out[prec] = g.download()
    a, b = out["fp64"][3:-3, 3:-3, 3:-3, :8], out["fp32"][3:-3, 3:-3, 3:-3, :8]
    for v in range(8):
        if p.iso and v == 4:
            continue
        den = np.abs(a[..., v]).sum()
        if den == 0:
            continue
        assert np.abs(b[..., v] - a[..., v]).sum() / den < 1e-4, v
