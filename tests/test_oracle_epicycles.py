"""The oracle's rotation source terms against an exact answer: in a uniform shearing box
(Omega = 1, q = 3/2, isothermal, no field) a uniform radial velocity v0 performs epicycles
at kappa = Omega, v_x = v0 cos(Omega t), dv_y = -(v0 / 2) sin(Omega t), with nothing else
moving.  The update integrates the Coriolis and tidal terms with a Crank-Nicolson rotation
(scheme.f90:1783-1831), which turns (v_x, 2 dv_y) by exactly 2 atan(Omega dt / 2) per step and
keeps v_x^2 + 4 dv_y^2: after one orbit the state must equal that rotation of the initial one
to round-off, with and without FARGO, and the density must not move."""
import math

import numpy as np
import pytest

from dumses_hybrid_b200 import Params
from _oracle import Oracle

V0 = 0.01


@pytest.mark.parametrize("fargo", [True, False])
def test_epicycles_follow_the_crank_nicolson_rotation(fargo):
    p = Params(ndim=3, iso=1, nx=8, ny=8, nz=4, xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5, zmin=-0.25, zmax=0.25,
               ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=fargo)
    u = np.zeros(p.shape, order="F")
    u[..., 0] = 1.0
    u[..., 1] = V0  # the velocities are the deviations from the background shear
    o = Oracle(p)
    o.set_state(u)
    o.boundary(0.0, 0.0)
    t, angle = 0.0, 0.0
    while t < 2.0 * math.pi:
        t, dt = o.step(t)
        angle += 2.0 * math.atan(0.5 * p.omega0 * dt)
    a = o.uin[3:-3, 3:-3, 3:-3]
    vx, vy = a[..., 1] / a[..., 0], a[..., 2] / a[..., 0]
    assert np.array_equal(a[..., 0], np.ones_like(a[..., 0]))
    assert np.allclose(vx, V0 * math.cos(angle), rtol=0, atol=1e-15)
    assert np.allclose(vy, -0.5 * V0 * math.sin(angle), rtol=0, atol=1e-15)
    assert np.abs(vx ** 2 + 4 * vy ** 2 - V0 ** 2).max() < 1e-14 * V0 ** 2
    assert np.abs(a[..., 3]).max() == 0.0
    # and the discrete orbit follows the continuous one up to the rotation's phase error (dt^2 / 12 per radian)
    assert abs(angle - p.omega0 * t) < 1e-3 and np.allclose(vx, V0 * math.cos(t), rtol=0, atol=1e-3 * V0)
