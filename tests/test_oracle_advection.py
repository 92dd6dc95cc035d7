"""The oracle's 3D hydrodynamics and its slope limiters against a known answer: a density
wave rho = 1 + 0.2 sin(2 pi (x + y + z)) carried by the uniform flow v = (1, 1, 1) at uniform
pressure (an entropy wave, exact solution a pure translation) through the periodic unit
cube is back at its initial position at t = 1.  The error must fall with resolution at the
rate of each limiter (scheme.f90:253-477): second order for MC (slope_type 2), about first
order at these resolutions for minmod (1) and the multidimensional limiter (3), which clip
the wave's extrema; the velocity and pressure stay uniform."""
import numpy as np
import pytest

from dumses_hybrid_b200 import Params
from _oracle import Oracle

GAMMA = 5.0 / 3.0


def wave_error(n: int, slope_type: int) -> float:
    """Mean |rho(t = 1) - rho(0)| over the amplitude 0.2, on n^3 cells (the last step ends at t = 1)."""
    p = Params(ndim=3, nx=n, ny=n, nz=n, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1, gamma=GAMMA, courant=0.8,
               slope_type=slope_type, riemann="hlld", riemann2d="hlld")
    u = np.zeros(p.shape, order="F")
    c = (np.arange(n + 6) - 2.5) / n
    x, y, z = np.meshgrid(c, c, c, indexing="ij")
    rho = 1.0 + 0.2 * np.sin(2 * np.pi * (x + y + z))
    u[..., 0] = rho
    u[..., 1:4] = rho[..., None]          # v = (1, 1, 1)
    u[..., 4] = 1.0 / (GAMMA - 1.0) + 1.5 * rho  # p = 1
    o = Oracle(p)
    o.set_state(u)
    o.boundary(0.0, 0.0)
    r0 = o.uin[3:-3, 3:-3, 3:-3, 0].copy()
    t = 0.0
    while t < 1.0:
        dt = min(o.compute_dt(), 1.0 - t)
        o.godunov(dt, t)
        o.boundary(t, dt)
        t = t + dt
    a = o.uin[3:-3, 3:-3, 3:-3]
    r1 = a[..., 0]
    v = a[..., 1:4] / r1[..., None]
    pg = (GAMMA - 1.0) * (a[..., 4] - 0.5 * (a[..., 1:4] ** 2).sum(axis=-1) / r1)
    assert np.abs(v - 1.0).max() < 1e-12 and np.abs(pg - 1.0).max() < 1e-12  # an entropy wave: v and p exact
    return float(np.abs(r1 - r0).mean() / 0.2)


@pytest.mark.parametrize("slope_type,rate", [(1, 1.7), (2, 3.0), (3, 1.7)])
def test_entropy_wave_converges_at_the_limiter_order(slope_type, rate):
    e8, e16 = wave_error(8, slope_type), wave_error(16, slope_type)
    print("slope_type", slope_type, "error 8^3", e8, "16^3", e16, "ratio", e8 / e16)
    # measured ratios: 2.05 (minmod), 5.4 (MC), 2.03 (multidimensional)
    assert e16 < e8 / rate


def test_mc_is_the_least_dissipative_limiter():
    errs = {s: wave_error(16, s) for s in (1, 2, 3)}
    assert errs[2] < errs[1] and errs[2] < errs[3], errs
