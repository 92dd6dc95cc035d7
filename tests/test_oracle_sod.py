"""The oracle's adiabatic path against an exact solution: Sod's shock tube (gamma = 1.4,
left rho = 1, p = 1, right rho = 0.125, p = 0.1, at rest, B = 0) on a 2D grid of 256 x 4
cells with zero-gradient x boundaries, run to t = 0.2 with the HLLD, HLL and LLF face
solvers.  The exact solution (the exact Riemann solver of Toro, "Riemann Solvers and
Numerical Methods for Fluid Dynamics", ch. 4) has a rarefaction, a contact and a shock; the
second-order scheme must approach it in L1, and the more dissipative solvers less closely.
The reference's shock-tube test (src/problem/shock_tube) has only a picture as its
reference output, so this pins the adiabatic EOS, the non-HLLD solvers and the 2D trace by
a known answer instead."""
import math

import numpy as np
import pytest

from dumses_hybrid_b200 import Params
from _oracle import Oracle

GAMMA = 1.4
LEFT = (1.0, 0.0, 1.0)     # rho, u, p
RIGHT = (0.125, 0.0, 0.1)
NX, NY = 256, 4


def exact_sod(x: np.ndarray, t: float, x0: float = 0.5) -> np.ndarray:
    """Density of the exact solution of the Riemann problem LEFT | RIGHT at x0, time t."""
    g = GAMMA
    rl, ul, pl = LEFT
    rr, ur, pr = RIGHT
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)

    def f(p, rk, pk, ck):  # pressure function and its derivative (Toro 4.6-4.7)
        if p > pk:
            a, b = 2.0 / ((g + 1.0) * rk), (g - 1.0) / (g + 1.0) * pk
            q = math.sqrt(a / (p + b))
            return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (b + p))
        r = p / pk
        return 2.0 * ck / (g - 1.0) * (r ** ((g - 1.0) / (2.0 * g)) - 1.0), r ** (-(g + 1.0) / (2.0 * g)) / (rk * ck)

    p = 0.5 * (pl + pr)
    for _ in range(50):  # Newton on f_L(p) + f_R(p) + u_R - u_L = 0
        fl, dl = f(p, rl, pl, cl)
        fr, dr = f(p, rr, pr, cr)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p = max(p - dp, 1e-12)
        if abs(dp) < 1e-14 * p:
            break
    us = 0.5 * (ul + ur) + 0.5 * (f(p, rr, pr, cr)[0] - f(p, rl, pl, cl)[0])
    # left rarefaction (p* < pL) and right shock (p* > pR) for Sod's data
    rls = rl * (p / pl) ** (1.0 / g)
    cls = cl * (p / pl) ** ((g - 1.0) / (2.0 * g))
    rrs = rr * ((p / pr + (g - 1.0) / (g + 1.0)) / ((g - 1.0) / (g + 1.0) * p / pr + 1.0))
    sr = ur + cr * math.sqrt((g + 1.0) / (2.0 * g) * p / pr + (g - 1.0) / (2.0 * g))
    s = (x - x0) / t
    rho = np.empty_like(x)
    head, tail = ul - cl, us - cls
    fan = (s > head) & (s < tail)
    rho[s <= head] = rl
    rho[fan] = rl * (2.0 / (g + 1.0) + (g - 1.0) / ((g + 1.0) * cl) * (ul - s[fan])) ** (2.0 / (g - 1.0))
    rho[(s >= tail) & (s < us)] = rls
    rho[(s >= us) & (s < sr)] = rrs
    rho[s >= sr] = rr
    return rho


def run(riemann: str) -> tuple[np.ndarray, np.ndarray, float]:
    p = Params(ndim=2, iso=0, nx=NX, ny=NY, nz=1, xmin=0.0, xmax=1.0, ymin=0.0, ymax=NY / NX, zmin=0.0, zmax=1.0,
               gamma=GAMMA, courant=0.8, slope_type=2, riemann=riemann, riemann2d="hlld", bdtypex="zero_gradient")
    u = np.zeros(p.shape, order="F")
    xc = (np.arange(NX + 6) - 2.5) / NX  # cell centres, ghosts included
    left = xc < 0.5
    u[..., 0] = np.where(left, LEFT[0], RIGHT[0])[:, None, None]
    u[..., 4] = (np.where(left, LEFT[2], RIGHT[2]) / (GAMMA - 1.0))[:, None, None]
    o = Oracle(p)
    o.set_state(u)
    o.boundary(0.0, 0.0)
    t = 0.0
    while t < 0.2:
        t, _ = o.step(t)
    rho = o.uin[3:3 + NX, 3:3 + NY, 0, 0].copy()  # a copy: the view dies with the oracle state
    return xc[3:3 + NX], rho, t


@pytest.mark.parametrize("riemann,bound", [("hlld", 0.007), ("hll", 0.0075), ("llf", 0.01)])
def test_sod_shock_tube_converges_to_the_exact_solution(riemann, bound):
    x, rho, t = run(riemann)
    assert np.allclose(rho, rho[:, :1])  # the y direction stays uniform
    exact = exact_sod(x, t)
    err = float(np.abs(rho[:, 0] - exact).mean() / np.abs(exact).mean())
    print(riemann, "t", t, "relative L1 of rho", err)
    # a second-order scheme at 256 cells, limited at the three waves: measured 0.34% (HLLD),
    # 0.36% (HLL), 0.47% (LLF); the bound allows about twice that
    assert err < bound
    # mass is conserved to round-off (nothing has reached the zero-gradient boundaries)
    assert abs(rho.sum() / NY / NX - (0.5 * LEFT[0] + 0.5 * RIGHT[0])) < 1e-13


def test_sod_dissipation_orders_the_solvers():
    errs = {}
    for riemann in ("hlld", "hll", "llf"):
        x, rho, t = run(riemann)
        errs[riemann] = float(np.abs(rho[:, 0] - exact_sod(x, t)).mean())
    assert errs["hlld"] <= errs["hll"] < errs["llf"], errs


def tube_3d(direction: int) -> np.ndarray:
    """Density profile of the HLLD shock tube along x, y or z of a 3D grid (256 cells along the
    tube, 4 across, zero-gradient ends) at t = 0.2 (the last step shortened to end there)."""
    n = [4, 4, 4]
    n[direction] = NX
    ext = [c / NX for c in n]
    bc = ["periodic"] * 3
    bc[direction] = "zero_gradient"
    p = Params(ndim=3, iso=0, nx=n[0], ny=n[1], nz=n[2], xmin=0.0, xmax=ext[0], ymin=0.0, ymax=ext[1], zmin=0.0,
               zmax=ext[2], gamma=GAMMA, courant=0.8, slope_type=2, riemann="hlld", riemann2d="hlld",
               bdtypex=bc[0], bdtypey=bc[1], bdtypez=bc[2])
    u = np.zeros(p.shape, order="F")
    c = (np.arange(NX + 6) - 2.5) / NX
    shape = [1, 1, 1]
    shape[direction] = NX + 6
    left = (c < 0.5).reshape(shape)
    u[..., 0] = np.where(left, LEFT[0], RIGHT[0])
    u[..., 4] = np.where(left, LEFT[2], RIGHT[2]) / (GAMMA - 1.0)
    o = Oracle(p)
    o.set_state(u)
    o.boundary(0.0, 0.0)
    t = 0.0
    while t < 0.2:
        dt = min(o.compute_dt(), 0.2 - t)
        o.godunov(dt, t)
        o.boundary(t, dt)
        t = t + dt
    rho = np.moveaxis(o.uin[3:-3, 3:-3, 3:-3, 0], direction, 0).copy()
    return rho[:, 0, 0], rho


def test_sod_shock_tube_is_the_same_along_x_y_and_z():
    """The solvers' direction permutations (solver.f90:116-160) and the trace's per-direction
    slopes: the tube along y and along z gives the x tube's profile, uniform across."""
    px, _ = tube_3d(0)
    x = (np.arange(NX) + 0.5) / NX
    assert np.abs(px - exact_sod(x, 0.2)).mean() / np.abs(exact_sod(x, 0.2)).mean() < 0.007
    for d in (1, 2):
        prof, full = tube_3d(d)
        assert np.allclose(full, prof[:, None, None], rtol=0, atol=1e-14)
        assert np.allclose(prof, px, rtol=0, atol=1e-12), (d, np.abs(prof - px).max())


def run_1d(riemann: str) -> tuple[np.ndarray, np.ndarray, float]:
    """The same tube with the reference's one-dimensional scheme (NDIM = 1: trace1d, the x
    solves only, every field updated by its x flux)."""
    p = Params(ndim=1, iso=0, nx=NX, ny=1, nz=1, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0,
               gamma=GAMMA, courant=0.8, slope_type=2, riemann=riemann, riemann2d="hlld", bdtypex="zero_gradient")
    u = np.zeros(p.shape, order="F")
    xc = (np.arange(NX + 6) - 2.5) / NX
    left = xc < 0.5
    u[:, 0, 0, 0] = np.where(left, LEFT[0], RIGHT[0])
    u[:, 0, 0, 4] = np.where(left, LEFT[2], RIGHT[2]) / (GAMMA - 1.0)
    o = Oracle(p)
    o.set_state(u)
    o.boundary(0.0, 0.0)
    t = 0.0
    while t < 0.2:
        t, _ = o.step(t)
    return xc[3:3 + NX], o.uin[3:3 + NX, 0, 0, 0].copy(), t


@pytest.mark.parametrize("riemann,bound", [("hlld", 0.007), ("llf", 0.01)])
def test_sod_shock_tube_in_one_dimension(riemann, bound):
    """The 1D scheme converges to the exact solution like the 2D one and conserves mass (its CFL
    step is dx / (c_f + |u|) alone, so its dt sequence differs from the 2D grid's)."""
    x, rho, t = run_1d(riemann)
    exact = exact_sod(x, t)
    err = float(np.abs(rho - exact).mean() / np.abs(exact).mean())
    print(riemann, "1D: t", t, "relative L1 of rho", err)
    assert err < bound
    assert abs(rho.sum() / NX - (0.5 * LEFT[0] + 0.5 * RIGHT[0])) < 1e-13
