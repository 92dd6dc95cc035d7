"""The oracle's MHD step is invariant under a rotation of the axes: the Orszag-Tang vortex
set up in the x-y plane of a 3D grid (32 x 32 cells, 4 across) and the same vortex turned
into the y-z and z-x planes (a cyclic permutation of the axes, a proper rotation) must give
the same fields, permuted, after the same steps.  Each orientation exercises other
direction permutations of the 1D solvers (solver.f90:116-160), other edge directions of the
2D EMF solvers and corner states (solver_magnetic.f90:81-108, scheme.f90:1555-1697) and other
constrained-transport terms; the reference's Orszag-Tang tests in x/y/z compare such
orientations by eye."""
import numpy as np
import pytest

from dumses_hybrid_b200 import Params
from _oracle import Oracle

N, M, STEPS = 32, 4, 12
GAMMA = 5.0 / 3.0


def vortex_xy() -> np.ndarray:
    """Orszag-Tang in the x-y plane: rho = 25/(36 pi), p = 5/(12 pi), v = (-sin 2 pi y,
    sin 2 pi x, 0), B = (-sin 2 pi y, sin 4 pi x, 0) / sqrt(4 pi), face B on the faces."""
    u = np.zeros((N + 6, N + 6, M + 6, 11), order="F")
    c = (np.arange(N + 6) - 2.5) / N
    x, y = np.meshgrid(c, c, indexing="ij")
    b0 = 1.0 / np.sqrt(4 * np.pi)
    rho = 25.0 / (36.0 * np.pi)
    vx, vy = -np.sin(2 * np.pi * y), np.sin(2 * np.pi * x)
    bx, by = -b0 * np.sin(2 * np.pi * y), b0 * np.sin(4 * np.pi * x)  # bx depends on y only, by on x only
    u[..., 0] = rho
    u[..., 1] = (rho * vx)[..., None]
    u[..., 2] = (rho * vy)[..., None]
    u[..., 5] = u[..., 8] = bx[..., None]
    u[..., 6] = u[..., 9] = by[..., None]
    u[..., 4] = (5.0 / (12.0 * np.pi) / (GAMMA - 1.0) + 0.5 * rho * (vx ** 2 + vy ** 2) + 0.5 * (bx ** 2 + by ** 2))[..., None]
    return u


def rotate(u: np.ndarray) -> np.ndarray:
    """The state turned by x -> y, y -> z, z -> x: u'[a, b, c] = R u[b, c, a]."""
    r = np.transpose(u, (2, 0, 1, 3)).copy(order="F")
    out = r.copy(order="F")
    for base in (1, 5, 8):  # momenta, left-face B, right-face B: (V_x, V_y, V_z) -> (V_z, V_x, V_y)
        out[..., base], out[..., base + 1], out[..., base + 2] = r[..., base + 2], r[..., base], r[..., base + 1]
    return out


def params(shape: tuple[int, int, int]) -> Params:
    nx, ny, nz = shape
    return Params(ndim=3, nx=nx, ny=ny, nz=nz, xmin=0, xmax=nx / N, ymin=0, ymax=ny / N, zmin=0, zmax=nz / N,
                  gamma=GAMMA, courant=0.8, slope_type=2, riemann="hlld", riemann2d="hlld")


def evolve(u: np.ndarray, shape) -> tuple[np.ndarray, list[float]]:
    o = Oracle(params(shape))
    o.set_state(u)
    o.boundary(0.0, 0.0)
    t, dts = 0.0, []
    for _ in range(STEPS):
        t, dt = o.step(t)
        dts.append(dt)
    return o.uin.copy(), dts


@pytest.mark.parametrize("turns", [1, 2])
def test_orszag_tang_is_the_same_in_every_plane(turns):
    u = vortex_xy()
    a, dts_a = evolve(u, (N, N, M))
    ur, ar = u, a
    shape = (N, N, M)
    for _ in range(turns):
        ur, ar = rotate(ur), rotate(ar)
        shape = (shape[2], shape[0], shape[1])
    b, dts_b = evolve(ur, shape)
    assert np.allclose(dts_a, dts_b, rtol=1e-13, atol=0)
    act = (slice(3, -3),) * 3
    for v in range(8):
        scale = max(np.abs(ar[act + (v,)]).max(), 1e-30)
        diff = np.abs(b[act + (v,)] - ar[act + (v,)]).max() / scale
        assert diff < 1e-11, (turns, v, diff)
