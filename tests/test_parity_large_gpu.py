"""Bit-exact parity with the oracle on the paths that only shifted or large grids take.

- FARGO with whole-cell shifts (0-8 cells per column, fargo.f90:59-93 with eps = 0) and
  with fractional multi-cell shifts (1-8 cells, fargo.f90:128-240 summing B over the
  traversed cells), through dg_fargo_update alone;
- the MRI + FARGO shearing box at 64 x 128 x 32 with a slow sound speed, so that most
  columns shift by one cell or more per step and every y line spans 9 FARGO segments;
- the 3D Orszag-Tang vortex at 128^3 (many 32-cell trace-core blocks per row);
- grids past 2^31 trace-core elements (64-bit indexing), checked by a property that does
  not depend on size: a periodic state tiled in y and z evolves into the tiled evolution
  of its tile, bit for bit, and the tile's evolution equals the oracle's.
"""
import numpy as np
import pytest

from dumses_hybrid_b200 import Context, Params, condinit
from _oracle import Oracle
from test_oracle_fargo import params as fargo_params, state as fargo_state
from test_parity_gpu import compare_states, run_pair

pytestmark = pytest.mark.gpu


def fargo_pair(p: Params, u0: np.ndarray, dt: float) -> None:
    o = Oracle(p)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    o.fargo_update(dt)
    with Context(p) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        g.fargo_update(dt)
        ug = g.download()
        # the active cells (the GPU writes the remap into the other state buffer, whose ghost
        # cells the next ghost fill makes; the reference remaps rho..E on the z ghosts too)
        act = (slice(3, 3 + p.nx), slice(3, 3 + p.ny), slice(3, 3 + p.nz), slice(0, 8))
        d = ug[act] != o.uin[act]
        assert not d.any(), (int(d.sum()), np.argwhere(d)[:5].tolist())
        # and the whole state after the ghost fill that follows, as in the reference's loop
        o.boundary(0.0, dt)
        g.boundary(0.0, dt)
        compare_states(g.download(), o.uin, p)


def shifts(p: Params, dt: float) -> np.ndarray:
    """FARGO shift of every x column, in cells (cell centres)."""
    dx, dy = (p.xmax - p.xmin) / p.nx, (p.ymax - p.ymin) / p.ny
    xc = p.xmin + dx / 2 + np.arange(p.nx) * dx
    return 1.5 * p.omega0 * np.abs(xc) * dt / dy


def test_fargo_whole_cell_shifts():
    p = fargo_params()
    dt = 2.0 / 3.0
    s = shifts(p, dt)
    assert np.allclose(s, np.round(s)) and round(s.max()) == 7
    fargo_pair(p, fargo_state(p), dt)


def test_fargo_fractional_multi_cell_shifts():
    p = fargo_params()
    dt = 0.65
    s = shifts(p, dt)
    assert s.min() < 1 < 6 < s.max() < 8 and not np.allclose(s, np.round(s))
    fargo_pair(p, fargo_state(p, seed=7), dt)


def test_fargo_long_lines_and_shifts_above_the_segment():
    # 8 x 64 columns: 65 y faces per line (5 segments of 16), shifts of 3-25 cells,
    # larger than a segment
    p = Params(**{**fargo_params().__dict__, "ny": 64, "ymax": 1.0})
    dt = 0.55
    s = shifts(p, dt)
    assert s.max() > 16
    fargo_pair(p, fargo_state_for(p, seed=9), dt)


def fargo_state_for(p: Params, seed: int) -> np.ndarray:
    """A random state with a discretely divergence-free face field on the grid of p."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = p.nx + 6, p.ny + 6, p.nz + 6
    dx, dy, dz = (p.xmax - p.xmin) / p.nx, (p.ymax - p.ymin) / p.ny, (p.zmax - p.zmin) / p.nz
    u = np.zeros(p.shape, order="F")
    u[..., 0] = 1.0 + 0.3 * rng.random((nx, ny, nz))
    u[..., 1:4] = 0.1 * rng.standard_normal((nx, ny, nz, 3))
    u[..., 4] = 1.5 + 0.1 * rng.random((nx, ny, nz))
    A = 1e-2 * rng.standard_normal((3, nx, ny, nz))
    A = np.pad(A[:, :, 3:-3, 3:-3], ((0, 0), (0, 0), (3, 3), (3, 3)), mode="wrap")
    Ax, Ay, Az = A
    u[:, :-1, :-1, 5] = np.diff(Az, axis=1)[:, :, :-1] / dy - np.diff(Ay, axis=2)[:, :-1, :] / dz
    u[:-1, :, :-1, 6] = np.diff(Ax, axis=2)[:-1, :, :] / dz - np.diff(Az, axis=0)[:, :, :-1] / dx
    u[:-1, :-1, :, 7] = np.diff(Ay, axis=0)[:, :-1, :] / dx - np.diff(Ax, axis=1)[:-1, :, :] / dy
    return u


# the shearing box with c_s = 0.03 and Omega = 1: the CFL step (which with FARGO ignores the
# background shear, physics.f90:68-70) moves columns at |x| = 0.5 by about 5 cells
MRI_SHIFTED = Params(ndim=3, iso=1, nx=64, ny=128, nz=32, xmin=-0.5, xmax=0.5, ymin=-1.0, ymax=1.0, zmin=-0.25,
                     zmax=0.25, ciso=0.03, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True)


def test_mri_fargo_64x128x32_multi_cell_shifts():
    p = MRI_SHIFTED
    u0 = condinit(p, "mri", beta=1000.0, amp=0.1, seed=17)
    o = Oracle(p)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    dt = o.compute_dt()
    s = shifts(p, dt)
    assert np.mean(s >= 1) > 0.75 and s.max() > 4, s
    o.close()
    run_pair(p, "mri", 4, beta=1000.0, amp=0.1, seed=17)
    run_pair(p, "mri", 3, use_run=True, beta=1000.0, amp=0.1, seed=17)


def test_orszag_tang_128_cubed():
    p = Params(ndim=3, nx=128, ny=128, nz=128, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1, gamma=5 / 3,
               courant=0.8)
    run_pair(p, "orszag_tang", 3)


def tile_yz(u_small: np.ndarray, p_small: Params, ty: int, tz: int) -> np.ndarray:
    """The interior of a reference-layout state tiled ty x tz times in y and z (ghosts zero;
    the ghost fill of the large grid makes them)."""
    nx, ny, nz = p_small.nx, p_small.ny, p_small.nz
    inner = u_small[:, 3:3 + ny, 3:3 + nz, :]
    big = np.zeros((nx + 6, ny * ty + 6, nz * tz + 6, 11), order="F")
    big[:, 3:3 + ny * ty, 3:3 + nz * tz, :] = np.tile(inner, (1, ty, tz, 1))
    return big


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tiled_shearing_box_past_2e31_core_elements(precision):
    """A 64 x 32 x 32 shearing box with FARGO (one tile) and the same state tiled 32 x 32 times in y
    and z (64 x 1024 x 1024 cells, 3.2e9 trace-core values): the shear-periodic x boundary, FARGO
    and every y/z stencil see a y/z-periodic state, the shear offset stays below the tile's length
    (1.5 Omega L_x t < L_y), so every cell of the large grid must end bit-identical to its tile's
    cell.  In FP64 the tile itself is checked against the oracle."""
    ps = Params(ndim=3, iso=1, nx=64, ny=32, nz=32, xmin=-0.5, xmax=0.5, ymin=-0.25, ymax=0.25, zmin=-0.25,
                zmax=0.25, ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True,
                precision=precision)
    ty = tz = 32
    pb = Params(**{**ps.__dict__, "ny": ps.ny * ty, "nz": ps.nz * tz, "ymin": -0.25 * ty, "ymax": 0.25 * ty,
                   "zmin": -0.25 * tz, "zmax": 0.25 * tz})
    assert (pb.ymax - pb.ymin) / pb.ny == (ps.ymax - ps.ymin) / ps.ny
    assert (pb.zmax - pb.zmin) / pb.nz == (ps.zmax - ps.zmin) / ps.nz
    u0 = condinit(ps, "mri", beta=1000.0, amp=0.1, seed=23)
    with Context(ps) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        u0 = g.download()  # the tile's state after its own ghost fill (right faces derived)
        ts, _ = g.run(4, 0.0)
        us = g.download()
    assert 1.5 * (ps.xmax - ps.xmin) * ts < ps.ymax - ps.ymin
    if precision == "fp64":
        run_pair(ps, "mri", 4, use_run=True, beta=1000.0, amp=0.1, seed=23)
    ub = tile_yz(u0, ps, ty, tz)
    del u0
    with Context(pb) as g:
        g.upload(ub)
        del ub
        g.boundary(0.0, 0.0)
        tb, _ = g.run(4, 0.0)
        big = g.download()
    assert tb == ts
    ny, nz = ps.ny, ps.nz
    small = us[:, 3:3 + ny, 3:3 + nz, :8]
    for a in range(ty):
        for b in range(tz):
            blk = big[:, 3 + a * ny:3 + (a + 1) * ny, 3 + b * nz:3 + (b + 1) * nz, :8]
            if not np.array_equal(blk, small):
                d = np.argwhere(blk != small)[:3]
                raise AssertionError(f"tile ({a}, {b}) differs from the single tile at {d.tolist()}")
