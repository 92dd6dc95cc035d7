"""The oracle's restatement of FARGO (fargo.f90:17-288) against a known answer: when the
orbital-advection shift of every column is a whole number of cells, the remap is a pure
translation.  Each x column is shifted along y by |v_K dt| / dy cells (v_K = -1.5 Omega x)
with the sub-cell fraction eps = 0, so the interpolation weights are 0 and 1 and the
parabolic correction (1/4 - (1/2 - eps)^2) vanishes; the face fields, moved through the
EMFs summed over the traversed cells and constrained transport, are translated the same
way, except B_y, which takes the shear's Omega effect.  The reference has no FARGO test
output, so this pins the restatement by the properties its algorithm must have."""
import numpy as np

from dumses_hybrid_b200 import Params
from _oracle import Oracle

NX, NY, NZ = 8, 16, 4


def params() -> Params:
    # dx = 1/8 and dy = dz = 1/16: cell centres x = (i - 4.5)/8, faces (i - 5)/8
    return Params(ndim=3, iso=1, nx=NX, ny=NY, nz=NZ, xmin=-0.5, xmax=0.5, ymin=0.0, ymax=1.0, zmin=0.0, zmax=0.25,
                  gamma=5.0 / 3.0, ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True)


def state(p: Params, seed: int = 11) -> np.ndarray:
    rng = np.random.default_rng(seed)
    u = np.zeros(p.shape, order="F")
    nx, ny, nz = p.nx + 6, p.ny + 6, p.nz + 6
    u[..., 0] = 1.0 + 0.3 * rng.random((nx, ny, nz))
    u[..., 1:4] = 0.1 * rng.standard_normal((nx, ny, nz, 3))
    u[..., 4] = 1.5 + 0.1 * rng.random((nx, ny, nz))
    # face fields from an edge vector potential: discretely divergence-free
    dx, dy, dz = 1.0 / 8, 1.0 / 16, 1.0 / 16
    A = 1e-2 * rng.standard_normal((3, nx, ny, nz))
    # periodic in y and z, as the ghost fill will make the field
    A = np.pad(A[:, :, 3:-3, 3:-3], ((0, 0), (0, 0), (3, 3), (3, 3)), mode="wrap")
    Ax, Ay, Az = A
    u[:, :-1, :-1, 5] = np.diff(Az, axis=1)[:, :, :-1] / dy - np.diff(Ay, axis=2)[:, :-1, :] / dz
    u[:-1, :, :-1, 6] = np.diff(Ax, axis=2)[:-1, :, :] / dz - np.diff(Az, axis=0)[:, :, :-1] / dx
    u[:-1, :-1, :, 7] = np.diff(Ay, axis=0)[:, :-1, :] / dx - np.diff(Ax, axis=1)[:-1, :, :] / dy
    return u


def best_shift(after: np.ndarray, before: np.ndarray) -> tuple[int, float]:
    """The cyclic shift s along y (axis 0 here) with after = roll(before, s), and its max error."""
    errs = [np.max(np.abs(after - np.roll(before, s, axis=0))) for s in range(before.shape[0])]
    s = int(np.argmin(errs))
    return s, float(errs[s])


def test_fargo_whole_cell_shift_is_a_translation():
    p = params()
    o = Oracle(p)
    o.set_state(state(p))
    o.boundary(0.0, 0.0)
    u0 = o.uin.copy()
    dt = 2.0 / 3.0  # 1.5 Omega |x| dt / dy = |16 x|: 1, 3, 5, 7 cells at the centres, 0, 2, 4, 6, 8 at the faces
    o.fargo_update(dt)
    u1 = o.uin
    act = (slice(3, 3 + NY), slice(3, 3 + NZ))
    for i in range(1, NX + 1):
        ii = i + 2  # array index of cell i (ghosts at 0..2)
        xc = (i - 4.5) / 8
        n = int(round(1.5 * abs(xc) * dt * 16))
        want = n if -1.5 * xc > 0 else -n  # material moves with v_K = -1.5 Omega x
        for v in range(5):  # rho, momenta, E: moved with the centre's shift
            before, after = u0[ii][act[0], act[1], v], u1[ii][act[0], act[1], v]
            s, err = best_shift(after, before)
            assert s == want % NY and err <= 1e-14 * np.max(np.abs(before)), (i, v, s, want, err)
        # B_z (at the cell's x) is moved through emfx, the sum of B_z over the traversed cells
        before, after = u0[ii][act[0], act[1], 7], u1[ii][act[0], act[1], 7]
        s, err = best_shift(after, before)
        assert s == want % NY and err <= 1e-13 * np.max(np.abs(before)), (i, 7, s, want, err)
    for i in range(2, NX + 1):  # B_x on the interior x faces, at x = (i - 5)/8
        ii = i + 2
        xf = (i - 5) / 8
        n = int(round(1.5 * abs(xf) * dt * 16))
        want = n if -1.5 * xf > 0 else -n
        before, after = u0[ii][act[0], act[1], 5], u1[ii][act[0], act[1], 5]
        s, err = best_shift(after, before)
        assert s == want % NY and err <= 1e-13 * np.max(np.abs(before)), (i, s, want, err)
    # B_y is not translated: the shear turns radial field into azimuthal field (the Omega
    # effect, dB_y = -(dE_z/dx) dt with E_z the translated B_x flux); what CT guarantees is
    # that the field stays divergence-free (after the ghost fill that follows FARGO in the
    # reference's loop, which brings the periodic y and z faces up to date)
    dx, dy, dz = 1.0 / 8, 1.0 / 16, 1.0 / 16
    u1 = u1.copy()
    o.boundary(0.0, dt)
    bx, by, bz = o.uin[..., 5], o.uin[..., 6], o.uin[..., 7]
    div = ((bx[4:-3, 3:-3, 3:-3] - bx[3:-4, 3:-3, 3:-3]) / dx + (by[3:-4, 4:-2, 3:-3] - by[3:-4, 3:-3, 3:-3]) / dy
           + (bz[3:-4, 3:-3, 4:-2] - bz[3:-4, 3:-3, 3:-3]) / dz)
    assert np.max(np.abs(div)) <= 1e-12 * np.max(np.abs(o.uin[..., 5:8])) / dx
    # and its y-average in each column moves by the curl of the y-averaged FARGO EMFs:
    # <E_z> = -v_K dt <B_x> on the column's x faces, <E_x> = v_K dt <B_z> on its z faces
    vk = lambda x: -1.5 * x
    ez = lambda f, k: -vk((f - 5) / 8) * dt * u0[f + 2, 3:3 + NY, k + 2, 5].mean()
    ex = lambda i, k: vk((i - 4.5) / 8) * dt * u0[i + 2, 3:3 + NY, k + 2, 7].mean()
    for i in range(2, NX):
        for k in range(1, NZ + 1):
            want = -(ez(i + 1, k) - ez(i, k)) / dx + (ex(i, k + 1) - ex(i, k)) / dz
            got = u1[i + 2, 3:3 + NY, k + 2, 6].mean() - u0[i + 2, 3:3 + NY, k + 2, 6].mean()
            assert abs(got - want) <= 1e-13, (i, k, got, want)


def test_fargo_fractional_shift_conserves_every_column():
    """With fractional shifts the remap interpolates (linear weights plus the parabolic slope
    correction) but stays conservative: every column keeps its sums of rho, momenta, E, B_x and
    B_z along y, and div B stays at round-off."""
    p = params()
    o = Oracle(p)
    o.set_state(state(p, seed=5))
    o.boundary(0.0, 0.0)
    u0 = o.uin.copy()
    o.fargo_update(0.137)
    u1 = o.uin.copy()
    act_y, act_z = slice(3, 3 + NY), slice(3, 3 + NZ)
    moved = False
    for i in range(1, NX + 1):
        for v in (0, 1, 2, 3, 4, 7):
            s0 = u0[i + 2, act_y, act_z, v].sum(axis=0)
            s1 = u1[i + 2, act_y, act_z, v].sum(axis=0)
            assert np.allclose(s1, s0, rtol=0, atol=1e-13 * np.abs(u0[..., v]).max() * NY), (i, v)
        moved = moved or not np.allclose(u1[i + 2, act_y, act_z, 0], u0[i + 2, act_y, act_z, 0])
    for i in range(2, NX + 1):
        s0, s1 = u0[i + 2, act_y, act_z, 5].sum(axis=0), u1[i + 2, act_y, act_z, 5].sum(axis=0)
        assert np.allclose(s1, s0, rtol=0, atol=1e-13 * np.abs(u0[..., 5]).max() * NY), i
    assert moved
    o.boundary(0.0, 0.137)
    b = o.uin
    dx, dy, dz = 1.0 / 8, 1.0 / 16, 1.0 / 16
    div = ((b[4:-3, 3:-3, 3:-3, 5] - b[3:-4, 3:-3, 3:-3, 5]) / dx + (b[3:-4, 4:-2, 3:-3, 6] - b[3:-4, 3:-3, 3:-3, 6]) / dy
           + (b[3:-4, 3:-3, 4:-2, 7] - b[3:-4, 3:-3, 3:-3, 7]) / dz)
    assert np.max(np.abs(div)) <= 1e-12 * np.max(np.abs(b[..., 5:8])) / dx
