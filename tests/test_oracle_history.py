"""The oracle's two history routines against exact sums.

The reference has two history routines of the same form (the history.f90 of a problem directory
replaces the default one at link time): the MRI problem's (src/problem/mri/history.f90) takes
the Maxwell stress of B_x and B_y and the Reynolds stress of v_x and v_y about their y-z means;
the default one of the other problems (src/subroutines/history.f90, NDIM 3) takes B_x with B_z
and v_x with v_z.  On a state with rho = 1, uniform face fields (bx, by, bz) and velocities
v = (A, C, D) cos(2 pi y) the sums are known exactly: the y-z means of the velocities vanish,
the discrete mean of cos^2 over a whole period of cell centres is 1/2, so reynolds = A C / 2
(MRI) or A D / 2 (default), maxwell = -bx by or -bx bz, magp = (bx^2 + by^2 + bz^2) / 2, the
mean field (bx, by, bz), the mass 1 and div B 0.  No reference output of the default routine
exists to compare with; this pins its restatement."""
import math

import numpy as np
import pytest

from dumses_hybrid_b200 import Params
from _oracle import Oracle

A, C, D = 0.3, -0.2, 0.7
BX, BY, BZ = 0.05, -0.02, 0.11


def state(p: Params) -> np.ndarray:
    u = np.zeros(p.shape, order="F")
    ny = p.ny
    dy = (p.ymax - p.ymin) / ny
    j = np.arange(-2, ny + 4)  # ghosted index i = -2 .. n+3 (3 ghost layers)
    y = p.ymin + (j - 0.5) * dy
    cy = np.cos(2.0 * math.pi * y)[None, :, None]
    u[..., 0] = 1.0
    u[..., 1] = A * cy
    u[..., 2] = C * cy
    u[..., 3] = D * cy
    u[..., 4] = 1.0
    for v, b in ((5, BX), (6, BY), (7, BZ), (8, BX), (9, BY), (10, BZ)):
        u[..., v] = b
    return u


@pytest.mark.parametrize("variant", ["mri", "default"])
def test_history_sums_are_exact_on_a_sine_shear(variant):
    p = Params(ndim=3, nx=6, ny=16, nz=5, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=0.5)
    o = Oracle(p)
    o.set_state(state(p))
    h = o.history(variant)
    second_v = C if variant == "mri" else D
    second_b = BY if variant == "mri" else BZ
    want = [1.0, -BX * second_b, A * second_v / 2, -BX * second_b + A * second_v / 2,
            0.5 * (BX * BX + BY * BY + BZ * BZ), BX, BY, BZ]
    for q, w in enumerate(want):
        assert abs(h[q] - w) <= 1e-13 * max(abs(w), 1.0), (variant, q, h[q], w)
    assert abs(h[8]) < 1e-12


def test_history_variants_differ_only_in_the_stresses():
    p = Params(ndim=3, nx=6, ny=16, nz=5, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=0.5)
    o = Oracle(p)
    o.set_state(state(p))
    hm, hd = o.history("mri"), o.history("default")
    assert np.array_equal(hm[[0, 4, 5, 6, 7, 8]], hd[[0, 4, 5, 6, 7, 8]])
    assert not np.isclose(hm[1], hd[1]) and not np.isclose(hm[2], hd[2])
