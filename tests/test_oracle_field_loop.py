"""The oracle's 2D EMF solvers against a known answer: a weak magnetic field loop advected by
the uniform flow v = (2, 1) across the periodic box [-1, 1] x [-0.5, 0.5] is back at its
initial position after t = 1 (the reference's magnetic_loop problem, whose test output is a
picture).  The scheme diffuses the loop's sharp edge, so the check is convergence: doubling
the resolution must bring B at t = 1 closer to the initial field, and keep more of the
magnetic energy, for each of the 2D solvers (HLLD, LLF, upwind, HLLA); LLF, the most
dissipative, must keep the least."""
import numpy as np
import pytest

from dumses_hybrid_b200 import Params, condinit
from _oracle import Oracle


def loop_at_t1(n: int, riemann2d: str) -> tuple[float, float]:
    """Relative L1 distance of B(t = 1) from B(0) and the fraction of magnetic energy kept,
    on a 2n x n grid (the last step shortened to end at t = 1 exactly)."""
    p = Params(ndim=2, nx=2 * n, ny=n, nz=1, xmin=-1, xmax=1, ymin=-0.5, ymax=0.5, courant=0.7, riemann="hlld",
               riemann2d=riemann2d)
    o = Oracle(p)
    o.set_state(condinit(p, "field_loop"))
    o.boundary(0.0, 0.0)
    b0 = o.uin[3:-3, 3:-3, 0, 5:7].copy()
    t = 0.0
    while t < 1.0:
        dt = min(o.compute_dt(), 1.0 - t)
        o.godunov(dt, t)
        o.boundary(t, dt)
        t = t + dt
    b1 = o.uin[3:-3, 3:-3, 0, 5:7]
    return float(np.abs(b1 - b0).sum() / np.abs(b0).sum()), float((b1 ** 2).sum() / (b0 ** 2).sum())


@pytest.mark.parametrize("riemann2d", ["hlld", "llf", "upwind", "hlla"])
def test_field_loop_returns_and_converges(riemann2d):
    e16, k16 = loop_at_t1(16, riemann2d)
    e32, k32 = loop_at_t1(32, riemann2d)
    print(riemann2d, "L1(B) 32x16", e16, "64x32", e32, "energy kept", k16, k32)
    assert e32 < e16 / 1.5  # closer to the known answer at twice the resolution
    assert k16 < k32 < 1.0  # numerical dissipation only removes magnetic energy, less when resolved


def test_llf_is_the_most_dissipative_emf():
    kept = {r: loop_at_t1(32, r)[1] for r in ("hlld", "llf", "upwind", "hlla")}
    assert kept["llf"] < min(kept["hlld"], kept["upwind"], kept["hlla"]), kept
