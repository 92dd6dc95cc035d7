"""The oracle's copy of the problem set-ups equals the library's host-side dg_condinit bit for
bit (ghosts included), so the CPU baseline can build the benchmark's initial state without
loading the library.  CPU only: dg_condinit is host code."""
import numpy as np
import pytest

from dumses_hybrid_b200 import Params, condinit
from _oracle import Oracle

MRI = Params(ndim=3, iso=1, nx=12, ny=20, nz=8, xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5, zmin=-0.5, zmax=0.5,
             ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True)
OT = Params(ndim=3, nx=10, ny=12, nz=14, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1, gamma=5 / 3, courant=0.8)
LOOP = Params(ndim=2, nx=32, ny=16, nz=1, xmin=-1, xmax=1, ymin=-0.5, ymax=0.5, courant=0.7)


@pytest.mark.parametrize("p,ic,kw", [
    (MRI, "mri", dict(beta=1000.0, amp=0.1, seed=2024)),
    (MRI, "mri", dict(beta=400.0, amp=0.1, seed=7)),
    (MRI, "mri_test", dict(beta=1000.0)),
    (OT, "orszag_tang", {}),
    (LOOP, "field_loop", {}),
])
def test_oracle_condinit_equals_library(p, ic, kw):
    o = Oracle(p)
    o.condinit(ic, **kw)
    u = condinit(p, ic, **kw)
    assert np.array_equal(o.uin, u)
    assert np.any(o.uin[..., 0] != 0)
    o.close()


def test_oracle_condinit_rejects_wrong_ndim():
    o = Oracle(LOOP)
    with pytest.raises(ValueError):
        o.condinit("orszag_tang")
    o.close()
