"""The bounds-checked build (libdumses_gpu_chk.so, step kernels compiled with
-DDG_CHECK_BOUNDS): every array access of the step kernels is checked against the device
buffers of the live contexts, and an access outside them is counted instead of made.  A
child process loads that build (DG_LIBRARY) and runs the step in every configuration the
parity tests cover, small grids: the FP64 results must still equal the oracle's and the
count of out-of-range accesses must be zero."""
import os
import pathlib
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = pathlib.Path(__file__).resolve().parent
CHILD = r'''
import sys
sys.path[:0] = [sys.argv[1], sys.argv[2]]
import numpy as np
import dumses_hybrid_b200 as dg
from dumses_hybrid_b200 import Context, Params, condinit
from _oracle import Oracle
from test_parity_gpu import compare_states

assert dg.load_library().dg_debug_oob_count() == 0, "not the checked build"

OT = Params(ndim=3, nx=16, ny=12, nz=10, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1, gamma=5 / 3, courant=0.8)
MRI = Params(ndim=3, iso=1, nx=16, ny=32, nz=16, xmin=-0.25, xmax=0.25, ymin=-0.5, ymax=0.5, zmin=-0.25, zmax=0.25,
             ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True)
ROT = Params(**{**MRI.__dict__, "fargo": False})
LOOP = Params(ndim=2, nx=32, ny=16, nz=1, xmin=-1, xmax=1, ymin=-0.5, ymax=0.5, courant=0.7)
cases = [(OT, "orszag_tang", {}), (Params(**{**OT.__dict__, "bdtypex": "zero_gradient", "slope_type": 3}), "orszag_tang", {}),
         (Params(**{**OT.__dict__, "riemann": "hll", "riemann2d": "hlla", "nu": 1e-3, "eta": 1e-3}), "orszag_tang", {}),
         (MRI, "mri", dict(beta=1000.0, amp=0.1, seed=5)), (ROT, "mri", dict(beta=1000.0, amp=0.1, seed=5)),
         (Params(**{**MRI.__dict__, "nu": 1e-3, "eta": 1e-3}), "mri", dict(beta=1000.0, amp=0.1, seed=5)),
         (LOOP, "field_loop", {}), (Params(**{**LOOP.__dict__, "nu": 1e-3, "eta": 1e-3}), "field_loop", {})]
for p, ic, kw in cases:
    u0 = condinit(p, ic, **kw)
    o = Oracle(p)
    o.set_state(u0)
    o.boundary(0.0, 0.0)
    t = 0.0
    for _ in range(3):
        t, _ = o.step(t)
    for prec in ("fp64", "fp32"):
        q = Params(**{**p.__dict__, "precision": prec})
        with Context(q) as g:
            g.upload(u0)
            g.boundary(0.0, 0.0)
            tg, _ = g.run(3, 0.0)
            u = g.download()
            if p.ndim == 3 and not p.nu and not p.eta:
                g.history()
        if prec == "fp64":
            assert tg == t
            compare_states(u, o.uin, p)
        else:
            assert np.isfinite(u[..., :8]).all()
print("OOB", dg.load_library().dg_debug_oob_count())
'''


def test_checked_build_has_no_out_of_range_access():
    from dumses_hybrid_b200 import build
    build.build()
    env = dict(os.environ, DG_LIBRARY=str(build.LIB_CHK))
    res = subprocess.run([sys.executable, "-c", CHILD, str(HERE.parent), str(HERE)], env=env, capture_output=True,
                         text=True, timeout=900)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-4000:]
    assert "OOB 0" in res.stdout, res.stdout[-2000:]
