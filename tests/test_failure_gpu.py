"""Failure detection without a GPU fault: a device-side wait that nothing completes runs out
of its time bound and is reported as DG_ERR_TIMEOUT; a non-finite state is reported by the
CFL pass as an error status; a host wait shorter than the queued work returns
DG_ERR_TIMEOUT.  After each, the device and the context stay usable."""
import ctypes

import numpy as np
import pytest

import dumses_hybrid_b200 as dg
from dumses_hybrid_b200 import Context, Params, condinit

pytestmark = pytest.mark.gpu

OT16 = Params(ndim=3, nx=16, ny=16, nz=16, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1, gamma=5 / 3, courant=0.8)


def selftest(arrive: int) -> tuple[int, float]:
    lib = dg.load_library()
    sec = ctypes.c_double()
    rc = lib.dg_wait_selftest(0, arrive, ctypes.byref(sec))
    return rc, sec.value


def one_step_ok(p: Params) -> None:
    with Context(p) as g:
        g.upload(condinit(p, "orszag_tang"))
        g.boundary(0.0, 0.0)
        t, dt = g.run(2, 0.0)
        assert t > 0 and dt > 0 and np.isfinite(g.download()[..., :8]).all()


def test_bounded_wait_completes_when_released():
    rc, sec = selftest(1)
    assert rc == dg.DG_OK and sec < 0.5


def test_bounded_wait_runs_out_and_device_stays_usable():
    rc, sec = selftest(0)
    assert rc == -4, dg.load_library().dg_last_error()  # DG_ERR_TIMEOUT
    assert 0.9 < sec < 30.0
    assert b"ran out" in dg.load_library().dg_last_error()
    one_step_ok(OT16)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_non_finite_state_is_an_error_status(precision):
    p = Params(**{**OT16.__dict__, "precision": precision})
    u = condinit(p, "orszag_tang")
    bad = u.copy(order="F")
    bad[8, 9, 10, 0] = np.nan  # one active cell's density
    with Context(p) as g:
        g.upload(bad)
        g.boundary(0.0, 0.0)
        with pytest.raises(dg.DumsesError) as e:
            g.compute_dt()
        assert e.value.code in (-5, -6)  # DG_ERR_STATE / DG_ERR_DT
        # the same context takes a good state and steps again
        g.upload(u)
        g.boundary(0.0, 0.0)
        assert g.compute_dt() > 0


def test_host_wait_bound_returns_timeout(monkeypatch):
    p = Params(**{**OT16.__dict__, "nx": 64, "ny": 64, "nz": 64})
    with Context(p) as g:
        g.upload(condinit(p, "orszag_tang"))
        g.boundary(0.0, 0.0)
        g.sync()
        monkeypatch.setenv("DG_SYNC_TIMEOUT_S", "1e-6")
        with pytest.raises(dg.DumsesError) as e:
            g.run(20, 0.0)
        assert e.value.code == -4  # DG_ERR_TIMEOUT: the steps were still running
        monkeypatch.delenv("DG_SYNC_TIMEOUT_S")
        g.sync()  # the queued work finishes; nothing was lost
        assert np.isfinite(g.download()[..., :8]).all()
