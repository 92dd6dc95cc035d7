"""Dumps streamed from the device and restarts into a context (output.f90:224-235,
restart.f90:212-221): the file must hold exactly the state the context downloads, and a run
restarted from it must continue bit for bit like the run that wrote it."""
import numpy as np
import pytest

import dumses_hybrid_b200 as dg
from dumses_hybrid_b200 import Context, Params, condinit

pytestmark = pytest.mark.gpu

MRI_FARGO = Params(ndim=3, iso=1, nx=16, ny=32, nz=16, xmin=-0.25, xmax=0.25, ymin=-0.5, ymax=0.5, zmin=-0.25,
                   zmax=0.25, ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True)
LOOP2D = Params(ndim=2, nx=32, ny=16, nz=1, xmin=-1, xmax=1, ymin=-0.5, ymax=0.5, courant=0.7)


def start(p: Params, ic: str, **kw) -> Context:
    g = Context(p)
    g.upload(condinit(p, ic, **kw))
    g.boundary(0.0, 0.0)
    return g


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_dump_is_the_downloaded_state(tmp_path, precision):
    p = Params(**{**MRI_FARGO.__dict__, "precision": precision})
    with start(p, "mri", beta=1000.0, amp=0.1, seed=5) as g:
        t, dt = g.run(3, 0.0)
        path = dg.dump_filename(1, 0, tmp_path)
        g.dump(path, t, dt)
        u = g.download()
    v, t2, dt2 = dg.read_dump(path, p)
    assert (t2, dt2) == (t, dt)
    assert np.array_equal(u, v)
    h = dg.dump_header(path)
    assert h["uin_bytes"] == u.size * 8 and (h["nx"], h["ny"], h["nz"]) == (p.nx, p.ny, p.nz)


def test_restart_continues_bit_for_bit(tmp_path):
    """Run 6 steps straight, or 3 steps, dump, restart in a new context and 3 more: same state, same time."""
    p = MRI_FARGO
    with start(p, "mri", beta=1000.0, amp=0.1, seed=5) as g:
        t_ref, _ = g.run(6, 0.0)
        u_ref = g.download()
    path = tmp_path / "d.bin"
    with start(p, "mri", beta=1000.0, amp=0.1, seed=5) as g:
        t, dt = g.run(3, 0.0)
        g.dump(path, t, dt)
    with Context(p) as g:
        t0, _ = g.restart(path)
        assert t0 == t
        t1, _ = g.run(3, t0)
        u = g.download()
    assert t1 == t_ref
    assert np.array_equal(u, u_ref)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_restart_2d_keeps_frozen_face(tmp_path, precision):
    """2D: uin var 11 (right z-face B) is never refreshed by the reference; it must survive a restart."""
    p = Params(**{**LOOP2D.__dict__, "precision": precision})
    path = tmp_path / "d.bin"
    with start(p, "field_loop") as g:
        t, dt = g.run(4, 0.0)
        g.dump(path, t, dt)
        u = g.download()
    with Context(p) as g:
        assert g.restart(path) == (t, dt)
        v = g.download()
    assert np.array_equal(u, v)


def test_restart_from_host_written_dump(tmp_path):
    """A dump written on the host (as a Fortran run would) loads into a context unchanged."""
    p = MRI_FARGO
    with start(p, "mri", beta=1000.0, amp=0.1, seed=9) as g:
        u0 = g.download()  # with ghosts filled
    path = tmp_path / "h.bin"
    dg.write_dump(path, p, u0, 0.0, 0.0)
    with Context(p) as g:
        g.restart(path)
        assert np.array_equal(g.download(), u0)


def test_restart_refuses_other_grid(tmp_path):
    path = tmp_path / "d.bin"
    with start(MRI_FARGO, "mri", beta=1000.0, amp=0.1, seed=5) as g:
        g.dump(path, 0.0, 0.0)
    other = Params(**{**MRI_FARGO.__dict__, "nz": 32})
    with Context(other) as g:
        with pytest.raises(dg.DumsesError, match="DG_ERR_ARG"):
            g.restart(path)
