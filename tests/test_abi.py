"""The C-ABI library on a machine without a GPU: it loads, exports every entry
point declared in include/dumses_gpu.h, builds initial conditions, validates
parameters and reports a missing device as an error code (no crash)."""
import ctypes
import pathlib
import re

import numpy as np
import pytest

import dumses_hybrid_b200 as dg

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "dumses_gpu.h").read_text()
    return sorted(set(re.findall(r"\b(dg_[a-z_0-9]+)\s*\(", text)))


def test_exports_every_declared_symbol():
    lib = dg.load_library()
    names = declared_functions()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), f"{n} declared but not exported"


def test_default_params_match_reference_defaults():
    lib = dg.load_library()
    p = dg.DgParams()
    lib.dg_default_params(ctypes.byref(p))
    # default_parameters, init.f90:244-302
    assert (p.nx, p.ny, p.nz) == (256, 256, 256)
    assert p.courant == 0.7 and p.slope_type == 2
    assert p.iriemann == 4 and p.iriemann2d == 4
    assert abs(p.gamma - 5.0 / 3.0) < 1e-15
    assert lib.dg_uin_size(ctypes.byref(p)) == 262 ** 3 * 11


def test_condinit_field_loop_div_free():
    P = dg.Params(ndim=2, nx=32, ny=16, nz=1, xmin=-1, xmax=1, ymin=-0.5, ymax=0.5)
    u = dg.condinit(P, "field_loop")
    assert u.shape == (38, 22, 1, 11)
    dx, dy = 2 / 32, 1 / 16
    bxl, byl = u[:-1, :-1, 0, 5], u[:-1, :-1, 0, 6]
    bxr, byr = u[:-1, :-1, 0, 8], u[:-1, :-1, 0, 9]
    div = (bxr - bxl) / dx + (byr - byl) / dy
    assert np.max(np.abs(div)) < 1e-12
    assert np.all(u[..., 0] == 1.0)


def test_condinit_mri_reproducible_and_bounded():
    P = dg.Params(ndim=3, iso=1, nx=8, ny=16, nz=8, xmin=-0.25, xmax=0.25, ymin=-0.5, ymax=0.5, zmin=-0.25,
                  zmax=0.25, ciso=1.0, omega0=1.0)
    a = dg.condinit(P, "mri", beta=1000.0, amp=0.1, seed=7)
    b = dg.condinit(P, "mri", beta=1000.0, amp=0.1, seed=7)
    c = dg.condinit(P, "mri", beta=1000.0, amp=0.1, seed=8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.max(np.abs(a[..., 1:4])) <= 0.05
    assert np.allclose(a[..., 7], np.sqrt(2.0 / 1000.0))


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_invalid_params_rejected_before_device_use():
    lib = dg.load_library()
    bad = dg.Params(ndim=4, nx=8, ny=8, nz=8).to_c()
    h = ctypes.c_void_p()
    rc = lib.dg_init(ctypes.byref(bad), ctypes.byref(h))
    assert rc == -8 and not h.value
    assert b"ndim" in lib.dg_last_error()
    bad = dg.Params(ndim=3, nx=8, ny=8, nz=8, bdtypey="shearingbox").to_c()
    assert lib.dg_init(ctypes.byref(bad), ctypes.byref(h)) == -8
    # ndim = 1: a single row, the FP64 path, slope types up to 2 (scheme.f90:313-315), no dissipation
    for kw, code in ((dict(ny=4), -1), (dict(precision="fp32"), -8), (dict(slope_type=3), -8), (dict(nu=1e-3), -8)):
        bad = dg.Params(**{**dict(ndim=1, nx=64, ny=1, nz=1), **kw}).to_c()
        assert lib.dg_init(ctypes.byref(bad), ctypes.byref(h)) == code, kw
        assert not h.value
    if not _has_gpu():  # a valid 1D grid passes validation and stops at the missing device
        good = dg.Params(ndim=1, nx=64, ny=1, nz=1).to_c()
        assert lib.dg_init(ctypes.byref(good), ctypes.byref(h)) in (-7, -2)


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_is_an_error_code():
    with pytest.raises(dg.DumsesError) as e:
        dg.Context(dg.Params(ndim=3, nx=8, ny=8, nz=8))
    assert e.value.code in (-7, -2)


def test_namelist_reader(tmp_path):
    nml = tmp_path / "input"
    nml.write_text("""&start_params tlim = 70000., verbose = .false. /
&scheme_params bdtypex = 'shearingbox', bdtypey = 'periodic', riemann = 'hlld', riemann2d = 'hlld',
 slope_type = 2, courant = 0.8, fargo = .true. /
&model_params nx = 32, ny = 64, nz = 32, xmin = -.5d0, xmax = .5d0, ymin = 0.d0, ymax = 4.d0,
 zmin = -.5d0, zmax = .5d0, Omega0 = 1.d-3, ciso = 1.d-3 /
""")
    p = dg.read_namelist(nml, ndim=3, iso=1)
    assert (p.nx, p.ny, p.nz) == (32, 64, 32)
    assert p.bdtypex == "shearingbox" and p.fargo
    assert p.omega0 == 1e-3 and p.courant == 0.8 and p.ymax == 4.0


def test_network_shape_matches_parameter_count_and_oracle():
    """dg_nn_shape and dg_nn_param_count are host-only calls: the library's network shape,
    its parameter count and the oracle's layer shapes for that shape agree (17-64-64-8 by
    default, 5832 parameters)."""
    from oracle import mlp_oracle as mo
    lib = dg.load_library()
    width, depth = dg.network_shape(lib)
    assert width in (32, 64, 128) and 1 <= depth <= 3
    shp = mo.shapes(width, depth)
    assert int(lib.dg_nn_param_count()) == sum(k * n + n for k, n in shp)
    assert (width, depth) != (64, 2) or int(lib.dg_nn_param_count()) == 5832
