"""The C++ driver (dumses_hybrid_b200/dg_driver, the reference's main program over the
C-ABI) without a GPU: it reads the reference's `input` namelist files to the same
parameters as the Python mirror (read_namelist, both with the defaults of
init.f90:244-302), and stops with the library's message, as the Fortran shims do,
on options the library does not build and on a missing device."""
import subprocess

import pytest

from dumses_hybrid_b200 import build, read_namelist

INPUT = """&start_params
	tlim    = 70000.
       ,verbose = .false.
       ,debug   = .false.
       /

&scheme_params
	bdtypex    = 'shearingbox'
       ,bdtypey    = 'periodic'
       ,bdtypez    = 'periodic'
       ,riemann    = 'hlld'
       ,riemann2d  = 'hlla'
       ,slope_type = 3
       ,courant    = 0.8
       ,fargo      = .true.
       /

&model_params
	nx     = 32
       ,ny     = 64
       ,nz     = 16
       ,xmin   = -.5d0
       ,xmax   = .5d0
       ,ymin   = 0.d0
       ,ymax   = 4.d0
       ,zmin   = -.5d0
       ,zmax   = .5D0
       ,Omega0 = 1.d-3
       ,ciso   = 1.d-3
       ,nu     = 2.5e-4
       /

&output_params
	dthist  = 100.
	dtdump  = 6283.
       ,io_type = 'binary'
	/

&mpi_params
	nxslice = 2
	nyslice = 4
	nzslice = 2
	/
"""


@pytest.fixture(scope="module")
def driver():
    build.build()
    assert build.DRIVER.exists()
    return str(build.DRIVER)


def run(driver, *args):
    return subprocess.run([driver, *map(str, args)], capture_output=True, text=True, timeout=60)


def printed(out: str) -> dict:
    kv = {}
    for tok in out.split():
        k, v = tok.split("=", 1)
        kv[k] = v
    return kv


@pytest.mark.parametrize("ndim,iso", [(3, 1), (3, 0), (2, 0)])
def test_driver_reads_the_namelist_like_the_python_mirror(driver, tmp_path, ndim, iso):
    path = tmp_path / "input"
    text = INPUT if ndim == 3 else INPUT.replace("'shearingbox'", "'periodic'")
    path.write_text(text)
    res = run(driver, path, "--ndim", ndim, "--iso", iso, "--print-params")
    assert res.returncode == 0, res.stderr
    got = printed(res.stdout)
    c = read_namelist(path, ndim=ndim, iso=iso).to_c()
    for k in ("ndim", "iso", "nx", "ny", "nz", "slope_type", "iriemann", "iriemann2d", "fargo"):
        assert int(got[k]) == getattr(c, k), k
    for k in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax", "gamma", "ciso", "omega0", "courant", "nu", "eta"):
        assert float(got[k]) == getattr(c, k), k
    assert [int(b) for b in got["bc"].split(",")] == list(c.bc)
    assert float(got["tlim"]) == 70000.0 and float(got["dthist"]) == 100.0 and float(got["dtdump"]) == 6283.0
    assert got["restart"] == "0" and got["io_type"] == "binary" and got["debug"] == "0"


def test_driver_defaults_are_the_reference_defaults(driver, tmp_path):
    """An input file that sets nothing gives default_parameters (init.f90:244-302)."""
    path = tmp_path / "input"
    path.write_text("&start_params /\n&scheme_params /\n&model_params /\n&output_params /\n&mpi_params /\n")
    got = printed(run(driver, path, "--print-params").stdout)
    c = read_namelist(path).to_c()
    for k in ("nx", "ny", "nz", "slope_type", "iriemann", "iriemann2d", "fargo"):
        assert int(got[k]) == getattr(c, k), k
    for k in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax", "gamma", "courant"):
        assert float(got[k]) == getattr(c, k), k
    assert (got["tlim"], got["dtdump"], got["dthist"], got["io_type"]) == ("1", "-1", "-1", "binary")


@pytest.mark.parametrize("change,message", [
    (("'hlld'\n       ,riemann2d", "'roe'\n       ,riemann2d"), "unsupported riemann"),
    (("io_type = 'binary'", "io_type = 'phdf5'"), "only 'binary' dumps"),
    (("ciso   = 1.d-3", "ciso   = 1.d-3\n       ,rhs    = .true."), "source terms"),
    (("'shearingbox'", "'reflexive'"), "unsupported boundary type"),
])
def test_driver_stops_on_what_the_library_does_not_build(driver, tmp_path, change, message):
    path = tmp_path / "input"
    assert change[0] in INPUT
    path.write_text(INPUT.replace(change[0], change[1], 1))
    res = run(driver, path, "--iso", 1, "--out", tmp_path / "out")
    assert res.returncode == 1 and message in res.stderr, res.stderr


def test_driver_without_a_device_stops_with_the_library_message(driver, tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible")
    path = tmp_path / "input"
    path.write_text(INPUT)
    res = run(driver, path, "--iso", 1, "--out", tmp_path / "out")
    assert res.returncode == 1 and "dg_init returned -7" in res.stderr, res.stderr


def test_driver_and_mirror_agree_on_namelist_details(driver, tmp_path):
    """Comments, upper-case names, D exponents, T/F logicals, double quotes, several
    assignments on a line: both readers see the same values."""
    text = """! a run of the MRI problem
&START_PARAMS TLIM = 2.5D1, restart = 0 /   ! stop time
&scheme_params
   BdTypeX = "shearingbox", bdtypey='periodic' ! riemann = 'llf' is a comment
   Riemann = 'HLLD', RIEMANN2D = 'upwind', slope_type = 1, Courant = 6.d-1, FARGO = T
/
&model_params nx = 24, NY = 40, nz = 8, xmin = -5.D-1, xmax = 5.D-1, ymin = -1.0, ymax = 1.0,
   zmin = -0.125, zmax = 0.125, omega0 = 1.5d0, CISO = 0.5, eta = 1.e-4 /
&output_params dthist = 0.5, dtdump = 2., io_type = 'binary' /
&mpi_params /
"""
    path = tmp_path / "input"
    path.write_text(text)
    res = run(driver, path, "--iso", 1, "--print-params")
    assert res.returncode == 0, res.stderr
    got = printed(res.stdout)
    c = read_namelist(path, ndim=3, iso=1).to_c()
    for k in ("nx", "ny", "nz", "slope_type", "iriemann", "iriemann2d", "fargo"):
        assert int(got[k]) == getattr(c, k), k
    for k in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax", "ciso", "omega0", "courant", "eta"):
        assert float(got[k]) == getattr(c, k), k
    assert [int(b) for b in got["bc"].split(",")] == list(c.bc)
    assert (c.iriemann, c.iriemann2d, c.fargo, c.bc[0]) == (4, 5, 1, 2)  # HLLD, upwind, FARGO, shearing box
    assert (float(got["tlim"]), float(got["dthist"]), float(got["dtdump"])) == (25.0, 0.5, 2.0)
