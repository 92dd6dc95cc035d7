"""The C++ driver (the reference's main program over the C-ABI, dumses.f90:37-185) on the
GPU against the oracle: the first dump is the initial state after its ghost fill, the
state after the loop is bit-identical to the oracle's after the same steps, the history
file has the oracle's rows (to its printed precision: the device sums run in another
order) at the same dthist crossings, dumps fall at the dtdump crossings, and a restart
from a dump continues bit for bit."""
import pathlib
import subprocess

import numpy as np
import pytest

from dumses_hybrid_b200 import Params, build, condinit, dump_header, read_dump
from _oracle import Oracle
from test_parity_gpu import compare_states

pytestmark = pytest.mark.gpu

OT = """&start_params tlim = 1.0 /
&scheme_params riemann = 'hlld', riemann2d = 'hlld', slope_type = 2, courant = 0.8 /
&model_params nx = 16, ny = 12, nz = 10, xmin = 0.d0, xmax = 1.d0, ymin = 0.d0, ymax = 1.d0,
              zmin = 0.d0, zmax = 1.d0, gamma = 1.6666666666666667d0 /
&output_params dtdump = -1., dthist = -1., io_type = 'binary' /
&mpi_params /
"""
OT_P = Params(ndim=3, nx=16, ny=12, nz=10, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1, gamma=5 / 3, courant=0.8)

MRI = """&start_params tlim = {tlim!r}, restart = {restart} /
&scheme_params bdtypex = 'shearingbox', riemann = 'hlld', riemann2d = 'hlld', slope_type = 2, courant = 0.8,
               fargo = .true. /
&model_params nx = 16, ny = 32, nz = 16, xmin = -0.25d0, xmax = 0.25d0, ymin = -0.5d0, ymax = 0.5d0,
              zmin = -0.25d0, zmax = 0.25d0, Omega0 = 1.d0, ciso = 1.d0 /
&output_params dtdump = {dtdump!r}, dthist = {dthist!r}, io_type = 'binary' /
&mpi_params /
"""
MRI_P = Params(ndim=3, iso=1, nx=16, ny=32, nz=16, xmin=-0.25, xmax=0.25, ymin=-0.5, ymax=0.5, zmin=-0.25,
               zmax=0.25, ciso=1.0, omega0=1.0, courant=0.8, bdtypex="shearingbox", fargo=True)
MRI_IC = dict(beta=1000.0, amp=0.1, seed=5)


def driver(tmp: pathlib.Path, text: str, *args) -> subprocess.CompletedProcess:
    build.build()
    (tmp / "input").write_text(text)
    res = subprocess.run([str(build.DRIVER), str(tmp / "input"), "--out", str(tmp), "--quiet", *map(str, args)],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    return res


def test_driver_orszag_tang_matches_the_oracle(tmp_path):
    driver(tmp_path, OT, "--ic", "orszag_tang", "--nsteps", 3, "--final-dump", tmp_path / "final.bin")
    o = Oracle(OT_P)
    o.set_state(condinit(OT_P, "orszag_tang"))
    o.boundary(0.0, 0.0)
    u0, t0, _ = read_dump(tmp_path / "output_000000" / "data.000000.bin", OT_P)
    assert t0 == 0.0
    compare_states(u0, o.uin, OT_P)
    t = 0.0
    for _ in range(3):
        t, dt = o.step(t)
    u, tg, dtg = read_dump(tmp_path / "final.bin", OT_P)
    assert (tg, dtg) == (t, dt)
    compare_states(u, o.uin, OT_P)


def test_driver_fp32_runs_the_same_loop(tmp_path):
    driver(tmp_path, OT, "--ic", "orszag_tang", "--nsteps", 3, "--precision", "fp32", "--final-dump",
           tmp_path / "final.bin")
    u, tg, _ = read_dump(tmp_path / "final.bin", OT_P)
    assert tg > 0 and np.isfinite(u[..., :8]).all()


def parse_history(path: pathlib.Path) -> np.ndarray:
    rows = []
    for line in path.read_text().splitlines():
        if line.startswith("#"):
            continue
        vals = []
        for tok in line.split():
            # Fortran 1PE with a three-digit exponent drops the E: d.ddddd+ddd
            if "E" not in tok and ("+" in tok[1:] or "-" in tok[1:]):
                k = max(tok.rfind("+"), tok.rfind("-"))
                tok = tok[:k] + "E" + tok[k:]
            vals.append(float(tok))
        rows.append(vals)
    return np.array(rows)


def test_driver_mri_history_dumps_and_end_time(tmp_path):
    """Shearing box with FARGO: history at every dthist crossing, dumps at every dtdump
    crossing, the run ending once time - dt > tlim (dumses.f90:115-159)."""
    o = Oracle(MRI_P)
    o.set_state(condinit(MRI_P, "mri", **MRI_IC))
    o.boundary(0.0, 0.0)
    tlim, dthist, dtdump = 0.05, 0.012, 0.02
    rows = o.run_history(tlim, dthist, 200)
    driver(tmp_path, MRI.format(tlim=tlim, restart=0, dtdump=dtdump, dthist=dthist), "--iso", 1, "--ic", "mri",
           "--beta", MRI_IC["beta"], "--amp", MRI_IC["amp"], "--seed", MRI_IC["seed"],
           "--final-dump", tmp_path / "final.bin")
    hist = parse_history(tmp_path / "history.txt")
    assert hist.shape == rows.shape, (hist.shape, rows.shape)
    ref = np.array([[float(f"{v:.5E}") for v in r] for r in rows])  # the oracle at printed precision
    scale = np.maximum(np.abs(ref), 1e-30)
    # time and dt are bit-identical (printed the same); the sums to 1 unit of the 6th digit
    assert np.array_equal(hist[:, :2], ref[:, :2])
    assert np.all(np.abs(hist[:, 2:] - ref[:, 2:]) <= 1.01e-5 * scale[:, 2:] + 1e-14 * np.abs(ref[:, 2:]).max()), \
        (hist - ref)[:, 2:]
    u, tg, _ = read_dump(tmp_path / "final.bin", MRI_P)
    assert tg > tlim
    compare_states(u, o.uin, MRI_P)
    # dumps: 0 at t = 0, then one per dtdump crossing, each stamped with its time
    dumps = sorted(p for p in tmp_path.glob("output_*/data.000000.bin"))
    times = [dump_header(p)["time"] for p in dumps]
    assert times[0] == 0.0 and len(dumps) == 1 + int(tg // dtdump) - (1 if tg % dtdump == 0 else 0)
    for n, t in enumerate(times[1:], 1):
        assert t > n * dtdump and t - dtdump * n < 0.01, (n, t)


def test_driver_restart_from_a_dump_matches_the_full_run(tmp_path):
    """restart = 1 reads output_000001 (init.f90:114-119) and continues the loop from its
    time: the end state equals that of the run that never stopped.  (Its later dumps fall
    at other times: the dump clock restarts at the restart time, dumses.f90:68.)"""
    tlim, dtdump = 0.03, 0.01
    ic = ("--iso", 1, "--ic", "mri", "--beta", MRI_IC["beta"], "--amp", MRI_IC["amp"], "--seed", MRI_IC["seed"])
    full = tmp_path / "full"
    full.mkdir()
    driver(full, MRI.format(tlim=tlim, restart=0, dtdump=dtdump, dthist=-1.0), *ic, "--final-dump", full / "end.bin")
    rest = tmp_path / "rest"
    (rest / "output_000001").mkdir(parents=True)
    (rest / "output_000001" / "data.000000.bin").write_bytes((full / "output_000001" / "data.000000.bin").read_bytes())
    driver(rest, MRI.format(tlim=tlim, restart=1, dtdump=dtdump, dthist=-1.0), "--iso", 1,
           "--final-dump", rest / "end.bin")
    a, ta, dta = read_dump(full / "end.bin", MRI_P)
    b, tb, dtb = read_dump(rest / "end.bin", MRI_P)
    assert (ta, dta) == (tb, dtb)
    assert np.array_equal(a, b)
