"""Generate the dump and history-file fixtures and check them with the reference's own reader.

The reference's Python tool dumpy (utils/dumpy/data/rd_dumses.py, rd_history.py) reads the
Fortran 'binary' dumps of output.f90:224-235 and the history.txt of the MRI history routine.
This script writes a small seeded dump and a three-line history file with this package,
reads both back with dumpy, checks every field, and records the result next to the files:

    dump/output_000001/data.000000.bin   4x3x3 grid, seeded uin, time 0.125, dt 1e-3
    history/history.txt                  three lines of seeded sums
    dump_golden.json                     parameters, seed, sha256, what dumpy read

dumpy imports h5py, netCDF4, tables and pylab at module level; none of them is used by the
binary or history readers, so they are replaced by empty modules here.  Run it where the
reference tree is present (python tests/golden/make_dump_golden.py <reference root>); the
tests only read the committed fixtures.
"""
from __future__ import annotations

import hashlib
import importlib.util
import json
import pathlib
import sys
import types

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

import dumses_hybrid_b200 as dg  # noqa: E402

PARAMS = dict(ndim=3, nx=4, ny=3, nz=3, xmin=-0.5, xmax=0.5, ymin=0.0, ymax=4.0, zmin=-0.25, zmax=0.25,
              gamma=5.0 / 3.0, ciso=0.0)
SEED = 2024
TIME, DT = 0.125, 1.0e-3
HIST_SEED = 7
HIST_TIMES = [(0.0, 2.5e-3), (0.1, 2.4e-3), (0.2, 2.3e-3)]


def seeded_uin(params: dg.Params, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal(params.shape))


def seeded_sums(seed: int, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, 9)) * 10.0 ** rng.integers(-6, 2, size=(n, 9))


def load_dumpy(root: pathlib.Path):
    for name in ("h5py", "netCDF4", "tables", "pylab"):
        sys.modules.setdefault(name, types.ModuleType(name))
    data = root / "utils" / "dumpy" / "data"
    spec = importlib.util.spec_from_file_location("dumpy_data", data / "__init__.py",
                                                  submodule_search_locations=[str(data)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dumpy_data"] = mod
    spec.loader.exec_module(mod)
    return mod


def main(root: pathlib.Path) -> None:
    params = dg.Params(**PARAMS)
    uin = seeded_uin(params, SEED)
    dump = dg.dump_filename(1, 0, HERE / "dump")
    dg.write_dump(dump, params, uin, TIME, DT)
    hist = HERE / "history" / "history.txt"
    hist.parent.mkdir(exist_ok=True)
    sums = seeded_sums(HIST_SEED, len(HIST_TIMES))
    for (t, dt), s in zip(HIST_TIMES, sums):
        dg.write_history(hist, t, dt, s)

    dumpy = load_dumpy(root)
    d = dumpy.DumsesData()
    d.load(idump=1, dir_=str(HERE / "dump") + "/", nghost=3, ndim=3)
    geo = dg.Params(**PARAMS)
    expect_meta = dict(nx=geo.nx, ny=geo.ny, nz=geo.nz, time=TIME, dt=DT, dx=(geo.xmax - geo.xmin) / geo.nx,
                       dy=(geo.ymax - geo.ymin) / geo.ny, dz=(geo.zmax - geo.zmin) / geo.nz, xmin=geo.xmin,
                       xmax=geo.xmax, ymin=geo.ymin, ymax=geo.ymax, zmin=geo.zmin, zmax=geo.zmax,
                       gamma=geo.gamma, ciso=geo.ciso)
    for k, v in expect_meta.items():
        assert getattr(d, k) == v, (k, getattr(d, k), v)
    act = uin[3:-3, 3:-3, 3:-3]  # DumsesData.load returns the active cells
    assert np.array_equal(d.rho, act[..., 0]) and np.array_equal(d.E, act[..., 4])
    assert np.array_equal(d.rhou, act[..., 1:4])
    assert np.array_equal(d.B, act[..., 5:8]) and np.array_equal(d.Br, act[..., 8:11])
    # the ghosted arrays of the file, through dumpy's per-file binary reader
    r = dumpy.rd_dumses.DumsesDataFactory.makeData("bin", geo.nx, geo.ny, geo.nz, 1, 1, 1, geo.nx, geo.ny, geo.nz, 1)
    full = r._load(idump=1, dir_=str(HERE / "dump") + "/", nghost=3, mype=0, ndim=3, ext="bin")
    assert np.array_equal(full["rho"], uin[..., 0]) and np.array_equal(full["E"], uin[..., 4])
    assert np.array_equal(full["rhou"], uin[..., 1:4])
    assert np.array_equal(full["B"], uin[..., 5:8]) and np.array_equal(full["Br"], uin[..., 8:11])

    h = dumpy.DumsesHistory()
    h.load(filedir=str(hist.parent) + "/")
    assert list(h.dict.keys()) == list(dg.HISTORY_KEYS), list(h.dict.keys())
    table = np.array([[t, dt, *s] for (t, dt), s in zip(HIST_TIMES, sums)])
    for c, k in enumerate(dg.HISTORY_KEYS):
        assert np.allclose(h.dict[k], table[:, c], rtol=1e-5, atol=0.0), k

    record = {
        "params": PARAMS, "seed": SEED, "time": TIME, "dt": DT,
        "dump": str(dump.relative_to(HERE)),
        "dump_sha256": hashlib.sha256(dump.read_bytes()).hexdigest(),
        "dump_bytes": dump.stat().st_size,
        "history": str(hist.relative_to(HERE)), "history_seed": HIST_SEED, "history_times": HIST_TIMES,
        "history_sha256": hashlib.sha256(hist.read_bytes()).hexdigest(),
        "checked_by": "utils/dumpy/data/rd_dumses.py DumsesData.load (metadata; rho, E, rhou, B, Br of the active "
                      "cells equal) and the binary data reader's _load (the ghosted arrays equal), "
                      "utils/dumpy/data/rd_history.py DumsesHistory.load (11 keys in order, values to 6 digits)",
    }
    (HERE / "dump_golden.json").write_text(json.dumps(record, indent=1) + "\n")
    print(json.dumps(record, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_dump_golden.py <reference project root>")
    main(pathlib.Path(sys.argv[1]))
