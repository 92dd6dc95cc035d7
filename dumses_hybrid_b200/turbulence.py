"""Saturated MRI turbulence in the FP64 and FP32 paths.

The shearing box of the reference's MRI problem at the size of its long test: 128 x 256 x
128 cells on [0.5, 1, 0.5] H (dx = dy = dz = H/256), Omega = 1, q = 1.5, isothermal with
c_s = 1, net vertical field beta = 1000, velocity kicks uniform in +-0.05 c_s (seeded),
shear-periodic x, FARGO on, HLLD/HLLD, MC slopes, CFL 0.8.  Each arithmetic runs from the
same initial state for `orbits` orbits, with the MRI history sums (the reference's
src/problem/mri/history.f90: volume averages of the Maxwell stress -BxBy, the Reynolds
stress rho vx dvy, the magnetic pressure, ...) sampled every `every` steps.

Once the flow is turbulent the FP64 and FP32 states decorrelate (any two round-offs do),
so what the FP32 path has to reproduce is the statistics of the saturated state: the
alpha stress (Maxwell + Reynolds over rho0 c_s^2 = 1) and the magnetic pressure, averaged
over the second half of the run, with standard errors from five block means.  Prints a
line per arm as it ends and one JSON line of results; --out saves the histories (.npz);
--max-minutes bounds the FP64 arm's wall time, the FP32 arm then runs to the same time.

  python -m dumses_hybrid_b200.turbulence --orbits 10
"""
from __future__ import annotations

import argparse
import json
import math
import pathlib
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

COLUMNS = ("time", "mass", "maxwell", "reynolds", "max+rey", "magp", "meanBx", "meanBy", "meanBz", "divB")


def box_params(precision: str, nx: int = 128, ny: int = 256, nz: int = 128):
    from dumses_hybrid_b200 import Params
    return Params(ndim=3, iso=1, nx=nx, ny=ny, nz=nz, xmin=-0.25, xmax=0.25, ymin=-0.5, ymax=0.5, zmin=-0.25,
                  zmax=0.25, gamma=5.0 / 3.0, ciso=1.0, omega0=1.0, courant=0.8, slope_type=2, riemann="hlld",
                  riemann2d="hlld", bdtypex="shearingbox", fargo=True, precision=precision)


def run(precision: str, u0: np.ndarray, tend: float, every: int, grid, max_s: float = 0.0,
        progress_s: float = 30.0) -> dict:
    """One arm to time tend, or until max_s seconds of wall time have passed (0: no limit).
    Prints a progress line (time, steps, last dt, alpha, magnetic pressure) every progress_s
    seconds, and ends the arm at the first non-finite history value or library error."""
    from dumses_hybrid_b200 import Context, DumsesError
    p = box_params(precision, *grid)
    rows, steps, t, dt = [], 0, 0.0, 0.0
    w0 = wlast = time.time()
    error = None
    with Context(p) as g:
        g.upload(u0)
        g.boundary(0.0, 0.0)
        rows.append([t, *g.history()])
        while t < tend and not (max_s > 0 and time.time() - w0 > max_s):
            try:
                t, dt = g.run(every, t)
            except DumsesError as e:
                error = str(e)
                break
            steps += every
            h = g.history()
            rows.append([t, *h])
            if not np.all(np.isfinite(h)):
                error = "non-finite history values"
                break
            if time.time() - wlast > progress_s:
                wlast = time.time()
                print(json.dumps({"arm": precision, "t": t, "orbits": t / (2 * math.pi), "steps": steps, "dt": dt,
                                  "alpha": float(h[3]), "magp": float(h[4]), "wall_s": wlast - w0}), flush=True)
        u = g.download()
    out = {"rows": np.array(rows), "steps": steps, "wall_s": time.time() - w0, "state": u, "stopped_early": t < tend,
           "error": error}
    print(json.dumps({"arm": precision, "steps": steps, "t_end": t, "wall_s": out["wall_s"],
                      "stopped_early": out["stopped_early"], "error": error}), flush=True)
    return out


def block_stats(t: np.ndarray, v: np.ndarray, t0: float, nblocks: int = 5) -> tuple[float, float]:
    """Mean of v over t >= t0 and the standard error of that mean from nblocks block means."""
    sel = v[t >= t0]
    blocks = np.array_split(sel, nblocks)
    means = np.array([b.mean() for b in blocks if len(b)])
    return float(sel.mean()), float(means.std(ddof=1) / math.sqrt(len(means)))


def main() -> None:
    from dumses_hybrid_b200 import condinit

    ap = argparse.ArgumentParser()
    ap.add_argument("--orbits", type=float, default=10.0)
    ap.add_argument("--every", type=int, default=200, help="steps between history samples")
    ap.add_argument("--grid", default="128,256,128")
    ap.add_argument("--out", default="", help="save both histories to this .npz")
    ap.add_argument("--max-minutes", type=float, default=0.0,
                    help="wall-time limit of the FP64 arm (0: none); the FP32 arm then runs to the time it reached")
    args = ap.parse_args()
    grid = tuple(int(s) for s in args.grid.split(","))
    tend = 2.0 * math.pi * args.orbits
    u0 = condinit(box_params("fp64", *grid), "mri", beta=1000.0, amp=0.1, seed=2024)
    arms = {"fp64": run("fp64", u0, tend, args.every, grid, 60.0 * args.max_minutes)}
    if args.out:
        np.savez(args.out, columns=np.array(COLUMNS), fp64=arms["fp64"]["rows"])
    tend = min(tend, float(arms["fp64"]["rows"][-1, 0]))  # the same physical time in both arms
    arms["fp32"] = run("fp32", u0, tend, args.every, grid)
    res = {"workload": f"shearing_box_mri_fargo_{grid[0]}x{grid[1]}x{grid[2]}_box_0.5x1x0.5", "orbits": args.orbits,
           "t_target": 2.0 * math.pi * args.orbits, "t_compared": tend, "history_every_steps": args.every,
           "averaged_over": "t >= t_compared / 2", "error": "standard error of the mean from 5 block means"}
    for prec, a in arms.items():
        r = a["rows"]
        out = {"steps": a["steps"], "t_end": float(r[-1, 0]), "wall_s": a["wall_s"], "stopped_early": a["stopped_early"]}
        for name in ("max+rey", "maxwell", "reynolds", "magp"):
            m, e = block_stats(r[:, 0], r[:, COLUMNS.index(name)], tend / 2)
            out[name] = {"mean": m, "stderr": e}
        magp0 = r[0, COLUMNS.index("magp")]
        grown = np.nonzero(r[:, COLUMNS.index("magp")] > 10.0 * magp0)[0]
        out["t_magp_10x"] = float(r[grown[0], 0]) if len(grown) else None
        out["max_abs_divB_sum"] = float(np.abs(r[:, COLUMNS.index("divB")]).max())
        out["finite"] = bool(np.isfinite(a["state"][..., :8]).all())
        res[prec] = out
    a64, a32 = res["fp64"]["max+rey"], res["fp32"]["max+rey"]
    res["alpha_fp32_minus_fp64_in_combined_stderr"] = (a32["mean"] - a64["mean"]) / math.hypot(a64["stderr"],
                                                                                              a32["stderr"])
    if args.out:
        np.savez(args.out, columns=np.array(COLUMNS), fp64=arms["fp64"]["rows"], fp32=arms["fp32"]["rows"])
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
