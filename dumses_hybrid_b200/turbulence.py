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

With --steps N every arm instead runs exactly N steps from the same initial state (the
arms' dt sequences then differ by round-off only), and the results add the relative L1
of each FP32 arm's final state against the FP64 arm's.  --arms fp64,fp32,fp32nn adds the
FP32 arm with the learned face flux (trained on the device first, as the benchmark
trains it) and its fallback fraction; --box cube puts the grid on [-0.5, 0.5]^3 H with
cubic cells; --beta sets the plasma beta of the net vertical field.  The 512^3 case at
beta = 400:

  python -m dumses_hybrid_b200.turbulence --grid 512,512,512 --box cube --beta 400 \
      --steps 3000 --every 100 --arms fp64,fp32,fp32nn --nn-stride 8
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


def box_params(precision: str, nx: int = 128, ny: int = 256, nz: int = 128, box: str = "c2"):
    """The shearing box on [0.5, 1, 0.5] H (box c2) or on the cube [-0.5, 0.5]^3 H (box cube)."""
    from dumses_hybrid_b200 import Params
    hx, hy, hz = (0.25, 0.5, 0.25) if box == "c2" else (0.5, 0.5, 0.5)
    return Params(ndim=3, iso=1, nx=nx, ny=ny, nz=nz, xmin=-hx, xmax=hx, ymin=-hy, ymax=hy, zmin=-hz,
                  zmax=hz, gamma=5.0 / 3.0, ciso=1.0, omega0=1.0, courant=0.8, slope_type=2, riemann="hlld",
                  riemann2d="hlld", bdtypex="shearingbox", fargo=True, precision=precision)


def run(precision: str, u0: np.ndarray, tend: float, every: int, grid, max_s: float = 0.0,
        progress_s: float = 30.0, box: str = "c2", nsteps: int = 0, net=None) -> dict:
    """One arm to time tend (or for exactly nsteps steps when nsteps > 0), or until max_s
    seconds of wall time have passed (0: no limit).  net: the learned face flux to attach
    (FP32).  Prints a progress line (time, steps, last dt, alpha, magnetic pressure) every
    progress_s seconds, and ends the arm at the first non-finite history value or library error."""
    from dumses_hybrid_b200 import Context, DumsesError
    p = box_params(precision, *grid, box=box)
    if net is not None:
        p.surrogate = True
    rows, steps, t, dt = [], 0, 0.0, 0.0
    w0 = wlast = time.time()
    error = None
    faces = fallback = 0
    with Context(p) as g:
        if net is not None:
            g.attach_surrogate(net)
        g.upload(u0)
        g.boundary(0.0, 0.0)
        rows.append([t, *g.history()])
        while (steps < nsteps if nsteps > 0 else t < tend) and not (max_s > 0 and time.time() - w0 > max_s):
            if nsteps > 0:
                every = min(every, nsteps - steps)
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
        if net is not None:
            faces, fallback = g.surrogate_stats()
        u = g.download()
    out = {"rows": np.array(rows), "steps": steps, "wall_s": time.time() - w0, "state": u,
           "stopped_early": (steps < nsteps) if nsteps > 0 else t < tend, "error": error}
    if net is not None:
        out["faces"], out["fallback_fraction"] = faces, fallback / max(faces, 1)
    print(json.dumps({"arm": precision, "steps": steps, "t_end": t, "wall_s": out["wall_s"],
                      "stopped_early": out["stopped_early"], "error": error}), flush=True)
    return out


def block_stats(t: np.ndarray, v: np.ndarray, t0: float, nblocks: int = 5) -> tuple[float, float]:
    """Mean of v over t >= t0 and the standard error of that mean from nblocks block means."""
    sel = v[t >= t0]
    blocks = np.array_split(sel, nblocks)
    means = np.array([b.mean() for b in blocks if len(b)])
    return float(sel.mean()), float(means.std(ddof=1) / math.sqrt(len(means)))


NAMES = ["rho", "rho_vx", "rho_vy", "rho_vz", "E", "Bx", "By", "Bz"]


def l1_rel(a64: np.ndarray, a: np.ndarray) -> dict:
    """Relative L1 of a against a64 over the active cells, per variable; the components of a
    vector (momentum, B) over the mean L1 of the whole vector."""
    a64, a = a64[3:-3, 3:-3, 3:-3], a[3:-3, 3:-3, 3:-3]
    out = {}
    for v, nm in enumerate(NAMES):
        lo, hi = {1: (1, 4), 2: (1, 4), 3: (1, 4), 5: (5, 8), 6: (5, 8), 7: (5, 8)}.get(v, (v, v + 1))
        den = float(sum(np.sum(np.abs(a64[..., w])) for w in range(lo, hi)) / (hi - lo))
        if den > 0:
            out[nm] = float(np.sum(np.abs(a[..., v] - a64[..., v])) / den)
    return out


def main() -> None:
    from dumses_hybrid_b200 import condinit

    ap = argparse.ArgumentParser()
    ap.add_argument("--orbits", type=float, default=10.0)
    ap.add_argument("--every", type=int, default=200, help="steps between history samples")
    ap.add_argument("--grid", default="128,256,128")
    ap.add_argument("--box", choices=["c2", "cube"], default="c2", help="[0.5,1,0.5] H (c2) or [-0.5,0.5]^3 H")
    ap.add_argument("--beta", type=float, default=1000.0, help="plasma beta of the net vertical field")
    ap.add_argument("--steps", type=int, default=0, help="run every arm for exactly this many steps (0: --orbits)")
    ap.add_argument("--arms", default="fp64,fp32", help="fp64 first, then any of fp32, fp32nn")
    ap.add_argument("--nn-stride", type=int, default=1, help="learned flux: harvest every stride-th face")
    ap.add_argument("--nn-epochs", type=float, default=3.0)
    ap.add_argument("--out", default="", help="save the histories to this .npz")
    ap.add_argument("--max-minutes", type=float, default=0.0,
                    help="wall-time limit of the FP64 arm (0: none); the FP32 arm then runs to the time it reached")
    args = ap.parse_args()
    grid = tuple(int(s) for s in args.grid.split(","))
    arm_names = [a for a in args.arms.split(",") if a]
    if arm_names[0] != "fp64":
        raise SystemExit("the first arm must be fp64 (the others are compared with it)")
    tend = 2.0 * math.pi * args.orbits
    u0 = condinit(box_params("fp64", *grid, box=args.box), "mri", beta=args.beta, amp=0.1, seed=2024)
    arms = {"fp64": run("fp64", u0, tend, args.every, grid, 60.0 * args.max_minutes, box=args.box, nsteps=args.steps)}
    s64 = arms["fp64"].pop("state")
    finite = {"fp64": bool(np.isfinite(s64[..., :8]).all())}
    l1 = {}
    if args.out:
        np.savez(args.out, columns=np.array(COLUMNS), fp64=arms["fp64"]["rows"])
    tend = min(tend, float(arms["fp64"]["rows"][-1, 0]))  # the same physical time in every arm
    nsteps = arms["fp64"]["steps"] if args.steps > 0 else 0
    nn_info = None
    for name in arm_names[1:]:
        net = None
        if name == "fp32nn":
            from dumses_hybrid_b200.surrogate import train_flux_net
            net, nn_info = train_flux_net(box_params("fp32", *grid, box=args.box), u0, stride=args.nn_stride,
                                          epochs=args.nn_epochs)
        arms[name] = run("fp32", u0, tend, args.every, grid, box=args.box, nsteps=nsteps, net=net)
        if net is not None:
            net.close()
        st = arms[name].pop("state")
        finite[name] = bool(np.isfinite(st[..., :8]).all())
        if nsteps > 0:
            l1[name] = l1_rel(s64, st)
        del st
    box = "0.5x1x0.5" if args.box == "c2" else "1x1x1"
    res = {"workload": f"shearing_box_mri_fargo_{grid[0]}x{grid[1]}x{grid[2]}_box_{box}_beta_{args.beta:g}",
           "orbits": args.orbits if args.steps == 0 else None, "steps_per_arm": args.steps or None,
           "t_target": 2.0 * math.pi * args.orbits, "t_compared": tend, "history_every_steps": args.every,
           "averaged_over": "t >= t_compared / 2", "error": "standard error of the mean from 5 block means"}
    r64 = arms["fp64"]["rows"]
    for prec, a in arms.items():
        r = a["rows"]
        out = {"steps": a["steps"], "t_end": float(r[-1, 0]), "orbits_reached": float(r[-1, 0]) / (2 * math.pi),
               "wall_s": a["wall_s"], "stopped_early": a["stopped_early"]}
        for nm in ("max+rey", "maxwell", "reynolds", "magp"):
            m, e = block_stats(r[:, 0], r[:, COLUMNS.index(nm)], tend / 2)
            out[nm] = {"mean": m, "stderr": e}
        magp0 = r[0, COLUMNS.index("magp")]
        grown = np.nonzero(r[:, COLUMNS.index("magp")] > 10.0 * magp0)[0]
        out["t_magp_10x"] = float(r[grown[0], 0]) if len(grown) else None
        out["max_abs_divB_sum"] = float(np.abs(r[:, COLUMNS.index("divB")]).max())
        out["finite"] = finite[prec]
        if prec != "fp64":
            n = min(len(r), len(r64))
            ia = COLUMNS.index("max+rey")
            # the alpha stress sample by sample, over the largest |alpha| of the FP64 arm
            out["alpha_max_abs_diff_over_max_alpha"] = float(np.abs(r[:n, ia] - r64[:n, ia]).max() /
                                                             max(np.abs(r64[:n, ia]).max(), 1e-300))
            if prec in l1:
                out["l1_rel_vs_fp64"] = l1[prec]
            if "fallback_fraction" in a:
                out["fallback_fraction"] = a["fallback_fraction"]
                out["faces"] = a["faces"]
        res[prec] = out
    if nn_info is not None:
        res["fp32nn"]["network"] = {k: nn_info[k] for k in ("samples", "adam_steps", "final_loss", "train_s")}
        res["fp32nn"]["network"]["held_out_error_ratio_mean"] = nn_info["held_out_error_ratio"]["mean"]
    a64 = res["fp64"]["max+rey"]
    for prec in arm_names[1:]:
        a = res[prec]["max+rey"]
        res[prec]["alpha_minus_fp64_in_combined_stderr"] = (a["mean"] - a64["mean"]) / max(
            math.hypot(a64["stderr"], a["stderr"]), 1e-300)
    if args.out:
        np.savez(args.out, columns=np.array(COLUMNS), **{k: v["rows"] for k, v in arms.items()})
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
