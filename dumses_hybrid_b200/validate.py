"""Accuracy of the FP32 mixed path, with and without the learned face flux, against the
FP64 plain path over a physical time.

Runs the arithmetics from the same initial state, each with its own CFL steps, for
the same number of steps reaching at least `orbits` orbits (t = 2 pi orbits / Omega
for the shearing box, t = 0.5 for Orszag-Tang), and prints the relative L1 error
sum|u - u64| / sum|u64| over the active cells for every variable (vector components
over the mean L1 of their vector), the times reached and the div B of the states, as
one JSON line.  The network of the FP32+NN arm is trained first on snapshots of the
same problem (dumses_hybrid_b200.surrogate).

  python -m dumses_hybrid_b200.validate --workload mri --n 256 --orbits 1
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


def main() -> None:
    from bench import WORKLOADS, initial_state, workload_params
    import dumses_hybrid_b200 as dg

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="mri")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--orbits", type=float, default=1.0)
    ap.add_argument("--chunk", type=int, default=200)
    ap.add_argument("--no-nn", action="store_true", help="skip the FP32 + learned face flux arm")
    args = ap.parse_args()
    from dumses_hybrid_b200.surrogate import train_flux_net

    p64 = workload_params(args.n, precision="fp64", kind=args.workload)
    p32 = workload_params(args.n, precision="fp32", kind=args.workload)
    tend = 2 * math.pi * args.orbits / p64.omega0 if args.workload == "mri" else 0.5 * args.orbits
    u0 = initial_state(p64, args.workload)
    res = {"workload": f"{WORKLOADS[args.workload]}_{args.n}^3", "t_target": tend}
    g64 = dg.Context(p64)
    g64.upload(u0)
    g64.boundary(0.0, 0.0)
    t, steps, w0 = 0.0, 0, time.time()
    while t < tend:
        t, _ = g64.run(args.chunk, t)
        steps += args.chunk
    res.update(steps=steps, t_fp64=t, wall_fp64_s=time.time() - w0)
    u64 = g64.download()
    g64.close()
    g32 = dg.Context(p32)
    g32.upload(u0)
    g32.boundary(0.0, 0.0)
    t32, w0 = 0.0, time.time()
    for _ in range(steps // args.chunk):
        t32, _ = g32.run(args.chunk, t32)
    res.update(t_fp32=t32, wall_fp32_s=time.time() - w0)
    u32 = g32.download()
    g32.close()
    unn = None
    if not args.no_nn:
        pnn = workload_params(args.n, precision="fp32", kind=args.workload)
        pnn.surrogate = True
        net, info = train_flux_net(pnn, u0)
        res["nn_training"] = info
        gnn = dg.Context(pnn)
        gnn.attach_surrogate(net)
        gnn.upload(u0)
        gnn.boundary(0.0, 0.0)
        tnn, w0 = 0.0, time.time()
        for _ in range(steps // args.chunk):
            tnn, _ = gnn.run(args.chunk, tnn)
        faces, fallback = gnn.surrogate_stats()
        res.update(t_fp32nn=tnn, wall_fp32nn_s=time.time() - w0, nn_fallback_fraction=fallback / max(faces, 1))
        unn = gnn.download()
        gnn.close()
        net.close()
    a64 = u64[3:-3, 3:-3, 3:-3]
    names = ["rho", "rho_vx", "rho_vy", "rho_vz", "E", "Bx", "By", "Bz"]

    def l1_vs(a):
        out = {}
        for v, nm in enumerate(names):
            group = {1: (1, 4), 2: (1, 4), 3: (1, 4), 5: (5, 8), 6: (5, 8), 7: (5, 8)}.get(v, (v, v + 1))
            den = float(np.sum(np.abs(a64[..., group[0]:group[1]])) / (group[1] - group[0]))
            if den > 0:
                out[nm] = float(np.sum(np.abs(a[..., v] - a64[..., v])) / den)
        return out

    res["l1_rel_normalisation"] = "per variable; vector components over the mean L1 of the vector"
    res["l1_rel_fp32_vs_fp64"] = l1_vs(u32[3:-3, 3:-3, 3:-3])
    if unn is not None:
        res["l1_rel_fp32nn_vs_fp64"] = l1_vs(unn[3:-3, 3:-3, 3:-3])
    dx = (p64.xmax - p64.xmin) / p64.nx

    def divb(u):
        bx, by, bz = u[..., 5], u[..., 6], u[..., 7]
        d = ((bx[4:-2, 3:-3, 3:-3] - bx[3:-3, 3:-3, 3:-3]) + (by[3:-3, 4:-2, 3:-3] - by[3:-3, 3:-3, 3:-3])
             + (bz[3:-3, 3:-3, 4:-2] - bz[3:-3, 3:-3, 3:-3])) / dx
        return float(np.max(np.abs(d)) * dx / max(np.max(np.abs(u[..., 5:8])), 1e-300))

    res["max_divB_dx_over_Bmax"] = {"fp64": divb(u64), "fp32": divb(u32)}
    if unn is not None:
        res["max_divB_dx_over_Bmax"]["fp32nn"] = divb(unn)
    res["finite"] = bool(np.isfinite(u32[..., :8]).all() and np.isfinite(u64[..., :8]).all()
                         and (unn is None or np.isfinite(unn[..., :8]).all()))
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
