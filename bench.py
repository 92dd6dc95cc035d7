#!/usr/bin/env python
"""Benchmark of the DUMSES Godunov MHD step on B200.

Headline workload: the 256^3 unstratified shearing-box MRI (isothermal, Omega = 1,
shear-periodic x, FARGO on, net vertical field beta = 1000, seeded velocity kicks),
HLLD face fluxes and HLLD edge EMFs, MC slopes, CFL 0.8 (--workload ot: the 3D
Orszag-Tang-type vortex on the periodic unit cube).  A step is one pass of the
reference loop body (compute_dt, godunov, fargo_update, boundary;
src/dumses.f90:82-120) over the whole grid.  By default three arithmetics run from
the same initial state: the FP64 plain path (bit-identical to the reference
arithmetic), the FP32 mixed path, and FP32 with the learned face flux (the
configuration the metric names, so the headline `value`).  The network of the last
is harvested and trained on the device before its timed region (dumses_hybrid_b200
.surrogate), and the line reports each FP32 arm's relative L1 error against the FP64
state after the same steps.

  value  zone-cycles/s with the state resident in HBM: K steps enqueued back to
         back (dg_run), timed with CUDA events on the library's stream.
  e2e    the same metric through the reference-facing C-ABI as the Fortran
         driver calls it: the state uploaded from pinned host memory, then per
         step dg_compute_dt (dt read back to the host), dg_godunov,
         dg_boundary, and the state downloaded at the end -- all inside the
         timed region.
  roofline  the dominant kernel's algorithmic HBM bytes (128 B per zone-cycle:
         read + write of the 8 conserved FP64 variables) per launch over its
         average CUDA-event duration, against the measured copy bandwidth; when
         the dominant kernel is the face network, its multiply-adds against the
         measured sustained BF16 tensor throughput.
  cpu_baseline  the CPU restatement of the reference (oracle/, C + OpenMP,
         FP64) on all host cores, on the same grid, initial state and step
         counts (the oracle builds the initial state itself).

--impl reference times that CPU implementation alone (the reference itself is
Fortran and no Fortran compiler exists on this image).
With torchrun and N > 1 the box is decomposed in z over the N processes (one GPU
each, dumses_hybrid_b200.slabs): every GPU owns an n^3 slab of an n x n x (n N)
box (weak scaling), the slabs exchange their 3-deep halos after every boundary
call with NCCL point-to-point operations and take the CFL minimum with an NCCL
all-reduce, as the reference's MPI ranks do (parallel.f90, physics.f90:123-129).
--slabs S puts S slabs on each process (S > 1 on one GPU runs the same
decomposed step with device copies for the halos).
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "zone-cycles/s at 256³: plain FP64 vs FP32+NN-flux at stated L1 vs FP64"
ALGO_BYTES_PER_ZONE = 128  # read + write of 8 conserved FP64 variables per zone-cycle
def nn_macs_per_face(width: int, depth: int) -> int:
    """The face network's multiply-adds per face: 17 -> width (x depth hidden layers) -> 8."""
    return 17 * width + (depth - 1) * width * width + width * 8


WORKLOADS = {"ot": "orszag_tang_3d", "mri": "shearing_box_mri_fargo"}


def workload_params(n: int, device: int = 0, precision: str = "fp64", kind: str = "ot", nu: float = 0.0,
                    eta: float = 0.0):
    """ot: the 3D Orszag-Tang-type vortex on the periodic unit cube (adiabatic).
    mri: the unstratified isothermal shearing box of the MRI set-up at n^3 with cubic cells on
    [-0.5,0.5]^3 H, Omega = 1, q = 1.5, c_s = 1, shear-periodic x, FARGO on.
    nu, eta > 0 add the dissipation step (viscosity, resistivity) after boundary."""
    from dumses_hybrid_b200 import Params
    if kind == "mri":
        return Params(ndim=3, iso=1, nx=n, ny=n, nz=n, xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5, zmin=-0.5,
                      zmax=0.5, gamma=5.0 / 3.0, ciso=1.0, omega0=1.0, courant=0.8, slope_type=2, riemann="hlld",
                      riemann2d="hlld", bdtypex="shearingbox", fargo=True, device=device, precision=precision,
                      nu=nu, eta=eta)
    return Params(ndim=3, nx=n, ny=n, nz=n, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0,
                  gamma=5.0 / 3.0, courant=0.8, slope_type=2, riemann="hlld", riemann2d="hlld", device=device,
                  precision=precision, nu=nu, eta=eta)


def initial_state(P, kind: str):
    from dumses_hybrid_b200 import condinit
    if kind == "mri":
        # net vertical field, beta = 1000, velocity kicks uniform in +-0.05 c_s, seed 2024
        return condinit(P, "mri", beta=1000.0, amp=0.1, seed=2024)
    return condinit(P, "orszag_tang")


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = ROOT / f".clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        try:
            self.f.close()
        except Exception:
            pass

    def summary(self) -> dict:
        try:
            lines = self.path.read_text().strip().splitlines()
            self.path.unlink()
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            if self.uuid and f[0] != self.uuid:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def rank_barrier(dist, cuda: bool = True) -> None:
    """All ranks meet before and after a timed region."""
    if dist is not None:
        dist.barrier()
    if cuda:
        import torch
        torch.cuda.synchronize()


def rank_max(x: float, dist, device: str = "cuda") -> float:
    """The largest value of x over the ranks (a timed region ends when its slowest rank does)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(steps: int, warmup: int, n: int = 256, kind: str = "mri", nu: float = 0.0, eta: float = 0.0) -> dict:
    """The CPU restatement of the reference (oracle/, C + OpenMP, FP64) on all host cores, on the
    same n^3 workload: the initial state is built by the oracle's own copy of the problem set-up
    (bit-identical to the library's), so this leg loads no product code."""
    sys.path.insert(0, str(ROOT / "tests"))
    from _oracle import Oracle, lib as oracle_lib
    cores = os.cpu_count() or 1
    oracle_lib().or_set_threads(cores)
    P = workload_params(n, kind=kind, nu=nu, eta=eta)
    o = Oracle(P)
    if kind == "mri":
        o.condinit("mri", beta=1000.0, amp=0.1, seed=2024)
    else:
        o.condinit("orszag_tang")
    o.boundary(0.0, 0.0)
    t = 0.0
    for _ in range(warmup):
        t, _ = o.step(t)
    t0 = time.perf_counter()
    for _ in range(steps):
        t, _ = o.step(t)
    el = time.perf_counter() - t0
    o.close()
    return {"value": n ** 3 * steps / el, "unit": "zone-cycles/s", "cores": cores, "kind": "port",
            "sample": f"the {n}^3 {WORKLOADS[kind]} workload itself (same grid, initial state and steps), {steps} timed "
                      f"steps after {warmup} warm-up, C restatement of the reference with OpenMP (FP64)",
            "seconds": el, "same_config": True}


def run_reference(args, rank: int) -> None:
    if rank != 0:
        return
    cb = cpu_baseline(max(args.steps, 1), max(args.warmup, 0), n=args.n, kind=args.workload, nu=args.nu, eta=args.eta)
    line = {"metric": METRIC, "value": cb["value"], "unit": "zone-cycles/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * cb["seconds"] / max(args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{WORKLOADS[args.workload]}_{args.n}^3", "grid": [args.n] * 3,
                       "solver": "hlld/hlld", "slope": "mc", "courant": 0.8},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "zone-cycles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256, help="grid edge (the headline workload is 256)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", choices=["fp64", "fp32", "fp32nn", "both"], default="both",
                    help="both: time the FP64 plain path, the FP32 mixed path and FP32 with the learned "
                         "face flux (headline) in one run")
    ap.add_argument("--nn-snapshots", type=int, default=2, help="training snapshots harvested")
    ap.add_argument("--nn-every", type=int, default=5, help="steps between snapshots")
    ap.add_argument("--nn-stride", type=int, default=1, help="harvest every stride-th face")
    ap.add_argument("--nn-epochs", type=float, default=3.0, help="passes over the harvested samples")
    ap.add_argument("--nn-batch", type=int, default=65536)
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="mri")
    ap.add_argument("--nu", type=float, default=0.0, help="viscosity: adds the dissipation step (default off)")
    ap.add_argument("--eta", type=float, default=0.0, help="resistivity: adds the dissipation step (default off)")
    ap.add_argument("--slabs", type=int, default=1,
                    help="z slabs per process: with N processes the box is n x n x (n N slabs), one n^3 slab "
                         "per slab (weak scaling); 1 with one process: the undecomposed n^3 box")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import datetime

    import numpy as np
    import torch

    import dumses_hybrid_b200 as dg
    from dumses_hybrid_b200 import build as dgbuild
    from dumses_hybrid_b200.surrogate import train_flux_net

    if rank == 0:
        dgbuild.build()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist.barrier()
        dgbuild.build()

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        pass

    def barrier():
        rank_barrier(dist, cuda=True)

    def max_over_ranks(x: float) -> float:
        return rank_max(x, dist, device="cuda")

    ncell = args.n ** 3
    nzslice = world * args.slabs

    def measure(precision: str, with_e2e: bool) -> dict:
        if nzslice > 1:
            return measure_slabs(precision, with_e2e)
        surrogate = precision == "fp32nn"
        P = workload_params(args.n, device=local_rank, precision="fp32" if surrogate else precision,
                            kind=args.workload, nu=args.nu, eta=args.eta)
        u0 = initial_state(P, args.workload)
        if surrogate:
            P.surrogate = True
            torch.cuda.synchronize()
            net, nn_info = train_flux_net(P, u0, snapshots=args.nn_snapshots, every=args.nn_every,
                                          stride=args.nn_stride, epochs=args.nn_epochs, batch=args.nn_batch)
            torch.cuda.synchronize()
        ctx = dg.Context(P)
        if surrogate:
            ctx.attach_surrogate(net)
        stream = torch.cuda.ExternalStream(ctx.stream)
        # device-resident timed region (value + per-kernel events for the roofline)
        ctx.upload(u0)
        ctx.boundary(0.0, 0.0)
        t_sim, _ = ctx.run(args.warmup, 0.0)
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx.profile(True)
        ctx.profile_read()
        launches0 = ctx.kernel_launches
        with ClockSampler(uuid) as clk:
            ev0.record(stream)
            t_sim, _ = ctx.run(args.steps, t_sim)
            ev1.record(stream)
            ev1.synchronize()
        barrier()
        out = {"launches": ctx.kernel_launches - launches0, "prof": ctx.profile_read(), "clocks": clk.summary()}
        if surrogate:
            faces, fallback = ctx.surrogate_stats()
            nn_info["faces_timed"] = faces
            nn_info["fallback_fraction"] = fallback / max(faces, 1)
            out["nn"] = nn_info
        ctx.profile(False)
        out["ms"] = max_over_ranks(ev0.elapsed_time(ev1))
        out["value"] = world * ncell * args.steps / (out["ms"] / 1e3)
        out["state"] = ctx.download() if rank == 0 else None
        out["sim_time"] = t_sim
        if with_e2e:
            # end-to-end through the reference-facing C-ABI, as the Fortran driver calls it
            nt = (args.n + 6) ** 3
            pinned = torch.empty((11, args.n + 6, args.n + 6, args.n + 6), dtype=torch.float64, pin_memory=True)
            host = pinned.numpy().T  # Fortran-ordered view (nx+6, ny+6, nz+6, 11)
            host[...] = u0
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.upload(host)
            ctx.boundary(0.0, 0.0)
            te = 0.0
            for _ in range(args.steps):
                dt = ctx.compute_dt()
                ctx.godunov(dt, te)
                if P.fargo:
                    ctx.fargo_update(dt)
                ctx.boundary(te, dt)
                ctx.dissipation(te, dt)
                te = te + dt
            ctx.download_into(host)
            e1.record(stream)
            e1.synchronize()
            barrier()
            ms_e2e = max_over_ranks(e0.elapsed_time(e1))
            out["e2e"] = {"value": world * ncell * args.steps / (ms_e2e / 1e3), "unit": "zone-cycles/s",
                          "h2d_bytes_per_step": 8 * nt * 8 / args.steps,
                          "d2h_bytes_per_step": (11 * nt * 8) / args.steps + 8,
                          "finite": bool(np.isfinite(host[..., :8]).all())}
        ctx.close()
        if surrogate:
            net.close()
        return out

    def measure_slabs(precision: str, with_e2e: bool) -> dict:
        """The box cut into nzslice z slabs of n^3 (args.slabs per process, one process per GPU):
        the reference's loop body over the slabs with the halo exchange (NCCL point-to-point
        between processes, device copies within one) and the CFL minimum over all slabs."""
        from dataclasses import replace as dc_replace

        from dumses_hybrid_b200.slabs import SlabSet, slab_params
        surrogate = precision == "fp32nn"
        P = workload_params(args.n, device=local_rank, precision="fp32" if surrogate else precision,
                            kind=args.workload, nu=args.nu, eta=args.eta)
        zlo, zhi = (-0.5 * nzslice, 0.5 * nzslice) if args.workload == "mri" else (0.0, float(nzslice))
        box = dc_replace(P, nz=args.n * nzslice, zmin=zlo, zmax=zhi)
        S = SlabSet(box, nzslice, dist=dist, device=local_rank)
        # each slab's own initial state: the workload's set-up on the slab's cells (velocity
        # kicks seeded per slab)
        u0s = []
        for sp in S.params:
            if args.workload == "mri":
                u0s.append(dg.condinit(sp, "mri", beta=1000.0, amp=0.1, seed=2024 + 7919 * sp.zposition))
            else:
                u0s.append(dg.condinit(sp, "orszag_tang"))
        nets = []
        if surrogate:
            for c, u in zip(S.ctxs, u0s):
                c.close()
            one = dc_replace(P, surrogate=False)
            S.ctxs = []
            for sp, u in zip(S.params, u0s):
                torch.cuda.synchronize()
                net, nn_info = train_flux_net(one, u, snapshots=args.nn_snapshots, every=args.nn_every,
                                              stride=args.nn_stride, epochs=args.nn_epochs, batch=args.nn_batch)
                nets.append(net)
                c = dg.Context(dc_replace(sp, surrogate=True))
                c.attach_surrogate(net)
                S.ctxs.append(c)
            S.params = [dc_replace(sp, surrogate=True) for sp in S.params]
            S.rebuild_exchange()
        stream = torch.cuda.ExternalStream(S.ctxs[0].stream)
        S.upload(u0s)
        S.boundary(0.0, 0.0)
        t_sim = 0.0
        for _ in range(args.warmup):
            t_sim, _ = S.step(t_sim)
        S.sync()
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        S.ctxs[0].profile(True)
        S.ctxs[0].profile_read()
        launches0 = sum(c.kernel_launches for c in S.ctxs)
        with ClockSampler(uuid) as clk:
            ev0.record(stream)
            for _ in range(args.steps):
                t_sim, _ = S.step(t_sim)
            S.sync()
            ev1.record(stream)
            ev1.synchronize()
        barrier()
        out = {"launches": sum(c.kernel_launches for c in S.ctxs) - launches0, "prof": S.ctxs[0].profile_read(),
               "clocks": clk.summary()}
        if surrogate:
            faces = fallback = 0
            for c in S.ctxs:
                a, b = c.surrogate_stats()
                faces, fallback = faces + a, fallback + b
            nn_info["faces_timed"] = faces
            nn_info["fallback_fraction"] = fallback / max(faces, 1)
            out["nn"] = nn_info
        S.ctxs[0].profile(False)
        out["ms"] = max_over_ranks(ev0.elapsed_time(ev1))
        out["value"] = nzslice * ncell * args.steps / (out["ms"] / 1e3)
        out["state"] = S.ctxs[0].download() if rank == 0 else None
        out["sim_time"] = t_sim
        if with_e2e:
            # end-to-end through the public API: every slab's state uploaded from pinned host
            # memory, the loop with the host-side CFL minimum and the exchange, the states downloaded
            nt = (args.n + 6) ** 3
            hosts = []
            for u in u0s:
                pinned = torch.empty((11, args.n + 6, args.n + 6, args.n + 6), dtype=torch.float64, pin_memory=True)
                h = pinned.numpy().T
                h[...] = u
                hosts.append(h)
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            S.upload(hosts)
            S.boundary(0.0, 0.0)
            te = 0.0
            for _ in range(args.steps):
                te, _ = S.step(te)
            for c, h in zip(S.ctxs, hosts):
                c.download_into(h)
            S.sync()
            e1.record(stream)
            e1.synchronize()
            barrier()
            ms_e2e = max_over_ranks(e0.elapsed_time(e1))
            out["e2e"] = {"value": nzslice * ncell * args.steps / (ms_e2e / 1e3), "unit": "zone-cycles/s",
                          "h2d_bytes_per_step": len(hosts) * 8 * nt * 8 / args.steps,
                          "d2h_bytes_per_step": len(hosts) * ((11 * nt * 8) / args.steps + 8),
                          "finite": bool(all(np.isfinite(h[..., :8]).all() for h in hosts))}
        S.close()
        for net in nets:
            net.close()
        return out

    precisions = ["fp64", "fp32", "fp32nn"] if args.precision == "both" else [args.precision]
    head = precisions[-1]
    res = {pr: measure(pr, with_e2e=(pr != "fp64" or len(precisions) == 1)) for pr in precisions}

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm_peak else "fallback"
    hbm_peak = hbm_peak or 6650.0

    def kernel_table(r):
        return {k: {"ms_total": v[0], "launches": v[1], "ms_per_launch": v[0] / max(v[1], 1)}
                for k, v in r["prof"].items()}

    def roofline(r, precision):
        kernels = kernel_table(r)
        dom = max(kernels, key=lambda k: kernels[k]["ms_total"])
        per_launch_s = kernels[dom]["ms_per_launch"] / 1e3
        if dom == "nn_faces":
            # the network's multiply-adds and the face kernel's algorithmic bytes over the faces of one
            # direction: per face the 16 trace-core values of each of its two cells (each cell's
            # values serve its two faces of the direction: 64 B per face) and the 6-value flux
            # record (24 B).  The roof is the one the operational intensity reaches first: the
            # tensor pipe above the ridge point (peak flop rate / copy bandwidth), HBM below it.
            from dumses_hybrid_b200 import network_shape
            width, depth = network_shape()
            macs = nn_macs_per_face(width, depth)
            faces = (args.n + 1) * args.n * args.n
            flops = 2.0 * macs * faces
            nbytes = (16 * 4 + 6 * 4) * faces
            tpeak = peaks.get("bf16_tflops_sustained")
            src = "measured (sustained)" if tpeak else "fallback"
            tpeak = tpeak or 1400.0
            t_ach = flops / per_launch_s / 1e12
            b_ach = nbytes / per_launch_s / 1e9
            intensity = flops / nbytes
            ridge = tpeak * 1e12 / (hbm_peak * 1e9)
            traffic = None
            tpath = ROOT / "profiles" / f"ncu_traffic_{args.workload}{args.n}_fp32nn.json"
            if tpath.exists():
                try:
                    traffic = json.loads(tpath.read_text()).get(dom)
                except Exception:
                    traffic = None
            shape = f"17-{'-'.join([str(width)] * depth)}-8 MLP"
            if intensity >= ridge:
                out = {"bound": "tensor", "kernel": dom, "achieved": t_ach, "peak": tpeak, "unit": "TFLOP/s",
                       "frac": t_ach / tpeak, "peak_source": src}
            else:
                out = {"bound": "hbm", "kernel": dom, "achieved": b_ach, "peak": hbm_peak, "unit": "GB/s",
                       "frac": b_ach / hbm_peak, "peak_source": peak_src}
            out.update({"traffic": traffic, "algorithmic_flops_per_launch": flops,
                        "algorithmic_bytes_per_launch": nbytes, "intensity_flop_per_byte": intensity,
                        "ridge_flop_per_byte": ridge, "tensor_frac": t_ach / tpeak, "hbm_frac": b_ach / hbm_peak,
                        "note": f"one launch per face direction; 2 x {macs} flops and 88 bytes per face ({shape})"})
            upath = ROOT / "profiles" / "pipe_util_mri128.json"
            if upath.exists():
                try:
                    util = json.loads(upath.read_text()).get("fp32nn", {}).get(dom)
                    if util:
                        pipe = max(("fma", "alu", "xu", "tensor"), key=lambda p: util[p])
                        out["binding"] = {"pipe": pipe, "pipe_frac": util[pipe], "tensor_frac": util["tensor"],
                                          "issue_frac": util["issue"], "warps_frac": util["warps"],
                                          "source": "profiles/pipe_util_mri128.json (ncu, 128^3)"}
                except Exception:
                    pass
            return out
        # the slot's time per step (the FP64 Riemann slot is six launches per step: faces and
        # edges of each direction) against the step's algorithmic bytes of the 8 state variables
        slot_s = kernels[dom]["ms_total"] / args.steps / 1e3
        launches_per_step = kernels[dom]["launches"] / args.steps
        achieved = ALGO_BYTES_PER_ZONE * ncell / slot_s / 1e9
        traffic = None
        tpath = ROOT / "profiles" / f"ncu_traffic_{args.workload}{args.n}_{precision}.json"
        if tpath.exists():
            try:
                traffic = json.loads(tpath.read_text()).get(dom)
            except Exception:
                traffic = None
        step = ALGO_BYTES_PER_ZONE * ncell * args.steps / (r["ms"] / 1e3) / 1e9 / world
        out = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
               "frac": achieved / hbm_peak, "traffic": traffic, "peak_source": peak_src,
               "algorithmic_bytes_per_step": ALGO_BYTES_PER_ZONE * ncell, "launches_per_step": launches_per_step,
               "note": "achieved = the step's algorithmic bytes over the kernel slot's time per step (the sum of "
                       "its launches); traffic = DRAM bytes of the slot per step",
               "step_achieved": step, "step_frac": step / hbm_peak}
        # the pipe that binds the dominant kernel, from the committed ncu summary of the same kernel
        upath = ROOT / "profiles" / "pipe_util_mri128.json"
        if upath.exists():
            try:
                util = json.loads(upath.read_text()).get(precision, {}).get(dom)
                if util:
                    pipe = max(("fp64", "fma", "alu", "xu", "tensor"), key=lambda p: util[p])
                    out["binding"] = {"pipe": pipe, "pipe_frac": util[pipe], "issue_frac": util["issue"],
                                      "dram_frac": util["dram"], "source": "profiles/pipe_util_mri128.json (ncu, 128^3)"}
            except Exception:
                pass
        return out

    arith = {"fp64": "fp64 (bit-exact)",
             "fp32": "fp32 trace/Riemann/CT, compensated fp32 hi/lo state, fp64 gas pressure/dt minimum/diagnostics",
             "fp32nn": "as fp32, with the learned bf16 face flux (tcgen05) on smooth faces and exact HLLD elsewhere"}
    h = res[head]
    line = {"metric": METRIC, "value": h["value"], "unit": "zone-cycles/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": h["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if head == "fp64" else "f32", "data": "synthetic",
            "config": {"workload": f"{WORKLOADS[args.workload]}_{args.n}^3", "grid": [args.n] * 3,
                       "arithmetic": arith[head], "solver": "hlld/hlld", "slope": "mc", "courant": 0.8,
                       "parallelism": (f"z slabs x{nzslice} ({world} processes, NCCL halo exchange)" if nzslice > 1
                                       else "one GPU"),
                       **({"box": [args.n, args.n, args.n * nzslice]} if nzslice > 1 else {}),
                       "l2": "working set 8-13 GB per step >> 126 MB L2, no flush needed",
                       **({"nu": args.nu, "eta": args.eta} if args.nu > 0 or args.eta > 0 else {})},
            "e2e": h["e2e"], "gpu_launches": h["launches"], "roofline": roofline(h, head if head != "fp32nn" else "fp32"),
            "kernels": kernel_table(h), "clocks": h["clocks"], "sim_time": h["sim_time"]}
    if "nn" in h:
        line["nn_flux"] = h["nn"]
    names = ["rho", "rho_vx", "rho_vy", "rho_vz", "E", "Bx", "By", "Bz"]

    def l1_vs(a64, a):
        # relative L1 per variable; vector components over the L1 norm of the whole vector
        out = {}
        for v, nm in enumerate(names):
            group = {1: (1, 4), 2: (1, 4), 3: (1, 4), 5: (5, 8), 6: (5, 8), 7: (5, 8)}.get(v, (v, v + 1))
            den = float(np.sum(np.abs(a64[..., group[0]:group[1]])) / (group[1] - group[0]))
            if den > 0:
                out[nm] = float(np.sum(np.abs(a[..., v] - a64[..., v])) / den)
        return out

    if "fp64" in res and head != "fp64":
        f = res["fp64"]
        a64 = f["state"][3:-3, 3:-3, 3:-3]
        line["fp64_plain_path"] = {"value": f["value"], "ms_per_step": f["ms"] / args.steps,
                                   "roofline": roofline(f, "fp64"), "kernels": kernel_table(f), "clocks": f["clocks"]}
        line["speedup_vs_fp64"] = h["value"] / f["value"]
        line["l1_rel_vs_fp64"] = {"after_steps": args.steps + args.warmup,
                                  "normalisation": "per variable; vector components over the mean L1 of the vector",
                                  **l1_vs(a64, h["state"][3:-3, 3:-3, 3:-3])}
        if head == "fp32nn" and "fp32" in res:
            g = res["fp32"]
            line["fp32_plain_path"] = {"value": g["value"], "ms_per_step": g["ms"] / args.steps,
                                       "speedup_vs_fp64": g["value"] / f["value"],
                                       "l1_rel_vs_fp64": l1_vs(a64, g["state"][3:-3, 3:-3, 3:-3]),
                                       "kernels": kernel_table(g), "clocks": g["clocks"], "e2e": g.get("e2e")}
    if world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(args.steps, args.warmup, n=args.n, kind=args.workload, nu=args.nu, eta=args.eta)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
