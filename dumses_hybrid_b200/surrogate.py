"""Training recipe of the learned face flux, shared by the benchmark and the validation.

The network (:class:`dumses_hybrid_b200.FluxNet`) learns HLLD minus LLF per interface
from interfaces that the code itself generates: snapshots of a plain FP32 run of the
same problem are harvested with FP64 HLLD labels, the inputs and outputs are
standardised, and Adam runs on the device in three equal phases at learning rates
1e-3, 3e-4 and 1e-4.  A later snapshot, not trained on, measures the network.
"""
from __future__ import annotations

import time

import numpy as np

from . import Context, FluxNet, Params

OUTPUTS = ["mass", "energy", "normal_momentum", "t1_momentum", "B_t1", "t2_momentum", "B_t2", "p_star"]


def held_out_ratio(net: FluxNet, x: np.ndarray, t: np.ndarray) -> np.ndarray:
    """Per output: L1 of (LLF + network - HLLD) over L1 of (LLF - HLLD), fluxes weighted by the jump."""
    y = net.forward(x)
    jump = x[:, 14:15]
    return np.sum(np.abs(y - t) * jump, 0) / np.maximum(np.sum(np.abs(t) * jump, 0), 1e-300)


def train_flux_net(params: Params, u0: np.ndarray, snapshots: int = 2, every: int = 5, stride: int = 1,
                   epochs: float = 3.0, batch: int = 65536, seed: int = 7) -> tuple[FluxNet, dict]:
    """Harvest `snapshots` states `every` steps apart from a plain FP32 run started at u0,
    train a network on them and measure it on the next snapshot.  Returns (net, info)."""
    t0 = time.perf_counter()
    net = FluxNet(device=params.device, seed=seed)
    pt = Params(**{**params.__dict__, "precision": "fp32", "surrogate": False})
    with Context(pt) as ctx, FluxNet(device=params.device, seed=seed + 1) as probe:
        ctx.upload(u0)
        ctx.boundary(0.0, 0.0)
        ts = 0.0
        for _ in range(snapshots):
            ts, _ = ctx.run(every, ts)
            net.harvest(ctx, stride=stride)
        ts, _ = ctx.run(every, ts)
        probe.harvest(ctx, stride=stride * 16 + 1)
        xh, th = probe.samples()
    t1 = time.perf_counter()
    ns = net.sample_count
    net.fit_envelope(0.0)
    net.fit_scaling()
    phase = max(1, int(epochs * ns / batch) // 3)
    for lr in (1e-3, 3e-4, 1e-4):
        loss = net.train(phase, batch=batch, lr=lr)
    t2 = time.perf_counter()
    ratio = held_out_ratio(net, xh, th)
    info = {"samples": int(ns), "batch": batch, "adam_steps": 3 * phase, "final_loss": float(loss),
            "harvest_s": t1 - t0, "train_s": t2 - t1, "train_samples_per_s": 3 * phase * batch / (t2 - t1),
            "held_out_faces": int(xh.shape[0]),
            "held_out_error_ratio": {
                "definition": "per output, L1 of (LLF + network - HLLD) over L1 of (LLF - HLLD) on held-out faces",
                "outputs": OUTPUTS, "ratio": [float(r) for r in ratio], "mean": float(np.mean(ratio))},
            "network": f"17-{'-'.join([str(net.shape[0])] * net.shape[1])}-8 SmeLU, bf16 weights, fp32 accumulate "
                       "(tcgen05), Adam, lr 1e-3 / 3e-4 / 1e-4 in three equal phases, standardised inputs and outputs"}
    return net, info
