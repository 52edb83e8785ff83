"""Device timings of the learned closure (tensor-core side) and of its cost
inside the solver step.

    python -m multiphysics_fvm_b200.closure_bench [--n 64 128] [--iters 20]

Per grid size: ms per forward pass and per training step (CUDA events on the
closure's stream) with the tensor FLOP rates they imply, and the device time
per SSPRK3 step of the 3D Kelvin-Helmholtz setup without and with the closure
attached (fixed dt).  FLOPs are those executed on the tensor cores (input
layer padded to 16 channels):
forward 2*27*(16*32 + 32*32 + 32*16) per cell, training step forward +
data gradients of layers 3 and 2 + weight gradients of all layers.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

FWD_FLOP = 2 * 27 * (16 * 32 + 32 * 32 + 32 * 16)
DGRAD_FLOP = 2 * 27 * (16 * 32 + 32 * 32)
TRAIN_FLOP = 2 * FWD_FLOP + DGRAD_FLOP


def measured_peak():
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d.get("bf16_tflops")), "measured"
    except Exception:
        return 1590.0, "fallback"


def random_state(n, rng):
    rho = rng.uniform(1.0, 2.0, (n, n, n))
    v = rng.uniform(-0.5, 0.5, (3, n, n, n))
    p = rng.uniform(2.0, 3.0, (n, n, n))
    return np.stack([rho, rho * v[0], rho * v[1], rho * v[2], p / 0.4 + 0.5 * rho * (v * v).sum(0)]).astype(np.float32)


def run(n: int, iters: int, rng) -> dict:
    import torch
    from . import closure as CL
    from .closure_train import new_sim
    net = CL.Closure((n, n, n), seed=1)
    net.set_norm(1.4, [1.5, 0, 0, 0, 2.5], [0.5] * 5, [0.01] * 5, [1.0] * 5)
    u = torch.from_numpy(random_state(n, rng)).cuda()
    d = torch.from_numpy((rng.standard_normal((5, n, n, n)) * 1e-3).astype(np.float32)).cuda()
    net.features(u)
    ms_fwd = net.time_forward(iters)
    ms_train = net.time_train(u, d, 2e-3, (1.0 / n,) * 3, 1e-3, iters)
    cells = n ** 3
    out = {"n": n, "cells": cells, "ms_forward": ms_fwd, "ms_train_step": ms_train,
           "tflops_forward": cells * FWD_FLOP / (ms_fwd * 1e9),
           "tflops_train": cells * TRAIN_FLOP / (ms_train * 1e9)}
    # solver step with and without the closure (KH 3D, fixed dt)
    steps = 50
    plain = new_sim(n, 0)
    closed = new_sim(n, 0)
    net.attach(closed, beta=0.05)
    dt = 0.4 / n / 3.0
    for sim in (plain, closed):
        sim.step(3, dt=dt)  # warm-up; also sets the fixed dt
    out["ms_step_plain"] = plain.time_steps(steps, fixed_dt=True) / steps
    out["ms_step_closure"] = closed.time_steps(steps, fixed_dt=True) / steps
    out["status"] = max(plain.status(), closed.status())
    plain.close()
    closed.close()
    net.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, nargs="+", default=[64, 128])
    ap.add_argument("--iters", type=int, default=20)
    a = ap.parse_args(argv)
    peak, kind = measured_peak()
    rng = np.random.default_rng(0)
    for n in a.n:
        r = run(n, a.iters, rng)
        r["peak_bf16_tflops"] = peak
        r["peak_kind"] = kind
        r["frac_forward"] = r["tflops_forward"] / peak
        r["frac_train"] = r["tflops_train"] / peak
        print(json.dumps(r))


if __name__ == "__main__":
    main()
