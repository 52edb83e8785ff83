"""Run a benchmark configuration for a few steps (used for profiling).

    python -m multiphysics_fvm_b200.run_config rt3d --n 256 --steps 2 [--precision fp32]
    python -m multiphysics_fvm_b200.run_config kh2d --n 256 --steps 200

Configurations: kh2d (2D sharp Kelvin-Helmholtz), kh3d (its 3D extrusion),
rt3d (3D Rayleigh-Taylor), maxwell_sph (spherical pulse), heat_cyl
(cylindrical hot spot), batch_c3 (96 mixed grids in one batch).  Prints the
device time per step; --autotune picks the block shape (tile rows, z-march
depth) first.
"""
from __future__ import annotations

import argparse
import math

import numpy as np

from . import backend
from .grid.geometry import build_grid


def make(name: str, n: int, precision: str | None = None):
    from .setups import kelvin_helmholtz_sharp as kh, rayleigh_taylor_3d as rt
    if name == "kh2d":
        s = kh.get_setup(n, n, 1)
    elif name == "kh3d":
        s = kh.get_setup(n, n, n, precision="fp32")
    elif name == "rt3d":
        s = rt.get_setup(n, n, n)
    elif name == "maxwell_sph":
        from .setups import maxwell_spherical_pulse as mx
        s = mx.get_setup(n // 2, n // 2, n)
    elif name == "heat_cyl":
        from .setups import heat_cylindrical_hotspot as hc
        s = hc.get_setup(3 * n // 4, n, n // 2)
    else:
        raise ValueError(f"unknown configuration {name!r}")
    if precision:
        s["precision"] = precision
    g = build_grid(s["coordinate_system"], s["grid_config"])
    U = s["physics"].allocate_u(s["grid_config"])
    s["initial_conditions"]["initializer"](U, s["physical_parameters"], g, s["initial_conditions"]["parameters"])
    return s, np.stack([U[k] for k in backend.VARIABLES[backend.physics_name(s["physics"])]])


def run_batch(steps: int, warmup: int, autotune: bool, seed: int = 0):
    """The batched configuration (setups/batch_mixed.py): 96 grids, per-grid dt."""
    from .setups import batch_mixed
    setups = batch_mixed.make_setups(seed=seed)
    states = batch_mixed.initial_states(setups)
    b = backend.Batch(setups)
    for i, U in enumerate(states):
        b[i].upload(U)
        b[i].set_time(0.0, math.inf, float(setups[i]["time_config"]["CFL"]))
    cells = sum(int(np.prod([s["grid_config"][k] for k in ("nx1", "nx2", "nx3")])) for s in setups)
    tuned = b.autotune() if autotune else None
    b.step(warmup)
    ms = b.time_steps(steps)
    st = max(b[i].status() for i in range(len(b)))
    print(f"batch_c3 grids={len(b)} cells={cells} tiles={b.tiles()} launches/stage={b.launches_per_stage()} autotune={tuned}: {ms / steps:.3f} ms/step, "
          f"{cells * steps / (ms / 1e3):.4e} cell-updates/s, status={st}")
    return cells * steps / (ms / 1e3)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("config")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--precision", default=None)
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--tile-rows", type=int, default=0, help="block shape (tile rows); 0: the default")
    ap.add_argument("--zchunk", type=int, default=0, help="z-march depth (planes per tile); 0: the default")
    ap.add_argument("--breakdown", action="store_true",
                    help="also time each launch of a few un-captured steps: stage kernels vs the rest")
    a = ap.parse_args()
    if a.config == "batch_c3":
        run_batch(a.steps, a.warmup, a.autotune)
        return
    s, U = make(a.config, a.n, a.precision)
    sim = backend.Simulation.from_setup(s, tile_ty=a.tile_rows, zchunk=a.zchunk)
    sim.upload(U)
    sim.set_time(0.0, math.inf, float(s["time_config"]["CFL"]))
    tuned = sim.autotune() if a.autotune else None
    sim.step(a.warmup)
    ms = sim.time_steps(a.steps)
    if tuned:
        print(f"autotuned tile rows {sim.tiling()[0]}, z-march depth {tuned[0]} ({tuned[1]:.3f} ms/step in the sweep)")
    print(f"{a.config} n={a.n} {s.get('precision')}: {ms / a.steps:.3f} ms/step, status={sim.status()}")
    if a.breakdown:
        n = max(3, min(a.steps, 10))
        st, ot, nl = sim.profile_steps(n)
        print(f"  per step: stage kernels {st / n:.3f} ms ({nl // n} launches), other kernels {ot / n:.3f} ms")


if __name__ == "__main__":
    main()
