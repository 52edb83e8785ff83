"""Batched configuration: many independent seeded setups advanced together.

64 two-dimensional Kelvin-Helmholtz grids (the sharp-interface profile of
kelvin_helmholtz_sharp) with nx1, nx2 each drawn log-uniformly in [64, 512] and a
seeded phase of the x2-velocity perturbation, plus 32 cylindrical heat grids
(heat_cylindrical_hotspot) with dimensions drawn uniformly between 32x64x32 and
128x256x64 and seeded hot-spot positions.  float32, SSPRK3, each grid with its
own CFL time step, 100 steps.  ``scale`` < 1 shrinks every grid (tests).
"""
from __future__ import annotations

import math

import numpy as np

from . import heat_cylindrical_hotspot as hc
from . import kelvin_helmholtz_sharp as kh


def make_setups(seed: int = 0, n_kh: int = 64, n_heat: int = 32, scale: float = 1.0, n_steps: int = 100):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_kh):
        nx, ny = (int(round(math.exp(rng.uniform(math.log(64), math.log(512))) * scale)) for _ in range(2))
        out.append(kh.get_setup(max(nx, 4), max(ny, 4), 1, seed=seed * 1000 + i, n_steps=n_steps,
                                precision="fp32", phase=float(rng.uniform(0, 2 * math.pi))))
    for i in range(n_heat):
        nr = max(int(rng.integers(32, 129) * scale), 4)
        nth = max(int(rng.integers(64, 257) * scale), 4)
        nz = max(int(rng.integers(32, 65) * scale), 4)
        centre = (float(rng.uniform(0.3, 0.8)), float(rng.uniform(0, 2 * math.pi)), float(rng.uniform(0.3, 0.7)))
        out.append(hc.get_setup(nr, nth, nz, n_steps=n_steps, precision="fp32", centre=centre))
    return out


def initial_states(setups):
    from ..backend import VARIABLES, physics_name
    from ..grid.geometry import build_grid
    states = []
    for s in setups:
        g = build_grid(s["coordinate_system"], s["grid_config"])
        U = s["physics"].allocate_u(s["grid_config"])
        s["initial_conditions"]["initializer"](U, s["physical_parameters"], g, s["initial_conditions"]["parameters"])
        states.append(np.stack([U[k] for k in VARIABLES[physics_name(s["physics"])]]))
    return states
