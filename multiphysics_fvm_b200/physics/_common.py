"""Shared implementation of the physics-module surface (allocate_u, compute_rhs,
compute_dt) on top of the device backend."""
from __future__ import annotations

import numpy as np

from .. import backend
from ..numerics import reconstructors, riemann_solvers, slope_limiters

_DEFAULT_SCHEMES = {"reconstructor": reconstructors.piecewise_constant, "slope_limiter": slope_limiters.minmod,
                    "riemann_solver": riemann_solvers.hll}


def allocate_u(physics: str, grid_config: dict) -> dict:
    sg = (grid_config["nx1"] + 2, grid_config["nx2"] + 2, grid_config["nx3"] + 2)
    return {k: np.zeros(sg) for k in backend.VARIABLES[physics]}


def compute_rhs(physics: str, U: dict, grid: dict, params: dict, space_schemes: dict) -> dict:
    sim = backend.cached_simulation(physics, grid, params, space_schemes)
    sim.upload(U)
    r = sim.residual()
    return {k: r[q] for q, k in enumerate(backend.VARIABLES[physics])}


def compute_dt(physics: str, U: dict, params: dict, grid: dict, cfl: float) -> float:
    sim = backend.cached_simulation(physics, grid, params, _DEFAULT_SCHEMES)
    if physics == "navier_stokes":
        sim.upload(U)
    return sim.compute_dt(cfl)
