"""Kelvin-Helmholtz with sharp shear interfaces (the reference's
setups/kelvin_helmholtz.py uses tanh layers; this profile is a step).

rho = 2, v1 = +0.5 where |x2 - 0.5| < 0.25, else rho = 1, v1 = -0.5; P = 2.5;
v2 = 0.01 sin(4 pi x1) + seeded uniform noise of amplitude 1e-3; v3 = 0.
Navier-Stokes, viscosity 0, gamma 1.4, periodic on every side, MUSCL minmod +
HLL + SSPRK3, CFL 0.4.  ``nz > 1`` extrudes the profile along x3 over [0, 1]
and (``noise_all=True``) puts the noise on all three velocity components.
"""
from __future__ import annotations

import numpy as np

from ..grid import boundary_conditions as bc
from ..numerics import diffusive_solvers, reconstructors, riemann_solvers, slope_limiters, time_integrators
from ..physics import navier_stokes


def initializer(U, params, grid, p):
    x = grid["cell"]["coordinates"]["x1"]
    y = grid["cell"]["coordinates"]["x2"]
    gamma = params["heat_capacity_ratio"]
    rng = np.random.default_rng(p["seed"])
    inner = np.abs(y - 0.5) < 0.25
    rho = np.where(inner, p["rho_inner"], p["rho_outer"])
    v1 = np.where(inner, p["shear_velocity"], -p["shear_velocity"])
    phase = p.get("phase", 0.0)
    v2 = p["amplitude"] * np.sin(2.0 * np.pi * p["wavenumber"] * x + phase)
    v2 = v2 + rng.uniform(-p["noise"], p["noise"], x.shape)
    v3 = np.zeros_like(x)
    if p.get("noise_all", False):
        v1 = v1 + rng.uniform(-p["noise"], p["noise"], x.shape)
        v3 = v3 + rng.uniform(-p["noise"], p["noise"], x.shape)
    I = (slice(1, -1),) * 3
    U["mass_density"][I] = rho
    U["momentum_x1"][I] = rho * v1
    U["momentum_x2"][I] = rho * v2
    U["momentum_x3"][I] = rho * v3
    U["energy_density"][I] = p["pressure"] / (gamma - 1.0) + 0.5 * rho * (v1 ** 2 + v2 ** 2 + v3 ** 2)


def get_setup(nx: int = 256, ny: int = 256, nz: int = 1, seed: int = 0, n_steps: int = 200,
              precision: str = "fp64", noise_all: bool | None = None, phase: float = 0.0) -> dict:
    if noise_all is None:
        noise_all = nz > 1
    params = {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 0.0, "gravitational_acceleration": [0.0, 0.0, 0.0]}
    names = navier_stokes.VARIABLES
    bcs = {v: {s: bc.periodic for s in ("left", "right", "bottom", "top", "front", "back")} for v in names}
    return {
        "physics": navier_stokes,
        "physical_parameters": params,
        "coordinate_system": "cartesian",
        "grid_config": {"x1_min": 0.0, "x1_max": 1.0, "nx1": nx, "x2_min": 0.0, "x2_max": 1.0, "nx2": ny,
                        "x3_min": 0.0, "x3_max": 1.0, "nx3": nz},
        "time_config": {"t_start": 0.0, "t_end": 5.0, "CFL": 0.4, "n_steps": n_steps},
        "time_integrator": time_integrators.rk3_ssp,
        "space_schemes": {"riemann_solver": riemann_solvers.hll, "reconstructor": reconstructors.muscl,
                          "slope_limiter": slope_limiters.minmod, "diffusive_solver": diffusive_solvers.centered},
        "boundary_conditions": bcs,
        "initial_conditions": {"initializer": initializer,
                               "parameters": {"rho_inner": 2.0, "rho_outer": 1.0, "shear_velocity": 0.5,
                                              "pressure": 2.5, "amplitude": 0.01, "wavenumber": 2,
                                              "noise": 1e-3, "seed": seed, "noise_all": noise_all,
                                              "phase": phase}},
        "save_config": {"saver": None, "output_frequency": 0, "directory": "./outputs/kelvin_helmholtz_sharp"},
        "precision": precision,
    }
