"""Gaussian hot spot in a cylindrical annulus.

Heat on r in [0.1, 1], theta in [0, 2 pi) (periodic), z in [0, 1] with
rho = cp = k = 1 (kappa = 1) and q = 0.  T = 1 + 10 exp(-|x - x0|^2 / (2 0.1^2))
in physical distance, hot spot at (r, theta, z) = (0.55, 0, 0.5).  Dirichlet
T = 1 on the r and z walls (ghost = 2 rho cp T_wall - interior).  Centred
diffusion with piecewise-constant face states + SSPRK3, CFL 0.4.
"""
from __future__ import annotations

import numpy as np

from ..grid import boundary_conditions as bc
from ..numerics import diffusive_solvers, reconstructors, slope_limiters, time_integrators
from ..physics import heat


def initializer(U, params, grid, p):
    r = grid["cell"]["coordinates"]["x1"]
    th = grid["cell"]["coordinates"]["x2"]
    z = grid["cell"]["coordinates"]["x3"]
    c = p["centre"]
    d2 = (r * np.cos(th) - c[0] * np.cos(c[1])) ** 2 + (r * np.sin(th) - c[0] * np.sin(c[1])) ** 2 + (z - c[2]) ** 2
    T = p["background"] + p["amplitude"] * np.exp(-d2 / (2.0 * p["width"] ** 2))
    U["internal_energy_density"][(slice(1, -1),) * 3] = params["mass_density"] * params["specific_heat_capacity"] * T


def get_setup(nr: int = 192, nth: int = 256, nz: int = 128, n_steps: int = 500, precision: str = "fp32",
              centre=(0.55, 0.0, 0.5)) -> dict:
    params = {"mass_density": 1.0, "specific_heat_capacity": 1.0, "thermal_conductivity": 1.0,
              "volumetric_heat_source": 0.0}
    wall = bc.dirichlet(params["mass_density"] * params["specific_heat_capacity"] * 1.0)
    bcs = {"internal_energy_density": {"left": wall, "right": wall, "bottom": bc.periodic, "top": bc.periodic,
                                       "front": wall, "back": wall}}
    return {
        "physics": heat,
        "physical_parameters": params,
        "coordinate_system": "cylindrical",
        "grid_config": {"x1_min": 0.1, "x1_max": 1.0, "nx1": nr, "x2_min": 0.0, "x2_max": 2 * np.pi, "nx2": nth,
                        "x3_min": 0.0, "x3_max": 1.0, "nx3": nz},
        "time_config": {"t_start": 0.0, "t_end": 1e30, "CFL": 0.4, "n_steps": n_steps},
        "time_integrator": time_integrators.rk3_ssp,
        "space_schemes": {"reconstructor": reconstructors.piecewise_constant, "slope_limiter": slope_limiters.minmod,
                          "diffusive_solver": diffusive_solvers.centered},
        "boundary_conditions": bcs,
        "initial_conditions": {"initializer": initializer,
                               "parameters": {"background": 1.0, "amplitude": 10.0, "width": 0.1,
                                              "centre": centre}},
        "save_config": {"saver": None, "output_frequency": 0, "directory": "./outputs/heat_cylindrical_hotspot"},
        "precision": precision,
    }
