"""Electromagnetic pulse in a spherical shell.

Maxwell on r in [0.1, 1], theta in [0.05 pi, 0.95 pi], phi in [0, 2 pi) with
mu = eps = 1 (c = 1), sigma = 0, rho_c = 0 and divergence-cleaning
coefficients 0.001 (the reference's electromagnetic_pulse.py:88-93 values).
Initial field: a Gaussian pulse of the cartesian z component of E, amplitude 1,
width 0.05 in physical distance, centred at (r, theta, phi) = (0.5, pi/2, 0),
projected on the spherical basis (E_r = E_z cos theta, E_theta = -E_z sin theta);
B = 0.  Perfect-conductor walls at r = 0.1, 1 and at both theta limits
(tangential D and normal B odd, the rest even); periodic in phi.
MUSCL monotonized-central + Rusanov + RK4, CFL 0.4.
"""
from __future__ import annotations

import numpy as np

from ..grid import boundary_conditions as bc
from ..numerics import reconstructors, riemann_solvers, slope_limiters, time_integrators
from ..physics import maxwell


def initializer(U, params, grid, p):
    r = grid["cell"]["coordinates"]["x1"]
    th = grid["cell"]["coordinates"]["x2"]
    ph = grid["cell"]["coordinates"]["x3"]
    x = r * np.sin(th) * np.cos(ph)
    y = r * np.sin(th) * np.sin(ph)
    z = r * np.cos(th)
    c = p["centre"]
    cx, cy, cz = (c[0] * np.sin(c[1]) * np.cos(c[2]), c[0] * np.sin(c[1]) * np.sin(c[2]), c[0] * np.cos(c[1]))
    Ez = p["amplitude"] * np.exp(-((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) / (2.0 * p["width"] ** 2))
    ep = params["electric_permittivity"]
    I = (slice(1, -1),) * 3
    for k in ("magnetic_field_x1", "magnetic_field_x2", "magnetic_field_x3", "electric_d_field_x3"):
        U[k][I] = 0.0
    U["electric_d_field_x1"][I] = ep * Ez * np.cos(th)
    U["electric_d_field_x2"][I] = -ep * Ez * np.sin(th)


def get_setup(nr: int = 128, nth: int = 128, nph: int = 256, n_steps: int = 200, precision: str = "fp32") -> dict:
    params = {"magnetic_permeability": 1.0, "electric_permittivity": 1.0, "electrical_conductivity": 0.0,
              "charge_density": 0.0, "magnetic_cleaning_coeff": 0.001, "electric_cleaning_coeff": 0.001}
    wall_r = bc.conducting_wall(maxwell.VARIABLES, 0)
    wall_t = bc.conducting_wall(maxwell.VARIABLES, 1)
    bcs = {v: {"left": wall_r[v], "right": wall_r[v], "bottom": wall_t[v], "top": wall_t[v],
               "front": bc.periodic, "back": bc.periodic} for v in maxwell.VARIABLES}
    return {
        "physics": maxwell,
        "physical_parameters": params,
        "coordinate_system": "spherical",
        "grid_config": {"x1_min": 0.1, "x1_max": 1.0, "nx1": nr, "x2_min": 0.05 * np.pi, "x2_max": 0.95 * np.pi,
                        "nx2": nth, "x3_min": 0.0, "x3_max": 2 * np.pi, "nx3": nph},
        "time_config": {"t_start": 0.0, "t_end": 1e30, "CFL": 0.4, "n_steps": n_steps},
        "time_integrator": time_integrators.rk4,
        "space_schemes": {"riemann_solver": riemann_solvers.rusanov, "reconstructor": reconstructors.muscl,
                          "slope_limiter": slope_limiters.monotonized_central},
        "boundary_conditions": bcs,
        "initial_conditions": {"initializer": initializer,
                               "parameters": {"amplitude": 1.0, "width": 0.05, "centre": (0.5, np.pi / 2, 0.0)}},
        "save_config": {"saver": None, "output_frequency": 0, "directory": "./outputs/maxwell_spherical_pulse"},
        "precision": precision,
    }
