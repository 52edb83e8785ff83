"""3D Rayleigh-Taylor on [0,0.5] x [0,0.5] x [0,1.5].

rho = 2 above x3 = 0.75 and 1 below; gravity (0, 0, -0.1); hydrostatic
pressure from the discrete trapezoid recurrence of the reference's
setups/rayleigh_taylor.py:84-89 (taken along x3), shifted so that the pressure
at the interface face x3 = 0.75 is 2.5; v3 = 0.01 (1+cos 4 pi x1)(1+cos 4 pi x2)
(1+cos 3 pi x3)/8 plus seeded uniform noise 1e-4.  Navier-Stokes with
mu = 1e-4, gamma 1.4; periodic in x1, x2; in x3 reflecting for momentum_x3 and
Neumann otherwise (the pattern of setups/rayleigh_taylor.py:143-147).  MUSCL
van Leer + HLL + rk3 (as written in the reference), float32, CFL 0.4.
"""
from __future__ import annotations

import numpy as np

from ..grid import boundary_conditions as bc
from ..numerics import diffusive_solvers, reconstructors, riemann_solvers, slope_limiters, time_integrators
from ..physics import navier_stokes


def initializer(U, params, grid, p):
    xc = grid["axes"]["centres"]
    x, y, z = xc[0], xc[1], xc[2]
    gamma = params["heat_capacity_ratio"]
    g = abs(params["gravitational_acceleration"][2])
    zi = p["interface"]
    rho_z = np.where(z > zi, p["rho_top"], p["rho_bottom"])
    P = np.zeros_like(z)
    for k in range(1, len(z)):
        P[k] = P[k - 1] - 0.5 * (rho_z[k] + rho_z[k - 1]) * g * (z[k] - z[k - 1])
    ka = int(np.searchsorted(z, zi))  # first cell above the interface
    if 0 < ka < len(z):
        P = P + (p["pressure_interface"] - 0.5 * (P[ka - 1] + P[ka]))
    else:
        P = P + p["pressure_interface"]
    rng = np.random.default_rng(p["seed"])
    shape = (len(x), len(y), len(z))
    v3 = (p["amplitude"] * (1 + np.cos(4 * np.pi * x))[:, None, None] * (1 + np.cos(4 * np.pi * y))[None, :, None]
          * (1 + np.cos(3 * np.pi * z))[None, None, :] / 8.0)
    v3 = v3 + rng.uniform(-p["noise"], p["noise"], shape)
    rho = np.broadcast_to(rho_z[None, None, :], shape)
    I = (slice(1, -1),) * 3
    U["mass_density"][I] = rho
    U["momentum_x1"][I] = 0.0
    U["momentum_x2"][I] = 0.0
    U["momentum_x3"][I] = rho * v3
    U["energy_density"][I] = P[None, None, :] / (gamma - 1.0) + 0.5 * rho * v3 ** 2


def get_setup(nx: int = 256, ny: int = 256, nz: int = 256, seed: int = 0, n_steps: int = 100,
              precision: str = "fp32") -> dict:
    params = {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 1e-4,
              "gravitational_acceleration": [0.0, 0.0, -0.1]}
    bcs = {}
    for v in navier_stokes.VARIABLES:
        zb = bc.reflecting if v == "momentum_x3" else bc.neumann
        bcs[v] = {"left": bc.periodic, "right": bc.periodic, "bottom": bc.periodic, "top": bc.periodic,
                  "front": zb, "back": zb}
    return {
        "physics": navier_stokes,
        "physical_parameters": params,
        "coordinate_system": "cartesian",
        "grid_config": {"x1_min": 0.0, "x1_max": 0.5, "nx1": nx, "x2_min": 0.0, "x2_max": 0.5, "nx2": ny,
                        "x3_min": 0.0, "x3_max": 1.5, "nx3": nz},
        "time_config": {"t_start": 0.0, "t_end": 1e30, "CFL": 0.4, "n_steps": n_steps},
        "time_integrator": time_integrators.rk3,
        "space_schemes": {"riemann_solver": riemann_solvers.hll, "reconstructor": reconstructors.muscl,
                          "slope_limiter": slope_limiters.van_leer, "diffusive_solver": diffusive_solvers.centered},
        "boundary_conditions": bcs,
        "initial_conditions": {"initializer": initializer,
                               "parameters": {"rho_top": 2.0, "rho_bottom": 1.0, "interface": 0.75,
                                              "pressure_interface": 2.5, "amplitude": 0.01, "noise": 1e-4,
                                              "seed": seed}},
        "save_config": {"saver": None, "output_frequency": 0, "directory": "./outputs/rayleigh_taylor_3d"},
        "precision": precision,
    }
