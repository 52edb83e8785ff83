"""Analytic known answers on the device, independent of the reference:

* free-stream preservation: a uniform state on a periodic cartesian grid has a
  zero residual (Navier-Stokes with viscosity and MUSCL, heat, Maxwell), in
  float32 and float64;
* Runge-Kutta orders on du/dt = lambda*u: a uniform Maxwell state with
  conductivity sigma only feels the Ohmic source, so each integrator's error
  at t = 1 must shrink by 2^p when dt halves (euler_explicit p = 1, rk3 as
  written in the reference p = 2, rk3_ssp p = 3, rk4 p = 4);
* Maxwell's HLL flux equals Rusanov's (symmetric wave speeds +-c).
"""
import math

import numpy as np
import pytest

from oracle import fvm_oracle as O
from tests.helpers import bcs_dict

pytestmark = pytest.mark.gpu

GRID = dict(x1_min=0.0, x1_max=1.0, x2_min=0.0, x2_max=0.75, x3_min=0.0, x3_max=0.5, nx1=16, nx2=12, nx3=8)
SH = (18, 14, 10)


def _schemes(lim="van_leer", riem="hll"):
    from multiphysics_fvm_b200.numerics import diffusive_solvers, reconstructors, riemann_solvers, slope_limiters
    return {"reconstructor": reconstructors.muscl, "slope_limiter": getattr(slope_limiters, lim),
            "riemann_solver": getattr(riemann_solvers, riem), "diffusive_solver": diffusive_solvers.centered}


def _sim(physics, prm, precision, integrator=None, **kw):
    from multiphysics_fvm_b200.backend import Simulation, VARIABLES
    from multiphysics_fvm_b200.numerics import time_integrators as ti
    nv = len(VARIABLES[physics])
    return Simulation(physics, "cartesian", GRID, prm, _schemes(**kw), bcs_dict(physics, [["periodic"] * 6] * nv),
                      getattr(ti, integrator) if integrator else None, precision=precision)


MAXWELL = {"magnetic_permeability": 1.0, "electric_permittivity": 1.0, "electrical_conductivity": 0.0,
           "charge_density": 0.0, "magnetic_cleaning_coeff": 0.001, "electric_cleaning_coeff": 0.001}


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("physics", ["navier_stokes", "heat", "maxwell"])
def test_free_stream_preservation(physics, precision):
    if physics == "navier_stokes":
        prm = {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 1e-3, "gravitational_acceleration": [0.0, 0.0, 0.0]}
        rho, v, p = 1.3, (0.2, -0.1, 0.3), 2.0
        U = np.stack([np.full(SH, x) for x in (rho, rho * v[0], rho * v[1], rho * v[2],
                                                 p / 0.4 + 0.5 * rho * sum(c * c for c in v))])
    elif physics == "heat":
        prm = {"mass_density": 1.0, "specific_heat_capacity": 1.0, "thermal_conductivity": 1.0,
               "volumetric_heat_source": 0.0}
        U = np.full((1,) + SH, 3.7)
    else:
        prm = MAXWELL
        U = np.stack([np.full(SH, x) for x in (0.3, -0.2, 0.1, 0.5, 0.25, -0.4)])
    sim = _sim(physics, prm, precision)
    sim.upload(U)
    r = sim.residual()
    tol = 1e-6 if precision == "fp32" else 1e-14
    assert np.max(np.abs(r)) <= tol * np.max(np.abs(U)), np.max(np.abs(r))


@pytest.mark.parametrize("integrator,order", [("euler_explicit", 1), ("rk3", 2), ("rk3_ssp", 3), ("rk4", 4)])
def test_runge_kutta_orders(integrator, order):
    prm = dict(MAXWELL, electrical_conductivity=1.0)
    U0 = np.stack([np.full(SH, x) for x in (0.3, -0.2, 0.1, 0.5, 0.25, -0.4)])
    rhs = O.maxwell_rhs(U0.copy(), O.Geometry("cartesian", GRID), prm,
                        dict(reconstructor="muscl", slope_limiter="van_leer", riemann_solver="hll"))
    lam = float(rhs[3, 0, 0, 0] / U0[3, 0, 0, 0])  # du/dt = lam * u for the D components
    assert lam != 0 and np.allclose(rhs[3:], lam * U0[3:, 1:-1, 1:-1, 1:-1])
    errs = []
    for n in (16, 32):
        sim = _sim("maxwell", prm, "fp64", integrator)
        sim.upload(U0)
        sim.set_time(0.0, math.inf, 0.4)
        sim.step(n, dt=1.0 / n)
        D = sim.download()[3:, 1:-1, 1:-1, 1:-1]
        errs.append(float(np.max(np.abs(D - U0[3:, 1:-1, 1:-1, 1:-1] * math.exp(lam)))))
        sim.close()
    p = math.log2(errs[0] / errs[1])
    assert abs(p - order) < 0.25, (integrator, errs, p)


def test_maxwell_hll_equals_rusanov():
    rng = np.random.default_rng(5)
    U = rng.uniform(-1.0, 1.0, (6,) + SH)
    res = []
    for riem in ("hll", "rusanov"):
        sim = _sim("maxwell", MAXWELL, "fp64", lim="monotonized_central", riem=riem)
        sim.upload(U)
        res.append(sim.residual())
    assert np.max(np.abs(res[0] - res[1])) <= 1e-13 * np.max(np.abs(res[1]))
