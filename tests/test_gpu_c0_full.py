"""Configuration C0 at its full size: 2D sharp Kelvin-Helmholtz, 256 x 256 x 1,
periodic, MUSCL minmod + HLL + SSPRK3, CFL 0.4, 200 steps with the device CFL
time step, against the float64 oracle run of the same 200 steps (the oracle
leg takes about a minute of CPU).

float64 build: relative L2 of the final state <= 1e-10 and the same simulated
time to 1e-12; float32 build: relative L2 <= 1e-4 (the 100-step tolerance,
here over 200 steps).
"""
import math

import numpy as np
import pytest

from oracle import fvm_oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

N_STEPS = 200


@pytest.fixture(scope="module")
def c0():
    from multiphysics_fvm_b200.grid.geometry import build_grid
    from multiphysics_fvm_b200.setups import kelvin_helmholtz_sharp as kh
    s = kh.get_setup(256, 256, 1, seed=0, n_steps=N_STEPS, precision="fp64")
    g = build_grid(s["coordinate_system"], s["grid_config"])
    U = s["physics"].allocate_u(s["grid_config"])
    s["initial_conditions"]["initializer"](U, s["physical_parameters"], g, s["initial_conditions"]["parameters"])
    U0 = np.stack([U[k] for k in ("mass_density", "momentum_x1", "momentum_x2", "momentum_x3", "energy_density")])
    Uo = U0.copy()
    bcs = [{sd: ("periodic", 0.0) for sd in O.SIDES} for _ in range(5)]
    dts = O.run("navier_stokes", Uo, s["physical_parameters"], O.Geometry("cartesian", s["grid_config"]),
                dict(reconstructor="muscl", slope_limiter="minmod", riemann_solver="hll"), bcs, "rk3_ssp", 0.4,
                N_STEPS)
    return s, U0, Uo, float(sum(dts))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-4)])
def test_c0_full_size_matches_oracle(c0, precision, tol):
    from multiphysics_fvm_b200.backend import Simulation
    s, U0, Uo, t_ref = c0
    s = dict(s, precision=precision)
    sim = Simulation.from_setup(s)
    sim.upload(U0)
    sim.set_time(0.0, math.inf, 0.4)
    sim.step(N_STEPS)
    assert sim.status() == 0
    t, steps, _ = sim.time()
    assert steps == N_STEPS
    assert abs(t - t_ref) <= (1e-12 if precision == "fp64" else 1e-5) * t_ref
    I = (slice(None),) + (slice(1, -1),) * 3
    err = rel_l2(sim.download()[I], Uo[I])
    assert err <= tol, err
