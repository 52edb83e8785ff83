"""The bounded waits of the stage kernels give up and report, without a fault.

Every wait of a stage kernel for a TMA plane (or a staged U0 / accumulator
tile) is bounded by the handle's wait limit (fvm_set_wait_limit, default 2 s).
Here every ring copy is made to expect 16 bytes more than it delivers, so no
ring wait can complete (a wait on something that never happens), and the limit
is 1 ms: the kernel must set FVM_ST_TIMEOUT, wait (bounded) for its own copies
in flight and return.  The same handle, with the default
limit restored and the state uploaded again, then runs clean steps whose result
is bitwise equal to a fresh handle's, so the context stayed usable.  No wait is
left without a limit and nothing traps.
"""
import math

import numpy as np
import pytest

from tests.helpers import bcs_dict, random_ns_state

pytestmark = pytest.mark.gpu

CASES = [
    # (physics, precision, viscosity, reconstructor): the register-blocked
    # float32 kernels (inviscid and viscous NS, piecewise-constant heat,
    # Maxwell) and the general ones (float64 NS, MUSCL heat)
    ("navier_stokes", "fp32", 0.0, "muscl"),
    ("navier_stokes", "fp32", 1e-3, "muscl"),
    ("navier_stokes", "fp64", 0.0, "muscl"),
    ("heat", "fp32", None, "muscl"),
    ("heat", "fp32", None, "piecewise_constant"),
    ("maxwell", "fp32", None, "muscl"),
]


def _make(physics, precision, mu, recon):
    from multiphysics_fvm_b200.backend import Simulation
    from multiphysics_fvm_b200.numerics import (diffusive_solvers, reconstructors, riemann_solvers,
                                                slope_limiters, time_integrators)
    n = (48, 40, 36)
    cfg = dict(x1_min=0, x1_max=1, x2_min=0, x2_max=0.8, x3_min=0, x3_max=0.7, nx1=n[0], nx2=n[1], nx3=n[2])
    sch = {"reconstructor": getattr(reconstructors, recon), "slope_limiter": slope_limiters.minmod,
           "riemann_solver": riemann_solvers.hll, "diffusive_solver": diffusive_solvers.centered}
    rng = np.random.default_rng(12)
    sh = tuple(x + 2 for x in n)
    if physics == "navier_stokes":
        prm = {"heat_capacity_ratio": 1.4, "dynamic_viscosity": mu, "gravitational_acceleration": [0, 0, 0]}
        U = random_ns_state(sh, rng)
        nv = 5
    elif physics == "heat":
        prm = {"mass_density": 1.0, "specific_heat_capacity": 1.0, "thermal_conductivity": 0.5,
               "volumetric_heat_source": 0.0}
        U = rng.uniform(1.0, 2.0, (1,) + sh)
        nv = 1
    else:
        prm = {"magnetic_permeability": 1.0, "electric_permittivity": 1.0, "electrical_conductivity": 0.0,
               "charge_density": 0.0, "magnetic_cleaning_coeff": 0.001, "electric_cleaning_coeff": 0.001}
        U = rng.uniform(-1.0, 1.0, (6,) + sh)
        nv = 6
    make = lambda: Simulation(physics, "cartesian", cfg, prm, sch,  # noqa: E731
                              bcs_dict(physics, [["periodic"] * 6] * nv), time_integrators.rk3_ssp,
                              precision=precision)
    return make, U


@pytest.mark.parametrize("physics,precision,mu,recon", CASES)
def test_short_wait_limit_reports_timeout_and_context_survives(physics, precision, mu, recon):
    from multiphysics_fvm_b200._lib import ST_TIMEOUT
    make, U = _make(physics, precision, mu, recon)
    sim = make()
    sim.upload(U)
    sim.set_time(0.0, math.inf, 0.4)
    sim.set_wait_limit(1_000_000, never_complete=True)  # the ring waits cannot complete
    sim.step(1)  # returns: no hang, no fault
    st = sim.status()
    assert st & ST_TIMEOUT, f"status {st:#x}"
    # the same handle recovers with the default limit
    sim.set_wait_limit(2_000_000_000)
    sim.clear_status()
    sim.upload(U)
    sim.set_time(0.0, math.inf, 0.4)
    sim.step(3)
    assert sim.status() == 0
    got = sim.download()
    sim.close()
    fresh = make()
    fresh.upload(U)
    fresh.set_time(0.0, math.inf, 0.4)
    fresh.step(3)
    assert fresh.status() == 0
    ref = fresh.download()
    fresh.close()
    assert np.array_equal(got, ref)
