"""Pipelined transfers (fvm_upload_async / fvm_step_async / fvm_download_async)
give bitwise the same states as the synchronous calls, including the ghost
edges and corners averaged on the device (src/solver.py:39-61), over a sequence
of uploads, steps and downloads in flight together."""
import math

import numpy as np
import pytest

from tests.helpers import bcs_dict, random_ns_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_async_pipeline_matches_sync_calls(precision):
    import torch
    from multiphysics_fvm_b200.backend import Simulation
    from multiphysics_fvm_b200.numerics import reconstructors, riemann_solvers, slope_limiters, time_integrators
    n = (40, 33, 21)
    cfg = dict(x1_min=0, x1_max=1, x2_min=0, x2_max=0.8, x3_min=0, x3_max=0.5, nx1=n[0], nx2=n[1], nx3=n[2])
    prm = {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 0.0, "gravitational_acceleration": [0, -0.1, 0]}
    sch = {"reconstructor": reconstructors.muscl, "slope_limiter": slope_limiters.minmod,
           "riemann_solver": riemann_solvers.hll}
    kinds = [["periodic"] * 2 + ["neumann", "neumann", ("dirichlet", 1.5) if q == 0 else "neumann", "neumann"]
             for q in range(5)]

    def make():
        s = Simulation("navier_stokes", "cartesian", cfg, prm, sch, bcs_dict("navier_stokes", kinds),
                       time_integrators.rk3_ssp, precision=precision)
        s.set_time(0.0, math.inf, 0.4)
        return s

    rng = np.random.default_rng(4)
    states = [random_ns_state(tuple(x + 2 for x in n), rng) for _ in range(3)]
    ref = []
    sim = make()
    for U in states:
        sim.upload(U)
        sim.step(2)
        ref.append(sim.download())
    sim.close()
    sim = make()
    pins = [torch.from_numpy(U).pin_memory().numpy() for U in states]
    outs = [torch.empty(U.shape, dtype=torch.float64).pin_memory().numpy() for U in states]
    for U, o in zip(pins, outs):
        sim.upload_async(U)
        sim.step_async(2)
        sim.download_async(o)
    sim.synchronize()
    assert sim.status() == 0
    sim.close()
    for r, o in zip(ref, outs):
        assert np.array_equal(r, o)
