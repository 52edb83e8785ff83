"""The benchmark configurations at their full sizes and step counts, where the
NumPy oracle would take hours: the float32 build against the float64 build of
the same kernels, which the other tests pin to the oracle to 1e-12 at reduced
sizes.  Tolerance: relative L2 of the final interior state <= 1e-4 (the
100-step bound), and the same simulated time to 1e-5.

* C1  3D Rayleigh-Taylor 256^3, viscous, MUSCL van Leer + HLL + rk3, 100 steps;
* C2a Maxwell, spherical 128x128x256, MUSCL MC + Rusanov + RK4, 200 steps;
* C2b heat, cylindrical 192x256x128, piecewise constant + SSPRK3, 500 steps.
"""
import math

import numpy as np
import pytest

from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

I3 = (slice(None),) + (slice(1, -1),) * 3


def _config(name):
    from multiphysics_fvm_b200 import run_config
    if name == "C1":
        return run_config.make("rt3d", 256)
    if name == "C2a":
        return run_config.make("maxwell_sph", 256)
    return run_config.make("heat_cyl", 256)


@pytest.mark.parametrize("name", ["C1", "C2a", "C2b"])
def test_full_size_fp32_matches_fp64_build(name):
    from multiphysics_fvm_b200.backend import Simulation
    s, U0 = _config(name)
    n_steps = int(s["time_config"]["n_steps"])
    out, times = {}, {}
    for precision in ("fp64", "fp32"):
        sim = Simulation.from_setup(dict(s, precision=precision))
        sim.upload(U0)
        sim.set_time(0.0, math.inf, float(s["time_config"]["CFL"]))
        sim.step(n_steps)
        assert sim.status() == 0, precision
        t, steps, _ = sim.time()
        assert steps == n_steps
        times[precision] = t
        out[precision] = sim.download()[I3]
        sim.close()
    assert abs(times["fp32"] - times["fp64"]) <= 1e-5 * times["fp64"]
    err = rel_l2(out["fp32"], out["fp64"])
    print(f"{name}: float32 vs float64 relative L2 {err:.2e}, t {times['fp64']:.6g}")
    assert err <= 1e-4, err
    assert np.all(np.isfinite(out["fp32"]))
