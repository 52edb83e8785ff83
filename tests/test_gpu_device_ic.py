"""Device-written initial state (fvm_init_kelvin_helmholtz) against the host
initializer of setups/kelvin_helmholtz_sharp: identical without noise; with
noise, every perturbation lies in [-noise, noise), has the uniform
distribution's moments, and repeats exactly for the same seed."""
import numpy as np
import pytest

from multiphysics_fvm_b200.grid.geometry import build_grid

pytestmark = pytest.mark.gpu


def _sim_and_host(n, noise, seed=3, precision="fp32"):
    from multiphysics_fvm_b200.backend import Simulation
    from multiphysics_fvm_b200.setups import kelvin_helmholtz_sharp as kh
    s = kh.get_setup(*n, seed=seed, precision=precision, noise_all=True)
    s["initial_conditions"]["parameters"]["noise"] = noise
    s["initial_conditions"]["parameters"]["phase"] = 0.7
    g = build_grid(s["coordinate_system"], s["grid_config"])
    U = s["physics"].allocate_u(s["grid_config"])
    s["initial_conditions"]["initializer"](U, s["physical_parameters"], g, s["initial_conditions"]["parameters"])
    host = np.stack([U[k] for k in ("mass_density", "momentum_x1", "momentum_x2", "momentum_x3", "energy_density")])
    sim = Simulation.from_setup(s)
    sim.init_kelvin_helmholtz(s["initial_conditions"]["parameters"], seed)
    return sim, host[:, 1:-1, 1:-1, 1:-1], s


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_device_state_equals_host_initializer_without_noise(precision):
    sim, host, _ = _sim_and_host((32, 48, 8), 0.0, precision=precision)
    dev = sim.download()[:, 1:-1, 1:-1, 1:-1]
    ref = host.astype(np.float32).astype(np.float64) if precision == "fp32" else host
    assert np.max(np.abs(dev - ref)) <= (2e-7 if precision == "fp32" else 1e-14) * np.max(np.abs(ref))


def test_device_noise_is_bounded_uniform_and_reproducible():
    n, noise = (64, 64, 32), 1e-3
    sim, host0, s = _sim_and_host(n, 0.0)  # clean reference profile (host)
    sim2, _, _ = _sim_and_host(n, noise)
    dev = sim2.download()[:, 1:-1, 1:-1, 1:-1]
    rho = dev[0]
    dv = [dev[c] / rho - host0[c] / host0[0] for c in (1, 2, 3)]
    for d in dv:
        assert np.all(np.abs(d) <= noise * (1 + 1e-4))
        assert abs(np.mean(d)) < 0.02 * noise
        assert abs(np.std(d) - noise / np.sqrt(3)) < 0.02 * noise
    sim3, _, _ = _sim_and_host(n, noise)
    assert np.array_equal(sim3.download(), sim2.download())
    sim4, _, _ = _sim_and_host(n, noise, seed=4)
    assert not np.array_equal(sim4.download(), sim2.download())
