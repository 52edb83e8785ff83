"""Batched persistent launch (many uneven grids, one launch per kernel
specialisation and stage, per-grid CFL dt) against the same grids advanced one
at a time, and the autotuner's state restoration.  Batched grids run the
tile-list kernels and single float32 grids the register-blocked ones, whose
float32 rounding differs: the states agree to relative L2 <= 1e-5 after 6
steps and the simulated times to 1e-6."""
import numpy as np
import pytest

from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def test_batch_matches_single_grids():
    from multiphysics_fvm_b200.backend import Batch, Simulation
    from multiphysics_fvm_b200.setups import batch_mixed
    setups = batch_mixed.make_setups(seed=3, n_kh=5, n_heat=3, scale=0.15, n_steps=6)
    states = batch_mixed.initial_states(setups)
    batch = Batch(setups)
    assert batch.tiles() > 0
    for i, U in enumerate(states):
        batch[i].upload(U)
        batch[i].set_time(0.0, float("inf"), setups[i]["time_config"]["CFL"])
    batch.step(6)
    for i, (s, U) in enumerate(zip(setups, states)):
        sim = Simulation.from_setup(s)
        sim.upload(U)
        sim.set_time(0.0, float("inf"), s["time_config"]["CFL"])
        sim.step(6)
        a, b = batch[i].download(), sim.download()
        assert rel_l2(a, b) <= 1e-5, (i, rel_l2(a, b))
        assert batch[i].time()[1] == 6 and batch[i].status() == 0
        assert abs(batch[i].time()[0] - sim.time()[0]) <= 1e-6 * sim.time()[0]  # per-grid dt
        sim.close()
    dts = {batch[i].time()[2] for i in range(len(setups))}
    assert len(dts) > 1  # grids advanced with different time steps
    batch.close()


def test_autotune_restores_state():
    from multiphysics_fvm_b200.backend import Batch, Simulation
    from multiphysics_fvm_b200.setups import batch_mixed, kelvin_helmholtz_sharp as kh
    s = kh.get_setup(40, 36, 30, precision="fp32")
    U = batch_mixed.initial_states([s])[0]
    sim = Simulation.from_setup(s)
    sim.upload(U)
    sim.set_time(0.0, float("inf"), 0.4)
    before = sim.download()
    z, ms = sim.autotune()
    assert 1 <= z <= 30 and ms > 0
    assert np.array_equal(sim.download(), before)
    assert sim.time()[1] == 0
    sim.close()
    setups = batch_mixed.make_setups(seed=5, n_kh=2, n_heat=2, scale=0.15)
    states = batch_mixed.initial_states(setups)
    b = Batch(setups)
    for i, U in enumerate(states):
        b[i].upload(U)
        b[i].set_time(0.0, float("inf"), 0.4)
    z, ms = b.autotune()
    assert z >= 1 and ms > 0
    for i, U in enumerate(states):
        got = b[i].download()[:, 1:-1, 1:-1, 1:-1]
        assert np.array_equal(got, U.astype(np.float32).astype(np.float64)[:, 1:-1, 1:-1, 1:-1])
    b.close()
