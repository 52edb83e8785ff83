"""Batched persistent launch (many uneven grids, one launch per kernel
specialisation and stage, per-grid CFL dt) against the same grids advanced one
at a time, and the autotuner's state restoration.  Batched grids run the
mixed launch (the register-blocked bodies of single grids over a tile list
covering every grid) when all grids are float32 inviscid navier_stokes or
piecewise-constant heat, else the tile-list kernels, whose float32 rounding
differs from the single grids' register-blocked kernels: the states agree to
relative L2 <= 1e-5 after 6 steps and the simulated times to 1e-6."""
import numpy as np
import pytest

from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("heat_rows", [0, 10])
def test_batch_matches_single_grids(heat_rows):
    """heat_rows 0: the heat grids on 20-row tiles (4-row strips), 10: 10-row
    tiles (2-row strips)."""
    from multiphysics_fvm_b200.backend import Batch, Simulation
    from multiphysics_fvm_b200.setups import batch_mixed
    setups = batch_mixed.make_setups(seed=3, n_kh=5, n_heat=3, scale=0.15, n_steps=6)
    states = batch_mixed.initial_states(setups)
    batch = Batch(setups, heat_tile_rows=heat_rows)
    assert batch.tiles() > 0
    assert batch.launches_per_stage() == 1  # inviscid navier_stokes + heat: one mixed launch
    assert batch[len(setups) - 1].tiling()[0] == (heat_rows or 20)
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


def _advance_pair(setups, n):
    from multiphysics_fvm_b200.backend import Batch, Simulation
    from multiphysics_fvm_b200.setups import batch_mixed
    states = batch_mixed.initial_states(setups)
    batch = Batch(setups)
    for i, U in enumerate(states):
        batch[i].upload(U)
        batch[i].set_time(0.0, float("inf"), setups[i]["time_config"]["CFL"])
    batch.step(n)
    out = []
    for i, (s, U) in enumerate(zip(setups, states)):
        sim = Simulation.from_setup(s)
        sim.upload(U)
        sim.set_time(0.0, float("inf"), s["time_config"]["CFL"])
        sim.step(n)
        out.append((batch[i].download(), sim.download(), batch[i].time(), sim.time(), batch[i].status()))
        sim.close()
    k = batch.launches_per_stage()
    batch.close()
    return k, out


def test_specialised_groups_match_single_grids():
    """A batch the mixed launch does not cover (a viscous navier_stokes grid and
    a MUSCL heat grid) runs one launch per kernel specialisation."""
    from multiphysics_fvm_b200.numerics import reconstructors
    from multiphysics_fvm_b200.setups import batch_mixed
    setups = batch_mixed.make_setups(seed=4, n_kh=3, n_heat=2, scale=0.15, n_steps=5)
    setups[1]["physical_parameters"] = dict(setups[1]["physical_parameters"], dynamic_viscosity=2e-3)
    setups[4]["space_schemes"] = dict(setups[4]["space_schemes"], reconstructor=reconstructors.muscl)
    k, out = _advance_pair(setups, 5)
    assert k >= 3
    for i, (a, b, ta, tb, st) in enumerate(out):
        assert st == 0 and ta[1] == 5
        assert rel_l2(a, b) <= 1e-5, (i, rel_l2(a, b))
        assert abs(ta[0] - tb[0]) <= 1e-6 * tb[0]


def test_mixed_launch_one_kind():
    """Mixed launches of navier_stokes grids only and of heat grids only."""
    from multiphysics_fvm_b200.setups import batch_mixed
    for n_kh, n_heat in ((4, 0), (0, 3)):
        setups = batch_mixed.make_setups(seed=6, n_kh=n_kh, n_heat=n_heat, scale=0.2, n_steps=4)
        k, out = _advance_pair(setups, 4)
        assert k == 1
        for i, (a, b, ta, tb, st) in enumerate(out):
            assert st == 0 and ta[1] == 4
            assert rel_l2(a, b) <= 1e-5, (n_kh, n_heat, i, rel_l2(a, b))


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
    assert b[len(setups) - 1].tiling()[0] in (20, 10)  # the heat tiles' rows the sweep kept
    b.step(2)
    assert max(b[i].status() for i in range(len(setups))) == 0
    b.close()


def test_batch_members_against_oracle():
    """Three members of a mixed batch (two 2-D Kelvin-Helmholtz grids and one
    cylindrical heat grid) against the oracle run of each setup from the same
    float32-rounded state: relative L2 <= 1e-5 after 3 steps, time to 1e-5."""
    import math
    from multiphysics_fvm_b200.backend import Batch, physics_name
    from multiphysics_fvm_b200.setups import batch_mixed
    from oracle import fvm_oracle as O
    from tests.helpers import oracle_bcs_of_setup, oracle_schemes_of_setup, setup_state, to_fp32
    setups = batch_mixed.make_setups(seed=7, n_kh=2, n_heat=1, scale=0.25, n_steps=3)
    states = [to_fp32(setup_state(s)) for s in setups]
    b = Batch(setups)
    assert b.launches_per_stage() == 1
    for i, U in enumerate(states):
        b[i].upload(U)
        b[i].set_time(0.0, math.inf, float(setups[i]["time_config"]["CFL"]))
    b.step(3)
    I3 = (slice(None),) + (slice(1, -1),) * 3
    for i, (s, U) in enumerate(zip(setups, states)):
        Uo = U.copy()
        dts = O.run(physics_name(s["physics"]), Uo, s["physical_parameters"],
                    O.Geometry(s["coordinate_system"], s["grid_config"]), oracle_schemes_of_setup(s),
                    oracle_bcs_of_setup(s), s["time_integrator"].__name__, float(s["time_config"]["CFL"]), 3)
        t, steps, _ = b[i].time()
        assert b[i].status() == 0 and steps == 3
        assert abs(t - sum(dts)) <= 1e-5 * sum(dts), (i, t, sum(dts))
        e = rel_l2(b[i].download()[I3], Uo[I3])
        assert e <= 1e-5, (i, physics_name(s["physics"]), e)
    b.close()


def test_batch_cfl_dt_bitwise_single_grid():
    """The batch's CFL reduction splits each grid over blocks in proportion to
    its cells; the maximum does not depend on the split, so the first step's dt
    of every navier_stokes member equals the single grid's bitwise (the grids
    span one to several reduction blocks)."""
    from multiphysics_fvm_b200.backend import Batch, Simulation
    from multiphysics_fvm_b200.setups import batch_mixed
    setups = batch_mixed.make_setups(seed=5, n_kh=6, n_heat=2, scale=0.3, n_steps=1)
    states = batch_mixed.initial_states(setups)
    batch = Batch(setups)
    for i, U in enumerate(states):
        batch[i].upload(U)
        batch[i].set_time(0.0, float("inf"), setups[i]["time_config"]["CFL"])
    batch.step(1)
    sizes = []
    for i, (s, U) in enumerate(zip(setups, states)):
        if s["grid_config"]["nx3"] != 1:
            continue
        sizes.append(s["grid_config"]["nx1"] * s["grid_config"]["nx2"])
        sim = Simulation.from_setup(s)
        sim.upload(U)
        sim.set_time(0.0, float("inf"), s["time_config"]["CFL"])
        sim.step(1)
        assert batch[i].time()[2] == sim.time()[2], (i, batch[i].time(), sim.time())
        sim.close()
    batch.close()
    assert max(sizes) > 2 * 2048 and min(sizes) < 2048, sizes
