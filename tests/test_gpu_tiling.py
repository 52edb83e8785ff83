"""The second block shape of the float32 kernels (for viscous cartesian
navier_stokes the 8-row register-blocked kernel against the default 6-row
general one, 16 rows against 8 for inviscid navier_stokes, 8 against 16 for
piecewise-constant heat): its residual
matches the oracle on a grid of many partial tiles, its steps are bitwise equal
to the default shape's (a cell's arithmetic does not depend on the tile it sits
in), and the autotuner picks one of the two shapes and leaves the state as it
found it."""
import math

import numpy as np
import pytest

from oracle import fvm_oracle as O
from tests.helpers import bcs_dict, oracle_schemes, random_ns_state, rel_l2, rel_linf, schemes_from_case, to_fp32

pytestmark = pytest.mark.gpu

N = (37, 19, 11)
CFG = dict(x1_min=0.0, x1_max=1.0, x2_min=0.0, x2_max=0.8, x3_min=0.0, x3_max=0.6, nx1=N[0], nx2=N[1], nx3=N[2])


def _sim(c, prm, tile_ty, integrator="rk3_ssp"):
    from multiphysics_fvm_b200.backend import Simulation, VARIABLES
    from multiphysics_fvm_b200.numerics import time_integrators as ti
    nv = len(VARIABLES[c["physics"]])
    return Simulation(c["physics"], "cartesian", CFG, prm, schemes_from_case(c),
                      bcs_dict(c["physics"], [["periodic"] * 6] * nv), getattr(ti, integrator), precision="fp32",
                      tile_ty=tile_ty)


CASES = [
    (dict(physics="navier_stokes", reconstructor="muscl", limiter="van_leer", riemann="hll"),
     {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 1e-3, "gravitational_acceleration": [0.1, -0.2, 0.3]}),
    (dict(physics="navier_stokes", reconstructor="muscl", limiter="minmod", riemann="hll"),
     {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 0.0, "gravitational_acceleration": [0.0, 0.0, 0.0]}),
    (dict(physics="heat", reconstructor="piecewise_constant", limiter=None, riemann=None),
     {"mass_density": 2.0, "specific_heat_capacity": 3.0, "thermal_conductivity": 0.7,
      "volumetric_heat_source": 0.25}),
]


def _state(c, rng):
    sh = tuple(x + 2 for x in N)
    if c["physics"] == "heat":
        return to_fp32((6.0 * rng.uniform(1.0, 2.0, sh))[None])
    return to_fp32(random_ns_state(sh, rng))


ALT_ROWS = [6, 16, 8]
SAME_KERNEL = [False, True, True]  # viscous: the two shapes are two kernels


@pytest.mark.parametrize("c,prm,alt,same", [cp + (a, sk) for cp, a, sk in zip(CASES, ALT_ROWS, SAME_KERNEL)],
                         ids=["ns_viscous", "ns_inviscid", "heat"])
def test_second_block_shape(c, prm, alt, same):
    c = dict(c, coords="cartesian", grid=CFG)
    rng = np.random.default_rng(13)
    U = _state(c, rng)
    ref = O.RHS[c["physics"]](U, O.Geometry("cartesian", CFG), prm, oracle_schemes(c))
    sims = {ty: _sim(c, prm, ty) for ty in (0, alt)}
    assert sims[alt].tiling()[0] == alt and sims[0].tiling()[0] != alt
    outs = {}
    for ty, sim in sims.items():
        sim.upload(U)
        assert rel_linf(sim.residual(), ref) <= 2e-6
        sim.upload(U)
        sim.set_time(0.0, math.inf, 0.3)
        sim.step(3)
        assert sim.status() == 0
        outs[ty] = sim.download()
    if same:
        assert np.array_equal(outs[0], outs[alt])
    else:  # two kernels with their own float32 rounding
        assert rel_l2(outs[0], outs[alt]) <= 1e-6


def test_autotune_chooses_a_shape_and_restores_the_state():
    c, prm = CASES[1]
    c = dict(c, coords="cartesian", grid=CFG)
    U = _state(c, np.random.default_rng(2))
    sim = _sim(c, prm, 0)
    sim.upload(U)
    sim.set_time(0.0, math.inf, 0.3)
    before = sim.download()
    z, ms = sim.autotune()
    ty, z2 = sim.tiling()
    assert ty in (8, 16) and z2 == z and ms > 0
    assert np.array_equal(sim.download(), before)
    t, steps, _ = sim.time()
    assert steps == 0 and t == 0.0


def test_unsupported_tile_rows_are_rejected():
    c, prm = CASES[1]
    c = dict(c, coords="cartesian", grid=CFG)
    with pytest.raises(ValueError, match="tile_ty"):
        _sim(c, prm, 5)


@pytest.mark.parametrize("integrator,stages", [("euler_explicit", 1), ("rk3_ssp", 3), ("rk4", 4)])
def test_step_launches_match_the_profiled_launches(integrator, stages):
    """fvm_step_launches (the bench line's gpu_launches) against the stage
    launches that fvm_profile_steps counts: per step a CFL reduction
    (navier_stokes), then per stage a ghost fill and the stage kernel."""
    for k, (c, prm) in enumerate(CASES[1:]):
        c = dict(c, coords="cartesian", grid=CFG)
        sim = _sim(c, prm, 0, integrator=integrator)
        sim.upload(_state(c, np.random.default_rng(5)))
        sim.set_time(0.0, math.inf, 0.3)
        _, _, launches = sim.profile_steps(2)
        assert launches == 2 * stages
        assert sim.step_launches() == (1 if c["physics"] == "navier_stokes" else 0) + 2 * stages
        sim.close()
