"""The curvilinear benchmark schemes, the Dirichlet wall and the heat / Maxwell
conserved totals, stepped through the CUDA path and compared with the NumPy
oracle (no self-comparison with the float64 build).

* C2a at reduced size: Maxwell on the spherical shell (setups/
  maxwell_spherical_pulse.py), MUSCL monotonized-central + Rusanov + RK4,
  conducting walls at both r and both theta limits, periodic phi, 24x20x32,
  50 steps (maxwell.py:603-729, time_integrators.py:162-221,
  boundary_conditions.py:13-91);
* C2b at reduced size: heat on the cylindrical annulus (setups/
  heat_cylindrical_hotspot.py), piecewise constant + SSPRK3, Dirichlet T = 1 on
  the r and z walls, 24x32x16, 100 steps (heat.py:354-473);
* one step of every integrator with Dirichlet values on several sides and
  variables, for all three physics and coordinate systems;
* heat rho*cp*T and Maxwell field / EM-energy totals against NumPy sums over
  the oracle geometry's volumes.

Tolerances: float64 build relative L2 <= 1e-10 after the run (single steps
relative L-inf <= 1e-12); float32 build relative L2 <= 1e-4 against the oracle
run from the same float32-rounded initial state; simulated time to 1e-12
(float64) / 1e-5 (float32); totals relative <= 1e-12 against NumPy on the same
state, <= 1e-6 against the oracle's after a run.
"""
import math

import numpy as np
import pytest

from oracle import fvm_oracle as O
from tests.helpers import (bcs_dict, oracle_bcs, oracle_bcs_of_setup, oracle_schemes_of_setup, random_ns_state,
                           rel_l2, rel_linf, setup_state, to_fp32)

pytestmark = pytest.mark.gpu

I3 = (slice(None),) + (slice(1, -1),) * 3
def _run_setup_against_oracle(s, physics, integrator, n_steps):
    from multiphysics_fvm_b200.backend import Simulation
    U0 = setup_state(s)
    geo = O.Geometry(s["coordinate_system"], s["grid_config"])
    sch = oracle_schemes_of_setup(s)
    bcs = oracle_bcs_of_setup(s)
    cfl = float(s["time_config"]["CFL"])
    results = {}
    for precision, tol, ttol in (("fp64", 1e-10, 1e-12), ("fp32", 1e-4, 1e-5)):
        Ui = U0 if precision == "fp64" else to_fp32(U0)
        Uo = Ui.copy()
        dts = O.run(physics, Uo, s["physical_parameters"], geo, sch, bcs, integrator, cfl, n_steps)
        sim = Simulation.from_setup(dict(s, precision=precision))
        sim.upload(Ui)
        sim.set_time(0.0, math.inf, cfl)
        sim.step(n_steps)
        assert sim.status() == 0, precision
        t, steps, _ = sim.time()
        assert steps == n_steps
        assert abs(t - sum(dts)) <= ttol * sum(dts), (precision, t, sum(dts))
        got = sim.download()[I3]
        err = rel_l2(got, Uo[I3])
        tot = sim.totals()
        sim.close()
        print(f"{physics} {precision}: relative L2 {err:.2e} after {n_steps} steps")
        assert err <= tol, (precision, err)
        results[precision] = (Uo, tot)
    return geo, results


def test_c2a_reduced_maxwell_spherical_against_oracle():
    from multiphysics_fvm_b200.setups import maxwell_spherical_pulse as mx
    s = mx.get_setup(24, 20, 32, n_steps=50)
    s["initial_conditions"]["parameters"]["width"] = 0.15  # resolved on the reduced grid
    geo, res = _run_setup_against_oracle(s, "maxwell", "rk4", 50)
    # field and EM-energy totals of the final state against NumPy sums of the oracle's
    prm = s["physical_parameters"]
    for precision, (Uo, tot) in res.items():
        ref = _maxwell_totals(Uo, geo.V, prm["magnetic_permeability"], prm["electric_permittivity"])
        scale = np.max(np.abs(ref[:6])) + 1e-300
        assert np.all(np.abs(tot[:6] - ref[:6]) <= 1e-6 * scale), (precision, tot, ref)
        assert abs(tot[6] - ref[6]) <= 1e-6 * ref[6], (precision, tot[6], ref[6])


def test_c2b_reduced_heat_cylindrical_dirichlet_against_oracle():
    from multiphysics_fvm_b200.setups import heat_cylindrical_hotspot as hc
    s = hc.get_setup(24, 32, 16, n_steps=100)
    s["initial_conditions"]["parameters"]["width"] = 0.2
    geo, res = _run_setup_against_oracle(s, "heat", "rk3_ssp", 100)
    for precision, (Uo, tot) in res.items():
        ref = float(np.sum(Uo[0][1:-1, 1:-1, 1:-1] * geo.V))
        assert abs(tot[0] - ref) <= 1e-6 * abs(ref), (precision, tot[0], ref)


def _maxwell_totals(U, V, mu, ep):
    I = (slice(1, -1),) * 3
    t = [float(np.sum(U[q][I] * V)) for q in range(6)]
    em = sum(U[q][I] ** 2 / mu for q in range(3)) + sum(U[q][I] ** 2 / ep for q in range(3, 6))
    return np.array(t + [float(np.sum(0.5 * em * V))])


def _random_state(physics, sh, rng):
    if physics == "navier_stokes":
        return random_ns_state(sh, rng)
    if physics == "heat":
        return (6.0 * rng.uniform(1.0, 2.0, sh))[None]
    return rng.uniform(-1.0, 1.0, (6,) + sh)


PARAMS = {
    "navier_stokes": {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 0.02,
                      "gravitational_acceleration": [0.0, -0.3, 0.1]},
    "heat": {"mass_density": 2.0, "specific_heat_capacity": 3.0, "thermal_conductivity": 0.7,
             "volumetric_heat_source": 0.25},
    "maxwell": {"magnetic_permeability": 1.3, "electric_permittivity": 0.8, "electrical_conductivity": 0.4,
                "charge_density": 0.05, "magnetic_cleaning_coeff": 0.002, "electric_cleaning_coeff": 0.003},
}
DOMAINS = {"cartesian": (0, 1, 0, 0.8, 0, 0.6), "cylindrical": (0.1, 1, 0, 2 * np.pi, 0, 1),
           "spherical": (0.1, 1, 0.05 * np.pi, 0.95 * np.pi, 0, 2 * np.pi)}


def _dirichlet_value(physics, q, rng):
    """Wall values that keep every ghost state physical: positive density and
    pressure for navier_stokes, positive rho*cp*T for heat."""
    if physics == "navier_stokes":
        return {0: 2.0, 4: 5.0}[q] * float(rng.uniform(0.95, 1.05)) if q in (0, 4) else float(rng.uniform(-0.1, 0.1))
    if physics == "heat":
        return 9.0 * float(rng.uniform(0.8, 1.2))
    return float(rng.uniform(-0.5, 0.5))


def _dirichlet_kinds(physics, nv, rng):
    """Dirichlet on several sides and variables, the other sides drawn from the
    reference's kinds (periodic in pairs only); every variable gets a Dirichlet
    side on each non-periodic axis.  Density and energy are never reflecting."""
    kinds = []
    for q in range(nv):
        row = []
        for ax in range(3):
            if ax == 1 and rng.integers(0, 3) == 0:
                row += ["periodic", "periodic"]
                continue
            for _ in range(2):
                k = int(rng.integers(0, 3))
                if k == 2 and physics == "navier_stokes" and q in (0, 4):
                    k = 0
                row.append(("dirichlet", _dirichlet_value(physics, q, rng)) if k == 0 else
                           ("neumann" if k == 1 else "reflecting"))
        for ax in range(3):
            if row[2 * ax] != "periodic" and not any(isinstance(row[2 * ax + s], tuple) for s in range(2)):
                row[2 * ax + 1] = ("dirichlet", _dirichlet_value(physics, q, rng))
        kinds.append(row)
    return kinds


@pytest.mark.parametrize("physics", ["navier_stokes", "heat", "maxwell"])
@pytest.mark.parametrize("coords", ["cartesian", "cylindrical", "spherical"])
def test_dirichlet_steps_against_oracle(physics, coords):
    from multiphysics_fvm_b200.backend import Simulation
    from multiphysics_fvm_b200.numerics import (diffusive_solvers, reconstructors, riemann_solvers,
                                                slope_limiters, time_integrators)
    rng = np.random.default_rng({"navier_stokes": 1, "heat": 2, "maxwell": 3}[physics] * 10 + len(coords))
    n = (11, 9, 7)
    dom = DOMAINS[coords]
    cfg = dict(x1_min=dom[0], x1_max=dom[1], x2_min=dom[2], x2_max=dom[3], x3_min=dom[4], x3_max=dom[5],
               nx1=n[0], nx2=n[1], nx3=n[2])
    nv = {"navier_stokes": 5, "heat": 1, "maxwell": 6}[physics]
    kinds = _dirichlet_kinds(physics, nv, rng)
    prm = PARAMS[physics]
    sch = {"reconstructor": reconstructors.muscl, "slope_limiter": slope_limiters.van_leer,
           "diffusive_solver": diffusive_solvers.centered}
    if physics != "heat":
        sch["riemann_solver"] = riemann_solvers.hll
    osch = dict(reconstructor="muscl", slope_limiter="van_leer", riemann_solver="hll" if physics != "heat" else None)
    geo = O.Geometry(coords, cfg)
    sh = tuple(x + 2 for x in n)
    for integrator in ("euler_explicit", "rk3", "rk3_ssp", "rk4"):
        U = _random_state(physics, sh, rng)
        dt = 0.2 * O.compute_dt(physics, U, prm, geo, 0.4)
        Uo = U.copy()
        O.integrate(integrator, physics, Uo, dt, prm, geo, osch, oracle_bcs(kinds))
        sim = Simulation(physics, coords, cfg, prm, sch, bcs_dict(physics, kinds),
                         getattr(time_integrators, integrator), precision="fp64")
        sim.upload(U)
        sim.step(1, dt=dt)
        assert sim.status() == 0
        e = rel_linf(sim.download()[I3], Uo[I3])
        sim.close()
        assert e <= 1e-12, (physics, coords, integrator, kinds, e)
    # three steps in float32 against the oracle on the same float32 input
    U = to_fp32(_random_state(physics, sh, rng))
    Uo = U.copy()
    dts = O.run(physics, Uo, prm, geo, osch, oracle_bcs(kinds), "rk3_ssp", 0.3, 3)
    sim = Simulation(physics, coords, cfg, prm, sch, bcs_dict(physics, kinds), time_integrators.rk3_ssp,
                     precision="fp32")
    sim.upload(U)
    sim.set_time(0.0, math.inf, 0.3)
    sim.step(3)
    assert sim.status() == 0
    t, _, _ = sim.time()
    assert abs(t - sum(dts)) <= 1e-5 * sum(dts)
    e = rel_l2(sim.download()[I3], Uo[I3])
    sim.close()
    assert e <= 1e-5, (physics, coords, e)


def test_dirichlet_ghost_faces_of_download():
    """Downloaded ghost faces are refreshed from the boundary conditions of the
    final interior: on a Dirichlet side, ghost = 2 value - adjacent interior."""
    from multiphysics_fvm_b200.backend import Simulation
    from multiphysics_fvm_b200.numerics import reconstructors, slope_limiters, diffusive_solvers
    rng = np.random.default_rng(7)
    n = (9, 8, 6)
    cfg = dict(x1_min=0, x1_max=1, x2_min=0, x2_max=1, x3_min=0, x3_max=1, nx1=n[0], nx2=n[1], nx3=n[2])
    kinds = [[("dirichlet", 5.0), ("dirichlet", 7.0), "neumann", ("dirichlet", 6.5), "periodic", "periodic"]]
    sim = Simulation("heat", "cartesian", cfg, PARAMS["heat"],
                     {"reconstructor": reconstructors.piecewise_constant, "slope_limiter": slope_limiters.minmod,
                      "diffusive_solver": diffusive_solvers.centered}, bcs_dict("heat", kinds), precision="fp64")
    U = _random_state("heat", tuple(x + 2 for x in n), rng)
    sim.upload(U)
    sim.set_time(0.0, math.inf, 0.4)
    sim.step(2)
    D = sim.download()[0]
    sim.close()
    J = (slice(1, -1), slice(1, -1))
    np.testing.assert_allclose(D[0][J], 2 * 5.0 - D[1][J], rtol=0, atol=1e-12)
    np.testing.assert_allclose(D[-1][J], 2 * 7.0 - D[-2][J], rtol=0, atol=1e-12)
    np.testing.assert_allclose(D[1:-1, -1, 1:-1], 2 * 6.5 - D[1:-1, -2, 1:-1], rtol=0, atol=1e-12)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("coords", ["cartesian", "cylindrical", "spherical"])
def test_heat_and_maxwell_totals_against_numpy(precision, coords):
    from multiphysics_fvm_b200.backend import Simulation
    from multiphysics_fvm_b200.numerics import reconstructors, riemann_solvers, slope_limiters
    rng = np.random.default_rng(5)
    n = (37, 19, 11)
    dom = DOMAINS[coords]
    cfg = dict(x1_min=dom[0], x1_max=dom[1], x2_min=dom[2], x2_max=dom[3], x3_min=dom[4], x3_max=dom[5],
               nx1=n[0], nx2=n[1], nx3=n[2])
    geo = O.Geometry(coords, cfg)
    sh = tuple(x + 2 for x in n)
    sch = {"reconstructor": reconstructors.muscl, "slope_limiter": slope_limiters.minmod,
           "riemann_solver": riemann_solvers.rusanov}
    # heat: the total of rho*cp*T
    U = _random_state("heat", sh, rng)
    U = to_fp32(U) if precision == "fp32" else U
    sim = Simulation("heat", coords, cfg, PARAMS["heat"], sch, bcs_dict("heat", [["periodic"] * 6]),
                     precision=precision)
    sim.upload(U)
    tot = sim.totals()
    sim.close()
    ref = float(np.sum(U[0][1:-1, 1:-1, 1:-1] * geo.V))
    assert abs(tot[0] - ref) <= 1e-12 * abs(ref), (tot, ref)
    # Maxwell with mu != epsilon: six field totals and 0.5 (B^2/mu + D^2/eps) V
    U = _random_state("maxwell", sh, rng)
    U = to_fp32(U) if precision == "fp32" else U
    prm = PARAMS["maxwell"]
    sim = Simulation("maxwell", coords, cfg, prm, sch, bcs_dict("maxwell", [["periodic"] * 6] * 6),
                     precision=precision)
    sim.upload(U)
    tot = sim.totals()
    sim.close()
    ref = _maxwell_totals(U, geo.V, prm["magnetic_permeability"], prm["electric_permittivity"])
    scale = np.sum(np.abs(U[:, 1:-1, 1:-1, 1:-1]) * geo.V, axis=(1, 2, 3))
    assert np.all(np.abs(tot[:6] - ref[:6]) <= 1e-12 * scale), (tot, ref)
    assert abs(tot[6] - ref[6]) <= 1e-12 * ref[6], (tot[6], ref[6])
    # swapping mu and epsilon must change the EM energy (the test would catch it)
    swapped = _maxwell_totals(U, geo.V, prm["electric_permittivity"], prm["magnetic_permeability"])
    assert abs(swapped[6] - ref[6]) > 1e-6 * ref[6]


def test_heat_totals_track_the_oracle_fp32():
    """The reference's heat flux is zero in the ghost cells (heat.py:95), so a
    boundary face carries half the interior flux and no wall kind conserves
    sum(rho cp T V) exactly.  The device totals after 200 float32 steps must
    follow the oracle's (relative <= 1e-6) and differ from the initial ones."""
    from multiphysics_fvm_b200.backend import Simulation
    from multiphysics_fvm_b200.numerics import reconstructors, slope_limiters, time_integrators
    rng = np.random.default_rng(9)
    n = (40, 24, 16)
    cfg = dict(x1_min=0, x1_max=1, x2_min=0, x2_max=0.6, x3_min=0, x3_max=0.4, nx1=n[0], nx2=n[1], nx3=n[2])
    prm = dict(PARAMS["heat"], volumetric_heat_source=0.0)
    U = to_fp32(_random_state("heat", tuple(x + 2 for x in n), rng))
    geo = O.Geometry("cartesian", cfg)
    Uo = U.copy()
    O.run("heat", Uo, prm, geo, dict(reconstructor="muscl", slope_limiter="van_leer", riemann_solver=None),
          oracle_bcs([["periodic"] * 6]), "rk3_ssp", 0.4, 200)
    ref0 = float(np.sum(U[0][1:-1, 1:-1, 1:-1] * geo.V))
    ref1 = float(np.sum(Uo[0][1:-1, 1:-1, 1:-1] * geo.V))
    sim = Simulation("heat", "cartesian", cfg, prm,
                     {"reconstructor": reconstructors.muscl, "slope_limiter": slope_limiters.van_leer},
                     bcs_dict("heat", [["periodic"] * 6]), time_integrators.rk3_ssp, precision="fp32")
    sim.upload(U)
    sim.set_time(0.0, math.inf, 0.4)
    t0 = sim.totals()
    sim.step(200)
    t1 = sim.totals()
    assert sim.status() == 0
    sim.close()
    assert abs(t0[0] - ref0) <= 1e-12 * abs(ref0)
    assert abs(t1[0] - ref1) <= 1e-6 * abs(ref0), (t1, ref1, ref0)
    assert abs(ref1 - ref0) > 1e-6 * abs(ref0)  # the reference scheme itself drifts here
