"""Heat and Maxwell CUDA paths vs the reference's golden vectors and the oracle.

float64 build: relative L-inf <= 1e-12 against NumPy; float32 single residual:
relative L-inf <= 2e-6 against the float64 oracle on the same float32 input.
"""
import numpy as np
import pytest

from oracle import fvm_oracle as O
from tests.helpers import bcs_dict, oracle_schemes, rel_linf, schemes_from_case, to_fp32

pytestmark = pytest.mark.gpu
I3 = (slice(None),) + (slice(1, -1),) * 3


def _sim(c, prm, precision, kinds=None, integrator=None):
    from multiphysics_fvm_b200.backend import Simulation, VARIABLES
    from multiphysics_fvm_b200.numerics import time_integrators as ti
    nv = len(VARIABLES[c["physics"]])
    bcs = bcs_dict(c["physics"], kinds or [["periodic"] * 6] * nv)
    return Simulation(c["physics"], c["coords"], c["grid"], prm, schemes_from_case(c), bcs,
                      getattr(ti, integrator) if integrator else None, precision=precision)


@pytest.mark.parametrize("physics", ["heat", "maxwell"])
def test_golden_residual(golden, physics):
    z, man, P = golden
    for c in man:
        if c["kind"] != "rhs" or c["physics"] != physics:
            continue
        prm = P[c["params"]]
        sim = _sim(c, prm, "fp64")
        sim.upload(z[c["name"] + "/U"])
        e = rel_linf(sim.residual(), z[c["name"] + "/rhs"])
        assert e <= 1e-12, (c["name"], c["coords"], c["reconstructor"], c["limiter"], c.get("riemann"), e)
        dt = sim.compute_dt(0.37)
        assert abs(dt - float(z[c["name"] + "/dt"])) <= 1e-12 * dt
        sim.close()
        U32 = to_fp32(z[c["name"] + "/U"])
        ref = O.RHS[physics](U32, O.Geometry(c["coords"], c["grid"]), prm, oracle_schemes(c))
        sim = _sim(c, prm, "fp32")
        sim.upload(U32)
        e = rel_linf(sim.residual(), ref)
        assert e <= 2e-6, (c["name"], c["coords"], c["reconstructor"], c["limiter"], e)
        sim.close()


@pytest.mark.parametrize("physics", ["heat", "maxwell"])
def test_golden_steps(golden, physics):
    z, man, P = golden
    for c in man:
        if c["kind"] != "step" or c["physics"] != physics:
            continue
        sim = _sim(c, P[c["params"]], "fp64", kinds=c["bcs"], integrator=c["integrator"])
        sim.upload(z[c["name"] + "/U"])
        sim.step(1, dt=float(z[c["name"] + "/dt"]))
        e = rel_linf(sim.download()[I3], z[c["name"] + "/U_after"][I3])
        assert e <= 1e-12, (c["name"], c["integrator"], e)
        sim.close()


@pytest.mark.parametrize("coords", ["cartesian", "cylindrical", "spherical"])
@pytest.mark.parametrize("physics,lim,riem", [("heat", None, None), ("heat", "van_leer", None),
                                              ("maxwell", "monotonized_central", "rusanov"),
                                              ("maxwell", "minmod", "hll")])
def test_multi_tile(coords, physics, lim, riem):
    rng = np.random.default_rng(3)
    n = (35, 17, 10)
    dom = {"cartesian": (0, 1, 0, 0.8, 0, 0.6), "cylindrical": (0.1, 1, 0, 2 * np.pi, 0, 1),
           "spherical": (0.1, 1, 0.05 * np.pi, 0.95 * np.pi, 0, 2 * np.pi)}[coords]
    cfg = dict(x1_min=dom[0], x1_max=dom[1], x2_min=dom[2], x2_max=dom[3], x3_min=dom[4], x3_max=dom[5],
               nx1=n[0], nx2=n[1], nx3=n[2])
    c = dict(physics=physics, coords=coords, grid=cfg, reconstructor="muscl" if lim else "piecewise_constant",
             limiter=lim, riemann=riem)
    sh = tuple(x + 2 for x in n)
    if physics == "heat":
        prm = {"mass_density": 2.0, "specific_heat_capacity": 3.0, "thermal_conductivity": 0.7,
               "volumetric_heat_source": 0.25}
        U = (6.0 * rng.uniform(1.0, 2.0, sh))[None]
    else:
        prm = {"magnetic_permeability": 1.3, "electric_permittivity": 0.8, "electrical_conductivity": 0.4,
               "charge_density": 0.05, "magnetic_cleaning_coeff": 0.002, "electric_cleaning_coeff": 0.003}
        U = rng.uniform(-1.0, 1.0, (6,) + sh)
    geo = O.Geometry(coords, cfg)
    ref = O.RHS[physics](U, geo, prm, oracle_schemes(c))
    sim = _sim(c, prm, "fp64")
    sim.upload(U)
    assert rel_linf(sim.residual(), ref) <= 1e-12
    sim.close()
    U32 = to_fp32(U)
    ref32 = O.RHS[physics](U32, geo, prm, oracle_schemes(c))
    sim = _sim(c, prm, "fp32")
    sim.upload(U32)
    assert rel_linf(sim.residual(), ref32) <= 2e-6
    sim.close()
