"""The register-blocked float32 kernels for cartesian Navier-Stokes
(stage_ns_strip.cuh inviscid, stage_ns_strip_visc.cuh with the Stokes stress)
against the oracle, on grids that cut every kind of tile edge: several
32-column tiles with a partial last one, partial row tiles of both block
shapes, z-march chunks of a few planes (so chunk boundaries fall inside the
grid), every limiter and both Riemann solvers, periodic and walled sides.

Tolerances: single residual relative L-inf <= 2e-6 against the float64 oracle
on the same float32 input; steps relative L2 <= 1e-5 after 4 steps of each
integrator (the 100-step bound is 1e-4); the two block shapes and every
z-chunk give bitwise equal steps.
"""
import math

import numpy as np
import pytest

from oracle import fvm_oracle as O
from tests.helpers import bcs_dict, oracle_bcs, random_ns_state, rel_l2, rel_linf, to_fp32

pytestmark = pytest.mark.gpu

N = (70, 40, 13)
CFG = dict(x1_min=0.0, x1_max=1.0, x2_min=0.0, x2_max=0.7, x3_min=0.0, x3_max=0.4, nx1=N[0], nx2=N[1], nx3=N[2])
PRM = {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 0.0, "gravitational_acceleration": [0.2, -0.1, 0.3]}
# block shapes (tile rows) of each kernel: inviscid 8 (default) and 16; the
# viscous strip kernel has one shape, the viscous grids' default 7 rows (their
# 6-row shape runs the general kernel)
SHAPES = {0.0: (0, 16), 0.02: (0, 7)}
LIMITERS = [("piecewise_constant", None), ("muscl", "minmod"), ("muscl", "monotonized_central"),
            ("muscl", "van_leer")]
WALLS = [["periodic"] * 2 + ["neumann", ("dirichlet", 1.7), "neumann", "neumann"],
         ["periodic"] * 2 + ["neumann", ("dirichlet", 0.05), "reflecting", "neumann"],
         ["periodic"] * 2 + ["reflecting", "reflecting", "neumann", "neumann"],
         ["periodic"] * 2 + ["neumann", ("dirichlet", 0.02), "reflecting", "reflecting"],
         ["periodic"] * 2 + ["neumann", ("dirichlet", 5.0), "neumann", ("dirichlet", 4.0)]]
I3 = (slice(None),) + (slice(1, -1),) * 3


def _sim(recon, lim, riem, kinds, tile_ty=0, zchunk=0, integrator="rk3_ssp", cfg=CFG, prm=PRM):
    from multiphysics_fvm_b200.backend import Simulation
    from multiphysics_fvm_b200.numerics import reconstructors, riemann_solvers, slope_limiters, time_integrators
    sch = {"reconstructor": getattr(reconstructors, recon), "slope_limiter": getattr(slope_limiters, lim or "minmod"),
           "riemann_solver": getattr(riemann_solvers, riem)}
    return Simulation("navier_stokes", "cartesian", cfg, prm, sch, bcs_dict("navier_stokes", kinds),
                      getattr(time_integrators, integrator), precision="fp32", zchunk=zchunk, tile_ty=tile_ty)


def _osch(recon, lim, riem):
    return dict(reconstructor=recon, slope_limiter=lim, riemann_solver=riem)


@pytest.mark.parametrize("mu", [0.0, 0.02])
@pytest.mark.parametrize("riem", ["hll", "rusanov"])
@pytest.mark.parametrize("recon,lim", LIMITERS)
def test_residual_against_oracle(recon, lim, riem, mu):
    rng = np.random.default_rng(21)
    prm = dict(PRM, dynamic_viscosity=mu)
    U = to_fp32(random_ns_state(tuple(x + 2 for x in N), rng))
    ref = O.ns_rhs(U, O.Geometry("cartesian", CFG), prm, _osch(recon, lim, riem))
    for ty, z in ((SHAPES[mu][0], 0), (SHAPES[mu][1], 5)):
        sim = _sim(recon, lim, riem, [["periodic"] * 6] * 5, tile_ty=ty, zchunk=z, prm=prm)
        sim.upload(U)
        e = rel_linf(sim.residual(), ref)
        sim.close()
        assert e <= 2e-6, (recon, lim, riem, mu, ty, z, e)


@pytest.mark.parametrize("mu", [0.0, 0.02])
@pytest.mark.parametrize("integrator", ["euler_explicit", "rk3", "rk3_ssp", "rk4"])
@pytest.mark.parametrize("recon,lim,riem", [("muscl", "minmod", "hll"), ("muscl", "van_leer", "rusanov"),
                                            ("muscl", "monotonized_central", "hll"),
                                            ("piecewise_constant", None, "rusanov")])
def test_walled_steps_against_oracle(recon, lim, riem, integrator, mu):
    rng = np.random.default_rng(22)
    prm = dict(PRM, dynamic_viscosity=mu)
    U = to_fp32(random_ns_state(tuple(x + 2 for x in N), rng))
    Uo = U.copy()
    dts = O.run("navier_stokes", Uo, prm, O.Geometry("cartesian", CFG), _osch(recon, lim, riem), oracle_bcs(WALLS),
                integrator, 0.3, 4)
    outs = []
    for ty, z in ((SHAPES[mu][0], 0), (SHAPES[mu][1], 4), (SHAPES[mu][0], 3)):
        sim = _sim(recon, lim, riem, WALLS, tile_ty=ty, zchunk=z, integrator=integrator, prm=prm)
        sim.upload(U)
        sim.set_time(0.0, math.inf, 0.3)
        sim.step(4)
        assert sim.status() == 0
        t, steps, _ = sim.time()
        assert steps == 4 and abs(t - sum(dts)) <= 1e-5 * sum(dts)
        outs.append(sim.download())
        sim.close()
        e = rel_l2(outs[-1][I3], Uo[I3])
        assert e <= 1e-5, (recon, lim, riem, integrator, mu, ty, z, e)
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])


@pytest.mark.parametrize("mu", [0.0, 0.02])
@pytest.mark.parametrize("n", [(45, 27, 1), (33, 17, 2), (7, 5, 3)])
def test_one_plane_and_thin_grids(n, mu):
    """nx3 = 1 and nx3 = 2 grids (the z-march has one or two output planes and
    reads ghost planes on both sides) and a grid narrower than one tile."""
    cfg = dict(CFG, nx1=n[0], nx2=n[1], nx3=n[2])
    rng = np.random.default_rng(sum(n))
    U = to_fp32(random_ns_state(tuple(x + 2 for x in n), rng))
    kinds = [["periodic"] * 4 + ["neumann", "neumann"]] * 5
    prm = dict(PRM, dynamic_viscosity=mu)
    ref = O.ns_rhs(U, O.Geometry("cartesian", cfg), prm, _osch("muscl", "van_leer", "hll"))
    sim = _sim("muscl", "van_leer", "hll", kinds, cfg=cfg, prm=prm, tile_ty=SHAPES[mu][0])
    sim.upload(U)
    e = rel_linf(sim.residual(), ref)
    sim.close()
    assert e <= 2e-6, (n, e)


FLAT_KINDS = [["periodic"] * 2 + ["neumann", ("dirichlet", 1.7), "neumann", "neumann"],
              ["periodic"] * 2 + ["neumann", ("dirichlet", 0.05), "periodic", "periodic"],
              ["periodic"] * 2 + ["reflecting", "reflecting", "neumann", "neumann"],
              ["periodic"] * 2 + ["neumann", ("dirichlet", 0.02), "neumann", "neumann"],
              ["periodic"] * 2 + ["neumann", ("dirichlet", 5.0), "periodic", "periodic"]]


@pytest.mark.parametrize("integrator", ["euler_explicit", "rk3", "rk3_ssp", "rk4"])
@pytest.mark.parametrize("recon,lim,riem", [("muscl", "minmod", "hll"), ("muscl", "van_leer", "rusanov")])
def test_one_plane_steps_against_oracle(recon, lim, riem, integrator):
    """nx3 = 1 with periodic or Neumann x3 sides for every variable: the x3
    fluxes cancel exactly and the kernel steps plane 1 alone (no x3 ring)."""
    cfg = dict(CFG, nx1=70, nx2=40, nx3=1)
    rng = np.random.default_rng(23)
    U = to_fp32(random_ns_state((72, 42, 3), rng))
    Uo = U.copy()
    dts = O.run("navier_stokes", Uo, PRM, O.Geometry("cartesian", cfg), _osch(recon, lim, riem),
                oracle_bcs(FLAT_KINDS), integrator, 0.3, 4)
    sim = _sim(recon, lim, riem, FLAT_KINDS, integrator=integrator, cfg=cfg)
    sim.upload(U)
    sim.set_time(0.0, math.inf, 0.3)
    sim.step(4)
    assert sim.status() == 0
    t, steps, _ = sim.time()
    assert steps == 4 and abs(t - sum(dts)) <= 1e-5 * sum(dts)
    e = rel_l2(sim.download()[I3], Uo[I3])
    sim.close()
    assert e <= 1e-5, (recon, lim, riem, integrator, e)
