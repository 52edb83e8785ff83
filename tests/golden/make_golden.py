"""Generate golden vectors for the finite-volume hot path from the reference itself.

Run once in a container that has the reference checked out (read-only):

    python tests/golden/make_golden.py /path/to/multiphysics-fvm

It imports the reference's own modules (``src.physics.*``, ``src.numerics.*``,
``src.grid.*``, ``src.solver``) with an ``h5py`` stub (``src/io.py`` imports
h5py at module top and it is not needed here), evaluates them on small seeded
states and writes ``tests/golden/golden.npz``:

* ``rhs``   -- ``physics.compute_rhs(U, grid, params, space_schemes)`` for every
  physics x coordinate system x reconstructor/limiter x Riemann solver;
* ``dt``    -- ``physics.compute_dt(U, params, grid, cfl)``;
* ``step``  -- one call of each time integrator (``time_integrators.*``) with
  the reference ``solver.apply_bcs`` and a mixed per-variable BC set.

Inputs are stored next to the outputs, so the tests need neither the reference
nor the generator.  Case metadata is a JSON string under key ``manifest``.
"""
from __future__ import annotations

import json
import os
import sys
import types

import numpy as np

PHYS_VARS = {
    "navier_stokes": ("mass_density", "momentum_x1", "momentum_x2", "momentum_x3", "energy_density"),
    "heat": ("internal_energy_density",),
    "maxwell": ("magnetic_field_x1", "magnetic_field_x2", "magnetic_field_x3",
                "electric_d_field_x1", "electric_d_field_x2", "electric_d_field_x3"),
}

DOMAINS = {
    "cartesian": dict(x1_min=0.0, x1_max=1.0, x2_min=0.0, x2_max=0.8, x3_min=0.0, x3_max=0.6),
    "cylindrical": dict(x1_min=0.1, x1_max=1.0, x2_min=0.0, x2_max=2 * np.pi, x3_min=0.0, x3_max=1.0),
    "spherical": dict(x1_min=0.1, x1_max=1.0, x2_min=0.05 * np.pi, x2_max=0.95 * np.pi,
                      x3_min=0.0, x3_max=2 * np.pi),
}

PARAMS = {
    "navier_stokes": {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 0.01,
                      "gravitational_acceleration": [0.1, -0.3, 0.2]},
    "navier_stokes_inviscid": {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 0.0,
                               "gravitational_acceleration": [0.0, 0.0, 0.0]},
    "heat": {"mass_density": 2.0, "specific_heat_capacity": 3.0,
             "thermal_conductivity": 0.7, "volumetric_heat_source": 0.25},
    "maxwell": {"magnetic_permeability": 1.3, "electric_permittivity": 0.8,
                "electrical_conductivity": 0.4, "charge_density": 0.05,
                "magnetic_cleaning_coeff": 0.002, "electric_cleaning_coeff": 0.003},
}

RECONS = [("piecewise_constant", None), ("muscl", "minmod"),
          ("muscl", "monotonized_central"), ("muscl", "van_leer")]
BC_KINDS = ("periodic", "neumann", "reflecting")
SIDES = ("left", "right", "bottom", "top", "front", "back")


def import_reference(root):
    sys.dont_write_bytecode = True
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    sys.path.insert(0, root)
    from src.numerics import (riemann_solvers, diffusive_solvers, reconstructors,
                              slope_limiters, time_integrators)
    from src.grid import geometry, boundary_conditions
    from src.physics import navier_stokes, heat, maxwell
    from src import solver
    return types.SimpleNamespace(
        riemann=riemann_solvers, diffusive=diffusive_solvers, recon=reconstructors,
        limiters=slope_limiters, integrators=time_integrators, geometry=geometry,
        bc=boundary_conditions, solver=solver,
        physics={"navier_stokes": navier_stokes, "heat": heat, "maxwell": maxwell})


def random_state(phys, shape, rng, params):
    """Seeded positive states with O(1) variation (ghosts included)."""
    if phys == "navier_stokes":
        g = params["heat_capacity_ratio"]
        rho = rng.uniform(1.0, 2.0, shape)
        v = [rng.uniform(-0.5, 0.5, shape) for _ in range(3)]
        P = rng.uniform(1.0, 2.0, shape)
        E = P / (g - 1.0) + 0.5 * rho * (v[0] ** 2 + v[1] ** 2 + v[2] ** 2)
        return np.stack([rho, rho * v[0], rho * v[1], rho * v[2], E])
    if phys == "heat":
        rc = params["mass_density"] * params["specific_heat_capacity"]
        return (rc * rng.uniform(1.0, 2.0, shape))[None]
    return rng.uniform(-1.0, 1.0, (6,) + shape)


def schemes(ref, phys, recon, lim, riem):
    s = {"reconstructor": getattr(ref.recon, recon),
         "slope_limiter": getattr(ref.limiters, lim) if lim else ref.limiters.minmod}
    if phys != "heat":
        s["riemann_solver"] = getattr(ref.riemann, riem)
    if phys != "maxwell":
        s["diffusive_solver"] = ref.diffusive.centered
    return s


def main(root):
    ref = import_reference(root)
    rng = np.random.default_rng(20261203)
    arrays, manifest = {}, []
    n_default = (5, 4, 3)

    def add(name, meta, **arrs):
        manifest.append(dict(name=name, **meta))
        for k, v in arrs.items():
            arrays[f"{name}/{k}"] = np.asarray(v)

    # ---- single residuals ------------------------------------------------
    cases = []
    for cs in DOMAINS:
        for recon, lim in RECONS:
            for riem in ("rusanov", "hll"):
                cases.append(("navier_stokes", "navier_stokes", cs, recon, lim, riem, n_default))
                cases.append(("maxwell", "maxwell", cs, recon, lim, riem, n_default))
            cases.append(("heat", "heat", cs, recon, lim, None, n_default))
        cases.append(("navier_stokes", "navier_stokes_inviscid", cs, "muscl", "van_leer", "hll", n_default))
    # thin and 2D grids
    cases.append(("navier_stokes", "navier_stokes", "cartesian", "muscl", "minmod", "hll", (6, 5, 1)))
    cases.append(("navier_stokes", "navier_stokes", "cylindrical", "muscl", "van_leer", "rusanov", (1, 4, 5)))
    cases.append(("maxwell", "maxwell", "spherical", "muscl", "monotonized_central", "rusanov", (4, 1, 5)))
    cases.append(("heat", "heat", "cylindrical", "muscl", "van_leer", None, (5, 6, 1)))

    for idx, (phys, pkey, cs, recon, lim, riem, n) in enumerate(cases):
        cfg = dict(DOMAINS[cs], nx1=n[0], nx2=n[1], nx3=n[2])
        grid = ref.geometry.build_grid(cs, cfg)
        prm = PARAMS[pkey]
        U = random_state(phys, (n[0] + 2, n[1] + 2, n[2] + 2), rng, prm)
        Ud = {k: U[q].copy() for q, k in enumerate(PHYS_VARS[phys])}
        rhs = ref.physics[phys].compute_rhs(Ud, grid, prm, schemes(ref, phys, recon, lim, riem))
        out = np.stack([rhs[k] for k in PHYS_VARS[phys]])
        dt = ref.physics[phys].compute_dt({k: U[q].copy() for q, k in enumerate(PHYS_VARS[phys])},
                                           prm, grid, 0.37)
        add(f"rhs{idx:03d}", dict(kind="rhs", physics=phys, params=pkey, coords=cs,
                                   grid=cfg, reconstructor=recon, limiter=lim, riemann=riem),
            U=U, rhs=out, dt=np.float64(dt))

    # ---- one integrator step with BCs ------------------------------------
    integ = ["euler_explicit", "rk3", "rk3_ssp", "rk4"]
    step_cases = []
    for phys, pkey, cs, recon, lim, riem in (
            ("navier_stokes", "navier_stokes", "cartesian", "muscl", "van_leer", "hll"),
            ("navier_stokes", "navier_stokes", "spherical", "muscl", "minmod", "rusanov"),
            ("heat", "heat", "cylindrical", "muscl", "monotonized_central", None),
            ("maxwell", "maxwell", "cylindrical", "muscl", "monotonized_central", "hll")):
        for it in integ:
            step_cases.append((phys, pkey, cs, recon, lim, riem, it))
    for idx, (phys, pkey, cs, recon, lim, riem, it) in enumerate(step_cases):
        n = (5, 4, 3)
        cfg = dict(DOMAINS[cs], nx1=n[0], nx2=n[1], nx3=n[2])
        grid = ref.geometry.build_grid(cs, cfg)
        prm = PARAMS[pkey]
        U = random_state(phys, (n[0] + 2, n[1] + 2, n[2] + 2), rng, prm)
        names = PHYS_VARS[phys]
        kinds = [[BC_KINDS[rng.integers(0, 3)] for _ in SIDES] for _ in names]
        if phys == "navier_stokes":
            # density and energy must stay positive in the ghosts: reflecting is
            # used on momentum only (as in setups/rayleigh_taylor.py:143-147)
            for q in (0, 4):
                kinds[q] = ["neumann" if k == "reflecting" else k for k in kinds[q]]
        # periodic must pair up on opposite sides
        for kk in kinds:
            for a in range(3):
                if (kk[2 * a] == "periodic") != (kk[2 * a + 1] == "periodic"):
                    kk[2 * a + 1] = kk[2 * a]
        bcs = {nm: {s: getattr(ref.bc, kinds[q][i]) for i, s in enumerate(SIDES)}
               for q, nm in enumerate(names)}
        Ud = {k: U[q].copy() for q, k in enumerate(names)}
        dt = 0.5 * ref.physics[phys].compute_dt({k: v.copy() for k, v in Ud.items()}, prm, grid, 0.4)
        getattr(ref.integrators, it)(ref.physics[phys].compute_rhs, Ud, dt, prm, grid,
                                     schemes(ref, phys, recon, lim, riem), bcs, ref.solver.apply_bcs)
        out = np.stack([Ud[k] for k in names])
        add(f"step{idx:03d}", dict(kind="step", physics=phys, params=pkey, coords=cs, grid=cfg,
                                    reconstructor=recon, limiter=lim, riemann=riem,
                                    integrator=it, bcs=kinds),
            U=U, U_after=out, dt=np.float64(dt))

    # ---- limiter truth table (includes the MC opposite-sign behaviour) ------
    a = np.array([1.0, 1.0, -1.0, 0.0, 2.0, -0.3, 1.0, 0.5, -2.0, 1e-300])
    b = np.array([-0.1, 0.5, -4.0, 3.0, 0.0, 0.7, 1.0, 2.0, -0.5, 1e-300])
    arrays["limiters/a"], arrays["limiters/b"] = a, b
    for nm in ("minmod", "monotonized_central", "van_leer"):
        arrays[f"limiters/{nm}"] = getattr(ref.limiters, nm)(a.copy(), b.copy())

    params_json = json.dumps(PARAMS)
    out_path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")
    np.savez_compressed(out_path, manifest=json.dumps(manifest), params=params_json, **arrays)
    print(f"wrote {out_path}: {len(manifest)} cases, {os.path.getsize(out_path)/1e3:.0f} kB")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
