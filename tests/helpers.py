"""Shared helpers for the parity tests (test infrastructure only)."""
from __future__ import annotations

import numpy as np

from oracle import fvm_oracle as O

SIDES = O.SIDES


def rel_linf(a, b):
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


def rel_l2(a, b):
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def schemes_from_case(c):
    from multiphysics_fvm_b200.numerics import reconstructors, riemann_solvers, slope_limiters, diffusive_solvers
    s = {"reconstructor": getattr(reconstructors, c["reconstructor"]),
         "slope_limiter": getattr(slope_limiters, c["limiter"] or "minmod")}
    if c.get("riemann"):
        s["riemann_solver"] = getattr(riemann_solvers, c["riemann"])
    s["diffusive_solver"] = diffusive_solvers.centered
    return s


def oracle_schemes(c):
    return dict(reconstructor=c["reconstructor"], slope_limiter=c["limiter"], riemann_solver=c.get("riemann"))


def bcs_dict(physics, kinds):
    """kinds: [var][side] names -> bcs dict of this package's selectors."""
    from multiphysics_fvm_b200.grid import boundary_conditions as bc
    from multiphysics_fvm_b200.backend import VARIABLES
    out = {}
    for q, v in enumerate(VARIABLES[physics]):
        row = {}
        for s, side in enumerate(SIDES):
            k = kinds[q][s]
            row[side] = bc.dirichlet(k[1]) if isinstance(k, tuple) else getattr(bc, k)
        out[v] = row
    return out


def oracle_bcs(kinds):
    return [{s: (k if isinstance(k, tuple) else (k, 0.0)) for s, k in zip(SIDES, kk)} for kk in kinds]


def random_ns_state(shape, rng, gam=1.4):
    rho = rng.uniform(1.0, 2.0, shape)
    v = [rng.uniform(-0.5, 0.5, shape) for _ in range(3)]
    P = rng.uniform(1.0, 2.0, shape)
    E = P / (gam - 1.0) + 0.5 * rho * (v[0] ** 2 + v[1] ** 2 + v[2] ** 2)
    return np.stack([rho, rho * v[0], rho * v[1], rho * v[2], E])


def to_fp32(U):
    return U.astype(np.float32).astype(np.float64)


KIND_NAMES = {0: "periodic", 1: "neumann", 2: "reflecting", 3: "dirichlet"}


def setup_state(s):
    """The setup's initial state as one [var, ...] array (ghosts included)."""
    from multiphysics_fvm_b200.backend import VARIABLES, physics_name
    from multiphysics_fvm_b200.grid.geometry import build_grid
    g = build_grid(s["coordinate_system"], s["grid_config"])
    U = s["physics"].allocate_u(s["grid_config"])
    s["initial_conditions"]["initializer"](U, s["physical_parameters"], g, s["initial_conditions"]["parameters"])
    return np.stack([U[k] for k in VARIABLES[physics_name(s["physics"])]])


def oracle_bcs_of_setup(s):
    """The setup's per-variable, per-side selectors as oracle (kind, value) pairs."""
    from multiphysics_fvm_b200.backend import bc_codes, physics_name
    rows = bc_codes(physics_name(s["physics"]), s["boundary_conditions"])
    return [{side: (KIND_NAMES[k], v) for side, (k, v) in zip(O.SIDES, row)} for row in rows]


def oracle_schemes_of_setup(s):
    ss = s["space_schemes"]
    name = lambda f: None if f is None else f.__name__  # noqa: E731
    return dict(reconstructor=name(ss["reconstructor"]), slope_limiter=name(ss.get("slope_limiter")),
                riemann_solver=name(ss.get("riemann_solver")))
