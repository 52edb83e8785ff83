"""heat physics module (reference: src/physics/heat.py).

A setup selects it with ``setup["physics"] = heat``.  The residual pieces the
reference exposes as separate functions (closure, fluxes, characteristic
speeds, sources) are fused into the device stage kernel; this module exposes
the reference's module-level entry points with the same signatures.
"""
from __future__ import annotations

from . import _common
from ..backend import VARIABLES as _V

PHYSICS = "heat"
VARIABLES = _V[PHYSICS]


def allocate_u(grid_config: dict) -> dict:
    """Zero host state with one ghost layer (src/physics/heat.py:13-37)."""
    return _common.allocate_u(PHYSICS, grid_config)


def compute_rhs(U: dict, grid: dict, params: dict, space_schemes: dict) -> dict:
    """Residual on the interior, computed on the device from U as given
    (ghosts are not refilled) (src/physics/heat.py:354-473)."""
    return _common.compute_rhs(PHYSICS, U, grid, params, space_schemes)


def compute_dt(U: dict, params: dict, grid: dict, cfl: float) -> float:
    """CFL time step, reduced on the device in float64 (src/physics/heat.py:305-351)."""
    return _common.compute_dt(PHYSICS, U, params, grid, cfl)


compute_rhs._fvm_physics = PHYSICS
