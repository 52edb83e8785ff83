"""Boundary conditions (reference: src/grid/boundary_conditions.py).

Selectors for the per-variable, per-side ``bcs`` dict of a setup.  The ghost
fill itself runs on the device before every stage (bc_fill_kernel), with the
reference's rules: ghost = opposite interior layer (periodic, :58-63),
adjacent interior (neumann, :31-36), minus adjacent interior (reflecting,
:85-90).  ``dirichlet(value)`` is new: ghost = 2*value - adjacent interior, so
the face value is ``value`` (in conserved units, e.g. rho*cp*T_wall for heat).
"""
from __future__ import annotations

from .. import _lib as L
from ..numerics._selector import selector

periodic = selector("boundary_condition", "periodic", L.BC_PERIODIC, "Periodic ghost fill.")
neumann = selector("boundary_condition", "neumann", L.BC_NEUMANN, "Zero-gradient ghost fill.")
reflecting = selector("boundary_condition", "reflecting", L.BC_REFLECTING, "Odd-symmetric ghost fill.")


def dirichlet(value: float):
    """Fixed face value: ghost = 2*value - adjacent interior."""
    return selector("boundary_condition", f"dirichlet({value!r})", (L.BC_DIRICHLET, float(value)),
                    "Dirichlet ghost fill.")


def conducting_wall(variables, normal_axis: int):
    """Perfect-conductor wall for Maxwell expressed with the reference's BC kinds:
    tangential D and normal B odd (reflecting), normal D and tangential B even
    (neumann).  Returns {variable: bc} for a wall normal to ``normal_axis`` (0..2)."""
    out = {}
    for v in variables:
        comp = int(v[-1]) - 1
        normal = comp == normal_axis
        if v.startswith("electric"):
            out[v] = neumann if normal else reflecting
        else:
            out[v] = reflecting if normal else neumann
    return out
