"""Riemann solvers (reference: src/numerics/riemann_solvers.py)."""
from .. import _lib as L
from ._selector import selector

rusanov = selector("riemann_solver", "rusanov", L.RUSANOV,
                   "Rusanov flux, speed max|lambda| over waves and sides (riemann_solvers.py:13-48).")
hll = selector("riemann_solver", "hll", L.HLL,
               "HLL flux with three-way selection on the extreme speeds (riemann_solvers.py:51-89).")
