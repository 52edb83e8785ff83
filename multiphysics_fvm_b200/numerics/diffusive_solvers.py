"""Diffusive solvers (reference: src/numerics/diffusive_solvers.py)."""
from ._selector import selector

centered = selector("diffusive_solver", "centered", 0, "Centred flux (Fd_L + Fd_R)/2 (diffusive_solvers.py:11-30).")
