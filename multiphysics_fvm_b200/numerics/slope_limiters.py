"""Slope limiters (reference: src/numerics/slope_limiters.py)."""
from .. import _lib as L
from ._selector import selector

minmod = selector("slope_limiter", "minmod", L.MINMOD, "Minmod (slope_limiters.py:13-39).")
monotonized_central = selector(
    "slope_limiter", "monotonized_central", L.MONOTONIZED_CENTRAL,
    "Monotonized central with the reference's three-sign test (slope_limiters.py:42-73): "
    "nonzero, +-1/3 min(...), for slopes of opposite sign.")
van_leer = selector("slope_limiter", "van_leer", L.VAN_LEER, "Van Leer harmonic mean (slope_limiters.py:76-105).")
