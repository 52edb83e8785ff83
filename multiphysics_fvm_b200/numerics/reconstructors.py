"""Interface reconstructors (reference: src/numerics/reconstructors.py)."""
from .. import _lib as L
from ._selector import selector

piecewise_constant = selector("reconstructor", "piecewise_constant", L.PIECEWISE_CONSTANT,
                              "First-order face states f_i, f_{i+1} (reconstructors.py:13-64).")
muscl = selector("reconstructor", "muscl", L.MUSCL,
                 "MUSCL: slope = limiter(bwd/L, fwd/L)*L, zero on ghosts (reconstructors.py:67-158).")
