"""multiphysics_fvm_b200: B200-native finite-volume residual + Runge-Kutta stages.

Drop-in for the hot path of nathanzimniak/multiphysics-fvm: setups keep the
reference's dict schema (physics module, integrator, space schemes, per-variable
per-side BCs, initializer) and ``solver.run(setup)`` advances them on the GPU
through the C ABI of ``libfvm_b200.so`` (include/fvm.h).
"""
from .backend import Simulation  # noqa: F401

__all__ = ["Simulation"]
