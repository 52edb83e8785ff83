"""Time integrators (reference: src/numerics/time_integrators.py).

Same signature as the reference, ``integrator(rhs, U, dt, params, grid,
space_schemes, bcs, apply_bcs)``; one call advances the host state dict ``U``
in place by one step.  The step runs on the device: the state is uploaded, every
stage applies the ghost fill of ``bcs`` and the fused residual + stage kernel,
and the result is written back into ``U``.  ``apply_bcs`` is accepted for
signature compatibility; the device applies ``bcs`` itself before each stage.
For a device-resident loop without per-step host copies use ``solver.run``.
"""
from __future__ import annotations

from .. import _lib as L
from .. import backend


def _physics_of(rhs) -> str:
    name = getattr(rhs, "_fvm_physics", None)
    if name:
        return name
    mod = (getattr(rhs, "__module__", "") or "").split(".")[-1]
    if mod in backend.PHYSICS_ID:
        return mod
    raise ValueError(f"cannot tell the physics of rhs={rhs!r}")


def _device_step(integrator, rhs, U, dt, params, grid, space_schemes, bcs):
    physics = _physics_of(rhs)
    sim = backend.cached_simulation(physics, grid, params, space_schemes, bcs, integrator)
    sim.upload(U)
    sim.step(1, dt=float(dt))
    sim.download_into(U)


def _make(name, enum, doc):
    def integrator(rhs, U, dt, params, grid, space_schemes, bcs, apply_bcs=None):
        _device_step(integrator, rhs, U, dt, params, grid, space_schemes, bcs)
    integrator.__name__ = integrator.__qualname__ = name
    integrator.__doc__ = doc
    integrator._fvm_id = ("time_integrator", enum)
    return integrator


euler_explicit = _make("euler_explicit", L.EULER_EXPLICIT, "Forward Euler (time_integrators.py:10-47).")
rk3 = _make("rk3", L.RK3, "Three-stage scheme exactly as the reference writes it (time_integrators.py:50-103); "
            "its third stage ignores k1 in the base point, which makes it second order.")
rk3_ssp = _make("rk3_ssp", L.RK3_SSP, "SSPRK3 (time_integrators.py:106-159).")
rk4 = _make("rk4", L.RK4, "Classical RK4 (time_integrators.py:162-221).")
