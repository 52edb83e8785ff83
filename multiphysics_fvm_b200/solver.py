"""Device-resident driver (reference: src/solver.py).

``run(setup)`` keeps the state on the GPU for the whole time loop: the grid's
metric tables, the ghost fill, the CFL reduction and the stage kernels all
run on the device, every step is one CUDA graph launch, and the state is
copied to the host only at output steps (``n % output_frequency == 0``, after
the step, labelled with the pre-step time as in src/solver.py:146-148).

Extensions of the setup schema: ``time_config["n_steps"]`` (step-counted run,
``t_end`` ignored), ``setup["precision"]`` ("fp32" | "fp64", default "fp64"),
``setup["restart_from"]`` (a snapshot written by ``io.save_snapshot`` through
this loop: the state, its time and the step count are taken from it instead of
the initial conditions; ``n_steps`` stays the total of the whole run, and the
output steps and labels continue the numbering of the interrupted run).
"""
from __future__ import annotations

import inspect
import math


from . import backend
from . import io
from .grid import geometry


def apply_bcs(U: dict, bcs: dict) -> None:
    """Fill ghost faces of every variable from ``bcs`` and average ghost edges
    and corners (src/solver.py:13-61), on the device (upload, ghost fill,
    download into ``U``)."""
    keys = tuple(U.keys())
    physics = next((p for p, v in backend.VARIABLES.items() if set(v) == set(keys)), None)
    if physics is None:
        raise ValueError(f"cannot tell the physics of state variables {keys}")
    shape = next(iter(U.values())).shape
    cfg = {"nx1": shape[0] - 2, "nx2": shape[1] - 2, "nx3": shape[2] - 2,
           "x1_min": 1.0, "x1_max": 2.0, "x2_min": 1.0, "x2_max": 2.0, "x3_min": 1.0, "x3_max": 2.0}
    grid = {"config": cfg, "coordinate_system": "cartesian"}
    from .physics._common import _DEFAULT_SCHEMES
    params = {"navier_stokes": {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 0.0,
                                "gravitational_acceleration": [0.0, 0.0, 0.0]},
              "heat": {"mass_density": 1.0, "specific_heat_capacity": 1.0, "thermal_conductivity": 1.0,
                       "volumetric_heat_source": 0.0},
              "maxwell": {"magnetic_permeability": 1.0, "electric_permittivity": 1.0,
                          "electrical_conductivity": 0.0, "charge_density": 0.0,
                          "magnetic_cleaning_coeff": 0.0, "electric_cleaning_coeff": 0.0}}[physics]
    sim = backend.cached_simulation(physics, grid, params, _DEFAULT_SCHEMES, bcs)
    sim.upload(U)
    sim.download_into(U)


def apply_ics(U: dict, params: dict, grid: dict, ics: dict) -> None:
    """Run the setup's initializer on the host state (src/solver.py:64-85)."""
    ics["initializer"](U, params, grid, ics["parameters"])


def _attach_closure(sim, spec):
    """Optional learned flux correction: ``setup["closure"] = {"weights": path
    or closure.Closure, "beta": 0.05, "fct": False}`` (navier_stokes, fp32,
    cartesian, periodic, rk3_ssp or euler_explicit).  ``beta`` and ``fct`` are
    optional: by default they are the values stored with the weights (the
    ones the network was selected with)."""
    if not spec:
        return
    from . import closure
    net = spec["weights"]
    if not isinstance(net, closure.Closure):
        net = closure.Closure(sim.n)
        net.load(spec["weights"])
    fct = spec.get("fct", net.meta.get("fct"))
    if fct is not None:
        net.set_limiter(bool(fct))
    beta = spec.get("beta")
    net.attach(sim, beta=None if beta is None else float(beta))


def _advance(sim, k: int) -> int:
    """Step up to ``k`` times; returns the steps taken (fewer once t > t_end)."""
    before = sim.time()[1]
    sim.step(k)
    return sim.time()[1] - before


def _accepts(fn, name: str) -> bool:
    try:
        return name in inspect.signature(fn).parameters
    except (TypeError, ValueError):
        return False


def run(setup: dict, verbose: bool = True):
    """Run a setup (src/solver.py:88-151) with the state resident on the device.
    Returns the Simulation (its final state via ``download()``)."""
    physics = setup["physics"]
    params = setup["physical_parameters"]
    tc = setup["time_config"]
    t_start, cfl = float(tc["t_start"]), float(tc["CFL"])
    n_steps = tc.get("n_steps")
    t_end = math.inf if n_steps is not None else float(tc["t_end"])
    save = setup.get("save_config") or {}
    saver = save.get("saver")
    out_freq = int(save.get("output_frequency", 0) or 0)
    U = physics.allocate_u(setup["grid_config"])
    n = 0
    if setup.get("restart_from"):
        t_start, n = io.restore_snapshot(setup["restart_from"], setup, U)
    else:
        grid = geometry.build_grid(setup["coordinate_system"], setup["grid_config"])
        apply_ics(U, params, grid, setup["initial_conditions"])
    sim = backend.Simulation.from_setup(setup)
    sim.upload(U)
    sim.set_time(t_start, t_end, cfl)
    _attach_closure(sim, setup.get("closure"))
    limit = n_steps if n_steps is not None else None
    takes_state_time = saver is not None and _accepts(saver, "state_time")
    while limit is None or n < limit:
        # Steps up to and including the next output step (step index k with
        # k % out_freq == 0, i.e. the step after which n == k + 1).
        if out_freq > 0:
            chunk = (1 - n) % out_freq or out_freq
        else:
            chunk = 1000 if limit is None else limit - n
        if limit is not None:
            chunk = min(chunk, limit - n)
        save_due = out_freq > 0 and (n + chunk - 1) % out_freq == 0
        if save_due and chunk > 1:  # stop before the output step to read its start time
            taken = _advance(sim, chunk - 1)
            n += taken
            if taken < chunk - 1:  # t passed t_end
                break
            chunk = 1
        t_pre = sim.time()[0]
        taken = _advance(sim, chunk)
        n += taken
        if save_due and taken == chunk:
            t, _, dt = sim.time()
            if verbose:
                pct = 100 * t_pre / t_end if math.isfinite(t_end) else 100 * n / max(limit or 1, 1)
                print(f"n = {n - 1:6d} | t = {t_pre:.2f}/{t_end:.2f} | dt = {dt:.2e} | {pct:.1f}%")
            if saver is not None:
                sim.download_into(U)
                extra = {"state_time": t} if takes_state_time else {}
                saver(U, setup, t_pre, n - 1, save.get("directory", "."), **extra)
        if taken < chunk:  # t passed t_end inside the chunk
            break
    status = sim.status()
    if status:
        raise FloatingPointError(f"device status word {status:#x} (NaN/Inf, rho<=0, P<=0 or bad dt)")
    return sim
