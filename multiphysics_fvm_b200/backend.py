"""Setup dict -> device simulation handle.

A setup (the reference's plugin surface, e.g. setups/kelvin_helmholtz.py:154-163)
selects its physics module, integrator, space schemes and boundary conditions
as Python callables.  This module maps those callables - this package's own or
the reference's functions of the same name - onto the enums of ``fvm_desc`` and
owns the device handle.  Unknown choices raise ``ValueError`` before anything
is launched, as the reference does (geometry.py:173, boundary_conditions.py:37).
"""
from __future__ import annotations

import ctypes as C
import math
from collections import OrderedDict

import numpy as np

from . import _lib as L

VARIABLES = {
    "navier_stokes": ("mass_density", "momentum_x1", "momentum_x2", "momentum_x3", "energy_density"),
    "heat": ("internal_energy_density",),
    "maxwell": ("magnetic_field_x1", "magnetic_field_x2", "magnetic_field_x3",
                "electric_d_field_x1", "electric_d_field_x2", "electric_d_field_x3"),
}
PHYSICS_ID = {"navier_stokes": L.NAVIER_STOKES, "heat": L.HEAT, "maxwell": L.MAXWELL}
COORDS = {"cartesian": L.CARTESIAN, "cylindrical": L.CYLINDRICAL, "spherical": L.SPHERICAL}
SIDES = ("left", "right", "bottom", "top", "front", "back")

# kind -> (module basename, {function name: enum})
SCHEMES = {
    "riemann_solver": ("riemann_solvers", {"rusanov": L.RUSANOV, "hll": L.HLL}),
    "reconstructor": ("reconstructors", {"piecewise_constant": L.PIECEWISE_CONSTANT, "muscl": L.MUSCL}),
    "slope_limiter": ("slope_limiters", {"minmod": L.MINMOD, "monotonized_central": L.MONOTONIZED_CENTRAL,
                                         "van_leer": L.VAN_LEER}),
    "diffusive_solver": ("diffusive_solvers", {"centered": 0}),
    "time_integrator": ("time_integrators", {"euler_explicit": L.EULER_EXPLICIT, "rk3": L.RK3,
                                             "rk3_ssp": L.RK3_SSP, "rk4": L.RK4}),
    "boundary_condition": ("boundary_conditions", {"periodic": L.BC_PERIODIC, "neumann": L.BC_NEUMANN,
                                                   "reflecting": L.BC_REFLECTING}),
}


def scheme_id(kind: str, fn):
    """Enum of a scheme callable: this package's callables carry ``_fvm_id``;
    the reference's are recognised by module and function name."""
    fid = getattr(fn, "_fvm_id", None)
    if fid is not None and fid[0] == kind:
        return fid[1]
    mod, table = SCHEMES[kind]
    name = getattr(fn, "__name__", None)
    modname = (getattr(fn, "__module__", "") or "").split(".")[-1]
    if name in table and modname == mod:
        return table[name]
    raise ValueError(f"Unknown {kind.replace('_', ' ')}: {fn!r}")


def physics_name(module) -> str:
    """'navier_stokes' | 'heat' | 'maxwell' for a physics module (ours or the reference's)."""
    name = getattr(module, "PHYSICS", None) or (getattr(module, "__name__", "") or "").split(".")[-1]
    if name not in PHYSICS_ID:
        raise ValueError(f"Unknown physics module: {module!r}")
    return name


def physics_params(name: str, p: dict) -> list[float]:
    """Ordered parameters of fvm_desc.params (include/fvm.h)."""
    if name == "navier_stokes":
        g = p["gravitational_acceleration"]
        return [p["heat_capacity_ratio"], p["dynamic_viscosity"], g[0], g[1], g[2]]
    if name == "heat":
        return [p["mass_density"], p["specific_heat_capacity"], p["thermal_conductivity"],
                p["volumetric_heat_source"]]
    return [p["magnetic_permeability"], p["electric_permittivity"], p["electrical_conductivity"],
            p["charge_density"], p["magnetic_cleaning_coeff"], p["electric_cleaning_coeff"]]


def bc_codes(name: str, bcs: dict):
    """[var][side] -> (kind, value) for every variable of the physics."""
    out = []
    for var in VARIABLES[name]:
        per = bcs[var]
        row = []
        for side in SIDES:
            fid = scheme_id("boundary_condition", per[side])
            row.append(fid if isinstance(fid, tuple) else (fid, 0.0))
        out.append(row)
    return out


def _key(x):
    if isinstance(x, dict):
        return tuple(sorted((k, _key(v)) for k, v in x.items()))
    if isinstance(x, (list, tuple)):
        return tuple(_key(v) for v in x)
    if callable(x):
        return (getattr(x, "__module__", None), getattr(x, "__name__", None), getattr(x, "_fvm_id", None))
    return x


class Simulation:
    """One device-resident simulation (an ``fvm_handle``).

    State arrays cross the boundary in the reference's layout: float64,
    ``(NV, nx1+2, nx2+2, nx3+2)`` with one ghost layer.
    """

    def __init__(self, physics: str, coordinate_system: str, grid_config: dict, params: dict,
                 space_schemes: dict, bcs: dict, integrator=None, precision: str = "fp64",
                 zchunk: int = 0, tile_ty: int = 0):
        lib = L.load()
        d = self._describe(physics, coordinate_system, grid_config, params, space_schemes, bcs, integrator,
                           precision, zchunk, tile_ty)
        h = C.c_void_p()
        L.check(lib.fvm_create(C.byref(d), C.byref(h)), "fvm_create")
        self._attach(h, lib, owned=True)

    def _describe(self, physics, coordinate_system, grid_config, params, space_schemes, bcs, integrator,
                  precision, zchunk, tile_ty):
        self.physics = physics
        self.nv = len(VARIABLES[physics])
        self.variables = VARIABLES[physics]
        self.n = (int(grid_config["nx1"]), int(grid_config["nx2"]), int(grid_config["nx3"]))
        if coordinate_system not in COORDS:
            raise ValueError(f"Unknown coordinate system: '{coordinate_system}'. "
                             "Expected one of: cartesian, cylindrical, spherical.")
        if precision not in ("fp32", "fp64"):
            raise ValueError(f"Unknown precision {precision!r} (fp32 or fp64)")
        d = L.FvmDesc()
        d.physics = PHYSICS_ID[physics]
        d.precision = L.FP64 if precision == "fp64" else L.FP32
        d.coords = COORDS[coordinate_system]
        d.nx1, d.nx2, d.nx3 = self.n
        for ax in (1, 2, 3):
            setattr(d, f"x{ax}_min", float(grid_config[f"x{ax}_min"]))
            setattr(d, f"x{ax}_max", float(grid_config[f"x{ax}_max"]))
        d.reconstructor = scheme_id("reconstructor", space_schemes["reconstructor"])
        lim = space_schemes.get("slope_limiter")
        d.limiter = scheme_id("slope_limiter", lim) if lim is not None else L.MINMOD
        if physics != "heat":
            d.riemann = scheme_id("riemann_solver", space_schemes["riemann_solver"])
        if physics != "maxwell" and "diffusive_solver" in space_schemes:
            scheme_id("diffusive_solver", space_schemes["diffusive_solver"])
        d.integrator = scheme_id("time_integrator", integrator) if integrator is not None else L.RK3_SSP
        for q, row in enumerate(bc_codes(physics, bcs)):
            for s, (kind, value) in enumerate(row):
                d.bc_kind[q][s] = kind
                d.bc_value[q][s] = float(value)
        for i, v in enumerate(physics_params(physics, params)):
            d.params[i] = float(v)
        d.zchunk = int(zchunk)
        d.tile_ty = int(tile_ty)
        self.desc = d
        self.precision = precision
        return d

    def _attach(self, h, lib, owned):
        self._h = h
        self._lib = lib
        self._owned = owned
        self._ghosted = (self.nv,) + tuple(x + 2 for x in self.n)

    # -- life cycle --------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value and getattr(self, "_owned", True):
            self._lib.fvm_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @classmethod
    def from_setup(cls, setup: dict, **kw):
        name = physics_name(setup["physics"])
        return cls(name, setup["coordinate_system"], setup["grid_config"], setup["physical_parameters"],
                   setup["space_schemes"], setup["boundary_conditions"], setup.get("time_integrator"),
                   precision=setup.get("precision", "fp64"), **kw)

    # -- state transfer ----------------------------------------------------
    def _stack(self, U) -> np.ndarray:
        if isinstance(U, dict):
            arr = np.stack([np.asarray(U[k], dtype=np.float64) for k in self.variables])
        else:
            arr = np.asarray(U, dtype=np.float64)
        if arr.shape != self._ghosted:
            raise ValueError(f"state shape {arr.shape} != {self._ghosted}")
        return np.ascontiguousarray(arr)

    def upload(self, U):
        arr = self._stack(U)
        L.check(self._lib.fvm_upload(self._h, L.dptr(arr)), "fvm_upload")

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self._ghosted, dtype=np.float64)
        L.check(self._lib.fvm_download(self._h, L.dptr(out)), "fvm_download")
        return out

    def upload_async(self, U: np.ndarray):
        """Enqueue the upload of a ghosted float64 state (NV, nx1+2, nx2+2,
        nx3+2); ``U`` (pinned for a truly asynchronous copy) must stay alive and
        unchanged until ``synchronize``."""
        if U.shape != self._ghosted or U.dtype != np.float64 or not U.flags.c_contiguous:
            raise ValueError(f"state must be C-contiguous float64 of shape {self._ghosted}")
        L.check(self._lib.fvm_upload_async(self._h, L.dptr(U)), "fvm_upload_async")

    def download_async(self, out: np.ndarray):
        """Enqueue the download of the state into ``out`` (valid after ``synchronize``)."""
        if out.shape != self._ghosted or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError(f"output must be C-contiguous float64 of shape {self._ghosted}")
        L.check(self._lib.fvm_download_async(self._h, L.dptr(out)), "fvm_download_async")

    def step_async(self, n_steps: int = 1):
        """Enqueue n_steps CFL steps without waiting for them."""
        L.check(self._lib.fvm_step_async(self._h, int(n_steps), 0), "fvm_step_async")

    def synchronize(self):
        L.check(self._lib.fvm_synchronize(self._h), "fvm_synchronize")

    def download_into(self, U: dict):
        arr = self.download()
        for q, k in enumerate(self.variables):
            U[k][...] = arr[q]

    def init_kelvin_helmholtz(self, ics: dict, seed: int):
        """Write the sharp Kelvin-Helmholtz state of setups/kelvin_helmholtz_sharp
        on the device (``ics`` = its initial_conditions parameters); the noise is
        a counter-based draw, not NumPy's."""
        keys = ("rho_inner", "rho_outer", "shear_velocity", "pressure", "amplitude", "wavenumber", "noise", "phase")
        prm = np.array([float(ics.get(k, 0.0)) for k in keys] + [1.0 if ics.get("noise_all") else 0.0])
        L.check(self._lib.fvm_init_kelvin_helmholtz(self._h, L.dptr(prm), C.c_ulonglong(int(seed))),
                "fvm_init_kelvin_helmholtz")

    # -- hot path ------------------------------------------------------------
    def residual(self) -> np.ndarray:
        out = np.empty((self.nv,) + self.n, dtype=np.float64)
        L.check(self._lib.fvm_residual(self._h, L.dptr(out)), "fvm_residual")
        return out

    def compute_dt(self, cfl: float) -> float:
        dt = C.c_double()
        L.check(self._lib.fvm_compute_dt(self._h, float(cfl), C.byref(dt)), "fvm_compute_dt")
        return dt.value

    def set_time(self, t: float = 0.0, t_end: float = math.inf, cfl: float = 0.4):
        L.check(self._lib.fvm_set_time(self._h, float(t), float(t_end), float(cfl)), "fvm_set_time")

    def step(self, n_steps: int = 1, dt: float | None = None):
        """Advance n_steps; dt=None uses the device CFL step (fvm_set_time's cfl)."""
        if dt is not None:
            L.check(self._lib.fvm_set_dt(self._h, float(dt)), "fvm_set_dt")
        L.check(self._lib.fvm_step(self._h, int(n_steps), 0 if dt is None else 1), "fvm_step")

    def time_steps(self, n_steps: int, fixed_dt: bool = False) -> float:
        ms = C.c_double()
        L.check(self._lib.fvm_time_steps(self._h, int(n_steps), 1 if fixed_dt else 0, C.byref(ms)),
                "fvm_time_steps")
        return ms.value

    def profile_steps(self, n_steps: int, fixed_dt: bool = False):
        st, ot, nl = C.c_double(), C.c_double(), C.c_int()
        L.check(self._lib.fvm_profile_steps(self._h, int(n_steps), 1 if fixed_dt else 0, C.byref(st),
                                            C.byref(ot), C.byref(nl)), "fvm_profile_steps")
        return st.value, ot.value, nl.value

    def time(self):
        t, dt, n = C.c_double(), C.c_double(), C.c_longlong()
        L.check(self._lib.fvm_get_time(self._h, C.byref(t), C.byref(n), C.byref(dt)), "fvm_get_time")
        return t.value, n.value, dt.value

    def totals(self) -> np.ndarray:
        nt = self.nv + (1 if self.physics == "maxwell" else 0)
        out = np.zeros(8, dtype=np.float64)
        L.check(self._lib.fvm_totals(self._h, L.dptr(out)), "fvm_totals")
        return out[:nt]

    def status(self) -> int:
        s = C.c_uint()
        L.check(self._lib.fvm_status(self._h, C.byref(s)), "fvm_status")
        return s.value

    def clear_status(self):
        L.check(self._lib.fvm_clear_status(self._h), "fvm_clear_status")

    def set_wait_limit(self, ns: int, never_complete: bool = False):
        """Limit (ns) of each wait of the stage kernels for a TMA plane; a wait
        that runs out sets the timeout status bit and the step returns.
        ``never_complete`` (tests of that path) makes every ring copy expect
        more bytes than it delivers, so every ring wait runs out."""
        L.check(self._lib.fvm_set_wait_limit(self._h, C.c_ulonglong(int(ns)), 1 if never_complete else 0),
                "fvm_set_wait_limit")

    def step_launches(self, dt_mode: int = 0) -> int:
        """Kernel launches of one step: CFL reduction, ghost fills, stage kernels."""
        n = C.c_int()
        L.check(self._lib.fvm_step_launches(self._h, int(dt_mode), C.byref(n)), "fvm_step_launches")
        return n.value

    def autotune(self):
        """Choose the z-march depth by timing candidates (state restored); returns (zchunk, ms/step)."""
        z, ms = C.c_int(), C.c_double()
        L.check(self._lib.fvm_autotune(self._h, C.byref(z), C.byref(ms)), "fvm_autotune")
        return z.value, ms.value

    def tiling(self):
        """(tile rows, z-march depth) the stage kernels run with."""
        ty, z = C.c_int(), C.c_int()
        L.check(self._lib.fvm_tiling(self._h, C.byref(ty), C.byref(z)), "fvm_tiling")
        return ty.value, z.value

    def info(self):
        nv, nb = C.c_int(), C.c_longlong()
        L.check(self._lib.fvm_info(self._h, C.byref(nv), C.byref(nb)), "fvm_info")
        return nv.value, nb.value


class Batch:
    """Independent grids advanced together by one persistent launch per kernel
    specialisation and stage (``fvm_batch_*``); each grid keeps its own CFL dt.
    ``setups`` are setup dicts (same integrator and precision; navier_stokes and
    heat may be mixed).  ``batch[i]`` is the i-th grid as a Simulation view."""

    def __init__(self, setups, heat_tile_rows: int = 0):
        """``heat_tile_rows``: 10 puts the heat grids of a one-launch (mixed)
        batch on 10-row tiles instead of 20 (``autotune`` times both)."""
        lib = L.load()
        descs = (L.FvmDesc * len(setups))()
        self.sims = []
        for i, s in enumerate(setups):
            sim = Simulation.__new__(Simulation)
            name = physics_name(s["physics"])
            descs[i] = sim._describe(name, s["coordinate_system"], s["grid_config"],
                                     s["physical_parameters"], s["space_schemes"], s["boundary_conditions"],
                                     s.get("time_integrator"), s.get("precision", "fp64"), 0,
                                     heat_tile_rows if name == "heat" else 0)
            self.sims.append(sim)
        b = C.c_void_p()
        L.check(lib.fvm_batch_create(descs, len(setups), C.byref(b)), "fvm_batch_create")
        self._b, self._lib = b, lib
        for i, sim in enumerate(self.sims):
            h = C.c_void_p()
            L.check(lib.fvm_batch_handle(b, i, C.byref(h)), "fvm_batch_handle")
            sim._attach(h, lib, owned=False)

    def __len__(self):
        return len(self.sims)

    def __getitem__(self, i) -> Simulation:
        return self.sims[i]

    def tiles(self) -> int:
        n, t = C.c_int(), C.c_longlong()
        L.check(self._lib.fvm_batch_size(self._b, C.byref(n), C.byref(t)), "fvm_batch_size")
        return t.value

    def launches_per_stage(self) -> int:
        """Kernel launches per Runge-Kutta stage (1 for a mixed
        navier_stokes + heat batch that runs as one launch)."""
        k = C.c_int()
        L.check(self._lib.fvm_batch_launches(self._b, C.byref(k)), "fvm_batch_launches")
        return k.value

    def step(self, n_steps: int = 1, fixed_dt: bool = False):
        L.check(self._lib.fvm_batch_step(self._b, int(n_steps), 1 if fixed_dt else 0), "fvm_batch_step")

    def time_steps(self, n_steps: int, fixed_dt: bool = False) -> float:
        ms = C.c_double()
        L.check(self._lib.fvm_batch_time_steps(self._b, int(n_steps), 1 if fixed_dt else 0, C.byref(ms)),
                "fvm_batch_time_steps")
        return ms.value

    def autotune(self):
        z, ms = C.c_int(), C.c_double()
        L.check(self._lib.fvm_batch_autotune(self._b, C.byref(z), C.byref(ms)), "fvm_batch_autotune")
        return z.value, ms.value

    def close(self):
        if getattr(self, "_b", None) is not None and self._b.value:
            for s in self.sims:
                s._h = None
            self._lib.fvm_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Cache:
    """Small LRU of simulations for the functional drop-in API (compute_rhs,
    compute_dt, integrators), keyed by everything that shapes the handle."""

    def __init__(self, size=4):
        self.size = size
        self.d: OrderedDict = OrderedDict()

    def get(self, key, make):
        if key in self.d:
            self.d.move_to_end(key)
            return self.d[key]
        sim = make()
        self.d[key] = sim
        while len(self.d) > self.size:
            _, old = self.d.popitem(last=False)
            old.close()
        return sim


CACHE = _Cache()


def cached_simulation(physics: str, grid: dict, params: dict, space_schemes: dict, bcs=None,
                      integrator=None, precision: str | None = None) -> Simulation:
    cs = grid.get("coordinate_system")
    if cs is None:
        raise ValueError("grid dict lacks 'coordinate_system': build it with multiphysics_fvm_b200.grid.geometry.build_grid")
    prec = precision or grid.get("precision", "fp64")
    if bcs is None:  # residual-only use: any valid BC set
        from .grid import boundary_conditions as bcm
        bcs = {v: {s: bcm.periodic for s in SIDES} for v in VARIABLES[physics]}
    key = (physics, cs, _key(grid["config"]), _key(params), _key(space_schemes), _key(bcs), _key(integrator), prec)
    return CACHE.get(key, lambda: Simulation(physics, cs, grid["config"], params, space_schemes, bcs,
                                             integrator, precision=prec))
