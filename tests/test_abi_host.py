"""CPU-side checks: the C-ABI library loads and exports every declared entry
point, the ctypes descriptor matches the header, and the setup -> descriptor
mapping accepts this package's and the reference's callables and rejects
unknown ones (no GPU work is launched here)."""
import ctypes
import os
import re
import subprocess
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fvm.h")
HEADERS = sorted(os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
                 if f.endswith(".h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        names |= set(re.findall(r"^int\s+(fvm_\w+)\s*\(", open(h).read(), flags=re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from multiphysics_fvm_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert {n for n, _, _ in _lib.SIGNATURES} == set(names)


def test_descriptor_layout_matches_header(tmp_path):
    from multiphysics_fvm_b200 import _lib
    c = tmp_path / "sz.c"
    c.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "fvm.h"\n'
                 'int main(){printf("%zu %zu %zu %zu\\n", sizeof(fvm_desc), offsetof(fvm_desc, bc_kind),'
                 ' offsetof(fvm_desc, params), offsetof(fvm_desc, zchunk));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    D = _lib.FvmDesc
    assert [int(x) for x in out] == [ctypes.sizeof(D), D.bc_kind.offset, D.params.offset, D.zchunk.offset]


def test_last_error_roundtrip():
    from multiphysics_fvm_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    d = _lib.FvmDesc()
    d.physics = 7  # unknown physics: rejected before any CUDA call
    assert lib.fvm_create(ctypes.byref(d), ctypes.byref(h)) == -1
    assert "physics" in _lib.last_error()
    d.physics = 0
    d.nx1 = d.nx2 = d.nx3 = 4
    d.coords = 5
    assert lib.fvm_create(ctypes.byref(d), ctypes.byref(h)) == -1
    assert "coordinate system" in _lib.last_error()


def _valid_desc():
    from multiphysics_fvm_b200 import _lib
    d = _lib.FvmDesc()
    d.physics, d.precision, d.coords = 0, 0, 0
    d.nx1 = d.nx2 = d.nx3 = 8
    d.x1_max = d.x2_max = d.x3_max = 1.0
    d.reconstructor, d.limiter, d.riemann, d.integrator = 1, 0, 1, 2
    d.params[0] = 1.4
    return d


@pytest.mark.parametrize("field,value,message", [
    ("precision", 7, "precision"),
    ("nx2", 0, "grid sizes"),
    ("nx1", 1 << 20, "grid too large"),
    ("reconstructor", 2, "reconstructor"),
    ("limiter", 3, "slope limiter"),
    ("riemann", 2, "riemann"),
    ("integrator", 4, "time integrator"),
    ("tile_ty", 5, "tile_ty"),
    ("bc", 4, "Unknown boundary condition"),
    ("periodic_one_side", 1, "both sides"),
])
def test_descriptor_rules_rejected_before_any_cuda_call(field, value, message):
    """fvm_create validates the descriptor first, so each rule is checked on
    the CPU: the call returns FVM_E_INVALID (-1) and fvm_last_error names it."""
    from multiphysics_fvm_b200 import _lib
    lib = _lib.load()
    d = _valid_desc()
    if field == "nx1":
        d.nx1 = d.nx2 = d.nx3 = value
    elif field == "bc":
        d.bc_kind[0][0] = value
    elif field == "periodic_one_side":
        d.bc_kind[2][2] = value  # neumann on the low x2 side, periodic on the high one
    else:
        setattr(d, field, value)
    h = ctypes.c_void_p()
    assert lib.fvm_create(ctypes.byref(d), ctypes.byref(h)) == -1
    assert message in _lib.last_error()
    assert not h.value


def test_scheme_ids_accept_package_and_reference_callables():
    from multiphysics_fvm_b200 import backend, _lib as L
    from multiphysics_fvm_b200.numerics import riemann_solvers, slope_limiters, time_integrators
    from multiphysics_fvm_b200.grid import boundary_conditions as bc
    assert backend.scheme_id("riemann_solver", riemann_solvers.hll) == L.HLL
    assert backend.scheme_id("slope_limiter", slope_limiters.monotonized_central) == L.MONOTONIZED_CENTRAL
    assert backend.scheme_id("time_integrator", time_integrators.rk3) == L.RK3
    assert backend.scheme_id("boundary_condition", bc.dirichlet(1.5)) == (L.BC_DIRICHLET, 1.5)

    # a function named like the reference's, in a module named like the reference's
    mod = types.ModuleType("src.numerics.riemann_solvers")
    exec("def rusanov(*a):\n    pass\n", mod.__dict__)
    mod.rusanov.__module__ = "src.numerics.riemann_solvers"
    assert backend.scheme_id("riemann_solver", mod.rusanov) == L.RUSANOV
    with pytest.raises(ValueError):
        backend.scheme_id("riemann_solver", lambda *a: None)
    with pytest.raises(ValueError):
        backend.physics_name(types.ModuleType("src.physics.mhd"))
    pm = types.ModuleType("src.physics.maxwell")
    assert backend.physics_name(pm) == "maxwell"


def test_selectors_refuse_host_calls():
    from multiphysics_fvm_b200.numerics import slope_limiters
    with pytest.raises(TypeError):
        slope_limiters.minmod(1.0, 2.0)


def test_conducting_wall_bc_set():
    from multiphysics_fvm_b200.grid import boundary_conditions as bc
    from multiphysics_fvm_b200.backend import VARIABLES
    w = bc.conducting_wall(VARIABLES["maxwell"], 0)
    assert w["electric_d_field_x1"] is bc.neumann and w["electric_d_field_x2"] is bc.reflecting
    assert w["magnetic_field_x1"] is bc.reflecting and w["magnetic_field_x3"] is bc.neumann


def test_lazy_grid_matches_oracle_geometry():
    import numpy as np
    from multiphysics_fvm_b200.grid.geometry import build_grid
    from oracle import fvm_oracle as O
    cfg = dict(x1_min=0.1, x1_max=1.0, x2_min=0.2, x2_max=2.9, x3_min=0.0, x3_max=1.0, nx1=5, nx2=4, nx3=3)
    for cs in ("cartesian", "cylindrical", "spherical"):
        g = build_grid(cs, cfg)
        o = O.Geometry(cs, cfg)
        assert np.array_equal(g["cell"]["geometry"]["volume"], o.V)
        for a, k in enumerate(("x1", "x2", "x3")):
            assert np.array_equal(g["cell"]["geometry"]["surface"][k], o.S[a])
            assert np.array_equal(g["cell"]["geometry"]["length"][k], o.L[a])
        assert g["cell"]["coordinates"]["x1"].shape == (5, 4, 3)
