"""fvm_totals_noalloc: the conserved-totals reduction for callers that cannot
allocate device memory (their host framework owns every allocation, or
allocation is forbidden once the run has started).  It keeps its partial sums
in a fixed array inside the library instead of a handle's buffer.

Checked through the C ABI against the regular entry point (fvm_totals on a
handle holding the same float32 state) on two calls in a row with different
states, so a second call cannot reuse what the first left in the shared array.
Tolerance: 1e-12 relative, as for the other float64 reductions.  This file is
collected last so that a run stopping at the first failure has run every other
test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from tests.helpers import bcs_dict, random_ns_state

pytestmark = pytest.mark.gpu


def _geometry_volumes(n, lo_hi):
    dl = []
    for a in range(3):
        lo, hi = lo_hi[a]
        d = (hi - lo) / n[a]
        xf = lo + np.arange(n[a] + 1) * d
        dl.append(xf[1:] - xf[:-1])
    return (dl[0][:, None, None] * dl[1][None, :, None]) * dl[2][None, None, :]


def test_totals_noalloc_matches_handle_totals():
    import torch
    from multiphysics_fvm_b200 import _lib
    from multiphysics_fvm_b200.backend import Simulation
    from multiphysics_fvm_b200.numerics import reconstructors, riemann_solvers, slope_limiters

    lib = _lib.load()
    n = (20, 18, 14)
    lo_hi = ((0.0, 1.0), (0.0, 0.8), (0.0, 0.6))
    cfg = dict(x1_min=0.0, x1_max=1.0, x2_min=0.0, x2_max=0.8, x3_min=0.0, x3_max=0.6,
               nx1=n[0], nx2=n[1], nx3=n[2])
    prm = {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 0.0, "gravitational_acceleration": [0, 0, 0]}
    sch = {"reconstructor": reconstructors.muscl, "slope_limiter": slope_limiters.minmod,
           "riemann_solver": riemann_solvers.hll}
    sim = Simulation("navier_stokes", "cartesian", cfg, prm, sch, bcs_dict("navier_stokes", [["periodic"] * 6] * 5),
                     precision="fp32")
    V = _geometry_volumes(n, lo_hi)
    vol = torch.tensor(V.reshape(-1), dtype=torch.float64, device="cuda")
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    for seed in (1, 2):  # two calls in a row on different states
        U = random_ns_state(tuple(x + 2 for x in n), np.random.default_rng(seed))
        sim.upload(U)
        expect = sim.totals()
        interior = U[:, 1:-1, 1:-1, 1:-1].astype(np.float32)  # the values the device state holds
        cells = torch.tensor(interior.reshape(5, -1), device="cuda")
        out.zero_()
        rc = lib.fvm_totals_noalloc(ctypes.c_void_p(cells.data_ptr()), ctypes.c_void_p(vol.data_ptr()), 5,
                                    ctypes.c_longlong(cells.shape[1]), ctypes.c_void_p(out.data_ptr()), None)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()[:5]
        np.testing.assert_allclose(got, expect, rtol=1e-12, atol=0.0)
    sim.close()


def test_totals_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from multiphysics_fvm_b200 import _lib
    lib = _lib.load()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    cells = torch.zeros(16, dtype=torch.float32, device="cuda")
    rc = lib.fvm_totals_noalloc(ctypes.c_void_p(cells.data_ptr()), ctypes.c_void_p(buf.data_ptr()), 9,
                                ctypes.c_longlong(1), ctypes.c_void_p(buf.data_ptr()), None)
    assert rc == -1 and "nvars" in _lib.last_error()


def test_totals_noalloc_full_scratch_against_numpy():
    """80^3 cells (more than 1024 blocks of 256, so the grid-stride loop runs)
    and nvars = 8 (every column of a scratch row), twice in a row, against a
    float64 NumPy sum: relative <= 1e-12 of the sum of magnitudes."""
    import torch
    from multiphysics_fvm_b200 import _lib
    lib = _lib.load()
    n = 80 ** 3
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    for seed in (3, 4):
        rng = np.random.default_rng(seed)
        cells_h = rng.uniform(-1.0, 2.0, (8, n)).astype(np.float32)
        vol_h = rng.uniform(0.5, 1.5, n) * 1e-6
        cells = torch.tensor(cells_h, device="cuda")
        vol = torch.tensor(vol_h, dtype=torch.float64, device="cuda")
        out.fill_(123.0)
        rc = lib.fvm_totals_noalloc(ctypes.c_void_p(cells.data_ptr()), ctypes.c_void_p(vol.data_ptr()), 8,
                                    ctypes.c_longlong(n), ctypes.c_void_p(out.data_ptr()), None)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        c64 = cells_h.astype(np.float64)
        expect = np.sum(c64 * vol_h[None, :], axis=1)
        scale = np.sum(np.abs(c64) * vol_h[None, :], axis=1)
        assert np.all(np.abs(got - expect) <= 1e-12 * scale), (got, expect)
