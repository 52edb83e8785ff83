"""Grid construction (reference: src/grid/geometry.py:14-194).

``build_grid`` returns the reference's grid dict (coordinates, volumes, face
areas, lengths, Lame coefficients and their log-derivatives) plus the keys
``coordinate_system`` and ``config`` that the device backend reads.  Entries
are computed on first access, so a setup's initializer that only reads cell
coordinates never materialises the other 3D arrays.  The device itself keeps
only 1D per-axis metric tables (built in C++ from the same expressions).
"""
from __future__ import annotations

import numpy as np


class _Lazy(dict):
    """dict whose callable-wrapped values are evaluated on first access."""

    class thunk:
        def __init__(self, f):
            self.f = f

    def __getitem__(self, k):
        v = dict.__getitem__(self, k)
        if isinstance(v, _Lazy.thunk):
            v = v.f()
            dict.__setitem__(self, k, v)
        return v

    def get(self, k, default=None):
        return self[k] if k in self else default


def build_grid(coordinate_system: str, grid_config: dict) -> dict:
    if coordinate_system not in ("cartesian", "cylindrical", "spherical"):
        raise ValueError(f"Unknown coordinate system: '{coordinate_system}'. "
                         "Expected one of: cartesian, cylindrical, spherical.")
    n = [int(grid_config[f"nx{a}"]) for a in (1, 2, 3)]
    lo = [float(grid_config[f"x{a}_min"]) for a in (1, 2, 3)]
    hi = [float(grid_config[f"x{a}_max"]) for a in (1, 2, 3)]
    d = [(hi[a] - lo[a]) / n[a] for a in range(3)]
    xc = [lo[a] + (np.arange(n[a]) + 0.5) * d[a] for a in range(3)]
    xf = [lo[a] + np.arange(n[a] + 1) * d[a] for a in range(3)]
    dl = [xf[a][1:] - xf[a][:-1] for a in range(3)]
    shape = tuple(n)
    T = _Lazy.thunk

    def mesh():
        return np.meshgrid(xc[0], xc[1], xc[2], indexing="ij")

    def b3(ti, tj, tk):
        return (ti[:, None, None] * tj[None, :, None]) * tk[None, None, :]

    one = [np.ones(k) for k in n]
    onef = [np.ones(k + 1) for k in n]
    cs = coordinate_system
    r, th = xc[0], xc[1]
    A = (xf[0][1:] ** 2 - xf[0][:-1] ** 2) / 2.0

    def volume():
        if cs == "cartesian":
            return b3(dl[0], dl[1], dl[2])
        if cs == "cylindrical":
            return b3(A, dl[1], dl[2])
        return b3((xf[0][1:] ** 3 - xf[0][:-1] ** 3) / 3.0, np.cos(xf[1][:-1]) - np.cos(xf[1][1:]), dl[2])

    def surface():
        if cs == "cartesian":
            return {"x1": b3(onef[0], dl[1], dl[2]), "x2": b3(dl[0], onef[1], dl[2]), "x3": b3(dl[0], dl[1], onef[2])}
        if cs == "cylindrical":
            return {"x1": b3(xf[0], dl[1], dl[2]), "x2": b3(dl[0], onef[1], dl[2]), "x3": b3(A, dl[1], onef[2])}
        C2 = np.cos(xf[1][:-1]) - np.cos(xf[1][1:])
        return {"x1": b3(xf[0] ** 2, C2, dl[2]), "x2": b3(A, np.sin(xf[1]), dl[2]), "x3": b3(A, dl[1], onef[2])}

    def length():
        L1 = b3(dl[0], one[1], one[2])
        L2 = b3(one[0], dl[1], one[2]) if cs == "cartesian" else b3(r, dl[1], one[2])
        if cs == "spherical":
            L3 = (r[:, None] * np.sin(th)[None, :])[:, :, None] * dl[2][None, None, :]
        else:
            L3 = b3(one[0], one[1], dl[2])
        return {"x1": L1, "x2": L2, "x3": L3}

    def lame():
        z = np.zeros(shape)
        o = np.ones(shape)
        if cs == "cartesian":
            h = {"x1": o, "x2": o.copy(), "x3": o.copy()}
            dd = {"x1": {"ln_hx1hx2hx3": z, "ln_hx2": z, "ln_hx3": z},
                  "x2": {"ln_hx1hx2hx3": z, "ln_hx1": z, "ln_hx3": z},
                  "x3": {"ln_hx1hx2hx3": z, "ln_hx1": z, "ln_hx2": z}}
        elif cs == "cylindrical":
            R = b3(r, one[1], one[2])
            h = {"x1": o, "x2": R, "x3": o.copy()}
            dd = {"x1": {"ln_hx1hx2hx3": 1.0 / R, "ln_hx2": 1.0 / R, "ln_hx3": z},
                  "x2": {"ln_hx1hx2hx3": z, "ln_hx1": z, "ln_hx3": z},
                  "x3": {"ln_hx1hx2hx3": z, "ln_hx1": z, "ln_hx2": z}}
        else:
            R = b3(r, one[1], one[2])
            TH = b3(one[0], th, one[2])
            h = {"x1": o, "x2": R, "x3": R * np.sin(TH)}
            dd = {"x1": {"ln_hx1hx2hx3": 2.0 / R, "ln_hx2": 1.0 / R, "ln_hx3": 1.0 / R},
                  "x2": {"ln_hx1hx2hx3": 1.0 / np.tan(TH), "ln_hx1": z, "ln_hx3": 1.0 / np.tan(TH)},
                  "x3": {"ln_hx1hx2hx3": z, "ln_hx1": z, "ln_hx2": z}}
        return {"coefficients": h, "derivatives": dd}

    coords = _Lazy()
    _m = {}

    def comp(a):
        def f():
            if "m" not in _m:
                _m["m"] = mesh()
            return _m["m"][a]
        return T(f)

    coords.update({"x1": comp(0), "x2": comp(1), "x3": comp(2)})
    geom = _Lazy()
    geom.update({"volume": T(volume), "surface": T(surface), "length": T(length)})
    cell = _Lazy()
    cell.update({"coordinates": coords,
                 "normal": {"x1": np.array([1.0, 0.0, 0.0]), "x2": np.array([0.0, 1.0, 0.0]),
                            "x3": np.array([0.0, 0.0, 1.0])},
                 "geometry": geom})
    grid = _Lazy()
    grid.update({"config": dict(grid_config), "coordinate_system": cs, "cell": cell, "lame": T(lame),
                 "axes": {"centres": xc, "faces": xf}})
    return grid
