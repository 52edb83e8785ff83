"""CPU oracle for the finite-volume residual + Runge-Kutta stage update.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA path: only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs may import it.  The product path (``multiphysics_fvm_b200``)
never imports it and has no CPU fallback.

It is a float64 NumPy restatement of the reference solver's hot path
(nathanzimniak/multiphysics-fvm, pure Python/NumPy).  Every function cites the
reference file:line it follows.  Expressions keep the reference's evaluation
order (left-to-right NumPy binary ops, no fused multiply-add) so that results
agree with the reference to round-off; the restatement is pinned against
golden vectors produced by the reference itself (``tests/golden``).

State layout: one float64 array ``U`` of shape ``(NV, nx1+2, nx2+2, nx3+2)``
(C order, one ghost layer, variable order as in the reference's
``allocate_u``).  Closure / face arrays follow the reference shapes.
"""
from __future__ import annotations

import numpy as np

VARIABLES = {
    # navier_stokes.py:35-39
    "navier_stokes": ("mass_density", "momentum_x1", "momentum_x2",
                      "momentum_x3", "energy_density"),
    # heat.py:34-35
    "heat": ("internal_energy_density",),
    # maxwell.py:35-40
    "maxwell": ("magnetic_field_x1", "magnetic_field_x2", "magnetic_field_x3",
                "electric_d_field_x1", "electric_d_field_x2", "electric_d_field_x3"),
}

SIDES = ("left", "right", "bottom", "top", "front", "back")
_SIDE_AXIS = {"left": (0, 0), "right": (0, 1), "bottom": (1, 0),
              "top": (1, 1), "front": (2, 0), "back": (2, 1)}


# ---------------------------------------------------------------------------
# Geometry (src/grid/geometry.py:14-194)
# ---------------------------------------------------------------------------
class Geometry:
    """Cell volumes, face areas, physical lengths and Lame data.

    Built from 1D per-axis tables with the same operation order as
    ``build_grid`` (geometry.py:37-171), so every value is bitwise equal to
    the reference's 3D arrays.  Attributes (interior-shaped unless noted):
    ``V``; ``S[a]`` face-shaped along axis a; ``L[a]``; ``h[a]``;
    ``dlnh[a][b]`` = d_a ln h_b (b != a); ``dlnh123[a]``; ``xc[a]`` 1D cell
    centres; ``xf[a]`` 1D faces.
    """

    def __init__(self, coordinate_system: str, cfg: dict):
        n = [cfg["nx1"], cfg["nx2"], cfg["nx3"]]
        lo = [cfg["x1_min"], cfg["x2_min"], cfg["x3_min"]]
        hi = [cfg["x1_max"], cfg["x2_max"], cfg["x3_max"]]
        self.n = tuple(n)
        self.coordinate_system = coordinate_system
        d = [(hi[a] - lo[a]) / n[a] for a in range(3)]                     # :37-39
        xc = [lo[a] + (np.arange(n[a]) + 0.5) * d[a] for a in range(3)]    # :42-44
        xf = [lo[a] + np.arange(n[a] + 1) * d[a] for a in range(3)]        # :47-49
        self.xc, self.xf = xc, xf
        dl = [xf[a][1:] - xf[a][:-1] for a in range(3)]                    # face differences
        shape = tuple(n)

        def outer(ti, tj, tk):
            """((ti*tj)*tk) broadcast to 3D, left-to-right like NumPy."""
            return (ti[:, None, None] * tj[None, :, None]) * tk[None, None, :]

        one = [np.ones(n[a]) for a in range(3)]
        onef = [np.ones(n[a] + 1) for a in range(3)]
        zero = np.zeros(shape)
        r, th = xc[0], xc[1]
        if coordinate_system == "cartesian":                               # :80-109
            self.V = outer(dl[0], dl[1], dl[2])
            S1 = outer(onef[0], dl[1], dl[2])
            S2 = outer(dl[0], onef[1], dl[2])
            S3 = outer(dl[0], dl[1], onef[2])
            self.L = [outer(dl[0], one[1], one[2]), outer(one[0], dl[1], one[2]),
                      outer(one[0], one[1], dl[2])]
            self.h = [np.ones(shape), np.ones(shape), np.ones(shape)]
            dl1 = [zero, zero, zero]            # d1 ln h2, d1 ln h3 (index by b)
            dl2 = [zero, zero, zero]
            dl3 = [zero, zero, zero]
            d123 = [zero, zero, zero]
        elif coordinate_system == "cylindrical":                           # :111-140
            A = (xf[0][1:] ** 2 - xf[0][:-1] ** 2) / 2.0
            self.V = outer(A, dl[1], dl[2])
            S1 = outer(xf[0], dl[1], dl[2])
            S2 = outer(dl[0], onef[1], dl[2])
            S3 = outer(A, dl[1], onef[2])
            self.L = [outer(dl[0], one[1], one[2]), outer(r, dl[1], one[2]),
                      outer(one[0], one[1], dl[2])]
            self.h = [np.ones(shape), outer(r, one[1], one[2]), np.ones(shape)]
            inv_r = outer(1.0 / r, one[1], one[2])
            dl1 = [zero, inv_r, zero]
            dl2 = [zero, zero, zero]
            dl3 = [zero, zero, zero]
            d123 = [inv_r, zero, zero]
        elif coordinate_system == "spherical":                             # :142-171
            B = (xf[0][1:] ** 3 - xf[0][:-1] ** 3) / 3.0
            A = (xf[0][1:] ** 2 - xf[0][:-1] ** 2) / 2.0
            C = np.cos(xf[1][:-1]) - np.cos(xf[1][1:])
            self.V = outer(B, C, dl[2])
            S1 = outer(xf[0] ** 2, C, dl[2])
            S2 = outer(A, np.sin(xf[1]), dl[2])
            S3 = outer(A, dl[1], onef[2])
            rs = r[:, None] * np.sin(th)[None, :]
            self.L = [outer(dl[0], one[1], one[2]), outer(r, dl[1], one[2]),
                      rs[:, :, None] * dl[2][None, None, :]]
            self.h = [np.ones(shape), outer(r, one[1], one[2]),
                      np.broadcast_to(rs[:, :, None], shape).copy()]
            inv_r = outer(1.0 / r, one[1], one[2])
            cot = outer(one[0], 1.0 / np.tan(th), one[2])
            dl1 = [zero, inv_r, inv_r]
            dl2 = [zero, zero, cot]
            dl3 = [zero, zero, zero]
            d123 = [outer(2.0 / r, one[1], one[2]), cot, zero]
        else:                                                              # :173
            raise ValueError(f"Unknown coordinate system: '{coordinate_system}'. "
                             "Expected one of: cartesian, cylindrical, spherical.")
        self.S = [S1, S2, S3]
        self.dlnh = [dl1, dl2, dl3]   # dlnh[a][b] = d_{x_a} ln h_{x_b}
        self.dlnh123 = d123


# ---------------------------------------------------------------------------
# Boundary conditions (src/grid/boundary_conditions.py:13-91, solver.py:13-61)
# ---------------------------------------------------------------------------
def _face_slab(field, side, depth):
    """View of the ghost (depth 0) or the layer ``depth`` cells inside it,
    restricted to the transverse interior ``[1:-1]`` (boundary_conditions.py:31-36)."""
    axis, high = _SIDE_AXIS[side]
    idx = [slice(1, -1)] * 3
    idx[axis] = (-1 - depth) if high else depth
    return tuple(idx)


def bc_fill_face(field, side, kind, value=0.0):
    """Fill one ghost face slab of one variable in place.

    kind: "periodic" (:58-63, ghost = opposite interior layer),
          "neumann" (:31-36, ghost = adjacent interior),
          "reflecting" (:85-90, ghost = -adjacent interior),
          "dirichlet" (not in the reference: ghost = 2*value - adjacent interior).
    """
    ghost = _face_slab(field, side, 0)
    inner = _face_slab(field, side, 1)
    if kind == "periodic":
        axis, high = _SIDE_AXIS[side]
        src = [slice(1, -1)] * 3
        src[axis] = 1 if high else -2
        field[ghost] = field[tuple(src)]
    elif kind == "neumann":
        field[ghost] = field[inner]
    elif kind == "reflecting":
        field[ghost] = -field[inner]
    elif kind == "dirichlet":
        field[ghost] = 2.0 * value - field[inner]
    else:
        raise ValueError(f"Unknown boundary condition kind: {kind!r}")


def fill_edges_corners(f):
    """Ghost edges = mean of the two adjacent ghost faces, corners = mean of
    three (solver.py:39-61).  Nothing in the residual reads them."""
    for a, b in ((0, 1), (0, 2), (1, 2)):
        c = 3 - a - b
        for ea in (0, -1):
            for eb in (0, -1):
                tgt = [slice(1, -1)] * 3
                tgt[a], tgt[b] = ea, eb
                p = list(tgt); p[a] = 1 if ea == 0 else -2
                q = list(tgt); q[b] = 1 if eb == 0 else -2
                f[tuple(tgt)] = 0.5 * (f[tuple(p)] + f[tuple(q)])
        del c
    for i in (0, -1):
        for j in (0, -1):
            for k in (0, -1):
                ii = 1 if i == 0 else -2
                jj = 1 if j == 0 else -2
                kk = 1 if k == 0 else -2
                f[i, j, k] = (f[ii, j, k] + f[i, jj, k] + f[i, j, kk]) / 3.0


def apply_bcs(U, bcs):
    """bcs: list over variables of dict side -> (kind, value).  solver.py:30-61."""
    for v, per_side in enumerate(bcs):
        for side in SIDES:
            kind, value = per_side[side]
            bc_fill_face(U[v], side, kind, value)
        fill_edges_corners(U[v])


# ---------------------------------------------------------------------------
# Slope limiters (src/numerics/slope_limiters.py) and reconstruction
# ---------------------------------------------------------------------------
def minmod(a, b):
    """slope_limiters.py:13-39."""
    return (np.sign(a) + np.sign(b)) / 2.0 * np.minimum(np.abs(a), np.abs(b))


def monotonized_central(a, b):
    """slope_limiters.py:42-73, including its sign test (sum of three signs / 3),
    which is nonzero for slopes of opposite sign."""
    c = 0.5 * (a + b)
    a2 = 2.0 * a
    b2 = 2.0 * b
    sgn = (np.sign(c) + np.sign(a2) + np.sign(b2)) / 3.0
    return sgn * np.minimum(np.abs(c), np.minimum(np.abs(a2), np.abs(b2)))


def van_leer(a, b):
    """slope_limiters.py:76-105."""
    sgn = (np.sign(a) + np.sign(b)) / 2.0
    den = np.abs(a) + np.abs(b)
    hm = np.zeros_like(a)
    m = den > 0.0
    hm[m] = 2.0 * a[m] * b[m] / den[m]
    return sgn * hm


LIMITERS = {"minmod": minmod, "monotonized_central": monotonized_central,
            "van_leer": van_leer}


def _transverse_interior(f, axis):
    idx = [slice(1, -1)] * 3
    idx[axis] = slice(None)
    return f[tuple(idx)]


def _shift(a, axis, lo, hi):
    idx = [slice(None)] * 3
    idx[axis] = slice(lo, hi)
    return a[tuple(idx)]


def reconstruct(f, L_axis, axis, scheme, limiter):
    """Left/right face states of a ghosted cell field along one axis.

    piecewise_constant: reconstructors.py:13-64.  muscl: reconstructors.py:67-158
    (slope = limiter(bwd/L, fwd/L)*L on interior cells, 0 on ghosts; L-state
    f_i + s_i/2, R-state f_{i+1} - s_{i+1}/2).  Returns face-shaped arrays.
    """
    g = _transverse_interior(f, axis)          # n_a+2 along axis, interior across
    if scheme == "piecewise_constant":
        return _shift(g, axis, None, -1), _shift(g, axis, 1, None)
    d = np.diff(g, axis=axis)                  # g[i+1]-g[i], n_a+1 entries
    bwd = _shift(d, axis, None, -1) / L_axis
    fwd = _shift(d, axis, 1, None) / L_axis
    s = np.zeros_like(g)
    idx = [slice(None)] * 3
    idx[axis] = slice(1, -1)
    s[tuple(idx)] = limiter(bwd, fwd) * L_axis
    left = _shift(g, axis, None, -1) + _shift(s, axis, None, -1) / 2.0
    right = _shift(g, axis, 1, None) - _shift(s, axis, 1, None) / 2.0
    return left, right


def central_gradient(f, L_axis, axis):
    """(f[i+1]-f[i-1])/(2 L) on interior cells of a ghosted array
    (navier_stokes.py:111-119, heat.py:85-87, maxwell.py:491-496)."""
    g = _transverse_interior(f, axis)
    return (_shift(g, axis, 2, None) - _shift(g, axis, None, -2)) / (2 * L_axis)


def _pad_zero(a):
    return np.pad(a, 1)


# ---------------------------------------------------------------------------
# Riemann and diffusive solvers (riemann_solvers.py, diffusive_solvers.py)
# ---------------------------------------------------------------------------
def rusanov(FL, FR, UL, UR, lamL, lamR):
    """riemann_solvers.py:13-48 (speed = max |lambda| over waves and sides)."""
    vs = np.maximum(np.maximum.reduce([np.abs(x) for x in lamL]),
                    np.maximum.reduce([np.abs(x) for x in lamR]))
    return [(fl + fr) / 2.0 - vs * (ur - ul) / 2.0
            for fl, fr, ul, ur in zip(FL, FR, UL, UR)]


def hll(FL, FR, UL, UR, lamL, lamR):
    """riemann_solvers.py:51-89 (three-way selection on the extreme speeds)."""
    smin = np.minimum(np.minimum.reduce(lamL), np.minimum.reduce(lamR))
    smax = np.maximum(np.maximum.reduce(lamL), np.maximum.reduce(lamR))
    out = []
    with np.errstate(divide="ignore", invalid="ignore"):
        for fl, fr, ul, ur in zip(FL, FR, UL, UR):
            mid = (smax * fl - smin * fr + smin * smax * (ur - ul)) / (smax - smin)
            out.append(np.where(smin >= 0.0, fl, np.where(smax <= 0.0, fr, mid)))
    return out


RIEMANN = {"rusanov": rusanov, "hll": hll}


def centered(FdL, FdR):
    """diffusive_solvers.py:11-30."""
    return [(a + b) / 2.0 for a, b in zip(FdL, FdR)]


def divergence(F, geo):
    """-(sum_a (F S)[+] - (F S)[-]) / V, the finite-volume divergence
    (navier_stokes.py:705-709, heat.py:471, maxwell.py:722-727)."""
    t = []
    for a in range(3):
        fs = F[a] * geo.S[a]
        t.append((_shift(fs, a, 1, None), _shift(fs, a, None, -1)))
    acc = t[0][0] - t[0][1] + t[1][0] - t[1][1] + t[2][0] - t[2][1]
    return -acc / geo.V


# ---------------------------------------------------------------------------
# Navier-Stokes (src/physics/navier_stokes.py)
# ---------------------------------------------------------------------------
def ns_pressure(U, gam):
    """Primitive velocity and ideal-gas pressure on all cells
    (navier_stokes.py:94-100).  Ghost edges and corners that a test leaves at
    zero give NaN here; no residual reads them (interior stencils slice the
    transverse 1:-1), so the division warnings are silenced."""
    rho = U[0]
    with np.errstate(invalid="ignore", divide="ignore"):
        v = [U[1] / rho, U[2] / rho, U[3] / rho]
        E = U[4] / rho
        P = (gam - 1.0) * rho * (E - (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / 2.0)
    return v, P


def ns_stress(v, geo, mu):
    """Stokes viscous stress on interior cells, zero-padded ghosts
    (navier_stokes.py:102-142).  Returns dict (a,b)->ghosted array."""
    g = [[central_gradient(v[c], geo.L[a], a) for a in range(3)] for c in range(3)]
    # g[c][a] = d v_c / d x_a
    vi = [x[1:-1, 1:-1, 1:-1] for x in v]
    h, dl = geo.h, geo.dlnh
    divv = (g[0][0] + g[1][1] + g[2][2]
            + vi[0] * (dl[0][1] + dl[0][2]) / h[0]
            + vi[1] * (dl[1][0] + dl[1][2]) / h[1]
            + vi[2] * (dl[2][0] + dl[2][1]) / h[2])
    t11 = mu * (2 * g[0][0] - (2.0 / 3.0) * divv)
    t22 = mu * (2 * (g[1][1] + vi[0] * dl[0][1] / h[0]) - (2.0 / 3.0) * divv)
    t33 = mu * (2 * (g[2][2] + vi[0] * dl[0][2] / h[0] + vi[1] * dl[1][2] / h[1])
                - (2.0 / 3.0) * divv)
    t12 = mu * (g[0][1] + g[1][0] - vi[1] * dl[0][1] / h[0] + vi[0] * dl[1][0] / h[1])
    t13 = mu * (g[0][2] + g[2][0] - vi[2] * dl[0][2] / h[0] + vi[0] * dl[2][0] / h[2])
    t23 = mu * (g[1][2] + g[2][1] - vi[2] * dl[1][2] / h[1] + vi[1] * dl[2][1] / h[2])
    T = {(0, 0): t11, (1, 1): t22, (2, 2): t33, (0, 1): t12, (0, 2): t13, (1, 2): t23}
    full = {}
    for (a, b), val in T.items():
        full[(a, b)] = _pad_zero(val)
        full[(b, a)] = full[(a, b)]
    return full


def ns_face_flux(Uf, Pf, Tf, a, gam):
    """Normal convective flux, normal diffusive flux and wave speeds of one
    face state along axis a (navier_stokes.py:159-316).  Tf[b] = face tau_{a b}
    (the a-row of the reconstructed stress)."""
    rho = Uf[0]
    v = [Uf[1] / rho, Uf[2] / rho, Uf[3] / rho]
    E = Uf[4] / rho
    va = v[a]
    Fc = [rho * va]
    for c in range(3):
        f = rho * v[c] * va
        if c == a:
            f = f + Pf
        Fc.append(f)
    Fc.append((rho * E + Pf) * va)
    if Tf is None:
        Fd = None
    else:
        Fd = [np.zeros_like(rho), -Tf[0], -Tf[1], -Tf[2],
              -Tf[0] * v[0] - Tf[1] * v[1] - Tf[2] * v[2]]
    cs = np.sqrt(gam * Pf / rho)
    lam = [va, va + (-cs), va + cs]
    return Fc, Fd, lam


def ns_rhs(U, geo, prm, sch):
    """Navier-Stokes residual (navier_stokes.py:588-711)."""
    gam = prm["heat_capacity_ratio"]
    mu = prm["dynamic_viscosity"]
    grav = prm["gravitational_acceleration"]
    v, P = ns_pressure(U, gam)
    T = ns_stress(v, geo, mu)
    lim = LIMITERS.get(sch.get("slope_limiter"))
    rec = sch["reconstructor"]
    riem = RIEMANN[sch["riemann_solver"]]
    F = []
    for a in range(3):
        UL, UR = zip(*[reconstruct(U[q], geo.L[a], a, rec, lim) for q in range(5)])
        PL, PR = reconstruct(P, geo.L[a], a, rec, lim)
        TL, TR = zip(*[reconstruct(T[(a, b)], geo.L[a], a, rec, lim) for b in range(3)])
        FcL, FdL, lamL = ns_face_flux(UL, PL, TL, a, gam)
        FcR, FdR, lamR = ns_face_flux(UR, PR, TR, a, gam)
        Fc = riem(FcL, FcR, UL, UR, lamL, lamR)
        Fd = centered(FdL, FdR)
        F.append([Fc[q] + Fd[q] for q in range(5)])
    src = ns_sources(U, P, T, v, geo, grav)
    return np.stack([divergence([F[0][q], F[1][q], F[2][q]], geo) + src[q]
                     for q in range(5)])


def ns_sources(U, P, T, v, geo, grav):
    """Geometric (navier_stokes.py:437-452) + gravity (:499-504) sources."""
    I = (slice(1, -1),) * 3
    rho = U[0][I]
    vi = [x[I] for x in v]
    Pi = P[I]
    t = {k: val[I] for k, val in T.items()}
    h, dl, d123 = geo.h, geo.dlnh, geo.dlnh123
    sgc = [0.0]
    sgd = [0.0]
    for c in range(3):
        o = [b for b in range(3) if b != c]
        # convective: P d_c ln(h1h2h3)/h_c + sum_b rho v_b v_b d_c ln h_b / h_c
        #             - sum_b rho v_c v_b d_b ln h_c / h_b
        s = (Pi * d123[c] / h[c]
             + rho * vi[o[0]] * vi[o[0]] * dl[c][o[0]] / h[c]
             + rho * vi[o[1]] * vi[o[1]] * dl[c][o[1]] / h[c]
             - rho * vi[c] * vi[o[0]] * dl[o[0]][c] / h[o[0]]
             - rho * vi[c] * vi[o[1]] * dl[o[1]][c] / h[o[1]])
        sgc.append(s)
        d = (t[(c, o[0])] * dl[o[0]][c] / h[o[0]]
             + t[(c, o[1])] * dl[o[1]][c] / h[o[1]]
             - t[(o[0], o[0])] * dl[c][o[0]] / h[c]
             - t[(o[1], o[1])] * dl[c][o[1]] / h[c])
        sgd.append(d)
    sgc.append(0.0)
    sgd.append(0.0)
    g1, g2, g3 = grav
    spg = [0.0, rho * g1, rho * g2, rho * g3,
           rho * (g1 * vi[0] + g2 * vi[1] + g3 * vi[2])]
    return [(sgc[q] + sgd[q]) + spg[q] for q in range(5)]


def ns_dt(U, prm, geo, cfl):
    """CFL time step (navier_stokes.py:512-585)."""
    gam = prm["heat_capacity_ratio"]
    mu = prm["dynamic_viscosity"]
    v, P = ns_pressure(U, gam)
    cs = np.sqrt(gam * P / U[0])
    I = (slice(1, -1),) * 3
    ml = [np.maximum.reduce([np.abs(v[a][I] + 0), np.abs(v[a][I] + (-cs[I])),
                             np.abs(v[a][I] + cs[I])]) for a in range(3)]
    nu = np.max(mu / U[0][I])
    rc = np.max(np.maximum.reduce([ml[a] / geo.L[a] for a in range(3)]))
    rd = np.max(2 * nu * (1 / geo.L[0] ** 2 + 1 / geo.L[1] ** 2 + 1 / geo.L[2] ** 2))
    return cfl / (rc + rd)


# ---------------------------------------------------------------------------
# Heat (src/physics/heat.py)
# ---------------------------------------------------------------------------
def heat_rhs(U, geo, prm, sch):
    """Heat residual (heat.py:354-473): centred diffusion of phi = -k grad T."""
    cp = prm["specific_heat_capacity"]
    k = prm["thermal_conductivity"]
    rho = prm["mass_density"]
    q = prm["volumetric_heat_source"]
    T = U[0] / (rho * cp)                                           # :74
    phi = [_pad_zero(-k * central_gradient(T, geo.L[a], a)) for a in range(3)]
    lim = LIMITERS.get(sch.get("slope_limiter"))
    F = []
    for a in range(3):
        L_, R_ = reconstruct(phi[a], geo.L[a], a, sch["reconstructor"], lim)
        F.append(0.0 + (L_ + R_) / 2.0)
    return (divergence(F, geo) + q)[None]


def heat_dt(prm, geo, cfl):
    """State-independent diffusive CFL step (heat.py:305-351)."""
    nu = prm["thermal_conductivity"] / (prm["mass_density"] * prm["specific_heat_capacity"])
    rd = np.max(2 * nu * (1 / geo.L[0] ** 2 + 1 / geo.L[1] ** 2 + 1 / geo.L[2] ** 2))
    return cfl / (0.0 + rd)


# ---------------------------------------------------------------------------
# Maxwell (src/physics/maxwell.py)
# ---------------------------------------------------------------------------
_EPS3 = {(0, 1, 2): 1, (1, 2, 0): 1, (2, 0, 1): 1,
         (0, 2, 1): -1, (2, 1, 0): -1, (1, 0, 2): -1}


def maxwell_face_flux(Uf, a, mu, ep):
    """Normal curl fluxes along axis a (maxwell.py:145-181): B_c row a is
    -eps_{c a b} E_b... written out component by component."""
    H = [Uf[0] / mu, Uf[1] / mu, Uf[2] / mu]
    E = [Uf[3] / ep, Uf[4] / ep, Uf[5] / ep]
    z = np.zeros_like(Uf[0])
    # magnetic flux tensor FB[c][a]: FB12=E3, FB13=-E2, FB23=E1, antisymmetric
    FB = [[z, E[2], -E[1]], [-E[2], z, E[0]], [E[1], -E[0], z]]
    FD = [[z, -H[2], H[1]], [H[2], z, -H[0]], [-H[1], H[0], z]]
    return [FB[c][a] for c in range(3)] + [FD[c][a] for c in range(3)]


def maxwell_rhs(U, geo, prm, sch):
    """Maxwell residual (maxwell.py:603-729) incl. divergence cleaning."""
    mu = prm["magnetic_permeability"]
    ep = prm["electric_permittivity"]
    c = 1 / np.sqrt(mu * ep)                                         # :256
    lim = LIMITERS.get(sch.get("slope_limiter"))
    riem = RIEMANN[sch["riemann_solver"]]
    F = []
    for a in range(3):
        UL, UR = zip(*[reconstruct(U[q], geo.L[a], a, sch["reconstructor"], lim)
                       for q in range(6)])
        FcL = maxwell_face_flux(UL, a, mu, ep)
        FcR = maxwell_face_flux(UR, a, mu, ep)
        shp = UL[0].shape
        lam = [np.full(shp, -c), np.full(shp, +c)]
        Fc = riem(FcL, FcR, UL, UR, lam, lam)
        F.append([x + 0.0 for x in Fc])
    src = maxwell_sources(U, geo, prm)
    return np.stack([divergence([F[0][q], F[1][q], F[2][q]], geo) + src[q]
                     for q in range(6)])


def maxwell_sources(U, geo, prm):
    """Geometric (maxwell.py:365-374), Ohmic (:414-420) and cleaning
    (:490-528) sources, summed as sg + sp + sc."""
    mu = prm["magnetic_permeability"]
    ep = prm["electric_permittivity"]
    sigma = prm["electrical_conductivity"]
    I = (slice(1, -1),) * 3
    B = [U[q][I] / mu for q in range(3)]      # H
    E = [U[q][I] / ep for q in range(3, 6)]
    h, dl = geo.h, geo.dlnh
    # flux tensors on cells; diagonal entries are the scalar 0.0
    FB = {(0, 1): E[2], (0, 2): -E[1], (1, 2): E[0]}
    FD = {(0, 1): -B[2], (0, 2): B[1], (1, 2): -B[0]}
    for T in (FB, FD):
        for (x, y) in list(T):
            T[(y, x)] = -T[(x, y)]
    sg = []
    for T in (FB, FD):
        for cc in range(3):
            o = [b for b in range(3) if b != cc]
            s = (T[(cc, o[0])] * dl[o[0]][cc] / h[o[0]]
                 + T[(cc, o[1])] * dl[o[1]][cc] / h[o[1]]
                 - 0.0 * dl[cc][o[0]] / h[cc]
                 - 0.0 * dl[cc][o[1]] / h[cc])
            sg.append(s)
    J = [-sigma * (U[q][I] / ep) for q in range(3, 6)]
    sp = [0.0, 0.0, 0.0, J[0], J[1], J[2]]
    sc = maxwell_cleaning(U, geo, prm)
    return [sg[q] + sp[q] + sc[q] for q in range(6)]


def maxwell_cleaning(U, geo, prm):
    """Divergence-cleaning source -chi grad(residual), residual edge-padded
    (maxwell.py:428-530)."""
    rho_c = prm["charge_density"]
    chiB = prm["magnetic_cleaning_coeff"]
    chiD = prm["electric_cleaning_coeff"]
    h, dl = geo.h, geo.dlnh
    I = (slice(1, -1),) * 3

    def div(q0):
        grads = [central_gradient(U[q0 + a], geo.L[a], a) for a in range(3)]
        c = [U[q0 + a][I] for a in range(3)]
        return (grads[0] + grads[1] + grads[2]
                + c[0] * (dl[0][1] + dl[0][2]) / h[0]
                + c[1] * (dl[1][0] + dl[1][2]) / h[1]
                + c[2] * (dl[2][0] + dl[2][1]) / h[2])

    rB = np.pad(div(0), 1, mode="edge")
    rD = np.pad(div(3) - rho_c, 1, mode="edge")
    out = [-chiB * central_gradient(rB, geo.L[a], a) for a in range(3)]
    out += [-chiD * central_gradient(rD, geo.L[a], a) for a in range(3)]
    return out


def maxwell_dt(prm, geo, cfl):
    """State-independent light-speed + cleaning CFL step (maxwell.py:533-600)."""
    c = 1 / np.sqrt(prm["magnetic_permeability"] * prm["electric_permittivity"])
    ml = max(abs(-c), abs(c))
    rc = np.max(np.maximum.reduce([np.full(geo.n, ml) / geo.L[a] for a in range(3)]))
    chi = max(prm["magnetic_cleaning_coeff"], prm["electric_cleaning_coeff"])
    rd = np.max(2.0 * chi * (1.0 / geo.L[0] ** 2 + 1.0 / geo.L[1] ** 2 + 1.0 / geo.L[2] ** 2))
    return cfl / (rc + rd)


RHS = {"navier_stokes": ns_rhs, "heat": heat_rhs, "maxwell": maxwell_rhs}


def compute_dt(physics, U, prm, geo, cfl):
    if physics == "navier_stokes":
        return ns_dt(U, prm, geo, cfl)
    if physics == "heat":
        return heat_dt(prm, geo, cfl)
    return maxwell_dt(prm, geo, cfl)


# ---------------------------------------------------------------------------
# Time integrators (src/numerics/time_integrators.py)
# ---------------------------------------------------------------------------
def integrate(integrator, physics, U, dt, prm, geo, sch, bcs):
    """One time step in place.  Stage combinations: euler_explicit :42-47,
    rk3 :87-103 (as written; second order), rk3_ssp :143-159, rk4 :199-221.
    ``apply_bcs`` runs before every stage."""
    rhs = RHS[physics]
    I = (slice(None),) + (slice(1, -1),) * 3
    U0 = U[I].copy()

    def stage():
        apply_bcs(U, bcs)
        return rhs(U, geo, prm, sch)

    if integrator == "euler_explicit":
        k1 = stage()
        U[I] += dt * k1
    elif integrator == "rk3":
        k1 = stage(); U[I] = U0 + 0.5 * dt * k1
        k2 = stage(); U[I] = U0 + dt * k2
        k3 = stage(); U[I] = U0 + (dt / 6.0) * (k1 + 4.0 * k2 + k3)
    elif integrator == "rk3_ssp":
        k1 = stage(); U[I] = U0 + dt * k1
        k2 = stage(); U[I] = 0.75 * U0 + 0.25 * (U[I] + dt * k2)
        k3 = stage(); U[I] = (1.0 / 3.0) * U0 + (2.0 / 3.0) * (U[I] + dt * k3)
    elif integrator == "rk4":
        k1 = stage(); U[I] = U0 + 0.5 * dt * k1
        k2 = stage(); U[I] = U0 + 0.5 * dt * k2
        k3 = stage(); U[I] = U0 + dt * k3
        k4 = stage(); U[I] = U0 + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
    else:
        raise ValueError(f"Unknown integrator {integrator!r}")


def run(physics, U, prm, geo, sch, bcs, integrator, cfl, n_steps, dt_fixed=None):
    """Step-counted time loop (solver.py:137-151 with a step count).
    Returns the list of dt values used."""
    dts = []
    for _ in range(n_steps):
        dt = dt_fixed if dt_fixed is not None else compute_dt(physics, U, prm, geo, cfl)
        integrate(integrator, physics, U, dt, prm, geo, sch, bcs)
        dts.append(dt)
    return dts
