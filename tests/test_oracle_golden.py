"""The oracle (CPU restatement) against golden vectors produced by the reference
itself (tests/golden/make_golden.py).  Bit-exact agreement is required."""
import numpy as np
import pytest

from oracle import fvm_oracle as O


def _cases(golden, kind):
    z, man, P = golden
    return [c for c in man if c["kind"] == kind]


def test_golden_fixture_is_complete(golden):
    z, man, P = golden
    rhs = [c for c in man if c["kind"] == "rhs"]
    steps = [c for c in man if c["kind"] == "step"]
    assert {c["physics"] for c in rhs} == {"navier_stokes", "heat", "maxwell"}
    assert {c["coords"] for c in rhs} == {"cartesian", "cylindrical", "spherical"}
    assert {(c["reconstructor"], c["limiter"]) for c in rhs if c["physics"] == "maxwell"} >= {
        ("piecewise_constant", None), ("muscl", "minmod"), ("muscl", "monotonized_central"), ("muscl", "van_leer")}
    assert {c["integrator"] for c in steps} == {"euler_explicit", "rk3", "rk3_ssp", "rk4"}


def test_oracle_residual_and_dt_bitexact(golden):
    z, man, P = golden
    for c in _cases(golden, "rhs"):
        nm = c["name"]
        geo = O.Geometry(c["coords"], c["grid"])
        sch = dict(reconstructor=c["reconstructor"], slope_limiter=c["limiter"], riemann_solver=c["riemann"])
        U = z[nm + "/U"].copy()
        with np.errstate(all="ignore"):
            r = O.RHS[c["physics"]](U, geo, P[c["params"]], sch)
            dt = O.compute_dt(c["physics"], U, P[c["params"]], geo, 0.37)
        assert np.array_equal(r, z[nm + "/rhs"]), nm
        assert dt == float(z[nm + "/dt"]), nm


def test_oracle_integrator_steps_bitexact(golden):
    z, man, P = golden
    I = (slice(None),) + (slice(1, -1),) * 3
    for c in _cases(golden, "step"):
        nm = c["name"]
        geo = O.Geometry(c["coords"], c["grid"])
        sch = dict(reconstructor=c["reconstructor"], slope_limiter=c["limiter"], riemann_solver=c["riemann"])
        bcs = [{s: (k, 0.0) for s, k in zip(O.SIDES, kk)} for kk in c["bcs"]]
        U = z[nm + "/U"].copy()
        with np.errstate(all="ignore"):
            O.integrate(c["integrator"], c["physics"], U, float(z[nm + "/dt"]), P[c["params"]], geo, sch, bcs)
        assert np.array_equal(U[I], z[nm + "/U_after"][I]), nm
        # ghosts too (faces, edges, corners written by apply_bcs before the last stage)
        assert np.array_equal(np.nan_to_num(U), np.nan_to_num(z[nm + "/U_after"])), nm


def test_limiter_truth_table(golden):
    z, _, _ = golden
    a, b = z["limiters/a"], z["limiters/b"]
    for nm, f in O.LIMITERS.items():
        assert np.array_equal(f(a.copy(), b.copy()), z[f"limiters/{nm}"]), nm
    # the reference's MC sign test leaves +-1/3 min(...) for opposite signs
    assert O.monotonized_central(np.array([1.0]), np.array([-0.1]))[0] == pytest.approx(0.2 / 3.0)


def test_known_answers():
    """Reference-independent checks of the oracle: free stream, RK orders."""
    geo = O.Geometry("cartesian", dict(x1_min=0, x1_max=1, x2_min=0, x2_max=1, x3_min=0, x3_max=1,
                                       nx1=6, nx2=5, nx3=4))
    U = np.ones((5, 8, 7, 6))
    U[1] *= 0.3
    U[4] = 2.5 / 0.4 + 0.5 * 0.09
    prm = {"heat_capacity_ratio": 1.4, "dynamic_viscosity": 1e-3, "gravitational_acceleration": [0, 0, 0]}
    for lim in ("minmod", "monotonized_central", "van_leer"):
        r = O.ns_rhs(U, geo, prm, dict(reconstructor="muscl", slope_limiter=lim, riemann_solver="hll"))
        assert np.max(np.abs(r)) < 1e-12
