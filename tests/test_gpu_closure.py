"""GPU parity of the learned-closure kernels against the float64 oracle
(oracle/closure_oracle.py), all through the C ABI:

* forward conv layers (tcgen05 implicit GEMM) and the feature kernel;
* the a-priori loss, its gradient, the data gradients and the weight/bias
  gradients (tcgen05 wgrad);
* Adam with bias correction over two steps;
* the box filter and the dense state copies;
* the per-stage correction (clip + positivity gate), standalone and inside
  the solver's captured step (Euler: bitwise against the composition of the
  plain step and the standalone correction; SSPRK3: against the oracle).

BF16 tolerances: a BF16 output may differ from the oracle's rounding of the
same float64 value by one BF16 ulp (at most 2^-7 relative) where the FP32
accumulation lands next to a rounding boundary; FP32 outputs and gradients
agree to 1e-4 of their largest magnitude.
"""
import math

import numpy as np
import pytest

from oracle import closure_oracle as co
from oracle import fvm_oracle as O

pytestmark = pytest.mark.gpu

GAMMA = 1.4
MEAN = np.array([1.5, 0.0, 0.0, 0.0, 2.5])
SCALE = np.array([0.5, 0.5, 0.5, 0.5, 0.5])


def _closure(n, seed=0, out_scale=None, loss_w=None):
    from multiphysics_fvm_b200.closure import Closure
    c = Closure(n, seed=seed)
    c.set_norm(GAMMA, MEAN, SCALE, out_scale if out_scale is not None else np.full(5, 0.05),
               loss_w if loss_w is not None else np.ones(5))
    return c


def _rand_params(rng, scale=1.0):
    dims = [(32, 16), (32, 32), (16, 32)]
    return [(rng.normal(0, scale * math.sqrt(2.0 / (27 * ci)), (27, cout, ci)).astype(np.float32),
             rng.normal(0, 0.1, cout).astype(np.float32)) for cout, ci in dims]


def _bf16_close(ours, ref, what):
    """Every element within one BF16 ulp of the oracle (plus a tiny floor)."""
    scale = max(float(np.max(np.abs(ref))), 1e-30)
    tol = 2.0 ** -7 * np.abs(ref) + 1e-5 * scale
    bad = np.abs(ours - ref) > tol
    assert not bad.any(), f"{what}: {bad.sum()} of {bad.size} elements off, max err {np.max(np.abs(ours - ref))}"


def _close(ours, ref, what, rel=1e-4):
    scale = max(float(np.max(np.abs(ref))), 1e-30)
    err = float(np.max(np.abs(ours - ref))) / scale
    assert err <= rel, f"{what}: max error {err:.3e} of max |ref|"


def _random_state(shape, rng):
    rho = rng.uniform(1.0, 2.0, shape)
    v = rng.uniform(-0.5, 0.5, (3,) + shape)
    p = rng.uniform(2.0, 3.0, shape)
    return np.stack([rho, rho * v[0], rho * v[1], rho * v[2], p / (GAMMA - 1) + 0.5 * rho * (v * v).sum(0)]
                    ).astype(np.float32)


GRIDS = [(64, 64, 32), (32, 16, 8)]


@pytest.fixture(params=GRIDS, ids=lambda g: "x".join(map(str, g)))
def net(request):
    n = request.param
    rng = np.random.default_rng(11)
    c = _closure(n)
    params = _rand_params(rng)
    c.set_weights(params)
    X0 = np.zeros((n[2], n[1], n[0], 16))
    X0[..., :5] = rng.normal(0, 1, (n[2], n[1], n[0], 5))
    c.set_buffer(0, X0)
    c.forward()
    yield c, params, rng
    c.close()


def test_forward_layers_match_oracle(net):
    c, params, _ = net
    Wb = [(co.bf16(W), b.astype(np.float64)) for W, b in params]
    X0, A1, A2, Z3 = c.buffer(0), c.buffer(1), c.buffer(2), c.buffer(3)
    assert np.count_nonzero(A1) > 0.2 * A1.size and np.count_nonzero(A2) > 0.2 * A2.size
    _bf16_close(A1, co.bf16(co.relu(co.conv3d(X0, *Wb[0]))), "layer 1")
    _bf16_close(A2, co.bf16(co.relu(co.conv3d(A1, *Wb[1]))), "layer 2")
    _close(Z3, co.conv3d(A2, *Wb[2]), "layer 3", rel=1e-5)


def test_backward_matches_oracle(net):
    import torch
    c, params, rng = net
    n = c.n
    Wb = [(co.bf16(W), b.astype(np.float64)) for W, b in params]
    X0, A1, A2, Z3 = (c.buffer(i).astype(np.float64) for i in range(4))
    D = rng.normal(0, 1e-3, (5, n[2], n[1], n[0])).astype(np.float32)
    s, w, dt, h = np.full(5, 0.05), np.ones(5), 2e-3, (1 / n[0], 1 / n[1], 1 / n[2])
    c.backward(torch.from_numpy(D).cuda(), dt, h)
    loss_ref, E_ref, G3_ref = co.loss_and_grad(Z3, D.astype(np.float64), s, w, dt, h)
    assert abs(c.loss() - loss_ref) <= 1e-5 * loss_ref
    _close(c.buffer(7), E_ref, "defect residual", rel=1e-5)
    G3, G2, G1 = (c.buffer(i).astype(np.float64) for i in (4, 5, 6))
    _bf16_close(G3, co.bf16(G3_ref), "dLoss/dZ3")
    _bf16_close(G2, co.bf16(co.conv3d_dgrad(G3, Wb[2][0]) * (A2 > 0)), "dgrad layer 3")
    _bf16_close(G1, co.bf16(co.conv3d_dgrad(G2, Wb[1][0]) * (A1 > 0)), "dgrad layer 2")
    ours = c.get_grads()
    refs = [(co.conv3d_wgrad(X0, G1), G1.sum((0, 1, 2))), (co.conv3d_wgrad(A1, G2), G2.sum((0, 1, 2))),
            (co.conv3d_wgrad(A2, G3), G3.sum((0, 1, 2)))]
    for layer, ((dw, db), (rw, rb)) in enumerate(zip(ours, refs), start=1):
        assert np.max(np.abs(rw)) > 0
        _close(dw, rw, f"dW{layer}")
        _close(db, rb, f"db{layer}")


def test_adam_two_steps_match_oracle(net):
    import torch
    c, _, rng = net
    n = c.n
    D = torch.from_numpy(rng.normal(0, 1e-3, (5, n[2], n[1], n[0])).astype(np.float32)).cuda()
    h = (1 / n[0], 1 / n[1], 1 / n[2])
    w0 = [(w.astype(np.float64), b.astype(np.float64)) for w, b in c.get_weights()]
    mom = [[np.zeros_like(w), np.zeros_like(w), np.zeros_like(b), np.zeros_like(b)] for w, b in w0]
    ref = [(w.copy(), b.copy()) for w, b in w0]
    for step in (1, 2):
        c.backward(D, 2e-3, h)
        grads = c.get_grads()
        c.adam(lr=1e-3)
        for layer in range(3):
            co.adam(ref[layer][0], grads[layer][0].astype(np.float64), mom[layer][0], mom[layer][1], step)
            co.adam(ref[layer][1], grads[layer][1].astype(np.float64), mom[layer][2], mom[layer][3], step)
        c.forward()  # repack check: the next backward uses the updated weights
    for (w, b), (rw, rb) in zip(c.get_weights(), ref):
        assert np.max(np.abs(w - rw)) <= 1e-6 * max(1.0, np.max(np.abs(rw)))
        assert np.max(np.abs(b - rb)) <= 1e-6 * max(1.0, np.max(np.abs(rb)))
    assert max(np.max(np.abs(w - w0w)) for (w, _), (w0w, _) in zip(c.get_weights(), w0)) > 1e-4


def test_features_match_oracle():
    import torch
    n = (32, 16, 8)
    rng = np.random.default_rng(3)
    u = _random_state((n[2], n[1], n[0]), rng)
    c = _closure(n)
    c.features(torch.from_numpy(u).cuda())
    _bf16_close(c.buffer(0), co.bf16(co.features(u.astype(np.float64), GAMMA, MEAN, SCALE)), "features")


def _kh_sim(n, integrator=None, seed=0):
    from multiphysics_fvm_b200.backend import Simulation
    from multiphysics_fvm_b200.setups import kelvin_helmholtz_sharp as kh
    s = kh.get_setup(n[0], n[1], n[2], seed=seed, precision="fp32", noise_all=True)
    if integrator is not None:
        s["time_integrator"] = integrator
    return s, Simulation.from_setup(s)


def test_filter_and_dense_copies():
    import torch
    from multiphysics_fvm_b200 import closure as CL
    n = (32, 32, 16)
    rng = np.random.default_rng(4)
    _, sim = _kh_sim(n)
    u = _random_state((n[2], n[1], n[0]), rng)
    ut = torch.from_numpy(u).cuda()
    CL.upload_dense(sim, ut)
    back = CL.download_dense(sim).cpu().numpy()
    assert np.array_equal(back, u)
    for f in (2, 4):
        ours = CL.filter_state(sim, f).cpu().numpy()
        _close(ours, co.box_filter(u.astype(np.float64), f), f"filter {f}", rel=1e-7)


@pytest.mark.parametrize("fct", [False, True], ids=["clip", "fct"])
def test_correct_dense_matches_oracle(fct):
    import torch
    n = (32, 32, 16)
    rng = np.random.default_rng(5)
    c = _closure(n, out_scale=np.full(5, 0.2))
    c.set_limiter(fct)
    c.set_weights(_rand_params(rng, scale=2.0))
    uin = _random_state((n[2], n[1], n[0]), rng)
    uout = (uin * (1 + 1e-3 * rng.standard_normal(uin.shape))).astype(np.float32)
    c.features(torch.from_numpy(uin).cuda())
    c.forward()
    Z3 = c.buffer(3).astype(np.float64)
    h = (1 / n[0], 1 / n[1], 1 / n[2])
    for beta, dt, coef in ((0.5, 1e-3, 1.0), (0.5, 1e-3, 0.25), (50.0, 5.0, 1.0)):
        out = torch.from_numpy(uout.copy()).cuda()
        nsw = c.correct_dense(torch.from_numpy(uin).cuda(), out, coef, dt, beta, h)
        ref, nref = co.correct(uin, uout.astype(np.float64), Z3, c.norm["out_scale"], beta, GAMMA, coef, dt, h,
                               fct=fct)
        ours = out.cpu().numpy()
        if nref == 0:
            assert nsw == 0
            _close(ours, ref, f"correction beta={beta}", rel=1e-5)
            assert np.max(np.abs(ours - uout)) > 1e-6  # the correction did something
        else:  # marginal cells may flip; all kept cells must be positive
            assert abs(nsw - nref) <= max(2, nref // 100)
            rho, _, p = co.primitives(ours.astype(np.float64), GAMMA)
            assert np.all(rho > 0) and np.all(p > 0)


@pytest.mark.parametrize("fct", [False, True], ids=["clip", "fct"])
def test_attached_euler_step_is_plain_step_plus_correction(fct):
    import torch
    from multiphysics_fvm_b200 import closure as CL
    from multiphysics_fvm_b200.numerics import time_integrators as ti
    n = (32, 32, 16)
    rng = np.random.default_rng(6)
    c = _closure(n, out_scale=np.full(5, 0.02))
    c.set_limiter(fct)
    c.set_weights(_rand_params(rng))
    _, sim = _kh_sim(n, ti.euler_explicit)
    _, ref = _kh_sim(n, ti.euler_explicit)
    u0 = _random_state((n[2], n[1], n[0]), rng)
    for s in (sim, ref):
        CL.upload_dense(s, torch.from_numpy(u0).cuda())
        s.set_time(0.0, math.inf, 0.4)
    c.attach(sim, beta=0.5)
    dt = 1e-3
    sim.step(1, dt=dt)
    ref.step(1, dt=dt)
    plain = CL.download_dense(ref)
    c.features(torch.from_numpy(u0).cuda())
    c.forward()
    nsw = c.correct_dense(torch.from_numpy(u0).cuda(), plain, 1.0, dt, 0.5, (1 / n[0], 1 / n[1], 1 / n[2]))
    ours = CL.download_dense(sim).cpu().numpy()
    assert np.array_equal(ours, plain.cpu().numpy())
    assert CL.Closure.switch_count(sim) == nsw
    assert not np.array_equal(ours, CL.download_dense(ref).cpu().numpy())


def test_attached_ssprk3_step_matches_oracle_composition():
    import torch
    from multiphysics_fvm_b200 import closure as CL
    n = (32, 32, 16)
    rng = np.random.default_rng(7)
    c = _closure(n, out_scale=np.full(5, 0.02))
    c.set_weights(_rand_params(rng))
    s, sim = _kh_sim(n)
    u0 = _random_state((n[2], n[1], n[0]), rng)
    CL.upload_dense(sim, torch.from_numpy(u0).cuda())
    sim.set_time(0.0, math.inf, 0.4)
    c.attach(sim, beta=0.5)
    dt = 1e-3
    sim.step(1, dt=dt)
    ours = CL.download_dense(sim).cpu().numpy().astype(np.float64)
    Z3 = c.buffer(3).astype(np.float64)  # from the step's base state
    # oracle: float64 residual (reference layout), the correction after each stage
    geo = O.Geometry("cartesian", s["grid_config"])
    prm = s["physical_parameters"]
    sch = dict(reconstructor="muscl", slope_limiter="minmod", riemann_solver="hll")
    bcs = [{sd: ("periodic", 0.0) for sd in O.SIDES} for _ in range(5)]
    h = (1 / n[0], 1 / n[1], 1 / n[2])

    def to_ref(d):  # dense (5, n3, n2, n1) -> ghosted (5, n1+2, n2+2, n3+2)
        U = np.zeros((5, n[0] + 2, n[1] + 2, n[2] + 2))
        U[:, 1:-1, 1:-1, 1:-1] = np.transpose(d, (0, 3, 2, 1))
        return U

    def from_ref(U):
        return np.transpose(U[:, 1:-1, 1:-1, 1:-1], (0, 3, 2, 1))

    def L(d):
        U = to_ref(d)
        O.apply_bcs(U, bcs)
        return np.transpose(O.ns_rhs(U, geo, prm, sch), (0, 3, 2, 1))

    s_out = np.array(c.norm["out_scale"])
    U0 = u0.astype(np.float64)
    U1, _ = co.correct(U0, U0 + dt * L(U0), Z3, s_out, 0.5, GAMMA, 1.0, dt, h)
    U2, _ = co.correct(U1, 0.75 * U0 + 0.25 * (U1 + dt * L(U1)), Z3, s_out, 0.5, GAMMA, 0.25, dt, h)
    U3, _ = co.correct(U2, U0 / 3 + 2.0 / 3.0 * (U2 + dt * L(U2)), Z3, s_out, 0.5, GAMMA, 2.0 / 3.0, dt, h)
    plain = U0.copy()
    Up = to_ref(U0)
    O.integrate("rk3_ssp", "navier_stokes", Up, dt, prm, geo, sch, bcs)
    plain = from_ref(Up)
    err = np.max(np.abs(ours - U3)) / np.max(np.abs(U3 - U0))
    gain = np.max(np.abs(U3 - plain)) / np.max(np.abs(U3 - U0))
    assert gain > 1e-3        # the closure changes the step measurably
    assert err < 2e-3 * 1.0   # float32 stages against float64 (relative to the update size)
    assert CL.Closure.switch_count(sim) == 0
