"""CPU checks of the closure oracle: its analytic gradients (conv data and
weight gradients, the a-priori loss gradient, the full 3-layer backward pass)
against central finite differences in float64, and its filter/correction
identities.  These pin the oracle that the GPU closure tests compare with."""
import numpy as np
import pytest

from oracle import closure_oracle as co


def rand_params(rng, scale=0.3):
    dims = [(32, 16), (32, 32), (16, 32)]
    return [(rng.normal(0, scale / np.sqrt(27 * ci), (27, cout, ci)), rng.normal(0, 0.05, cout))
            for cout, ci in dims]


def test_conv_adjoints():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(4, 5, 6, 3))
    W = rng.normal(size=(27, 2, 3))
    dY = rng.normal(size=(4, 5, 6, 2))
    Y = co.conv3d(X, W)
    # <conv(X), dY> = <X, dgrad(dY)> = <W, wgrad(X, dY)>
    lhs = np.sum(Y * dY)
    assert np.isclose(lhs, np.sum(X * co.conv3d_dgrad(dY, W)), rtol=1e-12)
    assert np.isclose(lhs, np.sum(W * co.conv3d_wgrad(X, dY)), rtol=1e-12)


def test_conv_direct_sum():
    rng = np.random.default_rng(1)
    X = rng.normal(size=(3, 4, 5, 2))
    W = rng.normal(size=(27, 3, 2))
    Y = co.conv3d(X, W)
    z, y, x = 1, 3, 4
    ref = np.zeros(3)
    for t, (dz, dy, dx) in enumerate(co.OFFSETS):
        ref += W[t] @ X[(z + dz) % 3, (y + dy) % 4, (x + dx) % 5]
    assert np.allclose(Y[z, y, x], ref, rtol=1e-13)


def _loss(params, X0, D, s, w, dt, h):
    _, _, Z3 = co.forward(X0, params)
    return co.loss_and_grad(Z3, D, s, w, dt, h)[0]


def test_full_backward_matches_finite_differences():
    rng = np.random.default_rng(2)
    n3, n2, n1 = 4, 4, 4
    X0 = np.zeros((n3, n2, n1, 16))
    X0[..., :5] = rng.normal(size=(n3, n2, n1, 5))
    params = rand_params(rng, scale=1.0)
    D = rng.normal(size=(5, n3, n2, n1)) * 1e-2
    s, w, dt, h = rng.uniform(0.5, 2, 5), rng.uniform(0.5, 2, 5), 0.01, (0.25, 0.3, 0.2)
    A1, A2, Z3 = co.forward(X0, params)
    _, _, G3 = co.loss_and_grad(Z3, D, s, w, dt, h)
    grads, _, _ = co.backward(X0, A1, A2, G3, params)
    eps = 1e-6
    for layer in range(3):
        W, b = params[layer]
        for _ in range(4):
            idx = tuple(rng.integers(0, d) for d in W.shape)
            old = W[idx]
            W[idx] = old + eps
            lp = _loss(params, X0, D, s, w, dt, h)
            W[idx] = old - eps
            lm = _loss(params, X0, D, s, w, dt, h)
            W[idx] = old
            fd = (lp - lm) / (2 * eps)
            assert np.isclose(grads[layer][0][idx], fd, rtol=1e-4, atol=1e-9), (layer, idx)
        k = int(rng.integers(0, b.shape[0]))
        old = b[k]
        b[k] = old + eps
        lp = _loss(params, X0, D, s, w, dt, h)
        b[k] = old - eps
        lm = _loss(params, X0, D, s, w, dt, h)
        b[k] = old
        assert np.isclose(grads[layer][1][k], (lp - lm) / (2 * eps), rtol=1e-4, atol=1e-9)


def test_correction_divergence_is_conservative_and_exact_for_uniform_flux():
    rng = np.random.default_rng(3)
    Z3 = rng.normal(size=(4, 6, 8, 16))
    s = np.ones(5)
    R = co.correction_divergence(Z3, s, (0.1, 0.2, 0.3))
    assert np.allclose(R.sum(axis=(1, 2, 3)), 0.0, atol=1e-10)  # periodic: a pure flux difference
    Zc = np.broadcast_to(rng.normal(size=16), Z3.shape)
    assert np.allclose(co.correction_divergence(Zc, s, (0.1, 0.2, 0.3)), 0.0)


def test_correct_respects_bounds_and_positivity():
    rng = np.random.default_rng(4)
    n = (4, 4, 8)
    rho = rng.uniform(0.5, 2, n)
    v = rng.normal(0, 0.3, (3,) + n)
    p = rng.uniform(1, 3, n)
    u = np.stack([rho, rho * v[0], rho * v[1], rho * v[2], p / 0.4 + 0.5 * rho * (v * v).sum(0)])
    Z3 = rng.normal(0, 1, n + (16,))
    new, nsw = co.correct(u, u.copy(), Z3, np.ones(5), 0.0, 1.4, 1.0, 0.01, (0.1, 0.1, 0.1))
    assert nsw == 0 and np.array_equal(new, u)   # beta = 0: no correction
    big, nsw = co.correct(u, u.copy(), Z3 * 1e6, np.ones(5), 1e6, 1.4, 1.0, 10.0, (0.1, 0.1, 0.1))
    rho2, _, p2 = co.primitives(big, 1.4)
    assert nsw > 0 and np.all(rho2 > 0) and np.all(p2 > 0)  # switched-off cells keep the plain state


def test_box_filter_conserves_totals():
    rng = np.random.default_rng(5)
    U = rng.normal(size=(5, 8, 8, 16))
    Ub = co.box_filter(U, 4)
    assert Ub.shape == (5, 2, 2, 4)
    assert np.allclose(Ub.sum(axis=(1, 2, 3)) * 64, U.sum(axis=(1, 2, 3)))


def test_adam_first_step_is_signed_lr():
    p = np.array([1.0, -2.0, 3.0])
    g = np.array([0.5, -0.1, 0.0])
    m, v = np.zeros(3), np.zeros(3)
    co.adam(p, g, m, v, 1, lr=1e-3)
    assert np.allclose(p, [1.0 - 1e-3, -2.0 + 1e-3, 3.0], atol=1e-9)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -1.5, 3.14159], np.float32)
    r = co.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -1.5
    assert abs(r[4] - 3.14159) < 2 ** -7 * 4


def test_fct_correction_creates_no_new_extrema_and_conserves():
    rng = np.random.default_rng(6)
    n = (4, 6, 8)
    rho = rng.uniform(1.0, 2.0, n)
    v = rng.normal(0, 0.3, (3,) + n)
    p = rng.uniform(2, 3, n)
    u = np.stack([rho, rho * v[0], rho * v[1], rho * v[2], p / 0.4 + 0.5 * rho * (v * v).sum(0)])
    Z3 = rng.normal(0, 1, n + (16,))
    big, nsw = co.correct(u, u.copy(), Z3, np.ones(5), 1e3, 1.4, 1.0, 1e-2, (0.1, 0.1, 0.1), fct=True)
    hi, lo = u.copy(), u.copy()
    for ax in (1, 2, 3):
        for sh in (1, -1):
            hi, lo = np.maximum(hi, np.roll(u, sh, axis=ax)), np.minimum(lo, np.roll(u, sh, axis=ax))
    assert nsw == 0
    assert np.all(big <= hi + 1e-12) and np.all(big >= lo - 1e-12)
    assert np.allclose(big.sum(axis=(1, 2, 3)), u.sum(axis=(1, 2, 3)), rtol=1e-12)
    assert np.max(np.abs(big - u)) > 1e-3  # the limited correction still acts
