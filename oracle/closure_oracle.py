"""CPU oracle for the learned flux-correction closure (test infrastructure only:
imported by tests/ and nowhere in the product path).

The reference (nathanzimniak/multiphysics-fvm) has no learned closure, so
there is nothing of it to pin this file to: it is a float64 NumPy statement of
the network, training and correction pieces the device kernels implement, used
as their value and gradient checker.  Its own gradients are pinned by finite
differences (tests/test_closure_oracle.py).  The closure acts on the MUSCL
face fluxes of the reference's navier_stokes residual
(src/physics/navier_stokes.py:627-660) inside the SSPRK3 stages
(src/numerics/time_integrators.py:106-159).

Conventions (shared with the device code):
* position arrays are (n3, n2, n1, C), x1 fastest; dense states (5, n3, n2, n1);
* tap t = (dz+1)*9 + (dy+1)*3 + (dx+1) for offsets in {-1, 0, 1}, weights
  W[t][co][ci]; all convolutions are periodic;
* output channel a*5 + q is the flux correction of conserved variable q on
  the +x_a face of a cell (a = 0, 1, 2 for x1, x2, x3), in units of s[q].
"""
from __future__ import annotations

import numpy as np

OFFSETS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def bf16(x):
    """Round to bfloat16 (nearest even) and return float64 values."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((b >> 16) & 1) + 0x7FFF
    return (((b + r) >> 16) << 16).astype(np.uint32).view(np.float32).astype(np.float64)


def conv3d(X, W, b=None):
    """Y[p, co] = sum_t sum_ci X[p + off_t, ci] W[t, co, ci] (+ b[co])."""
    Y = np.zeros(X.shape[:3] + (W.shape[1],))
    for t, (dz, dy, dx) in enumerate(OFFSETS):
        Xs = np.roll(X, shift=(-dz, -dy, -dx), axis=(0, 1, 2))
        Y += Xs @ W[t].T
    if b is not None:
        Y += b
    return Y


def conv3d_dgrad(dY, W):
    """dX[p, ci] = sum_t sum_co dY[p - off_t, co] W[t, co, ci]."""
    dX = np.zeros(dY.shape[:3] + (W.shape[2],))
    for t, (dz, dy, dx) in enumerate(OFFSETS):
        dYs = np.roll(dY, shift=(dz, dy, dx), axis=(0, 1, 2))
        dX += dYs @ W[t]
    return dX


def conv3d_wgrad(X, dY):
    """dW[t, co, ci] = sum_p dY[p, co] X[p + off_t, ci]."""
    C_out, C_in = dY.shape[3], X.shape[3]
    dW = np.zeros((27, C_out, C_in))
    Yf = dY.reshape(-1, C_out)
    for t, (dz, dy, dx) in enumerate(OFFSETS):
        Xs = np.roll(X, shift=(-dz, -dy, -dx), axis=(0, 1, 2)).reshape(-1, C_in)
        dW[t] = Yf.T @ Xs
    return dW


def relu(x):
    return np.maximum(x, 0.0)


def primitives(u, gamma):
    rho = u[0]
    v = u[1:4] / rho
    p = (gamma - 1.0) * (u[4] - 0.5 * rho * (v * v).sum(0))
    return rho, v, p


def features(u, gamma, mean, scale):
    """(rho, v1, v2, v3, p) normalised, channels 5..15 zero: (n3, n2, n1, 16)."""
    rho, v, p = primitives(np.asarray(u, np.float64), gamma)
    f = np.stack([rho, v[0], v[1], v[2], p])
    h = (f - np.asarray(mean)[:, None, None, None]) / np.asarray(scale)[:, None, None, None]
    X = np.zeros(u.shape[1:] + (16,))
    X[..., :5] = np.moveaxis(h, 0, -1)
    return X


def forward(X0, params):
    """params = [(W1, b1), (W2, b2), (W3, b3)] -> A1, A2, Z3."""
    (W1, b1), (W2, b2), (W3, b3) = params
    A1 = relu(conv3d(X0, W1, b1))
    A2 = relu(conv3d(A1, W2, b2))
    return A1, A2, conv3d(A2, W3, b3)


def _axis(a):
    """Array axis of face direction a in a (n3, n2, n1) array."""
    return 2 - a


def correction_divergence(Z3, s, h):
    """R[q] = -sum_a (F_a(p) - F_a(p - e_a)) / h_a with F_a = s_q Z3[..., a*5+q]; (5, n3, n2, n1)."""
    R = np.zeros((5,) + Z3.shape[:3])
    for a in range(3):
        for q in range(5):
            F = s[q] * Z3[..., a * 5 + q]
            R[q] -= (F - np.roll(F, 1, axis=_axis(a))) / h[a]
    return R


def loss_and_grad(Z3, D, s, w, dt, h):
    """A-priori loss of the network output against the target defect D:
    E = dt R(Z3) - D, loss = sum_q w_q sum_p E^2 / N, and dLoss/dZ3."""
    N = Z3.shape[0] * Z3.shape[1] * Z3.shape[2]
    E = dt * correction_divergence(Z3, s, h) - D
    loss = float(sum(w[q] * np.sum(E[q] ** 2) for q in range(5)) / N)
    G3 = np.zeros(Z3.shape[:3] + (16,))
    for a in range(3):
        for q in range(5):
            G3[..., a * 5 + q] = s[q] * (dt / h[a]) * (2.0 * w[q] / N) * (np.roll(E[q], -1, axis=_axis(a)) - E[q])
    return loss, E, G3


def backward(X0, A1, A2, G3, params):
    """Weight/bias gradients and the masked data gradients G2, G1."""
    (W1, _), (W2, _), (W3, _) = params
    dW3, db3 = conv3d_wgrad(A2, G3), G3.sum(axis=(0, 1, 2))
    G2 = conv3d_dgrad(G3, W3) * (A2 > 0)
    dW2, db2 = conv3d_wgrad(A1, G2), G2.sum(axis=(0, 1, 2))
    G1 = conv3d_dgrad(G2, W2) * (A1 > 0)
    dW1, db1 = conv3d_wgrad(X0, G1), G1.sum(axis=(0, 1, 2))
    return [(dW1, db1), (dW2, db2), (dW3, db3)], G2, G1


def adam(param, grad, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (Kingma & Ba 2015) in place; step counts from 1."""
    m[...] = b1 * m + (1 - b1) * grad
    v[...] = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    param[...] = param - lr * mh / (np.sqrt(vh) + eps)


def box_filter(U, f):
    """Volume average over f^3 blocks: dense (NV, n3, n2, n1) -> (NV, n3/f, n2/f, n1/f)."""
    nv, a, b, c = U.shape
    return U.reshape(nv, a // f, f, b // f, f, c // f, f).mean(axis=(2, 4, 6))


def correct(uin, uout, Z3, s, beta, gamma, coef, dt, h, fct=False):
    """Per-stage correction: face flux corrections s_q Z3 clipped to
    +-beta * max(|v_a| + c) * |U_q(p + e_a) - U_q(p)| (taken from the stage
    input uin), their divergence added to uout with weight coef*dt, and cells
    whose result has rho <= 0 or p <= 0 left at uout.  With ``fct`` the face
    transfers are first limited by flux-corrected transport (Zalesak 1979):
    the result stays within the min/max of uout over each cell and its six
    face neighbours.  Returns (new, count)."""
    uin = np.asarray(uin, np.float64)
    rho, v, p = primitives(uin, gamma)
    c = np.where((p > 0) & (rho > 0), np.sqrt(np.abs(gamma * p / rho)), 0.0)
    T = np.zeros((3,) + uin.shape)  # transfer through the +x_a face, from the cell to its upper neighbour
    for a in range(3):
        ax = _axis(a)
        sp = np.abs(v[a]) + c
        smax = np.maximum(sp, np.roll(sp, -1, axis=ax))
        for q in range(5):
            bound = beta * smax * np.abs(np.roll(uin[q], -1, axis=ax) - uin[q])
            T[a, q] = coef * dt * np.clip(s[q] * Z3[..., a * 5 + q], -bound, bound) / h[a]
    if fct:
        hi, lo = uout.copy(), uout.copy()
        pin, pout = np.zeros_like(uout), np.zeros_like(uout)
        for a in range(3):
            ax = _axis(a)
            for sh in (1, -1):
                nbv = np.roll(uout, sh, axis=ax + 1)
                hi, lo = np.maximum(hi, nbv), np.minimum(lo, nbv)
            tin = [-T[a], np.roll(T[a], 1, axis=ax + 1)]  # inflow through the +face and the -face
            for t in tin:
                pin += np.maximum(t, 0.0)
                pout += np.maximum(-t, 0.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            Rp = np.where(pin > 0, np.minimum(1.0, (hi - uout) / pin), 1.0)
            Rm = np.where(pout > 0, np.minimum(1.0, (uout - lo) / pout), 1.0)
        for a in range(3):
            ax = _axis(a) + 1
            Rp_up, Rm_up = np.roll(Rp, -1, axis=ax), np.roll(Rm, -1, axis=ax)
            T[a] *= np.where(T[a] >= 0, np.minimum(Rp_up, Rm), np.minimum(Rp, Rm_up))
    R = np.zeros_like(uin)
    for a in range(3):
        R -= T[a] - np.roll(T[a], 1, axis=_axis(a) + 1)
    un = uout + R
    ke = 0.5 * (un[1] ** 2 + un[2] ** 2 + un[3] ** 2) / un[0]
    pr = (gamma - 1.0) * (un[4] - ke)
    ok = (un[0] > 0) & (pr > 0) & np.isfinite(pr)
    return np.where(ok[None], un, uout), int((~ok).sum())
