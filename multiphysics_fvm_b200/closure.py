"""Learned flux-correction closure (host side).

The reference has no learned part.  This module drives the device network of
``include/fvm_closure.h``: a periodic 3x3x3 CNN (16 -> 32 -> 32 -> 16
channels, BF16 on the tensor cores) mapping the normalised primitive
variables of a coarse navier_stokes state to corrections of the MUSCL face
fluxes (output channel ``a*5 + q``: variable ``q`` on the ``+x_a`` face).
Attached to a :class:`~multiphysics_fvm_b200.backend.Simulation`, every step
runs the network on the step's base state and, after each Runge-Kutta stage,
adds the clipped, positivity-gated correction of that stage's residual.

Device arrays ("dense" states) are torch CUDA tensors of shape
``(5, n3, n2, n1)`` float32 (x1 fastest); torch is only the allocator here.
"""
from __future__ import annotations

import ctypes as C
import json

import numpy as np

from . import _lib as L

CB_X0, CB_A1, CB_A2, CB_Z3, CB_G3, CB_G2, CB_G1, CB_E = range(8)
LAYER_DIMS = [(32, 16), (32, 32), (16, 32)]  # (cout, cin)
_BUF = {CB_X0: (16, "bf16"), CB_A1: (32, "bf16"), CB_A2: (32, "bf16"), CB_Z3: (16, "f32"),
        CB_G3: (16, "bf16"), CB_G2: (32, "bf16"), CB_G1: (32, "bf16"), CB_E: (5, "f32")}


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise L.FvmError("the closure needs a CUDA device (there is no CPU fallback)")
    return torch


def _dev_ptr(t, shape=None):
    torch = _torch()
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise ValueError("expected a contiguous float32 CUDA tensor")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"tensor shape {tuple(t.shape)} != {tuple(shape)}")
    return C.c_void_p(t.data_ptr())


def bf16_to_f32(u16: np.ndarray) -> np.ndarray:
    return (u16.astype(np.uint32) << 16).view(np.float32)


def f32_to_bf16(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even float32 -> bfloat16 bits (as the device does)."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((b >> 16) & 1) + 0x7FFF
    return ((b + r) >> 16).astype(np.uint16)


class Closure:
    """Network, Adam state and workspace for one periodic grid (n1, n2, n3)."""

    def __init__(self, n, seed: int = 0):
        self._lib = L.load()
        self.n = tuple(int(x) for x in n)
        h = C.c_void_p()
        L.check(self._lib.fvm_closure_create(self.n[0], self.n[1], self.n[2], C.c_ulonglong(seed), C.byref(h)),
                "fvm_closure_create")
        self._h = h
        self.npos = self.n[0] * self.n[1] * self.n[2]
        self.norm = None
        self.fct = False
        self.meta = {}  # metadata of the loaded weights (selection beta, fct, ...)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.fvm_closure_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def dense_shape(self):
        return (5, self.n[2], self.n[1], self.n[0])

    # -- parameters ------------------------------------------------------------
    def set_norm(self, gamma, in_mean, in_scale, out_scale, loss_weight):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (in_mean, in_scale, out_scale, loss_weight)]
        L.check(self._lib.fvm_closure_set_norm(self._h, float(gamma), *[L.dptr(a) for a in arrs]),
                "fvm_closure_set_norm")
        self.norm = {"gamma": float(gamma), "in_mean": arrs[0].tolist(), "in_scale": arrs[1].tolist(),
                     "out_scale": arrs[2].tolist(), "loss_weight": arrs[3].tolist()}

    def set_limiter(self, fct: bool):
        """True: flux-corrected transport bound on top of the face clip (no
        new extrema); set before ``attach``."""
        L.check(self._lib.fvm_closure_set_limiter(self._h, 1 if fct else 0), "fvm_closure_set_limiter")
        self.fct = bool(fct)

    def get_weights(self):
        out = []
        for layer, (co, ci) in enumerate(LAYER_DIMS, start=1):
            w = np.empty((27, co, ci), np.float32)
            b = np.empty(co, np.float32)
            L.check(self._lib.fvm_closure_get_weights(self._h, layer, w.ctypes.data, b.ctypes.data),
                    "fvm_closure_get_weights")
            out.append((w, b))
        return out

    def set_weights(self, layers):
        for layer, ((w, b), (co, ci)) in enumerate(zip(layers, LAYER_DIMS), start=1):
            w = np.ascontiguousarray(w, dtype=np.float32).reshape(27, co, ci)
            b = np.ascontiguousarray(b, dtype=np.float32).reshape(co)
            L.check(self._lib.fvm_closure_set_weights(self._h, layer, w.ctypes.data, b.ctypes.data),
                    "fvm_closure_set_weights")

    def get_grads(self):
        out = []
        for layer, (co, ci) in enumerate(LAYER_DIMS, start=1):
            w = np.empty((27, co, ci), np.float32)
            b = np.empty(co, np.float32)
            L.check(self._lib.fvm_closure_get_grads(self._h, layer, w.ctypes.data, b.ctypes.data),
                    "fvm_closure_get_grads")
            out.append((w, b))
        return out

    def save(self, path: str, meta: dict | None = None):
        d = {}
        for i, (w, b) in enumerate(self.get_weights(), start=1):
            d[f"W{i}"], d[f"b{i}"] = w, b
        d["norm"] = np.array(json.dumps(self.norm))
        d["meta"] = np.array(json.dumps(meta or {}))
        np.savez(path, **d)

    def load(self, path: str) -> dict:
        z = np.load(path)
        self.set_weights([(z[f"W{i}"], z[f"b{i}"]) for i in (1, 2, 3)])
        norm = json.loads(str(z["norm"]))
        if norm:
            self.set_norm(norm["gamma"], norm["in_mean"], norm["in_scale"], norm["out_scale"], norm["loss_weight"])
        self.meta = json.loads(str(z["meta"])) if "meta" in z else {}
        return self.meta

    # -- workspace access (tests) ----------------------------------------------
    def buffer(self, which: int) -> np.ndarray:
        ch, kind = _BUF[which]
        n = self.npos * ch
        raw = np.empty(n, np.uint16 if kind == "bf16" else np.float32)
        L.check(self._lib.fvm_closure_buffer(self._h, which, raw.ctypes.data, raw.nbytes, 0), "fvm_closure_buffer")
        vals = bf16_to_f32(raw) if kind == "bf16" else raw
        if which == CB_E:
            return vals.reshape(5, self.n[2], self.n[1], self.n[0])
        return vals.reshape(self.n[2], self.n[1], self.n[0], ch)

    def set_buffer(self, which: int, values: np.ndarray):
        ch, kind = _BUF[which]
        v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
        raw = f32_to_bf16(v) if kind == "bf16" else v
        L.check(self._lib.fvm_closure_buffer(self._h, which, raw.ctypes.data, raw.nbytes, 1), "fvm_closure_buffer")

    # -- network ------------------------------------------------------------------
    def features(self, u):
        L.check(self._lib.fvm_closure_features(self._h, _dev_ptr(u, self.dense_shape)), "fvm_closure_features")

    def forward(self):
        L.check(self._lib.fvm_closure_forward(self._h), "fvm_closure_forward")

    def backward(self, defect, dt: float, h):
        hh = np.ascontiguousarray(h, dtype=np.float64)
        L.check(self._lib.fvm_closure_backward(self._h, _dev_ptr(defect, self.dense_shape), float(dt), L.dptr(hh)),
                "fvm_closure_backward")

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        L.check(self._lib.fvm_closure_adam(self._h, float(lr), float(beta1), float(beta2), float(eps)),
                "fvm_closure_adam")

    def train_step(self, u, defect, dt: float, h, lr: float = 1e-3):
        hh = np.ascontiguousarray(h, dtype=np.float64)
        L.check(self._lib.fvm_closure_train_step(self._h, _dev_ptr(u, self.dense_shape),
                                                 _dev_ptr(defect, self.dense_shape), float(dt), L.dptr(hh),
                                                 float(lr)), "fvm_closure_train_step")

    def time_forward(self, iters: int = 20) -> float:
        """Device ms per forward pass (from the current features)."""
        v = C.c_double()
        L.check(self._lib.fvm_closure_time_forward(self._h, int(iters), C.byref(v)), "fvm_closure_time_forward")
        return v.value

    def time_train(self, u, defect, dt: float, h, lr: float = 1e-3, iters: int = 20) -> float:
        """Device ms per full training step (the weights change)."""
        hh = np.ascontiguousarray(h, dtype=np.float64)
        v = C.c_double()
        L.check(self._lib.fvm_closure_time_train(self._h, _dev_ptr(u, self.dense_shape),
                                                 _dev_ptr(defect, self.dense_shape), float(dt), L.dptr(hh),
                                                 float(lr), int(iters), C.byref(v)), "fvm_closure_time_train")
        return v.value

    def loss(self) -> float:
        v = C.c_double()
        L.check(self._lib.fvm_closure_loss(self._h, C.byref(v)), "fvm_closure_loss")
        return v.value

    def correct_dense(self, uin, uout, coef: float, dt: float, beta: float, h) -> int:
        hh = np.ascontiguousarray(h, dtype=np.float64)
        n = C.c_ulonglong()
        L.check(self._lib.fvm_closure_correct_dense(self._h, _dev_ptr(uin, self.dense_shape),
                                                    _dev_ptr(uout, self.dense_shape), float(coef), float(dt),
                                                    float(beta), L.dptr(hh), C.byref(n)),
                "fvm_closure_correct_dense")
        return n.value

    # -- solver hook ---------------------------------------------------------------
    # the clip factor used when neither the caller nor the weights' metadata gives one
    DEFAULT_BETA = 0.05

    def attach(self, sim, beta: float | None = None):
        """Run the network in every step of ``sim``.  ``beta`` scales the face
        clip; None takes the value the loaded weights were selected with
        (their metadata), else DEFAULT_BETA."""
        if beta is None:
            beta = float(self.meta.get("beta", self.DEFAULT_BETA))
        L.check(self._lib.fvm_closure_attach(sim._h, self._h, float(beta)), "fvm_closure_attach")
        sim._closure = self  # keep the network alive while attached

    @staticmethod
    def detach(sim):
        L.check(L.load().fvm_closure_attach(sim._h, None, 0.0), "fvm_closure_attach")
        sim._closure = None

    @staticmethod
    def switch_count(sim) -> int:
        n = C.c_ulonglong()
        L.check(L.load().fvm_closure_switch_count(sim._h, C.byref(n)), "fvm_closure_switch_count")
        return n.value


# -- dense state transfer between a float32 Simulation and torch ---------------------
def filter_state(sim, factor: int, out=None):
    """f^3 box filter of ``sim``'s state -> dense (5, n3/f, n2/f, n1/f) CUDA tensor."""
    torch = _torch()
    n1, n2, n3 = sim.n
    shape = (sim.nv, n3 // factor, n2 // factor, n1 // factor)
    if out is None:
        out = torch.empty(shape, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    L.check(L.load().fvm_filter_state(sim._h, int(factor), _dev_ptr(out, shape)), "fvm_filter_state")
    return out


def upload_dense(sim, u):
    n1, n2, n3 = sim.n
    _torch().cuda.synchronize()
    L.check(L.load().fvm_upload_dense(sim._h, _dev_ptr(u, (sim.nv, n3, n2, n1))), "fvm_upload_dense")


def download_dense(sim, out=None):
    torch = _torch()
    n1, n2, n3 = sim.n
    shape = (sim.nv, n3, n2, n1)
    if out is None:
        out = torch.empty(shape, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    L.check(L.load().fvm_download_dense(sim._h, _dev_ptr(out, shape)), "fvm_download_dense")
    return out
