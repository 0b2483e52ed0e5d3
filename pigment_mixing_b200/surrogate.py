"""Return-map surrogate: data logging, GPU training and loading (thin layer over the C ABI).

The network (10 -> 64 -> 64 -> 6, GELU) is trained by the library's own FP32 forward/backward
kernels (``pm_mlp_train``) on samples the plain return map logs (``Simulation.enableSampleLog``),
and runs in the step as BF16 tensor-core inference with a consistency check (``Simulation.
setSurrogate`` + ``setReturnMap(RETURN_MAP_SURROGATE)``).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import call

NPARAMS = 5286
FEATURES = ("h0", "h1", "h2", "rate0", "rate1", "rate2", "yield", "viscosity", "flow_index", "E")
TARGETS = ("dh0", "dh1", "dh2", "dh_rate0", "dh_rate1", "dh_rate2")


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def train(x, y, epochs: int = 20, batch: int = 8192, lr: float = 3e-3, seed: int = 0, params=None):
    """Train on the current GPU; returns (params[NPARAMS], loss_history[epochs])."""
    x = np.ascontiguousarray(x, np.float32).reshape(-1, 10)
    y = np.ascontiguousarray(y, np.float32).reshape(-1, 6)
    p = np.zeros(NPARAMS, np.float32) if params is None else np.ascontiguousarray(params, np.float32).copy()
    hist = np.zeros(max(epochs, 1), np.float32)
    steps = C.c_uint32()
    call("pm_mlp_train", _fp(x), _fp(y), x.shape[0], int(epochs), int(batch), float(lr), int(seed),
         0 if params is None else 1, _fp(p), _fp(hist), C.byref(steps))
    return p, hist[:epochs]


def loss_grad(params, x, y):
    """(loss, grad[NPARAMS]) of one batch from the GPU training kernels."""
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32).reshape(-1, 10)
    y = np.ascontiguousarray(y, np.float32).reshape(-1, 6)
    loss = C.c_float()
    g = np.zeros(NPARAMS, np.float32)
    call("pm_mlp_loss_grad", _fp(p), _fp(x), _fp(y), x.shape[0], C.byref(loss), _fp(g))
    return float(loss.value), g


def infer(params, x):
    """BF16 tensor-core inference of raw features x[n,10] -> raw outputs [n,6]."""
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(x, np.float32).reshape(-1, 10)
    y = np.zeros((x.shape[0], 6), np.float32)
    call("pm_mlp_infer", _fp(p), _fp(x), x.shape[0], _fp(y))
    return y
