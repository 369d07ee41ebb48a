"""The learned warm start: a GELU MLP on the tensor cores (csrc/mlp.cu) that
maps one grid cell of one case to its steady primitive state, trained on
solved cases and used to start new solves closer to their steady state.
The reference has no counterpart; the solver's own residual still decides
convergence, so a warm start changes the path, not the answer.

A sample is the cell centroid (x, r) in body diameters and 8 case values
(nose family one-hot, fineness / 5, body length / 8, Mach / 5); a target is
(log rho / rho_inf, u / u_inf, v / u_inf, log p / p_inf).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native

FAMILIES = ("conical", "ogive", "parabolic", "ellipsoid", "haack")
SAMPLE = 10
TARGET = 4
FEATURES = 128
OUT_PAD = 128


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class WarmStartNet:
    """`hidden_layers` GELU layers of width 256; `batch` samples per Adam step."""

    def __init__(self, hidden_layers: int = 5, batch: int = 16384, seed: int = 1, width: int = 256):
        self._lib = _native.load()
        self.hidden_layers = hidden_layers
        self.batch = batch
        h = C.c_void_p()
        _native.check(self._lib.bs_mlp_create(hidden_layers, width, batch, seed, C.byref(h)), self._lib)
        self._h = h

    def destroy(self) -> None:
        if self._h:
            _native.check(self._lib.bs_mlp_destroy(self._h), self._lib)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def _call(self, name: str, *args) -> None:
        _native.check(getattr(self._lib, name)(self._h, *args), self._lib)

    def layer_shapes(self) -> list[tuple[int, int]]:
        """(out, in) of every layer's weight matrix."""
        dims = [FEATURES] + [256] * self.hidden_layers + [OUT_PAD]
        return [(dims[k + 1], dims[k]) for k in range(len(dims) - 1)]

    def param_count(self) -> int:
        n = C.c_int64()
        self._call("bs_mlp_param_count", C.byref(n))
        return n.value

    def params(self) -> np.ndarray:
        out = np.empty(self.param_count(), np.float32)
        self._call("bs_mlp_get_params", _ptr(out))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.param_count():
            raise ValueError("parameter count")
        self._call("bs_mlp_set_params", _ptr(p))

    def set_data(self, samples: np.ndarray, targets: np.ndarray) -> None:
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, SAMPLE)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1, TARGET)
        if len(s) != len(t):
            raise ValueError("samples and targets differ in length")
        self._call("bs_mlp_set_data", len(s), _ptr(s), _ptr(t))

    def train(self, steps: int, lr: float, seed: int = 1) -> np.ndarray:
        losses = np.empty(steps, np.float32)
        self._call("bs_mlp_train", steps, float(lr), seed, _ptr(losses))
        return losses

    def loss_grad(self, samples: np.ndarray, targets: np.ndarray) -> tuple[float, np.ndarray]:
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, SAMPLE)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1, TARGET)
        loss = np.zeros(1, np.float32)
        grads = np.empty(self.param_count(), np.float32)
        self._call("bs_mlp_loss_grad", len(s), _ptr(s), _ptr(t), _ptr(loss), _ptr(grads))
        return float(loss[0]), grads

    def predict(self, samples: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(samples, np.float32).reshape(-1, SAMPLE)
        out = np.empty((len(s), TARGET), np.float32)
        self._call("bs_mlp_predict", len(s), _ptr(s), _ptr(out))
        return out


# ---- samples and targets of a case --------------------------------------------

def case_values(case) -> np.ndarray:
    """The 8 case values of a workloads.Case."""
    nose = case.body.nose
    diameter = 2 * nose.base_radius
    v = np.zeros(8, np.float32)
    v[FAMILIES.index(nose.shape.kind)] = 1.0
    v[5] = nose.length / diameter / 5.0
    v[6] = (nose.length + case.body.cylinder_length) / diameter / 8.0
    v[7] = case.mach / 5.0
    return v


def cell_centroids(grid) -> tuple[np.ndarray, np.ndarray]:
    """Cell centres (mean of the four nodes), i fastest, in body diameters
    (grids are in body diameters already)."""
    X = grid.x.reshape(grid.nj + 1, grid.ni + 1)
    Y = grid.y.reshape(grid.nj + 1, grid.ni + 1)
    cx = 0.25 * (X[:-1, :-1] + X[:-1, 1:] + X[1:, :-1] + X[1:, 1:])
    cy = 0.25 * (Y[:-1, :-1] + Y[:-1, 1:] + Y[1:, :-1] + Y[1:, 1:])
    return cx.ravel(), cy.ravel()


def case_samples(case) -> np.ndarray:
    cx, cy = cell_centroids(case.config.grid)
    s = np.empty((len(cx), SAMPLE), np.float32)
    s[:, 0] = cx
    s[:, 1] = cy
    s[:, 2:] = case_values(case)
    return s


def targets_from_primitives(prims: np.ndarray, free) -> np.ndarray:
    """(rho, u, v, p) per cell to the network's normalised targets."""
    w = np.asarray(prims, np.float64).reshape(-1, 4)
    st = free.state
    speed = max(abs(st.u), 1e-12)
    t = np.empty((len(w), TARGET), np.float32)
    t[:, 0] = np.log(w[:, 0] / st.rho)
    t[:, 1] = w[:, 1] / speed
    t[:, 2] = w[:, 2] / speed
    t[:, 3] = np.log(w[:, 3] / st.p)
    return t


def primitives_from_prediction(pred: np.ndarray, free) -> np.ndarray:
    """The network's outputs back to (rho, u, v, p) per cell, flat."""
    p = np.asarray(pred, np.float64).reshape(-1, TARGET)
    st = free.state
    speed = abs(st.u)
    w = np.empty((len(p), 4))
    w[:, 0] = st.rho * np.exp(np.clip(p[:, 0], -20, 20))
    w[:, 1] = p[:, 1] * speed
    w[:, 2] = p[:, 2] * speed
    w[:, 3] = st.p * np.exp(np.clip(p[:, 3], -20, 20))
    return w.ravel()
