"""Learned ACA rank prediction: the library's 6 -> 64 -> 64 -> 1 perceptron
(BF16 weights, FP32 accumulation; training and inference are the library's
own CUDA kernels) over the features of a box's ACA problem.

Typical use: build a solver once with the fixed workspace bound, read its
ACA log (features and the ranks the adaptive ACA found), fit a model, and
install it on a context so that later solvers size each box's workspace from
the prediction.  The adaptive ACA (src/ACA.cpp:639-859) still decides every
rank; a box whose prediction was too small is rerun with a larger bound.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .kernel import Context, default_context

N_FEATURES = 6
FEATURES = ("centre distance / box side", "wavenumber x box side", "log2(1 + rows)", "log2(1 + columns)",
            "tree level", "leaf")


def num_params() -> int:
    n = C.c_int()
    _lib.check(_lib.lib().aifmm_mlp_num_params(C.byref(n)))
    return n.value


def _f32(a, cols=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    if cols is not None:
        a = a.reshape(-1, cols)
    return a


class RankMLP:
    """aifmm_mlp: the rank model on one context."""

    def __init__(self, ctx: Context | None = None, seed: int = 1):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        _lib.check(_lib.lib().aifmm_mlp_create(self.ctx.h, C.c_ulonglong(seed), C.byref(h)))
        self.h = h
        self.mean = np.zeros(N_FEATURES, dtype=np.float32)
        self.scale = np.ones(N_FEATURES, dtype=np.float32)

    def close(self):
        if getattr(self, "h", None):
            _lib.lib().aifmm_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_normalization(self, mean, scale) -> None:
        self.mean = _f32(mean).ravel()
        self.scale = _f32(scale).ravel()
        _lib.check(_lib.lib().aifmm_mlp_set_normalization(self.h, self.mean, self.scale))

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(num_params(), dtype=np.float32)
        _lib.check(_lib.lib().aifmm_mlp_get_params(self.h, out))
        return out

    @params.setter
    def params(self, p) -> None:
        _lib.check(_lib.lib().aifmm_mlp_set_params(self.h, _f32(p).ravel()))

    def infer(self, X) -> np.ndarray:
        """Predicted log2(1 + rank) for raw feature rows X (n x 6)."""
        X = _f32(X, N_FEATURES)
        y = np.zeros(len(X), dtype=np.float32)
        _lib.check(_lib.lib().aifmm_mlp_infer(self.h, X.ravel(), len(X), y))
        return y

    def predict_rank(self, X) -> np.ndarray:
        return np.maximum(0.0, np.exp2(self.infer(X).astype(np.float64)) - 1.0)

    def grad(self, X, t) -> tuple[np.ndarray, float]:
        """Gradient of the mean squared error against targets t, and the loss."""
        X = _f32(X, N_FEATURES)
        t = _f32(t).ravel()
        g = np.zeros(num_params(), dtype=np.float32)
        loss = C.c_float()
        _lib.check(_lib.lib().aifmm_mlp_grad(self.h, X.ravel(), t, len(X), g, C.byref(loss)))
        return g, float(loss.value)

    def train(self, X, t, epochs: int = 2000, lr: float = 3e-3) -> tuple[float, float]:
        X = _f32(X, N_FEATURES)
        t = _f32(t).ravel()
        l0, l1 = C.c_float(), C.c_float()
        _lib.check(_lib.lib().aifmm_mlp_train(self.h, X.ravel(), t, len(X), int(epochs), float(lr), C.byref(l0),
                                              C.byref(l1)))
        return float(l0.value), float(l1.value)

    def fit(self, X, ranks, epochs: int = 3000, lr: float = 3e-3) -> tuple[float, float]:
        """Normalise the features by their mean and spread, then train on
        log2(1 + rank)."""
        X = _f32(X, N_FEATURES)
        mean = X.mean(axis=0)
        sd = X.std(axis=0)
        self.set_normalization(mean, np.where(sd > 1e-6, 1.0 / np.maximum(sd, 1e-6), 1.0))
        return self.train(X, np.log2(1.0 + np.asarray(ranks, dtype=np.float64)), epochs, lr)


def set_rank_model(ctx: Context, model: RankMLP | None, margin: float = 1.25) -> None:
    """Solvers created on ctx afterwards size their ACA workspaces from the
    model (None: the fixed bound)."""
    _lib.check(_lib.lib().aifmm_ctx_set_rank_model(ctx.h, model.h if model is not None else None, float(margin)))


def aca_log(solver) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(features n x 6, first rank bound, rank found) of every ACA problem of
    the solver's build."""
    n = C.c_int()
    _lib.check(_lib.lib().aifmm_solver_aca_log(solver.h, None, None, None, 0, C.byref(n)))
    X = np.zeros((n.value, N_FEATURES), dtype=np.float32)
    r0 = np.zeros(n.value, dtype=np.int32)
    r = np.zeros(n.value, dtype=np.int32)
    _lib.check(_lib.lib().aifmm_solver_aca_log(solver.h, X.ctypes.data, r0.ctypes.data, r.ctypes.data, n.value,
                                               C.byref(n)))
    return X, r0, r
