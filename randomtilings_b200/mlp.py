"""The coordinate MLP of the learned warm start (include/rt_b200_mlp.h):
training and inference on the GPU through the library's own kernels."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi

IN, WIDTH, NPARAM = _capi.RT_MLP_IN, _capi.RT_MLP_WIDTH, _capi.RT_MLP_PARAMS


class CoordinateMLP:
    def __init__(self, device: int = 0, seed: int = 0):
        self._lib = _capi.load()
        h = ctypes.c_void_p()
        _capi.check(self._lib.rt_mlp_create(device, seed, ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.rt_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(NPARAM, dtype=np.float32)
        _capi.check(self._lib.rt_mlp_get_params(self._h, p.ctypes.data))
        return p

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == NPARAM
        _capi.check(self._lib.rt_mlp_set_params(self._h, p.ctypes.data))

    def predict(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, IN)
        y = np.zeros(x.shape[0], dtype=np.float32)
        _capi.check(self._lib.rt_mlp_predict(self._h, x.ctypes.data, x.shape[0], y.ctypes.data))
        return y

    def loss_grad(self, x, target) -> tuple[float, np.ndarray]:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, IN)
        t = np.ascontiguousarray(target, dtype=np.float32).reshape(-1)
        loss = ctypes.c_float()
        g = np.zeros(NPARAM, dtype=np.float32)
        _capi.check(self._lib.rt_mlp_loss_grad(self._h, x.ctypes.data, t.ctypes.data, x.shape[0], ctypes.byref(loss),
                                               g.ctypes.data))
        return loss.value, g

    def set_data(self, x, target) -> None:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, IN)
        t = np.ascontiguousarray(target, dtype=np.float32).reshape(-1)
        _capi.check(self._lib.rt_mlp_set_data(self._h, x.ctypes.data, t.ctypes.data, x.shape[0]))

    def train(self, steps: int, batch: int = 16384, lr: float = 1e-3, seed: int = 0) -> float:
        loss = ctypes.c_float()
        _capi.check(self._lib.rt_mlp_train(self._h, steps, batch, lr, seed, ctypes.byref(loss)))
        return loss.value
