"""Height functions of device-resident tilings (include/rt_b200_height.h).

The device counterpart of DominoTiler::TilingToHeightfunc
(src/Domino/DominoTiler.cpp:423-461) and LozengeTiler::TilingToHeightfunc
(src/Lozenge/LozengeTiler.cpp:95-138): same normalisation (0 at the first
boundary vertex, INT_MAX outside the domain).  Device buffers are passed as
raw addresses (int), e.g. torch tensors' data_ptr().
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi


class HeightPlan:
    def __init__(self, model: int, domain, device: int = 0):
        self._lib = _capi.load()
        d = np.ascontiguousarray(domain, dtype=np.int32).reshape(-1)
        h = ctypes.c_void_p()
        st = self._lib.rt_hplan_create(int(model), d.ctypes.data, d.size, int(device), ctypes.byref(h))
        if st != _capi.RT_OK:
            raise _capi.RtError(st, self._lib.rt_hplan_last_error(None).decode())
        self._h = h
        n, v = ctypes.c_int32(), ctypes.c_int64()
        self._check(self._lib.rt_hplan_info(h, ctypes.byref(n), ctypes.byref(v)))
        self.n, self.vertices, self.model = n.value, v.value, int(model)

    def _check(self, st: int) -> None:
        if st != _capi.RT_OK:
            raise _capi.RtError(st, self._lib.rt_hplan_last_error(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.rt_hplan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def heights(self, d_tiling: int, d_heights: int, stream: int = 0) -> None:
        self._check(self._lib.rt_hplan_heights(self._h, d_tiling, d_heights, stream or None))

    def accumulate(self, d_tiling: int, d_sum: int, stream: int = 0) -> None:
        self._check(self._lib.rt_hplan_accumulate(self._h, d_tiling, d_sum, stream or None))

    def error(self, d_tiling: int, d_ref: int, stream: int = 0) -> float:
        out = ctypes.c_double()
        self._check(self._lib.rt_hplan_error(self._h, d_tiling, d_ref, ctypes.byref(out), stream or None))
        return out.value
