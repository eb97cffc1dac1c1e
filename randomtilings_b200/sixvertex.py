"""The six-vertex model (square ice) with domain-wall boundary conditions.

The reference names the model beside its tilings (README.md:3) but ships no
code for it; this class follows its Tiler pattern -- extremal states, Walk,
CFTP -- over the C ABI of include/rt_b200_sixv.h.  A state is the height
function on the (n+1) x (n+1) faces of the n x n grid (int32, row-major): the
corner sums of an alternating-sign matrix.  Vertex weights are given per type
in the order a1, a2, b1, b2, c1, c2 (see the header for the types).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi


def _heights(h) -> tuple[np.ndarray, int]:
    a = np.ascontiguousarray(h, dtype=np.int32).reshape(-1)
    n1 = int(round(a.size ** 0.5))
    if n1 * n1 != a.size or n1 < 2:
        raise ValueError(f"heights of {a.size} entries are not an (n+1) x (n+1) array")
    return a, n1 - 1


class SixVertexTiler:
    """Heat-bath Glauber dynamics of the six-vertex model on the GPU."""

    def __init__(self, device: int = 0, weights=None):
        self._lib = _capi.load()
        h = ctypes.c_void_p()
        st = self._lib.rt_sixv_create(device, ctypes.byref(h))
        if st != _capi.RT_OK:
            raise _capi.RtError(st, "rt_sixv_create failed")
        self._h = h
        if weights is not None:
            self.SetWeights(*weights)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.rt_sixv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != _capi.RT_OK:
            msg = self._lib.rt_sixv_last_error(self._h)
            raise _capi.RtError(st, msg.decode() if msg else "")

    def SetWeights(self, a1: float, a2: float, b1: float, b2: float, c1: float, c2: float) -> None:
        w = np.array([a1, a2, b1, b2, c1, c2], dtype=np.float64)
        self._check(self._lib.rt_sixv_set_weights(self._h, w.ctypes.data))

    def Thresholds(self) -> tuple[np.ndarray, bool]:
        thr = np.zeros(16, dtype=np.uint32)
        mono = ctypes.c_int32()
        self._check(self._lib.rt_sixv_thresholds(self._h, thr.ctypes.data, ctypes.byref(mono)))
        return thr, bool(mono.value)

    @staticmethod
    def MinHeights(n: int) -> np.ndarray:
        out = np.zeros((n + 1) ** 2, dtype=np.int32)
        _capi.check(_capi.load().rt_sixv_dwbc_heights(n, out.ctypes.data, None))
        return out

    @staticmethod
    def MaxHeights(n: int) -> np.ndarray:
        out = np.zeros((n + 1) ** 2, dtype=np.int32)
        _capi.check(_capi.load().rt_sixv_dwbc_heights(n, None, out.ctypes.data))
        return out

    @staticmethod
    def IsValid(h) -> bool:
        a, n = _heights(h)
        return _capi.load().rt_sixv_check(a.ctypes.data, n) == _capi.RT_OK

    @staticmethod
    def HeightsToASM(h) -> np.ndarray:
        a, n = _heights(h)
        out = np.zeros(n * n, dtype=np.int32)
        _capi.check(_capi.load().rt_sixv_to_asm(a.ctypes.data, n, out.ctypes.data))
        return out.reshape(n, n)

    @staticmethod
    def VertexTypes(h) -> np.ndarray:
        a, n = _heights(h)
        out = np.zeros(n * n, dtype=np.int32)
        _capi.check(_capi.load().rt_sixv_vertex_types(a.ctypes.data, n, out.ctypes.data))
        return out.reshape(n, n)

    def Walk(self, h, sweeps: int, seed: int, chain: int = 0) -> None:
        """`sweeps` sweeps (four colour steps each) on the heights h, in place."""
        a, n = _heights(h)
        self._check(self._lib.rt_sixv_walk(self._h, a.ctypes.data, n, int(sweeps), int(seed) & (2**64 - 1), chain))
        if isinstance(h, np.ndarray) and not np.shares_memory(h, a):
            h.reshape(-1)[:] = a

    def CFTP(self, n: int, first_sweeps: int = 16, master_seed: int = 0, max_trials: int = 30):
        """An exact sample by coupling from the past; returns (heights, stats)."""
        out = np.zeros((n + 1) ** 2, dtype=np.int32)
        st = _capi.RtCftpStats()
        self._check(self._lib.rt_sixv_cftp(self._h, n, int(first_sweeps), int(master_seed), int(max_trials),
                                           out.ctypes.data, ctypes.byref(st)))
        return out, {"colour_steps": st.total_steps, "sweeps": st.total_steps // 4, "trials": st.trials,
                     "coalesced": bool(st.coalesced), "device_ms": st.device_ms}
