"""Exact projection of a real height surface onto a tiling's height function
(include/rt_b200_project.h), and the warm-start tiling built from it.

No reference counterpart for the projection itself; its output goes through
the reference's HeightfuncToTiling (rt_*_height_to_tiling here).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from .tilers import DominoTiler, LozengeTiler

INF = np.iinfo(np.int32).max
_CLS = {_capi.RT_DOMINO: DominoTiler, _capi.RT_LOZENGE: LozengeTiler}


def extremal_heights(model: int, domain) -> tuple[np.ndarray, np.ndarray]:
    """Height functions (h_min, h_max) of the domain's two extremal tilings."""
    cls = _CLS[model]
    a = np.asarray(cls.TilingToHeightfunc(cls.MinTiling(domain), domain), dtype=np.int64)
    b = np.asarray(cls.TilingToHeightfunc(cls.MaxTiling(domain), domain), dtype=np.int64)
    return np.minimum(a, b).astype(np.int32), np.maximum(a, b).astype(np.int32)


def project_heights(model: int, domain, hmin, hmax, target, device: int = 0) -> tuple[np.ndarray, dict]:
    lib = _capi.load()
    d = np.ascontiguousarray(domain, dtype=np.int32).reshape(-1)
    lo = np.ascontiguousarray(hmin, dtype=np.int32).reshape(-1)
    hi = np.ascontiguousarray(hmax, dtype=np.int32).reshape(-1)
    t = np.ascontiguousarray(target, dtype=np.float32).reshape(-1)
    if not (lo.size == hi.size == t.size):
        raise ValueError("hmin, hmax and target differ in size")
    out = np.zeros(lo.size, dtype=np.int32)
    st = _capi.RtProjectStats()
    _capi.check(lib.rt_project_heights(model, d.ctypes.data, d.size, lo.ctypes.data, hi.ctypes.data, t.ctypes.data,
                                       out.ctypes.data, lo.size, device, ctypes.byref(st)))
    return out, {"passes": st.passes, "lowered": st.lowered, "raised": st.raised, "device_ms": st.device_ms}


def warm_tiling(model: int, domain, target, device: int = 0) -> np.ndarray:
    """Tiling whose height function is the projection of `target`."""
    hmin, hmax = extremal_heights(model, domain)
    h, _ = project_heights(model, domain, hmin, hmax, target, device)
    return np.asarray(_CLS[model].HeightfuncToTiling(h, domain), dtype=np.int32)
