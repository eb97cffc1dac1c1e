"""Domains, extremal tilings and height functions (host C++ in librt_b200.so).

Thin numpy wrappers over include/rt_b200_host.h; the Tiler classes expose them
under the reference's static-method names.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi


def _arr(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32).reshape(-1))


def call(name: str, *args) -> np.ndarray:
    """Calls a builder: array arguments become (pointer, length) pairs."""
    lib = _capi.load()
    fn = getattr(lib, name)
    cargs, keep = [], []
    for a in args:
        if isinstance(a, (np.ndarray, list, tuple)):
            arr = _arr(a)
            keep.append(arr)
            cargs += [arr.ctypes.data, arr.size]
        else:
            cargs.append(int(a))
    n = ctypes.c_int64()
    _capi.check(fn(*cargs, None, 0, ctypes.byref(n)))
    out = np.zeros(max(n.value, 1), dtype=np.int32)
    _capi.check(fn(*cargs, out.ctypes.data, out.size, ctypes.byref(n)))
    return out[: n.value]


def aztec_rectangle(order: int, remove) -> np.ndarray:
    lib = _capi.load()
    rem = _arr(remove)
    n = ctypes.c_int64()
    _capi.check(lib.rt_domino_aztec_rectangle(order, rem.ctypes.data, rem.size, None, 0, ctypes.byref(n)))
    out = np.zeros(n.value, dtype=np.int32)
    _capi.check(lib.rt_domino_aztec_rectangle(order, rem.ctypes.data, rem.size, out.ctypes.data, out.size,
                                              ctypes.byref(n)))
    return out


def vertex_side(model: int, dlen: int) -> int:
    """Vertex side n of a domino (M x M faces) or lozenge (M x 2M triangles) domain."""
    m = int(round((dlen if model == _capi.RT_DOMINO else dlen // 2) ** 0.5))
    return m + 1


def extremal_tilings(model: int, domain, device: int = 0) -> tuple[dict, dict]:
    """MinTiling, MaxTiling and their height functions, computed on the GPU
    (include/rt_b200_extremal.h).  Returns ({"tmin", "tmax", "hmin", "hmax"},
    stats); the arrays equal the host functions' results."""
    lib = _capi.load()
    d = _arr(domain)
    n = vertex_side(model, d.size)
    out = {k: np.zeros(n * n, dtype=np.int32) for k in ("tmin", "tmax", "hmin", "hmax")}
    st = _capi.RtExtremalStats()
    _capi.check(lib.rt_extremal_tilings(model, d.ctypes.data, d.size, device, out["tmin"].ctypes.data,
                                        out["tmax"].ctypes.data, out["hmin"].ctypes.data, out["hmax"].ctypes.data,
                                        n * n, ctypes.byref(st)))
    stats = {k: getattr(st, k) for k, _ in _capi.RtExtremalStats._fields_}
    return out, stats


def write(name: str, filename: str, *arrays) -> None:
    """Calls an SVG / text writer of include/rt_b200_svg.h; None arrays pass NULL."""
    lib = _capi.load()
    cargs, keep = [], []
    for a in arrays:
        if a is None:
            cargs += [None, 0]
        else:
            arr = _arr(a)
            keep.append(arr)
            cargs += [arr.ctypes.data, arr.size]
    _capi.check(getattr(lib, name)(*cargs, str(filename).encode()))


def save_matrix(a, filename: str) -> None:
    write("rt_save_matrix", filename, a)


def load_matrix(filename: str) -> np.ndarray:
    lib = _capi.load()
    n = ctypes.c_int64()
    _capi.check(lib.rt_load_matrix(str(filename).encode(), None, 0, ctypes.byref(n)))
    out = np.zeros(max(n.value, 1), dtype=np.int32)
    _capi.check(lib.rt_load_matrix(str(filename).encode(), out.ctypes.data, out.size, ctypes.byref(n)))
    return out[: n.value]


def save_matrix_binary(a, filename: str) -> None:
    """Any int32 array in the compact binary format (include/rt_b200_svg.h)."""
    arr = _arr(a)
    _capi.check(_capi.load().rt_save_matrix_binary(arr.ctypes.data, arr.size, str(filename).encode()))


def load_matrix_binary(filename: str) -> np.ndarray:
    lib = _capi.load()
    n = ctypes.c_int64()
    _capi.check(lib.rt_load_matrix_binary(str(filename).encode(), None, 0, ctypes.byref(n)))
    out = np.zeros(max(n.value, 1), dtype=np.int32)
    _capi.check(lib.rt_load_matrix_binary(str(filename).encode(), out.ctypes.data, out.size, ctypes.byref(n)))
    return out[: n.value]


def extremal_tilings_device(model: int, domain, tmin=0, tmax=0, hmin=0, hmax=0, device: int = 0) -> dict:
    """rt_extremal_tilings_device: the same arrays as extremal_tilings written
    into caller-owned device buffers (device pointers as ints, 0 = not wanted,
    each n*n int32 on `device`; e.g. torch tensors' data_ptr()).  Returns the stats."""
    lib = _capi.load()
    d = _arr(domain)
    n = vertex_side(model, d.size)
    st = _capi.RtExtremalStats()
    _capi.check(lib.rt_extremal_tilings_device(model, d.ctypes.data, d.size, device, tmin or None, tmax or None,
                                               hmin or None, hmax or None, n * n, ctypes.byref(st)))
    return {k: getattr(st, k) for k, _ in _capi.RtExtremalStats._fields_}
