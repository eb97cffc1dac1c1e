"""Synthetic inputs of the benchmarks: the domains and start tilings are
built by the library's own builders (no dataset is involved)."""
from __future__ import annotations

import ctypes

from . import _capi
from .tilers import DominoTiler, LozengeTiler, RectTriangleTiler, TriangleDimerTiler


def mixed_chain_spec(seed: int) -> tuple[int, list[int]]:
    """(model, size parameters) of chain `seed` of the mixed batch workload
    (rt_mixed_chain_spec: type = seed mod 4, sizes from std::mt19937(seed))."""
    lib = _capi.load()
    model = ctypes.c_int32()
    p = (ctypes.c_int32 * 3)()
    _capi.check(lib.rt_mixed_chain_spec(int(seed), ctypes.byref(model), p))
    return model.value, list(p)


def start_tiling(model: int, p: list[int]):
    """Minimal tiling of the domain (p as mixed_chain_spec returns it); for the
    triangle dimers, which have no height function, the bibone hexagon's
    canonical start."""
    if model == _capi.RT_DOMINO:
        return DominoTiler.MinTiling(DominoTiler.AztecDiamond(p[0]))
    if model == _capi.RT_LOZENGE:
        return LozengeTiler.MinTiling(LozengeTiler.Hexagon(p[0], p[1], p[2]))
    if model == _capi.RT_TRIDIMER:
        return TriangleDimerTiler.BiboneHexagon(p[0])
    return RectTriangleTiler.minHex(p[0])


def mixed_chain(seed: int):
    """(model, start tiling) of chain `seed` of the mixed batch workload."""
    model, p = mixed_chain_spec(seed)
    return model, start_tiling(model, p)
