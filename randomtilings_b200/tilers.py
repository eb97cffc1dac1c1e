"""Python mirror of the reference's per-model Tiler classes over the C ABI.

Method names and argument meanings follow the reference
(src/Domino/DominoTiler.h, src/Lozenge/LozengeTiler.h,
src/RectTriangle/RectTriangleTiler.h, src/TriangleDimer/TriangleDimerTiler.h):
``LoadTinyMT(path, size)`` and ``Walk(tiling, steps, seed)`` mutate the
caller's tiling in place.  The OpenCL (context, queue, devices, source)
constructor arguments become a device ordinal plus kernel options.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi, builders
from ._capi import check


def _as_tiling(t) -> tuple[np.ndarray, int]:
    arr = np.ascontiguousarray(t, dtype=np.int32).reshape(-1)
    n = int(round(arr.size ** 0.5))
    if n * n != arr.size:
        raise ValueError(f"tiling of {arr.size} entries is not square")
    return arr, n


def _writeback(dst, src: np.ndarray) -> None:
    if isinstance(dst, np.ndarray):
        if dst.dtype == np.int32 and dst.flags.c_contiguous:
            if not np.shares_memory(dst, src):
                dst.reshape(-1)[:] = src
        else:
            dst.reshape(-1)[:] = src
    elif isinstance(dst, list):
        dst[:] = src.tolist()
    else:
        raise TypeError("tiling must be a numpy array or a list")


class _Tiler:
    MODEL = -1
    # common helpers (src/common/common.h:50-69)
    SaveMatrix = staticmethod(lambda a, f: builders.save_matrix(a, f))
    LoadMatrix = staticmethod(lambda f: builders.load_matrix(f))
    SaveMatrixBinary = staticmethod(lambda a, f: builders.save_matrix_binary(a, f))
    LoadMatrixBinary = staticmethod(lambda f: builders.load_matrix_binary(f))

    def __init__(self, device: int = 0, kernel: int = _capi.RT_KERNEL_DEFAULT, rng: int = _capi.RT_RNG_TINYMT,
                 q: float = 0.99, qcmp: int = _capi.RT_QCMP_FLOAT32, weights=None, stream=None, chain: int = 0):
        self._lib = _capi.load()
        cfg = _capi.RtConfig()
        self._lib.rt_config_default(ctypes.byref(cfg), self.MODEL)
        cfg.kernel = kernel
        cfg.rng = rng
        cfg.q = q
        cfg.qcmp = qcmp
        cfg.device = device
        cfg.chain = chain
        if weights is not None:
            for i, w in enumerate(weights):
                cfg.weights[i] = float(w)
        cfg.stream = stream
        h = ctypes.c_void_p()
        check(self._lib.rt_create(ctypes.byref(cfg), ctypes.byref(h)), None)
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.rt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status: int) -> None:
        check(status, self._h)

    # -- reference methods -------------------------------------------------
    def LoadTinyMT(self, params: str, size: int) -> None:
        self._check(self._lib.rt_load_rng_params(self._h, params.encode(), int(size)))

    def SetTinyMTTable(self, table) -> None:
        tab = np.ascontiguousarray(table, dtype=np.uint32).reshape(-1)
        self._check(self._lib.rt_set_rng_params(self._h, tab.ctypes.data, tab.size // 3))

    def Walk(self, t, steps: int, seed: int) -> None:
        arr, n = _as_tiling(t)
        self._check(self._lib.rt_walk(self._h, arr.ctypes.data, n, int(steps), int(seed)))
        _writeback(t, arr)

    def CFTP(self, tmax, tmin, first_steps: int = 1024, schedule: int = _capi.RT_CFTP_DOUBLING,
             master_seed: int = 345903, max_trials: int = 30):
        """Coupling from the past (Examples/AztecDiamondCftpEx.cpp:42-68) for a
        monotone kernel: dominoes with kernel=RT_KERNEL_CFTP, or either lozenge
        kernel.  Returns (tiling, stats dict)."""
        a, n = _as_tiling(tmax)
        b, n2 = _as_tiling(tmin)
        if n != n2:
            raise ValueError("tmax and tmin differ in size")
        out = np.zeros_like(a)
        st = _capi.RtCftpStats()
        self._check(self._lib.rt_cftp(self._h, a.ctypes.data, b.ctypes.data, n, int(first_steps), int(schedule),
                                      int(master_seed), int(max_trials), out.ctypes.data, ctypes.byref(st)))
        return out, {"total_steps": st.total_steps, "trials": st.trials, "coalesced": bool(st.coalesced),
                     "device_ms": st.device_ms}

    # -- device-resident form ---------------------------------------------
    def upload(self, t) -> None:
        arr, n = _as_tiling(t)
        self._check(self._lib.rt_upload(self._h, arr.ctypes.data, n))
        self._check(self._lib.rt_synchronize(self._h))

    def run(self, steps: int, seed: int) -> None:
        self._check(self._lib.rt_run(self._h, int(steps), int(seed)))

    def download(self, out: np.ndarray) -> None:
        self._check(self._lib.rt_download(self._h, out.ctypes.data))

    def synchronize(self) -> None:
        self._check(self._lib.rt_synchronize(self._h))

    def device_tiling(self) -> int:
        """Device address of the current tiling (N x N int32), merged on the
        handle's stream (rt_device_tiling)."""
        ptr = ctypes.c_void_p()
        self._check(self._lib.rt_device_tiling(self._h, ctypes.byref(ptr)))
        return ptr.value

    @property
    def stream(self) -> int:
        return self._lib.rt_stream(self._h) or 0

    def last_run_info(self) -> tuple[int, int]:
        ph, la = ctypes.c_int64(), ctypes.c_int64()
        self._check(self._lib.rt_last_run_info(self._h, ctypes.byref(ph), ctypes.byref(la)))
        return ph.value, la.value


class DominoTiler(_Tiler):
    MODEL = _capi.RT_DOMINO

    # static helpers (src/Domino/DominoTiler.h:83-107)
    Rectangle = staticmethod(lambda m, n: builders.call("rt_domino_rectangle", m, n))
    AztecRectangle = staticmethod(lambda n, remove: builders.aztec_rectangle(n, remove))
    AztecDiamond = staticmethod(lambda n: builders.call("rt_domino_aztec", n))
    MaxTiling = staticmethod(lambda d: builders.call("rt_domino_max_tiling", d))
    MinTiling = staticmethod(lambda d: builders.call("rt_domino_min_tiling", d))
    DomainToVertices = staticmethod(lambda d: builders.call("rt_domino_domain_to_vertices", d))
    TilingToDomain = staticmethod(lambda t: builders.call("rt_domino_tiling_to_domain", t))
    HeightfuncToTiling = staticmethod(lambda h, d: builders.call("rt_domino_height_to_tiling", h, d))
    TilingToHeightfunc = staticmethod(lambda t, d: builders.call("rt_domino_tiling_to_height", t, d))
    DomainToSVG = staticmethod(lambda d, f: builders.write("rt_domino_domain_svg", f, d))
    TilingToSVG = staticmethod(lambda t, f: builders.write("rt_domino_tiling_svg", f, t))
    MayaToSVG = staticmethod(lambda t, f: builders.write("rt_domino_maya_svg", f, t))

    @staticmethod
    def DimerToSVG(t, *args):  # DimerToSVG(t, filename) or DimerToSVG(t, d, filename)
        d, f = (None, args[0]) if len(args) == 1 else args
        builders.write("rt_domino_dimer_svg", f, t, d)

    @staticmethod
    def TwoPeriodicWeights(a: float, b: float):
        """(wh, wv) of the two-periodic weighting: every domino borders exactly
        one even lattice vertex (i + j even, a face of the dual graph) and takes
        its weight, a when that vertex's row is even, b when it is odd.  Flips
        at even vertices are then fair; at odd ones the vertical pair wins with
        probability a^2 / (a^2 + b^2) or b^2 / (a^2 + b^2), rows alternating."""
        wh, wv = np.zeros((2, 2)), np.zeros((2, 2))
        for r in range(2):
            for c in range(2):
                # horizontal domino on squares (r, c), (r, c+1): vertices (r, c+1), (r+1, c+1)
                row = r if (r + c + 1) % 2 == 0 else r + 1
                wh[r, c] = a if row % 2 == 0 else b
                # vertical domino on squares (r, c), (r+1, c): vertices (r+1, c), (r+1, c+1)
                wv[r, c] = a if (r + 1) % 2 == 0 else b
        return wh, wv

    def SetWeights(self, wh=None, wv=None) -> None:
        """Periodic domino weights for the heat-bath kernel (rt_set_domino_weights):
        wh / wv are P x P tables (P = 1, 2 or 4) of horizontal / vertical domino
        weights by the domino's top-left square (row mod P, column mod P);
        None returns to uniform weights."""
        if wh is None:
            self._check(_capi.load().rt_set_domino_weights(self._h, 0, None, None))
            return
        a = np.ascontiguousarray(wh, dtype=np.float64)
        b = np.ascontiguousarray(wv, dtype=np.float64)
        if a.ndim != 2 or a.shape[0] != a.shape[1] or b.shape != a.shape:
            raise ValueError("wh and wv must be P x P tables of the same shape")
        self._check(_capi.load().rt_set_domino_weights(self._h, a.shape[0], a.ctypes.data, b.ctypes.data))

    def Walk(self, t, steps, seed=None) -> None:  # noqa: N802 -- reference name
        """Walk(t, steps, seed) or Walk(t, [steps...], [seeds...]) (DominoTiler.h:73,76)."""
        if isinstance(steps, (list, tuple, np.ndarray)):
            st = np.ascontiguousarray(steps, dtype=np.int64)
            se = np.ascontiguousarray(seed, dtype=np.int64)
            if st.size != se.size:
                raise ValueError("steps and seeds must have the same length")
            arr, n = _as_tiling(t)
            self._check(self._lib.rt_walk_epochs(self._h, arr.ctypes.data, n, st.ctypes.data, se.ctypes.data,
                                                 int(st.size)))
            _writeback(t, arr)
        else:
            super().Walk(t, steps, seed)

class LozengeTiler(_Tiler):
    MODEL = _capi.RT_LOZENGE

    # static helpers (src/Lozenge/LozengeTiler.h:61-78)
    AlmostHexDomain = staticmethod(lambda n, m: builders.call("rt_lozenge_almost_hex", n, m))
    Hexagon = staticmethod(lambda a, b, c: builders.call("rt_lozenge_hexagon", a, b, c))  # no reference counterpart
    MaxTiling = staticmethod(lambda d: builders.call("rt_lozenge_max_tiling", d))
    MinTiling = staticmethod(lambda d: builders.call("rt_lozenge_min_tiling", d))
    DomainToVertices = staticmethod(lambda d: builders.call("rt_lozenge_domain_to_vertices", d))
    TilingToDomain = staticmethod(lambda t: builders.call("rt_lozenge_tiling_to_domain", t))
    HeightfuncToTiling = staticmethod(lambda h, d: builders.call("rt_lozenge_height_to_tiling", h, d))
    TilingToHeightfunc = staticmethod(lambda t, d: builders.call("rt_lozenge_tiling_to_height", t, d))
    DomainToSVG = staticmethod(lambda d, f: builders.write("rt_lozenge_domain_svg", f, d))
    TilingToSVG = staticmethod(lambda t, f: builders.write("rt_lozenge_tiling_svg", f, t))
    PrintDomain = staticmethod(lambda d, f: builders.write("rt_lozenge_print_domain", f, d))

    def SetWeights(self, w0=None, w1=None, w2=None) -> None:
        """Periodic lozenge weights for the uniform kernel (rt_set_lozenge_weights):
        P x P tables (P = 1, 2 or 4) for the lozenges covering the edge from
        (i, j) to (i, j+1), (i-1, j+1) and (i-1, j), indexed by (i mod P, j mod P);
        None returns to uniform weights."""
        if w0 is None:
            self._check(_capi.load().rt_set_lozenge_weights(self._h, 0, None, None, None))
            return
        t = [np.ascontiguousarray(w, dtype=np.float64) for w in (w0, w1, w2)]
        if t[0].ndim != 2 or t[0].shape[0] != t[0].shape[1] or any(w.shape != t[0].shape for w in t):
            raise ValueError("w0, w1 and w2 must be P x P tables of the same shape")
        self._check(_capi.load().rt_set_lozenge_weights(self._h, t[0].shape[0], *(w.ctypes.data for w in t)))

    @staticmethod
    def DimerToSVG(t, *args):
        d, f = (None, args[0]) if len(args) == 1 else args
        builders.write("rt_lozenge_dimer_svg", f, t, d)


class RectTriangleTiler(_Tiler):
    MODEL = _capi.RT_RECTTRI

    # static helpers (src/RectTriangle/RectTriangleTiler.h:60-66)
    maxHex = staticmethod(lambda n: builders.call("rt_recttri_max_hex", n))
    minHex = staticmethod(lambda n: builders.call("rt_recttri_min_hex", n))
    LozengeToRectTriangle = staticmethod(lambda tl, dl: builders.call("rt_recttri_from_lozenge", tl, dl))
    TilingToSVG = staticmethod(lambda t, f: builders.write("rt_recttri_tiling_svg", f, t))


class TriangleDimerTiler(_Tiler):
    MODEL = _capi.RT_TRIDIMER

    # static helpers (src/TriangleDimer/TriangleDimerTiler.h:182-195)
    IceCreamCone = staticmethod(lambda n, m: builders.call("rt_tridimer_ice_cream_cone", n, m))
    TestButterfly = staticmethod(lambda k: builders.call("rt_tridimer_test_butterfly", k))
    # no reference counterpart: a hexagon of side s edges less one corner, canonical start (rt_b200_host.h)
    BiboneHexagon = staticmethod(lambda s: builders.call("rt_tridimer_hexagon", s))
    TilingToTriangleFlips = staticmethod(lambda t: builders.call("rt_tridimer_triangle_flips", t))
    TilingToButterflyFlips = staticmethod(lambda t: builders.call("rt_tridimer_butterfly_flips", t))
    TilingToVertices = staticmethod(lambda t: builders.call("rt_tridimer_vertices", t))
    TilingToDomain = staticmethod(lambda t: builders.call("rt_tridimer_tiling_to_domain", t))
    DimerIndicator = staticmethod(lambda t, c: builders.call("rt_tridimer_dimer_indicator", t, c))
    DomainToSVG = staticmethod(lambda d, f: builders.write("rt_tridimer_domain_svg", f, d))
    TilingToSVG = staticmethod(lambda t, f: builders.write("rt_tridimer_tiling_svg", f, t))

    @staticmethod
    def DimerToSVG(t, *args):
        d, f = (None, args[0]) if len(args) == 1 else args
        builders.write("rt_tridimer_dimer_svg", f, t, d)
