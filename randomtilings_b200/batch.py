"""Many independent chains per launch (include/rt_b200_batch.h).

No reference counterpart: the reference runs one Tiler per lattice.  A Batch
holds chains of any of the four models and of uneven sizes; run(sweeps)
advances all of them in one CUDA graph (one persistent cluster launch per
kernel family).  Draws are the fast mode's, so chain c with key k equals a
fast-mode Tiler walk with chain=c and seed=k of sweeps x colours steps.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from .tilers import _as_tiling

# colour steps per sweep for each model
STEPS_PER_SWEEP = {_capi.RT_DOMINO: 2, _capi.RT_LOZENGE: 3, _capi.RT_RECTTRI: 3, _capi.RT_TRIDIMER: 30}
FAMILY_NAMES = ("domino", "domino_heat_bath", "lozenge", "", "rect_triangle", "triangle_dimer")


class BatchError(RuntimeError):
    pass


class Batch:
    def __init__(self, device: int = 0):
        self._lib = _capi.load()
        h = ctypes.c_void_p()
        self._check(self._lib.rt_batch_create(device, ctypes.byref(h)), None)
        self._h = h
        self._sizes: list[int] = []

    def _check(self, status: int, h="self") -> None:
        if status != _capi.RT_OK:
            handle = self._h if h == "self" else h
            msg = self._lib.rt_batch_last_error(handle)
            raise _capi.RtError(status, msg.decode() if msg else "")

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.rt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, model: int, tiling, key: int, chain: int | None = None, kernel: int = _capi.RT_KERNEL_DEFAULT,
            q: float = 0.0) -> int:
        """q: lozenge volume weight in (0, 1] (0 = uniform), see rt_chain.q."""
        arr, n = _as_tiling(tiling)
        c = _capi.RtChain()
        c.model, c.kernel, c.key = model, kernel, int(np.int64(np.uint64(key & (2**64 - 1))))
        c.q = float(q)
        c.chain = len(self._sizes) if chain is None else chain
        idx = ctypes.c_int64()
        self._check(self._lib.rt_batch_add(self._h, ctypes.byref(c), arr.ctypes.data, n, ctypes.byref(idx)))
        self._sizes.append(n)
        return idx.value

    def set_tuning(self, autotune: bool = True, cluster: int = 0, block: int = 0) -> None:
        self._check(self._lib.rt_batch_set_tuning(self._h, int(autotune), cluster, block))

    def set_sweeps_per_launch(self, sweeps: int) -> None:
        """> 0: launches of that many sweeps; 0: one launch per run; -1: the autotuner chooses."""
        self._check(self._lib.rt_batch_set_sweeps_per_launch(self._h, int(sweeps)))

    def run(self, sweeps: int) -> None:
        self._check(self._lib.rt_batch_run(self._h, int(sweeps)))

    def download(self, index: int) -> np.ndarray:
        n = self._sizes[index]
        out = np.zeros(n * n, dtype=np.int32)
        self._check(self._lib.rt_batch_download(self._h, int(index), out.ctypes.data))
        return out

    def device_tiling(self, index: int, d_tiling: int, stream: int = 0) -> None:
        """Chain `index`'s tiling into the device buffer at d_tiling (N*N int32)."""
        self._check(self._lib.rt_batch_device_tiling(self._h, int(index), d_tiling, stream or None))

    def info(self) -> dict:
        i = _capi.RtBatchInfo()
        self._check(self._lib.rt_batch_get_info(self._h, ctypes.byref(i)))
        plans = {FAMILY_NAMES[f]: {"cluster": i.cluster[f], "block": i.block[f], "clusters": i.clusters[f],
                                   "sweeps_per_launch": i.sweeps_per_launch[f]}
                 for f in range(6) if i.cluster[f]}
        return {"chains": i.chains, "plans": plans, "tune_ms": i.tune_ms, "run_ms": i.run_ms,
                "attempts": i.attempts, "algorithmic_bytes": i.algorithmic_bytes}

    def __len__(self) -> int:
        return len(self._sizes)
