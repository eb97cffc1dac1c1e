"""rt_walk_device_noalloc: the walk for callers that cannot let the library
allocate GPU memory (programs that hand out all device memory from their own
pool).  The caller owns the device tiling; the library uses only its built-in
scratch array.  Its result must equal the ordinary rt_walk bit for bit, on two
calls in a row (the second call reuses the scratch array the first one left
behind).  Collected last so that a failure here cannot hide other tests.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _noalloc(lib, cfg, d_ptr: int, n: int, steps: int, seed: int) -> None:
    from randomtilings_b200._capi import RtError

    buf = ctypes.create_string_buffer(512)
    st = lib.rt_walk_device_noalloc(ctypes.byref(cfg), ctypes.c_void_p(d_ptr), n, steps, seed, buf, len(buf))
    if st != 0:
        raise RtError(st, buf.value.decode())


@pytest.mark.parametrize("model,kernel,key", [
    (0, 0, "domino/aztec13/min"),
    (1, 0, "lozenge/hex13_5/min"),
    (1, 2, "lozenge/hex20_0/min"),
    (2, 0, "recttri/min_hex9"),
])
def test_noalloc_walk_matches_rt_walk_twice(model, kernel, key):
    import torch

    import randomtilings_b200 as rt
    from randomtilings_b200 import _capi

    lib = _capi.load()
    cfg = _capi.RtConfig()
    lib.rt_config_default(ctypes.byref(cfg), model)
    cfg.kernel = kernel
    t0 = np.array(golden("builders")[key], dtype=np.int32)
    n = int(round(t0.size ** 0.5))
    cls = {0: rt.DominoTiler, 1: rt.LozengeTiler, 2: rt.RectTriangleTiler}[model]

    # Caller-owned device tiling (the test allocates it; the entry point does not).
    dev = torch.from_numpy(t0.copy()).cuda()
    expect = t0.copy()
    ref = cls(kernel=kernel)
    for steps, seed in ((700, 11), (500, -3)):
        _noalloc(lib, cfg, dev.data_ptr(), n, steps, seed)
        ref.Walk(expect, steps, seed)
        got = dev.cpu().numpy()
        assert np.array_equal(got, expect)
    ref.close()


@pytest.mark.parametrize("steps", [10_000_000, 1 << 62, (1 << 63) - 1])
def test_noalloc_rejects_walks_beyond_its_scratch(steps):
    """Step counts whose schedule cannot fit the built-in array, up to the
    largest int64, are refused before anything touches the tiling."""
    import torch

    from randomtilings_b200 import _capi

    lib = _capi.load()
    cfg = _capi.RtConfig()
    lib.rt_config_default(ctypes.byref(cfg), 1)
    t0 = np.array(golden("builders")["lozenge/hex13_5/min"], dtype=np.int32)
    n = int(round(t0.size ** 0.5))
    dev = torch.from_numpy(t0.copy()).cuda()
    buf = ctypes.create_string_buffer(512)
    st = lib.rt_walk_device_noalloc(ctypes.byref(cfg), ctypes.c_void_p(dev.data_ptr()), n, steps, 1, buf,
                                    len(buf))
    assert st == _capi.RT_E_INVAL
    assert b"scratch" in buf.value
    assert np.array_equal(dev.cpu().numpy(), t0)  # rejected before touching the tiling
