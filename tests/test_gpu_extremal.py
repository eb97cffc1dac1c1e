"""Device extremal tilings (include/rt_b200_extremal.h) against the host
builders, which are byte-equal to the reference's MaxTiling / MinTiling /
TilingToHeightfunc (DominoTiler.cpp:214-461, LozengeTiler.cpp:95-318):
every output array equal, the same refusals for domains that cannot be
tiled."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host(model, d):
    import randomtilings_b200 as rt

    cls = rt.DominoTiler if model == 0 else rt.LozengeTiler
    tmin, tmax = np.asarray(cls.MinTiling(d)), np.asarray(cls.MaxTiling(d))
    return {"tmin": tmin, "tmax": tmax, "hmin": np.asarray(cls.TilingToHeightfunc(tmin, d)),
            "hmax": np.asarray(cls.TilingToHeightfunc(tmax, d))}


def _check(model, d):
    from randomtilings_b200 import builders

    dev, st = builders.extremal_tilings(model, d)
    ref = _host(model, d)
    for k in ("tmin", "tmax", "hmin", "hmax"):
        assert np.array_equal(dev[k], ref[k]), k
    assert st["passes"] >= 8 and st["boundary"] > 0
    return st


def _young(rows, pad=1):
    m = max(len(rows), max(rows)) + 2 * pad
    d = np.zeros((m, m), np.int32)
    for r, length in enumerate(rows):
        d[r + pad, pad:pad + length] = 1
    return d.reshape(-1)


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5, 7, 16, 31, 32, 33, 64, 100, 300])
def test_aztec_diamonds(order):
    import randomtilings_b200 as rt

    _check(0, rt.DominoTiler.AztecDiamond(order))


@pytest.mark.parametrize("abc", [(1, 1, 1), (1, 2, 3), (5, 5, 5), (7, 3, 9), (30, 31, 33), (64, 1, 64), (200, 150, 100)])
def test_hexagons(abc):
    import randomtilings_b200 as rt

    _check(1, rt.LozengeTiler.Hexagon(*abc))


@pytest.mark.parametrize("k,cut", [(10, 2), (6, 0), (9, 1), (40, 5), (120, 0)])
def test_almost_hex(k, cut):
    import randomtilings_b200 as rt

    _check(1, rt.LozengeTiler.AlmostHexDomain(k, cut))


@pytest.mark.parametrize("rc", [(2, 2), (1, 2), (2, 9 * 2), (4, 6), (7, 8), (64, 130), (97, 34)])
def test_rectangles(rc):
    from randomtilings_b200 import builders

    _check(0, builders.call("rt_domino_rectangle", *rc))


@pytest.mark.parametrize("order,removed", [(6, [1, 3]), (10, [0, 5]), (40, [3, 17, 30]), (64, [0, 63])])
def test_aztec_rectangles(order, removed):
    from randomtilings_b200 import builders

    _check(0, builders.aztec_rectangle(order, removed))


def test_young_diagrams_against_the_host_including_refusals():
    """Random Young-diagram domains, tileable or not: the device agrees with
    the host on every array or on the refusal."""
    from randomtilings_b200 import _capi, builders

    rng = np.random.default_rng(11)
    ok = refused = 0
    for _ in range(60):
        rows = sorted(rng.integers(1, 40, size=int(rng.integers(1, 40))).tolist(), reverse=True)
        if rng.random() < 0.5:
            rows = [r + (r & 1) for r in rows]  # even rows: tileable
        d = _young(rows)
        try:
            ref = _host(0, d)
        except _capi.RtError:
            with pytest.raises(_capi.RtError):
                builders.extremal_tilings(0, d)
            refused += 1
            continue
        dev, _ = builders.extremal_tilings(0, d)
        for k in ref:
            assert np.array_equal(dev[k], ref[k]), (rows, k)
        ok += 1
    assert ok > 20 and refused > 5, (ok, refused)


def test_large_aztec_and_hexagon_timing_is_reported():
    import randomtilings_b200 as rt

    st = _check(0, rt.DominoTiler.AztecDiamond(1000))
    assert st["n"] == 2006 and st["device_ms"] > 0
    st = _check(1, rt.LozengeTiler.Hexagon(500, 500, 500))
    assert st["n"] == 1008


@pytest.mark.parametrize("kind,size", [("aztec", (50,)), ("hexagon", (20, 30, 25))])
def test_warm_start_preparation_on_the_device(kind, size):
    from randomtilings_b200 import warmstart as ws

    spec = ws.DomainSpec(kind, size)
    a, b = ws.prepare(spec), ws.prepare(spec, 0)
    for f in ("tmin", "tmax", "hmin", "hmax", "idx"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert a.n == b.n


@pytest.mark.parametrize("model,make", [(0, lambda rt: rt.DominoTiler.AztecDiamond(60)),
                                        (1, lambda rt: rt.LozengeTiler.Hexagon(40, 30, 50))])
def test_device_outputs_equal_host_outputs(model, make):
    """rt_extremal_tilings_device writes the same arrays into device buffers,
    for every output or any subset of them."""
    import torch

    import randomtilings_b200 as rt
    from randomtilings_b200 import builders

    d = make(rt)
    ref, _ = builders.extremal_tilings(model, d)
    n2 = ref["tmin"].size
    names = ("tmin", "tmax", "hmin", "hmax")
    for subset in (names, ("tmin",), ("hmax", "tmax"), ("hmin",)):
        out = {k: torch.full((n2,), -7, dtype=torch.int32, device="cuda:0") for k in subset}
        st = builders.extremal_tilings_device(model, d, **{k: v.data_ptr() for k, v in out.items()})
        torch.cuda.synchronize()
        for k, v in out.items():
            assert np.array_equal(v.cpu().numpy(), ref[k]), (subset, k)
        assert st["passes"] >= 8


def test_device_outputs_must_be_device_memory():
    import randomtilings_b200 as rt
    from randomtilings_b200 import _capi, builders

    d = rt.DominoTiler.AztecDiamond(10)
    host = np.zeros(builders.vertex_side(0, len(d)) ** 2, dtype=np.int32)
    with pytest.raises(_capi.RtError):
        builders.extremal_tilings_device(0, d, tmin=host.ctypes.data)
