"""Weighted dominoes and lozenges on the GPU (rt_set_domino_weights,
rt_set_lozenge_weights): the walks with periodic weights are bit-equal to
the oracle's restatements (orc_domino_walk_weighted,
orc_lozenge_walk_weighted) in the TinyMT and Philox modes, on both walk
kernels, for single walks, epoch walks and CFTP; their samples follow the
weighted law (probability proportional to the product of the tile weights,
by exact enumeration on the Aztec diamond of order 3 and the 2 x 2 x 2
hexagon); and the handles refuse weights where they do not apply."""
from __future__ import annotations

from collections import Counter

import numpy as np
import pytest
from scipy import stats

from conftest import golden
from oracle import pyoracle as po
from test_weighted_oracle import LW, lozenge_tiling_weight, tiling_weight

pytestmark = pytest.mark.gpu

_rng = np.random.default_rng(31)
WEIGHTS = {
    1: (np.array([[1.0]]), np.array([[2.5]])),
    2: (np.array([[1.0, 0.3], [0.5, 2.0]]), np.array([[0.7, 1.5], [1.0, 0.2]])),
    4: (_rng.uniform(0.5, 2.0, (4, 4)), _rng.uniform(0.5, 2.0, (4, 4))),
}


@pytest.fixture(scope="module")
def rt():
    import randomtilings_b200 as rt

    rt.load()
    return rt


@pytest.fixture(params=["word", "generic"])
def kernel(request, monkeypatch):
    monkeypatch.setenv("RT_WALK_KERNEL", request.param)
    return request.param


def _tiler(rt, period, rng=None):
    from randomtilings_b200 import _capi

    tl = rt.DominoTiler(kernel=_capi.RT_KERNEL_CFTP, rng=_capi.RT_RNG_TINYMT if rng is None else rng)
    tl.SetWeights(*WEIGHTS[period])
    return tl


@pytest.mark.parametrize("period", [1, 2, 4])
@pytest.mark.parametrize("order", [5, 13, 40])
def test_bit_exact_walk_matches_oracle(rt, kernel, period, order):
    t = (golden("builders")[f"domino/aztec{order}/min"] if order != 40
         else rt.DominoTiler.MinTiling(rt.DominoTiler.AztecDiamond(40)))
    a = np.array(t, dtype=np.int32)
    _tiler(rt, period).Walk(a, 901, 77)
    wh, wv = WEIGHTS[period]
    assert np.array_equal(a, po.domino_walk_weighted(t, [901], [77], wh, wv, single_walk=True))


@pytest.mark.parametrize("period", [1, 2, 4])
def test_fast_epoch_walk_matches_oracle(rt, kernel, period):
    from randomtilings_b200 import _capi

    t = golden("builders")["domino/aztec13/max"]
    a = np.array(t, dtype=np.int32)
    _tiler(rt, period, _capi.RT_RNG_PHILOX).Walk(a, [300, 200, 57], [11, 2**40 + 3, 5])
    wh, wv = WEIGHTS[period]
    assert np.array_equal(a, po.domino_walk_weighted(t, [300, 200, 57], [11, 2**40 + 3, 5], wh, wv, fast=True))


@pytest.mark.parametrize("fast", [False, True])
def test_weighted_cftp_matches_oracle(rt, fast):
    from randomtilings_b200 import _capi

    b = golden("builders")
    tmax, tmin = b["domino/aztec13/max"], b["domino/aztec13/min"]
    tl = _tiler(rt, 2, _capi.RT_RNG_PHILOX if fast else None)
    got, st = tl.CFTP(tmax, tmin, first_steps=64, master_seed=123, max_trials=20)
    want, trials, total, ok = po.cftp(tmax, tmin, 64, 123, max_trials=20, fast=fast, weights=WEIGHTS[2])
    assert st["coalesced"] and ok and st["trials"] == trials and st["total_steps"] == total
    assert np.array_equal(got, want)


def test_equal_weights_and_reset_give_the_unweighted_walk(rt):
    from randomtilings_b200 import _capi

    t = golden("builders")["domino/aztec13/min"]
    plain = np.array(t, dtype=np.int32)
    rt.DominoTiler(kernel=_capi.RT_KERNEL_CFTP).Walk(plain, 500, 9)
    tl = rt.DominoTiler(kernel=_capi.RT_KERNEL_CFTP)
    tl.SetWeights(np.full((2, 2), 1.7), np.full((2, 2), 1.7))
    a = np.array(t, dtype=np.int32)
    tl.Walk(a, 500, 9)
    assert np.array_equal(a, plain)
    tl.SetWeights(*WEIGHTS[2])
    tl.SetWeights(None)
    a = np.array(t, dtype=np.int32)
    tl.Walk(a, 500, 9)
    assert np.array_equal(a, plain)


def test_weights_are_refused_where_they_do_not_apply(rt):
    from randomtilings_b200 import _capi

    one = np.ones((2, 2))
    with pytest.raises(_capi.RtError):
        rt.DominoTiler(kernel=_capi.RT_KERNEL_DEFAULT).SetWeights(one, one)  # not the heat bath
    with pytest.raises(_capi.RtError):
        rt.DominoTiler(kernel=_capi.RT_KERNEL_CFTP, rng=_capi.RT_RNG_PLANES).SetWeights(one, one)
    tl = rt.DominoTiler(kernel=_capi.RT_KERNEL_CFTP)
    for wh, wv in ((np.ones((3, 3)), np.ones((3, 3))), (one, -one), (one, np.full((2, 2), np.inf))):
        with pytest.raises(_capi.RtError):
            tl.SetWeights(wh, wv)


P_MIN = 1e-4  # deterministic keys and seeds; a right law fails with probability 1e-4


@pytest.mark.parametrize("period", [2, 4])
def test_samples_follow_the_weighted_law(rt, period):
    """Aztec diamond of order 3 (64 tilings): chain ends from independent
    Philox keys and CFTP samples follow P(T) ~ product of its domino weights."""
    from randomtilings_b200 import _capi

    b = golden("builders")
    tmax, tmin = b["domino/aztec3/max"], b["domino/aztec3/min"]
    wh, wv = WEIGHTS[period]
    tl = _tiler(rt, period, _capi.RT_RNG_PHILOX)
    ends = []
    for key in range(6400):
        a = np.array(tmin, dtype=np.int32)
        tl.Walk(a, 1000, key)
        ends.append(a)
    samples = [tl.CFTP(tmax, tmin, first_steps=16, master_seed=s)[0] for s in range(6400)]
    for got in (ends, samples):
        c = Counter(s.tobytes() for s in got)
        assert len(c) == 64
        keys = sorted(c)
        w = np.array([tiling_weight(np.frombuffer(k, dtype=np.int32), wh, wv) for k in keys])
        obs = np.array([c[k] for k in keys], dtype=float)
        assert stats.chisquare(obs, obs.sum() * w / w.sum()).pvalue > P_MIN
        assert stats.chisquare(obs).pvalue < 1e-6  # not the uniform law


# ---- lozenges ----
LWEIGHTS = {1: tuple(np.array([[w]]) for w in (1.0, 0.5, 1.8)), 2: LW,
            4: tuple(_rng.uniform(0.5, 2.0, (4, 4)) for _ in range(3))}


def _ltiler(rt, period, rng=None):
    from randomtilings_b200 import _capi

    tl = rt.LozengeTiler(rng=_capi.RT_RNG_TINYMT if rng is None else rng)
    tl.SetWeights(*LWEIGHTS[period])
    return tl


@pytest.mark.parametrize("period", [1, 2, 4])
@pytest.mark.parametrize("key", ["hex10_2", "hex20_0"])
def test_lozenge_walk_matches_oracle(rt, kernel, period, key):
    from randomtilings_b200 import _capi

    t = golden("builders")[f"lozenge/{key}/max"]
    a = np.array(t, dtype=np.int32)
    _ltiler(rt, period).Walk(a, 700, 31)
    assert np.array_equal(a, po.lozenge_walk_weighted(t, [700], [31], *LWEIGHTS[period]))
    b = np.array(t, dtype=np.int32)
    _ltiler(rt, period, _capi.RT_RNG_PHILOX).Walk(b, 700, 31 + 2**40)
    assert np.array_equal(b, po.lozenge_walk_weighted(t, [700], [31 + 2**40], *LWEIGHTS[period], fast=True))


@pytest.mark.parametrize("fast", [False, True])
def test_weighted_lozenge_cftp_matches_oracle(rt, fast):
    from randomtilings_b200 import _capi

    b = golden("builders")
    tmax, tmin = b["lozenge/hex10_2/max"], b["lozenge/hex10_2/min"]
    tl = _ltiler(rt, 2, _capi.RT_RNG_PHILOX if fast else None)
    got, st = tl.CFTP(tmax, tmin, first_steps=64, master_seed=77, max_trials=20)
    want, trials, total, ok = po.cftp(tmax, tmin, 64, 77, max_trials=20, model="lozenge", fast=fast, weights=LW)
    assert st["coalesced"] and ok and st["trials"] == trials and st["total_steps"] == total
    assert np.array_equal(got, want)


def test_lozenge_weights_are_refused_where_they_do_not_apply(rt):
    from randomtilings_b200 import _capi

    one = np.ones((2, 2))
    with pytest.raises(_capi.RtError):
        rt.LozengeTiler(kernel=2).SetWeights(one, one, one)  # the q-volume kernel
    with pytest.raises(_capi.RtError):
        rt.LozengeTiler(rng=_capi.RT_RNG_PLANES).SetWeights(one, one, one)
    with pytest.raises(_capi.RtError):
        rt.LozengeTiler().SetWeights(one, one, np.zeros((2, 2)))


def test_lozenge_samples_follow_the_weighted_law(rt):
    """2 x 2 x 2 hexagon (20 tilings): chain ends and CFTP samples."""
    from randomtilings_b200 import _capi

    d = rt.LozengeTiler.Hexagon(2, 2, 2)
    tmin, tmax = np.asarray(rt.LozengeTiler.MinTiling(d)), np.asarray(rt.LozengeTiler.MaxTiling(d))
    tl = _ltiler(rt, 2, _capi.RT_RNG_PHILOX)
    ends = []
    for key in range(4000):
        a = np.array(tmin, dtype=np.int32)
        tl.Walk(a, 600, key)
        ends.append(a)
    samples = [tl.CFTP(tmax, tmin, first_steps=16, master_seed=s)[0] for s in range(4000)]
    for got in (ends, samples):
        c = Counter(s.tobytes() for s in got)
        assert len(c) == 20
        keys = sorted(c)
        w = np.array([lozenge_tiling_weight(np.frombuffer(k, dtype=np.int32), *LW) for k in keys])
        obs = np.array([c[k] for k in keys], dtype=float)
        assert stats.chisquare(obs, obs.sum() * w / w.sum()).pvalue > P_MIN
        assert stats.chisquare(obs).pvalue < 1e-6
